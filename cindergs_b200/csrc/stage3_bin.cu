// Stage 3 (binning) on sm_100a: tile counting fused with a single-pass
// chained scan, key emission fused with the radix digit histograms, and tile
// range identification.
//
// Reference semantics: count_tiles_kernel / ellipse_intersects_tile_gpu
// (render/kernels/binning.rs:37-164), gpu_exclusive_scan (scan.rs:198-333),
// emit_tile_keys_kernel / _u64 (binning.rs:170-328), identify_tile_ranges*
// (binning.rs:333-417).
//
// Work distribution ("warp-ballot counting"): a warp owns 32 splats. Their
// candidate tiles (the tile AABB of each splat's tight extents, row-major)
// are concatenated and processed 32 at a time, one candidate per lane; each
// lane finds its candidate's owner by a 5-step search over the warp's
// candidate prefix sums, runs the exact ellipse-vs-tile test, and a ballot
// turns the hits into per-splat counts (and, in the emitter, into each
// entry's rank inside its splat). A splat with thousands of candidate tiles
// is spread over all 32 lanes instead of serialising one lane.
//
// Compiled with -fmad=false: the ellipse test's quadratic is rounded term by
// term as in the reference, so counts, offsets and keys are bit-exact.
#include "kernels.h"

namespace cgs {
namespace {

constexpr int kBinThreads = 256;
constexpr int kBinWarps = kBinThreads / 32;

struct WarpSplats {
  uint32_t base[kBinWarps][32];   // exclusive prefix of candidate counts
  uint32_t width[kBinWarps][32];  // tile-box width
  uint32_t x0[kBinWarps][32];
  uint32_t y0[kBinWarps][32];
  float mu_x[kBinWarps][32];
  float mu_y[kBinWarps][32];
  float ca[kBinWarps][32];
  float cb[kBinWarps][32];
  float cc[kBinWarps][32];
  float qcut[kBinWarps][32];
};

struct SplatBox {
  bool valid;
  uint32_t x0, x1, y0, y1;
  float mu_x, mu_y, ca, cb, cc, alpha, tz;
};

__device__ __forceinline__ uint32_t tile_coord(float v, int32_t hi) {
  // clamp(floor(v / 16) as i32, 0, hi) with Rust's saturating cast.
  const float f = floorf(v / 16.0f);
  int32_t i = __float2int_rz(f);  // saturates, NaN -> 0
  i = i < 0 ? 0 : (i > hi ? hi : i);
  return (uint32_t)i;
}

__device__ __forceinline__ SplatBox load_box(const BinArgs& a, uint32_t s, uint32_t active) {
  SplatBox b;
  b.valid = false;
  if (s >= active || a.tiles_x == 0 || a.tiles_y == 0) return b;
  const float4 cc4 = a.recs[s].cc;
  const uint32_t p = __float_as_uint(cc4.w);
  if (p == 0u) return b;
  const float4 geo = a.recs[s].geo;
  const float ext_x = (float)(p & 0xFFFFu), ext_y = (float)((p >> 16) & 0xFFFFu);
  b.mu_x = geo.x;
  b.mu_y = geo.y;
  b.ca = geo.z;
  b.cb = geo.w;
  b.cc = cc4.x;
  b.alpha = cc4.y;
  b.tz = cc4.z;
  const int32_t mx = (int32_t)a.tiles_x - 1, my = (int32_t)a.tiles_y - 1;
  b.x0 = tile_coord(b.mu_x - ext_x, mx);
  b.x1 = tile_coord(b.mu_x + ext_x, mx);
  b.y0 = tile_coord(b.mu_y - ext_y, my);
  b.y1 = tile_coord(b.mu_y + ext_y, my);
  // ellipse_intersects_tile_gpu returns false for every tile when alpha < 1/255.
  b.valid = !(b.alpha < (1.0f / 255.0f));
  return b;
}

__device__ __forceinline__ bool ellipse_hit(float mu_x, float mu_y, float ca, float cb, float cc,
                                            float qcut, uint32_t tx, uint32_t ty, uint32_t W,
                                            uint32_t H) {
  const uint32_t x_start = tx * 16u, y_start = ty * 16u;
  if (x_start >= W || y_start >= H) return false;
  const uint32_t x_end = min(x_start + 15u, W - 1u);
  const uint32_t y_end = min(y_start + 15u, H - 1u);
  const float dx0 = ((float)x_start + 0.5f) - mu_x;
  const float dx1 = ((float)x_end + 0.5f) - mu_x;
  const float dy0 = ((float)y_start + 0.5f) - mu_y;
  const float dy1 = ((float)y_end + 0.5f) - mu_y;
  const float x_near = clampf(0.0f, dx0, dx1);
  const float y1 = clampf(-cb * x_near / fmaxf(cc, 1e-12f), dy0, dy1);
  const float q1 = ca * x_near * x_near + 2.0f * cb * x_near * y1 + cc * y1 * y1;
  const float y_near = clampf(0.0f, dy0, dy1);
  const float x2 = clampf(-cb * y_near / fmaxf(ca, 1e-12f), dx0, dx1);
  const float q2 = ca * x2 * x2 + 2.0f * cb * x2 * y_near + cc * y_near * y_near;
  return fminf(q1, q2) <= qcut + 1e-4f;
}

__device__ __forceinline__ uint32_t seg_mask(int lo, int hi) {
  // bits [lo, hi) of a 32-bit mask, 0 <= lo <= hi <= 32
  if (hi <= lo) return 0u;
  const uint32_t upper = hi >= 32 ? 0xffffffffu : ((1u << hi) - 1u);
  const uint32_t lower = lo >= 32 ? 0xffffffffu : ((1u << lo) - 1u);
  return upper & ~lower;
}

// Stages one warp's splats in shared memory; returns this lane's candidate
// count and exclusive base, and the warp's total candidate count.
__device__ __forceinline__ void stage_warp(WarpSplats& ws, int warp, int lane, const SplatBox& b,
                                           uint32_t& ncand, uint32_t& base, uint32_t& total) {
  ncand = 0;
  if (b.valid) ncand = (b.x1 - b.x0 + 1u) * (b.y1 - b.y0 + 1u);
  uint32_t incl = ncand;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  base = incl - ncand;
  total = __shfl_sync(0xffffffffu, incl, 31);
  ws.base[warp][lane] = base;
  ws.width[warp][lane] = b.valid ? (b.x1 - b.x0 + 1u) : 1u;
  ws.x0[warp][lane] = b.x0;
  ws.y0[warp][lane] = b.y0;
  ws.mu_x[warp][lane] = b.mu_x;
  ws.mu_y[warp][lane] = b.mu_y;
  ws.ca[warp][lane] = b.ca;
  ws.cb[warp][lane] = b.cb;
  ws.cc[warp][lane] = b.cc;
  ws.qcut[warp][lane] = b.valid ? clampf(2.0f * cgs_logf(255.0f * b.alpha), 0.0f, 8.0f) : 0.0f;
  __syncwarp();
}

// Owner lane of candidate `item`: the largest lane whose base <= item.
__device__ __forceinline__ int find_owner(const WarpSplats& ws, int warp, uint32_t item) {
  int o = 0;
#pragma unroll
  for (int step = 16; step > 0; step >>= 1)
    if (ws.base[warp][o + step] <= item) o += step;
  return o;
}

__device__ __forceinline__ bool test_candidate(const WarpSplats& ws, int warp, int o,
                                               uint32_t item, const BinArgs& a, uint32_t& tile) {
  const uint32_t c = item - ws.base[warp][o];
  const uint32_t w = ws.width[warp][o];
  const uint32_t r = c / w;
  const uint32_t tx = ws.x0[warp][o] + (c - r * w);
  const uint32_t ty = ws.y0[warp][o] + r;
  tile = ty * a.tiles_x + tx;
  return ellipse_hit(ws.mu_x[warp][o], ws.mu_y[warp][o], ws.ca[warp][o], ws.cb[warp][o],
                     ws.cc[warp][o], ws.qcut[warp][o], tx, ty, a.width, a.height);
}

// Tile counts per splat, block exclusive scan, chained scan across blocks ->
// offsets[s]; the last block writes the entry total to fc->entries.
__global__ void __launch_bounds__(kBinThreads) k_count_scan(const BinArgs a) {
  __shared__ WarpSplats ws;
  __shared__ uint32_t s_tile;
  __shared__ uint32_t s_warp_sums[32];
  __shared__ uint32_t s_base;
  if (threadIdx.x == 0) s_tile = atomicAdd(&a.fc->tile_ctr[1], 1u);
  __syncthreads();
  const uint32_t tile = s_tile;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t active = a.n_rest + (a.split_count ? *a.split_count : 0u);
  const uint32_t s = tile * kBinThreads + threadIdx.x;
  const SplatBox b = load_box(a, s, active);
  uint32_t ncand, base, total;
  stage_warp(ws, warp, lane, b, ncand, base, total);
  uint32_t count = 0;
  for (uint32_t chunk = 0; chunk < total; chunk += 32) {
    const uint32_t item = chunk + lane;
    bool hit = false;
    if (item < total) {
      const int o = find_owner(ws, warp, item);
      uint32_t t;
      hit = test_candidate(ws, warp, o, item, a, t);
    }
    const uint32_t hits = __ballot_sync(0xffffffffu, hit);
    const int lo = base > chunk ? (int)min(base - chunk, 32u) : 0;
    const int hi = (base + ncand) > chunk ? (int)min(base + ncand - chunk, 32u) : 0;
    count += __popc(hits & seg_mask(lo, hi));
  }
  uint32_t agg;
  const uint32_t excl = block_exclusive_sum(count, s_warp_sums, &agg);
  if (threadIdx.x < 32) {
    const uint32_t pre = chained_scan_warp(a.status, tile, agg, &a.fc->status);
    if (threadIdx.x == 0) s_base = pre;
  }
  __syncthreads();
  if (s < a.max_n) a.offsets[s] = s_base + excl;
  const uint32_t num_tiles = (a.max_n + kBinThreads - 1) / kBinThreads;
  if (tile == num_tiles - 1 && threadIdx.x == 0) {
    const uint32_t e = s_base + agg;
    a.fc->entries = e;
    if (e > a.entry_cap) atomicOr(&a.fc->status, kStatusCapacity);
  }
}

// Key emission: 32-bit keys (tile << depth_bits | depth_q) or, for more than
// 65,535 tiles, (tile, raw depth bits) word pairs; plus the digit histograms
// of every radix pass, accumulated in shared memory and added to `hist`.
template <bool KEY64>
__global__ void __launch_bounds__(kBinThreads) k_emit(const BinArgs a) {
  __shared__ WarpSplats ws;
  __shared__ uint32_t s_off[kBinWarps][32];
  __shared__ uint32_t s_dq[kBinWarps][32];
  __shared__ uint32_t s_carry[kBinWarps][32];
  __shared__ uint32_t s_hist[8 * 256];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t radix = 1u << a.radix_bits, rmask = radix - 1u;
  const uint32_t passes_lo = KEY64 ? (32u + a.radix_bits - 1u) / a.radix_bits
                                   : (a.sort_bits + a.radix_bits - 1u) / a.radix_bits;
  const uint32_t passes_hi = KEY64 ? (a.tile_bits + a.radix_bits - 1u) / a.radix_bits : 0u;
  const uint32_t nbins = (passes_lo + passes_hi) * radix;
  for (uint32_t k = threadIdx.x; k < nbins; k += kBinThreads) s_hist[k] = 0u;
  __syncthreads();
  const uint32_t active = a.n_rest + (a.split_count ? *a.split_count : 0u);
  const uint32_t cap = a.entry_cap;
  const uint32_t s = blockIdx.x * kBinThreads + threadIdx.x;
  const SplatBox b = load_box(a, s, active);
  uint32_t ncand, base, total;
  stage_warp(ws, warp, lane, b, ncand, base, total);
  uint32_t dq = 0;
  if (b.valid) {
    if (KEY64) {
      dq = __float_as_uint(fmaxf(b.tz, 0.0f));
    } else {
      const uint32_t raw = __float_as_uint(fmaxf(b.tz, 1e-6f));
      const uint32_t rel = raw > a.depth_base_bits ? min(raw - a.depth_base_bits, 0x0FFFFFFFu) : 0u;
      dq = rel >> (28u - a.depth_bits);
    }
  }
  s_off[warp][lane] = (b.valid && s < a.max_n) ? a.offsets[s] : 0u;
  s_dq[warp][lane] = dq;
  s_carry[warp][lane] = 0u;
  __syncwarp();
  for (uint32_t chunk = 0; chunk < total; chunk += 32) {
    const uint32_t item = chunk + lane;
    bool hit = false;
    int o = 0;
    uint32_t tile = 0;
    if (item < total) {
      o = find_owner(ws, warp, item);
      hit = test_candidate(ws, warp, o, item, a, tile);
    }
    const uint32_t hits = __ballot_sync(0xffffffffu, hit);
    if (hit) {
      const uint32_t ob = ws.base[warp][o];
      const int sstart = ob > chunk ? (int)(ob - chunk) : 0;
      const uint32_t below = hits & lanemask_lt() & ~seg_mask(0, sstart);
      const uint32_t pos = s_off[warp][o] + s_carry[warp][o] + __popc(below);
      const uint32_t sid = blockIdx.x * kBinThreads + warp * 32 + o;
      if (pos < cap) {
        if (KEY64) {
          a.keys[pos] = tile;
          a.depths[pos] = s_dq[warp][o];
          a.ids[pos] = sid;
          const uint32_t d = s_dq[warp][o];
          for (uint32_t p = 0; p < passes_lo; ++p)
            atomicAdd(&s_hist[p * radix + ((d >> (p * a.radix_bits)) & rmask)], 1u);
          for (uint32_t p = 0; p < passes_hi; ++p)
            atomicAdd(&s_hist[(passes_lo + p) * radix + ((tile >> (p * a.radix_bits)) & rmask)], 1u);
        } else {
          const uint32_t key = a.depth_bits >= 32u ? s_dq[warp][o] : ((tile << a.depth_bits) | s_dq[warp][o]);
          a.keys[pos] = key;
          a.ids[pos] = sid;
          for (uint32_t p = 0; p < passes_lo; ++p)
            atomicAdd(&s_hist[p * radix + ((key >> (p * a.radix_bits)) & rmask)], 1u);
        }
      }
    }
    __syncwarp();
    const int lo = base > chunk ? (int)min(base - chunk, 32u) : 0;
    const int hi = (base + ncand) > chunk ? (int)min(base + ncand - chunk, 32u) : 0;
    s_carry[warp][lane] += __popc(hits & seg_mask(lo, hi));
    __syncwarp();
  }
  __syncthreads();
  for (uint32_t k = threadIdx.x; k < nbins; k += kBinThreads) {
    const uint32_t v = s_hist[k];
    if (v) atomicAdd(&a.hist[k], v);
  }
}

// identify_tile_ranges_kernel (binning.rs:356-391): boundaries of equal tile
// ids in the sorted words. Grid-stride over the device-side entry count.
__global__ void k_tile_ranges(const uint32_t* __restrict__ sorted, uint32_t shift,
                              const uint32_t* __restrict__ n_ptr, uint32_t total_tiles,
                              uint32_t* __restrict__ ranges) {
  const uint32_t n = *n_ptr;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t t = shift >= 32u ? 0u : (sorted[i] >> shift);
    if (t >= total_tiles) continue;
    if (i == 0) {
      ranges[2 * (size_t)t] = 0u;
    } else {
      const uint32_t prev = shift >= 32u ? 0u : (sorted[i - 1] >> shift);
      if (t != prev) {
        if (prev < total_tiles) ranges[2 * (size_t)prev + 1] = i;
        ranges[2 * (size_t)t] = i;
      }
    }
    if (i + 1 == n) ranges[2 * (size_t)t + 1] = n;
  }
}

// Generic single-pass exclusive scan: 4096 elements per tile (16 per thread,
// blocked), chained across tiles.
constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr uint32_t kScanTile = kScanThreads * kScanItems;

__global__ void __launch_bounds__(kScanThreads) k_scan_u32(const uint32_t* __restrict__ in,
                                                           uint32_t* __restrict__ out, uint32_t n,
                                                           uint32_t* d_total,
                                                           unsigned long long* status,
                                                           uint32_t* tile_ctr,
                                                           uint32_t* status_word) {
  __shared__ uint32_t s_tile, s_base;
  __shared__ uint32_t s_warp_sums[32];
  if (threadIdx.x == 0) s_tile = atomicAdd(tile_ctr, 1u);
  __syncthreads();
  const uint32_t tile = s_tile;
  const size_t start = (size_t)tile * kScanTile + (size_t)threadIdx.x * kScanItems;
  uint32_t v[kScanItems];
  uint32_t sum = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    v[k] = (start + k < n) ? in[start + k] : 0u;
    sum += v[k];
  }
  uint32_t agg;
  uint32_t excl = block_exclusive_sum(sum, s_warp_sums, &agg);
  if (threadIdx.x < 32) {
    const uint32_t pre = chained_scan_warp(status, tile, agg, status_word);
    if (threadIdx.x == 0) s_base = pre;
  }
  __syncthreads();
  uint32_t run = s_base + excl;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    if (start + k < n) out[start + k] = run;
    run += v[k];
  }
  const uint32_t num_tiles = (n + kScanTile - 1) / kScanTile;
  if (tile == num_tiles - 1 && threadIdx.x == 0) *d_total = s_base + agg;
}

}  // namespace

cudaError_t launch_count_scan(const BinArgs& a, cudaStream_t s) {
  if (a.max_n == 0) return cudaSuccess;
  k_count_scan<<<(a.max_n + kBinThreads - 1) / kBinThreads, kBinThreads, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_emit(const BinArgs& a, cudaStream_t s) {
  if (a.max_n == 0) return cudaSuccess;
  const uint32_t blocks = (a.max_n + kBinThreads - 1) / kBinThreads;
  if (a.key64)
    k_emit<true><<<blocks, kBinThreads, 0, s>>>(a);
  else
    k_emit<false><<<blocks, kBinThreads, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_tile_ranges(const uint32_t* sorted, uint32_t shift, const uint32_t* n_ptr,
                               uint32_t total_tiles, uint32_t* ranges, cudaStream_t s) {
  k_tile_ranges<<<148 * 8, 256, 0, s>>>(sorted, shift, n_ptr, total_tiles, ranges);
  return cudaGetLastError();
}

uint32_t scan_tiles(uint32_t n) { return (n + kScanTile - 1) / kScanTile; }

cudaError_t launch_scan_u32(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* d_total,
                            unsigned long long* status, uint32_t* tile_ctr, uint32_t* status_word,
                            cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  k_scan_u32<<<scan_tiles(n), kScanThreads, 0, s>>>(in, out, n, d_total, status, tile_ctr,
                                                    status_word);
  return cudaGetLastError();
}

}  // namespace cgs
