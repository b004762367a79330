// Stage 3 (binning) on sm_100a: one kernel that counts tile intersections,
// scans the counts in a single chained pass and emits the sort keys together
// with the radix digit histograms; and tile range identification.
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
  uint32_t magic[kBinWarps][32];  // ceil(2^32 / width): c / width == umulhi(c, magic)
  uint32_t owner_at[kBinWarps][32];  // lane whose candidates start at a chunk position
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
  const uint32_t w = b.valid ? (b.x1 - b.x0 + 1u) : 1u;
  ws.width[warp][lane] = w;
  ws.magic[warp][lane] = w <= 1u ? 0u : (uint32_t)(((1ull << 32) + w - 1u) / w);
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

// Owner lane of each lane's candidate in the chunk [chunk, chunk + 32): the
// starts of the candidate runs that begin inside the chunk are OR-reduced into
// a position mask; a lane's owner is the run starting at the highest set
// position not above it, or the run carried over from the previous chunk.
// `carry` holds that run's lane between chunks (the first run starts at 0).
__device__ __forceinline__ int chunk_owner(WarpSplats& ws, int warp, int lane, uint32_t chunk,
                                           uint32_t base, uint32_t ncand, int& carry) {
  const bool starts = ncand > 0u && base >= chunk && base - chunk < 32u;
  if (starts) ws.owner_at[warp][base - chunk] = (uint32_t)lane;
  const uint32_t smask = __reduce_or_sync(0xffffffffu, starts ? (1u << (base - chunk)) : 0u);
  __syncwarp();
  const uint32_t upto = smask & ((2u << lane) - 1u);
  const int o = upto ? (int)ws.owner_at[warp][31 - __clz(upto)] : carry;
  if (smask) carry = (int)ws.owner_at[warp][31 - __clz(smask)];
  __syncwarp();
  return o;
}

// Tile of candidate `item` of owner lane o (row-major over its tile box).
__device__ __forceinline__ void candidate_tile(const WarpSplats& ws, int warp, int o, uint32_t item,
                                               uint32_t& tx, uint32_t& ty) {
  const uint32_t c = item - ws.base[warp][o];
  const uint32_t w = ws.width[warp][o];
  const uint32_t r = w <= 1u ? c : __umulhi(c, ws.magic[warp][o]);
  tx = ws.x0[warp][o] + (c - r * w);
  ty = ws.y0[warp][o] + r;
}

__device__ __forceinline__ bool test_candidate(const WarpSplats& ws, int warp, int o,
                                               uint32_t item, const BinArgs& a, uint32_t& tile) {
  uint32_t tx, ty;
  candidate_tile(ws, warp, o, item, tx, ty);
  tile = ty * a.tiles_x + tx;
  return ellipse_hit(ws.mu_x[warp][o], ws.mu_y[warp][o], ws.ca[warp][o], ws.cb[warp][o],
                     ws.cc[warp][o], ws.qcut[warp][o], tx, ty, a.width, a.height);
}

// One pass of binning for a block of 256 splats, taken in depth-key order
// (slot s is splat order_ids[s]; Stage 2's depth keys were radix-sorted
// stably, so slots run by (depth key, splat index)):
//   1. counting: every candidate tile of the warp's 32 splats is tested once
//      (ballot per 32 candidates); the ballot masks are kept in shared memory;
//   2. block exclusive scan of the per-slot counts, chained across blocks
//      (decoupled look-back) -> each slot's first entry (written to `offsets`);
//   3. emission: the masks are walked again, each hit is written at
//      offset + (its rank inside the splat), row-major as in the reference,
//      with its 32-bit key (tile << depth_bits | depth_q) or, for more than
//      65,535 tiles, its (tile, raw depth bits) pair; the digit histograms of
//      the tile bits are accumulated at the same time.
// The entries therefore leave this kernel ordered by (depth, splat index), and
// a stable sort on the tile bits alone yields the reference's (tile, depth,
// splat index) order: sorting the splats once (N keys) replaces the depth
// passes over all entries.
// Entries at or beyond the key-buffer capacity are not written and set the
// capacity status bit (the host grows the buffers and runs Stage 3 again).
// The last block writes the frame's entry total.
constexpr int kMaskCap = 48;  // stored ballot masks per warp (1,536 candidates)

template <bool KEY64>
__global__ void __launch_bounds__(kBinThreads) k_bin(const BinArgs a) {
  __shared__ WarpSplats ws;
  __shared__ uint32_t s_off[kBinWarps][32];
  __shared__ uint32_t s_dq[kBinWarps][32];
  __shared__ uint32_t s_sid[kBinWarps][32];
  __shared__ uint32_t s_carry[kBinWarps][32];
  __shared__ uint32_t s_masks[kBinWarps][kMaskCap];
  __shared__ uint32_t s_hist[8 * 256];
  __shared__ uint32_t s_tile, s_base;
  __shared__ uint32_t s_warp_sums[32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t radix = 1u << a.radix_bits, rmask = radix - 1u;
  const uint32_t passes = (a.tile_bits + a.radix_bits - 1u) / a.radix_bits;
  const uint32_t tshift = KEY64 ? 0u : a.depth_bits;  // tile bits of the sort word
  const uint32_t nbins = passes * radix;
  if (threadIdx.x == 0) s_tile = atomicAdd(&a.fc->tile_ctr[1], 1u);
  for (uint32_t k = threadIdx.x; k < nbins; k += kBinThreads) s_hist[k] = 0u;
  __syncthreads();
  const uint32_t tile = s_tile;
  const uint32_t active = a.n_rest + (a.split_count ? *a.split_count : 0u);
  const uint32_t s = tile * kBinThreads + threadIdx.x;  // slot in depth order
  uint32_t sid = kInvalid, dq = 0;
  if (s < active && s < a.max_n) {
    sid = a.order_ids[s];
    dq = a.order_keys[s];
  }
  const SplatBox b = load_box(a, sid, active);
  uint32_t ncand, base, total;
  stage_warp(ws, warp, lane, b, ncand, base, total);

  // 1. count
  uint32_t count = 0;
  int carry = 0;
  for (uint32_t chunk = 0, c = 0; chunk < total; chunk += 32, ++c) {
    const uint32_t item = chunk + lane;
    const int o = chunk_owner(ws, warp, lane, chunk, base, ncand, carry);
    bool hit = false;
    if (item < total) {
      uint32_t t;
      hit = test_candidate(ws, warp, o, item, a, t);
    }
    const uint32_t hits = __ballot_sync(0xffffffffu, hit);
    if (c < (uint32_t)kMaskCap && lane == 0) s_masks[warp][c] = hits;
    const int lo = base > chunk ? (int)min(base - chunk, 32u) : 0;
    const int hi = (base + ncand) > chunk ? (int)min(base + ncand - chunk, 32u) : 0;
    count += __popc(hits & seg_mask(lo, hi));
  }

  // 2. scan
  uint32_t agg;
  const uint32_t excl = block_exclusive_sum(count, s_warp_sums, &agg);
  if (threadIdx.x < 32) {
    const uint32_t pre = chained_scan_warp(a.status, tile, agg, &a.fc->status);
    if (threadIdx.x == 0) s_base = pre;
  }
  __syncthreads();
  const uint32_t first = s_base + excl;
  if (s < a.max_n) a.offsets[s] = first;
  const uint32_t num_tiles = (a.max_n + kBinThreads - 1) / kBinThreads;
  if (tile == num_tiles - 1 && threadIdx.x == 0) {
    const uint32_t e = s_base + agg;
    a.fc->entries = e;
    if (e > a.entry_cap) atomicOr(&a.fc->status, kStatusCapacity);
  }

  // 3. emit
  s_off[warp][lane] = first;
  s_dq[warp][lane] = dq;
  s_sid[warp][lane] = sid;
  s_carry[warp][lane] = 0u;
  __syncwarp();
  const uint32_t cap = a.entry_cap;
  bool overflow = false;
  carry = 0;
  for (uint32_t chunk = 0, c = 0; chunk < total; chunk += 32, ++c) {
    const uint32_t item = chunk + lane;
    const int o = chunk_owner(ws, warp, lane, chunk, base, ncand, carry);
    uint32_t hits;
    uint32_t tile_id = 0;
    if (c < (uint32_t)kMaskCap) {
      hits = s_masks[warp][c];
      if ((hits >> lane) & 1u) {
        uint32_t tx, ty;
        candidate_tile(ws, warp, o, item, tx, ty);
        tile_id = ty * a.tiles_x + tx;
      }
    } else {
      bool hit = false;
      if (item < total) hit = test_candidate(ws, warp, o, item, a, tile_id);
      hits = __ballot_sync(0xffffffffu, hit);
    }
    if ((hits >> lane) & 1u) {
      const uint32_t ob = ws.base[warp][o];
      const int sstart = ob > chunk ? (int)(ob - chunk) : 0;
      const uint32_t below = hits & lanemask_lt() & ~seg_mask(0, sstart);
      const uint32_t pos = s_off[warp][o] + s_carry[warp][o] + __popc(below);
      const uint32_t osid = s_sid[warp][o];
      if (pos < cap) {
        uint32_t word;
        if (KEY64) {
          word = tile_id;
          a.depths[pos] = s_dq[warp][o];
        } else {
          word = a.depth_bits >= 32u ? s_dq[warp][o] : ((tile_id << a.depth_bits) | s_dq[warp][o]);
        }
        a.keys[pos] = word;
        a.ids[pos] = osid;
        for (uint32_t p = 0; p < passes; ++p)
          atomicAdd(&s_hist[p * radix + ((word >> (tshift + p * a.radix_bits)) & rmask)], 1u);
      } else {
        overflow = true;
      }
    }
    __syncwarp();
    const int lo = base > chunk ? (int)min(base - chunk, 32u) : 0;
    const int hi = (base + ncand) > chunk ? (int)min(base + ncand - chunk, 32u) : 0;
    s_carry[warp][lane] += __popc(hits & seg_mask(lo, hi));
    __syncwarp();
  }
  if (overflow) atomicOr(&a.fc->status, kStatusCapacity);
  __syncthreads();
  for (uint32_t k = threadIdx.x; k < nbins; k += kBinThreads) {
    const uint32_t v = s_hist[k];
    if (v) atomicAdd(&a.hist[k], v);
  }
}

// identify_tile_ranges_kernel (binning.rs:356-391): boundaries of equal tile
// ids in the sorted words. Each thread checks four consecutive words (one
// 128-bit load plus the word before them), grid-stride over the device-side
// entry count; boundaries are rare, so the writes are few.
__device__ __forceinline__ void range_edge(uint32_t i, uint32_t t, uint32_t prev, uint32_t n,
                                           uint32_t total_tiles, uint32_t* ranges) {
  if (t >= total_tiles) return;
  if (i == 0) {
    ranges[2 * (size_t)t] = 0u;
  } else if (t != prev) {
    if (prev < total_tiles) ranges[2 * (size_t)prev + 1] = i;
    ranges[2 * (size_t)t] = i;
  }
  if (i + 1 == n) ranges[2 * (size_t)t + 1] = n;
}

__global__ void k_tile_ranges(const uint32_t* __restrict__ sorted, uint32_t shift,
                              const uint32_t* __restrict__ n_ptr, uint32_t capacity,
                              uint32_t total_tiles, uint32_t* __restrict__ ranges) {
  const uint32_t n = min(*n_ptr, capacity);
  const uint32_t quads = (n + 3) / 4;
  for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < quads; q += gridDim.x * blockDim.x) {
    const uint32_t i0 = 4 * q;
    uint32_t w[4];
    if (i0 + 3 < n) {
      const uint4 v = __ldcs(reinterpret_cast<const uint4*>(sorted) + q);
      w[0] = v.x; w[1] = v.y; w[2] = v.z; w[3] = v.w;
    } else {
      for (int k = 0; k < 4; ++k) w[k] = i0 + k < n ? sorted[i0 + k] : 0u;
    }
    uint32_t prev = i0 > 0 ? (shift >= 32u ? 0u : (sorted[i0 - 1] >> shift)) : 0xFFFFFFFFu;
    for (int k = 0; k < 4; ++k) {
      const uint32_t i = i0 + k;
      if (i >= n) break;
      const uint32_t t = shift >= 32u ? 0u : (w[k] >> shift);
      range_edge(i, t, prev, n, total_tiles, ranges);
      prev = t;
    }
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

cudaError_t launch_bin(const BinArgs& a, cudaStream_t s) {
  if (a.max_n == 0) return cudaSuccess;
  const uint32_t blocks = (a.max_n + kBinThreads - 1) / kBinThreads;
  if (a.key64)
    k_bin<true><<<blocks, kBinThreads, 0, s>>>(a);
  else
    k_bin<false><<<blocks, kBinThreads, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_tile_ranges(const uint32_t* sorted, uint32_t shift, const uint32_t* n_ptr,
                               uint32_t capacity, uint32_t total_tiles, uint32_t* ranges,
                               cudaStream_t s) {
  k_tile_ranges<<<148 * 8, 256, 0, s>>>(sorted, shift, n_ptr, capacity, total_tiles, ranges);
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
