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
// Term tables: the reference's test evaluates the conic's quadratic at two
// points of a tile -- one whose x is the tile column's nearest x to the
// centre, one whose y is the tile row's nearest y -- each with a division
// that depends on the column alone or on the row alone. A warp therefore
// first evaluates, per splat, every column term (x edges, nearest x, the
// clamped-y division, a x^2) and every row term (y edges, nearest y, the
// clamped-x division, c y^2) of its 32 splats' tile boxes into shared memory;
// each candidate tile then combines one column and one row entry with ~20
// floating-point operations instead of evaluating the whole test. Every
// product and sum is rounded separately (explicit __fmul_rn/__fadd_rn, in the
// reference's operand order), so the test's result is the reference formula's
// bit for bit; counts, offsets and keys are bit-exact.
#include <algorithm>

#include "kernels.h"

namespace cgs {
namespace {

constexpr int kBinThreads = 256;
constexpr int kBinWarps = kBinThreads / 32;
constexpr int kMaskCap = 64;   // stored ballot masks per warp (2,048 candidates)
constexpr int kHitCap = 640;   // stored hit records per warp; a warp's 32 splats emit ~770
                               // entries at 1080p on average, the rest walk the masks again
constexpr int kTabCap = 384;   // term-table entries (tile columns + rows) per warp
constexpr uint32_t kMaxGroups = 8;  // tile groups of the record mode

// Per-splat constants of a warp's 32 splats, read by the lane that tests one
// of the splat's candidate tiles.
struct BinSplats {
  double2 rcp[kBinWarps][32]; // RN64(1 / max(c, 1e-12)), RN64(1 / max(a, 1e-12))
  uint4 box[kBinWarps][32];   // x0, y0, width (tiles), ceil(2^32 / width)
  float4 geo[kBinWarps][32];  // mu_x, mu_y, -b, 2b
  float4 con[kBinWarps][32];  // a, c, max(a, 1e-12), max(c, 1e-12)
  float4 kq[kBinWarps][32];   // a, 2b, c, q_max + 1e-4 (the term-table test)
  uint2 tb[kBinWarps][32];    // first column entry, first row entry in the term table
  uint32_t base[kBinWarps][32];  // exclusive prefix of the candidate counts
  uint32_t cpre[kBinWarps][32];  // exclusive prefix of the tile-box widths
  uint32_t rpre[kBinWarps][32];  // exclusive prefix of the tile-box heights
  uint32_t dq[kBinWarps][32];    // depth part of the key
  uint32_t sid[kBinWarps][32];   // splat index
  // owner lookup of warps with at most kMaskCap * 32 candidates: bit i of
  // word i / 32 set where a splat's candidates start, and the lane of the
  // k-th splat with candidates
  uint32_t sbits[kBinWarps][kMaskCap];
  uint32_t lor[kBinWarps][32];
};
constexpr size_t kBinSmem = sizeof(BinSplats) + sizeof(uint32_t) * kBinWarps * (2 * kMaskCap + kHitCap) +
                            sizeof(float4) * kBinWarps * kTabCap +
                            sizeof(uint32_t) * 1024;  // + tile-digit histograms (<= 4 x 256)

struct SplatBox {
  bool valid;
  uint32_t x0, x1, y0, y1;
  float mu_x, mu_y, ca, cb, cc, alpha;
};

__device__ __forceinline__ uint32_t tile_coord(float v, int32_t hi, float inv_tile) {
  // clamp(floor(v / tile) as i32, 0, hi) with Rust's saturating cast; the
  // tile size is a power of two, so v * (1 / tile) is the exact quotient.
  const float f = floorf(__fmul_rn(v, inv_tile));
  int32_t i = __float2int_rz(f);  // saturates, NaN -> 0
  i = i < 0 ? 0 : (i > hi ? hi : i);
  return (uint32_t)i;
}

__device__ __forceinline__ SplatBox load_box(const BinArgs& a, uint32_t s, uint32_t active) {
  SplatBox b;
  b.valid = false;
  b.x0 = b.x1 = b.y0 = b.y1 = 0;
  b.mu_x = b.mu_y = b.ca = b.cb = b.cc = b.alpha = 0.0f;
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
  const int32_t mx = (int32_t)a.tiles_x - 1, my = (int32_t)a.tiles_y - 1;
  const float itw = __uint_as_float((127u - a.tile_w_log2) << 23);  // 2^-lw
  const float ith = __uint_as_float((127u - a.tile_h_log2) << 23);
  b.x0 = tile_coord(__fsub_rn(b.mu_x, ext_x), mx, itw);
  b.x1 = tile_coord(__fadd_rn(b.mu_x, ext_x), mx, itw);
  b.y0 = tile_coord(__fsub_rn(b.mu_y, ext_y), my, ith);
  b.y1 = tile_coord(__fadd_rn(b.mu_y, ext_y), my, ith);
  // ellipse_intersects_tile_gpu returns false for every tile when alpha < 1/255.
  b.valid = !(b.alpha < (1.0f / 255.0f));
  return b;
}

// (float)v + 0.5f for v < 2^22, exactly: 2^23 + v is exact in binary32 and
// the subtraction of 2^23 - 0.5 is exact (Sterbenz), so the result equals the
// reference's integer-to-float conversion plus one half without a conversion.
__device__ __forceinline__ float pixel_center(uint32_t v) {
  return __fsub_rn(__int_as_float(0x4B000000u | v), 8388607.5f);
}

// n / d correctly rounded to binary32, for d > 0, from y = RN64(1 / d) (one
// binary64 reciprocal per splat instead of a binary32 division per tile).
// The binary64 product n * y is within 2^-52 (relative) of n / d. A quotient
// of two binary32 numbers is never closer than 2^-49 (relative) to a midpoint
// of two binary32 neighbours in the normal range: if n / d = m (1 + e) with m
// a midpoint, m = M 2^k with M odd and M >= 2^24, then n - d m is a nonzero
// multiple of 2^k ulp(d) -- an odd factor of M >= 2^24 cannot divide a 24-bit
// significand -- so |e| >= 2^-49. Hence n * y and n / d round to the same
// binary32 value. Results below 2^-125 in magnitude, where the binary32 grid
// is finer relative to the value than that argument assumes, use the binary32
// division itself; zero stays a signed zero.
__device__ __noinline__ float div_ieee(float n, float d) { return __fdiv_rn(n, d); }

__device__ __forceinline__ float div_rcp64(float n, float d, double y) {
  const double q = __dmul_rn((double)n, y);
  float r = __double2float_rn(q);
  // a call, so that the compiler cannot turn the rare case into a division
  // on every lane
  if (q != 0.0 && fabs(q) < 0x1p-125) r = div_ieee(n, d);
  return r;
}

// ellipse_intersects_tile_gpu (binning.rs:37-96) for tile (tx, ty) of the
// splat's tile box, in the reference's operand order, every operation rounded
// separately: the quadratic form is evaluated at the tile point nearest the
// centre along x (y minimised, clamped) and along y (x minimised, clamped).
// The reference's "tile starts outside the viewport" exit never fires for a
// tile of the clamped box. geo = (mu_x, mu_y, -b, 2b), con = (a, c, max(a,
// 1e-12), max(c, 1e-12)), rcp = their binary64 reciprocals (c term, a term),
// qlim = q_max + 1e-4. Used for warps whose term tables do not fit.
__device__ __forceinline__ bool tile_hit(uint32_t tx, uint32_t ty, uint32_t wm1, uint32_t hm1,
                                         uint32_t lw, uint32_t lh, const float4 geo,
                                         const float4 con, const double2 rcp, float qlim) {
  const uint32_t xs = tx << lw, ys = ty << lh;
  const float dx0 = __fsub_rn(pixel_center(xs), geo.x);
  const float dx1 = __fsub_rn(pixel_center(min(xs + ((1u << lw) - 1u), wm1)), geo.x);
  const float dy0 = __fsub_rn(pixel_center(ys), geo.y);
  const float dy1 = __fsub_rn(pixel_center(min(ys + ((1u << lh) - 1u), hm1)), geo.y);
  const float x_near = clampf(0.0f, dx0, dx1);
  const float y1 = clampf(div_rcp64(__fmul_rn(geo.z, x_near), con.w, rcp.x), dy0, dy1);
  const float q1 = __fadd_rn(__fadd_rn(__fmul_rn(__fmul_rn(con.x, x_near), x_near),
                                       __fmul_rn(__fmul_rn(geo.w, x_near), y1)),
                             __fmul_rn(__fmul_rn(con.y, y1), y1));
  const float y_near = clampf(0.0f, dy0, dy1);
  const float x2 = clampf(div_rcp64(__fmul_rn(geo.z, y_near), con.z, rcp.y), dx0, dx1);
  const float q2 = __fadd_rn(__fadd_rn(__fmul_rn(__fmul_rn(con.x, x2), x2),
                                       __fmul_rn(__fmul_rn(geo.w, x2), y_near)),
                             __fmul_rn(__fmul_rn(con.y, y_near), y_near));
  return fminf(q1, q2) <= qlim;
}

// Column terms of a splat's tile column tx (the parts of tile_hit that depend
// on the column alone): x edges, the y minimiser at the column's nearest x
// (before its clamp to the row), a x_near^2.
__device__ __forceinline__ float4 col_terms(uint32_t tx, uint32_t lw, uint32_t wm1, const float4 geo,
                                            const float4 con, const double2 rcp) {
  const uint32_t xs = tx << lw;
  const float dx0 = __fsub_rn(pixel_center(xs), geo.x);
  const float dx1 = __fsub_rn(pixel_center(min(xs + ((1u << lw) - 1u), wm1)), geo.x);
  const float x_near = clampf(0.0f, dx0, dx1);
  return make_float4(dx0, dx1, div_rcp64(__fmul_rn(geo.z, x_near), con.w, rcp.x),
                     __fmul_rn(__fmul_rn(con.x, x_near), x_near));
}

// Row terms of tile row ty: y edges, the x minimiser at the row's nearest y
// (before its clamp to the column), c y_near^2.
__device__ __forceinline__ float4 row_terms(uint32_t ty, uint32_t lh, uint32_t hm1, const float4 geo,
                                            const float4 con, const double2 rcp) {
  const uint32_t ys = ty << lh;
  const float dy0 = __fsub_rn(pixel_center(ys), geo.y);
  const float dy1 = __fsub_rn(pixel_center(min(ys + ((1u << lh) - 1u), hm1)), geo.y);
  const float y_near = clampf(0.0f, dy0, dy1);
  return make_float4(dy0, dy1, div_rcp64(__fmul_rn(geo.z, y_near), con.z, rcp.y),
                     __fmul_rn(__fmul_rn(con.y, y_near), y_near));
}

// tile_hit from a column entry, a row entry and kq = (a, 2b, c, qlim): the
// same operations on the same operands, the column/row-only ones taken from
// the tables.
__device__ __forceinline__ bool tab_hit(const float4 col, const float4 row, const float4 kq) {
  const float x_near = clampf(0.0f, col.x, col.y);
  const float y_near = clampf(0.0f, row.x, row.y);
  const float y1 = clampf(col.z, row.x, row.y);
  const float q1 = __fadd_rn(__fadd_rn(col.w, __fmul_rn(__fmul_rn(kq.y, x_near), y1)),
                             __fmul_rn(__fmul_rn(kq.z, y1), y1));
  const float x2 = clampf(row.z, col.x, col.y);
  const float q2 = __fadd_rn(__fadd_rn(__fmul_rn(__fmul_rn(kq.x, x2), x2),
                                       __fmul_rn(__fmul_rn(kq.y, x2), y_near)),
                             row.w);
  return fminf(q1, q2) <= kq.w;
}

__device__ __forceinline__ uint32_t seg_mask(int lo, int hi) {
  // bits [lo, hi) of a 32-bit mask, 0 <= lo <= hi <= 32
  if (hi <= lo) return 0u;
  const uint32_t upper = hi >= 32 ? 0xffffffffu : ((1u << hi) - 1u);
  const uint32_t lower = lo >= 32 ? 0xffffffffu : ((1u << lo) - 1u);
  return upper & ~lower;
}

// Lane of the warp's splat that owns item `item` of a concatenation: the last
// lane whose exclusive prefix is <= item (lanes with no items share the next
// lane's prefix and are skipped by "last").
__device__ __forceinline__ int find_owner(const uint32_t* base, uint32_t item) {
  int o = 0;
#pragma unroll
  for (int step = 16; step >= 1; step >>= 1)
    if (base[o + step] <= item) o += step;
  return o;
}

// Candidate `c` of a splat's tile box (row-major) -> row and column in the box.
__device__ __forceinline__ void box_rc(const uint4 box, uint32_t c, uint32_t& r, uint32_t& col) {
  r = box.z <= 1u ? c : __umulhi(c, box.w);
  col = c - r * box.z;
}

// Binning in depth-key order (slot s is splat order_ids[s]; Stage 2's depth
// keys were radix-sorted stably, so slots run by (depth key, splat index)).
// Persistent warps: each warp takes 32 consecutive slots at a time from a
// counter (so the 32-slot tiles are taken in increasing order). The 32
// splats' candidate tiles (each splat's tile box, row-major) are
// concatenated and tested 32 at a time, one per lane, so large and small
// splats share the lanes evenly.
//   0. term tables: the column and row terms of the 32 tile boxes (when they
//      fit; otherwise every candidate evaluates the whole test).
//   1. counting: ballot per 32 candidates; the masks, the hits before each
//      mask, and one record per hit (tile id or candidate index, owner lane)
//      are kept in shared memory. A slot's count is the number of hits inside
//      its candidate range, read from the masks.
//   2. direct mode: the tile's hit count enters a decoupled look-back over
//      the 32-slot tiles (published as soon as it is counted; sums saturate),
//      which gives the tile's first entry: the slots' scanned offsets are
//      written, and the hits, in candidate order (= the reference's emission
//      order: splat by splat, row-major), are written at their places in
//      depth order with their 32-bit keys (tile << depth_bits | depth_q) or,
//      beyond 65,535 tiles, (tile, raw depth bits) pairs; the block's digit
//      histograms of the tile bits are accumulated. A stable sort on the tile
//      bits alone then yields the reference's (tile, depth, splat index)
//      order. Record mode (the tile transpose) instead stages one record per
//      hit at an atomic position per tile group and leaves the counts.
//      Warps with more hits or candidates than the shared-memory stores hold
//      walk their candidates again for the rest.
// Entries at or beyond the buffer capacity are not written and set the
// capacity status bit (the host grows the buffers and runs Stage 3 again).
__global__ void __launch_bounds__(kBinThreads, 2) k_bin_count(const BinArgs a) {
  extern __shared__ __align__(16) unsigned char bin_smem[];
  BinSplats& sp = *reinterpret_cast<BinSplats*>(bin_smem);
  float4* s_tab = reinterpret_cast<float4*>(bin_smem + sizeof(BinSplats));  // [w][kTabCap]
  uint32_t* s_mask = reinterpret_cast<uint32_t*>(s_tab + kBinWarps * kTabCap);  // [w][kMaskCap]
  uint32_t* s_mrun = s_mask + kBinWarps * kMaskCap;  // [w][kMaskCap] hits before mask c
  uint32_t* s_hits = s_mrun + kBinWarps * kMaskCap;  // [w][kHitCap]
  uint32_t* s_grp = s_hits + kBinWarps * kHitCap;    // [warps][3][kMaxGroups]
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t wm1 = a.width - 1u, hm1 = a.height - 1u;
  const uint32_t lw = a.tile_w_log2, lh = a.tile_h_log2;
  // per warp, per tile group: the hits counted, the staging start and the
  // records written
  const uint32_t G = a.groups, gshift = a.group_shift;
  uint32_t* s_gcnt = s_grp + warp * 3 * kMaxGroups;
  uint32_t* s_gbase = s_gcnt + kMaxGroups;
  uint32_t* s_grun = s_gbase + kMaxGroups;
  const uint32_t lt = lanemask_lt();
  const uint32_t active = a.n_rest + (a.split_count ? *a.split_count : 0u);
  const uint32_t num_tiles = (a.max_n + 31u) / 32u;
  const uint32_t* wbase = sp.base[warp];
  float4* wtab = s_tab + warp * kTabCap;
  uint32_t* wmask = s_mask + warp * kMaskCap;
  uint32_t* wmrun = s_mrun + warp * kMaskCap;
  uint32_t* whits = s_hits + warp * kHitCap;
  const uint32_t cap = a.entry_cap;
  bool overflow = false;

  for (;;) {
    uint32_t tile = 0;
    if (lane == 0) tile = atomicAdd(&a.fc->tile_ctr[1], 1u);
    tile = __shfl_sync(0xffffffffu, tile, 0);
    if (tile >= num_tiles) break;
    const uint32_t s = tile * 32u + lane;  // slot in depth order
    uint32_t sid = kInvalid, dq = 0;
    if (s < active && s < a.max_n) {
      sid = a.order_ids[s];
      dq = a.order_keys[s];
    }
    const SplatBox b = load_box(a, sid, active);

    // Stage the warp's splats.
    const uint32_t bw = b.valid ? (b.x1 - b.x0 + 1u) : 0u;
    const uint32_t bh = b.valid ? (b.y1 - b.y0 + 1u) : 0u;
    const uint32_t ncand = bw * bh;
    uint32_t incl = ncand, cincl = bw, rincl = bh;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
      const uint32_t yc = __shfl_up_sync(0xffffffffu, cincl, o);
      const uint32_t yr = __shfl_up_sync(0xffffffffu, rincl, o);
      if (lane >= o) {
        incl += y;
        cincl += yc;
        rincl += yr;
      }
    }
    const uint32_t base = incl - ncand;
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    const uint32_t wt = __shfl_sync(0xffffffffu, cincl, 31);
    const uint32_t ht = __shfl_sync(0xffffffffu, rincl, 31);
    const bool tab = wt + ht <= (uint32_t)kTabCap;  // warp-uniform
    __syncwarp();  // the previous tile's readers are done with the warp's shared memory
    {
      const uint32_t w = b.valid ? bw : 1u;
      const float ca_ = fmaxf(b.ca, 1e-12f), cc_ = fmaxf(b.cc, 1e-12f);
      const float cb2 = __fmul_rn(2.0f, b.cb);
      const float qlim =
          __fadd_rn(b.valid ? clampf(__fmul_rn(2.0f, cgs_logf(__fmul_rn(255.0f, b.alpha))), 0.0f, 8.0f)
                            : 0.0f,
                    1e-4f);
      sp.box[warp][lane] =
          make_uint4(b.x0, b.y0, w, w <= 1u ? 0u : (uint32_t)(((1ull << 32) + w - 1u) / w));
      sp.geo[warp][lane] = make_float4(b.mu_x, b.mu_y, -b.cb, cb2);
      sp.con[warp][lane] = make_float4(b.ca, b.cc, ca_, cc_);
      sp.kq[warp][lane] = make_float4(b.ca, cb2, b.cc, qlim);
      sp.rcp[warp][lane] = make_double2(1.0 / (double)cc_, 1.0 / (double)ca_);
      sp.tb[warp][lane] = make_uint2(cincl - bw, wt + rincl - bh);
      sp.base[warp][lane] = base;
      sp.cpre[warp][lane] = cincl - bw;
      sp.rpre[warp][lane] = rincl - bh;
      sp.dq[warp][lane] = dq;
      sp.sid[warp][lane] = sid;
    }
    if (lane < (int)kMaxGroups) s_gcnt[lane] = 0u;
    const bool big = total > (uint32_t)kMaskCap * 32u;  // warp-uniform
    if (!big) {
#pragma unroll
      for (int k = lane; k < kMaskCap; k += 32) sp.sbits[warp][k] = 0u;
      const uint32_t nonempty = __ballot_sync(0xffffffffu, ncand > 0u);
      if (ncand > 0u) sp.lor[warp][__popc(nonempty & lt)] = (uint32_t)lane;
      __syncwarp();
      if (ncand > 0u) atomicOr(&sp.sbits[warp][base >> 5], 1u << (base & 31u));
    }
    __syncwarp();
    if (tab) {
      // 0. term tables: columns [0, wt), rows [wt, wt + ht)
      for (uint32_t i = lane; i < wt; i += 32) {
        const int o = find_owner(sp.cpre[warp], i);
        wtab[i] = col_terms(sp.box[warp][o].x + (i - sp.cpre[warp][o]), lw, wm1, sp.geo[warp][o],
                            sp.con[warp][o], sp.rcp[warp][o]);
      }
      for (uint32_t i = lane; i < ht; i += 32) {
        const int o = find_owner(sp.rpre[warp], i);
        wtab[wt + i] = row_terms(sp.box[warp][o].y + (i - sp.rpre[warp][o]), lh, hm1,
                                 sp.geo[warp][o], sp.con[warp][o], sp.rcp[warp][o]);
      }
      __syncwarp();
    }
    // the exact test of candidate ci of lane o's splat; tx, ty its tile
    auto test = [&](int o, uint32_t ci, uint32_t& tx, uint32_t& ty) -> bool {
      const uint4 bx = sp.box[warp][o];
      uint32_t r, c;
      box_rc(bx, ci, r, c);
      tx = bx.x + c;
      ty = bx.y + r;
      if (tab) {
        const uint2 t = sp.tb[warp][o];
        return tab_hit(wtab[t.x + c], wtab[t.y + r], sp.kq[warp][o]);
      }
      return tile_hit(tx, ty, wm1, hm1, lw, lh, sp.geo[warp][o], sp.con[warp][o], sp.rcp[warp][o],
                      sp.kq[warp][o].w);
    };

    // 1. count
    uint32_t run = 0;     // hits before the current chunk (warp-uniform)
    uint32_t own = 0;     // this lane's hits, accumulated only when `big`
    uint32_t starts = 0;  // splats starting before the current chunk
    const uint32_t upto = (2u << lane) - 1u;  // bits 0 .. lane
    for (uint32_t chunk = 0, c = 0; chunk < total; chunk += 32, ++c) {
      const uint32_t item = chunk + lane;
      bool hit = false;
      uint32_t rec = 0;
      // owner of `item`: the k-th splat with candidates, k = the starts at or
      // before it (a popcount instead of a search)
      uint32_t sb = 0;
      if (!big) sb = sp.sbits[warp][c];
      if (item < total) {
        const int o = big ? find_owner(wbase, item)
                          : (int)sp.lor[warp][starts + __popc(sb & upto) - 1u];
        const uint32_t ci = item - wbase[o];
        uint32_t tx, ty;
        hit = test(o, ci, tx, ty);
        rec = ((ty * a.tiles_x + tx) << 5) | (uint32_t)o;
      }
      const uint32_t hits = __ballot_sync(0xffffffffu, hit);
      if (lane == 0 && c < (uint32_t)kMaskCap) {
        wmask[c] = hits;
        wmrun[c] = run;
      }
      if (hit) {
        const uint32_t k = run + __popc(hits & lt);
        if (k < (uint32_t)kHitCap) whits[k] = rec;
      }
      if (big) {
        const int lo = base > chunk ? (int)min(base - chunk, 32u) : 0;
        const int hi = (base + ncand) > chunk ? (int)min(base + ncand - chunk, 32u) : 0;
        own += __popc(hits & seg_mask(lo, hi));
      }
      {  // hits per tile group (one counter update per group present)
        const uint32_t g = hit ? (rec >> 5) >> gshift : 0xFFFFFFFFu;
        const uint32_t peers = __match_any_sync(0xffffffffu, g);
        if (hit && lane == 31 - __clz(peers)) s_gcnt[g] += __popc(peers);
        __syncwarp();
      }
      run += __popc(hits);
      starts += __popc(sb);
    }
    __syncwarp();
    uint32_t count = own;
    if (!big) {
      // hits before this lane's first candidate, from the stored masks
      uint32_t before = run;
      if (base < total) {
        const uint32_t c = base >> 5;
        before = wmrun[c] + __popc(wmask[c] & ((1u << (base & 31u)) - 1u));
      }
      const uint32_t next = __shfl_down_sync(0xffffffffu, before, 1);
      count = (lane == 31 ? run : next) - before;
    }
    if (s < a.max_n) a.offsets[s] = count;  // scanned afterwards

    // 2. stage: one run per tile group, each in the hits' order: record =
    // tile << 5 | slot lane.
    {
      if (lane < (int)G) {
        const uint32_t gc = s_gcnt[lane];
        const unsigned long long gb64 =
            gc ? atomicAdd(&a.fc->stage_ctr, (unsigned long long)gc) : 0ull;
        const uint32_t gb = gb64 >= cap ? cap : (uint32_t)gb64;  // at or past cap: not staged
        a.tile_stage[(size_t)tile * G + lane] = gb;
        a.tile_count[(size_t)tile * G + lane] = gc;
        s_gbase[lane] = gb;
        s_grun[lane] = 0u;
      }
      __syncwarp();
      // called by the whole warp with the lanes' hits in order
      auto put_rec = [&](bool h, uint32_t rec) {
        const uint32_t g = h ? (rec >> 5) >> gshift : 0xFFFFFFFFu;
        const uint32_t peers = __match_any_sync(0xffffffffu, g);
        if (h) {
          const uint64_t pos = (uint64_t)s_gbase[g] + s_grun[g] + __popc(peers & lt);
          if (pos < cap)
            a.stage_keys[pos] = rec;
          else
            overflow = true;
        }
        __syncwarp();
        if (h && lane == 31 - __clz(peers)) s_grun[g] += __popc(peers);
        __syncwarp();
      };
      const uint32_t stored = min(run, (uint32_t)kHitCap);
      for (uint32_t k0 = 0; k0 < stored; k0 += 32) {
        const uint32_t k = k0 + lane;
        put_rec(k < stored, k < stored ? whits[k] : 0u);
      }
      if (run > (uint32_t)kHitCap) {
        uint32_t hrun = 0;
        for (uint32_t chunk = 0, c = 0; chunk < total; chunk += 32, ++c) {
          uint32_t hits;
          const uint32_t item = chunk + lane;
          if (c < (uint32_t)kMaskCap) {
            hits = wmask[c];
            hrun = wmrun[c];
            if (hrun + __popc(hits) <= (uint32_t)kHitCap) {
              hrun += __popc(hits);
              continue;
            }
          } else {
            bool hit = false;
            if (item < total) {
              const int o = find_owner(wbase, item);
              uint32_t tx, ty;
              hit = test(o, item - wbase[o], tx, ty);
            }
            hits = __ballot_sync(0xffffffffu, hit);
          }
          const uint32_t k = hrun + __popc(hits & lt);
          const bool sel = ((hits >> lane) & 1u) && k >= (uint32_t)kHitCap;
          uint32_t rec = 0;
          if (sel) {
            const int o = find_owner(wbase, item);
            uint32_t r, cc;
            box_rc(sp.box[warp][o], item - wbase[o], r, cc);
            rec = (((sp.box[warp][o].y + r) * a.tiles_x + sp.box[warp][o].x + cc) << 5) | (uint32_t)o;
          }
          put_rec(sel, rec);
          hrun += __popc(hits);
        }
      }
    }
  }
  if (overflow) atomicOr(&a.fc->status, kStatusCapacity);
}

// ---- Binning, direct mode ---------------------------------------------------
// The radix path's binning in one launch (the record mode of the tile
// transpose stays with k_bin_count). Per 32-slot tile (a warp's 32 splats in
// depth order, tiles taken from a counter in increasing order):
//   setup:  tile boxes, candidate and box-edge prefixes, per-splat constants
//           in shared memory; a start bit at each splat's first candidate and
//           the lane of each splat with candidates, so that a candidate's
//           splat is found by a popcount (no search);
//   tables: the column and row terms of the 32 tile boxes (tile_hit's
//           column-only and row-only parts);
//   count:  32 candidates per step, one per lane, ~20 rounded operations
//           each against the tables (the whole test when the tables do not
//           fit); the ballot masks and the hits before each are kept;
//   scan:   the tile's hit count enters a decoupled look-back over the 32-slot
//           tiles (saturating sums): the slots' scanned offsets and the tile's
//           first entry;
//   write:  the stored masks are walked again and every hit is written at
//           its place in depth order (key, splat index, 64-bit: depth word)
//           and counted in per-warp histograms of the entry sort's digits.
// The scan and write of a tile are deferred by one tile: a warp publishes the
// hit count of the tile it has just counted, then walks back and writes the
// tile it counted before, whose predecessors have had a whole count step to
// publish theirs. The state the write needs (owners, depth keys, splat
// indices, masks) is therefore kept for two tiles per warp. A tile with more
// candidates than the masks hold is scanned and written at once, testing the
// rest of its candidates again. Entries at or beyond the capacity are not
// written and set the capacity bit.
constexpr int kDirMaskCap = 64;   // stored ballot masks per warp and tile (2,048 candidates)
constexpr int kDirTabCap = 440;   // term-table entries per warp

struct DirSplats {
  // the tile being counted
  uint2 tb[kBinWarps][32];     // first column entry, first row entry in the term table
  uint2 xy[kBinWarps][32];     // box origin (tiles)
  float4 kq[kBinWarps][32];    // a, 2b, c, q_max + 1e-4
  float4 geo[kBinWarps][32];   // mu_x, mu_y, -b, 2b
  float4 con[kBinWarps][32];   // a, c, max(a, 1e-12), max(c, 1e-12)
  double2 rcp[kBinWarps][32];  // RN64(1 / max(c, 1e-12)), RN64(1 / max(a, 1e-12))
  uint32_t base[kBinWarps][32];
  uint32_t cpre[kBinWarps][32];
  uint32_t rpre[kBinWarps][32];
  // what the write needs, for two tiles (the one counted and the one before)
  uint4 own[2][kBinWarps][32];  // first candidate, ceil(2^32 / width) (0 if width 1), width, first tile id
  uint32_t dq[2][kBinWarps][32];
  uint32_t sid[2][kBinWarps][32];
  uint32_t lor[2][kBinWarps][32];             // lane of the k-th splat with candidates
  uint32_t sbits[2][kBinWarps][kDirMaskCap];  // start bit per splat's first candidate
  uint32_t mask[2][kBinWarps][kDirMaskCap];   // hit ballots
  uint32_t mrun[2][kBinWarps][kDirMaskCap];   // hits before each ballot
};
// tile-digit histograms: one per warp when a histogram has at most
// kDirWarpBins bins (no contention between warps), else one per block
constexpr uint32_t kDirWarpBins = 256;
constexpr size_t kDirSmem = sizeof(DirSplats) + sizeof(float4) * kBinWarps * kDirTabCap +
                            sizeof(uint32_t) * kBinWarps * kDirWarpBins;
static_assert(kBinWarps * kDirWarpBins >= 1024, "a block histogram of 4 x 256 bins fits");
// two blocks per SM: 228 KB of shared memory, 1 KB of it reserved per block
static_assert(2 * (kDirSmem + 1024) <= 233472, "two binning blocks per SM");

template <bool KEY64>
__global__ void __launch_bounds__(kBinThreads, 2) k_bin_direct(const BinArgs a) {
  extern __shared__ __align__(16) unsigned char dir_smem[];
  DirSplats& sp = *reinterpret_cast<DirSplats*>(dir_smem);
  float4* s_tab = reinterpret_cast<float4*>(dir_smem + sizeof(DirSplats));  // [w][kDirTabCap]
  uint32_t* s_hist = reinterpret_cast<uint32_t*>(s_tab + kBinWarps * kDirTabCap);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t radix = 1u << a.radix_bits, rmask = radix - 1u;
  const uint32_t tshift = KEY64 ? 0u : a.depth_bits;  // tile bits of the sort word
  const uint32_t passes = (a.tile_bits + a.radix_bits - 1u) / a.radix_bits;
  const uint32_t nbins = passes * radix;
  const uint32_t wm1 = a.width - 1u, hm1 = a.height - 1u;
  const uint32_t lw = a.tile_w_log2, lh = a.tile_h_log2;
  const bool warp_hist = nbins <= kDirWarpBins;
  const uint32_t hist_words = warp_hist ? kBinWarps * nbins : nbins;
  for (uint32_t k = threadIdx.x; k < hist_words; k += kBinThreads) s_hist[k] = 0u;
  __syncthreads();
  uint32_t* whist = warp_hist ? s_hist + warp * nbins : s_hist;
  const uint32_t lt = lanemask_lt();
  const uint32_t upto = (2u << lane) - 1u;  // lanes 0 .. lane
  const uint32_t active = a.n_rest + (a.split_count ? *a.split_count : 0u);
  const uint32_t num_tiles = (a.max_n + 31u) / 32u;
  const uint32_t* wbase = sp.base[warp];
  float4* wtab = s_tab + warp * kDirTabCap;
  const uint32_t cap = a.entry_cap;
  bool overflow = false;

  // owner (lane) of candidate `item` in write buffer q; sb = start bits of its
  // chunk, starts = splats starting before the chunk
  auto owner = [&](int q, bool big, uint32_t item, uint32_t sb, uint32_t starts) -> int {
    return big ? find_owner(wbase, item) : (int)sp.lor[q][warp][starts + __popc(sb & upto) - 1u];
  };
  // the test of candidate item of splat o (the tile being counted, buffer q)
  auto test = [&](int q, bool tab, int o, uint32_t item) -> bool {
    const uint4 ow = sp.own[q][warp][o];
    const uint32_t ci = item - ow.x;
    const uint32_t r = ow.y ? __umulhi(ci, ow.y) : ci;
    const uint32_t c = ci - r * ow.z;
    if (tab) {
      const uint2 t = sp.tb[warp][o];
      return tab_hit(wtab[t.x + c], wtab[t.y + r], sp.kq[warp][o]);
    }
    const uint2 xy = sp.xy[warp][o];
    return tile_hit(xy.x + c, xy.y + r, wm1, hm1, lw, lh, sp.geo[warp][o], sp.con[warp][o],
                    sp.rcp[warp][o], sp.kq[warp][o].w);
  };
  // Scan and write of a counted tile whose masks are in buffer q (a tile with
  // more candidates than the masks hold tests the rest again: only at once,
  // while its test state is the current one).
  auto scan_write = [&](int q, uint32_t tile, uint32_t total, bool big, bool tab, uint32_t run,
                        uint32_t count, uint32_t s) {
    const uint32_t wexcl = chained_resolve<true>(a.lookback, tile, run, &a.fc->status);
    {
      uint32_t cincl2 = count;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, cincl2, o);
        if (lane >= o) cincl2 += y;
      }
      if (s < a.max_n) a.offsets[s] = sat_add_u32(wexcl, cincl2 - count);
      if (tile == num_tiles - 1u && lane == 0) a.fc->entries = sat_add_u32(wexcl, run);
    }
    const uint32_t* qmask = sp.mask[q][warp];
    const uint32_t* qsbits = sp.sbits[q][warp];
    uint32_t hrun = 0, starts = 0;
#pragma unroll 2
    for (uint32_t chunk = 0, c = 0; chunk < total; chunk += 32, ++c) {
      const uint32_t item = chunk + lane;
      const uint32_t sb = big ? 0u : qsbits[c];
      uint32_t hits;
      if (c < (uint32_t)kDirMaskCap) {
        hits = qmask[c];
      } else {
        bool h = false;
        if (item < total) h = test(q, tab, owner(q, big, item, sb, starts), item);
        hits = __ballot_sync(0xffffffffu, h);
      }
      const bool hit = (hits >> lane) & 1u;
      uint32_t word = 0;
      if (hit) {
        const int o = owner(q, big, item, sb, starts);
        const uint4 ow = sp.own[q][warp][o];
        const uint32_t ci = item - ow.x;
        const uint32_t r = ow.y ? __umulhi(ci, ow.y) : ci;
        const uint32_t cc = ci - r * ow.z;
        const uint32_t tile_id = ow.w + r * a.tiles_x + cc;
        const uint32_t d = sp.dq[q][warp][o];
        word = KEY64 ? tile_id : (a.depth_bits >= 32u ? d : ((tile_id << a.depth_bits) | d));
        const uint64_t pos = (uint64_t)wexcl + hrun + __popc(hits & lt);
        if (pos < cap) {
          a.keys[pos] = word;
          a.ids[pos] = sp.sid[q][warp][o];
          if (KEY64) a.depths[pos] = d;
        } else {
          overflow = true;
        }
      }
      // the entry sort's digits (per-warp histograms)
      if (hit) {
        atomicAdd(&whist[(word >> tshift) & rmask], 1u);
        for (uint32_t p = 1; p < passes; ++p)
          atomicAdd(&whist[p * radix + ((word >> (tshift + p * a.radix_bits)) & rmask)], 1u);
      }
      hrun += __popc(hits);
      starts += __popc(sb);
    }
  };

  int cur = 0;        // write buffer of the tile being counted
  bool pend = false;  // a counted tile waits for its scan and write (buffer cur ^ 1)
  uint32_t p_tile = 0, p_total = 0, p_run = 0, p_count = 0, p_s = 0;
  for (;;) {
    uint32_t tile = 0;
    if (lane == 0) tile = atomicAdd(&a.fc->tile_ctr[1], 1u);
    tile = __shfl_sync(0xffffffffu, tile, 0);
    const bool have = tile < num_tiles;  // warp-uniform
    uint32_t s = 0, total = 0, run = 0, count = 0;
    bool big = false, tab = false;
    if (have) {
      s = tile * 32u + lane;  // slot in depth order
      uint32_t sid = kInvalid, dq = 0;
      if (s < active && s < a.max_n) {
        sid = a.order_ids[s];
        dq = a.order_keys[s];
      }
      const SplatBox b = load_box(a, sid, active);

      // ---- setup
      const uint32_t bw = b.valid ? (b.x1 - b.x0 + 1u) : 0u;
      const uint32_t bh = b.valid ? (b.y1 - b.y0 + 1u) : 0u;
      const uint32_t ncand = bw * bh;
      uint32_t incl = ncand, cincl = bw, rincl = bh;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        const uint32_t yc = __shfl_up_sync(0xffffffffu, cincl, o);
        const uint32_t yr = __shfl_up_sync(0xffffffffu, rincl, o);
        if (lane >= o) {
          incl += y;
          cincl += yc;
          rincl += yr;
        }
      }
      const uint32_t base = incl - ncand;
      total = __shfl_sync(0xffffffffu, incl, 31);
      const uint32_t wt = __shfl_sync(0xffffffffu, cincl, 31);
      const uint32_t ht = __shfl_sync(0xffffffffu, rincl, 31);
      tab = wt + ht <= (uint32_t)kDirTabCap;       // warp-uniform
      big = total > (uint32_t)kDirMaskCap * 32u;   // warp-uniform
      const uint32_t nonempty = __ballot_sync(0xffffffffu, ncand > 0u);
      __syncwarp();  // earlier readers are done with this buffer and the test state
      {
        const uint32_t w = b.valid ? bw : 1u;
        const float ca_ = fmaxf(b.ca, 1e-12f), cc_ = fmaxf(b.cc, 1e-12f);
        const float cb2 = __fmul_rn(2.0f, b.cb);
        const float qlim =
            __fadd_rn(b.valid ? clampf(__fmul_rn(2.0f, cgs_logf(__fmul_rn(255.0f, b.alpha))), 0.0f, 8.0f)
                              : 0.0f,
                      1e-4f);
        sp.own[cur][warp][lane] =
            make_uint4(base, w <= 1u ? 0u : (uint32_t)(((1ull << 32) + w - 1u) / w), w,
                       b.y0 * a.tiles_x + b.x0);
        sp.tb[warp][lane] = make_uint2(cincl - bw, wt + rincl - bh);
        sp.xy[warp][lane] = make_uint2(b.x0, b.y0);
        sp.kq[warp][lane] = make_float4(b.ca, cb2, b.cc, qlim);
        sp.geo[warp][lane] = make_float4(b.mu_x, b.mu_y, -b.cb, cb2);
        sp.con[warp][lane] = make_float4(b.ca, b.cc, ca_, cc_);
        sp.rcp[warp][lane] = make_double2(1.0 / (double)cc_, 1.0 / (double)ca_);
        sp.base[warp][lane] = base;
        sp.cpre[warp][lane] = cincl - bw;
        sp.rpre[warp][lane] = rincl - bh;
        sp.dq[cur][warp][lane] = dq;
        sp.sid[cur][warp][lane] = sid;
        if (ncand > 0u) sp.lor[cur][warp][__popc(nonempty & lt)] = (uint32_t)lane;
        if (!big) {
#pragma unroll
          for (int k = lane; k < kDirMaskCap; k += 32) sp.sbits[cur][warp][k] = 0u;
        }
      }
      __syncwarp();
      if (!big && ncand > 0u) atomicOr(&sp.sbits[cur][warp][base >> 5], 1u << (base & 31u));
      // ---- tables: columns [0, wt), rows [wt, wt + ht)
      if (tab) {
        for (uint32_t i = lane; i < wt; i += 32) {
          const int o = find_owner(sp.cpre[warp], i);
          wtab[i] = col_terms(sp.xy[warp][o].x + (i - sp.cpre[warp][o]), lw, wm1, sp.geo[warp][o],
                              sp.con[warp][o], sp.rcp[warp][o]);
        }
        for (uint32_t i = lane; i < ht; i += 32) {
          const int o = find_owner(sp.rpre[warp], i);
          wtab[wt + i] = row_terms(sp.xy[warp][o].y + (i - sp.rpre[warp][o]), lh, hm1,
                                   sp.geo[warp][o], sp.con[warp][o], sp.rcp[warp][o]);
        }
      }
      __syncwarp();
      // ---- count
      uint32_t* wmask = sp.mask[cur][warp];
      uint32_t* wmrun = sp.mrun[cur][warp];
      uint32_t own = 0;     // this lane's hits, accumulated only when `big`
      uint32_t starts = 0;  // splats starting before the current chunk
#pragma unroll 2
      for (uint32_t chunk = 0, c = 0; chunk < total; chunk += 32, ++c) {
        const uint32_t item = chunk + lane;
        const uint32_t sb = big ? 0u : sp.sbits[cur][warp][c];
        bool hit = false;
        if (item < total) hit = test(cur, tab, owner(cur, big, item, sb, starts), item);
        const uint32_t hits = __ballot_sync(0xffffffffu, hit);
        if (lane == 0 && c < (uint32_t)kDirMaskCap) {
          wmask[c] = hits;
          wmrun[c] = run;
        }
        if (big) {
          const int lo = base > chunk ? (int)min(base - chunk, 32u) : 0;
          const int hi = (base + ncand) > chunk ? (int)min(base + ncand - chunk, 32u) : 0;
          own += __popc(hits & seg_mask(lo, hi));
        }
        run += __popc(hits);
        starts += __popc(sb);
      }
      __syncwarp();
      count = own;
      if (!big) {
        // hits before this lane's first candidate, from the stored masks
        uint32_t before = run;
        if (base < total) {
          const uint32_t c = base >> 5;
          before = wmrun[c] + __popc(wmask[c] & ((1u << (base & 31u)) - 1u));
        }
        const uint32_t next = __shfl_down_sync(0xffffffffu, before, 1);
        count = (lane == 31 ? run : next) - before;
      }
      // publish this tile's hit count before any wait
      chained_publish(a.lookback, tile, run);
    }
    // ---- scan and write of the tile counted before this one
    if (pend) {
      scan_write(cur ^ 1, p_tile, p_total, false, false, p_run, p_count, p_s);
      pend = false;
    }
    if (!have) break;
    if (big) {
      scan_write(cur, tile, total, true, tab, run, count, s);
    } else {
      pend = true;
      p_tile = tile;
      p_total = total;
      p_run = run;
      p_count = count;
      p_s = s;
      cur ^= 1;
    }
  }
  if (overflow) atomicOr(&a.fc->status, kStatusCapacity);
  __syncthreads();
  for (uint32_t k = threadIdx.x; k < nbins; k += kBinThreads) {
    uint32_t v = 0;
    if (warp_hist) {
      for (int w = 0; w < kBinWarps; ++w) v += s_hist[w * nbins + k];
    } else {
      v = s_hist[k];
    }
    if (v) atomicAdd(&a.hist[k], v);
  }
}

// ---- Tile transpose ---------------------------------------------------------
// The binning kernel stages each 32-slot tile's hits in the reference's
// emission order. Sorting them stably by tile is a transpose of the
// (slot, tile) incidence from slot-major to tile-major; with few enough
// screen tiles it is done in one counting pass instead of radix passes:
//   k_chunk_counts: entries of every (tile, chunk) pair;
//   scan of the per-tile totals (launch_scan_u32) -> each tile's first entry;
//   k_column_scan:  per tile, exclusive scan over the chunks -> each
//                   (tile, chunk) pair's first entry; tile ranges;
//   k_chunk_place:  per (chunk, group of tiles): each warp counts its eighth
//                   of the chunk per tile, the counts are turned into per-warp
//                   bases, and each warp walks its records again in order,
//                   ranking equal tiles with match_any and per-warp counters,
//                   and writes every splat index to its final entry.
// The order inside a tile is chunk, then warp, then record order: the slots'
// (depth, splat index) order, as the reference's stable key sort gives.

// A warp's walk over the records of group g in the 32-slot tiles [w0, w1):
// the run descriptors (length, staging start) of 32 tiles at a time sit one
// per lane; their records are concatenated and taken 32 at a time, one per
// lane, in order. Each lane finds its record's run by a 5-step search over
// the runs' exclusive prefix (held in lanes).
struct RunWalk {
  uint32_t n, st, pre, total;  // this lane's run: length, start, exclusive prefix; sum
  __device__ __forceinline__ void load(const TransposeArgs& a, uint32_t wb, uint32_t w1,
                                       uint32_t g, int lane) {
    n = 0;
    st = 0;
    if (wb + lane < w1) {
      n = a.tile_count[(size_t)(wb + lane) * a.groups + g];
      st = a.tile_stage[(size_t)(wb + lane) * a.groups + g];
    }
    uint32_t incl = n;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    pre = incl - n;
    total = __shfl_sync(0xffffffffu, incl, 31);
  }
  // run (lane) holding record i (< total) of the concatenation, and its address
  __device__ __forceinline__ int find(uint32_t i, uint32_t& addr) const {
    int q = 0;
#pragma unroll
    for (int step = 16; step >= 1; step >>= 1)
      if (__shfl_sync(0xffffffffu, pre, q + step) <= i) q += step;
    addr = __shfl_sync(0xffffffffu, st, q) + (i - __shfl_sync(0xffffffffu, pre, q));
    return q;
  }
};

// Entries of every (tile, chunk) pair of one tile group, and per-tile totals.
// Block (chunk k, group g); warp w walks the w-th eighth of the chunk.
__global__ void __launch_bounds__(256) k_chunk_counts(const TransposeArgs a) {
  __shared__ uint32_t s_cnt[kTransposeGroupTiles];
  const uint32_t k = blockIdx.x, g = blockIdx.y;
  const uint32_t t0 = g * a.group_tiles;
  const uint32_t tn = min(a.group_tiles, a.num_tiles - t0);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (uint32_t t = threadIdx.x; t < tn; t += blockDim.x) s_cnt[t] = 0u;
  __syncthreads();
  const uint32_t sub = a.chunk_wtiles / 8;
  const uint32_t w0 = min(k * a.chunk_wtiles + warp * sub, a.num_wtiles);
  const uint32_t w1 = min(w0 + sub, a.num_wtiles);
  for (uint32_t wb = w0; wb < w1; wb += 32) {
    RunWalk rw;
    rw.load(a, wb, w1, g, lane);
    for (uint32_t i0 = 0; i0 < rw.total; i0 += 32) {
      uint32_t addr;
      rw.find(i0 + lane, addr);
      if (i0 + lane < rw.total && addr < a.capacity) {
        const uint32_t t = (__ldg(a.records + addr) >> 5) - t0;
        if (t < tn) atomicAdd(&s_cnt[t], 1u);
      }
    }
  }
  __syncthreads();
  for (uint32_t t = threadIdx.x; t < tn; t += blockDim.x) {
    const uint32_t c = s_cnt[t];
    a.cmat[(size_t)(t0 + t) * a.num_chunks + k] = c;
    if (c) atomicAdd(&a.totals[t0 + t], c);
  }
}

// One warp per tile: first entry of each (tile, chunk) pair, and the range.
__global__ void __launch_bounds__(256) k_column_scan(const TransposeArgs a) {
  const uint32_t t = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (t >= a.num_tiles) return;
  uint32_t run = a.tile_base[t];
  uint32_t* row = a.cmat + (size_t)t * a.num_chunks;
  for (uint32_t k0 = 0; k0 < a.num_chunks; k0 += 32) {
    const uint32_t k = k0 + lane;
    const uint32_t v = k < a.num_chunks ? row[k] : 0u;
    uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    if (k < a.num_chunks) row[k] = run + incl - v;
    run += __shfl_sync(0xffffffffu, incl, 31);
  }
  if (lane == 0) {
    const uint32_t total = a.totals[t], base = a.tile_base[t];
    a.ranges[2 * (size_t)t] = total ? base : 0u;
    a.ranges[2 * (size_t)t + 1] = total ? base + total : 0u;
  }
}

// Block (chunk k, tile group g): places the chunk's entries of the group.
// Shared memory: per-warp counters (two 16-bit counters per word: a warp's
// eighth of a chunk holds fewer than 2^16 slots, and so does a chunk) and the
// chunk's first entry per tile.
constexpr int kPlaceWarps = 8;

__global__ void __launch_bounds__(kPlaceWarps * 32) k_chunk_place(const TransposeArgs a) {
  constexpr uint32_t GW = kTransposeGroupTiles / 2;
  __shared__ uint32_t whist[kPlaceWarps * GW];
  __shared__ uint32_t obase[kTransposeGroupTiles];
  const uint32_t k = blockIdx.x, g = blockIdx.y;
  const uint32_t t0 = g * a.group_tiles;
  const uint32_t tn = min(a.group_tiles, a.num_tiles - t0);  // tiles of this group
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (uint32_t i = threadIdx.x; i < kPlaceWarps * GW; i += blockDim.x) whist[i] = 0u;
  for (uint32_t i = threadIdx.x; i < tn; i += blockDim.x)
    obase[i] = a.cmat[(size_t)(t0 + i) * a.num_chunks + k];
  // this warp's eighth of the chunk (at most 32 32-slot tiles per descriptor load)
  const uint32_t sub = a.chunk_wtiles / kPlaceWarps;
  const uint32_t w0 = min(k * a.chunk_wtiles + warp * sub, a.num_wtiles);
  const uint32_t w1 = min(w0 + sub, a.num_wtiles);
  __syncthreads();
  uint32_t* wh = whist + warp * GW;
  // 1. per-warp counts
  for (uint32_t wb = w0; wb < w1; wb += 32) {
    RunWalk rw;
    rw.load(a, wb, w1, g, lane);
    for (uint32_t i0 = 0; i0 < rw.total; i0 += 32) {
      uint32_t addr;
      rw.find(i0 + lane, addr);
      if (i0 + lane < rw.total && addr < a.capacity) {
        const uint32_t t = (__ldg(a.records + addr) >> 5) - t0;
        if (t < tn) atomicAdd(&wh[t >> 1], 1u << ((t & 1u) * 16u));
      }
    }
  }
  __syncthreads();
  // 2. counts -> per-warp exclusive bases (both halves of a word at once)
  for (uint32_t j = threadIdx.x; j < GW; j += blockDim.x) {
    uint32_t lo = 0, hi = 0;
#pragma unroll
    for (int w = 0; w < kPlaceWarps; ++w) {
      const uint32_t c = whist[w * GW + j];
      whist[w * GW + j] = lo | (hi << 16);
      lo += c & 0xFFFFu;
      hi += c >> 16;
    }
  }
  __syncthreads();
  // 3. stable placement: records in order, equal tiles ranked by lane; the
  // next batch's record and this batch's splat index are loaded ahead.
  const uint32_t lt = lanemask_lt();
  bool bad = false;
  for (uint32_t wb = w0; wb < w1; wb += 32) {
    RunWalk rw;
    rw.load(a, wb, w1, g, lane);
    auto fetch = [&](uint32_t i0, uint32_t& rec, uint32_t& wt) {
      uint32_t addr;
      const int q = rw.find(i0 + lane, addr);
      wt = wb + (uint32_t)q;
      rec = 0xFFFFFFFFu;
      if (i0 + lane < rw.total && addr < a.capacity) rec = __ldg(a.records + addr);
    };
    uint32_t rec, wt;
    if (rw.total) fetch(0, rec, wt);
    for (uint32_t i0 = 0; i0 < rw.total; i0 += 32) {
      const uint32_t sidx = rec == 0xFFFFFFFFu ? 0u : __ldg(a.order_ids + 32u * wt + (rec & 31u));
      uint32_t t = rec == 0xFFFFFFFFu ? 0xFFFFFFFFu : (rec >> 5) - t0;
      if (t >= tn) t = 0xFFFFFFFFu;
      uint32_t nrec = 0xFFFFFFFFu, nwt = wt;
      if (i0 + 32 < rw.total) fetch(i0 + 32, nrec, nwt);
      const uint32_t peers = __match_any_sync(0xffffffffu, t);
      const int leader = 31 - __clz(peers);
      uint32_t old = 0;
      if (lane == leader && t != 0xFFFFFFFFu) {
        const uint32_t sh = (t & 1u) * 16u;
        old = (atomicAdd(&wh[t >> 1], (uint32_t)__popc(peers) << sh) >> sh) & 0xFFFFu;
      }
      old = __shfl_sync(0xffffffffu, old, leader);
      if (t != 0xFFFFFFFFu) {
        const uint32_t pos = obase[t] + old + __popc(peers & lt);
        if (pos < a.capacity)
          a.ids_out[pos] = sidx;
        else
          bad = true;
      }
      rec = nrec;
      wt = nwt;
    }
  }
  if (bad) atomicOr(a.status_word, kStatusCapacity);
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

// [first, end) of every screen tile from the last sort pass's words:
// ranges[2 t] = ~first (0 when the tile is empty), ranges[2 t + 1] = end.
__global__ void k_ranges_fixup(uint32_t* __restrict__ ranges, uint32_t num_tiles) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= num_tiles) return;
  const uint32_t x = ranges[2 * (size_t)t];
  if (x != 0u) ranges[2 * (size_t)t] = ~x;
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

// Wait drill: one warp runs the chained scan as tile 1 of a status array
// whose tile 0 nothing publishes (two zeroed 64-bit words), so its look-back
// polls until `limit` and sets the timeout bit.
__global__ void k_drill_chained_scan(unsigned long long* status, uint32_t* status_word,
                                     uint32_t limit) {
  chained_scan_warp(status, 1u, 1u, status_word, limit);
}

}  // namespace

cudaError_t launch_drill_chained_scan(unsigned long long* status, uint32_t* status_word,
                                      uint32_t limit, cudaStream_t s) {
  k_drill_chained_scan<<<1, 32, 0, s>>>(status, status_word, limit);
  return cudaGetLastError();
}

// Persistent grid: as many blocks as fit on the device at once (at most one
// warp per 32-slot tile).
// Persistent grid of kernel K (k_bin_count or k_bin_direct) with `smem`
// bytes per block: as many blocks as fit on the device at once (at most one
// warp per 32-slot tile), or fewer when the launch shape asks.
template <typename K>
cudaError_t launch_persistent_bin(K kernel, size_t smem, int* resident, int* sm_count,
                                  const BinArgs& a, cudaStream_t s) {
  if (*resident == 0) {
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 0, per_sm = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kBinThreads, smem)) !=
        cudaSuccess)
      return e;
    *resident = std::max(1, sms * std::max(per_sm, 1));
    *sm_count = std::max(1, sms);
  }
  uint32_t want = (uint32_t)*resident;
  if (a.blocks_per_sm) want = std::min<uint32_t>(want, a.blocks_per_sm * (uint32_t)*sm_count);
  const uint32_t tiles = (a.max_n + 31u) / 32u;
  const uint32_t blocks = std::min<uint32_t>(want, (tiles + kBinWarps - 1) / kBinWarps);
  kernel<<<blocks, kBinThreads, smem, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_bin_count(const BinArgs& a, cudaStream_t s) {
  if (a.max_n == 0) return cudaSuccess;
  if (a.width >= (1u << 22) || a.height >= (1u << 22)) return cudaErrorInvalidValue;
  static int res[4] = {0, 0, 0, 0}, sms[4] = {0, 0, 0, 0};
  if (a.records) {
    if (a.key64) return cudaErrorInvalidValue;  // records hold 27-bit tile ids
    return launch_persistent_bin(k_bin_count, kBinSmem, &res[0], &sms[0], a, s);
  }
  if (!a.lookback) return cudaErrorInvalidValue;
  return a.key64 ? launch_persistent_bin(k_bin_direct<true>, kDirSmem, &res[3], &sms[3], a, s)
                 : launch_persistent_bin(k_bin_direct<false>, kDirSmem, &res[2], &sms[2], a, s);
}

cudaError_t launch_chunk_counts(const TransposeArgs& a, cudaStream_t s) {
  if (a.num_chunks == 0 || a.num_tiles == 0) return cudaSuccess;
  if (a.group_tiles > kTransposeGroupTiles || a.groups * a.group_tiles < a.num_tiles)
    return cudaErrorInvalidValue;
  k_chunk_counts<<<dim3(a.num_chunks, a.groups), 256, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_column_scan(const TransposeArgs& a, cudaStream_t s) {
  if (a.num_tiles == 0) return cudaSuccess;
  k_column_scan<<<(a.num_tiles + 7) / 8, 256, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_chunk_place(const TransposeArgs& a, cudaStream_t s) {
  if (a.num_chunks == 0 || a.num_tiles == 0) return cudaSuccess;
  if (a.group_tiles > kTransposeGroupTiles || a.groups * a.group_tiles < a.num_tiles ||
      a.chunk_wtiles % kPlaceWarps != 0 || a.chunk_wtiles > 2040u)
    return cudaErrorInvalidValue;
  k_chunk_place<<<dim3(a.num_chunks, a.groups), kPlaceWarps * 32, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_ranges_fixup(uint32_t* ranges, uint32_t num_tiles, cudaStream_t s) {
  if (num_tiles == 0) return cudaSuccess;
  k_ranges_fixup<<<(num_tiles + 255) / 256, 256, 0, s>>>(ranges, num_tiles);
  return cudaGetLastError();
}

cudaError_t launch_tile_ranges(const uint32_t* sorted, uint32_t shift, const uint32_t* n_ptr,
                               uint32_t capacity, uint32_t total_tiles, uint32_t* ranges,
                               uint32_t blocks, cudaStream_t s) {
  k_tile_ranges<<<blocks ? blocks : 148 * 8, 256, 0, s>>>(sorted, shift, n_ptr, capacity,
                                                         total_tiles, ranges);
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
