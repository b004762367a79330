// Stable LSD radix sort of 32-bit keys with one or two 32-bit payload words,
// "onesweep" style (one kernel per digit pass, no separate scan pass), on
// sm_100a. Replaces gpu_radix_sort_u32_pairs / gpu_radix_sort_u64_pairs
// (render/kernels/radix_sort.rs:292-477), whose 4-bit passes each ran a
// histogram kernel, a 1-3 level scan and a scatter kernel.
//
// Per pass and per 4096-key tile (256 threads x 16 keys, warp-striped so a
// warp's item j is 32 consecutive keys):
//   1. keys and payloads are loaded coalesced into registers;
//   2. each warp ranks its 512 keys by digit, 32 at a time (the lanes sharing
//      a digit found by __match_any_sync, by one ballot per digit bit, or by
//      shared-memory peer masks, chosen per pass), keeping a per-warp digit
//      counter in shared memory (stable: ranks follow key order);
//   3. per-digit counts are published to a chained look-back array, one thread
//      per digit, and the keys are reordered by digit in shared memory (tile-
//      local offsets only);
//   4. the digit threads then collect the exclusive prefix over earlier tiles
//      (tiles are taken in order from an atomic counter, so every tile waited
//      on belongs to a resident block; waits are bounded by kSpinLimit polls),
//      and each digit's run is written out as a contiguous, mostly coalesced
//      store.
// The global digit offsets come from digit histograms of all passes, which the
// Stage 3 binning kernel accumulates while it writes the keys (launch_histogram
// does the same for standalone sorts); k_digit_bases turns them into
// exclusive bases once per sort. HBM traffic per pass: one read and one write
// of keys and payloads (16 B per pair), plus 1 KiB of look-back words per tile.
#include "kernels.h"

namespace cgs {
namespace {

constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;
constexpr uint32_t kSortTile = kSortThreads * kSortItems;  // 4096
constexpr int kSortWarps = kSortThreads / 32;
// Reorder buffers hold one padding word per 32 keys: the lanes of a warp
// whose keys fall in different digits write positions about one digit run
// (~32 keys) apart, which without padding map to the same bank.
constexpr uint32_t kSortTileP = kSortTile + kSortTile / 32;
__device__ __forceinline__ uint32_t padded(uint32_t i) { return i + (i >> 5); }
// Look-back words: a flag (tile count published / inclusive prefix
// published) above the count. 32-bit words carry counts below 2^30 (splat
// sorts, the stand-alone sorts); 64-bit words any 32-bit count (the frame's
// tile entries, which may exceed 2^30).
template <typename W>
struct Lb;
template <>
struct Lb<uint32_t> {
  static constexpr uint32_t kAgg = 1u << 30, kPre = 2u << 30, kMask = (1u << 30) - 1u;
  static __device__ __forceinline__ uint32_t load(const uint32_t* p) { return ld_relaxed_u32(p); }
  static __device__ __forceinline__ void store(uint32_t* p, uint32_t w) { st_relaxed_u32(p, w); }
  static __device__ __forceinline__ uint32_t flag(uint32_t w) { return w & ~kMask; }
  static __device__ __forceinline__ uint32_t value(uint32_t w) { return w & kMask; }
  static __device__ __forceinline__ uint32_t make(uint32_t f, uint32_t v) { return f | (v & kMask); }
};
template <>
struct Lb<unsigned long long> {
  using W = unsigned long long;
  static constexpr W kAgg = 1ull << 32, kPre = 2ull << 32, kMask = 0xFFFFFFFFull;
  static __device__ __forceinline__ W load(const W* p) { return ld_relaxed_u64(p); }
  static __device__ __forceinline__ void store(W* p, W w) { st_relaxed_u64(p, w); }
  static __device__ __forceinline__ W flag(W w) { return w & ~kMask; }
  static __device__ __forceinline__ uint32_t value(W w) { return (uint32_t)w; }
  static __device__ __forceinline__ W make(W f, uint32_t v) { return f | (W)v; }
};

// Ranking modes of a pass: __match_any_sync (cheap when a warp's keys share
// few digits), one ballot per digit bit (a fixed cost), or shared-memory
// peer masks (each lane sets its bit in its digit's word; one warp barrier;
// cheapest for many distinct 8-bit digits).
constexpr uint32_t kRankMatch = 0, kRankBallot = 1, kRankSmem = 2;

struct PassArgs {
  const uint32_t* keys_in;
  const uint32_t* v0_in;
  const uint32_t* v1_in;
  uint32_t* keys_out;
  uint32_t* v0_out;
  uint32_t* v1_out;
  const uint32_t* n_ptr;
  uint32_t capacity;
  uint32_t shift;
  uint32_t dmask;          // digit mask of this pass (narrower on a final partial pass)
  const uint32_t* dbase;   // this pass's digit counts (each block scans them)
  void* status;            // this pass's [tiles][radix] look-back words (32- or 64-bit)
  void* clear_next;        // [tiles][clear_stride] words to zero for the next pass, or null
  uint32_t clear_stride;   // words per tile of clear_next (>= radix)
  uint32_t grid_tiles;     // tiles covered by the grid (all of clear_next)
  uint32_t* tile_ctr;
  uint32_t* status_word;
  uint32_t rank;           // how a warp finds the lanes sharing a digit: kRank*
  // last pass of a sort with ranges: per screen tile (key >> tile_shift,
  // below num_tiles), atomicMax of the complemented first entry and of the
  // end of every run of one tile in this block's output
  uint32_t* ranges;
  uint32_t tile_shift;
  uint32_t num_tiles;
};

// Exclusive prefix of digit d over the tiles before `tile`: walks back from
// tile - 1, adding published tile counts until a tile with its inclusive
// prefix. A word with neither flag is polled again (its tile is held by a
// resident block); after `limit` polls the wait gives up, sets
// kStatusLookbackTimeout and returns what it has. The words of four
// predecessors are read at once (independent loads), so a walk over tiles
// that have published only their counts costs one load latency per four
// tiles instead of one per tile.
template <typename W>
__device__ __forceinline__ uint32_t digit_lookback(const W* status, uint32_t tile, uint32_t R,
                                                   uint32_t d, uint32_t* status_word,
                                                   uint32_t limit) {
  constexpr int kAhead = 4;
  uint32_t excl = 0;
  long long pred = (long long)tile - 1;
  uint32_t spins = 0;
  while (pred >= 0) {
    W w[kAhead];
#pragma unroll
    for (int k = 0; k < kAhead; ++k)
      w[k] = pred - k >= 0 ? Lb<W>::load(status + (size_t)(pred - k) * R + d) : W(0);
    int used = 0;
    bool done = false;
#pragma unroll
    for (int k = 0; k < kAhead; ++k) {
      if (done || used < k || pred - k < 0) continue;
      if (Lb<W>::flag(w[k]) == 0) continue;  // not published: wait on it below
      excl += Lb<W>::value(w[k]);
      used = k + 1;
      if (Lb<W>::flag(w[k]) == Lb<W>::kPre) done = true;
    }
    if (done) break;
    pred -= used;
    if (used == 0) {  // the nearest unread predecessor has published nothing yet
      if (++spins > limit) {
        atomicOr(status_word, kStatusLookbackTimeout);
        break;
      }
      __nanosleep(32);
    }
  }
  return excl;
}

template <int RB, bool PAY2, typename W>
__global__ void __launch_bounds__(kSortThreads, PAY2 ? 3 : 4) k_onesweep(const PassArgs a) {
  constexpr uint32_t R = 1u << RB;
  W* const lb = static_cast<W*>(a.status);
  static_assert(R <= (uint32_t)kSortThreads, "one thread per digit");
  extern __shared__ __align__(16) uint32_t smem[];
  uint32_t* s_keys = smem;                       // [kSortTileP]
  uint32_t* s_v0 = s_keys + kSortTileP;          // [kSortTileP]
  uint32_t* s_v1 = s_v0 + kSortTileP;            // [kSortTileP] (PAY2)
  uint32_t* s_whist = s_v0 + (PAY2 ? 2 : 1) * kSortTileP;  // [warps][R]
  uint32_t* s_tstart = s_whist + kSortWarps * R;  // [R]
  uint32_t* s_goff = s_tstart + R;               // [R]
  uint32_t* s_misc = s_goff + R;                 // [40]: tile, warp sums
  uint32_t* s_wor = s_misc + 48;                 // [warps][3][R] peer masks (kRankSmem)

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  uint32_t n = *a.n_ptr;
  if (n > a.capacity) n = a.capacity;
  const uint32_t num_tiles = (n + kSortTile - 1) / kSortTile;
  if (tid == 0) s_misc[0] = atomicAdd(a.tile_ctr, 1u);
  for (uint32_t k = tid; k < kSortWarps * R; k += kSortThreads) s_whist[k] = 0u;
  if (a.rank == kRankSmem)
    for (uint32_t k = tid; k < kSortWarps * 3 * R; k += kSortThreads) s_wor[k] = 0u;
  __syncthreads();
  const uint32_t tile = s_misc[0];
  // Clear this tile's words of the other look-back buffer for the next pass
  // (the pass that used it has completed: passes are stream-ordered launches).
  // Every block of the grid clears its stride, so the whole buffer is clean
  // whatever radix the previous sort on it used.
  if (a.clear_next && tile < a.grid_tiles)
    for (uint32_t k = tid; k < a.clear_stride; k += kSortThreads)
      static_cast<W*>(a.clear_next)[(size_t)tile * a.clear_stride + k] = W(0);
  if (tile >= num_tiles) return;
  // this pass's exclusive digit base (thread d < R holds digit d's) from the
  // digit counts
  uint32_t dig_base;
  {
    uint32_t tot0;
    dig_base = block_exclusive_sum((uint32_t)tid < R ? a.dbase[tid] : 0u, s_misc + 8, &tot0);
  }

  // Load (warp-striped: a warp's item j is 32 consecutive keys). Full tiles,
  // all but the last, need no bounds checks.
  const size_t tile_base = (size_t)tile * kSortTile;
  const bool full = tile_base + kSortTile <= (size_t)n;
  const size_t first = tile_base + (size_t)warp * (32 * kSortItems) + lane;
  uint32_t k[kSortItems], v0[kSortItems], v1[kSortItems];
  uint32_t rk[kSortItems / 2];  // two 16-bit in-warp ranks per word (ranks < 512)
  if (full) {
#pragma unroll
    for (int j = 0; j < kSortItems; ++j) {
      k[j] = __ldcs(a.keys_in + first + 32 * j);
      v0[j] = __ldcs(a.v0_in + first + 32 * j);
      if (PAY2) v1[j] = __ldcs(a.v1_in + first + 32 * j);
    }
  } else {
#pragma unroll
    for (int j = 0; j < kSortItems; ++j) {
      const bool valid = first + 32 * j < n;
      k[j] = valid ? __ldcs(a.keys_in + first + 32 * j) : 0xFFFFFFFFu;
      v0[j] = valid ? __ldcs(a.v0_in + first + 32 * j) : 0u;
      if (PAY2) v1[j] = valid ? __ldcs(a.v1_in + first + 32 * j) : 0u;
    }
  }

  // Warp-level stable ranking by digit: the lanes holding the same digit
  // (match) take consecutive ranks after the warp's running count, which the
  // highest of them advances.
  uint32_t* wh = s_whist + warp * R;
  const uint32_t lt = lanemask_lt();
  uint32_t prev_d = 0;
  bool prev_lead = false;
#pragma unroll
  for (int j = 0; j < kSortItems; ++j) {
    const uint32_t d = (k[j] >> a.shift) & a.dmask;
    uint32_t peers;
    if (a.rank == kRankSmem) {
      // a step's words are cleared by their leaders one step later (after
      // that step's barrier, so every lane has read them); three buffers
      // keep a word from being reused before it is cleared
      uint32_t* wo = s_wor + (warp * 3 + (j % 3)) * R;
      atomicOr(&wo[d], 1u << lane);
      __syncwarp();
      peers = wo[d];
      if (j >= 1 && prev_lead) s_wor[(warp * 3 + ((j + 2) % 3)) * R + prev_d] = 0u;
    } else if (a.rank == kRankBallot) {
      peers = 0xffffffffu;
#pragma unroll
      for (int b = 0; b < RB; ++b) {
        const uint32_t m = __ballot_sync(0xffffffffu, (d >> b) & 1u);
        peers &= ((d >> b) & 1u) ? m : ~m;
      }
    } else {
      peers = __match_any_sync(0xffffffffu, d);
    }
    const int leader = 31 - __clz(peers);
    prev_lead = lane == leader;
    prev_d = d;
    uint32_t old = 0;
    if (lane == leader) old = atomicAdd(&wh[d], (uint32_t)__popc(peers));
    old = __shfl_sync(0xffffffffu, old, leader);
    const uint32_t r = old + __popc(peers & lt);
    if (j & 1)
      rk[j >> 1] |= r << 16;
    else
      rk[j >> 1] = r;
  }
  __syncthreads();
  // Per digit: exclusive prefix over warps, tile count (valid keys only).
  const uint32_t tile_valid = full ? kSortTile : (uint32_t)((size_t)n - tile_base);
  uint32_t my_count = 0;
  if ((uint32_t)tid < R) {
    uint32_t run = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w) {
      const uint32_t c = s_whist[w * R + tid];
      s_whist[w * R + tid] = run;
      run += c;
    }
    my_count = run;
  }
  uint32_t tot2;
  const uint32_t tstart = block_exclusive_sum(my_count, s_misc + 8, &tot2);
  // Publish the tile's counts, then reorder by digit through shared memory
  // (tile-local offsets only) before walking back for the global prefix, so
  // the walk starts later (its predecessors have had more time to publish
  // their prefixes) and the reorder does not wait for it.
  uint32_t agg = 0;
  if ((uint32_t)tid < R) {
    s_tstart[tid] = tstart;
    // Padding keys (past n) carry the largest digit and sit at the end of it.
    agg = my_count;
    if ((uint32_t)tid == a.dmask) agg -= (kSortTile - tile_valid);
    Lb<W>::store(lb + (size_t)tile * R + tid,
                 Lb<W>::make(tile == 0 ? Lb<W>::kPre : Lb<W>::kAgg, agg));
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < kSortItems; ++j) {
    const uint32_t d = (k[j] >> a.shift) & a.dmask;
    const uint32_t pos =
        padded(s_tstart[d] + wh[d] + ((rk[j >> 1] >> ((j & 1) * 16)) & 0xFFFFu));
    s_keys[pos] = k[j];
    s_v0[pos] = v0[j];
    if (PAY2) s_v1[pos] = v1[j];
  }
  if ((uint32_t)tid < R) {
    uint32_t excl = 0;
    if (tile != 0) {
      excl = digit_lookback<W>(lb, tile, R, (uint32_t)tid, a.status_word, kSpinLimit);
      Lb<W>::store(lb + (size_t)tile * R + tid, Lb<W>::make(Lb<W>::kPre, excl + agg));
    }
    s_goff[tid] = dig_base + excl - tstart;
  }
  __syncthreads();
  // Scatter: each digit's run is contiguous in the output.
  bool bad = false;
#pragma unroll
  for (int j = 0; j < kSortItems; ++j) {
    const uint32_t i = tid + kSortThreads * j;
    if (!full && i >= tile_valid) break;
    const uint32_t key = s_keys[padded(i)];
    const uint32_t g = s_goff[(key >> a.shift) & a.dmask] + i;
    if (g >= n) {  // inconsistent histogram: report instead of writing out of bounds
      bad = true;
      continue;
    }
    if (a.ranges) {
      // runs of one tile are contiguous here (one digit run, in input order,
      // which the earlier passes sorted by the lower tile bits) and in the
      // output (the run's positions are consecutive)
      const uint32_t t = a.tile_shift >= 32u ? 0u : key >> a.tile_shift;
      bool first = i == 0, last = i + 1 == tile_valid;
      if (!first) {
        const uint32_t pk = s_keys[padded(i - 1)];
        first = (a.tile_shift >= 32u ? 0u : pk >> a.tile_shift) != t;
      }
      if (!last) {
        const uint32_t nk = s_keys[padded(i + 1)];
        last = (a.tile_shift >= 32u ? 0u : nk >> a.tile_shift) != t;
      }
      if (t < a.num_tiles) {
        if (first) atomicMax(&a.ranges[2 * (size_t)t], ~g);
        if (last) atomicMax(&a.ranges[2 * (size_t)t + 1], g + 1u);
      }
    }
    a.keys_out[g] = key;
    a.v0_out[g] = s_v0[padded(i)];
    if (PAY2) a.v1_out[g] = s_v1[padded(i)];
  }
  if (bad) atomicOr(a.status_word, kStatusCapacity);
}

template <int RB, bool PAY2>
size_t onesweep_smem(uint32_t rank) {
  constexpr uint32_t R = 1u << RB;
  return sizeof(uint32_t) * ((PAY2 ? 3 : 2) * kSortTileP + kSortWarps * R + 3 * R + 48 +
                             (rank == kRankSmem ? kSortWarps * 3 * R : 0u));
}

template <int RB, bool PAY2, typename W>
cudaError_t launch_pass_w(const PassArgs& p, uint32_t grid, cudaStream_t s) {
  const size_t smem = onesweep_smem<RB, PAY2>(p.rank);
  // per device: set on every launch (a host-side attribute write)
  const cudaError_t e = cudaFuncSetAttribute(k_onesweep<RB, PAY2, W>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k_onesweep<RB, PAY2, W><<<grid, kSortThreads, smem, s>>>(p);
  return cudaGetLastError();
}

template <int RB, bool PAY2>
cudaError_t launch_pass(const PassArgs& p, uint32_t grid, bool wide, cudaStream_t s) {
  return wide ? launch_pass_w<RB, PAY2, unsigned long long>(p, grid, s)
              : launch_pass_w<RB, PAY2, uint32_t>(p, grid, s);
}

// Digit histograms of every pass in one read of the keys.
__global__ void k_histogram(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ n_ptr,
                            uint32_t capacity, uint32_t first_bit, uint32_t num_bits,
                            uint32_t radix_bits, uint32_t* __restrict__ hist) {
  __shared__ uint32_t s_hist[8 * 256];
  const uint32_t R = 1u << radix_bits;
  const uint32_t passes = (num_bits + radix_bits - 1) / radix_bits;
  for (uint32_t k = threadIdx.x; k < passes * R; k += blockDim.x) s_hist[k] = 0u;
  __syncthreads();
  uint32_t n = *n_ptr;
  if (n > capacity) n = capacity;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t key = keys[i];
    for (uint32_t p = 0; p < passes; ++p) {
      const uint32_t rem = num_bits - p * radix_bits;
      const uint32_t bits = rem < radix_bits ? rem : radix_bits;
      const uint32_t d = (key >> (first_bit + p * radix_bits)) & ((1u << bits) - 1u);
      atomicAdd(&s_hist[p * R + d], 1u);
    }
  }
  __syncthreads();
  for (uint32_t k = threadIdx.x; k < passes * R; k += blockDim.x)
    if (s_hist[k]) atomicAdd(&hist[k], s_hist[k]);
}

// Wait drill: one thread per digit walks back from tile 1 to a tile 0 whose
// words nothing publishes (status holds 2 x R zeroed words), so every walk
// polls until its limit and sets the timeout bit.
__global__ void k_drill_digit_lookback(const uint32_t* status, uint32_t R, uint32_t* status_word,
                                       uint32_t limit) {
  if (threadIdx.x < R) digit_lookback<uint32_t>(status, 1u, R, threadIdx.x, status_word, limit);
}

}  // namespace

cudaError_t launch_drill_digit_lookback(const uint32_t* status, uint32_t radix,
                                        uint32_t* status_word, uint32_t limit, cudaStream_t s) {
  if (radix == 0 || radix > 256) return cudaErrorInvalidValue;
  k_drill_digit_lookback<<<1, 256, 0, s>>>(status, radix, status_word, limit);
  return cudaGetLastError();
}

uint32_t sort_tiles(uint32_t capacity) { return (capacity + kSortTile - 1) / kSortTile; }

uint32_t sort_passes(uint32_t num_bits, uint32_t radix_bits) {
  return (num_bits + radix_bits - 1) / radix_bits;
}

cudaError_t launch_histogram(const uint32_t* keys, const uint32_t* n_ptr, uint32_t capacity,
                             uint32_t first_bit, uint32_t num_bits, uint32_t radix_bits,
                             uint32_t* hist, cudaStream_t s) {
  k_histogram<<<148 * 2, 512, 0, s>>>(keys, n_ptr, capacity, first_bit, num_bits, radix_bits,
                                      hist);
  return cudaGetLastError();
}

cudaError_t run_radix_sort(const SortArgs& a, int* out_src, cudaStream_t s) {
  const uint32_t rb = a.radix_bits < 4 ? 4u : (a.radix_bits > 8 ? 8u : a.radix_bits);
  const uint32_t R = 1u << rb;
  const uint32_t passes = sort_passes(a.num_bits, rb);
  const uint32_t tiles = sort_tiles(a.capacity);
  int src = a.src;
  const bool pay2 = a.vals2[0] != nullptr;
  const bool wide = a.wide_lookback;
  if (!wide && a.capacity > (1u << 30)) return cudaErrorInvalidValue;  // 30-bit counts
  for (uint32_t p = 0; p < passes; ++p) {
    PassArgs pa;
    pa.keys_in = a.keys[src];
    pa.v0_in = a.vals[src];
    pa.v1_in = pay2 ? a.vals2[src] : nullptr;
    pa.keys_out = a.keys[1 - src];
    pa.v0_out = a.vals[1 - src];
    pa.v1_out = pay2 ? a.vals2[1 - src] : nullptr;
    pa.n_ptr = a.n_ptr;
    pa.capacity = a.capacity;
    pa.shift = a.first_bit + p * rb;
    const uint32_t rem = a.num_bits - p * rb;
    pa.dmask = (1u << (rem < rb ? rem : rb)) - 1u;
    pa.dbase = a.hist + (size_t)p * R;
    if (a.status2[0]) {
      const int par = *a.parity;
      pa.status = a.status2[par];
      pa.clear_next = a.status2[par ^ 1];
      pa.clear_stride = a.lb_stride ? a.lb_stride : R;
      *a.parity = par ^ 1;
    } else {
      pa.status = static_cast<char*>(a.status) + (size_t)p * tiles * R * (wide ? 8 : 4);
      pa.clear_next = nullptr;
      pa.clear_stride = 0;
    }
    if (pa.clear_stride < R && pa.clear_next) return cudaErrorInvalidValue;
    pa.grid_tiles = tiles;
    pa.tile_ctr = a.tile_ctr + p;
    pa.status_word = a.status_word;
    pa.rank = ((a.smem_mask >> p) & 1u) ? kRankSmem : (((a.ballot_mask >> p) & 1u) ? kRankBallot : kRankMatch);
    pa.ranges = p + 1 == passes ? a.ranges : nullptr;
    pa.tile_shift = a.tile_shift;
    pa.num_tiles = a.num_tiles;
    cudaError_t e;
    switch (rb) {
      case 4: e = pay2 ? launch_pass<4, true>(pa, tiles, wide, s) : launch_pass<4, false>(pa, tiles, wide, s); break;
      case 5: e = pay2 ? launch_pass<5, true>(pa, tiles, wide, s) : launch_pass<5, false>(pa, tiles, wide, s); break;
      case 6: e = pay2 ? launch_pass<6, true>(pa, tiles, wide, s) : launch_pass<6, false>(pa, tiles, wide, s); break;
      case 7: e = pay2 ? launch_pass<7, true>(pa, tiles, wide, s) : launch_pass<7, false>(pa, tiles, wide, s); break;
      default: e = pay2 ? launch_pass<8, true>(pa, tiles, wide, s) : launch_pass<8, false>(pa, tiles, wide, s); break;
    }
    if (e != cudaSuccess) return e;
    src = 1 - src;
  }
  *out_src = src;
  return cudaSuccess;
}

}  // namespace cgs
