// Shared device-side definitions for the sm_100a splat pipeline kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "detmath.h"

namespace cgs {

constexpr uint32_t kInvalid = 0xFFFFFFFFu;

// Status bits written to FrameCounters::status by kernels that give up a
// bounded wait or detect a capacity overflow; the host maps them to
// CGS_E_TIMEOUT / CGS_E_CAPACITY after the frame.
constexpr uint32_t kStatusLookbackTimeout = 1u;
constexpr uint32_t kStatusCapacity = 2u;
constexpr uint32_t kStatusBarrierTimeout = 4u;
// A tensor-core wait gave up twice: MMAs may still be writing tensor memory
// that the kernel released on exit, so the device state is undefined and the
// context must be rebuilt.
constexpr uint32_t kStatusPoisoned = 8u;

// Upper bound on polls of a lookback or mbarrier wait before a kernel gives
// up, sets a status bit and carries on with whatever it has (the frame's
// result is then reported as an error instead of hanging the device).
constexpr uint32_t kSpinLimit = 1u << 22;

// Per-frame counters, cleared at the start of every frame.
struct FrameCounters {
  uint32_t surviving;    // Stage 2 survivors
  uint32_t active;       // splat slots of the frame (rest + split children), from Stage 2
  uint32_t entries;      // Stage 3 tile entries (binning total)
  uint32_t status;       // kStatus* bits
  uint32_t fetched;      // splat records the compositor gathered
  uint32_t tile_ctr[16]; // dynamic tile counters for chained-scan kernels
  uint32_t pad;
  unsigned long long stage_ctr;  // binning: staged entries so far (64 bits: never wraps)
};
// Largest tile-entry capacity of a frame (32-bit entry indices; a multiple
// of the radix sort's 4096-entry tiles; the entry sort's look-back words are
// 64 bits wide, so counts are not limited to 2^30).
constexpr uint32_t kMaxEntryCap = 0xFFFF0000u;

// Splat record written by Stage 2 and read by Stages 3 and 4: 48 bytes, three
// 16-byte words so one bulk copy moves a whole record.
struct __align__(16) SplatRec {
  float4 geo;   // mu_x, mu_y, conic a, conic b
  float4 cc;    // conic c, alpha_2d, t_z, extents (u32 bits: ext_x | ext_y << 16; 0 = culled)
  float4 rgb;   // r, g, b, unused
};
static_assert(sizeof(SplatRec) == 48, "SplatRec must be 48 bytes");

__device__ __forceinline__ float clampf(float x, float lo, float hi) {
  return fminf(fmaxf(x, lo), hi);
}

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Look-back status words carry their flag and value in one naturally aligned
// word, so a single-copy-atomic relaxed access at GPU scope is enough: no data
// other than the word itself is published through it, and no fence is needed.
__device__ __forceinline__ void st_relaxed_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_u32(uint32_t* p, uint32_t v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ uint32_t ld_relaxed_u32(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Block-wide exclusive sum over one u32 per thread (blockDim.x a multiple of
// 32, at most 1024). `warp_sums` is shared scratch of 32 words. Returns the
// exclusive prefix; *total receives the block sum.
__device__ __forceinline__ uint32_t block_exclusive_sum(uint32_t v, uint32_t* warp_sums,
                                                        uint32_t* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nwarps = blockDim.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t s = lane < nwarps ? warp_sums[lane] : 0u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    warp_sums[lane] = s;  // inclusive
  }
  __syncthreads();
  uint32_t warp_base = warp > 0 ? warp_sums[warp - 1] : 0u;
  *total = warp_sums[nwarps - 1];
  uint32_t excl = warp_base + x - v;
  __syncthreads();
  return excl;
}

// a + b, saturating at 2^32 - 1
__device__ __forceinline__ uint32_t sat_add_u32(uint32_t a, uint32_t b) {
  const uint32_t c = a + b;
  return c < a ? 0xFFFFFFFFu : c;
}

// Chained-scan ("decoupled look-back", Merrill & Garland 2016) of one value
// per tile. status[t] = flag << 32 | value with flag 1 = tile aggregate
// published, 2 = inclusive prefix published; the array must be zeroed before
// the launch. Tiles must be acquired in increasing order by running blocks
// (a dynamic tile counter), so every tile a block waits on is held by a block
// that is already resident and publishes its aggregate without waiting.
// Called by all lanes of ONE warp. chained_publish publishes the tile's
// aggregate (tile 0: its inclusive prefix); chained_resolve then walks back
// for its exclusive prefix, publishes the inclusive one and returns the
// exclusive one (with SAT, sums saturate at 2^32 - 1 instead of wrapping). A
// wait that exceeds `limit` polls sets kStatusLookbackTimeout and returns 0.
__device__ __forceinline__ void chained_publish(unsigned long long* status, uint32_t tile,
                                                uint32_t aggregate) {
  if ((threadIdx.x & 31) == 0)
    st_relaxed_u64(&status[tile], ((tile == 0 ? 2ull : 1ull) << 32) | aggregate);
}

template <bool SAT = false>
__device__ __forceinline__ uint32_t chained_resolve(unsigned long long* status, uint32_t tile,
                                                    uint32_t aggregate, uint32_t* status_word,
                                                    uint32_t limit = kSpinLimit) {
  const int lane = threadIdx.x & 31;
  if (tile == 0) return 0u;
  uint32_t exclusive = 0;
  long long pred = (long long)tile - 1;
  uint32_t spins = 0;
  bool timed_out = false;
  while (true) {
    long long mine = pred - lane;
    unsigned long long st = mine >= 0 ? ld_relaxed_u64(&status[mine]) : (2ull << 32);
    while (__any_sync(0xffffffffu, (st >> 32) == 0ull)) {
      if (++spins > limit) {
        timed_out = true;
        break;
      }
      if ((st >> 32) == 0ull) {
        __nanosleep(64);
        st = ld_relaxed_u64(&status[mine]);
      }
    }
    if (timed_out) break;
    uint32_t pmask = __ballot_sync(0xffffffffu, (st >> 32) == 2ull);
    int first_p = pmask ? (__ffs(pmask) - 1) : 32;
    uint32_t v = lane <= first_p ? (uint32_t)st : 0u;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const uint32_t w = __shfl_xor_sync(0xffffffffu, v, o);
      v = SAT ? sat_add_u32(v, w) : v + w;
    }
    exclusive = SAT ? sat_add_u32(exclusive, v) : exclusive + v;
    if (pmask) break;
    pred -= 32;
  }
  if (timed_out) {
    if (lane == 0) atomicOr(status_word, kStatusLookbackTimeout);
    exclusive = 0;
  }
  if (lane == 0)
    st_relaxed_u64(&status[tile], (2ull << 32) | (SAT ? sat_add_u32(exclusive, aggregate)
                                                      : exclusive + aggregate));
  return exclusive;
}

template <bool SAT = false>
__device__ __forceinline__ uint32_t chained_scan_warp(unsigned long long* status, uint32_t tile,
                                                      uint32_t aggregate, uint32_t* status_word,
                                                      uint32_t limit = kSpinLimit) {
  chained_publish(status, tile, aggregate);
  return chained_resolve<SAT>(status, tile, aggregate, status_word, limit);
}

}  // namespace cgs
