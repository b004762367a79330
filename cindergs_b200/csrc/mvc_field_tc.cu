// Fused inference of the learned MVC field on the 5th-generation tensor cores
// (tcgen05): per Gaussian, the network and its three forward-mode tangents,
// then either the position and deformation gradient on the current cage
// (x' = Pc^T h + pc + A3 x, F = Pc^T dh + A3; k_mvc_jacobian's layout) or the
// last hidden layer and its tangents as the cached code (bf16 [4][128]).
//
// One CTA per SM, three warpgroups; each warpgroup owns a tile of 32 items
// = 128 columns n = 8 (p / 2) + 2 s + p % 2 (item p, stream s = value, d/dx,
// d/dy, d/dz): the 16-byte chunk of columns 8 c .. 8 c + 7 holds items 2 c
// and 2 c + 1, and a stream of the two items sits in two adjacent columns,
// so the epilogue works on item pairs with packed f32x2 instructions.
// A hidden layer is one M = 128, N = 128 product per tile with the weights
// as A (K-major, as stored) and the activations as B in MN-major order
// (row k of the operand holds input k of every column), so the accumulator
// has TMEM lane = hidden unit and column = (item, stream): the thread that
// owns lane j reads the pre-activation and the three tangents of unit j of
// an item side by side, evaluates the SiLU and its slope once and scales
// its own tangents, and writes row j of the next layer's operand -- no
// exchange between threads and no barrier inside the epilogue. One elected
// thread per warpgroup issues the K = 16 steps and commits them to the
// warpgroup's mbarrier; the three warpgroups' products queue on the tensor
// pipe while the other warpgroups run their epilogues. The output
// projection takes the same shared-memory tile as an MN-major A operand
// (M = 128 columns of the tile) against Pc split into three bf16 terms
// (N = 16: columns 0-2, 3-5, 6-8), so that the products are exact and only
// the fp32 accumulation rounds; lane n of its accumulator is column n.
//
// Shared-memory operands use the 128-byte-swizzle canonical layouts:
// K-major (weights, Pc): rows of 64 bf16 (128 B), 8-row atoms of 1024 B,
// 16-byte chunk c of row r stored at chunk c ^ (r % 8); MN-major
// (activations): 128-byte rows of 64 consecutive columns, one row per input
// k, 8-row atoms of 1024 B (stride byte offset), the second 64 columns
// 16 KB further on (leading byte offset), chunk c of row k at c ^ (k % 8).
//
// Every mbarrier wait is bounded; a wait that gives up sets the status word
// and the warpgroup stops issuing work (TMEM is released at the end).
#include <cuda_bf16.h>

#include <algorithm>

#include "kernels.h"

namespace cgs {
namespace {

constexpr int kHid = kFieldHid, kIn = kFieldIn;
constexpr int kTcWG = 3;                 // warpgroups (tiles in flight) per CTA
constexpr uint32_t kTcCols = 128;        // TMEM columns per warpgroup
constexpr uint32_t kTcAlloc = 512;       // power of two >= kTcWG * kTcCols
constexpr uint32_t kTcWaitLimit = 1u << 20;
constexpr uint32_t kItems = 32;          // items per tile
constexpr uint32_t kMnBlock = 16384;     // bytes between the two 64-column halves of a tile

// shared memory map (bytes from the 1024-aligned base)
constexpr uint32_t kOffW1 = 0;                        // [128 x 64]   16 KB
constexpr uint32_t kOffW2 = kOffW1 + 128 * 64 * 2;    // [128 x 128]  32 KB each
constexpr uint32_t kOffW3 = kOffW2 + 128 * 128 * 2;
constexpr uint32_t kOffW4 = kOffW3 + 128 * 128 * 2;
constexpr uint32_t kOffP = kOffW4 + 128 * 128 * 2;    // [16 x 128]   4 KB
constexpr uint32_t kOffB = kOffP + 16 * 128 * 2;      // activation tile [128 k][128 n] per warpgroup
constexpr uint32_t kBTile = 128 * 128 * 2;
constexpr uint32_t kOffBias = kOffB + kTcWG * kBTile;  // 4 x 128 f32
constexpr uint32_t kOffMisc = kOffBias + 4 * 128 * 4;  // pc, A3, mbarriers, tmem
constexpr uint32_t kTcSmem = kOffMisc + 256 + 1024;    // + alignment slack
static_assert(kTcSmem <= 232448, "shared memory per CTA");
static_assert(kTcWG * kTcCols <= kTcAlloc, "TMEM columns");
static_assert(kOffB % 1024 == 0 && kBTile % 1024 == 0, "swizzle atoms are 1024-byte aligned");

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Byte offset of element (r, k) of a K-major swizzled operand with R rows.
__device__ __forceinline__ uint32_t sw_off(uint32_t R, uint32_t r, uint32_t k) {
  const uint32_t kb = k >> 6, kk = k & 63;
  const uint32_t chunk = (kk >> 3) ^ (r & 7);
  return kb * (R * 128) + (r >> 3) * 1024 + (r & 7) * 128 + chunk * 16 + (kk & 7) * 2;
}

// Byte offset of the 16-byte chunk holding columns 8 c .. 8 c + 7 (c < 16)
// of row k of an MN-major activation tile.
__device__ __forceinline__ uint32_t mn_chunk(uint32_t k, uint32_t c) {
  return (c >> 3) * kMnBlock + (k >> 3) * 1024 + (k & 7) * 128 + (((c & 7) ^ (k & 7)) << 4);
}

// Shared memory matrix descriptor, 128-byte swizzle: K-major operands
// (stride byte offset 1024 = next 8-row atom; the leading offset is unused)
// and MN-major operands (stride byte offset 1024 = next 8 rows of K, leading
// byte offset = next 64 columns of M or N).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr, uint32_t lbo = 16) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;  // leading byte offset
  d |= (uint64_t)(1024 >> 4) << 32;             // stride byte offset
  d |= (uint64_t)1 << 46;                       // descriptor version
  d |= (uint64_t)2 << 61;                       // 128-byte swizzle
  return d;
}

// Instruction descriptor: kind::f16, bf16 A and B, f32 accumulate; a_mn / b_mn
// select MN-major A / B.
__host__ __device__ constexpr uint32_t idesc_bf16(uint32_t M, uint32_t N, uint32_t a_mn,
                                                  uint32_t b_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (a_mn << 15) | (b_mn << 16) | ((N >> 3) << 17) |
         ((M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16_tc(uint32_t d_tmem, uint64_t a, uint64_t b,
                                            uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc));
}
__device__ __forceinline__ void mma_commit(uint32_t mbar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(mbar)
      : "memory");
}
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
  for (uint32_t i = 0; i < kTcWaitLimit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        "selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}
__device__ __forceinline__ void wg_sync(int wg) {
  asm volatile("bar.sync %0, 128;\n" ::"r"(1 + wg) : "memory");
}
__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
}

#define CGS_R8(i) "=r"(v[i]), "=r"(v[i + 1]), "=r"(v[i + 2]), "=r"(v[i + 3]), "=r"(v[i + 4]), \
                  "=r"(v[i + 5]), "=r"(v[i + 6]), "=r"(v[i + 7])
// 32 consecutive TMEM columns of this thread's lane into v[O .. O + 31]
// (no wait: the caller waits once for several loads).
template <int O, int NV>
__device__ __forceinline__ void tmem_ld32_nowait(uint32_t taddr, uint32_t (&v)[NV]) {
  static_assert(O + 32 <= NV, "tmem_ld32 range");
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, "
      "%28, %29, %30, %31}, [%32];\n"
      : CGS_R8(O), CGS_R8(O + 8), CGS_R8(O + 16), CGS_R8(O + 24)
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15}, [%16];\n"
      : CGS_R8(0), CGS_R8(8)
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}
#undef CGS_R8

__device__ __forceinline__ uint32_t pack2(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&v);
}

// Two f32 lanes in one 64-bit register pair, for the packed f32x2 arithmetic
// of sm_100 (one instruction for two IEEE-rounded products or sums).
__device__ __forceinline__ uint64_t f2_make(uint32_t lo, uint32_t hi) {
  uint64_t r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "r"(lo), "r"(hi));
  return r;
}
__device__ __forceinline__ uint64_t f2_splat(float x) {
  return f2_make(__float_as_uint(x), __float_as_uint(x));
}
__device__ __forceinline__ void f2_split(uint64_t a, float& lo, float& hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(a));
}
__device__ __forceinline__ uint64_t f2_add(uint64_t a, uint64_t b) {
  uint64_t d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ uint64_t f2_mul(uint64_t a, uint64_t b) {
  uint64_t d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ uint64_t f2_fma(uint64_t a, uint64_t b, uint64_t c) {
  uint64_t d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}
// bf16 pair (lo in the low half) of the two lanes, each rounded to nearest
__device__ __forceinline__ uint32_t f2_bf16(uint64_t a) {
  float lo, hi;
  f2_split(a, lo, hi);
  return pack2(lo, hi);
}
// 2^x and 1/x on the special-function unit, per lane
__device__ __forceinline__ uint64_t f2_ex2(uint64_t a) {
  float lo, hi;
  f2_split(a, lo, hi);
  asm("ex2.approx.ftz.f32 %0, %0;" : "+f"(lo));
  asm("ex2.approx.ftz.f32 %0, %0;" : "+f"(hi));
  return f2_make(__float_as_uint(lo), __float_as_uint(hi));
}
__device__ __forceinline__ uint64_t f2_rcp(uint64_t a) {
  float lo, hi;
  f2_split(a, lo, hi);
  asm("rcp.approx.ftz.f32 %0, %0;" : "+f"(lo));
  asm("rcp.approx.ftz.f32 %0, %0;" : "+f"(hi));
  return f2_make(__float_as_uint(lo), __float_as_uint(hi));
}

__device__ __forceinline__ float3 item_position(const FieldInfer& fi, uint32_t k_item) {
  const uint32_t gi = fi.gauss ? fi.gauss[fi.first + k_item] : fi.first + k_item;
  if (fi.points4) {
    const float4 x4 = fi.points4[gi];
    return make_float3(x4.x, x4.y, x4.z);
  }
  return make_float3(fi.points3[3 * (size_t)gi], fi.points3[3 * (size_t)gi + 1],
                     fi.points3[3 * (size_t)gi + 2]);
}

template <bool CODES>
__global__ void __launch_bounds__(kTcWG * 128, 1) k_field_infer_tc(FieldInfer fi) {
  extern __shared__ unsigned char tc_raw[];
  unsigned char* sm = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(tc_raw) + 1023) & ~(uintptr_t)1023);
  float* s_bias = reinterpret_cast<float*>(sm + kOffBias);
  float* s_misc = reinterpret_cast<float*>(sm + kOffMisc);  // pc[3], A3[9]
  uint64_t* s_mbar = reinterpret_cast<uint64_t*>(sm + kOffMisc + 64);   // [kTcWG]
  uint32_t* s_tmem = reinterpret_cast<uint32_t*>(sm + kOffMisc + 128);
  volatile uint32_t* s_ok = reinterpret_cast<uint32_t*>(sm + kOffMisc + 144);  // [kTcWG]
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int wg = warp >> 2, q4 = warp & 3;  // warpgroup, warp within it (TMEM lane quarter)
  const uint32_t j = 32u * (uint32_t)q4 + (uint32_t)lane;  // TMEM lane of this thread

  // ---- weights, biases and the projection into shared memory
  auto put_w = [&](uint32_t off, const __nv_bfloat16* W, uint32_t R, uint32_t K) {
    for (uint32_t c = tid; c < R * K / 8; c += blockDim.x) {
      const uint32_t row = c / (K / 8), k = (c % (K / 8)) * 8;
      *reinterpret_cast<uint4*>(sm + off + sw_off(R, row, k)) =
          *reinterpret_cast<const uint4*>(W + (size_t)row * K + k);
    }
  };
  put_w(kOffW1, fi.net.W1b, 128, kIn);
  put_w(kOffW2, fi.net.W2b, 128, kHid);
  put_w(kOffW3, fi.net.W3b, 128, kHid);
  put_w(kOffW4, fi.net.W4b, 128, kHid);
  for (int i = tid; i < kHid; i += blockDim.x) {
    s_bias[i] = fi.net.b1[i];
    s_bias[kHid + i] = fi.net.b2[i];
    s_bias[2 * kHid + i] = fi.net.b3[i];
    s_bias[3 * kHid + i] = fi.net.b4[i];
  }
  if (!CODES) {
    // B of the projection: row c, c+3, c+6 = the three bf16 terms of Pc[:, c]
    for (uint32_t i = tid; i < 16 * kHid; i += blockDim.x) {
      const uint32_t row = i / kHid, k = i % kHid;
      float v = 0.0f;
      if (row < 9) {
        const float p = fi.proj[3 * k + row % 3];
        const float t1 = __bfloat162float(__float2bfloat16_rn(p));
        const float t2 = __bfloat162float(__float2bfloat16_rn(p - t1));
        v = row < 3 ? t1 : (row < 6 ? t2 : p - t1 - t2);
      }
      *reinterpret_cast<__nv_bfloat16*>(sm + kOffP + sw_off(16, row, k)) = __float2bfloat16_rn(v);
    }
    if (tid < 12) s_misc[tid] = fi.proj[3 * kHid + tid];
  }
  if (tid < kTcWG) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&s_mbar[tid])));
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_u32(s_tmem)),
                 "r"(kTcAlloc));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
  }
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *s_tmem + (uint32_t)wg * kTcCols;
  const uint32_t t_row = tmem + ((uint32_t)q4 * 32u << 16);  // this warp's lanes
  const uint32_t mbar = smem_u32(&s_mbar[wg]);
  unsigned char* Bt = sm + kOffB + (uint32_t)wg * kBTile;
  const uint32_t b_addr = smem_u32(Bt);
  const uint32_t base_addr = smem_u32(sm);
  const uint32_t id_h = idesc_bf16(128, 128, 0, 1), id_p = idesc_bf16(128, 16, 1, 0);
  const bool leader = (tid & 127) == 0;
  uint32_t phase = 0;
  bool ok = true;
  // The leader waits for the commit; the warpgroup learns the outcome behind
  // a barrier (so every thread takes the same path) and orders its TMEM reads
  // after it with tcgen05.fence::after_thread_sync.
  auto wait_mma = [&]() {
    if (leader) s_ok[wg] = mbar_wait(mbar, phase) ? 1u : 0u;
    wg_sync(wg);
    ok = s_ok[wg] != 0u;
    phase ^= 1u;
    tc_fence_after();
    return ok;
  };
  // row j of the activation tile: 8 chunks of 16 B per 64-column half
  unsigned char* rowj = Bt + (j >> 3) * 1024 + (j & 7) * 128;
  const uint32_t swz = j & 7;

  const uint32_t tiles = (fi.count + kItems - 1) / kItems;
  for (uint32_t t = blockIdx.x * kTcWG + wg; t < tiles && ok; t += gridDim.x * kTcWG) {
    // ---- layer-1 operand: row k = feature k; column 4 p + s = the feature
    // of item p (s = 0) or its derivative along axis s - 1. Thread (q4, p)
    // evaluates the sine/cosine pairs i = 6 q4 .. 6 q4 + 5 (band i / 3,
    // axis i % 3) of item p and rows 4 q4 .. 4 q4 + 3 of {0, 1, 2, 51..63}.
    // (The previous tile's last product, which read this operand, has
    // completed: its wait came before.)
    {
      const uint32_t p = (uint32_t)lane, k_item = t * kItems + p;
      float3 x3 = make_float3(0.0f, 0.0f, 0.0f);
      if (k_item < fi.count) x3 = item_position(fi, k_item);
      if (CODES && q4 == 0 && k_item < fi.count)
        fi.code_pos[k_item] = make_float4(x3.x, x3.y, x3.z, 0.0f);
      const float inv_s = fi.enc[3];
      const float xh[3] = {(x3.x - fi.enc[0]) * inv_s, (x3.y - fi.enc[1]) * inv_s,
                           (x3.z - fi.enc[2]) * inv_s};
      // row k, streams 0-3 (a, b, c, d) of item p: the even lane of a pair
      // writes streams 0 and 1 of both items (the chunk's first 8 bytes), the
      // odd lane streams 2 and 3, after one exchange of packed halves. Every
      // call is made by the whole warp (k depends on the warp only).
      auto put4 = [&](uint32_t k, float a, float b, float c, float d) {
        const bool odd = (p & 1u) != 0u;
        const uint32_t keep = odd ? pack2(c, d) : pack2(a, b);
        const uint32_t give = odd ? pack2(a, b) : pack2(c, d);
        const uint32_t got = __shfl_xor_sync(0xffffffffu, give, 1);
        const uint32_t lo = odd ? got : keep, hi = odd ? keep : got;  // item 2 c, item 2 c + 1
        *reinterpret_cast<uint2*>(Bt + mn_chunk(k, p >> 1) + (p & 1) * 8) =
            make_uint2(__byte_perm(lo, hi, 0x5410), __byte_perm(lo, hi, 0x7632));
      };
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        // bands 2 q4 and 2 q4 + 1 of axis d: the second (twice the angle) from
        // the first by the double-angle identities (a few ulp, far below the
        // bf16 rounding of the operand)
        const int b = 2 * q4;
        const float w = (float)(1 << b) * 1.57079632679489662f;
        float sn, cs;
        sincosf(w * xh[d], &sn, &cs);
        const float sn2 = 2.0f * sn * cs, cs2 = (cs - sn) * (cs + sn);
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const float we = e ? 2.0f * w : w, se = e ? sn2 : sn, ce = e ? cs2 : cs;
          const float ds = we * ce * inv_s, dc = -we * se * inv_s;
          const uint32_t ks = 3u + 6u * (uint32_t)(b + e) + 2u * (uint32_t)d;
          put4(ks, se, d == 0 ? ds : 0.0f, d == 1 ? ds : 0.0f, d == 2 ? ds : 0.0f);
          put4(ks + 1, ce, d == 0 ? dc : 0.0f, d == 1 ? dc : 0.0f, d == 2 ? dc : 0.0f);
        }
      }
#pragma unroll
      for (int kk = 0; kk < 4; ++kk) {
        const int idx = 4 * q4 + kk;
        if (idx < 3)
          put4((uint32_t)idx, xh[idx], idx == 0 ? inv_s : 0.0f, idx == 1 ? inv_s : 0.0f,
               idx == 2 ? inv_s : 0.0f);
        else
          put4((uint32_t)(48 + idx), 0.0f, 0.0f, 0.0f, 0.0f);
      }
    }
    // ---- four hidden layers: D[j][n] = sum_k W[j][k] X[k][n]
#pragma unroll 1
    for (int l = 0; l < 4 && ok; ++l) {
      fence_async_smem();
      tc_fence_before();
      wg_sync(wg);
      if (leader) {
        tc_fence_after();
        const uint32_t woff = l == 0 ? kOffW1 : (l == 1 ? kOffW2 : (l == 2 ? kOffW3 : kOffW4));
        const uint32_t K = l == 0 ? kIn : kHid;
        for (uint32_t ks = 0; ks < K / 16; ++ks) {
          const uint32_t kb = ks >> 2, kin = (ks & 3) * 32;
          mma_bf16_tc(tmem, sw128_desc(base_addr + woff + kb * 16384 + kin),
                      sw128_desc(b_addr + ks * 2048, kMnBlock), id_h, ks > 0);
        }
        mma_commit(mbar);
      }
      if (!wait_mma()) break;
      const float bj = s_bias[l * kHid + j];
      // SiLU a = x sigmoid(x) and its slope a' = sg (1 + x (1 - sg)), with
      // sg = 1 / (1 + 2^(-x log2 e)) and x = pre-activation + bias
      constexpr float kLog2e = 1.4426950408889634f;
      const uint64_t b2 = f2_splat(bj), nl2 = f2_splat(-kLog2e), nbl2 = f2_splat(-bj * kLog2e);
      const uint64_t one2 = f2_splat(1.0f), mone2 = f2_splat(-1.0f);
      const bool last = l == 3;
#pragma unroll 1
      for (int h = 0; h < 2; ++h) {  // columns 64 h .. 64 h + 63 = items 16 h .. 16 h + 15
        uint32_t v[64];
        tmem_ld32_nowait<0>(t_row + (uint32_t)h * 64u, v);
        tmem_ld32_nowait<32>(t_row + (uint32_t)h * 64u + 32u, v);
        tmem_wait_ld();
        uint32_t o[32];
#pragma unroll
        for (int c = 0; c < 8; ++c) {  // items 16 h + 2 c and 16 h + 2 c + 1, lane-paired
          const uint32_t* w = v + 8 * c;
          const uint64_t acc = f2_make(w[0], w[1]);
          const uint64_t pre = f2_add(acc, b2);
          const uint64_t sg = f2_rcp(f2_add(f2_ex2(f2_fma(acc, nl2, nbl2)), one2));
          const uint64_t sl = f2_mul(sg, f2_fma(pre, f2_fma(sg, mone2, one2), one2));
          o[4 * c] = f2_bf16(f2_mul(pre, sg));
          o[4 * c + 1] = f2_bf16(f2_mul(f2_make(w[2], w[3]), sl));
          o[4 * c + 2] = f2_bf16(f2_mul(f2_make(w[4], w[5]), sl));
          o[4 * c + 3] = f2_bf16(f2_mul(f2_make(w[6], w[7]), sl));
        }
        if (CODES && last) {
          // code of an item: [stream][unit] bf16
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            const uint32_t k_item = t * kItems + 16u * (uint32_t)h + (uint32_t)i;
            if (k_item < fi.count) {
              unsigned short* dst =
                  reinterpret_cast<unsigned short*>(fi.codes + (size_t)k_item * (4 * kHid)) + j;
              const uint32_t* oc = o + 4 * (i >> 1);
              const uint32_t sh = (uint32_t)(i & 1) * 16u;
#pragma unroll
              for (int s = 0; s < 4; ++s) dst[s * kHid] = (unsigned short)(oc[s] >> sh);
            }
          }
        } else {
          unsigned char* rp = rowj + (uint32_t)h * kMnBlock;
#pragma unroll
          for (int c = 0; c < 8; ++c)
            *reinterpret_cast<uint4*>(rp + (((uint32_t)c ^ swz) << 4)) =
                make_uint4(o[4 * c], o[4 * c + 1], o[4 * c + 2], o[4 * c + 3]);
        }
      }
    }
    if (!ok) break;
    if (CODES) continue;
    // ---- output projection: D[n][c] = sum_k X[k][n] Pc'[c][k], N = 16
    fence_async_smem();
    tc_fence_before();
    wg_sync(wg);
    if (leader) {
      tc_fence_after();
      for (uint32_t ks = 0; ks < kHid / 16; ++ks) {
        const uint32_t kb = ks >> 2, kin = (ks & 3) * 32;
        mma_bf16_tc(tmem, sw128_desc(b_addr + ks * 2048, kMnBlock),
                    sw128_desc(base_addr + kOffP + kb * 2048 + kin), id_p, ks > 0);
      }
      mma_commit(mbar);
    }
    if (!wait_mma()) break;
    uint32_t v[16];
    tmem_ld16(t_row, v);
    // lane j = column n: item 2 (n / 8) + n % 2, stream (n / 2) % 4
    const uint32_t k_item = t * kItems + 2u * (j >> 3) + (j & 1u), s_st = (j >> 1) & 3u;
    if (k_item < fi.count) {
      float* out = reinterpret_cast<float*>(fi.xf) + 12 * (size_t)(fi.out_first + k_item);
      const float* pc = s_misc;
      const float* A3 = s_misc + 3;
      if (s_st == 0) {
        const float3 x3 = item_position(fi, k_item);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const float y =
              (__uint_as_float(v[c]) + __uint_as_float(v[3 + c])) + __uint_as_float(v[6 + c]);
          out[c] = y + pc[c] + (A3[3 * c] * x3.x + A3[3 * c + 1] * x3.y + A3[3 * c + 2] * x3.z);
        }
      } else {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const float y =
              (__uint_as_float(v[c]) + __uint_as_float(v[3 + c])) + __uint_as_float(v[6 + c]);
          out[3 + 3 * (s_st - 1) + c] = y + A3[3 * c + (s_st - 1)];
        }
      }
    }
  }
  if (!ok && leader) {
    if (fi.status) atomicOr(fi.status, kStatusBarrierTimeout);
    // the MMAs given up on, once more (bounded); if they still have not
    // completed, tensor memory may be written after the release below
    if (!mbar_wait(mbar, phase ^ 1u) && fi.status) atomicOr(fi.status, kStatusPoisoned);
  }
  // release TMEM once every warpgroup is done with it
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(*s_tmem),
                 "r"(kTcAlloc));
  }
}

// ---- training GEMMs: C = A B^T (+ bias), D = bf16(silu(C)) -------------------
// One CTA of 128 threads per 128 x 128 output tile. K is consumed in 64-wide
// blocks through a 4-stage ring: every thread copies its share of a block's
// A and B rows into shared memory with 16-byte cp.async (rows past M or N and
// columns past K zero-filled) in the K-major 128-byte-swizzle layout, one
// elected thread issues the block's four K = 16 tcgen05 MMAs into a 128-column
// TMEM accumulator and commits them to the stage's mbarrier, and the copies
// run two blocks ahead of the MMAs; a stage is refilled once the MMAs that
// read it have completed. The epilogue reads the accumulator row by row
// (TMEM lane = output row) and applies the bias and SiLU.
constexpr uint32_t kGmTile = 128, kGmBK = 64, kGmStages = 4, kGmAhead = 2;
constexpr uint32_t kGmStageBytes = 2 * kGmTile * kGmBK * 2;   // A and B, 32 KB
constexpr uint32_t kGmSmem = kGmStages * kGmStageBytes + 256 + 1024;

__device__ __forceinline__ void cp_async16_zfill(uint32_t dst, const void* src, uint32_t bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

constexpr uint32_t kGmMaxSplits = 16;

// C[r][c] = sum over splits z (in order) of ws[z][r][c].
__global__ void k_split_reduce(const float* __restrict__ ws, uint32_t splits, uint32_t M,
                               uint32_t N, float* __restrict__ C, uint32_t ldc) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= M * N) return;
  float acc = 0.0f;
  for (uint32_t z = 0; z < splits; ++z) acc += ws[(size_t)z * M * N + i];
  C[(size_t)(i / N) * ldc + i % N] = acc;
}

template <int EPI>
__global__ void __launch_bounds__(128, 1) k_gemm_tc(GemmArgs g) {
  extern __shared__ unsigned char gm_raw[];
  unsigned char* sm = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(gm_raw) + 1023) & ~(uintptr_t)1023);
  uint64_t* s_bar = reinterpret_cast<uint64_t*>(sm + kGmStages * kGmStageBytes);  // [stages]
  uint32_t* s_tmem = reinterpret_cast<uint32_t*>(s_bar + kGmStages);
  volatile uint32_t* s_ok = s_tmem + 1;  // [2], alternating by block
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t m0 = blockIdx.y * kGmTile, n0 = blockIdx.x * kGmTile;
  // split z of K: blocks [kb0, kb0 + nk) of the K range
  const uint32_t nkb = (g.K + kGmBK - 1) / kGmBK, per = (nkb + gridDim.z - 1) / gridDim.z;
  const uint32_t kb0 = min(nkb, blockIdx.z * per), nk = min(nkb, kb0 + per) - kb0;
  const bool split = gridDim.z > 1;
  if (tid < (int)kGmStages)
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&s_bar[tid])));
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_u32(s_tmem)),
                 "r"(kGmTile));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
  }
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *s_tmem;
  const uint32_t base = smem_u32(sm);
  const uint32_t idesc = idesc_bf16(kGmTile, kGmTile, 0, 0);

  // block kb of A rows m0.. and B rows n0.. into stage kb % stages
  auto load = [&](uint32_t kb) {
    const uint32_t st = base + (kb % kGmStages) * kGmStageBytes, k0 = (kb0 + kb) * kGmBK;
#pragma unroll 4
    for (uint32_t c = (uint32_t)tid; c < 2 * kGmTile * 8; c += 128) {
      const bool isb = c >= kGmTile * 8;
      const uint32_t cc = isb ? c - kGmTile * 8 : c, row = cc >> 3, ch = cc & 7;
      const uint32_t grow = (isb ? n0 : m0) + row, R = isb ? g.N : g.M, k = k0 + ch * 8;
      const __nv_bfloat16* mat = isb ? g.B : g.A;
      const void* src = mat;
      uint32_t bytes = 0;
      if (grow < R && k < g.K) {
        bytes = min(8u, g.K - k) * 2u;
        src = mat + (size_t)grow * (isb ? g.ldb : g.lda) + k;
      }
      cp_async16_zfill(st + (isb ? kGmTile * 128 : 0) + (row >> 3) * 1024 + (row & 7) * 128 +
                           ((ch ^ (row & 7)) << 4),
                       src, bytes);
    }
  };
#pragma unroll
  for (uint32_t p = 0; p < kGmAhead; ++p) {
    if (p < nk) load(p);
    cp_async_commit();
  }
  bool ok = true;
  uint32_t issued = 0;  // blocks whose MMAs were issued (block-uniform)
  for (uint32_t kb = 0; kb < nk; ++kb) {
    cp_async_wait<kGmAhead - 1>();  // this thread's copies of block kb have landed
    fence_async_smem();
    // the stage refilled below was read by the MMAs of block kb - ahead
    if (tid == 0 && kb >= kGmAhead) {
      const uint32_t q = kb - kGmAhead;
      s_ok[kb & 1u] = mbar_wait(smem_u32(&s_bar[q % kGmStages]), (q / kGmStages) & 1u) ? 1u : 0u;
    }
    __syncthreads();
    if (kb >= kGmAhead && s_ok[kb & 1u] == 0u) {
      ok = false;
      break;
    }
    if (tid == 0) {
      tc_fence_after();
      const uint32_t a = base + (kb % kGmStages) * kGmStageBytes, b = a + kGmTile * 128;
#pragma unroll
      for (uint32_t k16 = 0; k16 < kGmBK / 16; ++k16)
        mma_bf16_tc(tmem, sw128_desc(a + k16 * 32), sw128_desc(b + k16 * 32), idesc,
                    (kb > 0 || k16 > 0) ? 1u : 0u);
      mma_commit(smem_u32(&s_bar[kb % kGmStages]));
    }
    issued = kb + 1;
    if (kb + kGmAhead < nk) load(kb + kGmAhead);
    cp_async_commit();
  }
  cp_async_wait<0>();
  // the last commit covers every MMA issued before it
  if (tid == 0) {
    bool done = true;
    if (issued > 0) {
      const uint32_t q = issued - 1;
      done = mbar_wait(smem_u32(&s_bar[q % kGmStages]), (q / kGmStages) & 1u);
    }
    s_ok[0] = (ok && done) ? 1u : 0u;
    if ((!ok || !done) && g.status) {
      atomicOr(g.status, kStatusBarrierTimeout);
      // MMAs still running may write tensor memory after its release below
      if (!done) atomicOr(g.status, kStatusPoisoned);
    }
  }
  __syncthreads();
  ok = s_ok[0] != 0u;
  tc_fence_after();
  if (ok) {
    const uint32_t row = m0 + 32u * (uint32_t)warp + (uint32_t)lane;
    const uint32_t t_row = tmem + ((uint32_t)warp * 32u << 16);
    const bool vec_c = ((g.ldc & 3u) == 0u) && (((uintptr_t)g.C & 15u) == 0u);
    const bool vec_d = ((g.ldd & 7u) == 0u) && (((uintptr_t)g.D & 15u) == 0u);
#pragma unroll 1
    for (uint32_t c0 = 0; c0 < kGmTile; c0 += 32) {
      uint32_t v[32];
      if (nk > 0) {
        tmem_ld32_nowait<0>(t_row + c0, v);  // every lane of the warp loads (aligned)
        tmem_wait_ld();
      } else {
#pragma unroll
        for (int i = 0; i < 32; ++i) v[i] = 0u;
      }
      const uint32_t col0 = n0 + c0;
      if (row >= g.M || col0 >= g.N) continue;
      float x[32];
#pragma unroll
      for (int i = 0; i < 32; ++i) {
        x[i] = __uint_as_float(v[i]);
        if (EPI != kEpiF32 && col0 + i < g.N) x[i] += g.bias[col0 + i];
      }
      // a split's partial sums go to its slice of the workspace ([M][N] each)
      float* crow = split ? g.ws + ((size_t)blockIdx.z * g.M + row) * g.N + col0
                          : g.C + (size_t)row * g.ldc + col0;
      if (split) {
#pragma unroll
        for (int i = 0; i < 32; ++i)
          if (col0 + i < g.N) crow[i] = x[i];
        continue;
      }
      if (vec_c && col0 + 32 <= g.N) {
#pragma unroll
        for (int i = 0; i < 32; i += 4)
          *reinterpret_cast<float4*>(crow + i) = make_float4(x[i], x[i + 1], x[i + 2], x[i + 3]);
      } else {
#pragma unroll
        for (int i = 0; i < 32; ++i)
          if (col0 + i < g.N) crow[i] = x[i];
      }
      if (EPI == kEpiBiasSilu) {
        __nv_bfloat16* drow = g.D + (size_t)row * g.ldd + col0;
        if (vec_d && col0 + 32 <= g.N) {
#pragma unroll
          for (int i = 0; i < 32; i += 8) {
            uint32_t w[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              const float a0 = x[i + 2 * e], a1 = x[i + 2 * e + 1];
              w[e] = pack2(a0 * (1.0f / (1.0f + __expf(-a0))), a1 * (1.0f / (1.0f + __expf(-a1))));
            }
            *reinterpret_cast<uint4*>(drow + i) = make_uint4(w[0], w[1], w[2], w[3]);
          }
        } else {
#pragma unroll
          for (int i = 0; i < 32; ++i)
            if (col0 + i < g.N) drow[i] = __float2bfloat16_rn(x[i] * (1.0f / (1.0f + __expf(-x[i]))));
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem),
                 "r"(kGmTile));
}

}  // namespace

cudaError_t launch_field_infer_tc(const FieldInfer& fi, cudaStream_t s) {
  if (fi.count == 0) return cudaSuccess;
  const cudaError_t e =
      fi.codes ? cudaFuncSetAttribute(k_field_infer_tc<true>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem)
               : cudaFuncSetAttribute(k_field_infer_tc<false>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem);
  if (e != cudaSuccess) return e;
  static int sm_count = 0;
  if (sm_count == 0) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
      sm_count = 148;
  }
  const uint32_t tiles = (fi.count + kItems - 1) / kItems;
  const uint32_t blocks = std::min<uint32_t>((uint32_t)sm_count, (tiles + kTcWG - 1) / kTcWG);
  if (fi.codes)
    k_field_infer_tc<true><<<blocks, kTcWG * 128, kTcSmem, s>>>(fi);
  else
    k_field_infer_tc<false><<<blocks, kTcWG * 128, kTcSmem, s>>>(fi);
  return cudaGetLastError();
}

cudaError_t launch_gemm_nt(const GemmArgs& g, int epi, cudaStream_t s) {
  if (g.M == 0 || g.N == 0) return cudaSuccess;
  if ((g.lda & 7) || (g.ldb & 7)) return cudaErrorInvalidValue;
  if (((uintptr_t)g.A & 15) || ((uintptr_t)g.B & 15)) return cudaErrorInvalidValue;
  static int sm_count = 0;
  if (sm_count == 0) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
      sm_count = 148;
  }
  dim3 grid((g.N + kGmTile - 1) / kGmTile, (g.M + kGmTile - 1) / kGmTile, 1);
  // Long K over few tiles (the weight gradients: K = the batch): split K so
  // that the grid covers the SMs; the partial sums are added in split order
  // (deterministic) by k_split_reduce.
  const uint32_t tiles = grid.x * grid.y, nkb = (g.K + kGmBK - 1) / kGmBK;
  if (epi == kEpiF32 && g.ws && tiles * 2 <= (uint32_t)sm_count && nkb >= 8) {
    uint32_t z = std::min<uint32_t>({(uint32_t)sm_count / tiles, nkb / 4, kGmMaxSplits});
    while (z > 1 && (size_t)z * g.M * g.N > g.ws_floats) --z;
    grid.z = std::max<uint32_t>(1, z);
  }
  cudaError_t e;
  if (epi == kEpiF32) {
    e = cudaFuncSetAttribute(k_gemm_tc<kEpiF32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kGmSmem);
    if (e == cudaSuccess) k_gemm_tc<kEpiF32><<<grid, 128, kGmSmem, s>>>(g);
    if (e == cudaSuccess && grid.z > 1) {
      e = cudaGetLastError();
      const uint32_t n = g.M * g.N;
      if (e == cudaSuccess)
        k_split_reduce<<<(n + 255) / 256, 256, 0, s>>>(g.ws, grid.z, g.M, g.N, g.C, g.ldc);
    }
  } else if (epi == kEpiBias) {
    e = cudaFuncSetAttribute(k_gemm_tc<kEpiBias>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kGmSmem);
    if (e == cudaSuccess) k_gemm_tc<kEpiBias><<<grid, 128, kGmSmem, s>>>(g);
  } else {
    e = cudaFuncSetAttribute(k_gemm_tc<kEpiBiasSilu>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGmSmem);
    if (e == cudaSuccess) k_gemm_tc<kEpiBiasSilu><<<grid, 128, kGmSmem, s>>>(g);
  }
  return e != cudaSuccess ? e : cudaGetLastError();
}

}  // namespace cgs
