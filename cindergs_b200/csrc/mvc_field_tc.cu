// Fused inference of the learned MVC field on the 5th-generation tensor cores
// (tcgen05): per Gaussian, the network and its three forward-mode tangents,
// then either the position and deformation gradient on the current cage
// (x' = Pc^T h + pc + A3 x, F = Pc^T dh + A3; k_mvc_jacobian's layout) or the
// last hidden layer and its tangents as the cached code (bf16 [4][128]).
//
// One CTA per SM, two warpgroups; each warpgroup owns a tile of 32 items =
// 128 rows, stream-major (row 32 s + p: item p, stream s = value, d/dx,
// d/dy, d/dz), i.e. one M = 128 tcgen05.mma tile in which warp s of the
// warpgroup reads stream s of every item (tcgen05.ld 32x32b, lane = row).
// Per layer one elected thread issues the K = 16 steps into the
// warpgroup's 128-column TMEM accumulator and commits them to an mbarrier;
// then, 32 columns at a time, the value warp stages the pre-activations in
// shared memory, each of the four warps evaluates the SiLU and its slope for
// 8 of the columns of every item, and each warp takes back what its stream
// needs (the activation, or the slope times its tangent) and writes the
// bf16 result as the next layer's A operand. The sine/cosine pairs of the
// Fourier features are likewise computed once per item, 6 of the 24 pairs
// by each warp. Operands live in shared memory in
// the K-major, 128-byte-swizzle canonical layout: rows of 64 bf16 (128 B),
// 8-row atoms of 1024 B, 16-byte chunk c of row r stored at chunk
// c ^ (r % 8). The output projection is one more MMA with N = 16 against
// Pc split into three bf16 terms (columns 0-2, 3-5, 6-8), so that the
// products are exact and only the fp32 accumulation rounds.
//
// Every mbarrier wait is bounded; a wait that gives up sets the status word
// and the warpgroup stops issuing work (TMEM is released at the end).
#include <cuda_bf16.h>

#include <algorithm>

#include "kernels.h"

namespace cgs {
namespace {

constexpr int kHid = kFieldHid, kIn = kFieldIn;
constexpr int kTcWG = 2;                 // warpgroups (tiles in flight) per CTA
constexpr uint32_t kTcCols = 256;        // TMEM columns per warpgroup (128 hidden + 16 proj)
constexpr uint32_t kTcWaitLimit = 1u << 20;

// shared memory map (bytes from the 1024-aligned base)
constexpr uint32_t kOffW1 = 0;                        // [128 x 64]   16 KB
constexpr uint32_t kOffW2 = kOffW1 + 128 * 64 * 2;    // [128 x 128]  32 KB each
constexpr uint32_t kOffW3 = kOffW2 + 128 * 128 * 2;
constexpr uint32_t kOffW4 = kOffW3 + 128 * 128 * 2;
constexpr uint32_t kOffP = kOffW4 + 128 * 128 * 2;    // [16 x 128]   4 KB
constexpr uint32_t kOffA = kOffP + 16 * 128 * 2;      // [128 x 128] per warpgroup
constexpr uint32_t kOffBias = kOffA + kTcWG * 128 * 128 * 2;  // 4 x 128 f32
constexpr uint32_t kChunk = 64;                        // columns per epilogue step
constexpr uint32_t kXStride = kChunk + 4;                // floats per item row (bank spread)
constexpr uint32_t kOffX = kOffBias + 4 * 128 * 4;    // per warpgroup: exchange area
constexpr uint32_t kXBytes = 2 * 32 * kXStride * 4;      //   pre (then act), slope [32 item][68]
constexpr uint32_t kOffMisc = kOffX + kTcWG * kXBytes;   // pc, A3, mbarriers, tmem
constexpr uint32_t kTcSmem = kOffMisc + 256 + 1024;      // + alignment slack

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Byte offset of element (r, k) of a K-major swizzled operand with R rows.
__device__ __forceinline__ uint32_t sw_off(uint32_t R, uint32_t r, uint32_t k) {
  const uint32_t kb = k >> 6, kk = k & 63;
  const uint32_t chunk = (kk >> 3) ^ (r & 7);
  return kb * (R * 128) + (r >> 3) * 1024 + (r & 7) * 128 + chunk * 16 + (kk & 7) * 2;
}

// Shared memory matrix descriptor: K-major, 128-byte swizzle, SBO = 1024 B.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)1 << 16;              // leading byte offset (unused for this layout)
  d |= (uint64_t)(1024 >> 4) << 32;    // stride byte offset: next 8-row atom
  d |= (uint64_t)1 << 46;              // descriptor version
  d |= (uint64_t)2 << 61;              // 128-byte swizzle
  return d;
}

// Instruction descriptor: kind::f16, bf16 A and B (K-major), f32 accumulate.
__host__ __device__ constexpr uint32_t idesc_bf16(uint32_t M, uint32_t N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((N >> 3) << 17) | ((M >> 4) << 24);
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
// 32 consecutive TMEM columns of this thread's lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, "
      "%28, %29, %30, %31}, [%32];\n"
      : CGS_R8(0), CGS_R8(8), CGS_R8(16), CGS_R8(24)
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15}, [%16];\n"
      : CGS_R8(0), CGS_R8(8)
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}
#undef CGS_R8

__device__ __forceinline__ uint32_t pack2(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&v);
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
  const int wg = warp >> 2, r = tid & 127;  // warpgroup, row within its tile
  const int s_st = warp & 3, p = lane;      // stream (warp in the warpgroup), item (lane)
  float* X = reinterpret_cast<float*>(sm + kOffX + (uint32_t)wg * kXBytes);
  float* X_pre = X + p * kXStride;                 // this item's row: pre-activation, then act
  float* X_slp = X + (32 + p) * kXStride;          // this item's row: SiLU slope

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
                 "r"(kTcCols * kTcWG));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
  }
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *s_tmem + (uint32_t)wg * kTcCols;
  const uint32_t t_row = tmem + ((uint32_t)(warp & 3) * 32u << 16);  // this warp's lanes
  const uint32_t mbar = smem_u32(&s_mbar[wg]);
  unsigned char* A = sm + kOffA + (uint32_t)wg * 128 * 128 * 2;
  const uint32_t a_addr = smem_u32(A);
  const uint32_t base_addr = smem_u32(sm);
  const uint32_t id_h = idesc_bf16(128, 128), id_p = idesc_bf16(128, 16);
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

  const uint32_t tiles = (fi.count + 31) / 32;
  for (uint32_t t = blockIdx.x * kTcWG + wg; t < tiles && ok; t += gridDim.x * kTcWG) {
    const uint32_t k_item = t * 32 + p;
    const bool valid = k_item < fi.count;
    float xr[3] = {0.0f, 0.0f, 0.0f};
    if (valid) {
      const uint32_t gi = fi.gauss ? fi.gauss[fi.first + k_item] : fi.first + k_item;
      if (fi.points4) {
        const float4 x4 = fi.points4[gi];
        xr[0] = x4.x;
        xr[1] = x4.y;
        xr[2] = x4.z;
      } else {
        xr[0] = fi.points3[3 * (size_t)gi];
        xr[1] = fi.points3[3 * (size_t)gi + 1];
        xr[2] = fi.points3[3 * (size_t)gi + 2];
      }
    }
    // ---- layer-1 input row: features (value row) or their derivative along
    // one axis (tangent rows), bf16, K = 64. Pair i = 3 b + d (band b, axis
    // d): warp w computes pairs 6w .. 6w + 5 of every item.
    {
      const float inv_s = fi.enc[3];
      const float xh[3] = {(xr[0] - fi.enc[0]) * inv_s, (xr[1] - fi.enc[1]) * inv_s,
                           (xr[2] - fi.enc[2]) * inv_s};
      float* S = X;  // [24 pairs][32 items] x (sin, cos)
      wg_sync(wg);   // the previous tile's readers of the exchange area are done
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        const int i = 6 * s_st + k, b = i / 3, d = i % 3;
        const float w = (float)(1 << b) * 1.57079632679489662f;
        float sn, cs;
        sincosf(w * (d == 0 ? xh[0] : (d == 1 ? xh[1] : xh[2])), &sn, &cs);
        S[(2 * i) * 32 + p] = sn;
        S[(2 * i + 1) * 32 + p] = cs;
      }
      wg_sync(wg);
      const int ax = s_st - 1;  // tangent axis (-1 for the value row)
#pragma unroll 1
      for (int c = 0; c < kIn / 8; ++c) {
        float f8[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          const int j = c * 8 + e;
          float f = 0.0f;
          if (j < 3) {
            f = s_st == 0 ? xh[j] : (j == ax ? inv_s : 0.0f);
          } else if (j < 3 + 6 * kFieldBands) {
            const int q = j - 3, b = q / 6, d = (q % 6) >> 1, i = 3 * b + d;
            const bool is_cos = q & 1;
            if (s_st == 0) {
              f = S[(2 * i + (is_cos ? 1 : 0)) * 32 + p];
            } else if (d == ax) {
              const float w = (float)(1 << b) * 1.57079632679489662f;
              f = is_cos ? -w * S[(2 * i) * 32 + p] * inv_s : w * S[(2 * i + 1) * 32 + p] * inv_s;
            }
          }
          f8[e] = f;
        }
        *reinterpret_cast<uint4*>(A + sw_off(128, r, c * 8)) =
            make_uint4(pack2(f8[0], f8[1]), pack2(f8[2], f8[3]), pack2(f8[4], f8[5]),
                       pack2(f8[6], f8[7]));
      }
    }
    // ---- four hidden layers
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
          mma_bf16_tc(tmem, sw128_desc(a_addr + kb * 16384 + kin),
                      sw128_desc(base_addr + woff + kb * 16384 + kin), id_h, ks > 0);
        }
        mma_commit(mbar);
      }
      if (!wait_mma()) break;
      const float* bias = s_bias + l * kHid;
      const bool last = l == 3;
#pragma unroll 1
      for (int q = 0; q < kHid / (int)kChunk; ++q) {
        uint32_t v[kChunk];
        {
          uint32_t (&v0)[32] = *reinterpret_cast<uint32_t(*)[32]>(&v[0]);
          uint32_t (&v1)[32] = *reinterpret_cast<uint32_t(*)[32]>(&v[32]);
          tmem_ld32(t_row + (uint32_t)q * kChunk, v0);
          tmem_ld32(t_row + (uint32_t)q * kChunk + 32, v1);
        }
        const float* bq = bias + q * kChunk;
        if (s_st == 0) {
#pragma unroll
          for (int j = 0; j < (int)kChunk; j += 4)
            *reinterpret_cast<float4*>(X_pre + j) =
                make_float4(__uint_as_float(v[j]) + bq[j], __uint_as_float(v[j + 1]) + bq[j + 1],
                            __uint_as_float(v[j + 2]) + bq[j + 2], __uint_as_float(v[j + 3]) + bq[j + 3]);
        }
        wg_sync(wg);
        // SiLU and its slope for columns 16 w .. 16 w + 15 of this item (the
        // activation replaces the pre-activation)
#pragma unroll
        for (int k = 0; k < 16; k += 4) {
          const int j = 16 * s_st + k;
          const float4 pre4 = *reinterpret_cast<const float4*>(X_pre + j);
          const float pr[4] = {pre4.x, pre4.y, pre4.z, pre4.w};
          float ac[4], sl[4];
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const float sg = __fdividef(1.0f, 1.0f + __expf(-pr[e]));
            ac[e] = pr[e] * sg;
            sl[e] = sg * (1.0f + pr[e] * (1.0f - sg));
          }
          *reinterpret_cast<float4*>(X_pre + j) = make_float4(ac[0], ac[1], ac[2], ac[3]);
          *reinterpret_cast<float4*>(X_slp + j) = make_float4(sl[0], sl[1], sl[2], sl[3]);
        }
        wg_sync(wg);
        uint32_t outw[kChunk / 2];
        const float* src = s_st == 0 ? X_pre : X_slp;
#pragma unroll
        for (int j = 0; j < (int)kChunk; j += 4) {
          const float4 w4 = *reinterpret_cast<const float4*>(src + j);
          if (s_st == 0) {
            outw[j >> 1] = pack2(w4.x, w4.y);
            outw[(j >> 1) + 1] = pack2(w4.z, w4.w);
          } else {
            outw[j >> 1] = pack2(__uint_as_float(v[j]) * w4.x, __uint_as_float(v[j + 1]) * w4.y);
            outw[(j >> 1) + 1] =
                pack2(__uint_as_float(v[j + 2]) * w4.z, __uint_as_float(v[j + 3]) * w4.w);
          }
        }
#pragma unroll
        for (int c4 = 0; c4 < (int)kChunk / 8; ++c4)
          *reinterpret_cast<uint4*>(A + sw_off(128, r, q * kChunk + c4 * 8)) =
              make_uint4(outw[4 * c4], outw[4 * c4 + 1], outw[4 * c4 + 2], outw[4 * c4 + 3]);
        if (CODES && last && valid) {
          uint4* dst = reinterpret_cast<uint4*>(fi.codes + (size_t)k_item * (4 * kHid) +
                                                s_st * kHid + q * kChunk);
#pragma unroll
          for (int c4 = 0; c4 < (int)kChunk / 8; ++c4)
            dst[c4] = make_uint4(outw[4 * c4], outw[4 * c4 + 1], outw[4 * c4 + 2], outw[4 * c4 + 3]);
        }
        // (the next chunk's first writes come after every warp passed this
        // chunk's second barrier, i.e. after all reads of the pre-activations)
      }
    }
    if (!ok) break;
    if (CODES) {
      if (valid && s_st == 0) fi.code_pos[k_item] = make_float4(xr[0], xr[1], xr[2], 0.0f);
      continue;
    }
    // ---- output projection: N = 16 against the split Pc
    fence_async_smem();
    tc_fence_before();
    wg_sync(wg);
    if (leader) {
      tc_fence_after();
      for (uint32_t ks = 0; ks < kHid / 16; ++ks) {
        const uint32_t kb = ks >> 2, kin = (ks & 3) * 32;
        mma_bf16_tc(tmem + kHid, sw128_desc(a_addr + kb * 16384 + kin),
                    sw128_desc(base_addr + kOffP + kb * 2048 + kin), id_p, ks > 0);
      }
      mma_commit(mbar);
    }
    if (!wait_mma()) break;
    uint32_t v[16];
    tmem_ld16(t_row + kHid, v);
    if (valid) {
      float* out = reinterpret_cast<float*>(fi.xf) + 12 * (size_t)(fi.out_first + k_item);
      const float* pc = s_misc;
      const float* A3 = s_misc + 3;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float y = (__uint_as_float(v[c]) + __uint_as_float(v[3 + c])) + __uint_as_float(v[6 + c]);
        if (s_st == 0)
          out[c] = y + pc[c] + (A3[3 * c] * xr[0] + A3[3 * c + 1] * xr[1] + A3[3 * c + 2] * xr[2]);
        else
          out[3 + 3 * (s_st - 1) + c] = y + A3[3 * c + (s_st - 1)];
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
                 "r"(kTcCols * kTcWG));
  }
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
  const uint32_t tiles = (fi.count + 31) / 32;
  const uint32_t blocks = std::min<uint32_t>(148u, (tiles + kTcWG - 1) / kTcWG);
  if (fi.codes)
    k_field_infer_tc<true><<<blocks, kTcWG * 128, kTcSmem, s>>>(fi);
  else
    k_field_infer_tc<false><<<blocks, kTcWG * 128, kTcSmem, s>>>(fi);
  return cudaGetLastError();
}

}  // namespace cgs
