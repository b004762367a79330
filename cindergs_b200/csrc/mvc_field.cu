// Learned MVC weight field on sm_100a: a Fourier-feature encoding feeding a
// 4 x 128 SiLU MLP with BF16 weights and activations and FP32 accumulation on
// the tensor cores, whose V outputs are made a partition of unity by adding
// (1 - sum z) / V to each. It stands in for the exact mean value coordinates
// (deformation/mvc.rs:366-471) of the Gaussians it reproduces well enough.
//
// The partition-of-unity weights w0 are then projected onto the weights that
// also reproduce linear functions (sum_j w_j v_j = x on the rest cage), the
// two properties exact MVC has: w = w0 - Vb^T M (Vb w0 - [1; x]) with
// Vb = [1; rest vertices] (4 x V) and M = (Vb Vb^T)^-1, so affine cage
// motions are reproduced exactly and the network only carries the rest. The
// linear-precision residual r = sum_j w0_j v_j - x of the network's own
// weights decides which Gaussians fall back to exact MVC.
//
// Training (forward, backward, Adam) runs as separate kernels over batches of
// points with exact weights (mma.sync GEMMs: small, latency-bound shapes);
// inference for the frame is one fused tcgen05 kernel (mvc_field_tc.cu) that
// evaluates the network and its forward-mode Jacobian per Gaussian and emits
// the deformed position and deformation gradient in the layout of the exact
// path (k_mvc_jacobian), or keeps the last hidden layer as the Gaussian's
// code for k_field_apply. The weights enter the position linearly, so with
// A = v'^T Vb^T M (3 x 4, v' the current vertices) and A3 its last three
// columns, x' = sum_j w_j v'_j = v'^T w0 - A3 r = Pc^T h + pc + A3 x, where
// Pc (128 x 3), pc and A3 are formed once per frame from the output layer
// and the current and rest vertices; F = Pc^T dh/dx + A3.
//
// Network layout (row-major, out x in): W1 [128 x 64], W2..W4 [128 x 128],
// W5 [V x 128]; biases b1..b4 [128], b5 [V]. Features of x^ = (x - c) / s
// (c, s: centre and half of the largest extent of the rest cage): x^ (3), then
// sin and cos of w_b x^_d for bands b = 0..7 (w_b = 2^b pi / 2) and axes d,
// zero-padded to 64. Layer inputs (features, activations, tangents) are
// rounded to bf16 in training and inference alike.
#include <cuda_bf16.h>

#include <algorithm>

#include "field.h"
#include "kernels.h"

namespace cgs {
namespace {

constexpr int kIn = kFieldIn;    // 64 features
constexpr int kHid = kFieldHid;  // 128

__device__ __forceinline__ float sigmoid_fast(float x) { return 1.0f / (1.0f + __expf(-x)); }
__device__ __forceinline__ float silu_grad(float x) {
  const float s = sigmoid_fast(x);
  return s * (1.0f + x * (1.0f - s));
}

// Feature j of x^ (value) and its derivatives with respect to x (chain factor
// 1/s), for j in [0, 64).
__device__ __forceinline__ void feature(int j, const float* xh, float inv_s, float& f,
                                        float (&df)[3]) {
  f = 0.0f;
  df[0] = df[1] = df[2] = 0.0f;
  if (j < 3) {
    f = xh[j];
    df[j] = inv_s;
  } else if (j < 3 + 6 * kFieldBands) {
    const int q = j - 3, b = q / 6, d = (q % 6) >> 1;
    const float w = (float)(1 << b) * 1.57079632679489662f;
    float sn, cs;
    sincosf(w * xh[d], &sn, &cs);
    if ((q & 1) == 0) {
      f = sn;
      df[d] = w * cs * inv_s;
    } else {
      f = cs;
      df[d] = -w * sn * inv_s;
    }
  }
}

// ---- training kernels --------------------------------------------------------

__device__ __forceinline__ uint32_t mix32(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return (uint32_t)((z ^ (z >> 31)) >> 32);
}

// Batch gather and features: row r uses point idx = mix(seed, r) % n (or r
// when seed is 0); writes x [B*3], target weights [B x ldw] and features
// A0 [B x 64] (bf16).
__global__ void k_field_gather(FieldBatch fb) {
  const uint32_t r = blockIdx.x;
  if (r >= fb.B) return;
  const uint32_t idx = fb.seed ? mix32(((uint64_t)fb.seed << 32) | r) % fb.n : r % fb.n;
  __shared__ float xh[3];
  if (threadIdx.x < 3) {
    const float x = fb.points[3 * (size_t)idx + threadIdx.x];
    fb.x[3 * (size_t)r + threadIdx.x] = x;
    xh[threadIdx.x] = (x - fb.enc[threadIdx.x]) * fb.enc[3];
  }
  __syncthreads();
  if (fb.target)
    for (uint32_t j = threadIdx.x; j < fb.V; j += blockDim.x)
      fb.wt[(size_t)r * fb.ldw + j] = fb.target[(size_t)idx * fb.V + j];
  for (int j = threadIdx.x; j < kIn; j += blockDim.x) {
    float f, df[3];
    feature(j, xh, fb.enc[3], f, df);
    fb.a0[(size_t)r * kIn + j] = __float2bfloat16_rn(f);
  }
}

// out [C x R] bf16 = transpose of in [R x C] (fp32 or bf16).
template <typename T>
__global__ void k_transpose(const T* __restrict__ in, uint32_t R, uint32_t C, uint32_t ldi,
                            __nv_bfloat16* __restrict__ out, uint32_t ldo) {
  __shared__ float tile[32][33];
  const uint32_t c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const uint32_t r = r0 + k, c = c0 + threadIdx.x;
    tile[k][threadIdx.x] = (r < R && c < C) ? (float)in[(size_t)r * ldi + c] : 0.0f;
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const uint32_t c = c0 + k, r = r0 + threadIdx.x;
    if (c < C && r < R) out[(size_t)c * ldo + r] = __float2bfloat16_rn(tile[threadIdx.x][k]);
  }
}

// Sums of K values over the block (blockDim.x a multiple of 32, at most 1024);
// every thread gets the totals. red holds K x 32 floats.
template <int K>
__device__ __forceinline__ void block_sums(float (&v)[K], float* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < K; ++k) red[k * 32 + warp] = v[k];
  __syncthreads();
#pragma unroll
  for (int k = 0; k < K; ++k) {
    float t = 0.0f;
    for (int w = 0; w < nw; ++w) t += red[k * 32 + w];
    v[k] = t;
  }
}

// u = M[:, 1:4] r: the correction of the weights is u0 + v_j . (u1, u2, u3).
__device__ __forceinline__ void lp_correction(const float* M, const float (&r)[3], float (&u)[4]) {
#pragma unroll
  for (int a = 0; a < 4; ++a) u[a] = M[4 * a + 1] * r[0] + M[4 * a + 2] * r[1] + M[4 * a + 3] * r[2];
}

// Loss and dL/dz per batch row. w0 = z + (1 - sum z) / V; r = sum_j w0_j v_j
// - x; w = w0 - Vb^T M (Vb w0 - [1; x]) (Vb w0 = [1; x + r]). L = (1/B)
// sum_b sum_j (w - w*)^2 + lambda (1/B) sum_b |r|^2 / (3 s^2). dL/dw0 = Pi g
// + (2 lambda / (3 B s^2)) (r . v_j) with g = 2 (w - w*) / B and the
// projector Pi = I - Vb^T M Vb; dz = dL/dw0 - mean (the sum in w0). dz is
// written in fp32 and bf16; the loss terms (residual without lambda) are
// added to loss[0..1].
__global__ void k_field_loss(FieldLoss fl) {
  const uint32_t row = blockIdx.x;
  if (row >= fl.B) return;
  __shared__ float red[6 * 32];
  const float* z = fl.z + (size_t)row * fl.ldz;
  const float* wt = fl.wt + (size_t)row * fl.ldw;
  const float* x = fl.x + 3 * (size_t)row;
  float s1[1] = {0.0f};
  for (uint32_t j = threadIdx.x; j < fl.V; j += blockDim.x) s1[0] += z[j];
  block_sums<1>(s1, red);
  const float add = (1.0f - s1[0]) / (float)fl.V;
  float s3[3] = {0.0f, 0.0f, 0.0f};
  for (uint32_t j = threadIdx.x; j < fl.V; j += blockDim.x) {
    const float w0 = z[j] + add;
    const float4 v = fl.verts[j];
    s3[0] += w0 * v.x;
    s3[1] += w0 * v.y;
    s3[2] += w0 * v.z;
  }
  block_sums<3>(s3, red);
  const float r[3] = {s3[0] - x[0], s3[1] - x[1], s3[2] - x[2]};
  float u[4];
  lp_correction(fl.M, r, u);
  const float inv_b = 1.0f / (float)fl.B;
  // pass: squared error of w and Vb g (g = 2 e / B)
  float s5[5] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
  for (uint32_t j = threadIdx.x; j < fl.V; j += blockDim.x) {
    const float4 v = fl.verts[j];
    const float w = z[j] + add - (u[0] + (v.x * u[1] + v.y * u[2] + v.z * u[3]));
    const float e = w - wt[j];
    const float g = 2.0f * e * inv_b;
    s5[0] += e * e;
    s5[1] += g;
    s5[2] += g * v.x;
    s5[3] += g * v.y;
    s5[4] += g * v.z;
  }
  block_sums<5>(s5, red);
  float q[4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
    q[a] = fl.M[4 * a] * s5[1] + fl.M[4 * a + 1] * s5[2] + fl.M[4 * a + 2] * s5[3] +
           fl.M[4 * a + 3] * s5[4];
  const float cres = fl.lambda * 2.0f / (3.0f * (float)fl.B * fl.s2);
  auto grad_w0 = [&](uint32_t j) {
    const float4 v = fl.verts[j];
    const float w = z[j] + add - (u[0] + (v.x * u[1] + v.y * u[2] + v.z * u[3]));
    const float g = 2.0f * (w - wt[j]) * inv_b;
    return g - (q[0] + (v.x * q[1] + v.y * q[2] + v.z * q[3])) +
           cres * ((r[0] * v.x + r[1] * v.y) + r[2] * v.z);
  };
  float sg[1] = {0.0f};
  for (uint32_t j = threadIdx.x; j < fl.V; j += blockDim.x) sg[0] += grad_w0(j);
  block_sums<1>(sg, red);
  const float gmean = sg[0] / (float)fl.V;
  for (uint32_t j = threadIdx.x; j < fl.V; j += blockDim.x) {
    const float dz = grad_w0(j) - gmean;
    fl.dz[(size_t)row * fl.ldz + j] = dz;
    fl.dzb[(size_t)row * fl.ldz + j] = __float2bfloat16_rn(dz);
  }
  if (threadIdx.x == 0) {
    atomicAdd(&fl.loss[0], s5[0] * inv_b);
    atomicAdd(&fl.loss[1], ((r[0] * r[0] + r[1] * r[1]) + r[2] * r[2]) /
                               (3.0f * (float)fl.B * fl.s2));
  }
}

// dpre = dA * silu'(pre) (fp32 and bf16 copies), elementwise.
__global__ void k_silu_back(uint32_t n, const float* __restrict__ da,
                            const float* __restrict__ pre, float* __restrict__ dpre,
                            __nv_bfloat16* __restrict__ dpreb) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float v = da[i] * silu_grad(pre[i]);
  dpre[i] = v;
  dpreb[i] = __float2bfloat16_rn(v);
}

// Column sums of g [B x ld] over rows -> out [N] (bias gradients).
__global__ void k_colsum(const float* __restrict__ g, uint32_t B, uint32_t N, uint32_t ld,
                         float* __restrict__ out) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= N) return;
  float s = 0.0f;
  for (uint32_t r = 0; r < B; ++r) s += g[(size_t)r * ld + c];
  out[c] = s;
}

// Adam (Kingma & Ba 2015) on fp32 master weights, refreshing the bf16 copy:
// m = b1 m + (1-b1) g; v = b2 v + (1-b2) g^2; p -= lr mh / (sqrt(vh) + eps)
// with the bias corrections mh = m c1, vh = v c2.
__global__ void k_adam(uint32_t n, float* __restrict__ p, const float* __restrict__ g,
                       float* __restrict__ m, float* __restrict__ v,
                       __nv_bfloat16* __restrict__ pb, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.0f - b1) * gi;
  const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float pi = p[i] - lr * (mi * c1) / (sqrtf(vi * c2) + eps);
  p[i] = pi;
  if (pb) pb[i] = __float2bfloat16_rn(pi);
}

// ---- frame: per-frame projection and fused inference ---------------------------

// Per-frame projection of the output layer (one block of 1024 threads). For
// vertices u (rest or current), P_u[k] = sum_j W5[j][k] u_j - c_k ubar with
// c_k = sum_j W5[j][k], and p0_u = sum_j b5_j u_j + (1 - sum_j b5_j) ubar, so
// that sum_j w0_j u_j = P_u^T h + p0_u. Raw mode (verts == null): P_rest,
// p0_rest and A3 = 0, i.e. the network's own rest position sum_j w0_j v_j.
// Otherwise A = v'^T Vb^T M, Pc = P_cur - P_rest A3^T, pc = p0_cur - A3 p0_rest.
// proj = [Pc (128 x 3) | pc (3) | A3 (3 x 3, row-major)]. Both vertex sets
// are staged in shared memory; thread (g, k) sums vertices j = g mod 8 for
// hidden unit k and the eight partial sums are added in g order.
constexpr int kProjThreads = 1024, kProjGroups = kProjThreads / kHid;
__global__ void __launch_bounds__(kProjThreads) k_field_project(FieldNet net, uint32_t V,
                                                                const float4* __restrict__ rest,
                                                                const float4* __restrict__ verts,
                                                                const float* __restrict__ M,
                                                                float* __restrict__ proj) {
  extern __shared__ float4 pv[];  // [V] rest, [V] current
  __shared__ float red[22 * 32];
  __shared__ float part[kProjGroups][7][kHid];
  __shared__ float sh[20];
  const bool raw = verts == nullptr;
  for (uint32_t j = threadIdx.x; j < V; j += blockDim.x) {
    pv[j] = rest[j];
    pv[V + j] = raw ? make_float4(0.f, 0.f, 0.f, 0.f) : verts[j];
  }
  __syncthreads();
  // sums: rest (3), rest . b5 (3), sum b5 (1), current (3), current . b5 (3),
  // sum_j v'_j v_j^T (9)
  float t[22];
#pragma unroll
  for (int k = 0; k < 22; ++k) t[k] = 0.0f;
  for (uint32_t j = threadIdx.x; j < V; j += blockDim.x) {
    const float4 v = pv[j], c = pv[V + j];
    const float b = net.b5[j];
    t[0] += v.x; t[1] += v.y; t[2] += v.z;
    t[3] += b * v.x; t[4] += b * v.y; t[5] += b * v.z;
    t[6] += b;
    t[7] += c.x; t[8] += c.y; t[9] += c.z;
    t[10] += b * c.x; t[11] += b * c.y; t[12] += b * c.z;
    t[13] += c.x * v.x; t[14] += c.x * v.y; t[15] += c.x * v.z;
    t[16] += c.y * v.x; t[17] += c.y * v.y; t[18] += c.y * v.z;
    t[19] += c.z * v.x; t[20] += c.z * v.y; t[21] += c.z * v.z;
  }
  block_sums<22>(t, red);
  if (threadIdx.x == 0) {
    const float inv_v = 1.0f / (float)V;
    const float rb[3] = {t[0] * inv_v, t[1] * inv_v, t[2] * inv_v};
    float p0r[3];
    for (int q = 0; q < 3; ++q) p0r[q] = t[3 + q] + (1.0f - t[6]) * rb[q];
    for (int q = 0; q < 3; ++q) {
      sh[q] = rb[q];
      sh[3 + q] = p0r[q];
    }
    if (raw) {
      for (int q = 0; q < 3; ++q) proj[3 * kHid + q] = p0r[q];
      for (int k = 0; k < 9; ++k) proj[3 * kHid + 3 + k] = 0.0f;
    } else {
      const float cb[3] = {t[7] * inv_v, t[8] * inv_v, t[9] * inv_v};
      // S (3 x 4): column 0 = sum_j v'_j, columns 1..3 = sum_j v'_j v_j^T
      const float S[3][4] = {{t[7], t[13], t[14], t[15]},
                             {t[8], t[16], t[17], t[18]},
                             {t[9], t[19], t[20], t[21]}};
      float A3[3][3];
      for (int q = 0; q < 3; ++q)
        for (int d = 0; d < 3; ++d) {
          float acc = 0.0f;
          for (int k = 0; k < 4; ++k) acc += S[q][k] * M[4 * k + 1 + d];
          A3[q][d] = acc;
          sh[11 + 3 * q + d] = acc;
        }
      for (int q = 0; q < 3; ++q) {
        sh[6 + q] = cb[q];
        const float p0c = t[10 + q] + (1.0f - t[6]) * cb[q];
        proj[3 * kHid + q] =
            p0c - (A3[q][0] * p0r[0] + A3[q][1] * p0r[1] + A3[q][2] * p0r[2]);
        for (int d = 0; d < 3; ++d) proj[3 * kHid + 3 + 3 * q + d] = A3[q][d];
      }
    }
  }
  const uint32_t k = threadIdx.x % kHid, g = threadIdx.x / kHid;
  float acc[7] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};  // rest (3), current (3), c
  for (uint32_t j = g; j < V; j += kProjGroups) {
    const float w = __bfloat162float(net.W5b[(size_t)j * kHid + k]);
    const float4 v = pv[j], u = pv[V + j];
    acc[0] += w * v.x; acc[1] += w * v.y; acc[2] += w * v.z;
    acc[3] += w * u.x; acc[4] += w * u.y; acc[5] += w * u.z;
    acc[6] += w;
  }
#pragma unroll
  for (int q = 0; q < 7; ++q) part[g][q][k] = acc[q];
  __syncthreads();  // also publishes sh
  if (g != 0) return;
#pragma unroll
  for (int q = 0; q < 7; ++q) {
    float tot = 0.0f;
    for (int gg = 0; gg < kProjGroups; ++gg) tot += part[gg][q][k];
    acc[q] = tot;
  }
  float pr[3];
  for (int q = 0; q < 3; ++q) pr[q] = acc[q] - acc[6] * sh[q];
  if (raw) {
    for (int q = 0; q < 3; ++q) proj[3 * k + q] = pr[q];
  } else {
    for (int q = 0; q < 3; ++q) {
      const float pc = acc[3 + q] - acc[6] * sh[6 + q];
      proj[3 * k + q] = pc - (sh[11 + 3 * q] * pr[0] + sh[12 + 3 * q] * pr[1] +
                              sh[13 + 3 * q] * pr[2]);
    }
  }
}

// Final weights per row: w0 = z + (1 - sum z) / V, then the linear-precision
// projection w = w0 - (u0 + v_j . u[1..3]), u = M[:, 1:4] (sum_j w0_j v_j - x).
__global__ void k_field_weights(const float* __restrict__ z, uint32_t B, uint32_t V,
                                uint32_t ldz, const float* __restrict__ x,
                                const float4* __restrict__ verts, FieldMat M,
                                float* __restrict__ w) {
  const uint32_t row = blockIdx.x;
  if (row >= B) return;
  __shared__ float red[3 * 32];
  const float* zr = z + (size_t)row * ldz;
  float s1[1] = {0.0f};
  for (uint32_t j = threadIdx.x; j < V; j += blockDim.x) s1[0] += zr[j];
  block_sums<1>(s1, red);
  const float add = (1.0f - s1[0]) / (float)V;
  float s3[3] = {0.0f, 0.0f, 0.0f};
  for (uint32_t j = threadIdx.x; j < V; j += blockDim.x) {
    const float w0 = zr[j] + add;
    const float4 v = verts[j];
    s3[0] += w0 * v.x;
    s3[1] += w0 * v.y;
    s3[2] += w0 * v.z;
  }
  block_sums<3>(s3, red);
  const float* xr = x + 3 * (size_t)row;
  const float r[3] = {s3[0] - xr[0], s3[1] - xr[1], s3[2] - xr[2]};
  float u[4];
  lp_correction(M.m, r, u);
  for (uint32_t j = threadIdx.x; j < V; j += blockDim.x) {
    const float4 v = verts[j];
    w[(size_t)row * V + j] = zr[j] + add - (u[0] + (v.x * u[1] + v.y * u[2] + v.z * u[3]));
  }
}

// Linear-precision residual of the learned position on the rest cage.
__global__ void k_mvc_residual(uint32_t nb, const uint32_t* __restrict__ list,
                               const float4* __restrict__ rest_pos,
                               const float4* __restrict__ xf, float inv_scale, float threshold,
                               float* __restrict__ resid, uint32_t* __restrict__ flag) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nb) return;
  const float4 x = rest_pos[list[s]];
  const float4 y = xf[3 * (size_t)s];
  const float dx = y.x - x.x, dy = y.y - x.y, dz = y.z - x.z;
  const float r = sqrtf(dx * dx + dy * dy + dz * dz) * inv_scale;
  if (resid) resid[s] = r;
  flag[s] = (r > threshold || !(r == r)) ? 1u : 0u;
}

// Slots renumbered so the exact fallbacks come first (in slot order), then
// the learned ones: rank = exclusive scan of the fallback flags.
__global__ void k_mvc_reslot(uint32_t nb, const uint32_t* __restrict__ flag,
                             const uint32_t* __restrict__ rank, uint32_t nfb,
                             const uint32_t* __restrict__ list_in, uint32_t* __restrict__ list_out,
                             float4* __restrict__ bind_w) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nb) return;
  const uint32_t i = list_in[s];
  const uint32_t slot = flag[s] ? rank[s] : nfb + (s - rank[s]);
  list_out[slot] = i;
  bind_w[i] = make_float4(__uint_as_float(slot), 0.0f, 0.0f, 0.0f);
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const uint32_t a = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(a), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Per-frame output layer over cached codes (k_field_infer<true>) on the
// tensor cores. An item's code is four rows (h and its three tangents) of
// 128 bf16; x' and F are those rows times P (128 x 3) plus the affine terms,
// so four items make one 16-row MMA tile. Each warp owns a contiguous range
// of items and streams it through a kApStages-deep ring of 4-item stages
// with cp.async; the 16-byte chunks are placed with an XOR swizzle (chunk j
// of row r at j ^ (r % 8)) so that the ldmatrix reads are free of bank
// conflicts. Each stage is multiplied by P with mma.sync m16n8k16 (bf16 in,
// fp32 accumulate). P is split into three bf16 terms (hi + mid + lo, column
// n = 4 c + t of B holds term t of P[:, c]) held as B fragments in
// registers, so each output equals an fp32 dot product to within a few ulp.
// The kernel is bound by HBM (1,040 bytes per item); the MMAs replace the
// per-lane multiply-adds (48 per lane and item) that bounded a scalar form.
// Outputs go out in k_mvc_jacobian's layout: position, then F column-major.
constexpr int kApStages = 6, kApWarps = 8, kApItems = 4;
constexpr int kApCodeBytes = kApItems * 4 * kHid * 2;       // 4,096
constexpr int kApStageBytes = kApCodeBytes + kApItems * 16;  // + rest positions

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
  const uint32_t l = __bfloat16_as_ushort(__float2bfloat16_rn(lo));
  const uint32_t h = __bfloat16_as_ushort(__float2bfloat16_rn(hi));
  return l | (h << 16);
}
// term t (0 hi, 1 mid, 2 lo) of the three-term bf16 split of v
__device__ __forceinline__ float bf16_term(float v, int t) {
  const float hi = __bfloat162float(__float2bfloat16_rn(v));
  if (t == 0) return hi;
  const float mid = __bfloat162float(__float2bfloat16_rn(v - hi));
  if (t == 1) return mid;
  return v - hi - mid;  // rounded to bf16 when packed
}

__global__ void __launch_bounds__(kApWarps * 32, 1) k_field_apply(FieldInfer fi) {
  extern __shared__ __align__(128) unsigned char ap_smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, q = lane & 3;
  unsigned char* ring = ap_smem + (size_t)warp * kApStages * kApStageBytes;
  // B fragments of the split P: k = 16 kk + 2 q (+1) and + 8, n = 8 nt + g
  uint32_t bfr[8][2][2];
#pragma unroll
  for (int kk = 0; kk < 8; ++kk)
#pragma unroll
    for (int nt = 0; nt < 2; ++nt) {
      const int n = 8 * nt + g, c = n >> 2, t = n & 3;
#pragma unroll
      for (int r = 0; r < 2; ++r) {
        const int k = 16 * kk + 2 * q + 8 * r;
        float v0 = 0.0f, v1 = 0.0f;
        if (c < 3 && t < 3) {
          v0 = bf16_term(fi.proj[3 * k + c], t);
          v1 = bf16_term(fi.proj[3 * (k + 1) + c], t);
        }
        bfr[kk][nt][r] = pack_bf16x2(v0, v1);
      }
    }
  const float* pc = fi.proj + 3 * kHid;
  const float* A3 = pc + 3;
  const uint32_t gw = blockIdx.x * kApWarps + warp, nw = gridDim.x * kApWarps;
  const uint32_t per = (fi.count + nw - 1) / nw;
  const uint32_t i0 = min(fi.count, gw * per), i1 = min(fi.count, i0 + per);
  const uint32_t nstages = (i1 - i0 + kApItems - 1) / kApItems;
  const unsigned char* codes = reinterpret_cast<const unsigned char*>(fi.codes);
  auto issue = [&](uint32_t sidx) {
    const uint32_t it = i0 + kApItems * sidx;
    unsigned char* st = ring + (sidx % kApStages) * kApStageBytes;
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const uint32_t ch = lane + 32 * u;  // 16-byte chunk of the stage's 4 KB
      if (it + (ch >> 6) < i1) {
        const uint32_t r = ch >> 4, j = ch & 15;
        cp_async16(st + r * 256 + ((j ^ (r & 7)) << 4), codes + (size_t)it * 1024 + ch * 16);
      }
    }
    if (lane < kApItems && it + lane < i1) cp_async16(st + kApCodeBytes + 16 * lane, fi.code_pos + it + lane);
    cp_async_commit();
  };
#pragma unroll
  for (int k = 0; k < kApStages - 1; ++k) issue(k);
  for (uint32_t sidx = 0; sidx < nstages; ++sidx) {
    issue(sidx + kApStages - 1);
    cp_async_wait<kApStages - 1>();
    __syncwarp();
    const unsigned char* st = ring + (sidx % kApStages) * kApStageBytes;
    float d[2][4] = {{0.0f, 0.0f, 0.0f, 0.0f}, {0.0f, 0.0f, 0.0f, 0.0f}};
    const int mrow = (lane & 7) + ((lane >> 3) & 1) * 8;  // row this lane addresses
#pragma unroll
    for (int kk = 0; kk < 8; ++kk) {
      const int j = 2 * kk + (lane >> 4);
      const uint32_t addr =
          (uint32_t)__cvta_generic_to_shared(st + mrow * 256 + ((j ^ (mrow & 7)) << 4));
      uint32_t a0, a1, a2, a3;
      asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                   : "=r"(a0), "=r"(a1), "=r"(a2), "=r"(a3)
                   : "r"(addr));
#pragma unroll
      for (int nt = 0; nt < 2; ++nt)
        asm volatile(
            "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
            "{%8,%9}, {%0,%1,%2,%3};\n"
            : "+f"(d[nt][0]), "+f"(d[nt][1]), "+f"(d[nt][2]), "+f"(d[nt][3])
            : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(bfr[kk][nt][0]), "r"(bfr[kk][nt][1]));
    }
    // rows g and g + 8 = (item, stream); sum the terms of each output column
    const uint32_t it = i0 + kApItems * sidx;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      float s0 = d[0][2 * h] + d[0][2 * h + 1];  // c = q / 2
      float s1 = d[1][2 * h] + d[1][2 * h + 1];  // c = 2 (q < 2)
      s0 += __shfl_xor_sync(0xffffffffu, s0, 1);
      s1 += __shfl_xor_sync(0xffffffffu, s1, 1);
      const int row = g + 8 * h, item = row >> 2, stream = row & 3;
      if ((q & 1) || it + item >= i1) continue;
      const float4 x = *reinterpret_cast<const float4*>(st + kApCodeBytes + 16 * item);
      float* out = reinterpret_cast<float*>(fi.xf) + 12 * (size_t)(fi.out_first + it + item);
#pragma unroll
      for (int w = 0; w < 2; ++w) {
        if (w == 1 && q != 0) break;
        const int c = w == 0 ? (q >> 1) : 2;
        const float t = w == 0 ? s0 : s1;
        if (stream == 0)
          out[c] = (t + pc[c]) + (A3[3 * c] * x.x + A3[3 * c + 1] * x.y + A3[3 * c + 2] * x.z);
        else
          out[3 + 3 * (stream - 1) + c] = t + A3[3 * c + stream - 1];
      }
    }
    __syncwarp();  // every lane has read this stage before it is refilled
  }
  cp_async_wait<0>();
}

}  // namespace

cudaError_t launch_field_gather(const FieldBatch& b, cudaStream_t s) {
  if (b.B == 0) return cudaSuccess;
  k_field_gather<<<b.B, 128, 0, s>>>(b);
  return cudaGetLastError();
}

cudaError_t launch_transpose_f32(const float* in, uint32_t R, uint32_t C, uint32_t ldi,
                                 __nv_bfloat16* out, uint32_t ldo, cudaStream_t s) {
  if (R == 0 || C == 0) return cudaSuccess;
  k_transpose<float><<<dim3((C + 31) / 32, (R + 31) / 32), dim3(32, 8), 0, s>>>(in, R, C, ldi, out,
                                                                                ldo);
  return cudaGetLastError();
}

cudaError_t launch_transpose_bf16(const __nv_bfloat16* in, uint32_t R, uint32_t C, uint32_t ldi,
                                  __nv_bfloat16* out, uint32_t ldo, cudaStream_t s) {
  if (R == 0 || C == 0) return cudaSuccess;
  k_transpose<__nv_bfloat16><<<dim3((C + 31) / 32, (R + 31) / 32), dim3(32, 8), 0, s>>>(
      in, R, C, ldi, out, ldo);
  return cudaGetLastError();
}

cudaError_t launch_field_loss(const FieldLoss& l, cudaStream_t s) {
  if (l.B == 0) return cudaSuccess;
  k_field_loss<<<l.B, 128, 0, s>>>(l);
  return cudaGetLastError();
}

cudaError_t launch_silu_back(uint32_t n, const float* da, const float* pre, float* dpre,
                             __nv_bfloat16* dpreb, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  k_silu_back<<<(n + 255) / 256, 256, 0, s>>>(n, da, pre, dpre, dpreb);
  return cudaGetLastError();
}

cudaError_t launch_colsum(const float* g, uint32_t B, uint32_t N, uint32_t ld, float* out,
                          cudaStream_t s) {
  if (N == 0) return cudaSuccess;
  k_colsum<<<(N + 127) / 128, 128, 0, s>>>(g, B, N, ld, out);
  return cudaGetLastError();
}

cudaError_t launch_adam(uint32_t n, float* p, const float* g, float* m, float* v,
                        __nv_bfloat16* pb, float lr, float b1, float b2, float eps, float c1,
                        float c2, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  k_adam<<<(n + 255) / 256, 256, 0, s>>>(n, p, g, m, v, pb, lr, b1, b2, eps, c1, c2);
  return cudaGetLastError();
}

cudaError_t launch_field_project(const FieldNet& net, uint32_t V, const float4* rest,
                                 const float4* verts, const float* M, float* proj,
                                 cudaStream_t s) {
  // static shared memory (~32 KB) plus the two vertex sets
  const size_t smem = (size_t)V * 32;
  const cudaError_t e = cudaFuncSetAttribute(
      k_field_project, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k_field_project<<<1, kProjThreads, smem, s>>>(net, V, rest, verts, M, proj);
  return cudaGetLastError();
}

cudaError_t launch_field_infer(const FieldInfer& fi, cudaStream_t s) {
  return launch_field_infer_tc(fi, s);
}

cudaError_t launch_field_apply(const FieldInfer& fi, cudaStream_t s) {
  if (fi.count == 0) return cudaSuccess;
  if (!fi.codes || !fi.code_pos) return cudaErrorInvalidValue;
  const size_t smem = (size_t)kApWarps * kApStages * kApStageBytes;
  const cudaError_t e =
      cudaFuncSetAttribute(k_field_apply, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  // one block of eight warps per SM (the rings take 195 KB)
  const uint32_t blocks = std::min<uint32_t>(148u, (fi.count + kApWarps * kApItems - 1) / (kApWarps * kApItems));
  k_field_apply<<<blocks, kApWarps * 32, smem, s>>>(fi);
  return cudaGetLastError();
}

cudaError_t launch_field_weights(const float* z, uint32_t B, uint32_t V, uint32_t ldz,
                                 const float* x, const float4* verts, const FieldMat& M, float* w,
                                 cudaStream_t s) {
  if (B == 0) return cudaSuccess;
  k_field_weights<<<B, 128, 0, s>>>(z, B, V, ldz, x, verts, M, w);
  return cudaGetLastError();
}

cudaError_t launch_mvc_residual(uint32_t nb, const uint32_t* list, const float4* rest_pos,
                                const float4* xf, float inv_scale, float threshold, float* resid,
                                uint32_t* flag, cudaStream_t s) {
  if (nb == 0) return cudaSuccess;
  k_mvc_residual<<<(nb + 255) / 256, 256, 0, s>>>(nb, list, rest_pos, xf, inv_scale, threshold,
                                                  resid, flag);
  return cudaGetLastError();
}

cudaError_t launch_mvc_reslot(uint32_t nb, const uint32_t* flag, const uint32_t* rank,
                              uint32_t nfb, const uint32_t* list_in, uint32_t* list_out,
                              float4* bind_w, cudaStream_t s) {
  if (nb == 0) return cudaSuccess;
  k_mvc_reslot<<<(nb + 255) / 256, 256, 0, s>>>(nb, flag, rank, nfb, list_in, list_out, bind_w);
  return cudaGetLastError();
}

}  // namespace cgs
