// Mean value coordinates on sm_100a: exact 3D MVC weights for a closed
// triangle cage, the inside test, the binding of Gaussians (weights plus
// central-difference gradients) and the per-frame deformed position and
// deformation gradient from stored bindings.
//
// Reference semantics: PolyCageMesh::winding_number, compute_mvc_weights,
// jacobian_step_size, bind_gaussians, MvcBindings::local_jacobian and
// evaluate_position (deformation/mvc.rs:339-541, 58-78). Compiled with
// -fmad=false: products and sums are rounded one by one in the reference's
// (glam 0.28) operand order; per cage vertex the face contributions are added
// in ascending face order and the normaliser face by face, as the reference's
// sequential loop does, so only the transcendentals (asin, sin, atan2) can
// differ from the host restatement in their last bits.
#include <algorithm>

#include "kernels.h"

namespace cgs {
namespace {

constexpr int kMvcThreads = 128;
constexpr uint32_t kNone = 0xFFFFFFFFu;

struct F3 {
  float x, y, z;
};
__device__ __forceinline__ F3 f3(float4 v) { return {v.x, v.y, v.z}; }
__device__ __forceinline__ F3 sub(F3 a, F3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ float dot(F3 a, F3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
__device__ __forceinline__ float len(F3 a) { return sqrtf(dot(a, a)); }
__device__ __forceinline__ F3 cross(F3 a, F3 b) {
  return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
__device__ __forceinline__ float clampf1(float x, float lo, float hi) {
  return fminf(fmaxf(x, lo), hi);
}

// Shared memory of one evaluation: per vertex (unit direction, distance), per
// face (three contributions, kind: 0 regular or skipped, 1 boundary face).
struct EvalSmem {
  float4* dir;    // [V]
  float4* mu;     // [F]
  uint32_t* hit;  // [2]: first vertex within 1e-6, first boundary face
  float* total;   // [2]: normaliser, nearest vertex (as float bits)
};

// compute_mvc_weights (mvc.rs:366-471) at x: every thread of the block takes
// part; thread t returns in w[k] the weight of vertex t + k * blockDim.
template <int OWN>
__device__ __forceinline__ void mvc_eval(const MvcCage& c, F3 x, const EvalSmem& s, float (&w)[OWN]) {
  const int tid = threadIdx.x;
  if (tid == 0) {
    s.hit[0] = kNone;
    s.hit[1] = kNone;
  }
  __syncthreads();
  for (uint32_t j = tid; j < c.V; j += blockDim.x) {
    const F3 diff = sub(f3(c.verts[j]), x);
    const float d = len(diff);
    s.dir[j] = make_float4(diff.x / d, diff.y / d, diff.z / d, d);
    if (d < 1e-6f) atomicMin(&s.hit[0], j);
  }
  __syncthreads();
  const uint32_t vhit = s.hit[0];
  if (vhit == kNone) {
    const float PI_F = 3.14159265358979323846f;
    for (uint32_t f = tid; f < c.F; f += blockDim.x) {
      const uint4 t = c.tris[f];
      const float4 a0 = s.dir[t.x], a1 = s.dir[t.y], a2 = s.dir[t.z];
      const F3 u0 = f3(a0), u1 = f3(a1), u2 = f3(a2);
      const float d0 = a0.w, d1 = a1.w, d2 = a2.w;
      const float l0 = len(sub(u1, u2)), l1 = len(sub(u2, u0)), l2 = len(sub(u0, u1));
      const float t0 = 2.0f * asinf(clampf1(l0 * 0.5f, 0.0f, 1.0f));
      const float t1 = 2.0f * asinf(clampf1(l1 * 0.5f, 0.0f, 1.0f));
      const float t2 = 2.0f * asinf(clampf1(l2 * 0.5f, 0.0f, 1.0f));
      const float h = 0.5f * ((t0 + t1) + t2);
      float4 m = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      if (fabsf(PI_F - h) < 1e-5f) {
        // the point lies on this face (mvc.rs:396-408)
        m = make_float4(sinf(t0) * d1 * d2, sinf(t1) * d2 * d0, sinf(t2) * d0 * d1, 1.0f);
        atomicMin(&s.hit[1], f);
      } else {
        const float st0 = sinf(t0), st1 = sinf(t1), st2 = sinf(t2);
        if (!(fabsf(st0) < 1e-6f || fabsf(st1) < 1e-6f || fabsf(st2) < 1e-6f)) {
          const float sh = sinf(h);
          const float c0 = clampf1((2.0f * sh * sinf(h - t0)) / (st1 * st2) - 1.0f, -1.0f, 1.0f);
          const float c1 = clampf1((2.0f * sh * sinf(h - t1)) / (st2 * st0) - 1.0f, -1.0f, 1.0f);
          const float c2 = clampf1((2.0f * sh * sinf(h - t2)) / (st0 * st1) - 1.0f, -1.0f, 1.0f);
          const float det = dot(u2, cross(u0, u1));
          const float sg = det >= 0.0f ? 1.0f : -1.0f;
          const float s0 = sg * sqrtf(fmaxf(1.0f - c0 * c0, 0.0f));
          const float s1 = sg * sqrtf(fmaxf(1.0f - c1 * c1, 0.0f));
          const float s2 = sg * sqrtf(fmaxf(1.0f - c2 * c2, 0.0f));
          if (!(fabsf(s0) <= 1e-6f || fabsf(s1) <= 1e-6f || fabsf(s2) <= 1e-6f)) {
            m.x = ((t0 - c1 * t2) - c2 * t1) / (2.0f * d0 * st1 * s2);
            m.y = ((t1 - c2 * t0) - c0 * t2) / (2.0f * d1 * st2 * s0);
            m.z = ((t2 - c0 * t1) - c1 * t0) / (2.0f * d2 * st0 * s1);
          }
        }
      }
      s.mu[f] = m;
    }
  }
  __syncthreads();
  const uint32_t fhit = s.hit[1];
  if (tid == 0 && vhit == kNone && fhit == kNone) {
    // the normaliser, face by face as the reference accumulates it
    float total = 0.0f;
    for (uint32_t f = 0; f < c.F; ++f) {
      const float4 m = s.mu[f];
      total += (m.x + m.y) + m.z;
    }
    s.total[0] = total;
    uint32_t nearest = 0;
    if (!(fabsf(total) > 1e-12f)) {
      for (uint32_t j = 1; j < c.V; ++j)
        if (s.dir[j].w < s.dir[nearest].w) nearest = j;
    }
    s.total[1] = __uint_as_float(nearest);
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < OWN; ++k) {
    const uint32_t j = tid + k * blockDim.x;
    float v = 0.0f;
    if (j < c.V) {
      if (vhit != kNone) {
        v = j == vhit ? 1.0f : 0.0f;
      } else if (fhit != kNone) {
        const uint4 t = c.tris[fhit];
        const float4 m = s.mu[fhit];
        const float sum = (m.x + m.y) + m.z;
        if (fabsf(sum) > 1e-12f)
          v = j == t.x ? m.x / sum : (j == t.y ? m.y / sum : (j == t.z ? m.z / sum : 0.0f));
      } else {
        float acc = 0.0f;
        for (uint32_t e = c.vf_off[j]; e < c.vf_off[j + 1]; ++e) {
          const uint32_t fe = c.vf_list[e];
          const float4 m = s.mu[fe >> 2];
          const uint32_t corner = fe & 3u;
          acc += corner == 0 ? m.x : (corner == 1 ? m.y : m.z);
        }
        const float total = s.total[0];
        if (fabsf(total) > 1e-12f) {
          v = acc * (1.0f / total);
        } else {
          v = j == __float_as_uint(s.total[1]) ? 1.0f : acc;
        }
      }
    }
    w[k] = v;
  }
  __syncthreads();  // shared memory is reused by the next evaluation
}

constexpr int kMaxOwn = 8;  // V <= 8 * 128

__device__ __forceinline__ EvalSmem eval_smem(unsigned char* base, const MvcCage& c) {
  EvalSmem s;
  s.dir = reinterpret_cast<float4*>(base);
  s.mu = s.dir + c.V;
  s.hit = reinterpret_cast<uint32_t*>(s.mu + c.F);
  s.total = reinterpret_cast<float*>(s.hit + 2);
  return s;
}

// Exact weights of arbitrary points: w[i * V + j].
__global__ void __launch_bounds__(kMvcThreads, 1) k_mvc_weights(const MvcCage c, uint32_t n,
                                                            const float* __restrict__ pts,
                                                            float* __restrict__ w) {
  extern __shared__ __align__(16) unsigned char mvc_smem[];
  const EvalSmem s = eval_smem(mvc_smem, c);
  for (uint32_t i = blockIdx.x; i < n; i += gridDim.x) {
    const F3 x = {pts[3 * (size_t)i], pts[3 * (size_t)i + 1], pts[3 * (size_t)i + 2]};
    float wr[kMaxOwn];
    mvc_eval<kMaxOwn>(c, x, s, wr);
#pragma unroll
    for (int k = 0; k < kMaxOwn; ++k) {
      const uint32_t j = threadIdx.x + k * blockDim.x;
      if (j < c.V) w[(size_t)i * c.V + j] = wr[k];
    }
  }
}

// bind_gaussians (mvc.rs:498-541) for the bound Gaussians: weights and
// central-difference gradients, stored vertex-major, wg[j * nb + slot] =
// (w, dw/dx, dw/dy, dw/dz).
__global__ void __launch_bounds__(kMvcThreads, 1) k_mvc_bind_weights(const MvcCage c, uint32_t nb,
                                                                 const uint32_t* __restrict__ list,
                                                                 const float4* __restrict__ rest_pos,
                                                                 float h,
                                                                 float4* __restrict__ wg) {
  extern __shared__ __align__(16) unsigned char mvc_smem[];
  const EvalSmem s = eval_smem(mvc_smem, c);
  const float inv_2h = 0.5f / h;
  for (uint32_t slot = blockIdx.x; slot < nb; slot += gridDim.x) {
    const float4 p = rest_pos[list[slot]];
    float w0[kMaxOwn], wp[kMaxOwn], wm[kMaxOwn], g[3][kMaxOwn];
    mvc_eval<kMaxOwn>(c, {p.x, p.y, p.z}, s, w0);
#pragma unroll
    for (int axis = 0; axis < 3; ++axis) {
      F3 xp = {p.x, p.y, p.z}, xm = {p.x, p.y, p.z};
      if (axis == 0) { xp.x += h; xm.x -= h; }
      if (axis == 1) { xp.y += h; xm.y -= h; }
      if (axis == 2) { xp.z += h; xm.z -= h; }
      mvc_eval<kMaxOwn>(c, xp, s, wp);
      mvc_eval<kMaxOwn>(c, xm, s, wm);
#pragma unroll
      for (int k = 0; k < kMaxOwn; ++k) g[axis][k] = (wp[k] - wm[k]) * inv_2h;
    }
#pragma unroll
    for (int k = 0; k < kMaxOwn; ++k) {
      const uint32_t j = threadIdx.x + k * blockDim.x;
      if (j < c.V) wg[(size_t)j * nb + slot] = make_float4(w0[k], g[0][k], g[1][k], g[2][k]);
    }
  }
}

// winding_number (mvc.rs:339-357) >= 0.5 for Gaussians not bound to a tet cage;
// flag[i] = 1 marks a new MVC binding.
__global__ void k_mvc_inside(const MvcCage c, uint32_t n, const float4* __restrict__ rest_pos,
                             const uint32_t* __restrict__ bind_tet, uint32_t* __restrict__ flag) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t in = 0;
  if (bind_tet[i] == kNone) {
    const float4 p4 = rest_pos[i];
    const F3 p = {p4.x, p4.y, p4.z};
    float sum = 0.0f;
    bool on_vertex = false;
    for (uint32_t f = 0; f < c.F; ++f) {
      const uint4 t = c.tris[f];
      const F3 a = sub(f3(c.verts[t.x]), p), b = sub(f3(c.verts[t.y]), p),
               cc = sub(f3(c.verts[t.z]), p);
      const float la = len(a), lb = len(b), lc = len(cc);
      if (la < 1e-7f || lb < 1e-7f || lc < 1e-7f) {
        on_vertex = true;
        break;
      }
      const float det = dot(a, cross(b, cc));
      const float denom = ((la * lb * lc + dot(a, b) * lc) + dot(b, cc) * la) + dot(cc, a) * lb;
      sum += 2.0f * atan2f(det, denom);
    }
    const float wn = on_vertex ? 1.0f : sum / (4.0f * 3.14159265358979323846f);
    in = fabsf(wn) >= 0.5f ? 1u : 0u;
  }
  flag[i] = in;
}

// Bound Gaussians get consecutive slots in index order.
__global__ void k_mvc_compact(uint32_t n, const uint32_t* __restrict__ flag,
                              const uint32_t* __restrict__ slot_of, uint32_t* __restrict__ bind_tet,
                              float4* __restrict__ bind_w, uint32_t* __restrict__ list) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !flag[i]) return;
  const uint32_t slot = slot_of[i];
  list[slot] = i;
  bind_tet[i] = kMvcBound;
  bind_w[i] = make_float4(__uint_as_float(slot), 0.0f, 0.0f, 0.0f);
}

// Per frame: deformed position sum_j w_j v_j and deformation gradient
// F = sum_j v_j grad(w_j)^T of every stored binding (MvcBindings::local_jacobian,
// evaluate_position), vertex by vertex in order. xf[slot] = 3 float4:
// (x, y, z, F00), (F10, F20, F01, F11), (F21, F02, F12, F22), F column-major.
//
// One thread per slot. Each thread streams its own column of wg through a
// kJacStages-deep ring of kJacChunk vertices in shared memory with cp.async
// (16 bytes per vertex, the warp's copies of one vertex contiguous), so that
// up to (kJacStages - 1) * kJacChunk copies per thread are in flight even
// when there are only a few thousand slots; the sums stay sequential in j.
// A thread reads only the ring entries it copied itself, and in-order issue
// puts every read of a stage before the copy that refills it.
constexpr int kJacThreads = 128, kJacChunk = 8, kJacStages = 4;

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

__global__ void __launch_bounds__(kJacThreads) k_mvc_jacobian(uint32_t V, const float4* __restrict__ verts,
                                                              uint32_t nb, const float4* __restrict__ wg,
                                                              float4* __restrict__ xf) {
  extern __shared__ float4 s_v[];  // [V] vertices, then the ring
  float4* ring = s_v + V;          // [kJacStages][kJacChunk][kJacThreads]
  for (uint32_t j = threadIdx.x; j < V; j += blockDim.x) s_v[j] = verts[j];
  __syncthreads();
  const uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = slot < nb;
  const float4* row = wg + slot;
  const uint32_t chunks = (V + kJacChunk - 1) / kJacChunk;
  auto issue = [&](uint32_t c) {
    if (active && c < chunks) {
      float4* dst = ring + (size_t)(c % kJacStages) * kJacChunk * kJacThreads + threadIdx.x;
#pragma unroll
      for (int u = 0; u < kJacChunk; ++u) {
        const uint32_t j = c * kJacChunk + u;
        if (j < V) cp_async16(dst + u * kJacThreads, row + (size_t)j * nb);
      }
    }
    cp_async_commit();
  };
#pragma unroll
  for (int c = 0; c < kJacStages - 1; ++c) issue(c);
  float px = 0, py = 0, pz = 0, a0 = 0, a1 = 0, a2 = 0, b0 = 0, b1 = 0, b2 = 0, c0 = 0, c1 = 0,
        c2 = 0;
  for (uint32_t c = 0; c < chunks; ++c) {
    issue(c + kJacStages - 1);
    cp_async_wait<kJacStages - 1>();
    if (!active) continue;
    const float4* src = ring + (size_t)(c % kJacStages) * kJacChunk * kJacThreads + threadIdx.x;
#pragma unroll
    for (int u = 0; u < kJacChunk; ++u) {
      const uint32_t j = c * kJacChunk + u;
      if (j < V) {
        const float4 g = src[u * kJacThreads];
        const float4 v = s_v[j];
        px = px + v.x * g.x; py = py + v.y * g.x; pz = pz + v.z * g.x;
        a0 = a0 + v.x * g.y; a1 = a1 + v.y * g.y; a2 = a2 + v.z * g.y;
        b0 = b0 + v.x * g.z; b1 = b1 + v.y * g.z; b2 = b2 + v.z * g.z;
        c0 = c0 + v.x * g.w; c1 = c1 + v.y * g.w; c2 = c2 + v.z * g.w;
      }
    }
  }
  cp_async_wait<0>();
  if (!active) return;
  xf[3 * (size_t)slot] = make_float4(px, py, pz, a0);
  xf[3 * (size_t)slot + 1] = make_float4(a1, a2, b0, b1);
  xf[3 * (size_t)slot + 2] = make_float4(b2, c0, c1, c2);
}

size_t eval_smem_bytes(const MvcCage& c) { return (size_t)(c.V + c.F) * 16 + 32; }

template <typename K>
cudaError_t set_smem(K kernel, size_t bytes) {
  if (bytes <= 48 * 1024) return cudaSuccess;
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

}  // namespace

bool mvc_cage_fits(uint32_t V, uint32_t F) {
  return V >= 4 && F >= 4 && V <= (uint32_t)kMaxOwn * kMvcThreads && (V + F) * 16 + 32 <= 200 * 1024;
}

cudaError_t launch_mvc_weights(const MvcCage& c, uint32_t n, const float* pts, float* w,
                               cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  const size_t smem = eval_smem_bytes(c);
  cudaError_t e = set_smem(k_mvc_weights, smem);
  if (e != cudaSuccess) return e;
  k_mvc_weights<<<std::min<uint32_t>(n, 148u * 16u), kMvcThreads, smem, s>>>(c, n, pts, w);
  return cudaGetLastError();
}

cudaError_t launch_mvc_inside(const MvcCage& c, uint32_t n, const float4* rest_pos,
                              const uint32_t* bind_tet, uint32_t* flag, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  k_mvc_inside<<<(n + 255) / 256, 256, 0, s>>>(c, n, rest_pos, bind_tet, flag);
  return cudaGetLastError();
}

cudaError_t launch_mvc_compact(uint32_t n, const uint32_t* flag, const uint32_t* slot_of,
                               uint32_t* bind_tet, float4* bind_w, uint32_t* list,
                               cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  k_mvc_compact<<<(n + 255) / 256, 256, 0, s>>>(n, flag, slot_of, bind_tet, bind_w, list);
  return cudaGetLastError();
}

cudaError_t launch_mvc_bind_weights(const MvcCage& c, uint32_t nb, const uint32_t* list,
                                    const float4* rest_pos, float h, float4* wg, cudaStream_t s) {
  if (nb == 0) return cudaSuccess;
  const size_t smem = eval_smem_bytes(c);
  cudaError_t e = set_smem(k_mvc_bind_weights, smem);
  if (e != cudaSuccess) return e;
  k_mvc_bind_weights<<<std::min<uint32_t>(nb, 148u * 16u), kMvcThreads, smem, s>>>(
      c, nb, list, rest_pos, h, wg);
  return cudaGetLastError();
}

cudaError_t launch_mvc_jacobian(uint32_t V, const float4* verts, uint32_t nb, const float4* wg,
                                float4* xf, cudaStream_t s) {
  if (nb == 0) return cudaSuccess;
  const size_t smem = (size_t)V * 16 + (size_t)kJacStages * kJacChunk * kJacThreads * 16;
  cudaError_t e = set_smem(k_mvc_jacobian, smem);
  if (e != cudaSuccess) return e;
  k_mvc_jacobian<<<(nb + kJacThreads - 1) / kJacThreads, kJacThreads, smem, s>>>(V, verts, nb, wg,
                                                                                   xf);
  return cudaGetLastError();
}

}  // namespace cgs
