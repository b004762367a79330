// Host driver of the learned MVC weight field (mvc_field.cu): parameters,
// Adam state, training batches, and the per-frame projection.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "kernels.h"

namespace cgs {

struct FieldBuf {
  void* p = nullptr;
  size_t cap = 0;  // bytes
  FieldBuf() = default;
  FieldBuf(const FieldBuf&) = delete;
  FieldBuf& operator=(const FieldBuf&) = delete;
  ~FieldBuf() {
    if (p) cudaFree(p);
  }
  cudaError_t ensure(size_t bytes);  // grows, zero-filled; contents are not kept
  template <typename T>
  T* as() const {
    return reinterpret_cast<T*>(p);
  }
};

// Parameter block (fp32 master copy, gradients, Adam moments and a bf16 copy
// share this layout): W1 [128 x 64], b1, W2, b2, W3, b3, W4, b4 [128],
// W5 [V x 128], b5 [V]; every offset a multiple of 8 elements.
enum FieldParam { kW1, kB1, kW2, kB2, kW3, kB3, kW4, kB4, kW5, kB5, kFieldParams };

struct FieldState {
  uint32_t V = 0, ldV = 0;  // outputs, padded to 8
  uint32_t off[kFieldParams + 1] = {};  // element offsets, off[kFieldParams] = total
  float enc[4] = {};        // rest-cage centre xyz, 1 / s
  float scale = 1.0f;       // s: half of the largest rest-cage extent
  FieldMat M{};             // (Vb Vb^T)^-1, Vb = [1; rest vertices]
  uint32_t step = 0;        // Adam steps taken
  FieldBuf p32, g32, m1, m2, pb, enc_d, M_d, rest_d, proj, proj_rest, loss, wT, status;
  // training batch (B rows)
  uint32_t Bcap = 0;
  FieldBuf x, wt, a0, pre[4], h[4], z, dz, dzb, dzT, hT, dpre, dpreb, dpreT, dh;
  FieldBuf gemm_ws;  // split-K partial sums of the weight gradients (K = batch)

  uint32_t total() const { return off[kFieldParams]; }
  // New network for a cage of V vertices with the given rest vertices [V*4]
  // (float4 on the host): He-initialised hidden layers, zero hidden biases,
  // output weights N(0, 1e-6), output biases 1/V (uniform weights).
  cudaError_t init(uint32_t V, const float* rest_v4, uint64_t seed, cudaStream_t s);
  FieldNet net() const;
  cudaError_t ensure_batch(uint32_t B);
  // Forward over a batch (rows r -> points as FieldBatch::seed says), with
  // the loss and dL/dz when target is given, and the backward pass into g32
  // when backward is set. loss[0..1] accumulate in `loss`.
  cudaError_t forward(const float* points, const float* target, uint32_t n, uint32_t B,
                      uint32_t seed, const float4* rest_verts, float lambda, cudaStream_t s);
  cudaError_t backward(uint32_t B, cudaStream_t s);
  cudaError_t adam(float lr, cudaStream_t s);
  // Final (projected) weights of n points [n*3] into w [n*V].
  cudaError_t eval(uint32_t n, const float* points, float* w, cudaStream_t s);
  // Per-frame projection of the output layer for current vertices [V]
  // (float4), or the raw rest projection when verts is null.
  cudaError_t project(const float4* verts, float* out, cudaStream_t s) const;
};

cudaError_t launch_field_weights(const float* z, uint32_t B, uint32_t V, uint32_t ldz,
                                 const float* x, const float4* verts, const FieldMat& M, float* w,
                                 cudaStream_t s);
cudaError_t launch_mvc_reslot(uint32_t nb, const uint32_t* flag, const uint32_t* rank,
                              uint32_t nfb, const uint32_t* list_in, uint32_t* list_out,
                              float4* bind_w, cudaStream_t s);

}  // namespace cgs
