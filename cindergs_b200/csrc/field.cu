// Host driver of the learned MVC weight field: parameter block, batches,
// the training step sequence and the per-frame projection (field.h).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "field.h"

namespace cgs {

#define FIELD_TRY(x)                   \
  do {                                 \
    const cudaError_t e_ = (x);        \
    if (e_ != cudaSuccess) return e_;  \
  } while (0)

cudaError_t FieldBuf::ensure(size_t bytes) {
  if (bytes == 0) bytes = 16;
  if (bytes <= cap) return cudaSuccess;
  if (p) cudaFree(p);
  p = nullptr;
  cap = 0;
  FIELD_TRY(cudaMalloc(&p, bytes));
  cap = bytes;
  return cudaMemset(p, 0, bytes);
}

namespace {

uint64_t splitmix64(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Standard normal samples by the Box-Muller transform on splitmix64 uniforms.
double normal(uint64_t& s) {
  const double u1 = ((splitmix64(s) >> 11) + 1.0) * (1.0 / 9007199254740993.0);
  const double u2 = (splitmix64(s) >> 11) * (1.0 / 9007199254740992.0);
  return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
}

uint32_t pad8(uint32_t v) { return (v + 7u) & ~7u; }

// Inverse of a 4 x 4 matrix by Gauss-Jordan elimination with partial
// pivoting; false when singular.
bool invert4(const double (&a)[4][4], double (&inv)[4][4]) {
  double m[4][8];
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 8; ++j) m[i][j] = j < 4 ? a[i][j] : (j - 4 == i ? 1.0 : 0.0);
  for (int c = 0; c < 4; ++c) {
    int piv = c;
    for (int r = c + 1; r < 4; ++r)
      if (std::fabs(m[r][c]) > std::fabs(m[piv][c])) piv = r;
    if (!(std::fabs(m[piv][c]) > 0.0)) return false;
    if (piv != c)
      for (int j = 0; j < 8; ++j) std::swap(m[c][j], m[piv][j]);
    const double d = 1.0 / m[c][c];
    for (int j = 0; j < 8; ++j) m[c][j] *= d;
    for (int r = 0; r < 4; ++r)
      if (r != c) {
        const double f = m[r][c];
        for (int j = 0; j < 8; ++j) m[r][j] -= f * m[c][j];
      }
  }
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) inv[i][j] = m[i][j + 4];
  return true;
}

}  // namespace

cudaError_t FieldState::init(uint32_t nv, const float* rest_v4, uint64_t seed, cudaStream_t s) {
  V = nv;
  ldV = pad8(nv);
  const uint32_t sizes[kFieldParams] = {kFieldHid * kFieldIn, kFieldHid, kFieldHid * kFieldHid,
                                        kFieldHid,            kFieldHid * kFieldHid, kFieldHid,
                                        kFieldHid * kFieldHid, kFieldHid, nv * kFieldHid, nv};
  uint32_t o = 0;
  for (int k = 0; k < kFieldParams; ++k) {
    off[k] = o;
    o += pad8(sizes[k]);
  }
  off[kFieldParams] = o;
  // encoding: centre and half-extent of the rest cage's bounding box
  float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (uint32_t j = 0; j < nv; ++j)
    for (int d = 0; d < 3; ++d) {
      lo[d] = std::min(lo[d], rest_v4[4 * j + d]);
      hi[d] = std::max(hi[d], rest_v4[4 * j + d]);
    }
  scale = 0.5f * std::max(hi[0] - lo[0], std::max(hi[1] - lo[1], hi[2] - lo[2]));
  if (!(scale > 0.0f)) scale = 1.0f;
  for (int d = 0; d < 3; ++d) enc[d] = 0.5f * (lo[d] + hi[d]);
  enc[3] = 1.0f / scale;
  // M = (Vb Vb^T)^-1, Vb = [1; v_j] over the rest vertices
  double G[4][4] = {}, Gi[4][4];
  for (uint32_t j = 0; j < nv; ++j) {
    const double b[4] = {1.0, rest_v4[4 * j], rest_v4[4 * j + 1], rest_v4[4 * j + 2]};
    for (int a = 0; a < 4; ++a)
      for (int c = 0; c < 4; ++c) G[a][c] += b[a] * b[c];
  }
  if (!invert4(G, Gi)) return cudaErrorInvalidValue;  // degenerate (flat) cage
  for (int a = 0; a < 4; ++a)
    for (int c = 0; c < 4; ++c) M.m[4 * a + c] = (float)Gi[a][c];
  std::vector<float> h(o, 0.0f);
  uint64_t st = seed * 0x2545F4914F6CDD1Dull + 1;
  const int fan[4] = {kFieldIn, kFieldHid, kFieldHid, kFieldHid};
  const int wl[4] = {kW1, kW2, kW3, kW4};
  for (int l = 0; l < 4; ++l) {
    const double sd = std::sqrt(2.0 / fan[l]);
    for (uint32_t i = 0; i < sizes[wl[l]]; ++i) h[off[wl[l]] + i] = (float)(sd * normal(st));
  }
  for (uint32_t i = 0; i < sizes[kW5]; ++i) h[off[kW5] + i] = (float)(1e-3 * normal(st));
  for (uint32_t j = 0; j < nv; ++j) h[off[kB5] + j] = 1.0f / (float)nv;
  FIELD_TRY(p32.ensure((size_t)o * 4));
  FIELD_TRY(g32.ensure((size_t)o * 4));
  FIELD_TRY(m1.ensure((size_t)o * 4));
  FIELD_TRY(m2.ensure((size_t)o * 4));
  FIELD_TRY(pb.ensure((size_t)o * 2));
  FIELD_TRY(enc_d.ensure(16));
  FIELD_TRY(M_d.ensure(64));
  FIELD_TRY(rest_d.ensure((size_t)nv * 16));
  FIELD_TRY(proj.ensure((size_t)kFieldProj * 4));
  FIELD_TRY(proj_rest.ensure((size_t)kFieldProj * 4));
  FIELD_TRY(loss.ensure(16));
  FIELD_TRY(status.ensure(16));
  FIELD_TRY(wT.ensure((size_t)kFieldHid * std::max<uint32_t>(ldV, kFieldHid) * 2));
  FIELD_TRY(cudaMemsetAsync(m1.p, 0, (size_t)o * 4, s));
  FIELD_TRY(cudaMemsetAsync(m2.p, 0, (size_t)o * 4, s));
  FIELD_TRY(cudaMemsetAsync(g32.p, 0, (size_t)o * 4, s));
  FIELD_TRY(cudaMemcpyAsync(enc_d.p, enc, 16, cudaMemcpyHostToDevice, s));
  FIELD_TRY(cudaMemcpyAsync(M_d.p, M.m, 64, cudaMemcpyHostToDevice, s));
  FIELD_TRY(cudaMemcpyAsync(rest_d.p, rest_v4, (size_t)nv * 16, cudaMemcpyHostToDevice, s));
  step = 0;
  FIELD_TRY(cudaMemcpyAsync(p32.p, h.data(), (size_t)o * 4, cudaMemcpyHostToDevice, s));
  FIELD_TRY(launch_transpose_f32(p32.as<float>(), 1, o, o, pb.as<__nv_bfloat16>(), 1, s));
  return cudaStreamSynchronize(s);  // h goes out of scope
}

FieldNet FieldState::net() const {
  FieldNet n;
  const __nv_bfloat16* b = pb.as<__nv_bfloat16>();
  const float* f = p32.as<float>();
  n.W1b = b + off[kW1];
  n.W2b = b + off[kW2];
  n.W3b = b + off[kW3];
  n.W4b = b + off[kW4];
  n.W5b = b + off[kW5];
  n.b1 = f + off[kB1];
  n.b2 = f + off[kB2];
  n.b3 = f + off[kB3];
  n.b4 = f + off[kB4];
  n.b5 = f + off[kB5];
  return n;
}

cudaError_t FieldState::ensure_batch(uint32_t B) {
  if (B <= Bcap) return cudaSuccess;
  const size_t b = B, H = kFieldHid;
  FIELD_TRY(x.ensure(b * 12));
  FIELD_TRY(wt.ensure(b * ldV * 4));
  FIELD_TRY(a0.ensure(b * kFieldIn * 2));
  for (int l = 0; l < 4; ++l) {
    FIELD_TRY(pre[l].ensure(b * H * 4));
    FIELD_TRY(h[l].ensure(b * H * 2));
  }
  FIELD_TRY(z.ensure(b * ldV * 4));
  FIELD_TRY(dz.ensure(b * ldV * 4));
  FIELD_TRY(dzb.ensure(b * ldV * 2));
  FIELD_TRY(dzT.ensure((size_t)ldV * b * 2));
  FIELD_TRY(hT.ensure(H * b * 2));
  FIELD_TRY(dpre.ensure(b * H * 4));
  FIELD_TRY(dpreb.ensure(b * H * 2));
  FIELD_TRY(dpreT.ensure(H * b * 2));
  FIELD_TRY(dh.ensure(b * H * 4));
  FIELD_TRY(gemm_ws.ensure((size_t)16 * std::max<uint32_t>(ldV, kFieldHid) * H * 4));
  Bcap = B;
  return cudaSuccess;
}

cudaError_t FieldState::forward(const float* points, const float* target, uint32_t n, uint32_t B,
                                uint32_t seed, const float4* rest_verts, float lambda,
                                cudaStream_t s) {
  FIELD_TRY(ensure_batch(B));
  FieldBatch fb{};
  fb.points = points;
  fb.target = target;
  fb.n = n;
  fb.V = V;
  fb.B = B;
  fb.ldw = ldV;
  fb.seed = seed;
  fb.enc = enc_d.as<float>();
  fb.x = x.as<float>();
  fb.wt = wt.as<float>();
  fb.a0 = a0.as<__nv_bfloat16>();
  FIELD_TRY(launch_field_gather(fb, s));
  const FieldNet nt = net();
  const __nv_bfloat16* W[4] = {nt.W1b, nt.W2b, nt.W3b, nt.W4b};
  const float* bias[4] = {nt.b1, nt.b2, nt.b3, nt.b4};
  for (int l = 0; l < 4; ++l) {
    GemmArgs g{};
    g.status = status.as<uint32_t>();
    g.A = l == 0 ? a0.as<__nv_bfloat16>() : h[l - 1].as<__nv_bfloat16>();
    g.lda = g.K = l == 0 ? kFieldIn : kFieldHid;
    g.B = W[l];
    g.ldb = g.K;
    g.M = B;
    g.N = kFieldHid;
    g.C = pre[l].as<float>();
    g.ldc = kFieldHid;
    g.bias = bias[l];
    g.D = h[l].as<__nv_bfloat16>();
    g.ldd = kFieldHid;
    FIELD_TRY(launch_gemm_nt(g, kEpiBiasSilu, s));
  }
  GemmArgs g{};
  g.status = status.as<uint32_t>();
  g.A = h[3].as<__nv_bfloat16>();
  g.lda = g.K = kFieldHid;
  g.B = nt.W5b;
  g.ldb = kFieldHid;
  g.M = B;
  g.N = V;
  g.C = z.as<float>();
  g.ldc = ldV;
  g.bias = nt.b5;
  FIELD_TRY(launch_gemm_nt(g, kEpiBias, s));
  if (!target) return cudaSuccess;
  FieldLoss fl{};
  fl.z = z.as<float>();
  fl.wt = wt.as<float>();
  fl.x = x.as<float>();
  fl.verts = rest_verts;
  fl.B = B;
  fl.V = V;
  fl.ldz = ldV;
  fl.ldw = ldV;
  fl.lambda = lambda;
  fl.s2 = scale * scale;
  std::memcpy(fl.M, M.m, 64);
  fl.dz = dz.as<float>();
  fl.dzb = dzb.as<__nv_bfloat16>();
  fl.loss = loss.as<float>();
  return launch_field_loss(fl, s);
}

cudaError_t FieldState::backward(uint32_t B, cudaStream_t s) {
  if (B % 8) return cudaErrorInvalidValue;  // transposed operands have row length B
  const FieldNet nt = net();
  float* g = g32.as<float>();
  __nv_bfloat16* wTb = wT.as<__nv_bfloat16>();
  // output layer: dW5 = dz^T h4, db5 = sum_rows dz, dh4 = dz W5
  FIELD_TRY(launch_transpose_f32(dz.as<float>(), B, V, ldV, dzT.as<__nv_bfloat16>(), B, s));
  FIELD_TRY(launch_transpose_bf16(h[3].as<__nv_bfloat16>(), B, kFieldHid, kFieldHid,
                                  hT.as<__nv_bfloat16>(), B, s));
  GemmArgs gw{};
  gw.status = status.as<uint32_t>();
  gw.ws = gemm_ws.as<float>();
  gw.ws_floats = gemm_ws.cap / 4;
  gw.A = dzT.as<__nv_bfloat16>();
  gw.lda = B;
  gw.B = hT.as<__nv_bfloat16>();
  gw.ldb = B;
  gw.M = V;
  gw.N = kFieldHid;
  gw.K = B;
  gw.C = g + off[kW5];
  gw.ldc = kFieldHid;
  FIELD_TRY(launch_gemm_nt(gw, kEpiF32, s));
  FIELD_TRY(launch_colsum(dz.as<float>(), B, V, ldV, g + off[kB5], s));
  FIELD_TRY(launch_transpose_bf16(nt.W5b, V, kFieldHid, kFieldHid, wTb, ldV, s));
  GemmArgs gd{};
  gd.status = status.as<uint32_t>();
  gd.A = dzb.as<__nv_bfloat16>();
  gd.lda = ldV;
  gd.B = wTb;
  gd.ldb = ldV;
  gd.M = B;
  gd.N = kFieldHid;
  gd.K = V;
  gd.C = dh.as<float>();
  gd.ldc = kFieldHid;
  FIELD_TRY(launch_gemm_nt(gd, kEpiF32, s));
  const __nv_bfloat16* Wl[4] = {nt.W1b, nt.W2b, nt.W3b, nt.W4b};
  const int wk[4] = {kW1, kW2, kW3, kW4}, bk[4] = {kB1, kB2, kB3, kB4};
  for (int l = 3; l >= 0; --l) {
    FIELD_TRY(launch_silu_back(B * kFieldHid, dh.as<float>(), pre[l].as<float>(), dpre.as<float>(),
                               dpreb.as<__nv_bfloat16>(), s));
    FIELD_TRY(launch_transpose_f32(dpre.as<float>(), B, kFieldHid, kFieldHid,
                                   dpreT.as<__nv_bfloat16>(), B, s));
    const uint32_t kin = l == 0 ? kFieldIn : kFieldHid;
    const __nv_bfloat16* in = l == 0 ? a0.as<__nv_bfloat16>() : h[l - 1].as<__nv_bfloat16>();
    FIELD_TRY(launch_transpose_bf16(in, B, kin, kin, hT.as<__nv_bfloat16>(), B, s));
    GemmArgs gl{};
    gl.status = status.as<uint32_t>();
    gl.ws = gemm_ws.as<float>();
    gl.ws_floats = gemm_ws.cap / 4;
    gl.A = dpreT.as<__nv_bfloat16>();
    gl.lda = B;
    gl.B = hT.as<__nv_bfloat16>();
    gl.ldb = B;
    gl.M = kFieldHid;
    gl.N = kin;
    gl.K = B;
    gl.C = g + off[wk[l]];
    gl.ldc = kin;
    FIELD_TRY(launch_gemm_nt(gl, kEpiF32, s));
    FIELD_TRY(launch_colsum(dpre.as<float>(), B, kFieldHid, kFieldHid, g + off[bk[l]], s));
    if (l > 0) {
      FIELD_TRY(launch_transpose_bf16(Wl[l], kFieldHid, kFieldHid, kFieldHid, wTb, kFieldHid, s));
      GemmArgs gh{};
      gh.status = status.as<uint32_t>();
      gh.A = dpreb.as<__nv_bfloat16>();
      gh.lda = kFieldHid;
      gh.B = wTb;
      gh.ldb = kFieldHid;
      gh.M = B;
      gh.N = kFieldHid;
      gh.K = kFieldHid;
      gh.C = dh.as<float>();
      gh.ldc = kFieldHid;
      FIELD_TRY(launch_gemm_nt(gh, kEpiF32, s));
    }
  }
  return cudaSuccess;
}

cudaError_t FieldState::adam(float lr, cudaStream_t s) {
  ++step;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = (float)(1.0 / (1.0 - std::pow(0.9, (double)step)));
  const float c2 = (float)(1.0 / (1.0 - std::pow(0.999, (double)step)));
  return launch_adam(total(), p32.as<float>(), g32.as<float>(), m1.as<float>(), m2.as<float>(),
                     pb.as<__nv_bfloat16>(), lr, b1, b2, 1e-8f, c1, c2, s);
}

cudaError_t FieldState::eval(uint32_t n, const float* points, float* w, cudaStream_t s) {
  const uint32_t chunk = 65536;
  for (uint32_t done = 0; done < n; done += chunk) {
    const uint32_t B = std::min(chunk, n - done);
    FIELD_TRY(forward(points + 3 * (size_t)done, nullptr, B, B, 0, nullptr, 0.0f, s));
    FIELD_TRY(launch_field_weights(z.as<float>(), B, V, ldV, x.as<float>(), rest_d.as<float4>(), M,
                                   w + (size_t)done * V, s));
  }
  return cudaSuccess;
}

cudaError_t FieldState::project(const float4* verts, float* out, cudaStream_t s) const {
  return launch_field_project(net(), V, rest_d.as<float4>(), verts, M_d.as<float>(), out, s);
}

}  // namespace cgs
