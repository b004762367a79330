// Stage 1: tetrahedral cage deformation on sm_100a.
//
//  k_tet_transforms  per tet: J = D_s D_m^-1, largest singular value by
//                    Cardano on J^T J, rotation by 5 Newton-Schulz polar
//                    steps with chirality fix
//                    (render/kernels/deformation.rs:684-865).
//                    In frames the first blocks of the k_deform launch run
//                    these transforms (tet_transform) and publish a count,
//                    so Stage 1 is one launch; the Gaussian blocks of a
//                    deform with strain split wait for it (bounded).
//  k_deform<SPLIT>   per Gaussian: x' = sum w_k x_k, M = J S J^T (diag >= 1e-4,
//                    symmetrised), det-J opacity, 3D Mip filter, strain split
//                    along the major eigenvector
//                    (render/kernels/deformation.rs:874-1211).
//                    Split children are compacted deterministically: child
//                    slot = n + (number of splitting Gaussians with a lower
//                    index), from a block scan chained across blocks, instead
//                    of the reference's atomic counter whose order varies
//                    from run to run (deformation.rs:1191). Without the
//                    split the Gaussians evaluate their tet's J from the
//                    four vertices they load anyway (tet_jacobian, as the
//                    tet blocks do) and never wait; their blocks are
//                    persistent (as many as the SMs hold), and each thread
//                    loads its next Gaussian's 60 B while deforming the
//                    current one.
//  k_bind            GPU barycentric binding (TetMesh::bind_point,
//                    deformation/mod.rs:267-310).
//
// This file is compiled with -fmad=false: every product and sum is rounded
// separately, in the reference's operand order, so the host-side restatement
// reproduces it bit for bit. Memory layout: Gaussians as float4 (xyz,
// opacity) + float4 (xx, xy, xz, yy) + float2 (yz, zz) arrays, read and
// written coalesced with 128-bit accesses (40 B read + 20 B binding per
// Gaussian, 40 B written).
#include "kernels.h"

namespace cgs {
namespace {

constexpr int kDeformThreads = 256;

// J = D_s D_m^-1 of one tet from its four vertices (x[k] = vertex k's xyz)
// and its D_m^-1 (column-major), into j (column-major). The tet blocks and the
// Gaussians of a deform without strain split both evaluate it; with every
// operation rounded separately (-fmad=false) the two agree bit for bit.
__device__ __forceinline__ void tet_jacobian(const float (&x)[4][3], const float* __restrict__ a,
                                             float (&j)[9]) {
  const float x0x = x[0][0], x0y = x[0][1], x0z = x[0][2];
  const float ds_00 = x[1][0] - x0x, ds_10 = x[1][1] - x0y, ds_20 = x[1][2] - x0z;
  const float ds_01 = x[2][0] - x0x, ds_11 = x[2][1] - x0y, ds_21 = x[2][2] - x0z;
  const float ds_02 = x[3][0] - x0x, ds_12 = x[3][1] - x0y, ds_22 = x[3][2] - x0z;
  const float a_00 = a[0], a_10 = a[1], a_20 = a[2], a_01 = a[3], a_11 = a[4], a_21 = a[5];
  const float a_02 = a[6], a_12 = a[7], a_22 = a[8];
  j[0] = ds_00 * a_00 + ds_01 * a_10 + ds_02 * a_20;
  j[1] = ds_10 * a_00 + ds_11 * a_10 + ds_12 * a_20;
  j[2] = ds_20 * a_00 + ds_21 * a_10 + ds_22 * a_20;
  j[3] = ds_00 * a_01 + ds_01 * a_11 + ds_02 * a_21;
  j[4] = ds_10 * a_01 + ds_11 * a_11 + ds_12 * a_21;
  j[5] = ds_20 * a_01 + ds_21 * a_11 + ds_22 * a_21;
  j[6] = ds_00 * a_02 + ds_01 * a_12 + ds_02 * a_22;
  j[7] = ds_10 * a_02 + ds_11 * a_12 + ds_12 * a_22;
  j[8] = ds_20 * a_02 + ds_21 * a_12 + ds_22 * a_22;
}

// J, sigma_1 and R of tet t (compute_tet_transforms_kernel,
// deformation.rs:684-865).
__device__ __forceinline__ void tet_transform(uint32_t t, const float* __restrict__ verts,
                                              const uint4* __restrict__ elems,
                                              const float* __restrict__ inv_dm,
                                              float* __restrict__ J_out, float* __restrict__ R_out,
                                              float* __restrict__ S_out) {
  const uint4 e = elems[t];
  const uint32_t vi[4] = {e.x, e.y, e.z, e.w};
  float x[4][3];
#pragma unroll
  for (int k = 0; k < 4; ++k)
#pragma unroll
    for (int c = 0; c < 3; ++c) x[k][c] = verts[3 * (size_t)vi[k] + c];
  float jm[9];
  tet_jacobian(x, inv_dm + 9 * (size_t)t, jm);
  const float j_00 = jm[0], j_10 = jm[1], j_20 = jm[2];
  const float j_01 = jm[3], j_11 = jm[4], j_21 = jm[5];
  const float j_02 = jm[6], j_12 = jm[7], j_22 = jm[8];
  float* J = J_out + 9 * (size_t)t;
  J[0] = j_00; J[1] = j_10; J[2] = j_20; J[3] = j_01; J[4] = j_11; J[5] = j_21;
  J[6] = j_02; J[7] = j_12; J[8] = j_22;

  // Largest singular value: sqrt of the largest eigenvalue of C = J^T J.
  const float c00 = j_00 * j_00 + j_10 * j_10 + j_20 * j_20;
  const float c01 = j_00 * j_01 + j_10 * j_11 + j_20 * j_21;
  const float c02 = j_00 * j_02 + j_10 * j_12 + j_20 * j_22;
  const float c11 = j_01 * j_01 + j_11 * j_11 + j_21 * j_21;
  const float c12 = j_01 * j_02 + j_11 * j_12 + j_21 * j_22;
  const float c22 = j_02 * j_02 + j_12 * j_12 + j_22 * j_22;
  const float p1 = c01 * c01 + c02 * c02 + c12 * c12;
  if (p1 <= 1e-10f) {
    S_out[t] = sqrtf(fmaxf(fmaxf(c00, fmaxf(c11, c22)), 0.0f));
  } else {
    const float q = (c00 + c11 + c22) / 3.0f;
    const float d0 = c00 - q, d1 = c11 - q, d2 = c22 - q;
    const float p2 = d0 * d0 + d1 * d1 + d2 * d2 + 2.0f * p1;
    const float p = sqrtf(fmaxf(p2 / 6.0f, 1e-12f));
    const float inv_p = 1.0f / p;
    const float b00 = d0 * inv_p, b11 = d1 * inv_p, b22 = d2 * inv_p;
    const float b01 = c01 * inv_p, b02 = c02 * inv_p, b12 = c12 * inv_p;
    const float det_b = b00 * (b11 * b22 - b12 * b12) - b01 * (b01 * b22 - b12 * b02) +
                        b02 * (b01 * b12 - b11 * b02);
    const float r = clampf(0.5f * det_b, -1.0f, 1.0f);
    const float phi = cgs_acosf(r) / 3.0f;
    const float eig = q + 2.0f * p * cgs_cosf(phi);
    S_out[t] = sqrtf(fmaxf(eig, 0.0f));
  }

  // Polar rotation by Newton-Schulz steps R <- (R + R^-T) / 2.
  float* R = R_out + 9 * (size_t)t;
  const float det_j = j_00 * (j_11 * j_22 - j_12 * j_21) - j_01 * (j_10 * j_22 - j_12 * j_20) +
                      j_02 * (j_10 * j_21 - j_11 * j_20);
  const float abs_det = fabsf(det_j);
  if (abs_det < 1e-8f) {
    R[0] = 1.0f; R[1] = 0.0f; R[2] = 0.0f; R[3] = 0.0f; R[4] = 1.0f;
    R[5] = 0.0f; R[6] = 0.0f; R[7] = 0.0f; R[8] = 1.0f;
    return;
  }
  const float gamma = cgs_expf(-cgs_logf(abs_det) / 3.0f);
  float r00 = j_00 * gamma, r10 = j_10 * gamma, r20 = j_20 * gamma;
  float r01 = j_01 * gamma, r11 = j_11 * gamma, r21 = j_21 * gamma;
  float r02 = j_02 * gamma, r12 = j_12 * gamma, r22 = j_22 * gamma;
#pragma unroll
  for (int it = 0; it < 5; ++it) {
    const float cof00 = r11 * r22 - r21 * r12;
    const float cof10 = r21 * r02 - r01 * r22;
    const float cof20 = r01 * r12 - r11 * r02;
    const float cof01 = r12 * r20 - r22 * r10;
    const float cof11 = r22 * r00 - r02 * r20;
    const float cof21 = r02 * r10 - r12 * r00;
    const float cof02 = r10 * r21 - r20 * r11;
    const float cof12 = r20 * r01 - r00 * r21;
    const float cof22 = r00 * r11 - r10 * r01;
    const float det_r = r00 * cof00 + r10 * cof10 + r20 * cof20;
    if (fabsf(det_r) > 1e-12f) {
      const float inv_det = 1.0f / det_r;
      r00 = 0.5f * (r00 + cof00 * inv_det);
      r10 = 0.5f * (r10 + cof10 * inv_det);
      r20 = 0.5f * (r20 + cof20 * inv_det);
      r01 = 0.5f * (r01 + cof01 * inv_det);
      r11 = 0.5f * (r11 + cof11 * inv_det);
      r21 = 0.5f * (r21 + cof21 * inv_det);
      r02 = 0.5f * (r02 + cof02 * inv_det);
      r12 = 0.5f * (r12 + cof12 * inv_det);
      r22 = 0.5f * (r22 + cof22 * inv_det);
    }
  }
  const float det_final = r00 * (r11 * r22 - r21 * r12) + r10 * (r21 * r02 - r01 * r22) +
                          r20 * (r01 * r12 - r11 * r02);
  if (det_final < 0.0f) {
    r02 = -r02;
    r12 = -r12;
    r22 = -r22;
  }
  R[0] = r00; R[1] = r10; R[2] = r20; R[3] = r01; R[4] = r11; R[5] = r21;
  R[6] = r02; R[7] = r12; R[8] = r22;
}

__global__ void __launch_bounds__(128) k_tet_transforms(uint32_t T, const float* __restrict__ verts,
                                                        const uint4* __restrict__ elems,
                                                        const float* __restrict__ inv_dm,
                                                        float* __restrict__ J_out,
                                                        float* __restrict__ R_out,
                                                        float* __restrict__ S_out) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < T) tet_transform(t, verts, elems, inv_dm, J_out, R_out, S_out);
}

// 3D Mip filter Sigma + s I with opacity * sqrt(det / det_reg), in the operand
// order of deformation.rs:914-935 (shared by all three call sites).
__device__ __forceinline__ void mip3d(float& xx, float xy, float xz, float& yy, float yz,
                                      float& zz, float& alpha, float mip) {
  const float det_orig = fmaxf(
      xx * (yy * zz - yz * yz) - xy * (xy * zz - xz * yz) + xz * (xy * yz - xz * yy), 1e-24f);
  const float rxx = xx + mip, ryy = yy + mip, rzz = zz + mip;
  const float det_reg = fmaxf(
      rxx * (ryy * rzz - yz * yz) - xy * (xy * rzz - xz * yz) + xz * (xy * yz - xz * ryy),
      det_orig);
  const float comp = sqrtf(clampf(det_orig / det_reg, 0.0f, 1.0f));
  xx = rxx;
  yy = ryy;
  zz = rzz;
  alpha = clampf(alpha * comp, 0.0f, 1.0f);
}

// ---- CPU-path semantics for MVC-bound Gaussians ------------------------------
// The reference deforms polygon-cage (MVC) bindings only on its CPU path
// (PolyCageMesh::deform_scene_cpu, deformation/mvc.rs:564-749), so these
// helpers follow glam 0.28's Mat3 operation order and the f64 eigen-solver of
// math/covariance.rs instead of the GPU tet kernel's.
struct GM3 {
  float c[9];  // column-major: c[3 * col + row]
};
__device__ __forceinline__ GM3 gm3_mul(const GM3& A, const GM3& B) {
  GM3 C;
#pragma unroll
  for (int col = 0; col < 3; ++col)
#pragma unroll
    for (int row = 0; row < 3; ++row)
      C.c[3 * col + row] = (A.c[row] * B.c[3 * col] + A.c[3 + row] * B.c[3 * col + 1]) +
                           A.c[6 + row] * B.c[3 * col + 2];
  return C;
}
__device__ __forceinline__ GM3 gm3_t(const GM3& A) {
  GM3 T;
#pragma unroll
  for (int col = 0; col < 3; ++col)
#pragma unroll
    for (int row = 0; row < 3; ++row) T.c[3 * col + row] = A.c[3 * row + col];
  return T;
}
__device__ __forceinline__ void gcross(const float* a, const float* b, float* o) {
  o[0] = a[1] * b[2] - b[1] * a[2];
  o[1] = a[2] * b[0] - b[2] * a[0];
  o[2] = a[0] * b[1] - b[0] * a[1];
}
__device__ __forceinline__ float gdot(const float* a, const float* b) {
  return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2];
}
__device__ __forceinline__ float gm3_det(const GM3& A) {
  float x[3];
  gcross(A.c, A.c + 3, x);
  return gdot(A.c + 6, x);
}
// Mat3::inverse: cofactor columns by cross products, scaled by 1/det, transposed.
__device__ __forceinline__ GM3 gm3_inverse(const GM3& A) {
  float t0[3], t1[3], t2[3];
  gcross(A.c + 3, A.c + 6, t0);
  gcross(A.c + 6, A.c, t1);
  gcross(A.c, A.c + 3, t2);
  const float inv = 1.0f / gdot(A.c + 6, t2);
  GM3 R;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    R.c[3 * k + 0] = t0[k] * inv;
    R.c[3 * k + 1] = t1[k] * inv;
    R.c[3 * k + 2] = t2[k] * inv;
  }
  return R;
}
// higham_polar_decomposition (deformation/polar.rs:13-42), rotation only.
__device__ GM3 polar_rotation(const GM3& J) {
  GM3 r = {{1, 0, 0, 0, 1, 0, 0, 0, 1}};
  const float det = gm3_det(J);
  if (fabsf(det) < 1e-8f) return r;
  const float gamma = cgs_powf(fabsf(det), -1.0f / 3.0f);
#pragma unroll
  for (int k = 0; k < 9; ++k) r.c[k] = J.c[k] * gamma;
  for (int it = 0; it < 5; ++it) {
    const GM3 rit = gm3_t(gm3_inverse(r));
#pragma unroll
    for (int k = 0; k < 9; ++k) r.c[k] = 0.5f * (r.c[k] + rit.c[k]);
  }
  if (gm3_det(r) < 0.0f)
    for (int k = 6; k < 9; ++k) r.c[k] = -r.c[k];
  return r;
}
// symmetric_eigen_3x3 (math/covariance.rs:181-265): f64 cyclic Jacobi, 12
// sweeps; eigenvalues descending, right-handed basis (columns).
__device__ void sym_eigen3_f64(const float* cov, float* evals, GM3& basis) {
  double a[3][3] = {{cov[0], cov[1], cov[2]}, {cov[1], cov[3], cov[4]}, {cov[2], cov[4], cov[5]}};
  double v[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  for (int sweep = 0; sweep < 12; ++sweep) {
    for (int e = 0; e < 3; ++e) {
      const int p = e == 2 ? 1 : 0, q = e == 0 ? 1 : 2;
      const double apq = a[p][q];
      if (fabs(apq) <= 1e-15) continue;
      const double tau = (a[q][q] - a[p][p]) / (2.0 * apq);
      const double t = tau >= 0.0 ? 1.0 / (tau + sqrt(1.0 + tau * tau))
                                  : -1.0 / (-tau + sqrt(1.0 + tau * tau));
      const double c = 1.0 / sqrt(1.0 + t * t);
      const double s = t * c;
      const double app = a[p][p], aqq = a[q][q];
      a[p][p] = app - t * apq;
      a[q][q] = aqq + t * apq;
      a[p][q] = 0.0;
      a[q][p] = 0.0;
      const int r = 3 - p - q;  // the remaining index
      const double arp = a[r][p], arq = a[r][q];
      a[r][p] = c * arp - s * arq;
      a[p][r] = a[r][p];
      a[r][q] = s * arp + c * arq;
      a[q][r] = a[r][q];
      for (int k = 0; k < 3; ++k) {
        const double vrp = v[k][p], vrq = v[k][q];
        v[k][p] = c * vrp - s * vrq;
        v[k][q] = s * vrp + c * vrq;
      }
    }
  }
  double ev[3] = {a[0][0], a[1][1], a[2][2]};
  double vec[3][3];
  for (int k = 0; k < 3; ++k) {
    const double x = v[0][k], y = v[1][k], z = v[2][k];
    const double inv = 1.0 / sqrt((x * x + y * y) + z * z);
    vec[k][0] = x * inv;
    vec[k][1] = y * inv;
    vec[k][2] = z * inv;
  }
  int ord[3] = {0, 1, 2};  // stable sort by eigenvalue, descending
  for (int i = 1; i < 3; ++i)
    for (int j = i; j > 0 && ev[ord[j - 1]] < ev[ord[j]]; --j) {
      const int t = ord[j];
      ord[j] = ord[j - 1];
      ord[j - 1] = t;
    }
  for (int k = 0; k < 3; ++k) {
    evals[k] = (float)ev[ord[k]];
    for (int j = 0; j < 3; ++j) basis.c[3 * k + j] = (float)vec[ord[k]][j];
  }
  if (gm3_det(basis) < 0.0f)
    for (int j = 0; j < 3; ++j) basis.c[6 + j] = -basis.c[6 + j];
}
// covariance_determinant (math/covariance.rs:113-123) in f64, rounded to f32.
__device__ __forceinline__ float cov_det_f64(const float* c) {
  const double xx = c[0], xy = c[1], xz = c[2], yy = c[3], yz = c[4], zz = c[5];
  return (float)(xx * (yy * zz - yz * yz) - xy * (xy * zz - xz * yz) + xz * (xy * yz - xz * yy));
}
// apply_mip_filter_3d (math/covariance.rs:288-305).
__device__ __forceinline__ void mip3d_cpu(float* cov, float& alpha, float var) {
  const float d0 = fmaxf(cov_det_f64(cov), 1e-24f);
  cov[0] = cov[0] + var;
  cov[3] = cov[3] + var;
  cov[5] = cov[5] + var;
  const float dr = fmaxf(cov_det_f64(cov), d0);
  alpha = clampf(alpha * sqrtf(clampf(d0 / dr, 0.0f, 1.0f)), 0.0f, 1.0f);
}

// A Gaussian's Stage 1 inputs (60 B), loaded before the kernel waits for the
// tet transforms so that the first blocks' DRAM reads overlap that wait.
struct DeformIn {
  uint32_t tet_raw;
  float4 rp, rca, w;
  float2 rcb;
};

__device__ __forceinline__ DeformIn deform_load(const DeformArgs& a, uint32_t i) {
  DeformIn g;
  g.tet_raw = a.bind_tet[i];
  g.rp = a.rest_pos[i];
  g.rca = a.rest_cova[i];
  g.rcb = a.rest_covb[i];
  g.w = a.bind_w[i];
  return g;
}

// Deformed position, covariance and opacity of Gaussian i (and of its split
// child: cx, cy, cz) from its loaded inputs.
template <bool SPLIT>
__device__ __forceinline__ void deform_one(const DeformArgs& a, const DeformIn& g, bool& split,
                                           float& cx, float& cy, float& cz, float4& out_pos,
                                           float4& out_cova, float2& out_covb) {
  const uint32_t tet_raw = g.tet_raw;
  const float4 rp = g.rp, rca = g.rca;
  const float2 rcb = g.rcb;
  if (tet_raw == kMvcBound && a.mvc_xf) {
    // Polygon-cage binding (deform_scene_cpu, mvc.rs:616-749): position and
    // F from k_mvc_jacobian, rotation for SH, F S F^T, opacity unchanged.
    const uint32_t slot = __float_as_uint(g.w.x);
    const float4 q0 = a.mvc_xf[3 * (size_t)slot], q1 = a.mvc_xf[3 * (size_t)slot + 1],
                 q2 = a.mvc_xf[3 * (size_t)slot + 2];
    const GM3 Fm = {{q0.w, q1.x, q1.y, q1.z, q1.w, q2.x, q2.y, q2.z, q2.w}};
    const GM3 R = polar_rotation(Fm);
#pragma unroll
    for (int k = 0; k < 9; ++k) a.mvc_R[9 * (size_t)slot + k] = R.c[k];
    const GM3 S = {{rca.x, rca.y, rca.z, rca.y, rca.w, rcb.x, rca.z, rcb.x, rcb.y}};
    const GM3 m = gm3_mul(gm3_mul(Fm, S), gm3_t(Fm));
    float cv[6] = {m.c[0], m.c[1], m.c[2], m.c[4], m.c[5], m.c[8]};
    float alpha = rp.w;
    if (SPLIT && a.split_threshold > 0.0f) {
      // jacobian_singular_values (polar.rs:89-109): sigma_1 of F
      const GM3 C = gm3_mul(gm3_t(Fm), Fm);
      const float packed[6] = {C.c[0], C.c[1], C.c[2], C.c[4], C.c[5], C.c[8]};
      float ev[3];
      GM3 basis;
      sym_eigen3_f64(packed, ev, basis);
      split = sqrtf(fmaxf(ev[0], 0.0f)) > a.split_threshold;
    }
    if (!split) {
      if (a.mip > 0.0f) mip3d_cpu(cv, alpha, a.mip);
      out_pos = make_float4(q0.x, q0.y, q0.z, alpha);
    } else {
      // split_gaussian_along_major_axis (math/covariance.rs:331-378)
      float ev[3];
      GM3 B;
      sym_eigen3_f64(cv, ev, B);
      const float min_var = 1e-4f * 1e-4f;
      const GM3 D = {{fmaxf(ev[0] * 0.25f, min_var), 0, 0, 0, fmaxf(ev[1], min_var), 0, 0, 0,
                      fmaxf(ev[2], min_var)}};
      float ax[3] = {B.c[0], B.c[1], B.c[2]};
      const float len2 = gdot(ax, ax);
      if (len2 > 0.0f) {
        const float inv = 1.0f / sqrtf(len2);
        ax[0] *= inv; ax[1] *= inv; ax[2] *= inv;
      }
      const float om = 0.5f * sqrtf(fmaxf(ev[0], min_var));
      const GM3 cm = gm3_mul(gm3_mul(B, D), gm3_t(B));
      cv[0] = cm.c[0]; cv[1] = cm.c[1]; cv[2] = cm.c[2];
      cv[3] = cm.c[4]; cv[4] = cm.c[5]; cv[5] = cm.c[8];
      if (a.mip > 0.0f) mip3d_cpu(cv, alpha, a.mip);
      const float ox = ax[0] * om, oy = ax[1] * om, oz = ax[2] * om;
      out_pos = make_float4(q0.x + (-ox), q0.y + (-oy), q0.z + (-oz), alpha);
      cx = q0.x + ox;
      cy = q0.y + oy;
      cz = q0.z + oz;
    }
    out_cova = make_float4(cv[0], cv[1], cv[2], cv[3]);
    out_covb = make_float2(cv[4], cv[5]);
  } else if (tet_raw >= a.num_tets) {
    // Unbound: rest pose plus the Mip filter (deformation.rs:899-947).
    float xx = rca.x, xy = rca.y, xz = rca.z, yy = rca.w, yz = rcb.x, zz = rcb.y;
    float alpha = rp.w;
    if (a.mip > 0.0f) mip3d(xx, xy, xz, yy, yz, zz, alpha, a.mip);
    out_pos = make_float4(rp.x, rp.y, rp.z, alpha);
    out_cova = make_float4(xx, xy, xz, yy);
    out_covb = make_float2(yz, zz);
  } else {
    const float4 w = g.w;
    const uint4 e = __ldg(&a.elems[tet_raw]);
    const uint32_t vi[4] = {e.x, e.y, e.z, e.w};
    float x[4][3];
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
      for (int c = 0; c < 3; ++c) x[k][c] = __ldg(a.verts + 3 * (size_t)vi[k] + c);
    const float px = w.x * x[0][0] + w.y * x[1][0] + w.z * x[2][0] + w.w * x[3][0];
    const float py = w.x * x[0][1] + w.y * x[1][1] + w.z * x[2][1] + w.w * x[3][1];
    const float pz = w.x * x[0][2] + w.y * x[1][2] + w.z * x[2][2] + w.w * x[3][2];
    float jm[9];
    if (SPLIT) {
      // the tet blocks' J (this variant waited for them)
      const float* J = a.tet_J + 9 * (size_t)tet_raw;
#pragma unroll
      for (int k = 0; k < 9; ++k) jm[k] = __ldca(J + k);
    } else {
      // J of the Gaussian's tet evaluated here from the vertices just loaded,
      // as the tet blocks evaluate it, so this variant never waits for them
      tet_jacobian(x, a.inv_dm + 9 * (size_t)tet_raw, jm);
    }
    const float j_00 = jm[0], j_10 = jm[1], j_20 = jm[2];
    const float j_01 = jm[3], j_11 = jm[4], j_21 = jm[5];
    const float j_02 = jm[6], j_12 = jm[7], j_22 = jm[8];
    const float s_xx = rca.x, s_xy = rca.y, s_xz = rca.z, s_yy = rca.w, s_yz = rcb.x,
                s_zz = rcb.y;
    const float k_00 = j_00 * s_xx + j_01 * s_xy + j_02 * s_xz;
    const float k_01 = j_00 * s_xy + j_01 * s_yy + j_02 * s_yz;
    const float k_02 = j_00 * s_xz + j_01 * s_yz + j_02 * s_zz;
    const float k_10 = j_10 * s_xx + j_11 * s_xy + j_12 * s_xz;
    const float k_11 = j_10 * s_xy + j_11 * s_yy + j_12 * s_yz;
    const float k_12 = j_10 * s_xz + j_11 * s_yz + j_12 * s_zz;
    const float k_20 = j_20 * s_xx + j_21 * s_xy + j_22 * s_xz;
    const float k_21 = j_20 * s_xy + j_21 * s_yy + j_22 * s_yz;
    const float k_22 = j_20 * s_xz + j_21 * s_yz + j_22 * s_zz;
    const float m00 = fmaxf(1e-4f, k_00 * j_00 + k_01 * j_01 + k_02 * j_02);
    const float m01 = 0.5f * ((k_00 * j_10 + k_01 * j_11 + k_02 * j_12) +
                              (k_10 * j_00 + k_11 * j_01 + k_12 * j_02));
    const float m02 = 0.5f * ((k_00 * j_20 + k_01 * j_21 + k_02 * j_22) +
                              (k_20 * j_00 + k_21 * j_01 + k_22 * j_02));
    const float m11 = fmaxf(1e-4f, k_10 * j_10 + k_11 * j_11 + k_12 * j_12);
    const float m12 = 0.5f * ((k_10 * j_20 + k_11 * j_21 + k_12 * j_22) +
                              (k_20 * j_10 + k_21 * j_11 + k_22 * j_12));
    const float m22 = fmaxf(1e-4f, k_20 * j_20 + k_21 * j_21 + k_22 * j_22);
    const float det_j = j_00 * (j_11 * j_22 - j_12 * j_21) -
                        j_01 * (j_10 * j_22 - j_12 * j_20) + j_02 * (j_10 * j_21 - j_11 * j_20);
    const float s_det = clampf(det_j, 0.6f, 1.8f);
    const float safe_base = clampf(1.0f - rp.w, 1e-4f, 0.999f);
    const float alpha_prime = clampf(1.0f - cgs_powf(safe_base, 1.0f / s_det), 0.05f, 0.99f);
    split = SPLIT && a.split_threshold > 0.0f && __ldca(&a.tet_stretch[tet_raw]) > a.split_threshold;
    if (!split) {
      float xx = m00, yy = m11, zz = m22, alpha = alpha_prime;
      if (a.mip > 0.0f) mip3d(xx, m01, m02, yy, m12, zz, alpha, a.mip);
      out_pos = make_float4(px, py, pz, alpha);
      out_cova = make_float4(xx, m01, m02, yy);
      out_covb = make_float2(m12, zz);
    } else {
      // Major eigenpair of M by Cardano + cross products (deformation.rs:1066-1143).
      const float p1 = m01 * m01 + m02 * m02 + m12 * m12;
      float lambda0 = fmaxf(m00, fmaxf(m11, m22));
      float ux = 1.0f, uy = 0.0f, uz = 0.0f;
      if (p1 <= 1e-10f) {
        if (m11 >= m00 && m11 >= m22) {
          ux = 0.0f; uy = 1.0f; uz = 0.0f;
        } else if (m22 >= m00 && m22 >= m11) {
          ux = 0.0f; uy = 0.0f; uz = 1.0f;
        }
      } else {
        const float q = (m00 + m11 + m22) / 3.0f;
        const float d0 = m00 - q, d1 = m11 - q, d2 = m22 - q;
        const float p2 = d0 * d0 + d1 * d1 + d2 * d2 + 2.0f * p1;
        const float p = sqrtf(fmaxf(p2 / 6.0f, 1e-12f));
        const float inv_p = 1.0f / p;
        const float b00 = d0 * inv_p, b11 = d1 * inv_p, b22 = d2 * inv_p;
        const float b01 = m01 * inv_p, b02 = m02 * inv_p, b12 = m12 * inv_p;
        const float det_b = b00 * (b11 * b22 - b12 * b12) - b01 * (b01 * b22 - b12 * b02) +
                            b02 * (b01 * b12 - b11 * b02);
        const float r = clampf(0.5f * det_b, -1.0f, 1.0f);
        const float phi = cgs_acosf(r) / 3.0f;
        lambda0 = q + 2.0f * p * cgs_cosf(phi);
        const float r0x = m00 - lambda0, r0y = m01, r0z = m02;
        const float r1x = m01, r1y = m11 - lambda0, r1z = m12;
        const float r2x = m02, r2y = m12, r2z = m22 - lambda0;
        const float c01x = r0y * r1z - r0z * r1y, c01y = r0z * r1x - r0x * r1z,
                    c01z = r0x * r1y - r0y * r1x;
        const float n01 = c01x * c01x + c01y * c01y + c01z * c01z;
        const float c12x = r1y * r2z - r1z * r2y, c12y = r1z * r2x - r1x * r2z,
                    c12z = r1x * r2y - r1y * r2x;
        const float n12 = c12x * c12x + c12y * c12y + c12z * c12z;
        const float c02x = r0y * r2z - r0z * r2y, c02y = r0z * r2x - r0x * r2z,
                    c02z = r0x * r2y - r0y * r2x;
        const float n02 = c02x * c02x + c02y * c02y + c02z * c02z;
        if (n01 >= n12 && n01 >= n02 && n01 > 1e-12f) {
          const float inv = 1.0f / sqrtf(n01);
          ux = c01x * inv; uy = c01y * inv; uz = c01z * inv;
        } else if (n12 >= n02 && n12 > 1e-12f) {
          const float inv = 1.0f / sqrtf(n12);
          ux = c12x * inv; uy = c12y * inv; uz = c12z * inv;
        } else if (n02 > 1e-12f) {
          const float inv = 1.0f / sqrtf(n02);
          ux = c02x * inv; uy = c02y * inv; uz = c02z * inv;
        }
      }
      const float safe_l0 = fmaxf(lambda0, 1e-8f);
      const float offset_mag = 0.5f * sqrtf(safe_l0);
      const float dx = ux * offset_mag, dy = uy * offset_mag, dz = uz * offset_mag;
      const float shrink = 0.75f * safe_l0;
      float c00 = fmaxf(1e-8f, m00 - shrink * ux * ux);
      const float c01 = m01 - shrink * ux * uy;
      const float c02 = m02 - shrink * ux * uz;
      float c11 = fmaxf(1e-8f, m11 - shrink * uy * uy);
      const float c12 = m12 - shrink * uy * uz;
      float c22 = fmaxf(1e-8f, m22 - shrink * uz * uz);
      float child_alpha = alpha_prime;
      if (a.mip > 0.0f) mip3d(c00, c01, c02, c11, c12, c22, child_alpha, a.mip);
      out_pos = make_float4(px - dx, py - dy, pz - dz, child_alpha);
      out_cova = make_float4(c00, c01, c02, c11);
      out_covb = make_float2(c12, c22);
      cx = px + dx;
      cy = py + dy;
      cz = pz + dz;
    }
  }
}

template <bool SPLIT>
__global__ void __launch_bounds__(kDeformThreads, 4) k_deform(DeformArgs a) {
  __shared__ uint32_t s_tile;
  __shared__ uint32_t s_warp_sums[32];
  __shared__ uint32_t s_base;
  // Tickets in launch order: the first tet_blocks tickets compute the tet
  // transforms, the others are Gaussian tiles in increasing order (the chained
  // scan of the split children needs that order; every tile a block waits on
  // belongs to a block that took its ticket earlier, so it is resident).
  if (threadIdx.x == 0) s_tile = atomicAdd(&a.fc->tile_ctr[0], 1u);
  __syncthreads();
  uint32_t tile = s_tile;
  const uint32_t tet_blocks = a.fuse_tets ? (a.num_tets + kDeformThreads - 1) / kDeformThreads : 0u;
  if (tile < tet_blocks) {
    const uint32_t t = tile * kDeformThreads + threadIdx.x;
    if (t < a.num_tets)
      tet_transform(t, a.verts, a.elems, a.inv_dm, a.tet_J, a.tet_R, a.tet_stretch);
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();  // this block's J, R, sigma_1 before its completion count
      atomicAdd(&a.fc->tile_ctr[kTetsDoneCtr], 1u);
    }
    return;
  }
  tile -= tet_blocks;
  if (!SPLIT && tile == 0 && threadIdx.x == 0) *a.split_count = 0u;
  const uint32_t num_tiles = (a.n + kDeformThreads - 1) / kDeformThreads;
  if (tile >= num_tiles) return;
  uint32_t i = tile * kDeformThreads + threadIdx.x;
  DeformIn g{};
  if (i < a.n) g = deform_load(a, i);
  if (SPLIT && tet_blocks) {
    // Wait (bounded) until every tet block has published (the split needs
    // their sigma_1; without it the Gaussians evaluate their tets' J
    // themselves and the tet blocks only serve the later stages); the tet data is
    // then read with ld.global.ca (L1-cached, ordered after the acquire; no
    // SM has cached those lines earlier in this launch, and L1 holds no lines
    // from earlier launches), never through the incoherent read-only path. A
    // few hundred tets' J are read by every Gaussian: served from L1 instead
    // of hammering the same L2 lines.
    if (threadIdx.x == 0) {
      uint32_t spins = 0;
      while (ld_acquire_u32(&a.fc->tile_ctr[kTetsDoneCtr]) < tet_blocks) {
        if (++spins > kSpinLimit) {
          atomicOr(&a.fc->status, kStatusLookbackTimeout);
          break;
        }
        __nanosleep(64);
      }
    }
    __syncthreads();
  }
  if (!SPLIT) {
    // Persistent: the launch's Gaussian blocks take tiles tile, tile + stride,
    // ... and load the next tile's inputs before deforming the current one.
    const uint32_t stride = gridDim.x - tet_blocks;
    for (;;) {
      const uint32_t next = tile + stride;
      const uint32_t ni = next * kDeformThreads + threadIdx.x;
      DeformIn gn{};
      if (next < num_tiles && ni < a.n) gn = deform_load(a, ni);
      if (i < a.n) {
        bool split = false;
        float cx, cy, cz;
        float4 out_pos, out_cova;
        float2 out_covb;
        deform_one<false>(a, g, split, cx, cy, cz, out_pos, out_cova, out_covb);
        a.def_pos[i] = out_pos;
        a.def_cova[i] = out_cova;
        a.def_covb[i] = out_covb;
      }
      if (next >= num_tiles) break;
      tile = next;
      i = ni;
      g = gn;
    }
    return;
  }
  bool split = false;
  float cx = 0.0f, cy = 0.0f, cz = 0.0f;
  float4 out_pos = make_float4(0, 0, 0, 0), out_cova = make_float4(0, 0, 0, 0);
  float2 out_covb = make_float2(0, 0);
  if (i < a.n) {
    deform_one<SPLIT>(a, g, split, cx, cy, cz, out_pos, out_cova, out_covb);
    a.def_pos[i] = out_pos;
    a.def_cova[i] = out_cova;
    a.def_covb[i] = out_covb;
  }
  {
    uint32_t agg;
    const uint32_t excl = block_exclusive_sum(split ? 1u : 0u, s_warp_sums, &agg);
    if (threadIdx.x < 32) {
      const uint32_t base = chained_scan_warp(a.status, tile, agg, &a.fc->status);
      if (threadIdx.x == 0) s_base = base;
    }
    __syncthreads();
    const uint32_t base = s_base;
    if (split) {
      const size_t c = (size_t)a.n + base + excl;
      a.def_pos[c] = make_float4(cx, cy, cz, out_pos.w);
      a.def_cova[c] = out_cova;
      a.def_covb[c] = out_covb;
      a.split_meta[base + excl] = make_uint2(i, g.tet_raw);
    }
    if (tile == num_tiles - 1 && threadIdx.x == 0) *a.split_count = base + agg;
  }
}

// Barycentric binding, first tet with violation <= 1e-4 in index order,
// else the least-violating tet (strict <), as TetMesh::bind_point. Tet data
// (first rest vertex + D_m^-1, 12 floats) is staged through shared memory in
// chunks; the block keeps loading chunks while any of its points still searches.
constexpr int kBindThreads = 256;
constexpr int kBindChunk = 1024;

__global__ void __launch_bounds__(kBindThreads) k_bind(BindArgs a) {
  __shared__ float s_tet[kBindChunk * 12];
  const uint32_t i = blockIdx.x * kBindThreads + threadIdx.x;
  float px = 0, py = 0, pz = 0;
  bool searching = i < a.n;
  bool outside = false;
  if (searching) {
    const float4 p = a.points[i];
    px = p.x; py = p.y; pz = p.z;
    if (a.use_bounds) {
      outside = px < a.bmin[0] || px > a.bmax[0] || py < a.bmin[1] || py > a.bmax[1] ||
                pz < a.bmin[2] || pz > a.bmax[2];
      if (outside) searching = false;
    }
  }
  uint32_t found = kInvalid;
  float4 found_w = make_float4(0, 0, 0, 0);
  uint32_t best_tet = 0;
  float best_pen = __uint_as_float(0x7f800000u);
  float4 best_w = make_float4(1.0f, 0.0f, 0.0f, 0.0f);
  for (uint32_t c0 = 0; c0 < a.num_tets; c0 += kBindChunk) {
    if (!__syncthreads_or(searching)) break;
    const uint32_t cn = min((uint32_t)kBindChunk, a.num_tets - c0);
    for (uint32_t k = threadIdx.x; k < cn; k += kBindThreads) {
      const float* x0 = a.tet_x0 + 3 * (size_t)(c0 + k);
      const float* m = a.inv_dm + 9 * (size_t)(c0 + k);
      float* d = s_tet + 12 * k;
      d[0] = x0[0]; d[1] = x0[1]; d[2] = x0[2];
#pragma unroll
      for (int q = 0; q < 9; ++q) d[3 + q] = m[q];
    }
    __syncthreads();
    if (searching) {
      for (uint32_t k = 0; k < cn; ++k) {
        const float* d = s_tet + 12 * k;
        const float dx = px - d[0], dy = py - d[1], dz = pz - d[2];
        // glam Mat3 * Vec3: (c0 * x + c1 * y) + c2 * z
        const float w1 = (d[3] * dx + d[6] * dy) + d[9] * dz;
        const float w2 = (d[4] * dx + d[7] * dy) + d[10] * dz;
        const float w3 = (d[5] * dx + d[8] * dy) + d[11] * dz;
        const float w0 = 1.0f - ((w1 + w2) + w3);
        const float pen = ((fmaxf(-w0, 0.0f) + fmaxf(-w1, 0.0f)) + fmaxf(-w2, 0.0f)) +
                          fmaxf(-w3, 0.0f);
        if (pen <= 1e-4f) {
          found = c0 + k;
          found_w = make_float4(w0, w1, w2, w3);
          searching = false;
          break;
        }
        if (pen < best_pen) {
          best_pen = pen;
          best_tet = c0 + k;
          best_w = make_float4(w0, w1, w2, w3);
        }
      }
    }
    __syncthreads();
  }
  if (i >= a.n) return;
  if (outside) {
    a.bind_tet[i] = kInvalid;
    a.bind_w[i] = make_float4(0, 0, 0, 0);
  } else if (found != kInvalid) {
    a.bind_tet[i] = found;
    a.bind_w[i] = found_w;
  } else if (a.use_bounds && best_pen > 0.15f) {
    a.bind_tet[i] = kInvalid;
    a.bind_w[i] = make_float4(0, 0, 0, 0);
  } else if (a.num_tets == 0) {
    a.bind_tet[i] = kInvalid;
    a.bind_w[i] = make_float4(0, 0, 0, 0);
  } else {
    a.bind_tet[i] = best_tet;
    a.bind_w[i] = best_w;
  }
}

}  // namespace

cudaError_t launch_tet_transforms(const DeformArgs& a, cudaStream_t s) {
  if (a.num_tets == 0) return cudaSuccess;
  k_tet_transforms<<<(a.num_tets + 127) / 128, 128, 0, s>>>(a.num_tets, a.verts, a.elems,
                                                            a.inv_dm, a.tet_J, a.tet_R,
                                                            a.tet_stretch);
  return cudaGetLastError();
}

cudaError_t launch_deform(const DeformArgs& a, cudaStream_t s) {
  if (a.n == 0) return a.fuse_tets ? launch_tet_transforms(a, s) : cudaSuccess;
  const uint32_t tet_blocks = a.fuse_tets ? (a.num_tets + kDeformThreads - 1) / kDeformThreads : 0u;
  const uint32_t num_tiles = (a.n + kDeformThreads - 1) / kDeformThreads;
  if (a.split_threshold > 0.0f) {
    // one tile per block: the children's chained scan runs over the tiles
    k_deform<true><<<num_tiles + tet_blocks, kDeformThreads, 0, s>>>(a);
    return cudaGetLastError();
  }
  // Persistent Gaussian blocks: as many as the SMs hold beside the tet blocks.
  static int resident = 0;
  if (resident == 0) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess)
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_deform<false>, kDeformThreads, 0);
    if (e != cudaSuccess) return e;
    resident = std::max(1, sms * per_sm);
  }
  const uint32_t gauss_blocks =
      std::max<uint32_t>(1u, std::min<uint32_t>(num_tiles, (uint32_t)std::max<int>(1, resident - (int)tet_blocks)));
  k_deform<false><<<gauss_blocks + tet_blocks, kDeformThreads, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_bind(const BindArgs& a, cudaStream_t s) {
  if (a.n == 0) return cudaSuccess;
  k_bind<<<(a.n + kBindThreads - 1) / kBindThreads, kBindThreads, 0, s>>>(a);
  return cudaGetLastError();
}

}  // namespace cgs
