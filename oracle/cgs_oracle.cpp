// CPU oracle for the four-stage splat pipeline -- TEST INFRASTRUCTURE ONLY.
//
// This file restates the algorithms of the reference crate (CinderGS v2.0.0,
// Rust) in C++17 so that tests, the smoke check and the CPU-baseline leg of the
// benchmark can check the CUDA library against them. Nothing in the product
// (the cindergs_b200 package and its CUDA library) links, imports or calls it.
//
// Two modes are restated:
//  * "v2": the semantics of the reference's GPU kernels that its
//    GpuPipelineState::execute_frame_gpu wires up (render/kernels/*.rs). These
//    are the parity gates: Stage 3 integers bit-exact, Stage 1/2 floats within
//    1e-5 relative (bit-exact in practice, since both sides evaluate the same
//    IEEE operation sequence and the same deterministic transcendental
//    functions from cindergs_b200/csrc/detmath.h), Stage 4 RGB within 2e-3.
//  * "ref": the reference's own Rayon CPU backend (render_scene_cpu,
//    execute_cpu_reference_with_options): square-radius binning, full f32
//    depth keys, per-pixel SH. Its golden image hash pins this restatement.
//    Transcendentals use glibc, which is what Rust's f32 methods call on Linux.
//
// Build: see oracle/Makefile (-ffp-contract=off keeps every a*b+c unfused).
// Each function cites the reference file:line it follows.

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <numeric>
#include <thread>
#include <vector>

#include "../cindergs_b200/csrc/detmath.h"

namespace {

int g_threads = 0;

int num_threads() {
  if (g_threads > 0) return g_threads;
  unsigned h = std::thread::hardware_concurrency();
  return h == 0 ? 1 : (int)h;
}

// Static-chunk parallel loop over [0, n): the structure of parallel.rs's
// map_range / zip_fill_4 (chunked, order-independent per-element work).
void parallel_for(size_t n, const std::function<void(size_t, size_t)>& body) {
  int t = num_threads();
  if (n < 4096 || t <= 1) {
    body(0, n);
    return;
  }
  size_t chunks = (size_t)t * 4;
  size_t step = (n + chunks - 1) / chunks;
  std::atomic<size_t> next{0};
  std::vector<std::thread> pool;
  for (int k = 0; k < t; ++k) {
    pool.emplace_back([&]() {
      for (;;) {
        size_t c = next.fetch_add(1);
        size_t b = c * step;
        if (b >= n) break;
        body(b, std::min(n, b + step));
      }
    });
  }
  for (auto& th : pool) th.join();
}

inline float clampf(float x, float lo, float hi) { return std::fmin(std::fmax(x, lo), hi); }
inline uint32_t f2u(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }
inline float u2f(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }

// ---------------------------------------------------------------- v2 Stage 1
// compute_tet_transforms_kernel (render/kernels/deformation.rs:684-865).
void tet_transform_one(const float* verts, const uint32_t* e, const float* a, float* J, float* R,
                       float* stretch) {
  const float* x0 = verts + 3 * e[0];
  const float* x1 = verts + 3 * e[1];
  const float* x2 = verts + 3 * e[2];
  const float* x3 = verts + 3 * e[3];
  float ds_00 = x1[0] - x0[0], ds_10 = x1[1] - x0[1], ds_20 = x1[2] - x0[2];
  float ds_01 = x2[0] - x0[0], ds_11 = x2[1] - x0[1], ds_21 = x2[2] - x0[2];
  float ds_02 = x3[0] - x0[0], ds_12 = x3[1] - x0[1], ds_22 = x3[2] - x0[2];
  float a_00 = a[0], a_10 = a[1], a_20 = a[2], a_01 = a[3], a_11 = a[4], a_21 = a[5];
  float a_02 = a[6], a_12 = a[7], a_22 = a[8];
  float j_00 = ds_00 * a_00 + ds_01 * a_10 + ds_02 * a_20;
  float j_10 = ds_10 * a_00 + ds_11 * a_10 + ds_12 * a_20;
  float j_20 = ds_20 * a_00 + ds_21 * a_10 + ds_22 * a_20;
  float j_01 = ds_00 * a_01 + ds_01 * a_11 + ds_02 * a_21;
  float j_11 = ds_10 * a_01 + ds_11 * a_11 + ds_12 * a_21;
  float j_21 = ds_20 * a_01 + ds_21 * a_11 + ds_22 * a_21;
  float j_02 = ds_00 * a_02 + ds_01 * a_12 + ds_02 * a_22;
  float j_12 = ds_10 * a_02 + ds_11 * a_12 + ds_12 * a_22;
  float j_22 = ds_20 * a_02 + ds_21 * a_12 + ds_22 * a_22;
  J[0] = j_00; J[1] = j_10; J[2] = j_20; J[3] = j_01; J[4] = j_11; J[5] = j_21;
  J[6] = j_02; J[7] = j_12; J[8] = j_22;

  float c00 = j_00 * j_00 + j_10 * j_10 + j_20 * j_20;
  float c01 = j_00 * j_01 + j_10 * j_11 + j_20 * j_21;
  float c02 = j_00 * j_02 + j_10 * j_12 + j_20 * j_22;
  float c11 = j_01 * j_01 + j_11 * j_11 + j_21 * j_21;
  float c12 = j_01 * j_02 + j_11 * j_12 + j_21 * j_22;
  float c22 = j_02 * j_02 + j_12 * j_12 + j_22 * j_22;
  float p1 = c01 * c01 + c02 * c02 + c12 * c12;
  if (p1 <= 1e-10f) {
    float dmax = std::fmax(c00, std::fmax(c11, c22));
    *stretch = std::sqrt(std::fmax(dmax, 0.0f));
  } else {
    float q = (c00 + c11 + c22) / 3.0f;
    float d0 = c00 - q, d1 = c11 - q, d2 = c22 - q;
    float p2 = d0 * d0 + d1 * d1 + d2 * d2 + 2.0f * p1;
    float p = std::sqrt(std::fmax(p2 / 6.0f, 1e-12f));
    float inv_p = 1.0f / p;
    float b00 = d0 * inv_p, b11 = d1 * inv_p, b22 = d2 * inv_p;
    float b01 = c01 * inv_p, b02 = c02 * inv_p, b12 = c12 * inv_p;
    float det_b = b00 * (b11 * b22 - b12 * b12) - b01 * (b01 * b22 - b12 * b02) +
                  b02 * (b01 * b12 - b11 * b02);
    float r = clampf(0.5f * det_b, -1.0f, 1.0f);
    float phi = cgs_acosf(r) / 3.0f;
    float eig = q + 2.0f * p * cgs_cosf(phi);
    *stretch = std::sqrt(std::fmax(eig, 0.0f));
  }

  float det_j = j_00 * (j_11 * j_22 - j_12 * j_21) - j_01 * (j_10 * j_22 - j_12 * j_20) +
                j_02 * (j_10 * j_21 - j_11 * j_20);
  float abs_det = std::fabs(det_j);
  if (abs_det < 1e-8f) {
    const float id[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    std::memcpy(R, id, sizeof(id));
    return;
  }
  float gamma = cgs_expf(-cgs_logf(abs_det) / 3.0f);
  float r00 = j_00 * gamma, r10 = j_10 * gamma, r20 = j_20 * gamma;
  float r01 = j_01 * gamma, r11 = j_11 * gamma, r21 = j_21 * gamma;
  float r02 = j_02 * gamma, r12 = j_12 * gamma, r22 = j_22 * gamma;
  for (int it = 0; it < 5; ++it) {
    float cof00 = r11 * r22 - r21 * r12;
    float cof10 = r21 * r02 - r01 * r22;
    float cof20 = r01 * r12 - r11 * r02;
    float cof01 = r12 * r20 - r22 * r10;
    float cof11 = r22 * r00 - r02 * r20;
    float cof21 = r02 * r10 - r12 * r00;
    float cof02 = r10 * r21 - r20 * r11;
    float cof12 = r20 * r01 - r00 * r21;
    float cof22 = r00 * r11 - r10 * r01;
    float det_r = r00 * cof00 + r10 * cof10 + r20 * cof20;
    if (std::fabs(det_r) > 1e-12f) {
      float inv_det = 1.0f / det_r;
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
  float det_final = r00 * (r11 * r22 - r21 * r12) + r10 * (r21 * r02 - r01 * r22) +
                    r20 * (r01 * r12 - r11 * r02);
  if (det_final < 0.0f) {
    r02 = -r02;
    r12 = -r12;
    r22 = -r22;
  }
  R[0] = r00; R[1] = r10; R[2] = r20; R[3] = r01; R[4] = r11; R[5] = r21;
  R[6] = r02; R[7] = r12; R[8] = r22;
}

// 3D Mip filter on a packed covariance, in the operand order of
// deformation.rs:914-935 / :1031-1047 / :1150-1165 (det of the regularised
// matrix re-uses the off-diagonal terms unchanged).
inline void mip3d(float& xx, float xy, float xz, float& yy, float yz, float& zz, float& alpha,
                  float mip) {
  float det_orig = std::fmax(
      xx * (yy * zz - yz * yz) - xy * (xy * zz - xz * yz) + xz * (xy * yz - xz * yy), 1e-24f);
  float rxx = xx + mip, ryy = yy + mip, rzz = zz + mip;
  float det_reg = std::fmax(
      rxx * (ryy * rzz - yz * yz) - xy * (xy * rzz - xz * yz) + xz * (xy * yz - xz * ryy),
      det_orig);
  float comp = std::sqrt(clampf(det_orig / det_reg, 0.0f, 1.0f));
  xx = rxx;
  yy = ryy;
  zz = rzz;
  alpha = clampf(alpha * comp, 0.0f, 1.0f);
}

struct DeformOut {
  float pos[3], cov[6], opa;
  bool split;
  float cpos[3];  // second child
};

// deform_and_split_compact_kernel (render/kernels/deformation.rs:874-1211),
// per Gaussian.
DeformOut deform_one(size_t idx, uint32_t T, const float* verts, const uint32_t* elems,
                     const float* Jall, const float* stretch, const uint32_t* bind_tet,
                     const float* bind_w, const float* rest_pos, const float* rest_cov,
                     const float* rest_opa, float split_thr, float mip) {
  DeformOut o{};
  uint32_t tet_raw = bind_tet[idx];
  const float* rc = rest_cov + 6 * idx;
  if (tet_raw >= T) {
    for (int k = 0; k < 3; ++k) o.pos[k] = rest_pos[3 * idx + k];
    float xx = rc[0], xy = rc[1], xz = rc[2], yy = rc[3], yz = rc[4], zz = rc[5];
    float alpha = rest_opa[idx];
    if (mip > 0.0f) mip3d(xx, xy, xz, yy, yz, zz, alpha, mip);
    o.cov[0] = xx; o.cov[1] = xy; o.cov[2] = xz; o.cov[3] = yy; o.cov[4] = yz; o.cov[5] = zz;
    o.opa = alpha;
    return o;
  }
  const float* w = bind_w + 4 * idx;
  const uint32_t* e = elems + 4 * tet_raw;
  const float* v0 = verts + 3 * e[0];
  const float* v1 = verts + 3 * e[1];
  const float* v2 = verts + 3 * e[2];
  const float* v3 = verts + 3 * e[3];
  float px = w[0] * v0[0] + w[1] * v1[0] + w[2] * v2[0] + w[3] * v3[0];
  float py = w[0] * v0[1] + w[1] * v1[1] + w[2] * v2[1] + w[3] * v3[1];
  float pz = w[0] * v0[2] + w[1] * v1[2] + w[2] * v2[2] + w[3] * v3[2];
  const float* J = Jall + 9 * tet_raw;
  float j_00 = J[0], j_10 = J[1], j_20 = J[2], j_01 = J[3], j_11 = J[4], j_21 = J[5];
  float j_02 = J[6], j_12 = J[7], j_22 = J[8];
  float s_xx = rc[0], s_xy = rc[1], s_xz = rc[2], s_yy = rc[3], s_yz = rc[4], s_zz = rc[5];
  float k_00 = j_00 * s_xx + j_01 * s_xy + j_02 * s_xz;
  float k_01 = j_00 * s_xy + j_01 * s_yy + j_02 * s_yz;
  float k_02 = j_00 * s_xz + j_01 * s_yz + j_02 * s_zz;
  float k_10 = j_10 * s_xx + j_11 * s_xy + j_12 * s_xz;
  float k_11 = j_10 * s_xy + j_11 * s_yy + j_12 * s_yz;
  float k_12 = j_10 * s_xz + j_11 * s_yz + j_12 * s_zz;
  float k_20 = j_20 * s_xx + j_21 * s_xy + j_22 * s_xz;
  float k_21 = j_20 * s_xy + j_21 * s_yy + j_22 * s_yz;
  float k_22 = j_20 * s_xz + j_21 * s_yz + j_22 * s_zz;
  float m00 = std::fmax(1e-4f, k_00 * j_00 + k_01 * j_01 + k_02 * j_02);
  float m01 = 0.5f * ((k_00 * j_10 + k_01 * j_11 + k_02 * j_12) +
                      (k_10 * j_00 + k_11 * j_01 + k_12 * j_02));
  float m02 = 0.5f * ((k_00 * j_20 + k_01 * j_21 + k_02 * j_22) +
                      (k_20 * j_00 + k_21 * j_01 + k_22 * j_02));
  float m11 = std::fmax(1e-4f, k_10 * j_10 + k_11 * j_11 + k_12 * j_12);
  float m12 = 0.5f * ((k_10 * j_20 + k_11 * j_21 + k_12 * j_22) +
                      (k_20 * j_10 + k_21 * j_11 + k_22 * j_12));
  float m22 = std::fmax(1e-4f, k_20 * j_20 + k_21 * j_21 + k_22 * j_22);
  float det_j = j_00 * (j_11 * j_22 - j_12 * j_21) - j_01 * (j_10 * j_22 - j_12 * j_20) +
                j_02 * (j_10 * j_21 - j_11 * j_20);
  float s_det = clampf(det_j, 0.6f, 1.8f);
  float safe_base = clampf(1.0f - rest_opa[idx], 1e-4f, 0.999f);
  float alpha_prime = clampf(1.0f - cgs_powf(safe_base, 1.0f / s_det), 0.05f, 0.99f);
  bool should_split = split_thr > 0.0f && stretch[tet_raw] > split_thr;
  if (!should_split) {
    o.pos[0] = px; o.pos[1] = py; o.pos[2] = pz;
    float a = alpha_prime;
    float xx = m00, yy = m11, zz = m22;
    if (mip > 0.0f) mip3d(xx, m01, m02, yy, m12, zz, a, mip);
    o.cov[0] = xx; o.cov[1] = m01; o.cov[2] = m02; o.cov[3] = yy; o.cov[4] = m12; o.cov[5] = zz;
    o.opa = a;
    return o;
  }
  float p1 = m01 * m01 + m02 * m02 + m12 * m12;
  float lambda0 = std::fmax(m00, std::fmax(m11, m22));
  float ux = 1.0f, uy = 0.0f, uz = 0.0f;
  if (p1 <= 1e-10f) {
    if (m11 >= m00 && m11 >= m22) {
      ux = 0.0f; uy = 1.0f; uz = 0.0f;
    } else if (m22 >= m00 && m22 >= m11) {
      ux = 0.0f; uy = 0.0f; uz = 1.0f;
    }
  } else {
    float q = (m00 + m11 + m22) / 3.0f;
    float d0 = m00 - q, d1 = m11 - q, d2 = m22 - q;
    float p2 = d0 * d0 + d1 * d1 + d2 * d2 + 2.0f * p1;
    float p = std::sqrt(std::fmax(p2 / 6.0f, 1e-12f));
    float inv_p = 1.0f / p;
    float b00 = d0 * inv_p, b11 = d1 * inv_p, b22 = d2 * inv_p;
    float b01 = m01 * inv_p, b02 = m02 * inv_p, b12 = m12 * inv_p;
    float det_b = b00 * (b11 * b22 - b12 * b12) - b01 * (b01 * b22 - b12 * b02) +
                  b02 * (b01 * b12 - b11 * b02);
    float r = clampf(0.5f * det_b, -1.0f, 1.0f);
    float phi = cgs_acosf(r) / 3.0f;
    lambda0 = q + 2.0f * p * cgs_cosf(phi);
    float r0x = m00 - lambda0, r0y = m01, r0z = m02;
    float r1x = m01, r1y = m11 - lambda0, r1z = m12;
    float r2x = m02, r2y = m12, r2z = m22 - lambda0;
    float c01x = r0y * r1z - r0z * r1y, c01y = r0z * r1x - r0x * r1z, c01z = r0x * r1y - r0y * r1x;
    float n01 = c01x * c01x + c01y * c01y + c01z * c01z;
    float c12x = r1y * r2z - r1z * r2y, c12y = r1z * r2x - r1x * r2z, c12z = r1x * r2y - r1y * r2x;
    float n12 = c12x * c12x + c12y * c12y + c12z * c12z;
    float c02x = r0y * r2z - r0z * r2y, c02y = r0z * r2x - r0x * r2z, c02z = r0x * r2y - r0y * r2x;
    float n02 = c02x * c02x + c02y * c02y + c02z * c02z;
    if (n01 >= n12 && n01 >= n02 && n01 > 1e-12f) {
      float inv = 1.0f / std::sqrt(n01);
      ux = c01x * inv; uy = c01y * inv; uz = c01z * inv;
    } else if (n12 >= n02 && n12 > 1e-12f) {
      float inv = 1.0f / std::sqrt(n12);
      ux = c12x * inv; uy = c12y * inv; uz = c12z * inv;
    } else if (n02 > 1e-12f) {
      float inv = 1.0f / std::sqrt(n02);
      ux = c02x * inv; uy = c02y * inv; uz = c02z * inv;
    }
  }
  float safe_l0 = std::fmax(lambda0, 1e-8f);
  float offset_mag = 0.5f * std::sqrt(safe_l0);
  float dx = ux * offset_mag, dy = uy * offset_mag, dz = uz * offset_mag;
  float shrink = 0.75f * safe_l0;
  float c00 = std::fmax(1e-8f, m00 - shrink * ux * ux);
  float c01 = m01 - shrink * ux * uy;
  float c02 = m02 - shrink * ux * uz;
  float c11 = std::fmax(1e-8f, m11 - shrink * uy * uy);
  float c12 = m12 - shrink * uy * uz;
  float c22 = std::fmax(1e-8f, m22 - shrink * uz * uz);
  float child_alpha = alpha_prime;
  if (mip > 0.0f) {
    // deformation.rs:1150-1165: here the regularised determinant also uses
    // the updated diagonal, which mip3d() reproduces.
    mip3d(c00, c01, c02, c11, c12, c22, child_alpha, mip);
  }
  o.pos[0] = px - dx; o.pos[1] = py - dy; o.pos[2] = pz - dz;
  o.cov[0] = c00; o.cov[1] = c01; o.cov[2] = c02; o.cov[3] = c11; o.cov[4] = c12; o.cov[5] = c22;
  o.opa = child_alpha;
  o.split = true;
  o.cpos[0] = px + dx; o.cpos[1] = py + dy; o.cpos[2] = pz + dz;
  return o;
}

// ---------------------------------------------------------------- v2 Stage 2
// eval_sh_f32 (render/kernels/project.rs:798-895).
void eval_sh(const float* c, float dx, float dy, float dz, uint32_t deg, float* rgb) {
  float r = 0.28209479177387814f * c[0];
  float g = 0.28209479177387814f * c[1];
  float b = 0.28209479177387814f * c[2];
  if (deg >= 1) {
    float y1_m1 = -0.4886025119029199f * dy;
    float y1_0 = 0.4886025119029199f * dz;
    float y1_p1 = -0.4886025119029199f * dx;
    r += y1_m1 * c[3] + y1_0 * c[4] + y1_p1 * c[5];
    g += y1_m1 * c[18] + y1_0 * c[19] + y1_p1 * c[20];
    b += y1_m1 * c[33] + y1_0 * c[34] + y1_p1 * c[35];
    if (deg >= 2) {
      float xx = dx * dx, yy = dy * dy, zz = dz * dz;
      float xy = dx * dy, yz = dy * dz, xz = dx * dz;
      float y2_m2 = 1.0925484305920792f * xy;
      float y2_m1 = -1.0925484305920792f * yz;
      float y2_0 = 0.31539156525252005f * (2.0f * zz - xx - yy);
      float y2_p1 = -1.0925484305920792f * xz;
      float y2_p2 = 0.5462742152960396f * (xx - yy);
      r += y2_m2 * c[6] + y2_m1 * c[7] + y2_0 * c[8] + y2_p1 * c[9] + y2_p2 * c[10];
      g += y2_m2 * c[21] + y2_m1 * c[22] + y2_0 * c[23] + y2_p1 * c[24] + y2_p2 * c[25];
      b += y2_m2 * c[36] + y2_m1 * c[37] + y2_0 * c[38] + y2_p1 * c[39] + y2_p2 * c[40];
      if (deg >= 3) {
        float y3_m3 = -0.5900435899266435f * dy * (3.0f * xx - yy);
        float y3_m2 = 2.890611442640554f * xy * dz;
        float y3_m1 = -0.4570457994644658f * dy * (4.0f * zz - xx - yy);
        float y3_0 = 0.3731763325901154f * dz * (2.0f * zz - 3.0f * xx - 3.0f * yy);
        float y3_p1 = -0.4570457994644658f * dx * (4.0f * zz - xx - yy);
        float y3_p2 = 1.445305721320277f * dz * (xx - yy);
        float y3_p3 = -0.5900435899266435f * dx * (xx - 3.0f * yy);
        r += y3_m3 * c[11] + y3_m2 * c[12] + y3_m1 * c[13] + y3_0 * c[14] + y3_p1 * c[15] +
             y3_p2 * c[16] + y3_p3 * c[17];
        g += y3_m3 * c[26] + y3_m2 * c[27] + y3_m1 * c[28] + y3_0 * c[29] + y3_p1 * c[30] +
             y3_p2 * c[31] + y3_p3 * c[32];
        b += y3_m3 * c[41] + y3_m2 * c[42] + y3_m1 * c[43] + y3_0 * c[44] + y3_p1 * c[45] +
             y3_p2 * c[46] + y3_p3 * c[47];
      }
    }
  }
  rgb[0] = clampf(r + 0.5f, 0.0f, 1.0f);
  rgb[1] = clampf(g + 0.5f, 0.0f, 1.0f);
  rgb[2] = clampf(b + 0.5f, 0.0f, 1.0f);
}

// project_gaussians_v2_kernel (render/kernels/project.rs:1020-1289), per splat.
// Returns the packed extents (0 = culled); attrs is written only when visible.
uint32_t project_one(size_t idx, uint32_t n_rest, const float* pos, const float* cov,
                     const float* opa, const float* sh, const uint32_t* bind_tet,
                     const float* tet_R, uint32_t num_tets, const uint32_t* split_meta,
                     const float* cam, const float* cam_pos, float mip, float min_opa,
                     float min_rad, uint32_t sh_degree, uint32_t has_deform, float* attrs) {
  const float w00 = cam[0], w10 = cam[1], w20 = cam[2];
  const float w01 = cam[4], w11 = cam[5], w21 = cam[6];
  const float w02 = cam[8], w12 = cam[9], w22 = cam[10];
  const float w03 = cam[12], w13 = cam[13], w23 = cam[14];
  const float fx = cam[16], fy = cam[17], cx = cam[18], cy = cam[19];
  const float vw = cam[20], vh = cam[21], near_p = cam[22];
  float px = pos[3 * idx], py = pos[3 * idx + 1], pz = pos[3 * idx + 2];
  float tx = w00 * px + w01 * py + w02 * pz + w03;
  float ty = w10 * px + w11 * py + w12 * pz + w13;
  float tz = w20 * px + w21 * py + w22 * pz + w23;
  if (tz <= near_p) return 0;
  float op = opa[idx];
  if (op < min_opa) return 0;
  const float* c6 = cov + 6 * idx;
  float v_xx = c6[0], v_xy = c6[1], v_xz = c6[2], v_yy = c6[3], v_yz = c6[4], v_zz = c6[5];
  float alpha_3d = op;
  if (mip > 0.0f) {
    float det_orig = std::fmax(v_xx * (v_yy * v_zz - v_yz * v_yz) -
                                   v_xy * (v_xy * v_zz - v_xz * v_yz) +
                                   v_xz * (v_xy * v_yz - v_xz * v_yy),
                               1e-24f);
    v_xx += mip;
    v_yy += mip;
    v_zz += mip;
    float det_reg = std::fmax(v_xx * (v_yy * v_zz - v_yz * v_yz) -
                                  v_xy * (v_xy * v_zz - v_xz * v_yz) +
                                  v_xz * (v_xy * v_yz - v_xz * v_yy),
                              det_orig);
    float comp = std::sqrt(clampf(det_orig / det_reg, 0.0f, 1.0f));
    alpha_3d = clampf(op * comp, 0.0f, 1.0f);
    if (alpha_3d < min_opa) return 0;
  }
  float k00 = w00 * v_xx + w01 * v_xy + w02 * v_xz;
  float k01 = w00 * v_xy + w01 * v_yy + w02 * v_yz;
  float k02 = w00 * v_xz + w01 * v_yz + w02 * v_zz;
  float k10 = w10 * v_xx + w11 * v_xy + w12 * v_xz;
  float k11 = w10 * v_xy + w11 * v_yy + w12 * v_yz;
  float k12 = w10 * v_xz + w11 * v_yz + w12 * v_zz;
  float k20 = w20 * v_xx + w21 * v_xy + w22 * v_xz;
  float k21 = w20 * v_xy + w21 * v_yy + w22 * v_yz;
  float k22 = w20 * v_xz + w21 * v_yz + w22 * v_zz;
  float cam_xx = k00 * w00 + k01 * w01 + k02 * w02;
  float cam_xy = k00 * w10 + k01 * w11 + k02 * w12;
  float cam_xz = k00 * w20 + k01 * w21 + k02 * w22;
  float cam_yy = k10 * w10 + k11 * w11 + k12 * w12;
  float cam_yz = k10 * w20 + k11 * w21 + k12 * w22;
  float cam_zz = k20 * w20 + k21 * w21 + k22 * w22;
  float inv_tz = 1.0f / tz;
  float inv_tz2 = inv_tz * inv_tz;
  float j00 = fx * inv_tz;
  float j02 = -fx * tx * inv_tz2;
  float j11 = fy * inv_tz;
  float j12 = -fy * ty * inv_tz2;
  float m00 = j00 * cam_xx + j02 * cam_xz;
  float m01 = j00 * cam_xy + j02 * cam_yz;
  float m02 = j00 * cam_xz + j02 * cam_zz;
  float m11 = j11 * cam_yy + j12 * cam_yz;
  float m12 = j11 * cam_yz + j12 * cam_zz;
  float s_xx = m00 * j00 + m02 * j02;
  float s_xy = m01 * j11 + m02 * j12;
  float s_yy = m11 * j11 + m12 * j12;
  float raw_mid = 0.5f * (s_xx + s_yy);
  float raw_det = std::fmax(s_xx * s_yy - s_xy * s_xy, 0.0f);
  float raw_discr = std::sqrt(std::fmax(raw_mid * raw_mid - raw_det, 0.0f));
  float raw_lmax = std::fmax(raw_mid + raw_discr, 0.0f);
  if (3.0f * std::sqrt(raw_lmax) < min_rad) return 0;
  float sp_xx = s_xx + 0.3f, sp_xy = s_xy, sp_yy = s_yy + 0.3f;
  float det = sp_xx * sp_yy - sp_xy * sp_xy;
  if (det <= 1e-6f) return 0;
  float comp_2d = std::sqrt(clampf(raw_det / det, 0.0f, 1.0f));
  float alpha_2d = clampf(alpha_3d * comp_2d, 0.0f, 1.0f);
  if (alpha_2d < min_opa || alpha_2d <= (1.0f / 255.0f)) return 0;
  float q_max = clampf(2.0f * cgs_logf(255.0f * alpha_2d), 0.0f, 8.0f);
  float sigma_cut = std::sqrt(q_max);
  float ext_x = clampf(std::ceil(sigma_cut * std::sqrt(std::fmax(sp_xx, 0.0f))), 1.0f, 1024.0f);
  float ext_y = clampf(std::ceil(sigma_cut * std::sqrt(std::fmax(sp_yy, 0.0f))), 1.0f, 1024.0f);
  float mu_x = fx * tx * inv_tz + cx;
  float mu_y = fy * ty * inv_tz + cy;
  if (mu_x + ext_x < 0.0f || mu_x - ext_x >= vw || mu_y + ext_y < 0.0f || mu_y - ext_y >= vh)
    return 0;
  float inv_det = 1.0f / det;
  float a = sp_yy * inv_det;
  float b = -sp_xy * inv_det;
  float c = sp_xx * inv_det;
  float vx = px - cam_pos[0], vy = py - cam_pos[1], vz = pz - cam_pos[2];
  float inv_len = 1.0f / std::fmax(0.0001f, std::sqrt(vx * vx + vy * vy + vz * vz));
  float dx = vx * inv_len, dy = vy * inv_len, dz = vz * inv_len;
  size_t sh_idx = idx;
  uint32_t tet_raw = num_tets;
  if (idx < n_rest) {
    if (has_deform) tet_raw = bind_tet[idx];
  } else {
    size_t child = idx - n_rest;
    sh_idx = split_meta[2 * child];
    tet_raw = split_meta[2 * child + 1];
  }
  if (has_deform && tet_raw < num_tets) {
    const float* R = tet_R + 9 * (size_t)tet_raw;
    float ldx = R[0] * dx + R[1] * dy + R[2] * dz;
    float ldy = R[3] * dx + R[4] * dy + R[5] * dz;
    float ldz = R[6] * dx + R[7] * dy + R[8] * dz;
    dx = ldx;
    dy = ldy;
    dz = ldz;
  }
  float rgb[3];
  eval_sh(sh + 48 * sh_idx, dx, dy, dz, sh_degree, rgb);
  float* o = attrs + 10 * idx;
  o[0] = mu_x; o[1] = mu_y; o[2] = a; o[3] = b; o[4] = c; o[5] = alpha_2d;
  o[6] = rgb[0]; o[7] = rgb[1]; o[8] = rgb[2]; o[9] = tz;
  return ((uint32_t)ext_x & 0xFFFFu) | (((uint32_t)ext_y & 0xFFFFu) << 16);
}

// ---------------------------------------------------------------- v2 Stage 3
// Screen tile of the v2 Stages 3 and 4: the reference's 16x16 pixels unless
// set otherwise (8x8 and 32x16 are the library's other tile shapes; the
// functions below keep the reference's formulas on the other rectangle).
static uint32_t g_tile_w = 16, g_tile_h = 16;
static uint32_t tiles_across(uint32_t W) { return (W + g_tile_w - 1) / g_tile_w; }
static uint32_t tiles_down(uint32_t H) { return (H + g_tile_h - 1) / g_tile_h; }

// ellipse_intersects_tile_gpu (render/kernels/binning.rs:37-83).
bool ellipse_tile(float mu_x, float mu_y, float ca, float cb, float cc, float alpha, uint32_t tx,
                  uint32_t ty, uint32_t W, uint32_t H) {
  if (alpha < (1.0f / 255.0f) || W == 0 || H == 0) return false;
  uint32_t x_start = tx * g_tile_w, y_start = ty * g_tile_h;
  if (x_start >= W || y_start >= H) return false;
  uint32_t x_end = std::min(x_start + (g_tile_w - 1u), W - 1u);
  uint32_t y_end = std::min(y_start + (g_tile_h - 1u), H - 1u);
  float dx0 = ((float)x_start + 0.5f) - mu_x;
  float dx1 = ((float)x_end + 0.5f) - mu_x;
  float dy0 = ((float)y_start + 0.5f) - mu_y;
  float dy1 = ((float)y_end + 0.5f) - mu_y;
  float x_near = clampf(0.0f, dx0, dx1);
  float y1 = clampf(-cb * x_near / std::fmax(cc, 1e-12f), dy0, dy1);
  float q1 = ca * x_near * x_near + 2.0f * cb * x_near * y1 + cc * y1 * y1;
  float y_near = clampf(0.0f, dy0, dy1);
  float x2 = clampf(-cb * y_near / std::fmax(ca, 1e-12f), dx0, dx1);
  float q2 = ca * x2 * x2 + 2.0f * cb * x2 * y_near + cc * y_near * y_near;
  float min_quad = std::fmin(q1, q2);
  float q_cut = clampf(2.0f * cgs_logf(255.0f * alpha), 0.0f, 8.0f);
  return min_quad <= q_cut + 1e-4f;
}

struct TileBox {
  uint32_t x0, x1, y0, y1;
};

// Tile AABB of count_tiles_kernel / emit_tile_keys_kernel (binning.rs:139-142).
TileBox tile_box(float mu_x, float mu_y, float ext_x, float ext_y, uint32_t tiles_x,
                 uint32_t tiles_y) {
  auto fl = [](float v, int32_t hi, uint32_t tile) {
    float f = std::floor(v / (float)tile);
    int32_t i;
    if (!(f == f)) i = 0;
    else if (f >= 2147483520.0f) i = INT32_MAX;
    else if (f <= -2147483648.0f) i = INT32_MIN;
    else i = (int32_t)f;
    return (uint32_t)std::min(std::max(i, 0), hi);
  };
  int32_t mx = (int32_t)tiles_x - 1, my = (int32_t)tiles_y - 1;
  return {fl(mu_x - ext_x, mx, g_tile_w), fl(mu_x + ext_x, mx, g_tile_w),
          fl(mu_y - ext_y, my, g_tile_h), fl(mu_y + ext_y, my, g_tile_h)};
}

// ------------------------------------------------------------- ref CPU mode
// glam 0.28 operation order for the few composite ops the CPU path uses
// (scalar Mat3 columns, Mat4::transform_point3 as ((x*px + y*py) + z*pz) + w).

// evaluate_sh (render/rasterizer/sh.rs:29-137): same arithmetic as eval_sh
// for a full 48-float slice.

// project_ewa_splat (math/projection.rs:278-345) for view matrix `V`
// (column-major 16). Writes xy, depth, radius, conic.
void project_ewa_ref(const float* p, const float* c6, const float* V, float fx, float fy, float cx,
                     float cy, float vw, float vh, float near_p, float* xy, float* depth,
                     int32_t* radius, float* conic) {
  float tx = ((V[0] * p[0] + V[4] * p[1]) + V[8] * p[2]) + V[12];
  float ty = ((V[1] * p[0] + V[5] * p[1]) + V[9] * p[2]) + V[13];
  float tz = ((V[2] * p[0] + V[6] * p[1]) + V[10] * p[2]) + V[14];
  *depth = tz;
  xy[0] = xy[1] = 0.0f;
  conic[0] = conic[1] = conic[2] = 0.0f;
  *radius = 0;
  if (tz <= near_p) return;
  float inv_tz = 1.0f / tz;
  float inv_tz2 = inv_tz * inv_tz;
  float jac[4] = {fx * inv_tz, -fx * tx * inv_tz2, fy * inv_tz, -fy * ty * inv_tz2};
  // Sigma_cam = (W * Sigma) * W^T with W the upper-left 3x3 (columns V[0..3),
  // V[4..7), V[8..11)); glam Mat3 * Mat3 = columns of (c0*r.x + c1*r.y) + c2*r.z.
  float W[9] = {V[0], V[1], V[2], V[4], V[5], V[6], V[8], V[9], V[10]};
  float S[9] = {c6[0], c6[1], c6[2], c6[1], c6[3], c6[4], c6[2], c6[4], c6[5]};
  auto mul = [](const float* A, const float* B, float* C) {
    for (int col = 0; col < 3; ++col) {
      for (int row = 0; row < 3; ++row) {
        C[3 * col + row] = (A[row] * B[3 * col] + A[3 + row] * B[3 * col + 1]) +
                           A[6 + row] * B[3 * col + 2];
      }
    }
  };
  float WS[9], WT[9], Cm[9];
  mul(W, S, WS);
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) WT[3 * c + r] = W[3 * r + c];
  mul(WS, WT, Cm);
  float c_xx = Cm[0], c_xy = Cm[1], c_xz = Cm[2], c_yy = Cm[4], c_yz = Cm[5], c_zz = Cm[8];
  float j00 = jac[0], j02 = jac[1], j11 = jac[2], j12 = jac[3];
  float m00 = j00 * c_xx + j02 * c_xz;
  float m01 = j00 * c_xy + j02 * c_yz;
  float m02 = j00 * c_xz + j02 * c_zz;
  float m11 = j11 * c_yy + j12 * c_yz;
  float m12 = j11 * c_yz + j12 * c_zz;
  float sxx = m00 * j00 + m02 * j02;
  float sxy = m01 * j11 + m02 * j12;
  float syy = m11 * j11 + m12 * j12;
  // compute_conic_and_radius (projection.rs:143-172)
  float s_xx = sxx + 0.3f, s_xy = sxy, s_yy = syy + 0.3f;
  float det = s_xx * s_yy - s_xy * s_xy;
  if (det <= 1e-6f) return;
  float inv_det = 1.0f / det;
  float cn[3] = {s_yy * inv_det, -s_xy * inv_det, s_xx * inv_det};
  float mid = 0.5f * (s_xx + s_yy);
  float discr = std::sqrt(std::fmax(mid * mid - det, 0.1f));
  float l1 = mid + discr;
  float l2 = std::fmax(mid - discr, 0.1f);
  float lmax = std::fmax(l1, l2);
  float r = clampf(std::ceil(3.0f * std::sqrt(lmax)), 1.0f, 1024.0f);
  float mx = fx * tx * inv_tz + cx;
  float my = fy * ty * inv_tz + cy;
  xy[0] = mx;
  xy[1] = my;
  conic[0] = cn[0];
  conic[1] = cn[1];
  conic[2] = cn[2];
  if (mx + r < 0.0f || mx - r >= vw || my + r < 0.0f || my - r >= vh) {
    *radius = 0;
    return;
  }
  *radius = (int32_t)r;
}

// compute_gaussian_tile_bounds_xy (render/tiles/mod.rs:97-130).
bool tile_bounds_xy(float cxp, float cyp, float ex, float ey, uint32_t tiles_x, uint32_t tiles_y,
                    uint32_t W, uint32_t H, TileBox* out) {
  if (ex <= 0.0f || ey <= 0.0f || tiles_x == 0 || tiles_y == 0) return false;
  float min_x = cxp - ex, max_x = cxp + ex, min_y = cyp - ey, max_y = cyp + ey;
  if (max_x < 0.0f || min_x >= (float)W || max_y < 0.0f || min_y >= (float)H) return false;
  *out = tile_box(cxp, cyp, ex, ey, tiles_x, tiles_y);
  return !(out->x1 < out->x0 || out->y1 < out->y0);
}



// ------------------------------------------------------------- ref CPU frame
// Column-major 3x3 in glam 0.28's scalar Mat3 operation order.
struct M3 {
  float c[9];
  float at(int col, int row) const { return c[3 * col + row]; }
};
inline M3 m3_mul(const M3& A, const M3& B) {
  M3 C;
  for (int col = 0; col < 3; ++col)
    for (int row = 0; row < 3; ++row)
      C.c[3 * col + row] = (A.c[row] * B.c[3 * col] + A.c[3 + row] * B.c[3 * col + 1]) +
                           A.c[6 + row] * B.c[3 * col + 2];
  return C;
}
inline M3 m3_t(const M3& A) {
  M3 T;
  for (int col = 0; col < 3; ++col)
    for (int row = 0; row < 3; ++row) T.c[3 * col + row] = A.c[3 * row + col];
  return T;
}
inline void cross3(const float* a, const float* b, float* o) {
  o[0] = a[1] * b[2] - b[1] * a[2];
  o[1] = a[2] * b[0] - b[2] * a[0];
  o[2] = a[0] * b[1] - b[0] * a[1];
}
inline float dot3(const float* a, const float* b) { return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2]; }
inline float m3_det(const M3& A) {
  float x[3];
  cross3(A.c, A.c + 3, x);
  return dot3(A.c + 6, x);
}
inline M3 m3_inverse(const M3& A) {
  float t0[3], t1[3], t2[3];
  cross3(A.c + 3, A.c + 6, t0);
  cross3(A.c + 6, A.c, t1);
  cross3(A.c, A.c + 3, t2);
  const float det = dot3(A.c + 6, t2);
  const float inv = 1.0f / det;
  M3 R;
  for (int k = 0; k < 3; ++k) {
    R.c[3 * k + 0] = t0[k] * inv;
    R.c[3 * k + 1] = t1[k] * inv;
    R.c[3 * k + 2] = t2[k] * inv;
  }
  return R;
}

// symmetric_eigen_3x3 (math/covariance.rs:181-265): f64 cyclic Jacobi, 12
// sweeps, eigenvalues descending, right-handed basis (columns).
void sym_eigen3(const float* cov, float* evals, M3* basis) {
  double a[3][3] = {{cov[0], cov[1], cov[2]}, {cov[1], cov[3], cov[4]}, {cov[2], cov[4], cov[5]}};
  double v[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  const int pq[3][2] = {{0, 1}, {0, 2}, {1, 2}};
  for (int sweep = 0; sweep < 12; ++sweep) {
    for (auto& e : pq) {
      const int p = e[0], q = e[1];
      const double apq = a[p][q];
      if (std::fabs(apq) <= 1e-15) continue;
      const double tau = (a[q][q] - a[p][p]) / (2.0 * apq);
      const double t = tau >= 0.0 ? 1.0 / (tau + std::sqrt(1.0 + tau * tau))
                                  : -1.0 / (-tau + std::sqrt(1.0 + tau * tau));
      const double c = 1.0 / std::sqrt(1.0 + t * t);
      const double s = t * c;
      const double app = a[p][p], aqq = a[q][q];
      a[p][p] = app - t * apq;
      a[q][q] = aqq + t * apq;
      a[p][q] = 0.0;
      a[q][p] = 0.0;
      for (int r = 0; r < 3; ++r) {
        if (r == p || r == q) continue;
        const double arp = a[r][p], arq = a[r][q];
        a[r][p] = c * arp - s * arq;
        a[p][r] = a[r][p];
        a[r][q] = s * arp + c * arq;
        a[q][r] = a[r][q];
      }
      for (auto& row : v) {
        const double vrp = row[p], vrq = row[q];
        row[p] = c * vrp - s * vrq;
        row[q] = s * vrp + c * vrq;
      }
    }
  }
  struct P {
    double ev;
    double vec[3];
  } pr[3];
  for (int k = 0; k < 3; ++k) {
    double x = v[0][k], y = v[1][k], z = v[2][k];
    double inv = 1.0 / std::sqrt((x * x + y * y) + z * z);
    pr[k] = {a[k][k], {x * inv, y * inv, z * inv}};
  }
  std::stable_sort(pr, pr + 3, [](const P& l, const P& r) { return r.ev < l.ev; });
  M3 B;
  for (int k = 0; k < 3; ++k)
    for (int j = 0; j < 3; ++j) B.c[3 * k + j] = (float)pr[k].vec[j];
  if (m3_det(B) < 0.0f)
    for (int j = 0; j < 3; ++j) B.c[6 + j] = -B.c[6 + j];
  for (int k = 0; k < 3; ++k) evals[k] = (float)pr[k].ev;
  *basis = B;
}

// higham_polar_decomposition (deformation/polar.rs:13-42), rotation only.
M3 higham_polar(const M3& J) {
  const float det = m3_det(J);
  M3 I = {{1, 0, 0, 0, 1, 0, 0, 0, 1}};
  if (std::fabs(det) < 1e-8f) return I;
  const float gamma = powf(std::fabs(det), -1.0f / 3.0f);
  M3 r;
  for (int k = 0; k < 9; ++k) r.c[k] = J.c[k] * gamma;
  for (int it = 0; it < 5; ++it) {
    M3 rit = m3_t(m3_inverse(r));
    for (int k = 0; k < 9; ++k) r.c[k] = 0.5f * (r.c[k] + rit.c[k]);
  }
  if (m3_det(r) < 0.0f)
    for (int j = 0; j < 3; ++j) r.c[6 + j] = -r.c[6 + j];
  return r;
}

// ShRotator (render/rasterizer/sh_rotation.rs:1-460). Real SH of band l are
// homogeneous polynomials of degree l: Y_l(d) = B_l v_l(d) over the monomials
// v_l, and v_l(R^T d) = T_l v_l(d). The band's rotation matrix is
// M_l = (B_l T_l B_l^+)^T with B_l^+ = B_l^T (B_l B_l^T)^-1, built in f64 with
// the reference's operation order (poly_mul_linear, mat_mul, Gauss-Jordan with
// the last maximal pivot), rounded to f32, and applied to each channel's block
// with an f32 running sum (apply_block).

// Monomial order of exps_of (sh_rotation.rs:47-56): x exponent descending,
// then y descending.
int sh_exps(int d, int (*e)[3]) {
  int k = 0;
  for (int x = d; x >= 0; --x)
    for (int y = d - x; y >= 0; --y) {
      e[k][0] = x;
      e[k][1] = y;
      e[k][2] = d - x - y;
      ++k;
    }
  return k;
}
int sh_exp_index(int d, const int* e) {
  int k = 0;
  for (int x = d; x > e[0]; --x) k += d - x + 1;
  return k + (d - e[0] - e[1]);
}

// basis_rows (sh_rotation.rs:139-226) as integer monomial coefficients times
// the band constants: B[row * m + mono].
void sh_basis_rows(int l, double* B) {
  const double C1 = 0.4886025119029199, C2_0 = 1.0925484305920792, C2_2 = 0.31539156525252005,
               C2_4 = 0.5462742152960396, C3_0 = -0.5900435899266435, C3_1 = 2.890611442640554,
               C3_2 = -0.4570457994644658, C3_3 = 0.3731763325901154, C3_5 = 1.445305721320277;
  struct T { int row, mono; double k, c; };
  static const T t1[] = {{0, 1, 1, 0}, {1, 2, 1, 0}, {2, 0, 1, 0}};
  const int m = (l + 1) * (l + 2) / 2, n = 2 * l + 1;
  for (int i = 0; i < n * m; ++i) B[i] = 0.0;
  if (l == 1) {
    const double c[3] = {-C1, C1, -C1};
    for (const T& e : t1) B[e.row * m + e.mono] = e.k * c[e.row];
  } else if (l == 2) {
    // monomials xx xy xz yy yz zz
    const T t[] = {{0, 1, 1, C2_0}, {1, 4, 1, -C2_0}, {2, 0, -1, C2_2}, {2, 3, -1, C2_2},
                   {2, 5, 2, C2_2}, {3, 2, 1, -C2_0}, {4, 0, 1, C2_4}, {4, 3, -1, C2_4}};
    for (const T& e : t) B[e.row * m + e.mono] = e.k * e.c;
  } else {
    // monomials xxx xxy xxz xyy xyz xzz yyy yyz yzz zzz
    const T t[] = {{0, 1, 3, C3_0}, {0, 6, -1, C3_0}, {1, 4, 1, C3_1},  {2, 1, -1, C3_2},
                   {2, 6, -1, C3_2}, {2, 8, 4, C3_2}, {3, 2, -3, C3_3}, {3, 7, -3, C3_3},
                   {3, 9, 2, C3_3}, {4, 0, -1, C3_2}, {4, 3, -1, C3_2}, {4, 5, 4, C3_2},
                   {5, 2, 1, C3_5}, {5, 7, -1, C3_5}, {6, 0, 1, C3_0},  {6, 3, -3, C3_0}};
    for (const T& e : t) B[e.row * m + e.mono] = e.k * e.c;
  }
}

// mat_mul (sh_rotation.rs:228-245): out[i][j] = sum over k of a[i][k] b[k][j],
// k ascending, terms with a[i][k] == 0 skipped.
void sh_mat_mul(int r, int inner, int c, const double* a, const double* b, double* out) {
  for (int i = 0; i < r * c; ++i) out[i] = 0.0;
  for (int i = 0; i < r; ++i)
    for (int k = 0; k < inner; ++k) {
      const double aik = a[i * inner + k];
      if (aik == 0.0) continue;
      for (int j = 0; j < c; ++j) out[i * c + j] += aik * b[k * c + j];
    }
}

// invert (sh_rotation.rs:260-300): Gauss-Jordan, pivot = the last row of
// largest magnitude (Iterator::max_by), pivot row scaled by 1/pivot.
bool sh_invert(int n, const double* A, double* out) {
  double aug[10][20];
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < 2 * n; ++j) aug[i][j] = j < n ? A[i * n + j] : (j - n == i ? 1.0 : 0.0);
  for (int col = 0; col < n; ++col) {
    int piv = col;
    for (int r = col + 1; r < n; ++r)
      if (!(std::fabs(aug[piv][col]) > std::fabs(aug[r][col]))) piv = r;
    if (std::fabs(aug[piv][col]) < 1e-12) return false;
    if (piv != col)
      for (int j = 0; j < 2 * n; ++j) std::swap(aug[col][j], aug[piv][j]);
    const double inv = 1.0 / aug[col][col];
    for (int j = 0; j < 2 * n; ++j) aug[col][j] *= inv;
    for (int r = 0; r < n; ++r) {
      if (r == col) continue;
      const double f = aug[r][col];
      if (f == 0.0) continue;
      for (int j = 0; j < 2 * n; ++j) aug[r][j] -= f * aug[col][j];
    }
  }
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) out[i * n + j] = aug[i][n + j];
  return true;
}

// basis_for (sh_rotation.rs:307-330): B and B^+ = B^T (B B^T)^-1.
struct ShBasis {
  double B[70], P[70];
};
const ShBasis& sh_basis(int l) {
  static ShBasis cache[3];
  static bool ready[3] = {false, false, false};
  ShBasis& b = cache[l - 1];
  if (!ready[l - 1]) {
    const int m = (l + 1) * (l + 2) / 2, n = 2 * l + 1;
    sh_basis_rows(l, b.B);
    double Bt[70], G[49], Gi[49];
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < m; ++j) Bt[j * n + i] = b.B[i * m + j];
    sh_mat_mul(n, m, n, b.B, Bt, G);
    sh_invert(n, G, Gi);
    sh_mat_mul(m, n, n, Bt, Gi, b.P);
    ready[l - 1] = true;
  }
  return b;
}

// poly_mul_linear (sh_rotation.rs:332-352).
void sh_poly_mul_linear(const double* a, int deg, const double* lf, double* out) {
  int ea[10][3];
  const int na = sh_exps(deg, ea), nd = (deg + 2) * (deg + 3) / 2;
  for (int k = 0; k < nd; ++k) out[k] = 0.0;
  for (int ia = 0; ia < na; ++ia) {
    const double coeff = a[ia];
    if (coeff == 0.0) continue;
    for (int ax = 0; ax < 3; ++ax) {
      if (lf[ax] == 0.0) continue;
      int ne[3] = {ea[ia][0], ea[ia][1], ea[ia][2]};
      ne[ax] += 1;
      out[sh_exp_index(deg + 1, ne)] += coeff * lf[ax];
    }
  }
}

// sh_rotation_matrix (sh_rotation.rs:354-387): row-major f32 M_l.
void sh_rotation_matrix(const M3& R, int l, float* M) {
  const int m = (l + 1) * (l + 2) / 2, n = 2 * l + 1;
  // monomial_transform: the linear forms are the columns of R (rows of R^T).
  double lf[3][3];
  for (int a = 0; a < 3; ++a)
    for (int k = 0; k < 3; ++k) lf[a][k] = (double)R.at(a, k);
  int ex[10][3];
  sh_exps(l, ex);
  double T[100];
  for (int row = 0; row < m; ++row) {
    double poly[10] = {1.0}, next[10];
    int deg = 0;
    for (int a = 0; a < 3; ++a)
      for (int rep = 0; rep < ex[row][a]; ++rep) {
        sh_poly_mul_linear(poly, deg, lf[a], next);
        ++deg;
        for (int k = 0; k < (deg + 1) * (deg + 2) / 2; ++k) poly[k] = next[k];
      }
    for (int k = 0; k < m; ++k) T[row * m + k] = poly[k];
  }
  const ShBasis& b = sh_basis(l);
  double C[70], D[49];
  sh_mat_mul(n, m, m, b.B, T, C);
  sh_mat_mul(n, m, n, C, b.P, D);
  for (int row = 0; row < n; ++row)
    for (int col = 0; col < n; ++col) M[row * n + col] = (float)D[col * n + row];
}

struct ShRot {
  float M[3][49];
  int degree;
};
ShRot make_sh_rotator(const M3& R, int degree) {
  ShRot out;
  out.degree = degree < 0 ? 0 : (degree > 3 ? 3 : degree);
  for (int l = 1; l <= out.degree; ++l) sh_rotation_matrix(R, l, out.M[l - 1]);
  return out;
}

// ShRotator::apply / apply_block (sh_rotation.rs:389-440).
void apply_sh_rotation(const ShRot& r, float* c48) {
  static const int starts[3] = {0, 3, 8};
  for (int ch = 0; ch < 3; ++ch) {
    float* rest = c48 + 3 + 15 * ch;
    for (int l = 1; l <= r.degree; ++l) {
      const int n = 2 * l + 1;
      float* c = rest + starts[l - 1];
      float out[7];
      for (int row = 0; row < n; ++row) {
        float acc = 0.0f;
        for (int col = 0; col < n; ++col) acc += r.M[l - 1][row * n + col] * c[col];
        out[row] = acc;
      }
      for (int j = 0; j < n; ++j) c[j] = out[j];
    }
  }
}

struct RefTet {
  M3 J, R;
  float max_stretch;
};

// tet_transforms (deformation/cpu_reference.rs:61-93).
RefTet ref_tet_transform(const float* verts, const uint32_t* e, const float* inv) {
  float c0[3], c1[3], c2[3];
  const float* x0 = verts + 3 * e[0];
  for (int k = 0; k < 3; ++k) {
    c0[k] = verts[3 * e[1] + k] - x0[k];
    c1[k] = verts[3 * e[2] + k] - x0[k];
    c2[k] = verts[3 * e[3] + k] - x0[k];
  }
  M3 ds = {{c0[0], c0[1], c0[2], c1[0], c1[1], c1[2], c2[0], c2[1], c2[2]}};
  M3 idm;
  std::memcpy(idm.c, inv, 36);
  RefTet t;
  t.J = m3_mul(ds, idm);
  t.R = higham_polar(t.J);
  M3 C = m3_mul(m3_t(t.J), t.J);
  const float packed[6] = {C.at(0, 0), C.at(0, 1), C.at(0, 2), C.at(1, 1), C.at(1, 2), C.at(2, 2)};
  float ev[3];
  M3 basis;
  sym_eigen3(packed, ev, &basis);
  t.max_stretch = std::sqrt(std::fmax(ev[0], 0.0f));
  return t;
}

// apply_mip_filter_3d (math/covariance.rs:288-305): f64 determinants.
void ref_mip3d(float* cov, float* opa, float var) {
  if (var <= 0.0f) return;
  auto det = [](const float* c) {
    const double xx = c[0], xy = c[1], xz = c[2], yy = c[3], yz = c[4], zz = c[5];
    return (float)(xx * (yy * zz - yz * yz) - xy * (xy * zz - xz * yz) + xz * (xy * yz - xz * yy));
  };
  const float d0 = std::fmax(det(cov), 1e-24f);
  float reg[6] = {cov[0] + var, cov[1], cov[2], cov[3] + var, cov[4], cov[5] + var};
  const float dr = std::fmax(det(reg), d0);
  const float comp = std::sqrt(clampf(d0 / dr, 0.0f, 1.0f));
  std::memcpy(cov, reg, 24);
  *opa = clampf(*opa * comp, 0.0f, 1.0f);
}

// ---------------------------------------------------------------- MVC (ref)
// PolyCageMesh (deformation/mvc.rs) in f32 with glam 0.28's Vec3/Mat3 order:
// length = sqrt(dot), dot = (x*x + y*y) + z*z, Vec3 / f32 per component.
struct V3 {
  float x, y, z;
};
inline V3 v3(const float* p) { return {p[0], p[1], p[2]}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3 operator/(V3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
inline float vdot(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline float vlen(V3 a) { return std::sqrt(vdot(a, a)); }
inline V3 vcross(V3 a, V3 b) {
  return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}

// winding_number (mvc.rs:339-357).
float mvc_winding(uint32_t F, const float* verts, const uint32_t* tris, V3 p) {
  float sum = 0.0f;
  for (uint32_t f = 0; f < F; ++f) {
    const V3 a = v3(verts + 3 * tris[3 * f]) - p;
    const V3 b = v3(verts + 3 * tris[3 * f + 1]) - p;
    const V3 c = v3(verts + 3 * tris[3 * f + 2]) - p;
    const float la = vlen(a), lb = vlen(b), lc = vlen(c);
    if (la < 1e-7f || lb < 1e-7f || lc < 1e-7f) return 1.0f;
    const float det = vdot(a, vcross(b, c));
    const float denom = ((la * lb * lc + vdot(a, b) * lc) + vdot(b, c) * la) + vdot(c, a) * lb;
    sum += 2.0f * std::atan2(det, denom);
  }
  return sum / (4.0f * (float)M_PI);
}

// compute_mvc_weights (mvc.rs:366-471), Ju, Schaefer & Warren 2005.
void mvc_weights(uint32_t V, uint32_t F, const float* verts, const uint32_t* tris, V3 x,
                 float* w) {
  std::vector<float> dists(V);
  std::vector<V3> dirs(V);
  for (uint32_t i = 0; i < V; ++i) {
    const V3 diff = v3(verts + 3 * i) - x;
    const float d = vlen(diff);
    if (d < 1e-6f) {
      for (uint32_t j = 0; j < V; ++j) w[j] = 0.0f;
      w[i] = 1.0f;
      return;
    }
    dists[i] = d;
    dirs[i] = diff / d;
  }
  for (uint32_t j = 0; j < V; ++j) w[j] = 0.0f;
  float total = 0.0f;
  const float PI_F = (float)M_PI;
  for (uint32_t f = 0; f < F; ++f) {
    const uint32_t i0 = tris[3 * f], i1 = tris[3 * f + 1], i2 = tris[3 * f + 2];
    const V3 u0 = dirs[i0], u1 = dirs[i1], u2 = dirs[i2];
    const float l0 = vlen(u1 - u2), l1 = vlen(u2 - u0), l2 = vlen(u0 - u1);
    const float t0 = 2.0f * std::asin(clampf(l0 * 0.5f, 0.0f, 1.0f));
    const float t1 = 2.0f * std::asin(clampf(l1 * 0.5f, 0.0f, 1.0f));
    const float t2 = 2.0f * std::asin(clampf(l2 * 0.5f, 0.0f, 1.0f));
    const float h = 0.5f * ((t0 + t1) + t2);
    if (std::fabs(PI_F - h) < 1e-5f) {
      const float w0 = std::sin(t0) * dists[i1] * dists[i2];
      const float w1 = std::sin(t1) * dists[i2] * dists[i0];
      const float w2 = std::sin(t2) * dists[i0] * dists[i1];
      const float sum = (w0 + w1) + w2;
      for (uint32_t j = 0; j < V; ++j) w[j] = 0.0f;
      if (std::fabs(sum) > 1e-12f) {
        w[i0] = w0 / sum;
        w[i1] = w1 / sum;
        w[i2] = w2 / sum;
      }
      return;
    }
    const float st0 = std::sin(t0), st1 = std::sin(t1), st2 = std::sin(t2);
    if (std::fabs(st0) < 1e-6f || std::fabs(st1) < 1e-6f || std::fabs(st2) < 1e-6f) continue;
    const float sh = std::sin(h);
    const float c0 = clampf((2.0f * sh * std::sin(h - t0)) / (st1 * st2) - 1.0f, -1.0f, 1.0f);
    const float c1 = clampf((2.0f * sh * std::sin(h - t1)) / (st2 * st0) - 1.0f, -1.0f, 1.0f);
    const float c2 = clampf((2.0f * sh * std::sin(h - t2)) / (st0 * st1) - 1.0f, -1.0f, 1.0f);
    const float det = vdot(u2, vcross(u0, u1));  // Mat3::from_cols(u0,u1,u2).determinant()
    const float sg = det >= 0.0f ? 1.0f : -1.0f;
    const float s0 = sg * std::sqrt(std::fmax(1.0f - c0 * c0, 0.0f));
    const float s1 = sg * std::sqrt(std::fmax(1.0f - c1 * c1, 0.0f));
    const float s2 = sg * std::sqrt(std::fmax(1.0f - c2 * c2, 0.0f));
    if (std::fabs(s0) <= 1e-6f || std::fabs(s1) <= 1e-6f || std::fabs(s2) <= 1e-6f) continue;
    const float mu0 = ((t0 - c1 * t2) - c2 * t1) / (2.0f * dists[i0] * st1 * s2);
    const float mu1 = ((t1 - c2 * t0) - c0 * t2) / (2.0f * dists[i1] * st2 * s0);
    const float mu2 = ((t2 - c0 * t1) - c1 * t0) / (2.0f * dists[i2] * st0 * s1);
    w[i0] += mu0;
    w[i1] += mu1;
    w[i2] += mu2;
    total += (mu0 + mu1) + mu2;
  }
  if (std::fabs(total) > 1e-12f) {
    const float inv = 1.0f / total;
    for (uint32_t j = 0; j < V; ++j) w[j] *= inv;
  } else {
    uint32_t best = 0;
    for (uint32_t i = 1; i < V; ++i)
      if (dists[i] < dists[best]) best = i;
    w[best] = 1.0f;
  }
}

// jacobian_step_size (mvc.rs:484-494).
float mvc_step(uint32_t V, const float* verts) {
  V3 mn = {INFINITY, INFINITY, INFINITY}, mx = {-INFINITY, -INFINITY, -INFINITY};
  for (uint32_t i = 0; i < V; ++i) {
    const V3 p = v3(verts + 3 * i);
    mn = {std::fmin(mn.x, p.x), std::fmin(mn.y, p.y), std::fmin(mn.z, p.z)};
    mx = {std::fmax(mx.x, p.x), std::fmax(mx.y, p.y), std::fmax(mx.z, p.z)};
  }
  const float diag = std::fmax(vlen(mx - mn), 1e-3f);
  return clampf(diag * 1e-3f, 1e-5f, 1e-2f);
}

}  // namespace


extern "C" {

// Screen tile shape of the v2 functions (width, height in pixels).
void orc_set_tile_shape(uint32_t w, uint32_t h) {
  g_tile_w = w ? w : 16u;
  g_tile_h = h ? h : 16u;
}

void orc_set_threads(int n) { g_threads = n; }
int orc_get_threads(void) { return num_threads(); }

// ------------------------------------------------------------ v2 entry points

void orc_tet_transforms(uint32_t T, const float* verts, const uint32_t* elems,
                        const float* inv_dm, float* J, float* R, float* stretch) {
  parallel_for(T, [&](size_t b, size_t e) {
    for (size_t t = b; t < e; ++t)
      tet_transform_one(verts, elems + 4 * t, inv_dm + 9 * t, J + 9 * t, R + 9 * t, stretch + t);
  });
}

// Stage 1 (deformation.rs:874-1211). Children are placed at n + (number of
// splitting Gaussians before the parent), i.e. ordered by parent index (the
// order gpu_bridge.rs:383 sorts the reference's atomically placed children
// into). Outputs hold 2n slots; returns the number of children.
uint32_t orc_deform_split(uint32_t n, uint32_t T, const float* verts, const uint32_t* elems,
                          const float* J, const float* stretch, const uint32_t* bind_tet,
                          const float* bind_w, const float* rest_pos, const float* rest_cov,
                          const float* rest_opa, float split_thr, float mip, float* out_pos,
                          float* out_cov, float* out_opa, uint32_t* out_meta) {
  std::vector<uint8_t> split(n, 0);
  std::vector<float> cpos((size_t)n * 3);
  parallel_for(n, [&](size_t b, size_t e) {
    for (size_t i = b; i < e; ++i) {
      DeformOut o = deform_one(i, T, verts, elems, J, stretch, bind_tet, bind_w, rest_pos,
                               rest_cov, rest_opa, split_thr, mip);
      std::memcpy(out_pos + 3 * i, o.pos, 12);
      std::memcpy(out_cov + 6 * i, o.cov, 24);
      out_opa[i] = o.opa;
      split[i] = o.split;
      std::memcpy(&cpos[3 * i], o.cpos, 12);
    }
  });
  uint32_t k = 0;
  for (uint32_t i = 0; i < n; ++i) {
    if (!split[i]) continue;
    size_t c = (size_t)n + k;
    std::memcpy(out_pos + 3 * c, &cpos[3 * i], 12);
    std::memcpy(out_cov + 6 * c, out_cov + 6 * (size_t)i, 24);
    out_opa[c] = out_opa[i];
    out_meta[2 * (size_t)k] = i;
    out_meta[2 * (size_t)k + 1] = bind_tet[i];
    ++k;
  }
  return k;
}

// Stage 2 (project.rs:1020-1289). attrs [active*10] (written for visible
// splats only, zeros elsewhere), ext [active]. Returns the survivor count.
uint64_t orc_project_v2(uint32_t active, uint32_t n_rest, const float* pos, const float* cov,
                        const float* opa, const float* sh, const uint32_t* bind_tet,
                        const float* tet_R, uint32_t num_tets, const uint32_t* split_meta,
                        const float* cam24, const float* cam_pos3, float mip, float min_opa,
                        float min_rad, uint32_t sh_degree, uint32_t has_deform, float* attrs,
                        uint32_t* ext) {
  std::atomic<uint64_t> surv{0};
  parallel_for(active, [&](size_t b, size_t e) {
    uint64_t local = 0;
    for (size_t i = b; i < e; ++i) {
      std::memset(attrs + 10 * i, 0, 40);
      ext[i] = project_one(i, n_rest, pos, cov, opa, sh, bind_tet, tet_R, num_tets, split_meta,
                           cam24, cam_pos3, mip, min_opa, min_rad, sh_degree, has_deform, attrs);
      local += ext[i] != 0;
    }
    surv += local;
  });
  return surv.load();
}

// count_tiles_kernel (binning.rs:92-164). Returns the sum of counts.
uint64_t orc_count_tiles(uint32_t n, const float* attrs, const uint32_t* ext, uint32_t W,
                         uint32_t H, uint32_t* counts) {
  uint32_t tiles_x = tiles_across(W), tiles_y = tiles_down(H);
  std::atomic<uint64_t> total{0};
  parallel_for(n, [&](size_t b, size_t e) {
    uint64_t local = 0;
    for (size_t i = b; i < e; ++i) {
      uint32_t p = ext[i];
      counts[i] = 0;
      if (p == 0 || tiles_x == 0 || tiles_y == 0) continue;
      const float* a = attrs + 10 * i;
      TileBox tb = tile_box(a[0], a[1], (float)(p & 0xFFFF), (float)((p >> 16) & 0xFFFF), tiles_x,
                            tiles_y);
      uint32_t c = 0;
      for (uint32_t ty = tb.y0; ty <= tb.y1; ++ty)
        for (uint32_t tx = tb.x0; tx <= tb.x1; ++tx)
          c += ellipse_tile(a[0], a[1], a[2], a[3], a[4], a[5], tx, ty, W, H);
      counts[i] = c;
      local += c;
    }
    total += local;
  });
  return total.load();
}

// Exclusive scan (scan.rs:198-333 / tiles/cpu_reference.rs:100-115).
uint64_t orc_scan(uint64_t n, const uint32_t* in, uint32_t* out) {
  uint64_t acc = 0;
  for (uint64_t i = 0; i < n; ++i) {
    out[i] = (uint32_t)acc;
    acc += in[i];
  }
  return acc;
}

// compute_packed_key_bits (binning.rs:12-20).
void orc_packed_key_bits(uint32_t total_tiles, uint32_t* tile_bits, uint32_t* depth_bits) {
  uint32_t tb = total_tiles <= 1 ? 1u : 32u - (uint32_t)__builtin_clz(total_tiles - 1);
  *tile_bits = tb;
  *depth_bits = std::min(32u - std::min(tb, 32u), 28u);
}

// emit_tile_keys_kernel (binning.rs:170-250): 32-bit keys.
void orc_emit_keys32(uint32_t n, const float* attrs, const uint32_t* ext, const uint32_t* offsets,
                     uint32_t W, uint32_t H, float near_plane, uint32_t depth_bits,
                     uint32_t* keys, uint32_t* ids) {
  uint32_t tiles_x = tiles_across(W), tiles_y = tiles_down(H);
  uint32_t base = f2u(std::fmax(near_plane, 1e-6f)) & 0x7F800000u;
  parallel_for(n, [&](size_t b, size_t e) {
    for (size_t i = b; i < e; ++i) {
      uint32_t p = ext[i];
      if (p == 0 || tiles_x == 0 || tiles_y == 0) continue;
      const float* a = attrs + 10 * i;
      uint32_t raw = f2u(std::fmax(a[9], 1e-6f));
      uint32_t rel = raw > base ? std::min(raw - base, 0x0FFFFFFFu) : 0u;
      uint32_t dq = rel >> (28u - depth_bits);
      TileBox tb = tile_box(a[0], a[1], (float)(p & 0xFFFF), (float)((p >> 16) & 0xFFFF), tiles_x,
                            tiles_y);
      uint64_t cur = offsets[i];
      for (uint32_t ty = tb.y0; ty <= tb.y1; ++ty)
        for (uint32_t tx = tb.x0; tx <= tb.x1; ++tx)
          if (ellipse_tile(a[0], a[1], a[2], a[3], a[4], a[5], tx, ty, W, H)) {
            uint32_t tile = ty * tiles_x + tx;
            keys[cur] = depth_bits >= 32 ? dq : ((tile << depth_bits) | dq);
            ids[cur] = (uint32_t)i;
            ++cur;
          }
    }
  });
}

// emit_tile_keys_u64_kernel (binning.rs:256-328).
void orc_emit_keys64(uint32_t n, const float* attrs, const uint32_t* ext, const uint32_t* offsets,
                     uint32_t W, uint32_t H, uint32_t* tiles, uint32_t* depths, uint32_t* ids) {
  uint32_t tiles_x = tiles_across(W), tiles_y = tiles_down(H);
  parallel_for(n, [&](size_t b, size_t e) {
    for (size_t i = b; i < e; ++i) {
      uint32_t p = ext[i];
      if (p == 0 || tiles_x == 0 || tiles_y == 0) continue;
      const float* a = attrs + 10 * i;
      uint32_t d = f2u(std::fmax(a[9], 0.0f));
      TileBox tb = tile_box(a[0], a[1], (float)(p & 0xFFFF), (float)((p >> 16) & 0xFFFF), tiles_x,
                            tiles_y);
      uint64_t cur = offsets[i];
      for (uint32_t ty = tb.y0; ty <= tb.y1; ++ty)
        for (uint32_t tx = tb.x0; tx <= tb.x1; ++tx)
          if (ellipse_tile(a[0], a[1], a[2], a[3], a[4], a[5], tx, ty, W, H)) {
            tiles[cur] = ty * tiles_x + tx;
            depths[cur] = d;
            ids[cur] = (uint32_t)i;
            ++cur;
          }
    }
  });
}

// Stable sort by the low key_bits of the key: the result of the reference's
// LSD radix sort (radix_sort.rs:292-368), which is stable.
void orc_sort_pairs32(uint64_t n, uint32_t* keys, uint32_t* vals, uint32_t key_bits) {
  uint32_t mask = key_bits >= 32 ? 0xFFFFFFFFu : ((1u << key_bits) - 1u);
  std::vector<uint64_t> idx(n);
  for (uint64_t i = 0; i < n; ++i) idx[i] = ((uint64_t)(keys[i] & mask) << 32) | (uint32_t)i;
  std::sort(idx.begin(), idx.end());
  std::vector<uint32_t> k2(n), v2(n);
  for (uint64_t i = 0; i < n; ++i) {
    uint32_t src = (uint32_t)idx[i];
    k2[i] = keys[src];
    v2[i] = vals[src];
  }
  std::memcpy(keys, k2.data(), n * 4);
  std::memcpy(vals, v2.data(), n * 4);
}

// Stable sort of (tile, depth, id) by (tile, depth) (radix_sort.rs:377-477).
void orc_sort_triples64(uint64_t n, uint32_t* tiles, uint32_t* depths, uint32_t* ids) {
  std::vector<uint64_t> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](uint64_t a, uint64_t b) {
    if (tiles[a] != tiles[b]) return tiles[a] < tiles[b];
    return depths[a] < depths[b];
  });
  std::vector<uint32_t> t2(n), d2(n), i2(n);
  for (uint64_t i = 0; i < n; ++i) {
    t2[i] = tiles[order[i]];
    d2[i] = depths[order[i]];
    i2[i] = ids[order[i]];
  }
  std::memcpy(tiles, t2.data(), n * 4);
  std::memcpy(depths, d2.data(), n * 4);
  std::memcpy(ids, i2.data(), n * 4);
}

// clear_tile_ranges_kernel + identify_tile_ranges[_u32_tile]_kernel
// (binning.rs:333-417): tile id = key >> shift.
void orc_tile_ranges(uint64_t n, const uint32_t* sorted, uint32_t shift, uint32_t total_tiles,
                     uint32_t* ranges) {
  std::memset(ranges, 0, (size_t)total_tiles * 8);
  for (uint64_t i = 0; i < n; ++i) {
    uint32_t t = shift >= 32 ? 0u : (sorted[i] >> shift);
    if (t >= total_tiles) continue;
    if (i == 0) {
      ranges[2 * t] = 0;
    } else {
      uint32_t prev = shift >= 32 ? 0u : (sorted[i - 1] >> shift);
      if (t != prev) {
        if (prev < total_tiles) ranges[2 * prev + 1] = (uint32_t)i;
        ranges[2 * t] = (uint32_t)i;
      }
    }
    if (i + 1 == n) ranges[2 * t + 1] = (uint32_t)n;
  }
}

// tile_compositor_v2_kernel (render/kernels/compositor.rs:727-883) with both
// output modes: rgba8 tight [H][W][4] (round-half-even, WGSL round) and f32.
void orc_composite_v2(uint32_t W, uint32_t H, const float* attrs, const uint32_t* sorted_ids,
                      const uint32_t* ranges, const float* bg, uint8_t* rgba8, float* rgba_f32) {
  uint32_t tiles_x = tiles_across(W);
  parallel_for((size_t)W * H, [&](size_t b, size_t e) {
    for (size_t pix = b; pix < e; ++pix) {
      uint32_t px = (uint32_t)(pix % W), py = (uint32_t)(pix / W);
      uint32_t tile = (py / g_tile_h) * tiles_x + (px / g_tile_w);
      uint32_t rs = ranges[2 * tile], re = ranges[2 * tile + 1];
      bool empty = rs >= re;
      float cr = 0, cg = 0, cb = 0, t = 1.0f;
      float pcx = (float)px + 0.5f, pcy = (float)py + 0.5f;
      if (!empty) {
        for (uint32_t k = rs; k < re; ++k) {
          const float* a = attrs + 10 * (size_t)sorted_ids[k];
          float op = a[5];
          if (!(op > 0.003921569f)) continue;
          float dx = pcx - a[0], dy = pcy - a[1];
          float q = -0.5f * (a[2] * dx * dx + 2.0f * a[3] * dx * dy + a[4] * dy * dy);
          if (q > 0.0f) q = 0.0f;
          if (q >= -4.0f) {
            float alpha = std::fmin(0.99f, op * cgs_expf(q));
            if (alpha >= 0.003921569f) {
              float w = alpha * t;
              cr += w * a[6];
              cg += w * a[7];
              cb += w * a[8];
              t *= 1.0f - alpha;
              if (t < 0.001f) {
                t = 0.0f;
                break;
              }
            }
          }
        }
      }
      float fr = clampf(cr + t * bg[0], 0.0f, 1.0f);
      float fg = clampf(cg + t * bg[1], 0.0f, 1.0f);
      float fb = clampf(cb + t * bg[2], 0.0f, 1.0f);
      float fa = empty ? bg[3] : clampf(1.0f - t, 0.0f, 1.0f);
      if (rgba_f32) {
        rgba_f32[4 * pix] = fr;
        rgba_f32[4 * pix + 1] = fg;
        rgba_f32[4 * pix + 2] = fb;
        rgba_f32[4 * pix + 3] = fa;
      }
      if (rgba8) {
        float v[4] = {fr, fg, fb, fa};
        for (int ch = 0; ch < 4; ++ch)
          rgba8[4 * pix + ch] = (uint8_t)clampf(std::nearbyint(v[ch] * 255.0f), 0.0f, 255.0f);
      }
    }
  });
}


// Ellipse-vs-tile test (render/tiles/mod.rs:139-184; same formula as
// binning.rs:37-83) for unit tests.
int orc_ellipse_tile(float mu_x, float mu_y, float a, float b, float c, float alpha, uint32_t tx,
                     uint32_t ty, uint32_t W, uint32_t H) {
  return ellipse_tile(mu_x, mu_y, a, b, c, alpha, tx, ty, W, H) ? 1 : 0;
}

// compute_conic_and_extents (math/projection.rs:187-222); returns 0 when culled.
int orc_conic_extents(float sxx_in, float sxy_in, float syy_in, float alpha, float* conic,
                      int32_t* ext) {
  const float s_xx = sxx_in + 0.3f, s_xy = sxy_in, s_yy = syy_in + 0.3f;
  const float det = s_xx * s_yy - s_xy * s_xy;
  if (det <= 1e-6f) return 0;
  float sigma = 0.0f;
  if (!(alpha <= 1.0f / 255.0f)) sigma = std::sqrt(clampf(2.0f * logf(255.0f * alpha), 0.0f, 8.0f));
  if (sigma <= 0.0f) return 0;
  const float inv_det = 1.0f / det;
  conic[0] = s_yy * inv_det;
  conic[1] = -s_xy * inv_det;
  conic[2] = s_xx * inv_det;
  ext[0] = (int32_t)clampf(std::ceil(sigma * std::sqrt(std::fmax(s_xx, 0.0f))), 1.0f, 1024.0f);
  ext[1] = (int32_t)clampf(std::ceil(sigma * std::sqrt(std::fmax(s_yy, 0.0f))), 1.0f, 1024.0f);
  return 1;
}

// Deterministic transcendental functions exposed for their unit tests.
float orc_detmath(int which, float x, float y) {
  switch (which) {
    case 0: return cgs_logf(x);
    case 1: return cgs_expf(x);
    case 2: return cgs_acosf(x);
    case 3: return cgs_cosf(x);
    case 4: return cgs_powf(x, y);
    default: return 0.0f;
  }
}


// TetMesh::bind_point (deformation/mod.rs:267-310): first tet whose
// barycentric violation is <= 1e-4, else the least-violating one; with bounds,
// points outside [bmin, bmax] or with best violation > 0.15 are unbound.
// glam Mat3 * Vec3 is (c0 x + c1 y) + c2 z.
void orc_bind_points(uint32_t n, const float* pts, uint32_t T, const float* x0,
                     const float* inv_dm, int use_bounds, const float* bmin, const float* bmax,
                     uint32_t* out_tet, float* out_w) {
  parallel_for(n, [&](size_t b, size_t e) {
    for (size_t i = b; i < e; ++i) {
      const float px = pts[3 * i], py = pts[3 * i + 1], pz = pts[3 * i + 2];
      float* w = out_w + 4 * i;
      if (use_bounds && (px < bmin[0] || px > bmax[0] || py < bmin[1] || py > bmax[1] ||
                         pz < bmin[2] || pz > bmax[2])) {
        out_tet[i] = 0xFFFFFFFFu;
        w[0] = w[1] = w[2] = w[3] = 0.0f;
        continue;
      }
      uint32_t best = 0;
      float best_pen = INFINITY;
      float bw[4] = {1.0f, 0.0f, 0.0f, 0.0f};
      bool found = false;
      for (uint32_t t = 0; t < T; ++t) {
        const float* d = inv_dm + 9 * (size_t)t;
        const float dx = px - x0[3 * t], dy = py - x0[3 * t + 1], dz = pz - x0[3 * t + 2];
        const float w1 = (d[0] * dx + d[3] * dy) + d[6] * dz;
        const float w2 = (d[1] * dx + d[4] * dy) + d[7] * dz;
        const float w3 = (d[2] * dx + d[5] * dy) + d[8] * dz;
        const float w0 = 1.0f - ((w1 + w2) + w3);
        const float pen = ((std::fmax(-w0, 0.0f) + std::fmax(-w1, 0.0f)) + std::fmax(-w2, 0.0f)) +
                          std::fmax(-w3, 0.0f);
        if (pen <= 1e-4f) {
          out_tet[i] = t;
          w[0] = w0; w[1] = w1; w[2] = w2; w[3] = w3;
          found = true;
          break;
        }
        if (pen < best_pen) {
          best_pen = pen;
          best = t;
          bw[0] = w0; bw[1] = w1; bw[2] = w2; bw[3] = w3;
        }
      }
      if (found) continue;
      if ((use_bounds && best_pen > 0.15f) || T == 0) {
        out_tet[i] = 0xFFFFFFFFu;
        w[0] = w[1] = w[2] = w[3] = 0.0f;
      } else {
        out_tet[i] = best;
        std::memcpy(w, bw, 16);
      }
    }
  });
}

// ------------------------------------------------------------ ref CPU entry points

// fibonacci_cluster (scene/synthetic.rs:6-44), glibc f32 transcendentals.
void orc_fibonacci_cluster(uint32_t count, float radius, const float* center, float* pos,
                           float* cov, float* opa, float* sh) {
  const float golden = (1.0f + std::sqrt(5.0f)) / 2.0f;
  const float SH_C0 = 0.28209479f;
  const float two_pi = 2.0f * 3.14159265358979323846f;
  for (uint32_t i = 0; i < count; ++i) {
    float t = ((float)i + 0.5f) / (float)count;
    float r = radius * cbrtf(t);
    float theta = acosf(clampf(1.0f - 2.0f * t, -1.0f, 1.0f));
    float phi = two_pi * ((float)i / golden);
    pos[3 * i] = center[0] + r * sinf(theta) * cosf(phi);
    pos[3 * i + 1] = center[1] + r * sinf(theta) * sinf(phi);
    pos[3 * i + 2] = center[2] + r * cosf(theta);
    const float c6[6] = {0.0004f, 0.0f, 0.0f, 0.0004f, 0.0f, 0.0004f};
    std::memcpy(cov + 6 * i, c6, 24);
    opa[i] = 0.88f;
    float* s = sh + 48 * (size_t)i;
    std::memset(s, 0, 48 * 4);
    float cr = 0.5f + 0.5f * sinf((float)i * 0.02f);
    float cg = 0.5f + 0.5f * sinf((float)i * 0.02f + 2.094f);
    float cb = 0.5f + 0.5f * sinf((float)i * 0.02f + 4.188f);
    s[0] = (cr - 0.5f) / SH_C0;
    s[1] = (cg - 0.5f) / SH_C0;
    s[2] = (cb - 0.5f) / SH_C0;
  }
}

// project_scene_cpu (render/mod.rs:143-221).
void orc_ref_project_scene(uint32_t n, const float* pos, const float* cov, const float* cam24,
                           float* xy, float* depths, int32_t* radii, float* conics) {
  parallel_for(n, [&](size_t b, size_t e) {
    for (size_t i = b; i < e; ++i)
      project_ewa_ref(pos + 3 * i, cov + 6 * i, cam24, cam24[16], cam24[17], cam24[18], cam24[19],
                      cam24[20], cam24[21], cam24[22], xy + 2 * i, depths + i, radii + i,
                      conics + 3 * i);
  });
}

// bin_and_sort_gaussians_cpu (render/tiles/cpu_reference.rs:248-303): square
// radius bounds, entries (tile, f32 depth bits, id) sorted lexicographically,
// ranges by binary search. Returns the entry count; with out_* null only counts.
uint64_t orc_ref_bin_and_sort(uint32_t n, const float* xy, const float* depths,
                              const int32_t* radii, uint32_t W, uint32_t H, uint32_t* out_tiles,
                              uint32_t* out_depth_bits, uint32_t* out_ids, uint32_t* ranges) {
  uint32_t tiles_x = (W + 15) / 16, tiles_y = (H + 15) / 16, total_tiles = tiles_x * tiles_y;
  std::vector<uint32_t> cnt(n);
  parallel_for(n, [&](size_t b, size_t e) {
    for (size_t i = b; i < e; ++i) {
      cnt[i] = 0;
      if (radii[i] <= 0) continue;
      TileBox tb;
      float r = (float)radii[i];
      if (tile_bounds_xy(xy[2 * i], xy[2 * i + 1], r, r, tiles_x, tiles_y, W, H, &tb))
        cnt[i] = (tb.x1 - tb.x0 + 1) * (tb.y1 - tb.y0 + 1);
    }
  });
  std::vector<uint64_t> off(n + 1, 0);
  for (uint32_t i = 0; i < n; ++i) off[i + 1] = off[i] + cnt[i];
  uint64_t total = off[n];
  if (!out_tiles) return total;
  struct E {
    uint32_t tile, depth, id;
  };
  std::vector<E> ent(total);
  parallel_for(n, [&](size_t b, size_t e) {
    for (size_t i = b; i < e; ++i) {
      if (!cnt[i]) continue;
      TileBox tb;
      float r = (float)radii[i];
      tile_bounds_xy(xy[2 * i], xy[2 * i + 1], r, r, tiles_x, tiles_y, W, H, &tb);
      uint64_t c = off[i];
      for (uint32_t ty = tb.y0; ty <= tb.y1; ++ty)
        for (uint32_t tx = tb.x0; tx <= tb.x1; ++tx)
          ent[c++] = {ty * tiles_x + tx, f2u(depths[i]), (uint32_t)i};
    }
  });
  std::sort(ent.begin(), ent.end(), [](const E& a, const E& b) {
    if (a.tile != b.tile) return a.tile < b.tile;
    if (a.depth != b.depth) return a.depth < b.depth;
    return a.id < b.id;
  });
  for (uint64_t i = 0; i < total; ++i) {
    out_tiles[i] = ent[i].tile;
    out_depth_bits[i] = ent[i].depth;
    out_ids[i] = ent[i].id;
  }
  std::memset(ranges, 0, (size_t)total_tiles * 8);
  for (uint64_t i = 0; i < total;) {
    uint64_t j = i;
    while (j < total && ent[j].tile == ent[i].tile) ++j;
    ranges[2 * ent[i].tile] = (uint32_t)i;
    ranges[2 * ent[i].tile + 1] = (uint32_t)j;
    i = j;
  }
  return total;
}

// rasterize_scene_cpu (render/rasterizer/cpu_reference.rs:120-240) with the
// quantisation of RasterizedImage::from_pixels (:58-72, round half away from 0).
void orc_ref_rasterize(uint32_t W, uint32_t H, const float* xy, const float* conics,
                       const float* opa, const float* sh, const float* pos,
                       const uint32_t* sorted_ids, const uint32_t* ranges, const float* bg,
                       const float* cam_pos, uint32_t sh_degree, uint8_t* rgba8,
                       float* rgba_f32) {
  uint32_t tiles_x = (W + 15) / 16;
  parallel_for((size_t)W * H, [&](size_t b, size_t e) {
    for (size_t pix = b; pix < e; ++pix) {
      uint32_t px = (uint32_t)(pix % W), py = (uint32_t)(pix / W);
      uint32_t tile = (py / 16) * tiles_x + (px / 16);
      uint32_t rs = ranges[2 * tile], re = ranges[2 * tile + 1];
      float out[4];
      if (rs >= re) {
        out[0] = bg[0]; out[1] = bg[1]; out[2] = bg[2]; out[3] = bg[3];
      } else {
        float pcx = (float)px + 0.5f, pcy = (float)py + 0.5f;
        float cr = 0, cg = 0, cb = 0, t = 1.0f;
        for (uint32_t k = rs; k < re; ++k) {
          if (t < 0.001f) {
            t = 0.0f;
            break;
          }
          uint32_t g = sorted_ids[k];
          float dx = pcx - xy[2 * g], dy = pcy - xy[2 * g + 1];
          float a = conics[3 * g], bb = conics[3 * g + 1], c = conics[3 * g + 2];
          float q = -0.5f * (a * dx * dx + 2.0f * bb * dx * dy + c * dy * dy);
          if (q > 0.0f) q = 0.0f;
          if (q < -4.0f) continue;
          float alpha = std::fmin(opa[g] * expf(q), 0.99f);
          if (alpha < (1.0f / 255.0f)) continue;
          float vx = pos[3 * g] - cam_pos[0], vy = pos[3 * g + 1] - cam_pos[1],
                vz = pos[3 * g + 2] - cam_pos[2];
          float ls = (vx * vx + vy * vy) + vz * vz;
          float dxn = 0, dyn = 0, dzn = 1;
          if (ls > 1e-8f) {
            float rl = 1.0f / std::sqrt(ls);
            dxn = vx * rl;
            dyn = vy * rl;
            dzn = vz * rl;
          }
          float rgb[3];
          eval_sh(sh + 48 * (size_t)g, dxn, dyn, dzn, sh_degree, rgb);
          float w = alpha * t;
          cr += w * rgb[0];
          cg += w * rgb[1];
          cb += w * rgb[2];
          t *= 1.0f - alpha;
        }
        out[0] = clampf(cr + t * bg[0], 0.0f, 1.0f);
        out[1] = clampf(cg + t * bg[1], 0.0f, 1.0f);
        out[2] = clampf(cb + t * bg[2], 0.0f, 1.0f);
        out[3] = clampf(1.0f - t, 0.0f, 1.0f);
      }
      for (int ch = 0; ch < 4; ++ch) {
        if (rgba_f32) rgba_f32[4 * pix + ch] = out[ch];
        if (rgba8) rgba8[4 * pix + ch] = (uint8_t)std::round(clampf(out[ch], 0.0f, 1.0f) * 255.0f);
      }
    }
  });
}

// FNV-1a over the RGBA8 bytes (RasterizedImage::pixel_hash, cpu_reference.rs:105-112).
uint64_t orc_pixel_hash(uint64_t nbytes, const uint8_t* rgba8) {
  uint64_t h = 0xcbf29ce484222325ull;
  for (uint64_t i = 0; i < nbytes; ++i) {
    h ^= rgba8[i];
    h *= 0x00000100000001b3ull;
  }
  return h;
}

// render_scene_cpu (render/mod.rs:288-305): project, square-radius bin, raster.
uint64_t orc_ref_render_scene(uint32_t n, const float* pos, const float* cov, const float* opa,
                              const float* sh, const float* cam24, uint32_t W, uint32_t H,
                              const float* bg, const float* cam_pos, uint32_t sh_degree,
                              uint8_t* rgba8, float* rgba_f32) {
  std::vector<float> xy(2 * (size_t)n), depths(n), conics(3 * (size_t)n);
  std::vector<int32_t> radii(n);
  orc_ref_project_scene(n, pos, cov, cam24, xy.data(), depths.data(), radii.data(), conics.data());
  uint32_t tiles = ((W + 15) / 16) * ((H + 15) / 16);
  uint64_t total =
      orc_ref_bin_and_sort(n, xy.data(), depths.data(), radii.data(), W, H, nullptr, nullptr,
                           nullptr, nullptr);
  std::vector<uint32_t> t(total), d(total), ids(total), ranges(2 * (size_t)tiles);
  orc_ref_bin_and_sort(n, xy.data(), depths.data(), radii.data(), W, H, t.data(), d.data(),
                       ids.data(), ranges.data());
  orc_ref_rasterize(W, H, xy.data(), conics.data(), opa, sh, pos, ids.data(), ranges.data(), bg,
                    cam_pos, sh_degree, rgba8, rgba_f32);
  return total;
}

}  // extern "C"

extern "C" {

// ellipse_intersects_tile (render/tiles/mod.rs:139-184): the CPU-side twin of
// the kernels' test, 16x16 tiles, with the cutoff from glibc logf (Rust's
// f32::ln on Linux) instead of the deterministic logarithm of the v2 mode.
int orc_ref_ellipse_tile(float mu_x, float mu_y, float a, float b, float c, float alpha,
                         uint32_t tx, uint32_t ty, uint32_t W, uint32_t H) {
  if (alpha < (1.0f / 255.0f) || W == 0 || H == 0) return 0;
  const uint32_t x_start = tx * 16u, y_start = ty * 16u;
  if (x_start >= W || y_start >= H) return 0;
  const float dx0 = ((float)x_start + 0.5f) - mu_x;
  const float dx1 = ((float)std::min(x_start + 15u, W - 1u) + 0.5f) - mu_x;
  const float dy0 = ((float)y_start + 0.5f) - mu_y;
  const float dy1 = ((float)std::min(y_start + 15u, H - 1u) + 0.5f) - mu_y;
  const float x_near = clampf(0.0f, dx0, dx1);
  const float y1 = clampf(-b * x_near / std::fmax(c, 1e-12f), dy0, dy1);
  const float q1 = a * x_near * x_near + 2.0f * b * x_near * y1 + c * y1 * y1;
  const float y_near = clampf(0.0f, dy0, dy1);
  const float x2 = clampf(-b * y_near / std::fmax(a, 1e-12f), dx0, dx1);
  const float q2 = a * x2 * x2 + 2.0f * b * x2 * y_near + c * y_near * y_near;
  const float q_cut = clampf(2.0f * logf(255.0f * alpha), 0.0f, 8.0f);
  return std::fmin(q1, q2) <= q_cut + 1e-4f ? 1 : 0;
}

// compute_gaussian_tile_bounds_xy (render/tiles/mod.rs:97-130), 16x16 tiles:
// returns 0 when culled or off screen, else 1 with box = tx0, tx1, ty0, ty1.
int orc_ref_tile_bounds_xy(float cxp, float cyp, float ex, float ey, uint32_t tiles_x,
                           uint32_t tiles_y, uint32_t W, uint32_t H, uint32_t* box) {
  const uint32_t tw = g_tile_w, th = g_tile_h;
  g_tile_w = g_tile_h = 16;
  TileBox tb{};
  const bool ok = tile_bounds_xy(cxp, cyp, ex, ey, tiles_x, tiles_y, W, H, &tb);
  g_tile_w = tw;
  g_tile_h = th;
  if (!ok) return 0;
  box[0] = tb.x0;
  box[1] = tb.x1;
  box[2] = tb.y0;
  box[3] = tb.y1;
  return 1;
}

// pack_relative_depth_bits (render/kernels/binning.rs:25-31).
uint32_t orc_pack_depth(float tz, float near_plane, uint32_t depth_bits) {
  const uint32_t db = std::min(depth_bits, 28u);
  const uint32_t base = f2u(std::fmax(near_plane, 1e-6f)) & 0x7F800000u;
  const uint32_t raw = f2u(std::fmax(tz, 1e-6f));
  const uint32_t rel = raw > base ? std::min(raw - base, 0x0FFFFFFFu) : 0u;
  return rel >> (28u - db);
}

// Reference CPU tet transforms (for tests): J, R column-major, max stretch.
void orc_ref_tet_transforms(uint32_t T, const float* verts, const uint32_t* elems,
                            const float* inv_dm, float* J, float* R, float* stretch) {
  for (uint32_t t = 0; t < T; ++t) {
    RefTet r = ref_tet_transform(verts, elems + 4 * t, inv_dm + 9 * t);
    std::memcpy(J + 9 * t, r.J.c, 36);
    std::memcpy(R + 9 * t, r.R.c, 36);
    stretch[t] = r.max_stretch;
  }
}

// sh_rotation_matrix (sh_rotation.rs:367-385) for band l in 1..3: the row-major
// (2l+1)^2 f32 matrix for rotation R (column-major 9).
void orc_sh_rotation_matrix(const float* R9, uint32_t l, float* out) {
  M3 R;
  std::memcpy(R.c, R9, 36);
  sh_rotation_matrix(R, (int)l, out);
}

// Rotates SH coefficients [n*48] in place by rotation R (column-major 9) up to
// `degree` (ShRotator::apply).
void orc_ref_sh_rotate(uint32_t n, float* sh, const float* R9, uint32_t degree) {
  M3 R;
  std::memcpy(R.c, R9, 36);
  ShRot r = make_sh_rotator(R, (int)std::min(degree, 3u));
  for (uint32_t i = 0; i < n; ++i) apply_sh_rotation(r, sh + 48 * (size_t)i);
}

// deform_cage_scene_cpu (deformation/cpu_reference.rs:157-404) for one tet
// cage set: position sum, J S J^T with the 1e-4 floor, det-J opacity rule,
// SH coefficients rotated per tet (degree sh_degree), then the sequential
// strain split with the f64 eigen-solver and the 3D Mip filter. Children are
// appended in parent order. Returns the output count (n + children).
static uint32_t ref_deform_scene(uint32_t n, const float* pos, const float* cov, const float* opa,
                                 const float* sh, uint32_t T, const float* verts,
                                 const uint32_t* elems, const float* inv_dm,
                                 const uint32_t* bind_tet, const float* bind_w,
                                 uint32_t sh_degree, float split_thr, float mip,
                                 std::vector<float>& dpos, std::vector<float>& dcov,
                                 std::vector<float>& dopa, std::vector<float>& dsh) {
  dpos.assign(pos, pos + 3 * (size_t)n);
  dcov.assign(cov, cov + 6 * (size_t)n);
  dopa.assign(opa, opa + n);
  dsh.assign(sh, sh + 48 * (size_t)n);
  const bool has_cages = T > 0;
  uint32_t total = n;
  if (has_cages) {
    std::vector<RefTet> tets(T);
    for (uint32_t t = 0; t < T; ++t) tets[t] = ref_tet_transform(verts, elems + 4 * t, inv_dm + 9 * t);
    const uint32_t deg = std::min(sh_degree, 3u);
    std::vector<ShRot> rots;
    if (deg > 0) {
      rots.resize(T);
      for (uint32_t t = 0; t < T; ++t) rots[t] = make_sh_rotator(tets[t].R, (int)deg);
    }
    parallel_for(n, [&](size_t b, size_t e) {
      for (size_t i = b; i < e; ++i) {
        const uint32_t tr = bind_tet[i];
        if (tr >= T) {
          float c6[6];
          std::memcpy(c6, cov + 6 * i, 24);
          float a = opa[i];
          if (mip > 0.0f) ref_mip3d(c6, &a, mip);
          std::memcpy(&dcov[6 * i], c6, 24);
          dopa[i] = a;
          continue;
        }
        const uint32_t* el = elems + 4 * tr;
        const float* w = bind_w + 4 * i;
        for (int k = 0; k < 3; ++k)
          dpos[3 * i + k] = ((w[0] * verts[3 * el[0] + k] + w[1] * verts[3 * el[1] + k]) +
                             w[2] * verts[3 * el[2] + k]) + w[3] * verts[3 * el[3] + k];
        const float* c = cov + 6 * i;
        M3 S = {{c[0], c[1], c[2], c[1], c[3], c[4], c[2], c[4], c[5]}};
        const M3& J = tets[tr].J;
        M3 m = m3_mul(m3_mul(J, S), m3_t(J));
        float* o = &dcov[6 * i];
        o[0] = std::fmax(m.at(0, 0), 1e-4f);
        o[1] = 0.5f * (m.at(0, 1) + m.at(1, 0));
        o[2] = 0.5f * (m.at(0, 2) + m.at(2, 0));
        o[3] = std::fmax(m.at(1, 1), 1e-4f);
        o[4] = 0.5f * (m.at(1, 2) + m.at(2, 1));
        o[5] = std::fmax(m.at(2, 2), 1e-4f);
        const float s_det = clampf(m3_det(J), 0.6f, 1.8f);
        const float safe_base = clampf(1.0f - opa[i], 1e-4f, 0.999f);
        dopa[i] = clampf(1.0f - powf(safe_base, 1.0f / s_det), 0.05f, 0.99f);
        if (deg > 0) apply_sh_rotation(rots[tr], &dsh[48 * i]);
      }
    });
    // Split pass (cpu_reference.rs:304-393), sequential as in the reference.
    for (uint32_t i = 0; i < n; ++i) {
      const uint32_t tr = bind_tet[i];
      const bool split = split_thr > 0.0f && tr < T && tets[tr].max_stretch > split_thr;
      if (!split) {
        if (split_thr > 0.0f || mip > 0.0f) {
          if (tr < T && mip > 0.0f) ref_mip3d(&dcov[6 * i], &dopa[i], mip);
        }
        continue;
      }
      float ev[3];
      M3 B;
      sym_eigen3(&dcov[6 * i], ev, &B);
      const float min_var = 1e-4f * 1e-4f;
      const float l0 = std::fmax(ev[0] * 0.25f, min_var), l1 = std::fmax(ev[1], min_var),
                  l2 = std::fmax(ev[2], min_var);
      float ax[3] = {B.c[0], B.c[1], B.c[2]};
      const float len2 = dot3(ax, ax);
      if (len2 > 0.0f) {
        const float inv = 1.0f / std::sqrt(len2);
        for (auto& a : ax) a *= inv;
      }
      const float om = 0.5f * std::sqrt(std::fmax(ev[0], min_var));
      M3 D = {{l0, 0, 0, 0, l1, 0, 0, 0, l2}};
      M3 cm = m3_mul(m3_mul(B, D), m3_t(B));
      float cc[6] = {cm.at(0, 0), cm.at(0, 1), cm.at(0, 2), cm.at(1, 1), cm.at(1, 2), cm.at(2, 2)};
      float ca[6], cb[6];
      std::memcpy(ca, cc, 24);
      std::memcpy(cb, cc, 24);
      float aa = dopa[i], ab = dopa[i];
      if (mip > 0.0f) {
        ref_mip3d(ca, &aa, mip);
        ref_mip3d(cb, &ab, mip);
      }
      float center[3] = {dpos[3 * i], dpos[3 * i + 1], dpos[3 * i + 2]};
      for (int k = 0; k < 3; ++k) dpos[3 * i + k] = center[k] + (-(ax[k] * om));
      std::memcpy(&dcov[6 * i], ca, 24);
      dopa[i] = aa;
      for (int k = 0; k < 3; ++k) dpos.push_back(center[k] + ax[k] * om);
      dcov.insert(dcov.end(), cb, cb + 6);
      dopa.push_back(ab);
      dsh.insert(dsh.end(), dsh.begin() + 48 * (size_t)i, dsh.begin() + 48 * (size_t)i + 48);
      ++total;
    }
  }
  return total;
}

// deform_cage_scene_cpu / deform_scene_adaptive_cpu restated (ref mode, one
// tet cage set, see ref_deform_scene). Outputs hold 2n slots (out_sh 2n x 48);
// returns the output count.
uint32_t orc_ref_deform(uint32_t n, const float* pos, const float* cov, const float* opa,
                        const float* sh, uint32_t T, const float* verts, const uint32_t* elems,
                        const float* inv_dm, const uint32_t* bind_tet, const float* bind_w,
                        uint32_t sh_degree, float split_thr, float mip, float* out_pos,
                        float* out_cov, float* out_opa, float* out_sh) {
  std::vector<float> dpos, dcov, dopa, dsh;
  const uint32_t total = ref_deform_scene(n, pos, cov, opa, sh, T, verts, elems, inv_dm, bind_tet,
                                          bind_w, sh_degree, split_thr, mip, dpos, dcov, dopa, dsh);
  std::memcpy(out_pos, dpos.data(), sizeof(float) * 3 * (size_t)total);
  std::memcpy(out_cov, dcov.data(), sizeof(float) * 6 * (size_t)total);
  std::memcpy(out_opa, dopa.data(), sizeof(float) * (size_t)total);
  if (out_sh) std::memcpy(out_sh, dsh.data(), sizeof(float) * 48 * (size_t)total);
  return total;
}

// execute_cpu_reference_with_options (render/pipeline.rs:420-507) for one tet
// cage set: deform_cage_scene_cpu (SH coefficients rotated per tet, strain
// split with the f64 eigen-solver, 3D Mip filter), project_scene_cull_cpu
// (sequential loop, render/mod.rs:226-285), bin_and_sort_active (square radius,
// tiles/cpu_reference.rs:307-402) and rasterize_scene_cpu. `verts` are the
// current flattened cage vertices; bind_tet holds global tet indices.
// Returns the number of tile entries; *out_splits receives the child count.
uint64_t orc_ref_frame(uint32_t n, const float* pos, const float* cov, const float* opa,
                       const float* sh, uint32_t T, const float* verts, const uint32_t* elems,
                       const float* inv_dm, const uint32_t* bind_tet, const float* bind_w,
                       const float* cam24, uint32_t W, uint32_t H, const float* bg,
                       const float* cam_pos, uint32_t sh_degree, float split_thr, float mip,
                       uint8_t* rgba8, uint32_t* out_splits) {
  const bool has_cages = T > 0;
  std::vector<float> dpos, dcov, dopa, dsh;
  const uint32_t total = ref_deform_scene(n, pos, cov, opa, sh, T, verts, elems, inv_dm, bind_tet,
                                          bind_w, sh_degree, split_thr, mip, dpos, dcov, dopa, dsh);
  if (out_splits) *out_splits = total - n;
  // project_scene_cull_cpu: sequential loop (render/mod.rs:248).
  std::vector<float> xy(2 * (size_t)total), depth(total), conic(3 * (size_t)total),
      copa(total);
  std::vector<int32_t> radius(total);
  const float fx = cam24[16], fy = cam24[17], cx = cam24[18], cy = cam24[19];
  const float vw = cam24[20], vh = cam24[21], near_p = cam24[22];
  const float mip2 = has_cages ? 0.0f : mip;
  const bool cull = split_thr > 0.0f || mip > 0.0f;
  if (!cull) {
    orc_ref_project_scene(total, dpos.data(), dcov.data(), cam24, xy.data(), depth.data(),
                          radius.data(), conic.data());
    copa = dopa;
  } else {
    for (uint32_t i = 0; i < total; ++i) {
      const float* p = &dpos[3 * i];
      const float* V = cam24;
      const float tx = ((V[0] * p[0] + V[4] * p[1]) + V[8] * p[2]) + V[12];
      const float ty = ((V[1] * p[0] + V[5] * p[1]) + V[9] * p[2]) + V[13];
      const float tz = ((V[2] * p[0] + V[6] * p[1]) + V[10] * p[2]) + V[14];
      depth[i] = tz;
      radius[i] = 0;
      copa[i] = 0.0f;
      xy[2 * i] = xy[2 * i + 1] = 0.0f;
      conic[3 * i] = conic[3 * i + 1] = conic[3 * i + 2] = 0.0f;
      if (tz <= near_p) continue;
      float c6[6];
      std::memcpy(c6, &dcov[6 * i], 24);
      float a3 = dopa[i];
      if (mip2 > 0.0f) ref_mip3d(c6, &a3, mip2);
      if (a3 < 1.0f / 255.0f) continue;
      const float inv_tz = 1.0f / tz, inv_tz2 = inv_tz * inv_tz;
      const float j00 = fx * inv_tz, j02 = -fx * tx * inv_tz2, j11 = fy * inv_tz,
                  j12 = -fy * ty * inv_tz2;
      M3 Wm = {{V[0], V[1], V[2], V[4], V[5], V[6], V[8], V[9], V[10]}};
      M3 S = {{c6[0], c6[1], c6[2], c6[1], c6[3], c6[4], c6[2], c6[4], c6[5]}};
      M3 Cm = m3_mul(m3_mul(Wm, S), m3_t(Wm));
      const float c_xx = Cm.c[0], c_xy = Cm.c[1], c_xz = Cm.c[2], c_yy = Cm.c[4], c_yz = Cm.c[5],
                  c_zz = Cm.c[8];
      const float m00 = j00 * c_xx + j02 * c_xz, m01 = j00 * c_xy + j02 * c_yz,
                  m02 = j00 * c_xz + j02 * c_zz, m11 = j11 * c_yy + j12 * c_yz,
                  m12 = j11 * c_yz + j12 * c_zz;
      const float sxx = m00 * j00 + m02 * j02, sxy = m01 * j11 + m02 * j12,
                  syy = m11 * j11 + m12 * j12;
      const float raw_mid = 0.5f * (sxx + syy);
      const float raw_det = sxx * syy - sxy * sxy;
      const float raw_discr = std::sqrt(std::fmax(raw_mid * raw_mid - raw_det, 0.0f));
      const float rlmax = std::fmax(raw_mid + raw_discr, 0.0f);
      if (3.0f * std::sqrt(rlmax) < 0.5f) continue;
      // apply_ewa_low_pass_2d (covariance.rs:310-330)
      const float det_o = std::fmax(sxx * syy - sxy * sxy, 0.0f);
      const float rx = sxx + 0.3f, ry = syy + 0.3f;
      const float det_r = std::fmax(rx * ry - sxy * sxy, 1e-12f);
      const float a2 = clampf(a3 * std::sqrt(clampf(det_o / det_r, 0.0f, 1.0f)), 0.0f, 1.0f);
      if (a2 < 1.0f / 255.0f) continue;
      const float det = rx * ry - sxy * sxy;
      if (det <= 1e-6f) continue;
      const float inv_det = 1.0f / det;
      const float cn[3] = {ry * inv_det, -sxy * inv_det, rx * inv_det};
      const float mid = 0.5f * (rx + ry);
      const float discr = std::sqrt(std::fmax(mid * mid - det, 0.1f));
      const float lmax = std::fmax(mid + discr, std::fmax(mid - discr, 0.1f));
      const float r = clampf(std::ceil(3.0f * std::sqrt(lmax)), 1.0f, 1024.0f);
      const float mx = fx * tx * inv_tz + cx, my = fy * ty * inv_tz + cy;
      xy[2 * i] = mx;
      xy[2 * i + 1] = my;
      conic[3 * i] = cn[0];
      conic[3 * i + 1] = cn[1];
      conic[3 * i + 2] = cn[2];
      if (mx + r < 0.0f || mx - r >= vw || my + r < 0.0f || my - r >= vh) continue;
      radius[i] = (int32_t)r;
      copa[i] = a2;
    }
  }
  // Binning: bin_and_sort_active when culling projection ran, else bin_and_sort.
  const uint32_t tiles = ((W + 15) / 16) * ((H + 15) / 16);
  const uint64_t e = orc_ref_bin_and_sort(total, xy.data(), depth.data(), radius.data(), W, H,
                                          nullptr, nullptr, nullptr, nullptr);
  std::vector<uint32_t> t(e), d(e), ids(e), ranges(2 * (size_t)tiles);
  orc_ref_bin_and_sort(total, xy.data(), depth.data(), radius.data(), W, H, t.data(), d.data(),
                       ids.data(), ranges.data());
  orc_ref_rasterize(W, H, xy.data(), conic.data(), copa.data(), dsh.data(), dpos.data(),
                    ids.data(), ranges.data(), bg, cam_pos, sh_degree, rgba8, nullptr);
  return e;
}

// ------------------------------------------------------------ MVC (ref)
float orc_mvc_winding(uint32_t F, const float* verts, const uint32_t* tris, const float* p) {
  return mvc_winding(F, verts, tris, v3(p));
}

void orc_mvc_weights(uint32_t n, const float* pts, uint32_t V, const float* verts, uint32_t F,
                     const uint32_t* tris, float* w) {
  parallel_for(n, [&](size_t b, size_t e) {
    for (size_t i = b; i < e; ++i) mvc_weights(V, F, verts, tris, v3(pts + 3 * i), w + V * i);
  });
}

float orc_mvc_step(uint32_t V, const float* verts) { return mvc_step(V, verts); }

// bind_gaussians (mvc.rs:498-541): inside flag, weights and central-difference
// gradients (w, dw/dx, dw/dy, dw/dz) per point and cage vertex.
void orc_mvc_bind(uint32_t n, const float* pts, uint32_t V, const float* verts, uint32_t F,
                  const uint32_t* tris, uint8_t* inside, float* wg /* [n][V][4] */) {
  const float h = mvc_step(V, verts);
  const float inv_2h = 0.5f / h;
  parallel_for(n, [&](size_t b, size_t e) {
    std::vector<float> wp(V), wm(V);
    for (size_t i = b; i < e; ++i) {
      const V3 p = v3(pts + 3 * i);
      float* out = wg + 4 * (size_t)V * i;
      const bool in = std::fabs(mvc_winding(F, verts, tris, p)) >= 0.5f;
      inside[i] = in ? 1 : 0;
      if (!in) {
        for (uint32_t j = 0; j < 4 * V; ++j) out[j] = 0.0f;
        continue;
      }
      mvc_weights(V, F, verts, tris, p, wp.data());
      for (uint32_t j = 0; j < V; ++j) out[4 * j] = wp[j];
      for (int axis = 0; axis < 3; ++axis) {
        float pp[3] = {p.x, p.y, p.z}, pm[3] = {p.x, p.y, p.z};
        pp[axis] += h;
        pm[axis] -= h;
        mvc_weights(V, F, verts, tris, v3(pp), wp.data());
        mvc_weights(V, F, verts, tris, v3(pm), wm.data());
        for (uint32_t j = 0; j < V; ++j) out[4 * j + 1 + axis] = (wp[j] - wm[j]) * inv_2h;
      }
    }
  });
}

// deform_scene_cpu (mvc.rs:564-749) without the SH coefficient rotation:
// position sum w v, F = sum v g^T (MvcBindings::local_jacobian), rotation by
// higham_polar_decomposition, covariance F S F^T, opacity unchanged, strain
// split and 3D Mip. Returns the output count; out_R gets each input Gaussian's
// rotation (identity when unbound), split children are appended in parent
// order.
uint32_t orc_mvc_deform(uint32_t n, const float* pos, const float* cov, const float* opa,
                        const uint8_t* inside, const float* wg, uint32_t V, const float* dverts,
                        float split_thr, float mip, float* out_pos, float* out_cov,
                        float* out_opa, uint32_t* out_parent, float* out_R) {
  std::vector<float> P(pos, pos + 3 * (size_t)n), C(cov, cov + 6 * (size_t)n), A(opa, opa + n);
  std::vector<M3> Fs(n);
  std::vector<uint8_t> split(n, 0);
  for (uint32_t i = 0; i < n; ++i) {
    M3 I = {{1, 0, 0, 0, 1, 0, 0, 0, 1}};
    if (out_R) std::memcpy(out_R + 9 * (size_t)i, I.c, 36);
    if (!inside[i]) continue;
    const float* row = wg + 4 * (size_t)V * i;
    V3 p = {0, 0, 0}, c0 = {0, 0, 0}, c1 = {0, 0, 0}, c2 = {0, 0, 0};
    for (uint32_t j = 0; j < V; ++j) {
      const V3 v = v3(dverts + 3 * j);
      p = p + v * row[4 * j];
      c0 = c0 + v * row[4 * j + 1];
      c1 = c1 + v * row[4 * j + 2];
      c2 = c2 + v * row[4 * j + 3];
    }
    M3 Fm = {{c0.x, c0.y, c0.z, c1.x, c1.y, c1.z, c2.x, c2.y, c2.z}};
    Fs[i] = Fm;
    const M3 R = higham_polar(Fm);
    if (out_R) std::memcpy(out_R + 9 * (size_t)i, R.c, 36);
    const float* c = cov + 6 * (size_t)i;
    M3 S = {{c[0], c[1], c[2], c[1], c[3], c[4], c[2], c[4], c[5]}};
    M3 m = m3_mul(m3_mul(Fm, S), m3_t(Fm));
    P[3 * i] = p.x;
    P[3 * i + 1] = p.y;
    P[3 * i + 2] = p.z;
    float* o = &C[6 * (size_t)i];
    o[0] = m.at(0, 0); o[1] = m.at(0, 1); o[2] = m.at(0, 2);
    o[3] = m.at(1, 1); o[4] = m.at(1, 2); o[5] = m.at(2, 2);
    if (split_thr > 0.0f) {
      M3 Cg = m3_mul(m3_t(Fm), Fm);
      const float packed[6] = {Cg.at(0, 0), Cg.at(0, 1), Cg.at(0, 2), Cg.at(1, 1), Cg.at(1, 2),
                               Cg.at(2, 2)};
      float ev[3];
      M3 basis;
      sym_eigen3(packed, ev, &basis);
      split[i] = std::sqrt(std::fmax(ev[0], 0.0f)) > split_thr ? 1 : 0;
    }
  }
  std::vector<uint32_t> parent;
  uint32_t total = n;
  for (uint32_t i = 0; i < n; ++i) {
    if (!split[i]) {
      if (mip > 0.0f) ref_mip3d(&C[6 * (size_t)i], &A[i], mip);
      continue;
    }
    float ev[3];
    M3 B;
    sym_eigen3(&C[6 * (size_t)i], ev, &B);
    const float min_var = 1e-4f * 1e-4f;
    const float l0 = std::fmax(ev[0] * 0.25f, min_var), l1 = std::fmax(ev[1], min_var),
                l2 = std::fmax(ev[2], min_var);
    float ax[3] = {B.c[0], B.c[1], B.c[2]};
    const float len2 = dot3(ax, ax);
    if (len2 > 0.0f) {
      const float inv = 1.0f / std::sqrt(len2);
      for (auto& v : ax) v *= inv;
    }
    const float om = 0.5f * std::sqrt(std::fmax(ev[0], min_var));
    M3 D = {{l0, 0, 0, 0, l1, 0, 0, 0, l2}};
    M3 cm = m3_mul(m3_mul(B, D), m3_t(B));
    float cc[6] = {cm.at(0, 0), cm.at(0, 1), cm.at(0, 2), cm.at(1, 1), cm.at(1, 2), cm.at(2, 2)};
    float ca[6], cb[6];
    std::memcpy(ca, cc, 24);
    std::memcpy(cb, cc, 24);
    float aa = A[i], ab = A[i];
    if (mip > 0.0f) {
      ref_mip3d(ca, &aa, mip);
      ref_mip3d(cb, &ab, mip);
    }
    float center[3] = {P[3 * i], P[3 * i + 1], P[3 * i + 2]};
    for (int k = 0; k < 3; ++k) P[3 * i + k] = center[k] + (-(ax[k] * om));
    std::memcpy(&C[6 * (size_t)i], ca, 24);
    A[i] = aa;
    for (int k = 0; k < 3; ++k) P.push_back(center[k] + ax[k] * om);
    C.insert(C.end(), cb, cb + 6);
    A.push_back(ab);
    parent.push_back(i);
    ++total;
  }
  if (out_pos) std::memcpy(out_pos, P.data(), 12 * (size_t)total);
  if (out_cov) std::memcpy(out_cov, C.data(), 24 * (size_t)total);
  if (out_opa) std::memcpy(out_opa, A.data(), 4 * (size_t)total);
  if (out_parent && !parent.empty()) std::memcpy(out_parent, parent.data(), 4 * parent.size());
  return total;
}


// ------------------------------------------------------------ cage springs
// CageSpringSimulator (deformation/dynamics.rs:75-313) for one cage: rest,
// current and velocity [V*3], pinned [V] (0/1), collision planes [P*8]
// (nx, ny, nz, offset, restitution, friction, pad, pad).

static float spring_min(float a, float b) {  // f32::min: NaN yields the other
  if (std::isnan(a)) return b;
  if (std::isnan(b)) return a;
  return a < b ? a : b;
}
static float spring_max(float a, float b) {
  if (std::isnan(a)) return b;
  if (std::isnan(b)) return a;
  return a > b ? a : b;
}
// damping_coefficient / frame_damping (dynamics.rs:137-148)
float orc_spring_frame_damping(float damping, float dt) {
  float r = damping;
  if (r < 1.0e-4f) r = 1.0e-4f;
  if (r > 0.9999f) r = 0.9999f;
  const float c = -logf(r) * 60.0f;
  return expf(-c * dt);
}

// CollisionPlane::resolve_contact (dynamics.rs:57-71).
static void spring_contact(const float* pl, float* p, float* v) {
  const float d = ((pl[0] * p[0] + pl[1] * p[1]) + pl[2] * p[2]) - pl[3];
  if (d >= 0.0f) return;
  for (int k = 0; k < 3; ++k) p[k] = p[k] - pl[k] * d;
  const float vn = (v[0] * pl[0] + v[1] * pl[1]) + v[2] * pl[2];
  if (vn < 0.0f) {
    float vnorm[3], vtan[3];
    for (int k = 0; k < 3; ++k) vnorm[k] = pl[k] * vn;
    for (int k = 0; k < 3; ++k) vtan[k] = v[k] - vnorm[k];
    const float keep = 1.0f - pl[5];
    for (int k = 0; k < 3; ++k) v[k] = vtan[k] * keep - vnorm[k] * pl[4];
  }
}

// CageSpringSimulator::step (dynamics.rs:249-277).
void orc_spring_step(uint32_t V, const float* rest, float* cur, float* vel, const uint8_t* pinned,
                     float stiffness, float damping, float mass, uint32_t num_planes,
                     const float* planes, float dt) {
  const float dt_sim = spring_min(dt, 0.033f);
  if (!(dt_sim > 0.0f)) return;
  const float inv_mass = 1.0f / spring_max(mass, 0.001f);
  const float gamma = orc_spring_frame_damping(damping, dt_sim);
  const float kim = stiffness * inv_mass;
  for (uint32_t i = 0; i < V; ++i) {
    float* x = cur + 3 * (size_t)i;
    float* v = vel + 3 * (size_t)i;
    if (pinned && pinned[i]) {
      v[0] = v[1] = v[2] = 0.0f;
      continue;
    }
    for (int k = 0; k < 3; ++k) {
      const float accel = (rest[3 * (size_t)i + k] - x[k]) * kim;
      v[k] = (v[k] + accel * dt_sim) * gamma;
      x[k] = x[k] + v[k] * dt_sim;
    }
    for (uint32_t q = 0; q < num_planes; ++q) spring_contact(planes + 8 * (size_t)q, x, v);
  }
}

// CageSpringSimulator::trigger_jiggle_impulse (dynamics.rs:280-305).
void orc_spring_impulse(uint32_t V, const float* rest, float* vel, const uint8_t* pinned,
                        float magnitude) {
  if (V == 0) return;
  float c[3] = {0.0f, 0.0f, 0.0f};
  for (uint32_t i = 0; i < V; ++i)
    for (int k = 0; k < 3; ++k) c[k] = c[k] + rest[3 * (size_t)i + k];
  for (int k = 0; k < 3; ++k) c[k] = c[k] / (float)V;
  for (uint32_t i = 0; i < V; ++i) {
    if (pinned && pinned[i]) continue;
    float d[3];
    for (int k = 0; k < 3; ++k) d[k] = rest[3 * (size_t)i + k] - c[k];
    const float rcp = 1.0f / sqrtf((d[0] * d[0] + d[1] * d[1]) + d[2] * d[2]);
    float r[3] = {0.0f, 0.0f, 0.0f};  // normalize_or_zero
    if (std::isfinite(rcp) && rcp > 0.0f)
      for (int k = 0; k < 3; ++k) r[k] = d[k] * rcp;
    float imp[3];
    if ((r[0] * r[0] + r[1] * r[1]) + r[2] * r[2] > 1e-4f) {
      for (int k = 0; k < 3; ++k) imp[k] = r[k] * magnitude;
    } else {
      imp[0] = 0.0f * magnitude;
      imp[1] = 1.0f * magnitude;
      imp[2] = 0.0f * magnitude;
    }
    for (int k = 0; k < 3; ++k) vel[3 * (size_t)i + k] = vel[3 * (size_t)i + k] + imp[k];
  }
}

}  // extern "C"
