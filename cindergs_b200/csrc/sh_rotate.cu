// SH coefficient rotation and the deformed-scene export on sm_100a.
//
//  k_sh_basis      once per context: for bands l = 1..3 the constant matrix
//                  B_l of the real SH basis over the degree-l monomials and
//                  its right pseudo-inverse B_l^+ = B_l^T (B_l B_l^T)^-1
//                  (basis_rows / basis_for, render/rasterizer/sh_rotation.rs:
//                  139-330).
//  k_sh_rotators   one thread per rotation (a tet's or an MVC slot's polar
//                  rotation): the monomial transform T_l(R^T) and the f32
//                  band matrices M_l = (B_l T_l B_l^+)^T
//                  (sh_rotation_matrix, sh_rotation.rs:332-385), 84 floats per
//                  rotation (M1 9, M2 25, M3 49, one pad).
//  k_sh_apply      rotates coefficient blocks in place by a table row
//                  (ShRotator::apply, sh_rotation.rs:389-440).
//  k_export        one thread per deformed splat: position, covariance and
//                  opacity from Stage 1's output, SH of the splat (a child's
//                  are its parent's) rotated by its tet's or MVC slot's
//                  rotation, written as a structure-of-arrays chunk for the
//                  host (write_deformed + deform_cage_scene_cpu's per-tet
//                  ShRotator, deformation/cpu_reference.rs:157-404).
//
// Live frames never rotate coefficients: Stage 2 evaluates the rest-pose SH
// along R^T d. Coefficient rotation is for exporting a deformed scene.
//
// This file is compiled with -fmad=false: the f64 construction follows the
// reference's operation order (poly_mul_linear's accumulation order, mat_mul
// over k ascending with zero terms skipped, Gauss-Jordan with the last
// maximal pivot) and the f32 application keeps its running sum, so the
// matrices and the rotated coefficients equal the host restatement bit for
// bit.
#include <cuda_fp16.h>

#include "kernels.h"

namespace cgs {
namespace {

struct ShBasisDev {
  double B[3][70];  // row-major (2l+1) x m_l
  double P[3][70];  // row-major m_l x (2l+1)
};

__device__ __forceinline__ int mono_count(int d) { return (d + 1) * (d + 2) / 2; }

// Monomial order of exps_of (sh_rotation.rs:47-56): x exponent descending,
// then y descending. Index of (x, y, d - x - y):
__device__ __forceinline__ int mono_index(int d, int x, int y) {
  int k = 0;
  for (int xp = d; xp > x; --xp) k += d - xp + 1;
  return k + (d - x - y);
}
__device__ __forceinline__ void mono_exps(int d, int k, int* e) {
  int idx = 0;
  for (int x = d; x >= 0; --x)
    for (int y = d - x; y >= 0; --y) {
      if (idx == k) {
        e[0] = x;
        e[1] = y;
        e[2] = d - x - y;
        return;
      }
      ++idx;
    }
}

// mat_mul (sh_rotation.rs:228-245): out[i][j] = sum over k ascending of
// a[i][k] b[k][j], skipping a[i][k] == 0.
__device__ void mat_mul(int r, int inner, int c, const double* a, const double* b, double* out) {
  for (int i = 0; i < r * c; ++i) out[i] = 0.0;
  for (int i = 0; i < r; ++i)
    for (int k = 0; k < inner; ++k) {
      const double aik = a[i * inner + k];
      if (aik == 0.0) continue;
      for (int j = 0; j < c; ++j) out[i * c + j] += aik * b[k * c + j];
    }
}

// basis_rows (sh_rotation.rs:139-226): integer monomial coefficients of each
// real SH row times the band constant.
__device__ void basis_rows(int l, double* B) {
  const double C1 = 0.4886025119029199, C2_0 = 1.0925484305920792, C2_2 = 0.31539156525252005,
               C2_4 = 0.5462742152960396, C3_0 = -0.5900435899266435, C3_1 = 2.890611442640554,
               C3_2 = -0.4570457994644658, C3_3 = 0.3731763325901154, C3_5 = 1.445305721320277;
  const int m = mono_count(l), n = 2 * l + 1;
  for (int i = 0; i < n * m; ++i) B[i] = 0.0;
  auto put = [&](int row, int mono, double k, double c) { B[row * m + mono] = k * c; };
  if (l == 1) {  // x y z
    put(0, 1, 1.0, -C1);
    put(1, 2, 1.0, C1);
    put(2, 0, 1.0, -C1);
  } else if (l == 2) {  // xx xy xz yy yz zz
    put(0, 1, 1.0, C2_0);
    put(1, 4, 1.0, -C2_0);
    put(2, 0, -1.0, C2_2);
    put(2, 3, -1.0, C2_2);
    put(2, 5, 2.0, C2_2);
    put(3, 2, 1.0, -C2_0);
    put(4, 0, 1.0, C2_4);
    put(4, 3, -1.0, C2_4);
  } else {  // xxx xxy xxz xyy xyz xzz yyy yyz yzz zzz
    put(0, 1, 3.0, C3_0);
    put(0, 6, -1.0, C3_0);
    put(1, 4, 1.0, C3_1);
    put(2, 1, -1.0, C3_2);
    put(2, 6, -1.0, C3_2);
    put(2, 8, 4.0, C3_2);
    put(3, 2, -3.0, C3_3);
    put(3, 7, -3.0, C3_3);
    put(3, 9, 2.0, C3_3);
    put(4, 0, -1.0, C3_2);
    put(4, 3, -1.0, C3_2);
    put(4, 5, 4.0, C3_2);
    put(5, 2, 1.0, C3_5);
    put(5, 7, -1.0, C3_5);
    put(6, 0, 1.0, C3_0);
    put(6, 3, -3.0, C3_0);
  }
}

__global__ void k_sh_basis(ShBasisDev* out) {
  const int l = threadIdx.x + 1;
  if (l > 3) return;
  const int m = mono_count(l), n = 2 * l + 1;
  double* B = out->B[l - 1];
  basis_rows(l, B);
  double Bt[70], G[49];
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < m; ++j) Bt[j * n + i] = B[i * m + j];
  mat_mul(n, m, n, B, Bt, G);
  // invert (sh_rotation.rs:260-300): Gauss-Jordan, pivot = the last row of
  // the largest magnitude, pivot row multiplied by 1 / pivot. The Gram
  // matrix of a band is far from singular.
  double aug[7][14];
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < 2 * n; ++j) aug[i][j] = j < n ? G[i * n + j] : (j - n == i ? 1.0 : 0.0);
  for (int col = 0; col < n; ++col) {
    int piv = col;
    for (int r = col + 1; r < n; ++r)
      if (!(fabs(aug[piv][col]) > fabs(aug[r][col]))) piv = r;
    if (piv != col)
      for (int j = 0; j < 2 * n; ++j) {
        const double t = aug[col][j];
        aug[col][j] = aug[piv][j];
        aug[piv][j] = t;
      }
    const double inv = 1.0 / aug[col][col];
    for (int j = 0; j < 2 * n; ++j) aug[col][j] *= inv;
    for (int r = 0; r < n; ++r) {
      if (r == col) continue;
      const double f = aug[r][col];
      if (f == 0.0) continue;
      for (int j = 0; j < 2 * n; ++j) aug[r][j] -= f * aug[col][j];
    }
  }
  double Gi[49];
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) Gi[i * n + j] = aug[i][n + j];
  mat_mul(m, n, n, Bt, Gi, out->P[l - 1]);
}

// sh_rotation_matrix (sh_rotation.rs:354-387) for band L: the f32 matrix
// M[row * n + col] = D[col][row], D = B T B^+.
template <int L>
__device__ void band_matrix(const double (*lf)[3], const ShBasisDev& basis, float* M) {
  constexpr int m = (L + 1) * (L + 2) / 2, n = 2 * L + 1;
  double T[m * m];
  for (int row = 0; row < m; ++row) {
    int e[3];
    mono_exps(L, row, e);
    // poly_mul_linear (sh_rotation.rs:332-352), one factor of the row's
    // monomial at a time, x factors first.
    double poly[10] = {1.0, 0, 0, 0, 0, 0, 0, 0, 0, 0}, next[10];
    int deg = 0;
    for (int a = 0; a < 3; ++a)
      for (int rep = 0; rep < e[a]; ++rep) {
        const int nd = mono_count(deg + 1), na = mono_count(deg);
        for (int k = 0; k < nd; ++k) next[k] = 0.0;
        for (int ia = 0; ia < na; ++ia) {
          const double coeff = poly[ia];
          if (coeff == 0.0) continue;
          int ea[3];
          mono_exps(deg, ia, ea);
          for (int ax = 0; ax < 3; ++ax) {
            if (lf[a][ax] == 0.0) continue;
            int ne[3] = {ea[0], ea[1], ea[2]};
            ne[ax] += 1;
            next[mono_index(deg + 1, ne[0], ne[1])] += coeff * lf[a][ax];
          }
        }
        ++deg;
        for (int k = 0; k < nd; ++k) poly[k] = next[k];
      }
    for (int k = 0; k < m; ++k) T[row * m + k] = poly[k];
  }
  double C[n * m], D[n * n];
  mat_mul(n, m, m, basis.B[L - 1], T, C);
  mat_mul(n, m, n, C, basis.P[L - 1], D);
  for (int row = 0; row < n; ++row)
    for (int col = 0; col < n; ++col) M[row * n + col] = (float)D[col * n + row];
}

__global__ void __launch_bounds__(128) k_sh_rotators(uint32_t count, const float* __restrict__ rot,
                                                     const ShBasisDev* __restrict__ basis,
                                                     uint32_t degree, float* __restrict__ table) {
  const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= count) return;
  // monomial_transform: the linear forms are the columns of R (rows of R^T);
  // R is column-major.
  double lf[3][3];
  for (int a = 0; a < 3; ++a)
    for (int k = 0; k < 3; ++k) lf[a][k] = (double)rot[9 * (size_t)r + 3 * a + k];
  float* M = table + (size_t)r * kShRotStride;
  if (degree >= 1) band_matrix<1>(lf, *basis, M);
  if (degree >= 2) band_matrix<2>(lf, *basis, M + 9);
  if (degree >= 3) band_matrix<3>(lf, *basis, M + 34);
}

// apply_block (sh_rotation.rs:389-400) on the three channel blocks of a band.
template <int L>
__device__ __forceinline__ void apply_band(const float* __restrict__ M, float* c) {
  constexpr int n = 2 * L + 1, start = L == 1 ? 0 : (L == 2 ? 3 : 8);
#pragma unroll
  for (int ch = 0; ch < 3; ++ch) {
    float* b = c + 3 + 15 * ch + start;
    float out[n];
#pragma unroll
    for (int row = 0; row < n; ++row) {
      float acc = 0.0f;
#pragma unroll
      for (int col = 0; col < n; ++col) acc += __ldg(M + row * n + col) * b[col];
      out[row] = acc;
    }
#pragma unroll
    for (int j = 0; j < n; ++j) b[j] = out[j];
  }
}
__device__ __forceinline__ void apply_rotator(const float* __restrict__ M, uint32_t degree,
                                              float* c) {
  if (degree >= 1) apply_band<1>(M, c);
  if (degree >= 2) apply_band<2>(M + 9, c);
  if (degree >= 3) apply_band<3>(M + 34, c);
}

__global__ void __launch_bounds__(256) k_sh_apply(uint64_t n, float* __restrict__ sh,
                                                  const float* __restrict__ table,
                                                  uint32_t num_rot, const uint32_t* __restrict__ index,
                                                  uint32_t degree, uint32_t* __restrict__ bad) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t r = index ? index[i] : (uint32_t)(i % num_rot);
  if (r >= num_rot) {
    atomicAdd(bad, 1u);  // left unchanged, reported to the host
    return;
  }
  float c[48];
  float4* p = reinterpret_cast<float4*>(sh + 48 * i);
#pragma unroll
  for (int j = 0; j < 12; ++j) {
    const float4 v = p[j];
    c[4 * j] = v.x; c[4 * j + 1] = v.y; c[4 * j + 2] = v.z; c[4 * j + 3] = v.w;
  }
  apply_rotator(table + (size_t)r * kShRotStride, degree, c);
#pragma unroll
  for (int j = 0; j < 12; ++j) p[j] = make_float4(c[4 * j], c[4 * j + 1], c[4 * j + 2], c[4 * j + 3]);
}

__global__ void __launch_bounds__(256) k_export(const ExportArgs a) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= a.count) return;
  const uint32_t i = a.first + j;
  const float4 p = a.pos[i];
  const float4 ca = a.cova[i];
  const float2 cb = a.covb[i];
  if (a.out_pos) {
    a.out_pos[3 * (size_t)j] = p.x;
    a.out_pos[3 * (size_t)j + 1] = p.y;
    a.out_pos[3 * (size_t)j + 2] = p.z;
  }
  if (a.out_cov) {
    float* o = a.out_cov + 6 * (size_t)j;
    o[0] = ca.x; o[1] = ca.y; o[2] = ca.z; o[3] = ca.w; o[4] = cb.x; o[5] = cb.y;
  }
  if (a.out_opa) a.out_opa[j] = p.w;
  if (!a.out_sh) return;
  // The splat's SH source and rotation: a child carries (parent, tet).
  uint32_t src = i, tet = kInvalid;
  if (i < a.n_rest) {
    if (a.bind_tet) tet = a.bind_tet[i];
  } else {
    const uint2 m = a.split_meta[i - a.n_rest];
    src = m.x;
    tet = m.y;
  }
  float c[48];
  if (!a.sh_f16) {
    const float4* s = reinterpret_cast<const float4*>(a.sh);
#pragma unroll
    for (int q = 0; q < 12; ++q) {
      const float4 v = __ldg(&s[(size_t)q * a.sh_stride + src]);
      c[4 * q] = v.x; c[4 * q + 1] = v.y; c[4 * q + 2] = v.z; c[4 * q + 3] = v.w;
    }
  } else {
    const uint4* s = reinterpret_cast<const uint4*>(a.sh);
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      const uint4 v = __ldg(&s[(size_t)q * a.sh_stride + src]);
      const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
      for (int h = 0; h < 4; ++h) {
        const float2 f = __half22float2(*reinterpret_cast<const __half2*>(&w[h]));
        c[8 * q + 2 * h] = f.x;
        c[8 * q + 2 * h + 1] = f.y;
      }
    }
  }
  if (a.table && a.degree > 0) {
    const float* M = nullptr;
    if (tet < a.num_tets)
      M = a.table + (size_t)tet * kShRotStride;
    else if (tet == kMvcBound && a.mvc)
      M = a.table + ((size_t)a.num_tets + __float_as_uint(a.bind_w[src].x)) * kShRotStride;
    if (M) apply_rotator(M, a.degree, c);
  }
  float* o = a.out_sh + 48 * (size_t)j;
#pragma unroll
  for (int k = 0; k < 48; ++k) o[k] = c[k];
}

}  // namespace

size_t sh_basis_bytes() { return sizeof(ShBasisDev); }

cudaError_t launch_sh_basis(void* basis, cudaStream_t s) {
  k_sh_basis<<<1, 32, 0, s>>>(reinterpret_cast<ShBasisDev*>(basis));
  return cudaGetLastError();
}

cudaError_t launch_sh_rotators(uint32_t count, const float* rot, const void* basis, uint32_t degree,
                               float* table, cudaStream_t s) {
  if (count == 0 || degree == 0) return cudaSuccess;
  k_sh_rotators<<<(count + 127) / 128, 128, 0, s>>>(
      count, rot, reinterpret_cast<const ShBasisDev*>(basis), degree > 3 ? 3u : degree, table);
  return cudaGetLastError();
}

cudaError_t launch_sh_apply(uint64_t n, float* sh, const float* table, uint32_t num_rot,
                            const uint32_t* index, uint32_t degree, uint32_t* bad, cudaStream_t s) {
  if (n == 0 || degree == 0) return cudaSuccess;
  const uint64_t blocks = (n + 255) / 256;
  k_sh_apply<<<(unsigned)blocks, 256, 0, s>>>(n, sh, table, num_rot, index,
                                              degree > 3 ? 3u : degree, bad);
  return cudaGetLastError();
}

cudaError_t launch_export(const ExportArgs& a, cudaStream_t s) {
  if (a.count == 0) return cudaSuccess;
  ExportArgs b = a;
  if (b.degree > 3) b.degree = 3;
  k_export<<<(a.count + 255) / 256, 256, 0, s>>>(b);
  return cudaGetLastError();
}

}  // namespace cgs
