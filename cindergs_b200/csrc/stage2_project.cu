// Stage 2: EWA projection with the 3D/2D Mip filter, tight opacity-aware
// extents and inverse-ray spherical harmonics, on sm_100a
// (project_gaussians_v2_kernel, render/kernels/project.rs:1020-1289;
//  eval_sh_f32, project.rs:798-895).
//
// One thread per splat. Inputs are read coalesced with 128-bit loads: the
// position/opacity and covariance words (40 B), and for visible splats the
// 48 SH coefficients from a planar layout (plane j holds coefficients
// 4j..4j+3 of every Gaussian as one float4, so a warp's load of a plane is
// 512 contiguous bytes; f16 storage keeps 8 coefficients per 16-byte word).
// Output is one 48-byte SplatRec per splat (culled splats write only the
// extents word, 0). The survivor count is a warp-aggregated atomic.
//
// Compiled with -fmad=false and the deterministic log of detmath.h, so the
// extents and the values Stage 3 turns into integers are bit-identical to the
// host restatement.
#include <cuda_fp16.h>

#include "kernels.h"

namespace cgs {
namespace {

constexpr int kProjectThreads = 256;     // default block size
constexpr int kProjectMaxThreads = 512;  // largest block size a launch shape may ask for

struct ShCoeffs {
  float c[48];
};

__device__ __forceinline__ void load_sh(const ProjectArgs& a, uint32_t g, uint32_t deg,
                                        ShCoeffs& s) {
  const int planes = deg == 0 ? 1 : 12;
  if (!a.sh_f16) {
    const float4* p = reinterpret_cast<const float4*>(a.sh);
#pragma unroll
    for (int j = 0; j < 12; ++j) {
      if (j < planes) {
        const float4 v = __ldg(&p[(size_t)j * a.sh_stride + g]);
        s.c[4 * j] = v.x; s.c[4 * j + 1] = v.y; s.c[4 * j + 2] = v.z; s.c[4 * j + 3] = v.w;
      }
    }
  } else {
    const uint4* p = reinterpret_cast<const uint4*>(a.sh);
    const int hplanes = deg == 0 ? 1 : 6;
#pragma unroll
    for (int j = 0; j < 6; ++j) {
      if (j < hplanes) {
        const uint4 v = __ldg(&p[(size_t)j * a.sh_stride + g]);
        const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const __half2 h = *reinterpret_cast<const __half2*>(&w[q]);
          const float2 f = __half22float2(h);
          s.c[8 * j + 2 * q] = f.x;
          s.c[8 * j + 2 * q + 1] = f.y;
        }
      }
    }
  }
}

// eval_sh_f32 (project.rs:798-895), same operand order.
__device__ __forceinline__ float3 eval_sh(const float* c, float dx, float dy, float dz,
                                          uint32_t deg) {
  float r = 0.28209479177387814f * c[0];
  float g = 0.28209479177387814f * c[1];
  float b = 0.28209479177387814f * c[2];
  if (deg >= 1) {
    const float y1_m1 = -0.4886025119029199f * dy;
    const float y1_0 = 0.4886025119029199f * dz;
    const float y1_p1 = -0.4886025119029199f * dx;
    r += y1_m1 * c[3] + y1_0 * c[4] + y1_p1 * c[5];
    g += y1_m1 * c[18] + y1_0 * c[19] + y1_p1 * c[20];
    b += y1_m1 * c[33] + y1_0 * c[34] + y1_p1 * c[35];
    if (deg >= 2) {
      const float xx = dx * dx, yy = dy * dy, zz = dz * dz;
      const float xy = dx * dy, yz = dy * dz, xz = dx * dz;
      const float y2_m2 = 1.0925484305920792f * xy;
      const float y2_m1 = -1.0925484305920792f * yz;
      const float y2_0 = 0.31539156525252005f * (2.0f * zz - xx - yy);
      const float y2_p1 = -1.0925484305920792f * xz;
      const float y2_p2 = 0.5462742152960396f * (xx - yy);
      r += y2_m2 * c[6] + y2_m1 * c[7] + y2_0 * c[8] + y2_p1 * c[9] + y2_p2 * c[10];
      g += y2_m2 * c[21] + y2_m1 * c[22] + y2_0 * c[23] + y2_p1 * c[24] + y2_p2 * c[25];
      b += y2_m2 * c[36] + y2_m1 * c[37] + y2_0 * c[38] + y2_p1 * c[39] + y2_p2 * c[40];
      if (deg >= 3) {
        const float y3_m3 = -0.5900435899266435f * dy * (3.0f * xx - yy);
        const float y3_m2 = 2.890611442640554f * xy * dz;
        const float y3_m1 = -0.4570457994644658f * dy * (4.0f * zz - xx - yy);
        const float y3_0 = 0.3731763325901154f * dz * (2.0f * zz - 3.0f * xx - 3.0f * yy);
        const float y3_p1 = -0.4570457994644658f * dx * (4.0f * zz - xx - yy);
        const float y3_p2 = 1.445305721320277f * dz * (xx - yy);
        const float y3_p3 = -0.5900435899266435f * dx * (xx - 3.0f * yy);
        r += y3_m3 * c[11] + y3_m2 * c[12] + y3_m1 * c[13] + y3_0 * c[14] + y3_p1 * c[15] +
             y3_p2 * c[16] + y3_p3 * c[17];
        g += y3_m3 * c[26] + y3_m2 * c[27] + y3_m1 * c[28] + y3_0 * c[29] + y3_p1 * c[30] +
             y3_p2 * c[31] + y3_p3 * c[32];
        b += y3_m3 * c[41] + y3_m2 * c[42] + y3_m1 * c[43] + y3_0 * c[44] + y3_p1 * c[45] +
             y3_p2 * c[46] + y3_p3 * c[47];
      }
    }
  }
  return make_float3(clampf(r + 0.5f, 0.0f, 1.0f), clampf(g + 0.5f, 0.0f, 1.0f),
                     clampf(b + 0.5f, 0.0f, 1.0f));
}

// At most 64 registers a thread (two 512-thread or four 256-thread blocks per
// SM): the kernel waits on its dependent loads (position, then the survivor's
// covariance and SH), and the fourth 256-thread block hides more of that
// latency than the two registers it costs (8 bytes spilled): 0.068 -> 0.064 ms
// at 1.1M Gaussians.
__global__ void __launch_bounds__(kProjectMaxThreads, 2) k_project(const ProjectArgs a) {
  const uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t active = a.n_rest + (a.split_count ? *a.split_count : 0u);
  bool visible = false;
  if (idx < active && idx < a.max_n) {
    const float w00 = a.cam[0], w10 = a.cam[1], w20 = a.cam[2];
    const float w01 = a.cam[4], w11 = a.cam[5], w21 = a.cam[6];
    const float w02 = a.cam[8], w12 = a.cam[9], w22 = a.cam[10];
    const float w03 = a.cam[12], w13 = a.cam[13], w23 = a.cam[14];
    const float fx = a.cam[16], fy = a.cam[17], cx = a.cam[18], cy = a.cam[19];
    const float vw = a.cam[20], vh = a.cam[21], near_p = a.cam[22];
    const float4 p4 = a.pos[idx];
    const float px = p4.x, py = p4.y, pz = p4.z;
    const float tx = w00 * px + w01 * py + w02 * pz + w03;
    const float ty = w10 * px + w11 * py + w12 * pz + w13;
    const float tz = w20 * px + w21 * py + w22 * pz + w23;
    uint32_t ext_packed = 0;
    float mu_x = 0, mu_y = 0, ca = 0, cb = 0, cc = 0, alpha_2d = 0;
    const float op = p4.w;
    if (tz > near_p && !(op < a.min_opacity)) {
      const float4 ca4 = a.cova[idx];
      const float2 cb2 = a.covb[idx];
      float v_xx = ca4.x, v_xy = ca4.y, v_xz = ca4.z, v_yy = ca4.w, v_yz = cb2.x, v_zz = cb2.y;
      float alpha_3d = op;
      bool alive = true;
      if (a.mip > 0.0f) {
        const float det_orig = fmaxf(v_xx * (v_yy * v_zz - v_yz * v_yz) -
                                         v_xy * (v_xy * v_zz - v_xz * v_yz) +
                                         v_xz * (v_xy * v_yz - v_xz * v_yy),
                                     1e-24f);
        v_xx += a.mip;
        v_yy += a.mip;
        v_zz += a.mip;
        const float det_reg = fmaxf(v_xx * (v_yy * v_zz - v_yz * v_yz) -
                                        v_xy * (v_xy * v_zz - v_xz * v_yz) +
                                        v_xz * (v_xy * v_yz - v_xz * v_yy),
                                    det_orig);
        const float comp = sqrtf(clampf(det_orig / det_reg, 0.0f, 1.0f));
        alpha_3d = clampf(op * comp, 0.0f, 1.0f);
        if (alpha_3d < a.min_opacity) alive = false;
      }
      if (alive) {
        const float k00 = w00 * v_xx + w01 * v_xy + w02 * v_xz;
        const float k01 = w00 * v_xy + w01 * v_yy + w02 * v_yz;
        const float k02 = w00 * v_xz + w01 * v_yz + w02 * v_zz;
        const float k10 = w10 * v_xx + w11 * v_xy + w12 * v_xz;
        const float k11 = w10 * v_xy + w11 * v_yy + w12 * v_yz;
        const float k12 = w10 * v_xz + w11 * v_yz + w12 * v_zz;
        const float k20 = w20 * v_xx + w21 * v_xy + w22 * v_xz;
        const float k21 = w20 * v_xy + w21 * v_yy + w22 * v_yz;
        const float k22 = w20 * v_xz + w21 * v_yz + w22 * v_zz;
        const float cam_xx = k00 * w00 + k01 * w01 + k02 * w02;
        const float cam_xy = k00 * w10 + k01 * w11 + k02 * w12;
        const float cam_xz = k00 * w20 + k01 * w21 + k02 * w22;
        const float cam_yy = k10 * w10 + k11 * w11 + k12 * w12;
        const float cam_yz = k10 * w20 + k11 * w21 + k12 * w22;
        const float cam_zz = k20 * w20 + k21 * w21 + k22 * w22;
        const float inv_tz = 1.0f / tz;
        const float inv_tz2 = inv_tz * inv_tz;
        const float j00 = fx * inv_tz;
        const float j02 = -fx * tx * inv_tz2;
        const float j11 = fy * inv_tz;
        const float j12 = -fy * ty * inv_tz2;
        const float m00 = j00 * cam_xx + j02 * cam_xz;
        const float m01 = j00 * cam_xy + j02 * cam_yz;
        const float m02 = j00 * cam_xz + j02 * cam_zz;
        const float m11 = j11 * cam_yy + j12 * cam_yz;
        const float m12 = j11 * cam_yz + j12 * cam_zz;
        const float s_xx = m00 * j00 + m02 * j02;
        const float s_xy = m01 * j11 + m02 * j12;
        const float s_yy = m11 * j11 + m12 * j12;
        const float raw_mid = 0.5f * (s_xx + s_yy);
        const float raw_det = fmaxf(s_xx * s_yy - s_xy * s_xy, 0.0f);
        const float raw_discr = sqrtf(fmaxf(raw_mid * raw_mid - raw_det, 0.0f));
        const float raw_lmax = fmaxf(raw_mid + raw_discr, 0.0f);
        if (!(3.0f * sqrtf(raw_lmax) < a.min_radius)) {
          const float sp_xx = s_xx + 0.3f, sp_xy = s_xy, sp_yy = s_yy + 0.3f;
          const float det = sp_xx * sp_yy - sp_xy * sp_xy;
          if (det > 1e-6f) {
            const float comp_2d = sqrtf(clampf(raw_det / det, 0.0f, 1.0f));
            alpha_2d = clampf(alpha_3d * comp_2d, 0.0f, 1.0f);
            if (!(alpha_2d < a.min_opacity || alpha_2d <= (1.0f / 255.0f))) {
              const float q_max = clampf(2.0f * cgs_logf(255.0f * alpha_2d), 0.0f, 8.0f);
              const float sigma_cut = sqrtf(q_max);
              const float ext_x = clampf(ceilf(sigma_cut * sqrtf(fmaxf(sp_xx, 0.0f))), 1.0f, 1024.0f);
              const float ext_y = clampf(ceilf(sigma_cut * sqrtf(fmaxf(sp_yy, 0.0f))), 1.0f, 1024.0f);
              mu_x = fx * tx * inv_tz + cx;
              mu_y = fy * ty * inv_tz + cy;
              if (!(mu_x + ext_x < 0.0f || mu_x - ext_x >= vw || mu_y + ext_y < 0.0f ||
                    mu_y - ext_y >= vh)) {
                const float inv_det = 1.0f / det;
                ca = sp_yy * inv_det;
                cb = -sp_xy * inv_det;
                cc = sp_xx * inv_det;
                ext_packed = ((uint32_t)ext_x & 0xFFFFu) | (((uint32_t)ext_y & 0xFFFFu) << 16);
                visible = true;
              }
            }
          }
        }
      }
    }
    SplatRec* rec = a.out + idx;
    if (visible) {
      const float vx = px - a.cam_pos[0], vy = py - a.cam_pos[1], vz = pz - a.cam_pos[2];
      const float inv_len = 1.0f / fmaxf(0.0001f, sqrtf(vx * vx + vy * vy + vz * vz));
      float dx = vx * inv_len, dy = vy * inv_len, dz = vz * inv_len;
      uint32_t sh_idx = idx;
      uint32_t tet_raw = a.num_tets;
      if (idx < a.n_rest) {
        if (a.bind_tet) tet_raw = a.bind_tet[idx];
      } else {
        const uint2 m = a.split_meta[idx - a.n_rest];
        sh_idx = m.x;
        tet_raw = m.y;
      }
      const float* R = nullptr;
      if (a.tet_R && tet_raw < a.num_tets)
        R = a.tet_R + 9 * (size_t)tet_raw;
      else if (a.mvc_R && tet_raw == kMvcBound)
        R = a.mvc_R + 9 * (size_t)__float_as_uint(a.bind_w[sh_idx].x);
      if (R) {
        const float ldx = __ldg(R + 0) * dx + __ldg(R + 1) * dy + __ldg(R + 2) * dz;
        const float ldy = __ldg(R + 3) * dx + __ldg(R + 4) * dy + __ldg(R + 5) * dz;
        const float ldz = __ldg(R + 6) * dx + __ldg(R + 7) * dy + __ldg(R + 8) * dz;
        dx = ldx;
        dy = ldy;
        dz = ldz;
      }
      const uint32_t deg = a.sh_degree > 3 ? 3u : a.sh_degree;
      ShCoeffs sh;
      load_sh(a, sh_idx, deg, sh);
      const float3 rgb = eval_sh(sh.c, dx, dy, dz, deg);
      rec->geo = make_float4(mu_x, mu_y, ca, cb);
      rec->cc = make_float4(cc, alpha_2d, tz, __uint_as_float(ext_packed));
      rec->rgb = make_float4(rgb.x, rgb.y, rgb.z, 0.0f);
    } else {
      rec->cc = make_float4(0.0f, 0.0f, tz, 0.0f);
    }
    if (a.depth_keys) {
      // The depth part of the splat's tile keys (emit_tile_keys_kernel,
      // binning.rs:170-328): Stage 3 sorts the splats by it once, then emits
      // their entries in that order and sorts the entries by tile alone.
      uint32_t dk = 0xFFFFFFFFu;
      if (visible) {
        if (a.key64) {
          dk = __float_as_uint(fmaxf(tz, 0.0f));
        } else {
          const uint32_t raw = __float_as_uint(fmaxf(tz, 1e-6f));
          const uint32_t rel =
              raw > a.depth_base_bits ? min(raw - a.depth_base_bits, 0x0FFFFFFFu) : 0u;
          dk = rel >> (28u - a.depth_bits);
        }
      }
      a.depth_keys[idx] = dk;
      a.depth_ids[idx] = idx;
    }
  }
  if (idx == 0) a.fc->active = active < a.max_n ? active : a.max_n;
  const uint32_t vote = __ballot_sync(0xffffffffu, visible);
  if ((threadIdx.x & 31) == 0 && vote) atomicAdd(&a.fc->surviving, (uint32_t)__popc(vote));
}

// Rest-scene layout: interleaved SoA (pos N*3, cov N*6, opa N, sh N*48) to
// float4 (xyz, opacity), float4 (xx, xy, xz, yy), float2 (yz, zz) and SH planes.
__global__ void k_scene_layout(uint32_t n, const float* __restrict__ pos,
                               const float* __restrict__ cov, const float* __restrict__ opa,
                               const void* __restrict__ sh, int sh_f16, float4* __restrict__ out_pos,
                               float4* __restrict__ out_cova, float2* __restrict__ out_covb,
                               void* __restrict__ out_sh) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  out_pos[i] = make_float4(pos[3 * (size_t)i], pos[3 * (size_t)i + 1], pos[3 * (size_t)i + 2], opa[i]);
  const float* c = cov + 6 * (size_t)i;
  out_cova[i] = make_float4(c[0], c[1], c[2], c[3]);
  out_covb[i] = make_float2(c[4], c[5]);
  if (!sh_f16) {
    const float4* src = reinterpret_cast<const float4*>(sh) + 12 * (size_t)i;
    float4* dst = reinterpret_cast<float4*>(out_sh);
#pragma unroll
    for (int j = 0; j < 12; ++j) dst[(size_t)j * n + i] = src[j];
  } else {
    const uint4* src = reinterpret_cast<const uint4*>(sh) + 6 * (size_t)i;
    uint4* dst = reinterpret_cast<uint4*>(out_sh);
#pragma unroll
    for (int j = 0; j < 6; ++j) dst[(size_t)j * n + i] = src[j];
  }
}

// QuantizedGaussianSceneSoa (scene/soa.rs:429-608) into the resident layout:
// covariances from three words of f16 pairs ((xx, xy), (xz, yy), (yz, zz),
// first value in the low half), SH from the degree-trimmed words (DC rgb,
// then each channel's higher-order coefficients, two f16 per word) into the
// 48-coefficient channel-major f16 planes with zeros above the degree. f16
// to f32 is exact, so this equals uploading the dequantized scene.
__global__ void k_scene_decode_quantized(uint32_t n, const float* __restrict__ pos,
                                         const uint32_t* __restrict__ cov_words,
                                         const float* __restrict__ opa,
                                         const uint32_t* __restrict__ sh_words, uint32_t sh_degree,
                                         float4* __restrict__ out_pos, float4* __restrict__ out_cova,
                                         float2* __restrict__ out_covb, uint4* __restrict__ out_sh) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  out_pos[i] = make_float4(pos[3 * (size_t)i], pos[3 * (size_t)i + 1], pos[3 * (size_t)i + 2], opa[i]);
  const uint32_t* cw = cov_words + 3 * (size_t)i;
  auto lo = [](uint32_t w) { return __half2float(__ushort_as_half((unsigned short)(w & 0xFFFFu))); };
  auto hi = [](uint32_t w) { return __half2float(__ushort_as_half((unsigned short)(w >> 16))); };
  const uint32_t w0 = cw[0], w1 = cw[1], w2 = cw[2];
  out_cova[i] = make_float4(lo(w0), hi(w0), lo(w1), hi(w1));
  out_covb[i] = make_float2(lo(w2), hi(w2));
  const uint32_t deg = sh_degree > 3 ? 3 : sh_degree;
  const uint32_t bases = deg == 0 ? 1 : (deg == 1 ? 4 : (deg == 2 ? 9 : 16));
  const uint32_t rest = bases - 1, words = (bases * 3 + 1) / 2;
  const uint32_t* sw = sh_words + (size_t)words * i;
  uint32_t half_bits[48];
#pragma unroll
  for (int k = 0; k < 48; ++k) {
    int l;
    if (k < 3) l = k;
    else if (k < 18) l = (uint32_t)(k - 3) < rest ? 3 + (k - 3) : -1;
    else if (k < 33) l = (uint32_t)(k - 18) < rest ? 3 + (int)rest + (k - 18) : -1;
    else l = (uint32_t)(k - 33) < rest ? 3 + 2 * (int)rest + (k - 33) : -1;
    half_bits[k] = l < 0 ? 0u : (sw[l >> 1] >> (16 * (l & 1))) & 0xFFFFu;
  }
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    const uint32_t* h = half_bits + 8 * j;
    out_sh[(size_t)j * n + i] = make_uint4(h[0] | (h[1] << 16), h[2] | (h[3] << 16),
                                           h[4] | (h[5] << 16), h[6] | (h[7] << 16));
  }
}

}  // namespace

cudaError_t launch_scene_decode_quantized(uint32_t n, const float* pos, const uint32_t* cov_words,
                                          const float* opa, const uint32_t* sh_words,
                                          uint32_t sh_degree, float4* out_pos, float4* out_cova,
                                          float2* out_covb, void* out_sh, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  k_scene_decode_quantized<<<(n + 255) / 256, 256, 0, s>>>(
      n, pos, cov_words, opa, sh_words, sh_degree, out_pos, out_cova, out_covb,
      reinterpret_cast<uint4*>(out_sh));
  return cudaGetLastError();
}

cudaError_t launch_project(const ProjectArgs& a, cudaStream_t s) {
  if (a.max_n == 0) return cudaSuccess;
  const uint32_t t = a.threads ? a.threads : kProjectThreads;
  if (t != 128 && t != 256 && t != 512) return cudaErrorInvalidValue;
  k_project<<<(a.max_n + t - 1) / t, t, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_scene_layout(uint32_t n, const float* pos, const float* cov, const float* opa,
                                const void* sh, int sh_f16, float4* out_pos, float4* out_cova,
                                float2* out_covb, void* out_sh, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  k_scene_layout<<<(n + 255) / 256, 256, 0, s>>>(n, pos, cov, opa, sh, sh_f16, out_pos, out_cova,
                                                 out_covb, out_sh);
  return cudaGetLastError();
}

}  // namespace cgs
