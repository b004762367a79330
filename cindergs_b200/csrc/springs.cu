// Cage spring dynamics on the device (CageSpringSimulator,
// deformation/dynamics.rs:75-313): semi-implicit Euler springs toward the
// rest pose with frame-rate independent exponential damping, pinned
// vertices and collision half-spaces, stepping the resident tet-cage
// vertices in place so that a sequence of frames needs no host vertex upload.
//
//  k_springs_step     one thread per cage vertex, `steps` steps of
//                     CageSpringSimulator::step (dynamics.rs:249-277) with
//                     CollisionPlane::resolve_contact (:57-71) after each.
//                     Vertices are independent, so several steps in one
//                     launch equal several calls.
//  k_springs_impulse  trigger_jiggle_impulse (dynamics.rs:280-305): an
//                     outward radial velocity pulse from each cage's rest
//                     centroid (summed on the host in vertex order).
//
// Per-cage scalars (stiffness / mass, the damping factor exp(-c dt), the
// clamped dt) are computed on the host with the C library's logf / expf, as
// the reference does. Compiled with -fmad=false: each product and sum is
// rounded separately, in the reference's order.
#include "kernels.h"

namespace cgs {
namespace {

// CollisionPlane::resolve_contact: plane = (nx, ny, nz, offset),
// (restitution, friction, -, -).
__device__ __forceinline__ void contact(const float4 pa, const float4 pb, float& x, float& y,
                                        float& z, float& vx, float& vy, float& vz) {
  const float d = ((pa.x * x + pa.y * y) + pa.z * z) - pa.w;
  if (d >= 0.0f) return;
  x = x - pa.x * d;
  y = y - pa.y * d;
  z = z - pa.z * d;
  const float vn = (vx * pa.x + vy * pa.y) + vz * pa.z;
  if (vn < 0.0f) {
    const float nx = pa.x * vn, ny = pa.y * vn, nz = pa.z * vn;
    const float keep = 1.0f - pb.y;
    vx = (vx - nx) * keep - nx * pb.x;
    vy = (vy - ny) * keep - ny * pb.x;
    vz = (vz - nz) * keep - nz * pb.x;
  }
}

__global__ void __launch_bounds__(128) k_springs_step(SpringArgs a) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.V) return;
  const float4 r = a.rest[i];
  const uint32_t c = __float_as_uint(r.w);
  if (c >= a.num_cages) return;  // vertex of no spring cage
  const SpringCageDev p = a.cages[c];
  if (!(p.dt > 0.0f)) return;
  if (a.pinned[i]) {
    a.vel[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    return;
  }
  float* xp = a.verts + 3 * (size_t)i;
  float x = xp[0], y = xp[1], z = xp[2];
  float4 v = a.vel[i];
  const uint32_t first = p.planes & 0xFFFFu, np = p.planes >> 16;
  for (uint32_t s = 0; s < a.steps; ++s) {
    const float ax = (r.x - x) * p.kim, ay = (r.y - y) * p.kim, az = (r.z - z) * p.kim;
    v.x = (v.x + ax * p.dt) * p.gamma;
    v.y = (v.y + ay * p.dt) * p.gamma;
    v.z = (v.z + az * p.dt) * p.gamma;
    x = x + v.x * p.dt;
    y = y + v.y * p.dt;
    z = z + v.z * p.dt;
    for (uint32_t q = 0; q < np; ++q)
      contact(a.planes[2 * (first + q)], a.planes[2 * (first + q) + 1], x, y, z, v.x, v.y, v.z);
  }
  xp[0] = x;
  xp[1] = y;
  xp[2] = z;
  a.vel[i] = v;
}

__global__ void __launch_bounds__(128) k_springs_impulse(SpringArgs a, float magnitude) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.V) return;
  const float4 r = a.rest[i];
  const uint32_t c = __float_as_uint(r.w);
  if (c >= a.num_cages || a.pinned[i]) return;
  const SpringCageDev p = a.cages[c];
  const float dx = r.x - p.cx, dy = r.y - p.cy, dz = r.z - p.cz;
  // Vec3::normalize_or_zero
  const float rcp = 1.0f / sqrtf((dx * dx + dy * dy) + dz * dz);
  float ux = 0.0f, uy = 0.0f, uz = 0.0f;
  if (isfinite(rcp) && rcp > 0.0f) {
    ux = dx * rcp;
    uy = dy * rcp;
    uz = dz * rcp;
  }
  float ix, iy, iz;
  if ((ux * ux + uy * uy) + uz * uz > 1e-4f) {
    ix = ux * magnitude;
    iy = uy * magnitude;
    iz = uz * magnitude;
  } else {
    ix = 0.0f * magnitude;
    iy = 1.0f * magnitude;
    iz = 0.0f * magnitude;
  }
  float4 v = a.vel[i];
  v.x = v.x + ix;
  v.y = v.y + iy;
  v.z = v.z + iz;
  a.vel[i] = v;
}

}  // namespace

cudaError_t launch_springs_step(const SpringArgs& a, cudaStream_t s) {
  if (a.V == 0 || a.steps == 0) return cudaSuccess;
  k_springs_step<<<(a.V + 127) / 128, 128, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_springs_impulse(const SpringArgs& a, float magnitude, cudaStream_t s) {
  if (a.V == 0) return cudaSuccess;
  k_springs_impulse<<<(a.V + 127) / 128, 128, 0, s>>>(a, magnitude);
  return cudaGetLastError();
}

}  // namespace cgs
