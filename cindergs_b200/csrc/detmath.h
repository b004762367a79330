// Deterministic single-precision elementary functions shared by the CUDA
// kernels and the host code that must reproduce their results bit for bit.
//
// Stage 1-3 of the splat pipeline feed transcendental results into integer
// decisions: the tile extents `ceil(sqrt(2 ln(255 a)) * sqrt(s))`, the
// ellipse-vs-tile cutoff `2 ln(255 a)` (render/kernels/binning.rs:79,
// render/kernels/project.rs:1193-1204), the polar pre-scale
// `exp(-ln|det J| / 3)` and the Cardano eigenvalue `q + 2p cos(acos(r)/3)`
// (render/kernels/deformation.rs:753-787, :810). The reference lowers these to
// whatever the WGSL driver provides, so its last bits are unpinned. Here every
// such call goes through the functions below, which use only IEEE-754 +, -, *,
// / and sqrt (each correctly rounded on both host and device) in a fixed
// order, so a host build and an sm_100a build produce identical bits.
//
// Methods (all textbook, none taken from a vendor library):
//   log:  x = m 2^e with m in [sqrt(1/2), sqrt(2)); ln m = 2 atanh(s),
//         s = (m-1)/(m+1), odd power series of atanh to s^11; e ln 2 is added
//         as a two-part constant (Cody & Waite range reduction).
//   exp:  x = k ln2 + r with |r| <= ln2/2 (two-part ln 2), Taylor series of
//         e^r to r^7, scaled by 2^k built from the exponent bits.
//   acos: asin Maclaurin series to a^23 on [0, 1/2]; for |x| > 1/2 the
//         half-angle identity acos x = 2 asin(sqrt((1-x)/2)).
//   cos:  Maclaurin series to x^12, accurate on [-pi/2, pi/2] (the callers
//         only pass acos(.)/3 in [0, pi/3]).
// Accuracy versus glibc is a few ulp; the unit tests pin that bound.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define CGS_HD __host__ __device__ __forceinline__
#else
#define CGS_HD static inline
#endif

// Arithmetic that must never be fused into an FMA by the compiler.
#if defined(__CUDA_ARCH__)
#define CGS_MUL(a, b) __fmul_rn((a), (b))
#define CGS_ADD(a, b) __fadd_rn((a), (b))
#define CGS_SUB(a, b) __fsub_rn((a), (b))
#define CGS_DIV(a, b) __fdiv_rn((a), (b))
#define CGS_SQRT(a) __fsqrt_rn((a))
#else
#include <math.h>
#define CGS_MUL(a, b) ((a) * (b))
#define CGS_ADD(a, b) ((a) + (b))
#define CGS_SUB(a, b) ((a) - (b))
#define CGS_DIV(a, b) ((a) / (b))
#define CGS_SQRT(a) sqrtf((a))
#endif

CGS_HD uint32_t cgs_f2u(float f) {
#if defined(__CUDA_ARCH__)
  return __float_as_uint(f);
#else
  union { float f; uint32_t u; } v;
  v.f = f;
  return v.u;
#endif
}

CGS_HD float cgs_u2f(uint32_t u) {
#if defined(__CUDA_ARCH__)
  return __uint_as_float(u);
#else
  union { float f; uint32_t u; } v;
  v.u = u;
  return v.f;
#endif
}

// Natural logarithm. ln(0) = -inf, ln(x<0) = NaN, ln(inf) = inf.
CGS_HD float cgs_logf(float x) {
  uint32_t bits = cgs_f2u(x);
  if (x != x || (bits >> 31)) return x == 0.0f ? cgs_u2f(0xff800000u) : cgs_u2f(0x7fc00000u);
  if (x == 0.0f) return cgs_u2f(0xff800000u);
  if ((bits & 0x7f800000u) == 0x7f800000u) return x;  // +inf
  int e = 0;
  if ((bits & 0x7f800000u) == 0) {  // subnormal: scale into the normal range
    x = CGS_MUL(x, 8388608.0f);     // 2^23, exact
    bits = cgs_f2u(x);
    e = -23;
  }
  e += (int)((bits >> 23) & 0xffu) - 127;
  float m = cgs_u2f((bits & 0x007fffffu) | 0x3f800000u);  // [1, 2)
  if (m > 1.41421356f) {
    m = CGS_MUL(m, 0.5f);
    e += 1;
  }
  const float s = CGS_DIV(CGS_SUB(m, 1.0f), CGS_ADD(m, 1.0f));
  const float z = CGS_MUL(s, s);
  float p = CGS_ADD(0.111111111f, CGS_MUL(z, 0.0909090909f));  // 1/9 + z/11
  p = CGS_ADD(0.142857143f, CGS_MUL(z, p));                     // 1/7
  p = CGS_ADD(0.2f, CGS_MUL(z, p));                             // 1/5
  p = CGS_ADD(0.333333333f, CGS_MUL(z, p));                     // 1/3
  p = CGS_ADD(1.0f, CGS_MUL(z, p));
  const float r = CGS_MUL(CGS_MUL(2.0f, s), p);
  const float fe = (float)e;
  const float ln2_hi = 0.693145751953125f;        // 0x3f317200, low 9 bits clear
  const float ln2_lo = 1.42860676533018e-06f;     // ln 2 - ln2_hi
  return CGS_ADD(CGS_ADD(CGS_MUL(fe, ln2_lo), r), CGS_MUL(fe, ln2_hi));
}

// e^x.
CGS_HD float cgs_expf(float x) {
  if (x != x) return x;
  if (x > 88.7228394f) return cgs_u2f(0x7f800000u);
  if (x < -103.972084f) return 0.0f;
  const float log2e = 1.44269504f;
  float kf = CGS_MUL(x, log2e);
  // round half away from zero to an integer, exactly representable here
  kf = (kf >= 0.0f) ? (float)(int)CGS_ADD(kf, 0.5f) : -(float)(int)CGS_ADD(-kf, 0.5f);
  const int k = (int)kf;
  const float ln2_hi = 0.693145751953125f;
  const float ln2_lo = 1.42860676533018e-06f;
  const float r = CGS_SUB(CGS_SUB(x, CGS_MUL(kf, ln2_hi)), CGS_MUL(kf, ln2_lo));
  float p = CGS_ADD(0.00138888889f, CGS_MUL(r, 0.000198412698f));  // 1/720 + r/5040
  p = CGS_ADD(0.00833333333f, CGS_MUL(r, p));                        // 1/120
  p = CGS_ADD(0.0416666667f, CGS_MUL(r, p));                         // 1/24
  p = CGS_ADD(0.166666667f, CGS_MUL(r, p));                          // 1/6
  p = CGS_ADD(0.5f, CGS_MUL(r, p));
  p = CGS_ADD(1.0f, CGS_MUL(r, p));
  p = CGS_ADD(1.0f, CGS_MUL(r, p));
  if (k > 127) {  // e^x close to FLT_MAX: scale in two steps
    p = CGS_MUL(p, 2.0f);
    return CGS_MUL(p, cgs_u2f((uint32_t)(k - 1 + 127) << 23));
  }
  if (k < -125) {  // subnormal result: scale in two steps
    p = CGS_MUL(p, cgs_u2f((uint32_t)(k + 64 + 127) << 23));
    return CGS_MUL(p, 5.42101086e-20f);  // 2^-64, exact
  }
  return CGS_MUL(p, cgs_u2f((uint32_t)(k + 127) << 23));
}

// asin on [0, 1/2] by its Maclaurin series (terms to a^23).
CGS_HD float cgs_asin_small(float a) {
  const float z = CGS_MUL(a, a);
  // c_n = C(2n, n) / (4^n (2n + 1)), n = 1..11, evaluated by Horner in z
  float p = CGS_ADD(0.00839033580f, CGS_MUL(z, 0.00731252587f));  // c10, c11
  p = CGS_ADD(0.00976160952f, CGS_MUL(z, p));  // c9
  p = CGS_ADD(0.0115518009f, CGS_MUL(z, p));   // c8
  p = CGS_ADD(0.0139648438f, CGS_MUL(z, p));   // c7
  p = CGS_ADD(0.0173527644f, CGS_MUL(z, p));   // c6
  p = CGS_ADD(0.0223721591f, CGS_MUL(z, p));   // c5
  p = CGS_ADD(0.0303819444f, CGS_MUL(z, p));   // c4
  p = CGS_ADD(0.0446428571f, CGS_MUL(z, p));   // c3
  p = CGS_ADD(0.075f, CGS_MUL(z, p));          // c2
  p = CGS_ADD(0.166666667f, CGS_MUL(z, p));    // c1
  return CGS_ADD(a, CGS_MUL(CGS_MUL(a, z), p));
}

// arccos on [-1, 1]; callers clamp their argument first.
CGS_HD float cgs_acosf(float x) {
  const float pi = 3.14159274f;
  const float pio2 = 1.57079637f;
  const float a = x < 0.0f ? -x : x;
  if (a <= 0.5f) {
    const float s = cgs_asin_small(a);
    return x < 0.0f ? CGS_ADD(pio2, s) : CGS_SUB(pio2, s);
  }
  const float t = CGS_MUL(CGS_SUB(1.0f, a), 0.5f);
  const float h = CGS_MUL(2.0f, cgs_asin_small(CGS_SQRT(t)));
  return x < 0.0f ? CGS_SUB(pi, h) : h;
}

// cos on [-pi/2, pi/2] by its Maclaurin series (terms to x^12).
CGS_HD float cgs_cosf(float x) {
  const float z = CGS_MUL(x, x);
  float p = CGS_ADD(-2.75573192e-07f, CGS_MUL(z, 2.08767570e-09f));  // -1/10! + z/12!
  p = CGS_ADD(2.48015873e-05f, CGS_MUL(z, p));   // 1/8!
  p = CGS_ADD(-0.00138888889f, CGS_MUL(z, p));   // -1/6!
  p = CGS_ADD(0.0416666667f, CGS_MUL(z, p));     // 1/4!
  p = CGS_ADD(-0.5f, CGS_MUL(z, p));
  return CGS_ADD(1.0f, CGS_MUL(z, p));
}

// b^e for b > 0, as exp(e ln b).
CGS_HD float cgs_powf(float b, float e) { return cgs_expf(CGS_MUL(e, cgs_logf(b))); }
