// Reference-faithful FP32 arithmetic of the plain form.
//
// The plain FP32 form must reproduce the reference's images to 1e-5 relative
// RMS.  Its forward bilinear splat makes every image pixel depend on the
// target position of its source pixels at O(1) per pixel of shift, and the
// reference evaluates those positions through an FP32 chain of degree-based
// trigonometry built with --use_fast_math (FIPkernels.cu:73-171, 289-376,
// reference Makefile:13).  An independent formula (even an exact one) moves
// targets by 1e-3..1e-1 pixel and the images by ~3e-3 relative RMS.  So the
// functions below evaluate the same steps, in the same order and types
// (including the double-precision promotions that the reference's double
// M_PI literal causes), and this header is only included by translation units
// compiled with --use_fast_math, like the reference.  The precision form uses
// the exact closed form instead (fip_precise.cu).
#pragma once

#include "fip_common.cuh"

// Quadrature of the ES kernel's Fourier transform used for the grid-correction
// taper (FIPkernels.cu:14-29).  Same values as the reference: the taper (and
// so every image pixel) depends on them bit for bit.
__constant__ float fip_quad_nodes[14] = {
    0.9964425f, 0.98130317f, 0.95425928f, 0.91563303f, 0.86589252f,
    0.80564137f, 0.73561088f, 0.65665109f, 0.56972047f, 0.47587422f,
    0.37625152f, 0.27206163f, 0.16456928f, 0.05507929f};
__constant__ float fip_quad_weights[14] = {
    0.00912428f, 0.02113211f, 0.03290143f, 0.04427293f, 0.05510735f,
    0.06527292f, 0.07464621f, 0.08311342f, 0.09057174f, 0.09693066f,
    0.10211297f, 0.10605577f, 0.10871119f, 0.11004701f};
__constant__ float fip_quad_kernel[14] = {
    7.71381676e-07f, 4.06901586e-06f, 2.09164257e-05f, 1.01923695e-04f,
    4.61199576e-04f, 1.90183990e-03f, 7.02391280e-03f, 2.28652529e-02f,
    6.46725327e-02f, 1.56933676e-01f, 3.23208771e-01f, 5.60024174e-01f,
    8.10934691e-01f, 9.76937533e-01f};

namespace fipref {

// Correctly rounded double quotient x / d for the constant divisors of the
// chain (180 and pi), by one Markstein correction of the product with the
// rounded reciprocal: q0 = x * (1/d), e = x - q0 * d (exact with an FMA),
// q = q0 + e * (1/d) (P. Markstein, "Computation of elementary functions on
// the IBM RISC System/6000 processor", IBM J. Res. Dev. 34(1), 1990).  This
// equals the IEEE division the reference performs (verified against the
// reference's own targets), at three FP64 operations instead of a division.
__device__ __forceinline__ double div_const(double x, double d, double rinv) {
  const double q0 = x * rinv;
  const double e = fma(-q0, d, x);
  return fma(e, rinv, q0);
}
#define FIP_INV_180 (1.0 / 180.0)
#define FIP_INV_PI (1.0 / FIP_M_PI)
// (double)a * M_PI / 180.0, as the reference evaluates the degree-to-radian
// conversion inside sinf/cosf arguments (FIPkernels.cu:96-97, 116, 135).
__device__ __forceinline__ float deg_to_rad_arg(float a) {
  return (float)div_const((double)a * FIP_M_PI, 180.0, FIP_INV_180);
}
// (double)(v * 180.0f) / M_PI, the radian-to-degree step of the reference's
// atan2/acos/asin helpers (FIPkernels.cu:145, 157, 169).
__device__ __forceinline__ float rad_to_deg_ret(float v180) {
  return (float)div_const((double)v180, FIP_M_PI, FIP_INV_PI);
}

// fmodf(a, 90.0f) == 0, i.e. a is an exact multiple of 90.  fmod is exact,
// so for |a| < 90 it equals a, and for 90 <= |a| < 180 it equals |a| - 90
// (Sterbenz); only larger angles need the library call.
__device__ __forceinline__ bool multiple_of_90(float a) {
  const float m = fabsf(a);
  if (m < 90.0f) return a == 0.0f;
  if (m < 180.0f) return m == 90.0f;
  return fmodf(a, 90.0f) == 0;
}

// computeCeil/computeFloor semantics (FIPkernels.cu:47-61): equal to
// ceilf/floorf, returned as a signed integer.
__device__ __forceinline__ long ceil_l(float v) { return v < 0 ? -(long)floorf(-v) : (long)ceilf(v); }
__device__ __forceinline__ long floor_l(float v) { return v < 0 ? -(long)ceilf(-v) : (long)floorf(v); }

// ES gridding kernel exp(beta (sqrt(1 - x^2) - 1)), 0 outside |x| <= 1
// (FIPkernels.cu:67-71).
__device__ __forceinline__ float es(float x) {
  const float beta = FIP_ES_BETA;
  const float xx = x * x;
  return (xx > float(1.0)) ? float(0.0) : exp(beta * (sqrt(float(1.0) - xx) - float(1.0)));
}

// Grid-correction taper value at distance t (FIPkernels.cu:173-186).
__device__ __forceinline__ float taper(size_t t, size_t g) {
  const int support = FIP_SUPPORT;
  const float norm = FIP_CONV_NORM;
  float tn = static_cast<float>(t) / g;
  float corr = 0.0;
  float angle;
  for (int i = 0; i < 14; ++i) {
    angle = FIP_M_PI * tn * support * fip_quad_nodes[i];
    corr += fip_quad_kernel[i] * fip_quad_weights[i] * cosf(angle);
  }
  return corr * support / norm;
}

// Degree-based trigonometry with exact values at multiples of 90 degrees
// (FIPkernels.cu:73-171).
__device__ __forceinline__ void sincos_deg(float a, float& s, float& c) {
  if (multiple_of_90(a)) {
    int i = static_cast<int>(fabsf((float)floor_l(a / 90.0f + 0.5f))) % 4;
    switch (i) {
      case 0: s = 0.0f; c = 1.0f; break;
      case 1: s = (a > 0.0f) ? 1.0f : -1.0f; c = 0.0f; break;
      case 2: s = 0.0f; c = -1.0f; break;
      default: s = (a > 0.0f) ? -1.0f : 1.0f; c = 0.0f; break;
    }
  } else {
    const float arg = deg_to_rad_arg(a);
    s = sinf(arg);
    c = cosf(arg);
  }
}

__device__ __forceinline__ float sin_deg(float a) {
  if (multiple_of_90(a)) {
    int i = static_cast<int>(fabsf((float)floor_l(a / 90.0f - 0.5f))) % 4;
    return i == 0 ? 1.0f : (i == 2 ? -1.0f : 0.0f);
  }
  return sinf(deg_to_rad_arg(a));
}

__device__ __forceinline__ float cos_deg(float a) {
  if (multiple_of_90(a)) {
    int i = static_cast<int>(fabsf((float)floor_l(a / 90.0f + 0.5f))) % 4;
    return i == 0 ? 1.0f : (i == 2 ? -1.0f : 0.0f);
  }
  return cosf(deg_to_rad_arg(a));
}

__device__ __forceinline__ float atan2_deg(float y, float x) {
  if (y == 0.0f) return (x >= 0.0f) ? 0.0f : 180.0f;
  if (x == 0.0f) return (y > 0.0f) ? 90.0f : -90.0f;
  return rad_to_deg_ret(atan2f(y, x) * 180.0f);
}

__device__ __forceinline__ float acos_deg(float v) {
  if (v >= 1.0f && v - 1.0f < 1e-10) return 0.0f;
  if (v == 0.0f) return 90.0f;
  if (v <= -1.0f && v + 1.0f > -1e-10) return 180.0f;
  return rad_to_deg_ret(acosf(v) * 180.0f);
}

__device__ __forceinline__ float asin_deg(float v) {
  if (v <= -1.0f && v + 1.0f > -1e-10) return -90.0f;
  if (v == 0.0f) return 0.0f;
  if (v >= 1.0f && v - 1.0f < 1e-10) return 90.0f;
  return rad_to_deg_ret(asinf(v) * 180.0f);
}

// Per-snapshot constants of the pixel mapping.
struct Frame {
  float v0, v1, v3, v4, v8;  // V[0][0], V[0][1], V[1][0], V[1][1], V[2][2]
  float v6, v7;              // V[2][0], V[2][1]
  float dc;                  // cell in degrees: (float)((double)cell / pi * 180)
};

// The slant-step terms of the chain that depend on theta alone
// (FIPkernels.cu:344-359, 366): r = r0 cos(theta) and z r0 with
// z = 1 - sin(theta) (small-angle forms below 1e-5 rad), in the chain's
// FP32 steps.
__device__ __forceinline__ void theta_terms(float theta, float& r, float& zr0) {
  float t = (90.0f - fabsf(theta)) / 180.0f * FIP_M_PI;
  float z, costhe;
  if (t < 1.0e-5f) {
    if (theta > 0.0f) {
      z = t * t / 2.0f;
    } else {
      z = 2.0f - t * t / 2.0f;
    }
    costhe = t;
  } else {
    z = 1.0f - sin_deg(theta);
    costhe = cos_deg(theta);
  }
  const float r0 = 180.0f / FIP_M_PI;
  r = r0 * costhe;
  zr0 = z * r0;
}

// theta_terms tabulated over theta in [80, 90] degrees, indexed by the bit
// pattern of theta (every FP32 value in the range, 1,310,721 entries): the
// values are the chain's own FP32 results, so a lookup returns the same bits
// as the evaluation (two trigonometric calls, two FP64 conversions) at a
// fraction of the instructions.  Fields within 10 degrees of the phase
// centre (r < cos 80 deg) map every pixel through the table; the rest
// evaluate.
constexpr unsigned kThetaTabLo = 0x42A00000u;  // 80.0f
constexpr unsigned kThetaTabHi = 0x42B40000u;  // 90.0f
constexpr int kThetaTabSize = (int)(kThetaTabHi - kThetaTabLo) + 1;

// Target (LL, MM) of source pixel (column i, row j), relative to the image
// centre: the plane-pixel coordinates of FIPkernels.cu:296-297 followed by
// the SIN -> slant-SIN step of FIPkernels.cu:307-374 and the centring of
// :385-386.  di = N.
// ttab: the theta_terms table, or null to evaluate them.
__device__ __forceinline__ void pixel_target(const Frame& f, int i, int j, int di,
                                             float& LL, float& MM,
                                             const float2* __restrict__ ttab = nullptr) {
  // Integer-to-float conversions are exact below 2^24, whatever the integer
  // type, so 32-bit indices give the reference's values.
  const int half = di / 2;
  float p1 = (-f.v0 * (static_cast<float>(i) - static_cast<float>(half)) +
              f.v3 * (static_cast<float>(j) - static_cast<float>(half))) /
                 fabsf(f.v8) +
             static_cast<float>(half);
  float p2 = (-f.v1 * (static_cast<float>(i) - static_cast<float>(half)) +
              f.v4 * (static_cast<float>(j) - static_cast<float>(half))) /
                 fabsf(f.v8) +
             static_cast<float>(half);

  float xi = f.v6 / f.v8;
  float eta = f.v7 / f.v8;
  float dc = f.dc;
  float x = -dc * (p1 - (static_cast<float>(di) / 2.0f + 1.0f));
  float y = dc * (p2 - (static_cast<float>(di) / 2.0f + 1.0f));
  float r0 = 180.0f / FIP_M_PI;
  float x0 = x / r0;
  float y0 = y / r0;
  float r2 = x0 * x0 + y0 * y0;
  float phi;
  if (r2 != 0.0f) {
    phi = atan2_deg(x0, -y0);
  } else {
    phi = 0.0f;
  }
  float theta;
  bool mapped = true;
  if (r2 < 0.5f) {
    theta = acos_deg(sqrtf(r2));
  } else if (r2 <= 1.0f) {
    theta = asin_deg(sqrtf(1.0f - r2));
  } else {
    mapped = false;
    theta = 0.0f;
  }
  if (mapped) {
    float sinphi, cosphi;
    sincos_deg(phi, sinphi, cosphi);
    x = sinphi;
    y = cosphi;
    float r, zr0;
    const unsigned tb = __float_as_uint(theta) - kThetaTabLo;
    if (ttab && tb < (unsigned)kThetaTabSize) {
      const float2 q = __ldg(&ttab[tb]);
      r = q.x;
      zr0 = q.y;
    } else {
      theta_terms(theta, r, zr0);
    }
    float w = xi * xi + eta * eta;
    if (w == 0.0f) {
      x = r * x;
      y = -r * y;
    } else {
      float z1 = xi * zr0;
      float z2 = eta * zr0;
      x = r * x + z1;
      y = -r * y + z2;
    }
    p1 = -1.0f / static_cast<float>(dc) * x + static_cast<float>(di) / 2.0f + 1.0f;
    p2 = 1.0f / static_cast<float>(dc) * y + static_cast<float>(di) / 2.0f + 1.0f;
  }
  LL = p1 - static_cast<float>(half);
  MM = p2 - static_cast<float>(half);
}

}  // namespace fipref
