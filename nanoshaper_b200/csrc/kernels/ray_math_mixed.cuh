// Mixed-precision ray-patch arithmetic: FP32 in patch-local coordinates for the bulk of the work,
// FP64 only where it decides the result.
//
//   * sphere hits: the discriminant and square root in FP32 on local offsets, then one FP64
//     Newton correction of the square root against the FP64 discriminant; near-tangent rays
//     (|disc| below a threshold) fall back to the double-precision test;
//   * torus hits: quartic coefficients in FP64, real roots isolated in FP32 with the same
//     Ferrari-type resolvent as the double-precision solver, each root polished by two FP64
//     Newton steps on the FP64 polynomial; whenever the FP32 isolation is near a decision boundary
//     (discriminant, resolvent root, merging roots, small derivative) the candidate falls back to
//     the double-precision solver;
//   * feasibility: plane and sphere tests in FP32 on local coordinates; a test whose FP32 value is
//     within a tolerance of zero is re-evaluated in FP64 from the double-precision pool.
// Hit points therefore carry FP64 accuracy and the accept/reject decisions equal the
// double-precision ones except where the FP64 value itself sits within rounding of zero.
#pragma once
#include <stdint.h>

#include "ray_math.cuh"

namespace nsg {

// FP32 tolerances of the fallback tests (in A, A^2 or relative units as noted).
constexpr float kDiscTol = 1e-3f;     // sphere discriminant r^2 - dx^2 - dy^2 [A^2]
constexpr float kPlaneTol = 1e-3f;    // plane test value [A] (planes are unit normals)
constexpr float kSphereTol = 1e-2f;   // clipping-sphere test |p-s|^2 - r^2 [A^2]
constexpr float kRelTol = 1e-4f;      // relative closeness of quartic decision quantities

// Cubic resolvent root in FP32 (same branch structure as the double-precision restatement).
__device__ __forceinline__ float real_cubic_f32(float b, float c, float d) {
  float p = -(1.0f / 3.0f) * b * b + c;
  float q = (2.f / 27.f) * b * b * b - (1.f / 3.f) * b * c + d;
  float D3p = (1.f / 27.f) * p * p * p;
  float D3 = D3p + 0.25f * q * q;
  if (fabsf(c) < b * b * 1.E-6f && fabsf(d) < fabsf(b) * 1.E-6f) {
    return c / b - b - d / (b * b);
  } else if (fabsf(d / c) < 4.E-4f) {
    float ratio = d / c;
    if (D3 <= 0.f) {
      return 0.5f * (ratio - b + sqrtf((b - ratio) * (b - ratio) - 4.f * (c - ratio * (b - ratio))));
    } else {
      float eps = -ratio * ratio * (b - ratio) / (3.f * ratio * ratio - 2.f * b * ratio + c);
      return eps - ratio;
    }
  } else {
    if (D3 >= 0.f) {
      float radD3 = sqrtf(D3);
      float A = cbrtf(radD3 - 0.5f * q);
      float psu3A = cbrtf(radD3 + 0.5f * q);
      return A - psu3A - (1.f / 3.f) * b;
    } else {
      float Aarg = acosf(-0.5f * q / sqrtf(-D3p));
      return 2.f * sqrtf(-(1.f / 3.f) * p) * cosf((1.f / 3.f) * Aarg) - (1.f / 3.f) * b;
    }
  }
}

// FP32 root isolation of the monic quartic; returns the number of roots, or -1 when a decision
// is too close to call in FP32.
__device__ __forceinline__ int quartic_f32(float roots[4], float b, float c, float d, float e) {
  float b_2 = 0.5f * b;
  float b_4 = 0.25f * b;
  float p = c - 1.5f * (b_2 * b_2);
  float q = d + b_2 * (b_2 * b_2 - c);
  float r = e + b_4 * (b_4 * (c - 3.0f * b_4 * b_4) - d);
  if (fabsf(p) > 3.E+3f || fabsf(r) > 3.E+3f || fabsf(q) > 3.E+3f) return -1;  // reciprocal variant: FP64
  float f = p * p - 4.f * r;
  float t1 = 4.f * r * (p * p), t2 = p * (q * q), t3 = 16.f * (r * r);
  float t4 = 128.f * p * r, t5 = 27.f * (q * q);
  float delta = 4.f * f * (t1 - t2 - t3) + (q * q) * (t4 - t5);
  float dscale = fabsf(4.f * f) * (fabsf(t1) + fabsf(t2) + fabsf(t3)) + (q * q) * (fabsf(t4) + fabsf(t5));
  if (!(fabsf(delta) > kRelTol * dscale)) return -1;
  if (fabsf(delta) > 1.E+14f) return -1;
  int num_sol;
  if (delta < 0.f) {
    num_sol = 2;
  } else {
    if (fabsf(p) < kRelTol * (fabsf(c) + 1.f) || fabsf(f) < kRelTol * (p * p + fabsf(4.f * r))) return -1;
    if (p < 0.f && f > 0.f) num_sol = 4;
    else return 0;
  }
  float m = real_cubic_f32(p, 0.25f * (p * p) - r, (-0.125f) * (q * q));
  float mscale = fabsf(p) + sqrtf(fabsf(r)) + 1e-30f;
  if (!(fabsf(m) > kRelTol * mscale)) return -1;
  if (m <= 0.f) return 0;
  float p1 = -2.f * (p + m);
  float p2 = sqrtf(2.f * (q * q) / m);
  float coeff = sqrtf(2.f * m);
  float sdmax = p1 + p2;
  float sscale = fabsf(p1) + fabsf(p2);
  if (!(fabsf(sdmax) > kRelTol * sscale) || sdmax < 0.f) return -1;
  float sq = (q >= 0.f) ? -coeff : coeff;
  roots[0] = 0.5f * (sq - sqrtf(sdmax)) - 0.25f * b;
  roots[1] = 0.5f * (sq + sqrtf(sdmax)) - 0.25f * b;
  if (num_sol == 4) {
    float sdmin = p1 - p2;
    if (!(fabsf(sdmin) > kRelTol * sscale) || sdmin < 0.f) return -1;
    roots[2] = 0.5f * (-sq - sqrtf(sdmin)) - 0.25f * b;
    roots[3] = 0.5f * (-sq + sqrtf(sdmin)) - 0.25f * b;
  }
  return num_sol;
}

// Two Newton steps on the FP64 monic quartic; returns false when the derivative is too small
// for the polish to be trusted (a root of multiplicity > 1 is close) or when the FP32 estimate
// was not already close to a root.
__device__ __forceinline__ bool polish_root(double B, double C, double D, double E, double& x) {
  for (int it = 0; it < 2; it++) {
    double f = (((x + B) * x + C) * x + D) * x + E;
    double fp = ((4.0 * x + 3.0 * B) * x + 2.0 * C) * x + D;
    double scale = fabs(D) + fabs(C) + fabs(B) + 1.0;
    if (!(fabs(fp) > 1e-3 * scale)) return false;
    double step = f / fp;
    if (it == 0 && !(fabs(step) < 1e-3 * (fabs(x) + 1.0))) return false;
    x -= step;
  }
  return true;
}

// Plane test value in FP64 (from the double-precision pool) when the FP32 one is undecided.
__device__ __forceinline__ double plane_value(float4 lw, const double4* pl, int q, const float* pl32,
                                              const double* p64) {
  float v = (lw.x * pl32[0] + lw.y * pl32[1]) + (lw.z * pl32[2] + lw.w);
  if (fabsf(v) > kPlaneTol) return (double)v;
  return plane_test_f64(pl[q], p64);
}

// Feasibility with FP32 tests on patch-local coordinates (pl32 = hit - patch centre) and FP64
// re-evaluation of undecided tests (p64 = absolute hit point).
__device__ __forceinline__ bool feasible_mixed(const double* P, int kind, int first, int cnt,
                                               const double4* __restrict__ pool, const float4* __restrict__ pool32,
                                               const int8_t* __restrict__ pflag, const float* pl32,
                                               const double* p64) {
  const double4* pl = pool + first;
  const float4* lp = pool32 + first;
  if (kind == NS_FACE_REG || kind == NS_FACE_SING) {
    for (int q = 0; q < cnt; q++)
      if (plane_value(lp[q], pl, q, pl32, p64) > 0) return false;
    return true;
  }
  if (kind == NS_POINT) {
    for (int q = 0; q < cnt; q++) {
      float4 s = lp[q];
      float ex = pl32[0] - s.x, ey = pl32[1] - s.y, ez = pl32[2] - s.z;
      float dd = (ex * ex + ey * ey) + (ez * ez - s.w);
      if (fabsf(dd) > kSphereTol) {
        if (dd < 0.f) return false;
        continue;
      }
      double4 sd = pl[q];
      double d64 = (sd.x - p64[0]) * (sd.x - p64[0]) + (sd.y - p64[1]) * (sd.y - p64[1]) + (sd.z - p64[2]) * (sd.z - p64[2]);
      d64 -= sd.w;
      if (d64 < 0) return false;
    }
    return true;
  }
  double sir = P[kSir];
  if (sir >= 0.) {
    double dd = (P[kTC] - p64[0]) * (P[kTC] - p64[0]) + (P[kTC + 1] - p64[1]) * (P[kTC + 1] - p64[1]) +
                (P[kTC + 2] - p64[2]) * (P[kTC + 2] - p64[2]);
    if (dd < sir * sir) return false;
  }
  if (cnt == 0) return true;
  const int8_t* fl = pflag + first;
  for (int q = 0; q + 1 < cnt; q += 2) {
    double t0 = plane_value(lp[q], pl, q, pl32, p64);
    if (fl[q]) {
      if (t0 > 0) continue;
      if (plane_value(lp[q + 1], pl, q + 1, pl32, p64) > 0) continue;
      return true;
    } else {
      if (t0 <= 0) return true;
      if (plane_value(lp[q + 1], pl, q + 1, pl32, p64) <= 0) return true;
    }
  }
  return false;
}

}  // namespace nsg
