// Mixed-precision ray-patch arithmetic: FP32 in patch-local coordinates for the bulk of the work,
// FP64 only where it decides the result.
//
//   * sphere hits: the discriminant and square root in FP32 on local offsets, then one FP64
//     Newton correction of the square root against the FP64 discriminant; near-tangent rays
//     (|disc| below a threshold) fall back to the double-precision test;
//   * torus hits: every decision of the Ferrari-type solver (discriminant and root count,
//     resolvent branch and sign, which root pairs are real) in FP64 with the double-precision
//     solver's expressions; its transcendental steps (cube roots, arccos, cos) and the root
//     estimates in FP32, the resolvent root refined by FP64 Newton steps and each quartic root
//     polished by two FP64 Newton steps on the FP64 polynomial; a decision within rounding of its
//     threshold, merging roots or a small derivative defer the candidate to the double-precision
//     solver;
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

// Estimate of the resolvent root chosen by the double-precision solver (real_cubic_f64): the
// branch decisions are taken in FP64 with the same expressions, so the same root is approximated;
// the chosen closed form (Cardano cube roots, or the trigonometric form) is evaluated in FP32.
__device__ __forceinline__ float real_cubic_mixed(double b, double c, double d) {
  const double p = -(1.0 / 3.0) * b * b + c;
  const double q = (2. / 27.) * b * b * b - (1. / 3.) * b * c + d;
  const double D3p = (1. / 27.) * p * p * p;
  const double D3 = D3p + 0.25 * q * q;
  const float bf = (float)b;
  if (fabs(c) < b * b * 1.E-6 && fabs(d) < fabs(b) * 1.E-6) {
    return (float)(c / b - b - d / (b * b));
  } else if (fabs(d / c) < 4.E-4) {
    const double ratio = d / c;
    if (D3 <= 0.) return (float)(0.5 * (ratio - b + sqrt((b - ratio) * (b - ratio) - 4. * (c - ratio * (b - ratio)))));
    return (float)(-ratio * ratio * (b - ratio) / (3. * ratio * ratio - 2. * b * ratio + c) - ratio);
  } else if (D3 >= 0.) {
    const float radD3 = sqrtf((float)D3);
    const float hq = (float)(0.5 * q);
    return cbrtf(radD3 - hq) - cbrtf(radD3 + hq) - (1.f / 3.f) * bf;
  } else {
    const float Aarg = acosf((float)(-0.5 * q / sqrt(-D3p)));
    return 2.f * sqrtf((float)(-(1. / 3.) * p)) * cosf((1.f / 3.f) * Aarg) - (1.f / 3.f) * bf;
  }
}

// Root isolation of the monic quartic x^4 + b x^3 + c x^2 + d x + e, following the
// double-precision solver (quartic_f64): the depressed coefficients, the discriminant and the
// root-count decision in FP64 with the same operation sequence; the resolvent root estimated in
// FP32 on the same branch and refined by FP64 Newton steps on the resolvent cubic; the
// square-root arguments that decide which root pairs are real in FP64; the root estimates in
// FP32 (each is polished on the FP64 quartic afterwards).  Returns the number of roots, or -1
// when a decision is within rounding of its threshold (the resolvent refinement did not converge,
// the resolvent root or a square-root argument is near zero) or the coefficients need the
// reciprocal variant.
__device__ __forceinline__ int quartic_mixed(float roots[4], double b, double c, double d, double e) {
  const double b_2 = 0.5 * b;
  const double b_4 = 0.25 * b;
  const double p = c - 1.5 * (b_2 * b_2);
  const double q = d + b_2 * (b_2 * b_2 - c);
  const double r = e + b_4 * (b_4 * (c - 3.0 * b_4 * b_4) - d);
  const double f = p * p - 4. * r;
  const double delta =
      4. * f * (4. * r * (p * p) - p * (q * q) - 16. * (r * r)) + (q * q) * (128. * p * r - 27. * (q * q));
  if (e != 0. && (fabs(p) > 3.E+3 || fabs(r) > 3.E+3 || fabs(q) > 3.E+3 || fabs(delta) > 1.E+14)) return -1;
  int num_sol;
  if (delta < 0. || (delta == 0. && (p >= 0. || f < 0.)))
    num_sol = 2;
  else if ((p < 0. && f > 0.) || (delta == 0. && p == 0. && r == 0.))
    num_sol = 4;
  else
    return 0;
  // resolvent m^3 + p m^2 + (p^2/4 - r) m - q^2/8
  const double cb = p, cc = 0.25 * (p * p) - r, cd = (-0.125) * (q * q);
  double m = (double)real_cubic_mixed(cb, cc, cd);
  const double mscale = fabs(p) + sqrt(fabs(r)) + 1e-30;
  for (int it = 0; it < 3; it++) {
    const double g = ((m + cb) * m + cc) * m + cd;
    const double gp = (3.0 * m + 2.0 * cb) * m + cc;
    if (!(fabs(gp) > 1e-8 * (mscale * mscale + 1e-30))) return -1;
    const double step = g / gp;
    m -= step;
    if (it == 2 && !(fabs(step) <= 1e-12 * (fabs(m) + 1e-6 * mscale))) return -1;
  }
  if (!(fabs(m) > 1e-9 * mscale) || fabs(m) < 1.E-13) return -1;
  if (m <= 0.) return 0;
  const double p1 = -2. * (p + m);
  const double p2 = sqrt(2. * (q * q) / m);
  const double sscale = fabs(p1) + fabs(p2);
  const double sdmax = p1 + p2;
  if (!(fabs(sdmax) > 1e-9 * sscale)) return -1;
  const float coeff = sqrtf((float)(2. * m));
  const float b4f = (float)b_4;
  const float sq = (q >= 0.) ? -coeff : coeff;
  int n = 0;
  if (sdmax > 0.) {
    const float s = sqrtf((float)sdmax);
    roots[n++] = 0.5f * (sq - s) - b4f;
    roots[n++] = 0.5f * (sq + s) - b4f;
  }
  if (num_sol == 4) {
    const double sdmin = p1 - p2;
    if (!(fabs(sdmin) > 1e-9 * sscale)) return -1;
    if (sdmin > 0.) {
      const float s = sqrtf((float)sdmin);
      roots[n++] = 0.5f * (-sq - s) - b4f;
      roots[n++] = 0.5f * (-sq + s) - b4f;
    }
  }
  return n;
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
