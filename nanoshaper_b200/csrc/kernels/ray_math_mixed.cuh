// Mixed-precision ray-patch arithmetic: FP32 in patch-local coordinates for the bulk of the work,
// FP64 only where it decides the result.
//
//   * sphere hits: the discriminant and square root in FP32 on local offsets, then one FP64
//     Newton correction of the square root against the FP64 discriminant; near-tangent rays
//     (|disc| below a threshold) fall back to the double-precision test;
//   * torus hits: the FP32 discriminant only screens near-tangent rays; the clipping-sphere entry
//     and the quartic are the double-precision path's operations (built without fused
//     multiply-adds, its decisions guarded: a discriminant, resolvent root or square-root argument
//     within rounding of its threshold defers the candidate), because the reference's solver is
//     ill-conditioned for some rays and another rounding would move their roots by up to 1e-4 A;
//     measured on B200, an FP32 isolation followed by FP64 Newton polishing costs more FP64 issue
//     than the FP64 solver itself;
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

// The double-precision quartic solver (quartic_f64: the reference's Ferrari-type
// quarticEqSolutions, src/tools.cpp:525-639) with every decision guarded: it returns -1 when the
// discriminant, the resolvent root or a square-root argument lies within relative rounding of its
// threshold, or when the coefficients need the reciprocal variant.  Otherwise the roots equal
// those of quartic_f64 on the same coefficients (the same operation sequence), with complex pairs
// (negative square-root arguments) left out instead of returned as NaN.
__device__ __forceinline__ int quartic_guarded(double roots[4], double b, double c, double d, double e) {
  constexpr double kRel = 1e-10;
  const double b_2 = 0.5 * b;
  const double b_4 = 0.25 * b;
  const double p = c - 1.5 * (b_2 * b_2);
  const double q = d + b_2 * (b_2 * b_2 - c);
  const double r = e + b_4 * (b_4 * (c - 3.0 * b_4 * b_4) - d);
  const double f = p * p - 4. * r;
  const double t1 = 4. * r * (p * p), t2 = p * (q * q), t3 = 16. * (r * r), t4 = 128. * p * r, t5 = 27. * (q * q);
  const double delta = 4. * f * (t1 - t2 - t3) + (q * q) * (t4 - t5);
  if (e != 0. && (fabs(p) > 3.E+3 || fabs(r) > 3.E+3 || fabs(q) > 3.E+3 || fabs(delta) > 1.E+14)) return -1;
  const double dscale = fabs(4. * f) * (fabs(t1) + fabs(t2) + fabs(t3)) + (q * q) * (fabs(t4) + fabs(t5));
  if (!(fabs(delta) > kRel * dscale)) return -1;
  int num_sol;
  if (delta < 0.) {
    num_sol = 2;
  } else {
    if (!(fabs(p) > kRel * (fabs(c) + 1.5 * b_2 * b_2)) || !(fabs(f) > kRel * (p * p + fabs(4. * r)))) return -1;
    if (p < 0. && f > 0.) num_sol = 4;
    else return 0;
  }
  const double m = real_cubic_f64(p, 0.25 * (p * p) - r, (-0.125) * (q * q));
  const double mscale = fabs(p) + sqrt(fabs(r)) + 1e-300;
  if (!(fabs(m) > kRel * mscale) || fabs(m) < 1.E-13) return -1;
  if (m <= 0) return 0;
  const double p1 = -2. * (p + m);
  const double p2 = sqrt(2. * (q * q) / m);
  const double coeff = sqrt(2. * m);
  const double sscale = fabs(p1) + fabs(p2);
  const double sdmax = p1 + p2;
  if (!(fabs(sdmax) > kRel * sscale)) return -1;
  int n = 0;
  if (sdmax > 0.) {
    roots[n++] = 0.5 * (((q >= 0.) ? -coeff : coeff) - sqrt(sdmax)) - 0.25 * b;
    roots[n++] = 0.5 * (((q >= 0.) ? -coeff : coeff) + sqrt(sdmax)) - 0.25 * b;
  }
  if (num_sol == 4) {
    const double sdmin = p1 - p2;
    if (!(fabs(sdmin) > kRel * sscale)) return -1;
    if (sdmin > 0.) {
      roots[n++] = 0.5 * (((q >= 0.) ? coeff : -coeff) - sqrt(sdmin)) - 0.25 * b;
      roots[n++] = 0.5 * (((q >= 0.) ? coeff : -coeff) + sqrt(sdmin)) - 0.25 * b;
    }
  }
  return n;
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
// kTorus: the patch is an edge (torus) patch; otherwise a point (atom) or face (probe) patch.
template <bool kTorus>
__device__ __forceinline__ bool feasible_mixed(const double* P, int kind, int first, int cnt,
                                               const double4* __restrict__ pool, const float4* __restrict__ pool32,
                                               const int8_t* __restrict__ pflag, const float* pl32,
                                               const double* p64) {
  const double4* pl = pool + first;
  const float4* lp = pool32 + first;
  if (!kTorus && (kind == NS_FACE_REG || kind == NS_FACE_SING)) {
    for (int q = 0; q < cnt; q++)
      if (plane_value(lp[q], pl, q, pl32, p64) > 0) return false;
    return true;
  }
  if (!kTorus) {
    // a point patch: the hit is feasible unless it lies inside one of the clip spheres; four entries are loaded
    // ahead of their tests so that the loads of a group overlap
    const auto inside = [&](float4 s, int q) {
      float ex = pl32[0] - s.x, ey = pl32[1] - s.y, ez = pl32[2] - s.z;
      float dd = (ex * ex + ey * ey) + (ez * ez - s.w);
      if (fabsf(dd) > kSphereTol) return dd < 0.f;
      double4 sd = pl[q];
      double d64 = (sd.x - p64[0]) * (sd.x - p64[0]) + (sd.y - p64[1]) * (sd.y - p64[1]) + (sd.z - p64[2]) * (sd.z - p64[2]);
      d64 -= sd.w;
      return d64 < 0;
    };
    int q = 0;
    for (; q + 4 <= cnt; q += 4) {
      const float4 s0 = lp[q], s1 = lp[q + 1], s2 = lp[q + 2], s3 = lp[q + 3];
      if (inside(s0, q) || inside(s1, q + 1) || inside(s2, q + 2) || inside(s3, q + 3)) return false;
    }
    for (; q < cnt; q++)
      if (inside(lp[q], q)) return false;
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
