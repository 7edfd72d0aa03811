// Device arithmetic of the SES ray tracer: ray-sphere, ray-torus (analytical quartic) and the
// patch feasibility tests.  The double-precision functions evaluate exactly the operation
// sequence of the reference (raySphere src/tools.cpp:833-861, realCubicSolution :350-391,
// quarticEqSolutions :525-639, rayTorus :907-1098, ConnollySurface::isFeasible
// src/ConnollySurface.cpp:4769-5019); the translation unit is compiled with --fmad=false so that
// every product and sum rounds separately, as on the host.
#pragma once
#include <stdint.h>

#include "../ns_types.h"

namespace nsg {

__device__ __forceinline__ double rintp(double x) { return floor(x + 0.5); }

// Field offsets of a patch record (NS_PATCH_F64 doubles, see ns_types.h).
constexpr int kC = 0, kR = 3, kTC = 4, kMajor = 7, kSir = 8, kInv = 9;

__device__ __forceinline__ bool ray_sphere_f64(const double* orig, const double* dir, const double* c, double r,
                                               double* t1, double* t2) {
  double temp0 = orig[0] - c[0], temp1 = orig[1] - c[1], temp2 = orig[2] - c[2];
  double A = dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2];
  double B = temp0 * dir[0] + temp1 * dir[1] + temp2 * dir[2];
  double C = temp0 * temp0 + temp1 * temp1 + temp2 * temp2 - r * r;
  double det = B * B - A * C;
  if (det < 0.) return false;
  det = sqrt(det);
  double a = (-B - det) / A;
  double b = (-B + det) / A;
  if (b < a) { double tt = a; a = b; b = tt; }
  *t1 = a;
  *t2 = b;
  return true;
}

__device__ __forceinline__ double real_cubic_f64(double b, double c, double d) {
  double p = -(1.0 / 3.0) * b * b + c;
  double q = (2. / 27.) * b * b * b - (1. / 3.) * b * c + d;
  double D3p = (1. / 27.) * p * p * p;
  double D3 = D3p + 0.25 * q * q;
  if (fabs(c) < b * b * 1.E-6 && fabs(d) < fabs(b) * 1.E-6) {
    return c / b - b - d / (b * b);
  } else if (fabs(d / c) < 4.E-4) {
    double ratio = d / c;
    if (D3 <= 0.) {
      return 0.5 * (ratio - b + sqrt((b - ratio) * (b - ratio) - 4. * (c - ratio * (b - ratio))));
    } else {
      double eps = -ratio * ratio * (b - ratio) / (3. * ratio * ratio - 2. * b * ratio + c);
      return eps - ratio;
    }
  } else {
    if (D3 >= 0.) {
      double radD3 = sqrt(D3);
      double A = cbrt(radD3 - 0.5 * q);
      double psu3A = cbrt(radD3 + 0.5 * q);
      return A - psu3A - (1. / 3.) * b;
    } else {
      double Aarg = acos(-0.5 * q / sqrt(-D3p));
      return 2. * sqrt(-(1. / 3.) * p) * cos((1. / 3.) * Aarg) - (1. / 3.) * b;
    }
  }
}

__device__ __forceinline__ int quartic_f64(double roots[4], double b, double c, double d, double e) {
  double b_2 = 0.5 * b;
  double b_4 = 0.25 * b;
  double p = c - 1.5 * (b_2 * b_2);
  double q = d + b_2 * (b_2 * b_2 - c);
  double r = e + b_4 * (b_4 * (c - 3.0 * b_4 * b_4) - d);
  double f = p * p - 4. * r;
  double delta = 4. * f * (4. * r * (p * p) - p * (q * q) - 16. * (r * r)) + (q * q) * (128. * p * r - 27. * (q * q));
  bool change_variant = false;
  if (e != 0. && (fabs(p) > 3.E+3 || fabs(r) > 3.E+3 || fabs(q) > 3.E+3 || fabs(delta) > 1.E+14)) {
    double dsu2e = 0.5 * d / e;
    change_variant = true;
    p = -1.5 * dsu2e * dsu2e + c / e;
    q = dsu2e * (dsu2e * dsu2e - c / e) + b / e;
    r = dsu2e * (-3. / 16. * (dsu2e * dsu2e * dsu2e) + 0.25 * dsu2e * (c / e) - 0.5 * b / e) + 1. / e;
    f = p * p - 4. * r;
    delta = 4. * f * (4. * r * (p * p) - p * (q * q) - 16. * (r * r)) + (q * q) * (128. * p * r - 27. * (q * q));
  }
  int num_sol;
  if (delta < 0. || (delta == 0. && (p >= 0. || f < 0.)))
    num_sol = 2;
  else if ((p < 0. && f > 0.) || (delta == 0. && p == 0. && r == 0.))
    num_sol = 4;
  else
    return 0;
  double m = real_cubic_f64(p, 0.25 * (p * p) - r, (-0.125) * (q * q));
  if (m <= 0) return 0;
  double coeff, p1, p2, p3 = 0, sol_delta_max;
  if (m < 1.E-14) {
    p1 = p + p;
    p2 = (q * q) / f;
    p3 = 2. * sqrt(f);
    sol_delta_max = p3 - p1 - p2;
    coeff = 2. * fabs(q) / f;
  } else {
    p1 = -2. * (p + m);
    p2 = sqrt(2. * (q * q) / m);
    sol_delta_max = p1 + p2;
    coeff = sqrt(2. * m);
  }
  roots[0] = 0.5 * (((q >= 0.) ? -coeff : coeff) - sqrt(sol_delta_max));
  roots[1] = 0.5 * (((q >= 0.) ? -coeff : coeff) + sqrt(sol_delta_max));
  if (num_sol == 4) {
    double sol_delta_min = (m < 1.E-14) ? (-p1 - p2 - p3) : (p1 - p2);
    roots[2] = 0.5 * (((q >= 0.) ? coeff : -coeff) - sqrt(sol_delta_min));
    roots[3] = 0.5 * (((q >= 0.) ? coeff : -coeff) + sqrt(sol_delta_min));
  }
  if (change_variant) {
    for (int i = 0; i < num_sol; i++) roots[i] = 1. / (roots[i] - 0.25 * d / e);
  } else {
    for (int i = 0; i < num_sol; i++) roots[i] -= 0.25 * b;
  }
  return num_sol;
}

// Torus quartic coefficients for a ray starting at orig1 (already moved to the clipping-sphere
// entry) along axis vc.
__device__ __forceinline__ void torus_coeffs_f64(const double* P, double probe, int vc, const double* orig1,
                                                 double* B, double* C, double* D, double* E) {
  const double* inv = P + kInv;
  double temp0 = orig1[0] - P[kTC], temp1 = orig1[1] - P[kTC + 1], temp2 = orig1[2] - P[kTC + 2];
  double pp[3];
#pragma unroll
  for (int i = 0; i < 3; i++) pp[i] = inv[3 * i + 0] * temp0 + inv[3 * i + 1] * temp1 + inv[3 * i + 2] * temp2;
  double r2 = probe * probe;
  double R2 = P[kMajor] * P[kMajor];
  double pd = pp[0] * inv[0 * 3 + vc] + pp[1] * inv[1 * 3 + vc] + pp[2] * inv[2 * 3 + vc];
  double p2 = pp[0] * pp[0] + pp[1] * pp[1] + pp[2] * pp[2];
  double coeff = p2 - r2 - R2;
  double iz = inv[2 * 3 + vc];
  *B = 4 * pd;
  *C = 2 * coeff + 4 * pd * pd + 4 * R2 * iz * iz;
  *D = 4 * pd * coeff + 8 * R2 * pp[2] * iz;
  *E = coeff * coeff - 4 * R2 * (r2 - pp[2] * pp[2]);
}

// rayTorus: t[0] holds the clipping-sphere entry on input; the accepted torus hits are written
// to t[0..n-1] in root order.
__device__ __forceinline__ int ray_torus_f64(const double* P, double probe, int vc, const double* orig,
                                             double ray_dir, double t[4]) {
  double orig1[3] = {orig[0], orig[1], orig[2]};
  orig1[vc] += t[0] * ray_dir;
  double B, C, D, E;
  torus_coeffs_f64(P, probe, vc, orig1, &B, &C, &D, &E);
  double roots[4];
  int nr = quartic_f64(roots, B, C, D, E);
  double t0 = t[0];
  int n = 0;
  for (int i = 0; i < nr; i++) {
    if (roots[i] < 0) continue;
    double point[3] = {orig1[0], orig1[1], orig1[2]};
    point[vc] += roots[i];
    double dd = (P[0] - point[0]) * (P[0] - point[0]) + (P[1] - point[1]) * (P[1] - point[1]) +
                (P[2] - point[2]) * (P[2] - point[2]);
    if (dd < P[kR] * P[kR]) t[n++] = t0 + roots[i] / ray_dir;
  }
  return n;
}

__device__ __forceinline__ double plane_test_f64(const double4 w, const double* p) {
  return (w.x * p[0] + w.y * p[1] + w.z * p[2]) + w.w;
}

// isFeasible over the patch-set encoding (see ns_types.h).
__device__ __forceinline__ bool feasible_f64(const double* P, int kind, int first, int cnt,
                                             const double4* __restrict__ pool, const int8_t* __restrict__ pflag,
                                             const double* p) {
  const double4* pl = pool + first;
  if (kind == NS_FACE_REG || kind == NS_FACE_SING) {
    for (int q = 0; q < cnt; q++)
      if (plane_test_f64(pl[q], p) > 0) return false;
    return true;
  }
  if (kind == NS_POINT) {
    for (int q = 0; q < cnt; q++) {
      double4 s = pl[q];
      double dd = (s.x - p[0]) * (s.x - p[0]) + (s.y - p[1]) * (s.y - p[1]) + (s.z - p[2]) * (s.z - p[2]);
      dd -= s.w;
      if (dd < 0) return false;
    }
    return true;
  }
  double sir = P[kSir];
  if (sir >= 0.) {
    double dd = (P[kTC] - p[0]) * (P[kTC] - p[0]) + (P[kTC + 1] - p[1]) * (P[kTC + 1] - p[1]) +
                (P[kTC + 2] - p[2]) * (P[kTC + 2] - p[2]);
    if (dd < sir * sir) return false;
  }
  if (cnt == 0) return true;
  const int8_t* fl = pflag + first;
  for (int q = 0; q + 1 < cnt; q += 2) {
    double t0 = plane_test_f64(pl[q], p);
    if (fl[q]) {
      if (t0 > 0) continue;
      if (plane_test_f64(pl[q + 1], p) > 0) continue;
      return true;
    } else {
      if (t0 <= 0) return true;
      if (plane_test_f64(pl[q + 1], p) <= 0) return true;
    }
  }
  return false;
}

// rayQuadricIntersectionX/Y/Z of the skin surface (src/SkinSurface.cpp:4632-4709): a ray of unit
// direction along axis VC from o against the quadric Q (coding q11, q22, q33, q44, q12, q23, q34,
// q13, q24, q14); t[0..1] in Angstrom from o, operation for operation as the reference.
template <int VC>
__device__ __forceinline__ bool ray_quadric_f64(const double* Q, const double* o, double* t) {
  const double q44 = Q[3], q33 = Q[2], q22 = Q[1], q11 = Q[0], q34 = Q[6], q24 = Q[8], q23 = Q[5], q14 = Q[9],
               q13 = Q[7], q12 = Q[4];
  double a, b;
  if (VC == 0) {
    a = q11;
    if (a == 0) return false;
    b = q14 + o[2] * q13 + o[1] * q12 + o[0] * q11;
  } else if (VC == 1) {
    a = q22;
    if (a == 0) return false;
    b = q24 + o[2] * q23 + o[1] * q22 + o[0] * q12;
  } else {
    a = q33;
    if (a == 0) return false;
    b = q34 + o[2] * q33 + o[1] * q23 + o[0] * q13;
  }
  const double c = q44 + (o[2] + o[2]) * q34 + (o[2] * o[2]) * q33 + (o[1] + o[1]) * q24 + (2 * o[1] * o[2]) * q23 +
                   (o[1] * o[1]) * q22 + (o[0] + o[0]) * q14 + (2 * o[0] * o[2]) * q13 + (2 * o[0] * o[1]) * q12 +
                   (o[0] * o[0]) * q11;
  double delta = b * b - a * c;
  if (delta < 0) return false;
  delta = sqrt(delta);
  t[0] = (-b - delta) / a;
  t[1] = (-b + delta) / a;
  return true;
}

// SkinSurface::isFeasible (src/SkinSurface.cpp:4374-4448) over the cell's planes: outside the cell
// when a plane test is positive (Del0 planes are stored negated, see ns_types.h).
__device__ __forceinline__ bool feasible_skin_f64(const double4* __restrict__ pool, int first, int cnt,
                                                  const double* p) {
  const double4* pl = pool + first;
  for (int q = 0; q < cnt; q++)
    if (plane_test_f64(pl[q], p) > 0) return false;
  return true;
}

// MeshSurface::intersect_triangle (src/MeshSurface.cpp:1487-1553, the non-culling branch) for a
// ray from orig with direction dir (the full ray, so t is the ray parameter), operation for
// operation; EPS = 1e-5 (src/MeshSurface.h:21).  Returns the parameter t and the barycentric u, v.
__device__ __forceinline__ bool ray_triangle_f64(const double* orig, const double* dir, const double* v0,
                                                 const double* v1, const double* v2, double* t, double* uo,
                                                 double* vo) {
  constexpr double kEps = 1e-5;
  double edge1[3], edge2[3], tvec[3], pvec[3], qvec[3];
  edge1[0] = v1[0] - v0[0]; edge1[1] = v1[1] - v0[1]; edge1[2] = v1[2] - v0[2];
  edge2[0] = v2[0] - v0[0]; edge2[1] = v2[1] - v0[1]; edge2[2] = v2[2] - v0[2];
  pvec[0] = dir[1] * edge2[2] - dir[2] * edge2[1];
  pvec[1] = dir[2] * edge2[0] - dir[0] * edge2[2];
  pvec[2] = dir[0] * edge2[1] - dir[1] * edge2[0];
  const double det = edge1[0] * pvec[0] + edge1[1] * pvec[1] + edge1[2] * pvec[2];
  if (det > -kEps && det < kEps) return false;
  const double inv_det = 1.0 / det;
  tvec[0] = orig[0] - v0[0]; tvec[1] = orig[1] - v0[1]; tvec[2] = orig[2] - v0[2];
  const double u = (tvec[0] * pvec[0] + tvec[1] * pvec[1] + tvec[2] * pvec[2]) * inv_det;
  if (u < 0.0 || u > 1.0) return false;
  qvec[0] = tvec[1] * edge1[2] - tvec[2] * edge1[1];
  qvec[1] = tvec[2] * edge1[0] - tvec[0] * edge1[2];
  qvec[2] = tvec[0] * edge1[1] - tvec[1] * edge1[0];
  const double v = (dir[0] * qvec[0] + dir[1] * qvec[1] + dir[2] * qvec[2]) * inv_det;
  if (v < 0.0 || u + v > 1.0) return false;
  *t = (edge2[0] * qvec[0] + edge2[1] * qvec[1] + edge2[2] * qvec[2]) * inv_det;
  *uo = u;
  *vo = v;
  return true;
}

}  // namespace nsg
