// Chain rule from one patch's surface-parameter derivatives to its atoms, shared by the host
// (host/grad.cpp) and the device (kernels/chain.cu).
//
// Per-patch parameters (NS_GRAD_PER_PATCH slots):
//   point patch  (atom sphere)   : centre c (3), radius r (1)       -> the atom itself
//   facet patch  (probe sphere)  : centre p (3)                     -> the three atoms it touches:
//       |p - c_a| = r_a + probe, so J dp = [(p - c_a).dc_a + (r_a + probe) dr_a]_a with J rows
//       (p - c_a); with lambda = J^-T g: d/dc_a = lambda_a (p - c_a), d/dr_a = lambda_a (r_a + probe)
//   edge patch   (torus)         : centre tc (3), axis u (3), R (1) -> atoms i, j: the circle where
//       the expanded spheres meet (ConnollySurface torus construction,
//       src/ConnollySurface.cpp:1296-1420), differentiated in forward mode over c_i, c_j, r_i, r_j.
#pragma once
#include <math.h>
#include <stdint.h>

#include "ns_types.h"

namespace nsg {

struct D8 {
  double v;
  double d[8];
};

NS_HD D8 d8_cst(double v) {
  D8 r;
  r.v = v;
  for (int k = 0; k < 8; k++) r.d[k] = 0.0;
  return r;
}
NS_HD D8 d8_var(double v, int k) {
  D8 r = d8_cst(v);
  r.d[k] = 1.0;
  return r;
}
NS_HD D8 d8_add(const D8& a, const D8& b) {
  D8 r;
  r.v = a.v + b.v;
  for (int k = 0; k < 8; k++) r.d[k] = a.d[k] + b.d[k];
  return r;
}
NS_HD D8 d8_sub(const D8& a, const D8& b) {
  D8 r;
  r.v = a.v - b.v;
  for (int k = 0; k < 8; k++) r.d[k] = a.d[k] - b.d[k];
  return r;
}
NS_HD D8 d8_mul(const D8& a, const D8& b) {
  D8 r;
  r.v = a.v * b.v;
  for (int k = 0; k < 8; k++) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
  return r;
}
NS_HD D8 d8_div(const D8& a, const D8& b) {
  D8 r;
  r.v = a.v / b.v;
  for (int k = 0; k < 8; k++) r.d[k] = (a.d[k] * b.v - a.v * b.d[k]) / (b.v * b.v);
  return r;
}
NS_HD D8 d8_sqrt(const D8& a) {
  D8 r;
  r.v = sqrt(a.v);
  for (int k = 0; k < 8; k++) r.d[k] = a.d[k] / (2.0 * r.v);
  return r;
}

NS_HD double det3(const double M[3][3]) {
  return M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) - M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0]) +
         M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0]);
}

// Adds the patch's contribution to the atom derivatives through add(atom, slot, value); patch_atoms
// indexes into atoms (x, y, z, r per atom).  Returns false when a facet's system is singular.
template <class Add>
NS_HD bool chain_patch(int kind, const double* P, const int32_t* pa, const double* atoms, double probe,
                       const double* g, Add add) {
  bool any = false;
  for (int k = 0; k < NS_GRAD_PER_PATCH; k++) any |= g[k] != 0.0;
  if (!any) return true;
  if (kind == NS_POINT) {
    for (int k = 0; k < 4; k++) add(pa[0], k, g[k]);
    return true;
  }
  if (kind == NS_FACE_REG || kind == NS_FACE_SING) {
    double J[3][3], JT[3][3];
    for (int a = 0; a < 3; a++)
      for (int d = 0; d < 3; d++) J[a][d] = P[d] - atoms[4 * pa[a] + d];
    for (int a = 0; a < 3; a++)
      for (int d = 0; d < 3; d++) JT[d][a] = J[a][d];
    const double det = det3(JT);
    if (!(fabs(det) > 0.0)) return false;
    for (int a = 0; a < 3; a++) {
      double M[3][3];
      for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) M[r][c] = c == a ? g[r] : JT[r][c];
      const double lam = det3(M) / det;
      for (int d = 0; d < 3; d++) add(pa[a], d, lam * J[a][d]);
      add(pa[a], 3, lam * (atoms[4 * pa[a] + 3] + probe));
    }
    return true;
  }
  const double* ci = atoms + 4 * pa[0];
  const double* cj = atoms + 4 * pa[1];
  D8 xi[3], xj[3], diff[3];
  for (int d = 0; d < 3; d++) {
    xi[d] = d8_var(ci[d], d);
    xj[d] = d8_var(cj[d], 3 + d);
    diff[d] = d8_sub(xj[d], xi[d]);
  }
  const D8 ri = d8_add(d8_var(ci[3], 6), d8_cst(probe)), rj = d8_add(d8_var(cj[3], 7), d8_cst(probe));
  const D8 w1 = d8_mul(ri, ri), w2 = d8_mul(rj, rj);
  const D8 dij2 = d8_add(d8_add(d8_mul(diff[0], diff[0]), d8_mul(diff[1], diff[1])), d8_mul(diff[2], diff[2]));
  const D8 ratio = d8_mul(d8_sub(d8_add(w1, dij2), w2), d8_cst(0.5));
  const D8 bigR = d8_sqrt(d8_sub(w1, d8_div(d8_mul(ratio, ratio), dij2)));
  const D8 cof = d8_div(ratio, dij2);
  const D8 dn = d8_sqrt(dij2);
  double gin[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int d = 0; d < 3; d++) {
    const D8 tc = d8_add(xi[d], d8_mul(cof, diff[d]));
    const D8 u = d8_div(diff[d], dn);
    for (int k = 0; k < 8; k++) gin[k] += g[d] * tc.d[k] + g[3 + d] * u.d[k];
  }
  for (int k = 0; k < 8; k++) gin[k] += g[6] * bigR.d[k];
  for (int d = 0; d < 3; d++) {
    add(pa[0], d, gin[d]);
    add(pa[1], d, gin[3 + d]);
  }
  add(pa[0], 3, gin[6]);
  add(pa[1], 3, gin[7]);
  return true;
}

}  // namespace nsg
