// Chain rule from per-patch surface parameters to atom coordinates and radii (host).
//
// The device adjoint (kernels/grad.cuh) gives, for every patch, the derivative of an output (ray
// cast volume, marching-cubes area) with respect to the parameters of the patch's surface:
//   point patch  (atom sphere)   : centre c (3), radius r (1)
//   facet patch  (probe sphere)  : centre p (3); the probe radius is fixed
//   edge patch   (torus)         : centre tc (3), axis u (3), major radius R (1)
// This file maps those to the atoms: an atom sphere is the atom itself; a probe centre p touches
// the three expanded spheres |p - c_a| = r_a + probe, differentiated implicitly; a torus is the
// circle where the expanded spheres of atoms i, j meet (tc, R) around the axis c_j - c_i
// (torus_geom in ses_builder.cpp, src/ConnollySurface.cpp:1296-1420), differentiated in forward
// mode over the 8 inputs c_i, c_j, r_i, r_j.
#include <cmath>
#include <cstring>

#include "../ns_types.h"
#include "host_api.h"

namespace {

// Forward-mode dual number with 8 derivative slots.
struct D8 {
  double v;
  double d[8];
};

D8 cst(double v) {
  D8 r;
  r.v = v;
  for (double& x : r.d) x = 0.0;
  return r;
}
D8 var(double v, int k) {
  D8 r = cst(v);
  r.d[k] = 1.0;
  return r;
}
D8 operator+(const D8& a, const D8& b) {
  D8 r;
  r.v = a.v + b.v;
  for (int k = 0; k < 8; k++) r.d[k] = a.d[k] + b.d[k];
  return r;
}
D8 operator-(const D8& a, const D8& b) {
  D8 r;
  r.v = a.v - b.v;
  for (int k = 0; k < 8; k++) r.d[k] = a.d[k] - b.d[k];
  return r;
}
D8 operator*(const D8& a, const D8& b) {
  D8 r;
  r.v = a.v * b.v;
  for (int k = 0; k < 8; k++) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
  return r;
}
D8 operator/(const D8& a, const D8& b) {
  D8 r;
  r.v = a.v / b.v;
  for (int k = 0; k < 8; k++) r.d[k] = (a.d[k] * b.v - a.v * b.d[k]) / (b.v * b.v);
  return r;
}
D8 dsqrt(const D8& a) {
  D8 r;
  r.v = std::sqrt(a.v);
  for (int k = 0; k < 8; k++) r.d[k] = a.d[k] / (2.0 * r.v);
  return r;
}

// Solves the 3x3 system M x = b (Cramer); returns false when M is singular.
bool solve3(const double M[3][3], const double* b, double* x) {
  double det = M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) - M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0]) +
               M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0]);
  if (!(std::fabs(det) > 0.0)) return false;
  for (int c = 0; c < 3; c++) {
    double A[3][3];
    memcpy(A, M, sizeof A);
    for (int r = 0; r < 3; r++) A[r][c] = b[r];
    x[c] = (A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) - A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]) +
            A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0])) /
           det;
  }
  return true;
}

}  // namespace

extern "C" {

// grad_atoms (n_atoms x 4: x, y, z, r) += d out / d atoms, from the per-patch parameter gradients
// gpatch (n_patches x NS_GRAD_PER_PATCH).  atoms_xyzr are the atoms the patches were built from
// (after any jitter); patch_atoms holds 3 atom indices per patch (nsg_patchset_atoms).
int nsg_ses_chain_grad(const double* atoms_xyzr, int64_t n_atoms, double probe, int64_t n_patches,
                       const int32_t* i32, const double* f64, const int32_t* patch_atoms, const double* gpatch,
                       double* grad_atoms) {
  if (!atoms_xyzr || !i32 || !f64 || !patch_atoms || !gpatch || !grad_atoms || n_atoms < 0 || n_patches < 0)
    return NSG_ERR_ARG;
  int n_bad = 0;
  for (int64_t p = 0; p < n_patches; p++) {
    const int kind = i32[NS_PATCH_I32 * p];
    const int32_t* pa = patch_atoms + 3 * p;
    const double* g = gpatch + NS_GRAD_PER_PATCH * p;
    bool any = false;
    for (int k = 0; k < NS_GRAD_PER_PATCH; k++) any |= g[k] != 0.0;
    if (!any) continue;
    for (int q = 0; q < 3; q++)
      if (pa[q] >= n_atoms) return NSG_ERR_ARG;
    if (kind == NS_POINT) {
      double* o = grad_atoms + 4 * pa[0];
      for (int k = 0; k < 4; k++) o[k] += g[k];
    } else if (kind == NS_FACE_REG || kind == NS_FACE_SING) {
      // J dp = [(p - c_a).dc_a + (r_a + probe) dr_a]_a with J rows (p - c_a); lambda = J^-T g
      const double* P = f64 + NS_PATCH_F64 * p;
      double J[3][3], JT[3][3], lam[3];
      for (int a = 0; a < 3; a++)
        for (int d = 0; d < 3; d++) J[a][d] = P[d] - atoms_xyzr[4 * pa[a] + d];
      for (int a = 0; a < 3; a++)
        for (int d = 0; d < 3; d++) JT[d][a] = J[a][d];
      if (!solve3(JT, g, lam)) {
        n_bad++;
        continue;
      }
      for (int a = 0; a < 3; a++) {
        double* o = grad_atoms + 4 * pa[a];
        for (int d = 0; d < 3; d++) o[d] += lam[a] * J[a][d];
        o[3] += lam[a] * (atoms_xyzr[4 * pa[a] + 3] + probe);
      }
    } else {
      // torus of atoms i, j: tc, u, R as functions of (c_i, c_j, r_i, r_j)
      const double* ci = atoms_xyzr + 4 * pa[0];
      const double* cj = atoms_xyzr + 4 * pa[1];
      D8 xi[3], xj[3];
      for (int d = 0; d < 3; d++) {
        xi[d] = var(ci[d], d);
        xj[d] = var(cj[d], 3 + d);
      }
      D8 ri = var(ci[3], 6) + cst(probe), rj = var(cj[3], 7) + cst(probe);
      D8 w1 = ri * ri, w2 = rj * rj;
      D8 diff[3] = {xj[0] - xi[0], xj[1] - xi[1], xj[2] - xi[2]};
      D8 dij2 = diff[0] * diff[0] + diff[1] * diff[1] + diff[2] * diff[2];
      D8 ratio = (w1 + dij2 - w2) * cst(0.5);
      D8 bigR = dsqrt(w1 - ratio * ratio / dij2);
      D8 cof = ratio / dij2;
      D8 dn = dsqrt(dij2);
      D8 out[7];
      for (int d = 0; d < 3; d++) {
        out[d] = xi[d] + cof * diff[d];  // tc
        out[3 + d] = diff[d] / dn;       // u
      }
      out[6] = bigR;
      double gin[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      for (int o = 0; o < 7; o++)
        for (int k = 0; k < 8; k++) gin[k] += g[o] * out[o].d[k];
      double* oi = grad_atoms + 4 * pa[0];
      double* oj = grad_atoms + 4 * pa[1];
      for (int d = 0; d < 3; d++) {
        oi[d] += gin[d];
        oj[d] += gin[3 + d];
      }
      oi[3] += gin[6];
      oj[3] += gin[7];
    }
  }
  return n_bad ? NSG_ERR_GEOMETRY : NSG_OK;
}

}  // extern "C"
