// ORACLE — test infrastructure only.  CPU restatement of the reference's grid ray-casting surface
// path, used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as the checker.
// It is never linked into, called by or loaded from the product library.
//
// Restates, for the patch-based ray tracer of an SES patch set:
//   * per-patch ray casting     ConnollySurface::getPatchIntersectionData
//                               (src/ConnollySurface.cpp:4319-4590), raySphere (src/tools.cpp:833-861),
//                               rayTorus (src/tools.cpp:907-1098), quarticEqSolutions
//                               (src/tools.cpp:525-639), realCubicSolution (src/tools.cpp:350-391),
//                               ConnollySurface::isFeasible (src/ConnollySurface.cpp:4769-5019)
//   * pixel binning and sort    countPixelIntersections / copyPatchIntersections /
//                               reorderPatchIntersections (src/Surface.cpp:4941-5095)
//   * interval fill             setVerticesAndGridsWithIntersectionData (src/Surface.cpp:5101-6251)
//                               with NEW_INTERSECTION_FILTERING: a ray with an odd hit count is
//                               skipped (the emptiness test precedes the closure test, :5279-5287)
//   * volume                    src/Surface.cpp:1680-1684
//   * cavities                  getCavitiesWithBilevelStatusMap (src/Surface.cpp:1994-2126),
//                               floodFillWithBilevelStatusMap2 (:4284-4554), fillCavities (:2355-2484)
//   * vertex assembly           assembleVerticesList (src/Surface.cpp:7415-7667)
//   * marching cubes            triangulateSurface / getVertices / triangulationKernel / getTriangles
//                               (src/Surface.cpp:9909-10300, 8002-8327, 9075-9318, 14526-14780)
// For skin patch sets (mixed cells):
//   * per-cell ray casting      SkinSurface::getPatchIntersectionData (src/SkinSurface.cpp:3422-3760),
//                               rayQuadricIntersectionX/Y/Z (:4632-4709), isFeasible (:4374-4448)
// For blobby surfaces:
//   * field, marching cubes     BlobbySurface::build (src/BlobbySurface.cpp:83-229), getVertices
//                               with a scalar field (src/Surface.cpp:8143-8327), triangulationKernel
//                               (:9075-9318), vertexInterp (:14516-14523), classifyCube (:14526-14545)
//   * smoothing                 smoothSurface (src/Surface.cpp:13089-13354)
//   * OFF round trip            saveMesh "%.3f" (src/Surface.cpp:10857-10960), loadOFF "%f"
//                               (src/MeshSurface.cpp:2350-2479), done here with snprintf / sscanf
//   * ray casting               MeshSurface::getRayIntersection + intersect_triangle
//                               (src/MeshSurface.cpp:1487-1553, 1756-1855)
// Single-threaded by default so that volume and area are summed in the reference's serial order.
// Compile without FMA contraction (-ffp-contract=off) so that every operation rounds as written.
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <deque>
#include <stack>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include "../nanoshaper_b200/csrc/mc_cases.h"
#include "../nanoshaper_b200/csrc/ns_types.h"

namespace {

inline double rintp(double x) { return floor(x + 0.5); }

struct Patches {
  int64_t n;
  const double* f64;
  const int32_t* i32;
  const double* pool;
  const int8_t* flag;
  double probe;
};

// raySphere (src/tools.cpp:833-861)
bool ray_sphere(const double* orig, const double* dir, const double* c, double r, double* t1, double* t2) {
  double temp[3], A, B, C;
  A = dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2];
  temp[0] = orig[0] - c[0]; temp[1] = orig[1] - c[1]; temp[2] = orig[2] - c[2];
  B = temp[0] * dir[0] + temp[1] * dir[1] + temp[2] * dir[2];
  C = temp[0] * temp[0] + temp[1] * temp[1] + temp[2] * temp[2] - r * r;
  double det = B * B - A * C;
  if (det < 0.) return false;
  det = sqrt(det);
  *t1 = (-B - det) / A;
  *t2 = (-B + det) / A;
  if (*t2 < *t1) { double tt = *t1; *t1 = *t2; *t2 = tt; }
  return true;
}

// Branch counters of the torus path (the op model of the bench's roofline and the candidates'
// branch mix): torus candidates, clipping-sphere misses, quartic outcomes, resolvent-cubic branches.
enum {
  kOpTorusCand, kOpTorusNoSphere, kOpQuarticNone, kOpQuarticM0, kOpQuartic2, kOpQuartic4, kOpQuarticRecip,
  kOpCubicSmallC, kOpCubicRatioSqrt, kOpCubicRatioEps, kOpCubicCbrt, kOpCubicAcos, kOpSphereCand,
  kOpSphereMiss, kOpRootTest, kOpRootIn, kOpFeasTest, kOpPlaneTest, kOpClipTest, kOpSirTest,
  kOpCount
};
std::atomic<uint64_t> g_ops[kOpCount];
thread_local uint64_t t_ops[kOpCount];
inline void op_count(int k) { t_ops[k]++; }
// Adds this thread's counts to the totals (end of a tracing worker).
inline void op_flush() {
  for (int k = 0; k < kOpCount; k++) {
    g_ops[k].fetch_add(t_ops[k], std::memory_order_relaxed);
    t_ops[k] = 0;
  }
}

// realCubicSolution (src/tools.cpp:350-391)
double real_cubic(double b, double c, double d) {
  double p = -(1.0 / 3.0) * b * b + c;
  double q = (2. / 27.) * b * b * b - (1. / 3.) * b * c + d;
  double D3p = (1. / 27.) * p * p * p;
  double D3 = D3p + 0.25 * q * q;
  if (fabs(c) < b * b * 1.E-6 && fabs(d) < fabs(b) * 1.E-6) {
    op_count(kOpCubicSmallC);
    return c / b - b - d / (b * b);
  } else if (fabs(d / c) < 4.E-4) {
    double ratio = d / c;
    if (D3 <= 0.) {
      op_count(kOpCubicRatioSqrt);
      return 0.5 * (ratio - b + sqrt((b - ratio) * (b - ratio) - 4. * (c - ratio * (b - ratio))));
    } else {
      op_count(kOpCubicRatioEps);
      double eps = -ratio * ratio * (b - ratio) / (3. * ratio * ratio - 2. * b * ratio + c);
      return eps - ratio;
    }
  } else {
    if (D3 >= 0.) {
      op_count(kOpCubicCbrt);
      double radD3 = sqrt(D3);
      double A = cbrt(radD3 - 0.5 * q);
      double psu3A = cbrt(radD3 + 0.5 * q);
      return A - psu3A - (1. / 3.) * b;
    } else {
      op_count(kOpCubicAcos);
      double Aarg = acos(-0.5 * q / sqrt(-D3p));
      return 2. * sqrt(-(1. / 3.) * p) * cos((1. / 3.) * Aarg) - (1. / 3.) * b;
    }
  }
}

// quarticEqSolutions (src/tools.cpp:525-639)
void quartic(double roots[4], double b, double c, double d, double e, int* num_sol) {
  double b_2 = 0.5 * b;
  double b_4 = 0.25 * b;
  double p = c - 1.5 * (b_2 * b_2);
  double q = d + b_2 * (b_2 * b_2 - c);
  double r = e + b_4 * (b_4 * (c - 3.0 * b_4 * b_4) - d);
  double f = p * p - 4. * r;
  double delta = 4. * f * (4. * r * (p * p) - p * (q * q) - 16. * (r * r)) + (q * q) * (128. * p * r - 27. * (q * q));
  bool change_variant = false;
  if (e != 0. && (fabs(p) > 3.E+3 || fabs(r) > 3.E+3 || fabs(q) > 3.E+3 || fabs(delta) > 1.E+14)) {
    op_count(kOpQuarticRecip);
    double dsu2e = 0.5 * d / e;
    change_variant = true;
    p = -1.5 * dsu2e * dsu2e + c / e;
    q = dsu2e * (dsu2e * dsu2e - c / e) + b / e;
    r = dsu2e * (-3. / 16. * (dsu2e * dsu2e * dsu2e) + 0.25 * dsu2e * (c / e) - 0.5 * b / e) + 1. / e;
    f = p * p - 4. * r;
    delta = 4. * f * (4. * r * (p * p) - p * (q * q) - 16. * (r * r)) + (q * q) * (128. * p * r - 27. * (q * q));
  }
  if (delta < 0. || (delta == 0. && (p >= 0. || f < 0.)))
    *num_sol = 2;
  else if ((p < 0. && f > 0.) || (delta == 0. && p == 0. && r == 0.))
    *num_sol = 4;
  else {
    op_count(kOpQuarticNone);
    *num_sol = 0;
    return;
  }
  op_count(*num_sol == 2 ? kOpQuartic2 : kOpQuartic4);
  double m = real_cubic(p, 0.25 * (p * p) - r, (-0.125) * (q * q));
  if (m <= 0) {
    op_count(kOpQuarticM0);
    *num_sol = 0;
    return;
  }
  double coeff;
  if (*num_sol >= 2) {
    double sol_delta_min, sol_delta_max, p1, p2, p3;
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
    if (*num_sol == 4) {
      if (m < 1.E-14)
        sol_delta_min = -p1 - p2 - p3;
      else
        sol_delta_min = p1 - p2;
      roots[2] = 0.5 * (((q >= 0.) ? coeff : -coeff) - sqrt(sol_delta_min));
      roots[3] = 0.5 * (((q >= 0.) ? coeff : -coeff) + sqrt(sol_delta_min));
    }
  }
  if (change_variant) {
    for (int i = 0; i < *num_sol; i++) roots[i] = 1. / (roots[i] - 0.25 * d / e);
  } else {
    for (int i = 0; i < *num_sol; i++) roots[i] -= 0.25 * b;
  }
}

// rayTorus with the analytical solver (src/tools.cpp:907-1098)
bool ray_torus(const double* invrot, const double* tc, const double* sc, double probe, double major,
               double radius, int vc, const double* orig, const double* dir, double t[4], int& numInt) {
  double roots[4], pp[3], temp[3], orig1[3];
  double ray_dir = dir[vc];
  orig1[0] = orig[0]; orig1[1] = orig[1]; orig1[2] = orig[2];
  orig1[vc] += t[0] * ray_dir;
  temp[0] = orig1[0] - tc[0]; temp[1] = orig1[1] - tc[1]; temp[2] = orig1[2] - tc[2];
  for (int i = 0; i < 3; i++) pp[i] = invrot[3 * i + 0] * temp[0] + invrot[3 * i + 1] * temp[1] + invrot[3 * i + 2] * temp[2];
  double r2 = probe * probe;
  double R2 = major * major;
  double pd = pp[0] * invrot[0 * 3 + vc] + pp[1] * invrot[1 * 3 + vc] + pp[2] * invrot[2 * 3 + vc];
  double p2 = pp[0] * pp[0] + pp[1] * pp[1] + pp[2] * pp[2];
  double coeff = p2 - r2 - R2;
  double B = 4 * pd;
  double C = 2 * coeff + 4 * pd * pd + 4 * R2 * invrot[2 * 3 + vc] * invrot[2 * 3 + vc];
  double D = 4 * pd * coeff + 8 * R2 * pp[2] * invrot[2 * 3 + vc];
  double E = coeff * coeff - 4 * R2 * (r2 - pp[2] * pp[2]);
  int numroots;
  quartic(roots, B, C, D, E, &numroots);
  if (numroots == 0) return false;
  double t0 = t[0];
  numInt = 0;
  for (int i = 0; i < numroots; i++) {
    if (roots[i] < 0) continue;
    op_count(kOpRootTest);
    double point[3] = {orig1[0], orig1[1], orig1[2]};
    point[vc] += roots[i];
    double dd = (sc[0] - point[0]) * (sc[0] - point[0]) + (sc[1] - point[1]) * (sc[1] - point[1]) +
                (sc[2] - point[2]) * (sc[2] - point[2]);
    if (dd < radius * radius) {
      op_count(kOpRootIn);
      t[numInt++] = t0 + roots[i] / ray_dir;
    }
  }
  return numInt != 0;
}

inline double dist2(const double* a, const double* b) {
  return (a[0] - b[0]) * (a[0] - b[0]) + (a[1] - b[1]) * (a[1] - b[1]) + (a[2] - b[2]) * (a[2] - b[2]);
}
inline double plane_test(const double* w, const double* p) { return (w[0] * p[0] + w[1] * p[1] + w[2] * p[2]) + w[3]; }

// SkinSurface::isFeasible (src/SkinSurface.cpp:4374-4448): a point is outside the cell when a plane
// test is positive (the planes of Del0 cells are stored negated, which turns the reference's
// "val < 0" test of those cells into the same "> 0" test exactly).
bool feasible_skin(const Patches& P, int64_t it, const double* p) {
  const int32_t* ir = P.i32 + NS_PATCH_I32 * it;
  const double* pool = P.pool + 4 * (int64_t)ir[1];
  for (int q = 0; q < ir[2]; q++)
    if (plane_test(pool + 4 * q, p) > 0) return false;
  return true;
}

// rayQuadricIntersectionX/Y/Z with a unit direction along axis vc (src/SkinSurface.cpp:4632-4709);
// Q in the reference's coding q11, q22, q33, q44, q12, q23, q34, q13, q24, q14.
bool ray_quadric(const double* Q, int vc, const double* o, double t[2]) {
  double q44 = Q[3], q33 = Q[2], q22 = Q[1], q11 = Q[0], q34 = Q[6], q24 = Q[8], q23 = Q[5], q14 = Q[9], q13 = Q[7],
         q12 = Q[4];
  double a, b;
  if (vc == 0) {
    a = q11;
    if (a == 0) return false;
    b = q14 + o[2] * q13 + o[1] * q12 + o[0] * q11;
  } else if (vc == 1) {
    a = q22;
    if (a == 0) return false;
    b = q24 + o[2] * q23 + o[1] * q22 + o[0] * q12;
  } else {
    a = q33;
    if (a == 0) return false;
    b = q34 + o[2] * q33 + o[1] * q23 + o[0] * q13;
  }
  double c = q44 + (o[2] + o[2]) * q34 + (o[2] * o[2]) * q33 + (o[1] + o[1]) * q24 + (2 * o[1] * o[2]) * q23 +
             (o[1] * o[1]) * q22 + (o[0] + o[0]) * q14 + (2 * o[0] * o[2]) * q13 + (2 * o[0] * o[1]) * q12 +
             (o[0] * o[0]) * q11;
  double delta = b * b - a * c;
  if (delta < 0) return false;
  delta = sqrt(delta);
  t[0] = (-b - delta) / a;
  t[1] = (-b + delta) / a;
  return true;
}

// MeshSurface::intersect_triangle, non-culling branch (src/MeshSurface.cpp:1487-1553), EPS 1e-5.
bool ray_triangle(const double* orig, const double* dir, const double* v0, const double* v1, const double* v2,
                  double* t) {
  const double EPS = 1e-5;
  double edge1[3], edge2[3], tvec[3], pvec[3], qvec[3];
  for (int k = 0; k < 3; k++) {
    edge1[k] = v1[k] - v0[k];
    edge2[k] = v2[k] - v0[k];
  }
  pvec[0] = dir[1] * edge2[2] - dir[2] * edge2[1];
  pvec[1] = dir[2] * edge2[0] - dir[0] * edge2[2];
  pvec[2] = dir[0] * edge2[1] - dir[1] * edge2[0];
  double det = edge1[0] * pvec[0] + edge1[1] * pvec[1] + edge1[2] * pvec[2];
  if (det > -EPS && det < EPS) return false;
  double inv_det = 1.0 / det;
  for (int k = 0; k < 3; k++) tvec[k] = orig[k] - v0[k];
  double u = (tvec[0] * pvec[0] + tvec[1] * pvec[1] + tvec[2] * pvec[2]) * inv_det;
  if (u < 0.0 || u > 1.0) return false;
  qvec[0] = tvec[1] * edge1[2] - tvec[2] * edge1[1];
  qvec[1] = tvec[2] * edge1[0] - tvec[0] * edge1[2];
  qvec[2] = tvec[0] * edge1[1] - tvec[1] * edge1[0];
  double v = (dir[0] * qvec[0] + dir[1] * qvec[1] + dir[2] * qvec[2]) * inv_det;
  if (v < 0.0 || u + v > 1.0) return false;
  *t = (edge2[0] * qvec[0] + edge2[1] * qvec[1] + edge2[2] * qvec[2]) * inv_det;
  return true;
}

// isFeasible (src/ConnollySurface.cpp:4769-5019) over the patch-set encoding.
bool feasible(const Patches& P, int64_t it, const double* p) {
  const int32_t* ir = P.i32 + NS_PATCH_I32 * it;
  const double* fr = P.f64 + NS_PATCH_F64 * it;
  int kind = ir[0];
  const double* pool = P.pool + 4 * (int64_t)ir[1];
  const int8_t* flg = P.flag + ir[1];
  int cnt = ir[2];
  op_count(kOpFeasTest);
  if (kind == NS_FACE_REG || kind == NS_FACE_SING) {
    for (int q = 0; q < cnt; q++) {
      op_count(kOpPlaneTest);
      if (plane_test(pool + 4 * q, p) > 0) return false;
    }
    return true;
  }
  if (kind == NS_POINT) {
    for (int q = 0; q < cnt; q++) {
      op_count(kOpClipTest);
      double dd = dist2(pool + 4 * q, p);
      dd -= pool[4 * q + 3];
      if (dd < 0) return false;
    }
    return true;
  }
  double r = fr[8];
  if (r >= 0.) {
    op_count(kOpSirTest);
    double dd = dist2(fr + 4, p);
    if (dd < r * r) return false;
  }
  if (cnt == 0) return true;
  for (int q = 0; q + 1 < cnt; q += 2) {
    op_count(kOpPlaneTest);
    double t0 = plane_test(pool + 4 * q, p);
    if (flg[q]) {
      if (t0 > 0) continue;
      op_count(kOpPlaneTest);
      if (plane_test(pool + 4 * (q + 1), p) > 0) continue;
      return true;
    } else {
      if (t0 <= 0) return true;
      op_count(kOpPlaneTest);
      if (plane_test(pool + 4 * (q + 1), p) <= 0) return true;
    }
  }
  return false;
}

struct Hit {
  int64_t pixel;
  double t;
  int32_t patch;
};

struct Oracle {
  NsGrid g;
  Patches P;
  int flags;
  double cav_vol;
  int nthreads;
  int panels[2];
  int numPanels;
  int64_t NMAX;
  // products
  std::vector<int64_t> pix_off;  // pixel -> first hit
  std::vector<double> pix_t;
  std::vector<int32_t> pix_pid;  // patch of every hit
  std::vector<int32_t> status;
  std::vector<uint32_t> bits;
  // epsilon map ((k*ny + j)*nx + i)*3 + axis and ideb map (flag 32); boundary grid points and their
  // projection (flag 64)
  std::vector<int32_t> eps;
  std::vector<uint8_t> ideb;
  std::vector<int32_t> ibgp, bgp_type, bgp_flag;
  std::vector<double> scspos, scsnor;
  int aux_max_dim = 50;
  bool eps_on() const { return (flags & 32) != 0; }
  double volPanel[3] = {0, 0, 0};
  int flagsum = 0;
  double volume = 0;
  std::vector<double> vert;        // analytic vertices before assembly: x y z
  std::vector<int32_t> vert_edge;  // ix iy iz dir
  std::vector<int32_t> vert_pid;   // patch of every analytic vertex
  std::vector<int32_t> vpid;       // patch of every assembled analytic vertex
  std::vector<double> normals;     // vertex normals (Compute_Vertex_Normals)
  std::vector<double> vlist;       // assembled vertex list
  std::vector<int32_t> vkey;       // edge of every assembled vertex (ix iy iz dir)
  std::vector<int32_t> tris;
  double area = 0;
  int ncav = 0;
  std::vector<double> cav_size;
  std::vector<int32_t> cav_filled;
  std::vector<int64_t> ray_hits;  // per pixel id: number of hits (for tests)
  int64_t n_hits = 0;
  // optional sample: only rays whose second pixel index n lies in [slab_lo*na, slab_hi*na)
  double slab_lo = 0.0, slab_hi = 1.0;
  int64_t n_lo(int64_t na) const { return (int64_t)(slab_lo * na); }
  int64_t n_hi(int64_t na) const { return slab_hi >= 1.0 ? na : (int64_t)(slab_hi * na); }
  int64_t rays_cast = 0;

  double X(int64_t i) const { return ns_coord(g.xmin, g.side, i); }
  double Y(int64_t i) const { return ns_coord(g.ymin, g.side, i); }
  double Z(int64_t i) const { return ns_coord(g.zmin, g.side, i); }
  double coord(int d, int64_t i) const { return d == 0 ? X(i) : (d == 1 ? Y(i) : Z(i)); }
  int64_t Nd(int d) const { return d == 0 ? g.nx : (d == 1 ? g.ny : g.nz); }
  double mind(int d) const { return d == 0 ? g.xmin : (d == 1 ? g.ymin : g.zmin); }
  double maxd(int d) const { return d == 0 ? g.xmax : (d == 1 ? g.ymax : g.zmax); }

  // One skin cell (SkinSurface::getPatchIntersectionData, src/SkinSurface.cpp:3422-3760): the box
  // of the cell culls the grid and the pixels, the atom disc culls Del0 pixels, rays of unit
  // direction start at min + delta, hits are stored as t / (max - min).
  void trace_skin(int64_t it, std::vector<Hit>& out) const {
    const int32_t* ir = P.i32 + NS_PATCH_I32 * it;
    const double* fr = P.f64 + NS_PATCH_F64 * it;
    const int kind = ir[0];
    const double* down = fr + NS_SKIN_LO;
    const double* up = fr + NS_SKIN_HI;
    const double* Q = fr + NS_SKIN_Q;
    const double dacc = NS_DELTA;
    for (int d = 0; d < 3; d++) if (down[d] > maxd(d) + NS_EPS_INT) return;
    for (int d = 0; d < 3; d++) if (up[d] < mind(d) - (g.hside - dacc + NS_EPS_INT)) return;
    int64_t i_start[3], i_end[3];
    for (int d = 0; d < 3; d++) {
      i_start[d] = (int64_t)rintp(fmax(0., (down[d] - mind(d))) * g.scale);
      i_end[d] = (int64_t)rintp(fmax(0., up[d] - mind(d)) * g.scale);
      if (i_end[d] >= Nd(d)) i_end[d] = Nd(d) - 1;
    }
    int64_t pixels[3] = {1 + i_end[0] - i_start[0], 1 + i_end[1] - i_start[1], 1 + i_end[2] - i_start[2]};
    for (int phase = 0; phase < 2; phase++) {
      if (panels[phase] == 0) continue;
      double delta = (phase == 0) ? 0. : dacc - g.hside;
      for (int panel = 0; panel < panels[phase]; panel++) {
        int fd, ld, vc;
        if (panel == 0) { fd = 1; ld = 2; vc = 0; }
        else if (panel == 1) { fd = 0; ld = 1; vc = 2; }
        else { fd = 0; ld = 2; vc = 1; }
        double pa[3];
        pa[vc] = mind(vc) + delta;
        const double ray_dir = maxd(vc) - mind(vc);
        int64_t npix = pixels[fd] * pixels[ld];
        for (int64_t rp = 0; rp < npix; rp++) {
          int64_t n = rp / pixels[fd];
          int64_t m = rp - n * pixels[fd];
          n += i_start[ld];
          m += i_start[fd];
          if (n < n_lo(Nd(ld)) || n >= n_hi(Nd(ld))) continue;
          pa[fd] = coord(fd, m) + delta;
          if (pa[fd] < down[fd] || pa[fd] > up[fd]) continue;
          pa[ld] = coord(ld, n) + delta;
          if (pa[ld] < down[ld] || pa[ld] > up[ld]) continue;
          if (kind == NS_SKIN_POINT) {
            double dx = fr[fd] - pa[fd];
            double dy = fr[ld] - pa[ld];
            if (dx * dx + dy * dy > fr[3] * fr[3]) continue;
          }
          if (kind == NS_MESH_TRI) {
            // the mesh caster's ray runs from the first to the last node (+ delta) of the axis
            double dir[3] = {0., 0., 0.};
            dir[vc] = (coord(vc, Nd(vc) - 1) + delta) - (coord(vc, 0) + delta);
            double o[3] = {pa[0], pa[1], pa[2]};
            o[vc] = coord(vc, 0) + delta;
            double tt;
            if (ray_triangle(o, dir, fr, fr + 3, fr + 6, &tt)) {
              int64_t pid = (n * NMAX + m) * numPanels + (panels[0] * phase + panel);
              out.push_back({pid, tt, (int32_t)it});
            }
            continue;
          }
          double t[2];
          if (!ray_quadric(Q, vc, pa, t)) continue;
          for (int i = 0; i < 2; i++) {
            double ip[3] = {pa[0], pa[1], pa[2]};
            ip[vc] += t[i];
            if (!feasible_skin(P, it, ip)) continue;
            int64_t pid = (n * NMAX + m) * numPanels + (panels[0] * phase + panel);
            out.push_back({pid, t[i] / ray_dir, (int32_t)it});
          }
        }
      }
    }
  }

  void trace_patch(int64_t it, std::vector<Hit>& out) const {
    const int32_t* ir = P.i32 + NS_PATCH_I32 * it;
    const double* fr = P.f64 + NS_PATCH_F64 * it;
    int kind = ir[0];
    if (ns_has_box(kind)) {
      trace_skin(it, out);
      return;
    }
    const double* sc = fr;
    double radius = fr[3];
    bool doTorus = (kind == NS_EDGE_REG || kind == NS_EDGE_SING);
    double down[3] = {sc[0] - radius, sc[1] - radius, sc[2] - radius};
    double up[3] = {sc[0] + radius, sc[1] + radius, sc[2] + radius};
    const double dacc = NS_DELTA;
    // CELL_CULLING
    for (int d = 0; d < 3; d++) if (down[d] > maxd(d) + NS_EPS_INT) return;
    for (int d = 0; d < 3; d++) if (up[d] < mind(d) - (g.hside - dacc + NS_EPS_INT)) return;
    int64_t i_start[3], i_end[3];
    for (int d = 0; d < 3; d++) {
      i_start[d] = (int64_t)rintp(fmax(0., down[d] - mind(d)) * g.scale);
      i_end[d] = (int64_t)rintp(fmax(0., up[d] - mind(d)) * g.scale);
      if (i_end[d] >= Nd(d)) i_end[d] = Nd(d) - 1;
    }
    int64_t pixels[3] = {1 + i_end[0] - i_start[0], 1 + i_end[1] - i_start[1], 1 + i_end[2] - i_start[2]};
    for (int phase = 0; phase < 2; phase++) {
      if (panels[phase] == 0) continue;
      double delta = (phase == 0) ? 0. : dacc - g.hside;
      for (int panel = 0; panel < panels[phase]; panel++) {
        int fd, ld, vc;
        if (panel == 0) { fd = 1; ld = 2; vc = 0; }
        else if (panel == 1) { fd = 0; ld = 1; vc = 2; }
        else { fd = 0; ld = 2; vc = 1; }
        double pa[3], dir[3] = {0., 0., 0.};
        pa[vc] = coord(vc, 0) + delta;
        double ray_dir = coord(vc, Nd(vc) - 1) - coord(vc, 0);
        dir[vc] = ray_dir;
        int64_t npix = pixels[fd] * pixels[ld];
        for (int64_t rp = 0; rp < npix; rp++) {
          int64_t n = rp / pixels[fd];
          int64_t m = rp - n * pixels[fd];
          n += i_start[ld];
          m += i_start[fd];
          if (n < n_lo(Nd(ld)) || n >= n_hi(Nd(ld))) continue;
          pa[fd] = coord(fd, m) + delta;
          if (pa[fd] < down[fd] || pa[fd] > up[fd]) continue;
          pa[ld] = coord(ld, n) + delta;
          if (pa[ld] < down[ld] || pa[ld] > up[ld]) continue;
          double dx = sc[fd] - pa[fd];
          double dy = sc[ld] - pa[ld];
          if (dx * dx + dy * dy > radius * radius) continue;
          double t[4];
          op_count(doTorus ? kOpTorusCand : kOpSphereCand);
          if (!ray_sphere(pa, dir, sc, radius, &t[0], &t[1])) {
            op_count(doTorus ? kOpTorusNoSphere : kOpSphereMiss);
            continue;
          }
          int numInt = 0;
          if (!doTorus) numInt = 2;
          else ray_torus(fr + 9, fr + 4, sc, P.probe, fr[7], radius, vc, pa, dir, t, numInt);
          for (int i = 0; i < numInt; i++) {
            double ip[3] = {pa[0], pa[1], pa[2]};
            ip[vc] += t[i] * ray_dir;
            if (!feasible(P, it, ip)) continue;
            int64_t pid = (n * NMAX + m) * numPanels + (panels[0] * phase + panel);
            out.push_back({pid, t[i], (int32_t)it});
          }
        }
      }
    }
  }

  // Runs f(lo, hi) over [a, b) split into contiguous blocks, one per thread.
  template <class F>
  void parallel_rows(int64_t a, int64_t b, F&& f) const {
    const int nt = std::max(1, nthreads);
    if (nt <= 1 || b - a < 2 * nt) {
      f(a, b);
      return;
    }
    std::vector<std::thread> th;
    const int64_t step = (b - a + nt - 1) / nt;
    for (int t = 0; t < nt; t++) {
      const int64_t lo = a + t * step, hi = std::min(b, lo + step);
      if (lo < hi) th.emplace_back([&f, lo, hi] { f(lo, hi); });
    }
    for (auto& x : th) x.join();
  }

  void trace() {
    std::vector<std::vector<Hit>> per(std::max(1, nthreads));
    auto work = [&](int tid) {
      for (int64_t it = tid; it < P.n; it += std::max(1, nthreads)) trace_patch(it, per[tid]);
      op_flush();
    };
    if (nthreads <= 1) work(0);
    else {
      std::vector<std::thread> th;
      for (int t = 0; t < nthreads; t++) th.emplace_back(work, t);
      for (auto& x : th) x.join();
    }
    int64_t npix = NMAX * NMAX * numPanels;
    pix_off.assign(npix + 1, 0);
    for (auto& v : per)
      for (auto& h : v) pix_off[h.pixel + 1]++;
    for (int64_t i = 0; i < npix; i++) pix_off[i + 1] += pix_off[i];
    n_hits = pix_off[npix];
    pix_t.resize(n_hits);
    pix_pid.resize(n_hits);
    std::vector<int64_t> fill(pix_off.begin(), pix_off.end() - 1);
    for (auto& v : per)
      for (auto& h : v) {
        pix_pid[fill[h.pixel]] = h.patch;
        pix_t[fill[h.pixel]++] = h.t;
      }
    // per pixel by t (the patch of each hit follows it; equal t keep their patch order)
    std::vector<std::pair<double, int32_t>> tmp;
    for (int64_t i = 0; i < npix; i++) {
      const int64_t a = pix_off[i], b = pix_off[i + 1];
      if (b - a < 2) continue;
      tmp.clear();
      for (int64_t q = a; q < b; q++) tmp.push_back({pix_t[q], pix_pid[q]});
      std::stable_sort(tmp.begin(), tmp.end(), [](const std::pair<double, int32_t>& x,
                                                  const std::pair<double, int32_t>& y) { return x.first < y.first; });
      for (int64_t q = a; q < b; q++) {
        pix_t[q] = tmp[q - a].first;
        pix_pid[q] = tmp[q - a].second;
      }
    }
  }

  // 32x compressed bit grid accessors (src/tools.h:1364-1413); bit = 1 means outside.
  bool rbit(int64_t i, int64_t j, int64_t k) const {
    int64_t f = (k * g.ny + j) * g.nx + i;
    return (bits[f >> 5] >> (f & 31)) & 1u;
  }
  void clear_bit(int64_t i, int64_t j, int64_t k) {
    int64_t f = (k * g.ny + j) * g.nx + i;
    if ((f >> 5) < (int64_t)bits.size()) bits[f >> 5] &= ~(1u << (f & 31));
  }

  // Pairs of a ray's sorted hits under NEW_INTERSECTION_FILTERING (src/Surface.cpp:5262-5282).
  void pairs_of(int64_t id, std::vector<std::pair<int64_t, int64_t>>& pr) const {
    pr.clear();
    int64_t s = pix_off[id], vsize = pix_off[id + 1] - s;
    if (vsize == 0 || (vsize & 1)) return;
    for (int64_t i = 0; i < vsize; i += 2)
      if (fabs(pix_t[s + i + 1] - pix_t[s + i]) >= NS_EPS_INT) pr.push_back({s + i, s + i + 1});
  }

  void fill_panel(int panel) {
    int64_t na, nb;
    if (panel == 0) { na = g.nz; nb = g.ny; }
    else if (panel == 1) { na = g.ny; nb = g.nx; }
    else { na = g.nz; nb = g.nx; }
    std::vector<std::pair<int64_t, int64_t>> pr;
    // phase 0 of panels 1 and 2: the epsilon map's node rays along z and y (src/Surface.cpp:6698-6898)
    if (eps_on() && panel > 0) {
      flagsum++;
      const int vc = panel == 1 ? 2 : 1;
      const int64_t n0 = n_lo(na), n1 = n_hi(na);
      rays_cast += (n1 - n0) * nb;
      double pa[3], pb[3];
      pa[vc] = coord(vc, 0);
      pb[vc] = coord(vc, Nd(vc) - 1);
      for (int64_t n = n0; n < n1; n++) {
        if (panel == 1) pa[1] = Y(n);
        else pa[2] = Z(n);
        for (int64_t m = 0; m < nb; m++) {
          int64_t id = (n * NMAX + m) * numPanels + panel;
          pairs_of(id, pr);
          if (pr.empty()) continue;
          pa[0] = X(m);
          double dir = pb[vc] - pa[vc];
          double lvi = 0.0;
          for (auto& q : pr) {
            double lim1 = pa[vc] + dir * pix_t[q.first];
            double lim2 = pa[vc] + dir * pix_t[q.second];
            lvi += lim2 - lim1;
            int64_t c1 = (int64_t)rintp((lim1 - mind(vc)) * g.scale);
            int64_t c2 = (int64_t)rintp((lim2 - mind(vc)) * g.scale);
            c1 = c1 < 0 ? 0 : (c1 >= Nd(vc) ? Nd(vc) - 1 : c1);
            c2 = c2 < 0 ? 0 : (c2 >= Nd(vc) ? Nd(vc) - 1 : c2);
            if (c2 < c1) continue;
            for (int64_t c = c1; c < c2; c++) {
              if (coord(vc, c) <= lim2 - g.hside) {
                if (panel == 1) eps[3 * ((c * g.ny + n) * g.nx + m) + 2] = NS_EPS_INSIDE;
                else eps[3 * ((n * g.ny + c) * g.nx + m) + 1] = NS_EPS_INSIDE;
              }
            }
          }
          volPanel[panel] += lvi;
        }
      }
    }
    // phase 0: status map along x (only panel 0 when the status map is built)
    if (panels[0] > 0 && panel == 0) {
      flagsum++;
      const int64_t n0 = n_lo(na), n1 = n_hi(na);
      rays_cast += (n1 - n0) * nb;
      // rows are independent (each writes its own status row); the interval sums are kept per
      // ray and added afterwards in the reference's serial ray order
      std::vector<double> lv((size_t)(n1 - n0) * nb, 0.0);
      auto rows = [&](int64_t nn0, int64_t nn1) {
        std::vector<std::pair<int64_t, int64_t>> prl;
        double pa[3], pb[3];
        pa[0] = X(0); pb[0] = X(g.nx - 1);
        for (int64_t n = nn0; n < nn1; n++) {
          pa[2] = Z(n);
          for (int64_t m = 0; m < nb; m++) {
            int64_t id = (n * NMAX + m) * numPanels + panel;
            pairs_of(id, prl);
            if (prl.empty()) continue;
            pa[1] = Y(m);
            double dir = pb[0] - pa[0];
            double lvi = 0.0;
            for (auto& q : prl) {
              double lim1 = pa[0] + dir * pix_t[q.first];
              double lim2 = pa[0] + dir * pix_t[q.second];
              lvi += lim2 - lim1;
              int64_t i1 = (int64_t)rintp((lim1 - g.xmin) * g.scale);
              int64_t i2 = (int64_t)rintp((lim2 - g.xmin) * g.scale);
              i1 = i1 < 0 ? 0 : (i1 >= g.nx ? g.nx - 1 : i1);
              i2 = i2 < 0 ? 0 : (i2 >= g.nx ? g.nx - 1 : i2);
              if (i2 < i1) continue;
              for (int64_t ix = i1; ix <= i2; ix++) {
                double xx = X(ix);
                const int64_t f = (n * g.ny + m) * g.nx + ix;
                if (eps_on() && xx <= lim2 - g.hside) eps[3 * f] = NS_EPS_INSIDE;
                if (xx <= lim2 && xx >= lim1) {
                  status[f] = NS_STATUS_INSIDE;
                  if (eps_on()) ideb[f] = 0;
                }
              }
            }
            lv[(size_t)(n - n0) * nb + m] = lvi;
          }
        }
      };
      parallel_rows(n0, n1, rows);
      for (double v : lv) volPanel[panel] += v;
    }
    if (!(flags & 2)) return;  // accurate triangulation rays
    flagsum++;
    double delta = NS_DELTA - g.hside;
    int vc = panel == 0 ? 0 : (panel == 1 ? 2 : 1);
    double pa[3], pb[3];
    pa[vc] = coord(vc, 0) + delta;
    pb[vc] = coord(vc, Nd(vc) - 1) + delta;
    rays_cast += (n_hi(na) - n_lo(na)) * nb;
    for (int64_t n = n_lo(na); n < n_hi(na); n++) {
      if (panel == 0) pa[2] = Z(n) + delta;
      else if (panel == 1) pa[1] = Y(n) + delta;
      else pa[2] = Z(n) + delta;
      for (int64_t m = 0; m < nb; m++) {
        int64_t id = (n * NMAX + m) * numPanels + (panels[0] + panel);
        pairs_of(id, pr);
        if (pr.empty()) continue;
        if (panel == 0) pa[1] = Y(m) + delta;
        else pa[0] = X(m) + delta;
        double dir = pb[vc] - pa[vc];
        double lvi = 0.0;
        for (auto& q : pr) {
          double lim1 = pa[vc] + dir * pix_t[q.first];
          double lim2 = pa[vc] + dir * pix_t[q.second];
          lvi += lim2 - lim1;
          int64_t a = (int64_t)rintp((lim1 - mind(vc)) * g.scale);
          int64_t b = (int64_t)rintp((lim2 - mind(vc)) * g.scale);
          if (b <= a) continue;
          double v1[3] = {pa[0], pa[1], pa[2]}, v2[3] = {pa[0], pa[1], pa[2]};
          v1[vc] = lim1;
          v2[vc] = lim2;
          int32_t e1[4], e2[4];
          if (panel == 0) {
            for (int64_t i = a + 1; i <= b; i++) clear_bit(i, m, n);
            int32_t t1[4] = {(int32_t)a, (int32_t)m, (int32_t)n, NS_X_DIR};
            int32_t t2[4] = {(int32_t)b, (int32_t)m, (int32_t)n, NS_X_DIR};
            memcpy(e1, t1, sizeof e1); memcpy(e2, t2, sizeof e2);
          } else if (panel == 1) {
            for (int64_t k = a + 1; k <= b; k++) clear_bit(m, n, k);
            int32_t t1[4] = {(int32_t)m, (int32_t)n, (int32_t)a, NS_Z_DIR};
            int32_t t2[4] = {(int32_t)m, (int32_t)n, (int32_t)b, NS_Z_DIR};
            memcpy(e1, t1, sizeof e1); memcpy(e2, t2, sizeof e2);
          } else {
            for (int64_t j = a + 1; j <= b; j++) clear_bit(m, j, n);
            int32_t t1[4] = {(int32_t)m, (int32_t)a, (int32_t)n, NS_Y_DIR};
            int32_t t2[4] = {(int32_t)m, (int32_t)b, (int32_t)n, NS_Y_DIR};
            memcpy(e1, t1, sizeof e1); memcpy(e2, t2, sizeof e2);
          }
          if (flags & 8) {  // analytic vertices are kept only for the triangulation
            vert.insert(vert.end(), v1, v1 + 3);
            vert_edge.insert(vert_edge.end(), e1, e1 + 4);
            vert_pid.push_back(pix_pid[q.first]);
            vert.insert(vert.end(), v2, v2 + 3);
            vert_edge.insert(vert_edge.end(), e2, e2 + 4);
            vert_pid.push_back(pix_pid[q.second]);
          }
        }
        volPanel[panel] += lvi;
      }
    }
  }

  // Flood fill of one 6-connected region of value idold with idnew, in the scanline order of
  // floodFillWithBilevelStatusMap2; returns the visited nodes in fill order.
  void flood(int64_t si, int64_t sj, int64_t sk, int idold, int idnew, std::vector<int64_t>* nodes) {
    auto S = [&](int64_t i, int64_t j, int64_t k) -> int32_t& { return status[(k * g.ny + j) * g.nx + i]; };
    std::deque<std::array<int64_t, 3>> zq;
    zq.push_back({si, sj, sk});
    while (!zq.empty()) {
      auto tr = zq.front();
      zq.pop_front();
      int64_t i = tr[0], j = tr[1], k = tr[2];
      if (S(i, j, k) == idnew) continue;
      std::stack<std::pair<int64_t, int64_t>> xy;
      xy.push({i, j});
      while (!xy.empty()) {
        auto d = xy.top();
        xy.pop();
        i = d.first;
        j = d.second;
        bool spanLeft = false, spanRight = false;
        int64_t i1 = i;
        while (i1 >= 0 && S(i1, j, k) == idold) i1--;
        i1++;
        while (i1 < g.nx) {
          if (S(i1, j, k) != idold) break;
          S(i1, j, k) = idnew;
          if (nodes) nodes->push_back((k * g.ny + j) * g.nx + i1);
          if (k < g.nz - 1 && S(i1, j, k + 1) == idold) zq.push_back({i1, j, k + 1});
          if (k > 0 && S(i1, j, k - 1) == idold) zq.push_back({i1, j, k - 1});
          if (!spanLeft && j > 0) {
            if (S(i1, j - 1, k) == idold) { xy.push({i1, j - 1}); spanLeft = true; }
          } else if (spanLeft && j > 0) {
            if (S(i1, j - 1, k) != idold) spanLeft = false;
          }
          if (!spanRight && j < g.ny - 1) {
            if (S(i1, j + 1, k) == idold) { xy.push({i1, j + 1}); spanRight = true; }
          } else if (spanRight && j < g.ny - 1) {
            if (S(i1, j + 1, k) != idold) spanRight = false;
          }
          i1++;
        }
      }
    }
  }

  void cavities() {
    int id = NS_STATUS_TEMPORARY_OUT;
    int times = 0;
    std::vector<std::vector<int64_t>> cav_nodes;
    // search cursors: the scan restarts from the beginning in the reference; since nodes only
    // ever leave the TEMPORARY_OUT state, resuming from the last hit position is equivalent.
    int64_t cur_up = 0, cur_dn = 0;
    const int64_t plane = g.nx * g.ny;
    const int64_t total = plane * g.nz;
    while (true) {
      int64_t found = -1;
      if (times % 2 == 0) {
        for (int64_t s = cur_up; s < total; s++)
          if (status[s] == NS_STATUS_TEMPORARY_OUT) { found = s; break; }
        if (found >= 0) cur_up = found;
      } else {
        for (int64_t s = cur_dn; s < total; s++) {
          int64_t k = g.nz - 1 - s / plane;
          int64_t f = k * plane + (s % plane);
          if (status[f] == NS_STATUS_TEMPORARY_OUT) { found = f; cur_dn = s; break; }
        }
      }
      times++;
      if (found < 0) break;
      id++;
      int64_t k = found / plane, j = (found % plane) / g.nx, i = found % g.nx;
      std::vector<int64_t> nodes;
      flood(i, j, k, NS_STATUS_TEMPORARY_OUT, id, id >= NS_STATUS_FIRST_CAV ? &nodes : nullptr);
      if (id >= NS_STATUS_FIRST_CAV) cav_nodes.push_back(std::move(nodes));
    }
    ncav = id - NS_STATUS_OUT;
    double cubeVol = g.side * g.side * g.side;
    cav_size.assign(cav_nodes.size(), 0);
    cav_filled.assign(cav_nodes.size(), 0);
    for (size_t c = 0; c < cav_nodes.size(); c++) {
      double cv = cav_nodes[c].size() * cubeVol;
      cav_size[c] = cv;
      if (cv <= cav_vol) {
        cav_filled[c] = 1;
        if (eps_on())
          for (int64_t f : cav_nodes[c]) {
            for (int a = 0; a < 3; a++) eps[3 * f + a] = NS_EPS_INSIDE;
            eps[3 * (f - 1)] = NS_EPS_INSIDE;
            eps[3 * (f - g.nx) + 1] = NS_EPS_INSIDE;
            eps[3 * (f - plane) + 2] = NS_EPS_INSIDE;
            ideb[f] = 0;
          }
        if (flags & 2)
          for (int64_t f : cav_nodes[c]) {
            int64_t k = f / plane, j = (f % plane) / g.nx, i = f % g.nx;
            for (int dk = 0; dk < 2; dk++)
              for (int dj = 0; dj < 2; dj++)
                for (int di = 0; di < 2; di++) clear_bit(i + di, j + dj, k + dk);
          }
      }
    }
  }

  // projectToSphere (src/tools.cpp:1112-1120)
  static double project_sphere(const double* y, const double* c, double r, double* proj) {
    double dist = sqrt((y[0] - c[0]) * (y[0] - c[0]) + (y[1] - c[1]) * (y[1] - c[1]) + (y[2] - c[2]) * (y[2] - c[2]));
    dist = r / dist;
    for (int d = 0; d < 3; d++) proj[d] = y[d] - c[d];
    for (int d = 0; d < 3; d++) proj[d] = c[d] + dist * proj[d];
    return sqrt((proj[0] - y[0]) * (proj[0] - y[0]) + (proj[1] - y[1]) * (proj[1] - y[1]) +
                (proj[2] - y[2]) * (proj[2] - y[2]));
  }
  // projectToCircle (src/ConnollySurface.cpp:5693-5703) with point2plane (src/tools.cpp:277-287)
  static void project_circle(const double* p, double radius, const double* c, const double* w, double* proj) {
    const double den = w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
    const double val = (w[0] * p[0] + w[1] * p[1] + w[2] * p[2]) + w[3];
    const double cc = val / den;
    for (int d = 0; d < 3; d++) proj[d] = p[d] - w[d] * cc;
    for (int d = 0; d < 3; d++) proj[d] = proj[d] - c[d];
    radius /= sqrt(proj[0] * proj[0] + proj[1] * proj[1] + proj[2] * proj[2]);
    for (int d = 0; d < 3; d++) proj[d] = c[d] + radius * proj[d];
  }
  // projectToTorus (src/ConnollySurface.cpp:5705-5733); the rotation back is the transpose of the
  // stored inverse frame
  static double project_torus(const double* y, const double* f, double probe, double* proj) {
    const double* inv = f + 9;
    const double* tc = f + 4;
    double temp[3], pp[3];
    for (int d = 0; d < 3; d++) temp[d] = y[d] - tc[d];
    for (int i = 0; i < 3; i++) pp[i] = inv[3 * i] * temp[0] + inv[3 * i + 1] * temp[1] + inv[3 * i + 2] * temp[2];
    const double zero3[3] = {0., 0., 0.};
    const double torus_plane[4] = {0., 0., 1., 0.};
    double major[3];
    project_circle(pp, f[7], zero3, torus_plane, major);
    // plane3points (src/tools.cpp:258-274), normalised
    const double p2[3] = {0., 0., 1.}, p3[3] = {0., 0., -1.};
    double w[4];
    w[0] = major[1] * (p2[2] - p3[2]) + p2[1] * (p3[2] - major[2]) + p3[1] * (major[2] - p2[2]);
    w[1] = major[2] * (p2[0] - p3[0]) + p2[2] * (p3[0] - major[0]) + p3[2] * (major[0] - p2[0]);
    w[2] = major[0] * (p2[1] - p3[1]) + p2[0] * (p3[1] - major[1]) + p3[0] * (major[1] - p2[1]);
    w[3] = -(w[0] * major[0] + w[1] * major[1] + w[2] * major[2]);
    const double nrm = sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
    for (int d = 0; d < 4; d++) w[d] /= nrm;
    double loc[3];
    project_circle(pp, probe, major, w, loc);
    for (int i = 0; i < 3; i++) pp[i] = inv[i] * loc[0] + inv[3 + i] * loc[1] + inv[6 + i] * loc[2];
    for (int d = 0; d < 3; d++) proj[d] = pp[d] + tc[d];
    return sqrt((proj[0] - y[0]) * (proj[0] - y[0]) + (proj[1] - y[1]) * (proj[1] - y[1]) +
                (proj[2] - y[2]) * (proj[2] - y[2]));
  }

  // Mesh surfaces (MeshSurface, src/MeshSurface.cpp): the projection plane of a triangle
  // (plane3points src/tools.cpp:258-274, normalised and its offset recomputed as in
  // preProcessTriangles :674-684), point2plane (:2034-2044), inTriangle (:2010-2032, the
  // denominator multiplied rather than divided, as there) and point2triangle (:1864-2008: the
  // nearest of the three edge projections when the plane projection falls outside; its "normal"
  // is A + B t normalised, as there).  Returns whether the plane projection fell inside.
  static void mesh_plane(const double* f, double w[4]) {
    const double *a = f, *b = f + 3, *c = f + 6;
    w[0] = a[1] * (b[2] - c[2]) + b[1] * (c[2] - a[2]) + c[1] * (a[2] - b[2]);
    w[1] = a[2] * (b[0] - c[0]) + b[2] * (c[0] - a[0]) + c[2] * (a[0] - b[0]);
    w[2] = a[0] * (b[1] - c[1]) + b[0] * (c[1] - a[1]) + c[0] * (a[1] - b[1]);
    const double norm = sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
    w[0] /= norm;
    w[1] /= norm;
    w[2] /= norm;
    w[3] = -(a[0] * (b[1] * c[2] - c[1] * b[2]) + b[0] * (c[1] * a[2] - a[1] * c[2]) + c[0] * (a[1] * b[2] - b[1] * a[2]));
    w[3] /= norm;
  }
  static bool mesh_project(const double* P, const double* f, double* proj, double* dist, double* normal) {
    const double *A = f, *B = f + 3, *C = f + 6;
    double w[4];
    mesh_plane(f, w);
    const double den = w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
    const double dd = sqrt(den);
    const double val = (w[0] * P[0] + w[1] * P[1] + w[2] * P[2]) + w[3];
    for (int d = 0; d < 3; d++) proj[d] = P[d] - w[d] * (val / den);
    *dist = fabs(val / dd);
    double v0[3], v1[3], v2[3];
    for (int d = 0; d < 3; d++) {
      v0[d] = C[d] - A[d];
      v1[d] = B[d] - A[d];
      v2[d] = proj[d] - A[d];
    }
    auto dot = [](const double* x, const double* y) { return x[0] * y[0] + x[1] * y[1] + x[2] * y[2]; };
    const double d00 = dot(v0, v0), d01 = dot(v0, v1), d02 = dot(v0, v2), d11 = dot(v1, v1), d12 = dot(v1, v2);
    const double inv = d00 * d11 - d01 * d01;
    const double u = (d11 * d02 - d01 * d12) * inv, v = (d00 * d12 - d01 * d02) * inv;
    if (u > 0 && v > 0 && u + v < 1) {
      for (int d = 0; d < 3; d++) normal[d] = w[d];
      return true;
    }
    // edges AB, AC, BC: clamp the plane projection's parameter, distance from P
    const double* E[3][2] = {{A, B}, {A, C}, {B, C}};
    double res[3][3], de[3], tt[3];
    for (int e = 0; e < 3; e++) {
      const double *S = E[e][0], *T = E[e][1];
      double t2[3], t1[3];
      for (int d = 0; d < 3; d++) {
        t2[d] = T[d] - S[d];
        t1[d] = proj[d] - S[d];
      }
      const double l2 = dot(t2, t2);
      double t = dot(t1, t2);
      if (t < 0.0) {
        for (int d = 0; d < 3; d++) t1[d] = P[d] - S[d];
        de[e] = sqrt(dot(t1, t1));
        for (int d = 0; d < 3; d++) res[e][d] = S[d];
        t = 0.0;
      } else if (t > l2) {
        for (int d = 0; d < 3; d++) t1[d] = P[d] - T[d];
        de[e] = sqrt(dot(t1, t1));
        for (int d = 0; d < 3; d++) res[e][d] = T[d];
        t = 1.0;
      } else {
        t /= l2;
        for (int d = 0; d < 3; d++) res[e][d] = S[d] + t2[d] * t;
        for (int d = 0; d < 3; d++) t1[d] = res[e][d] - P[d];
        de[e] = sqrt(dot(t1, t1));
      }
      tt[e] = t;
    }
    const int k = (de[0] <= de[1] && de[0] <= de[2]) ? 0 : ((de[1] <= de[0] && de[1] <= de[2]) ? 1 : 2);
    for (int d = 0; d < 3; d++) proj[d] = res[k][d];
    *dist = de[k];
    for (int d = 0; d < 3; d++) normal[d] = E[k][0][d] + E[k][1][d] * tt[k];
    const double nn = sqrt(dot(normal, normal));
    for (int d = 0; d < 3; d++) normal[d] /= nn;
    return false;
  }

  // Boundary grid points (src/Surface.cpp:1488-1546) and the projection of the external ones
  // (Surface::projector, src/Surface.cpp:4657-4676; ConnollySurface::getProjection,
  // src/ConnollySurface.cpp:5822-5912) over the auxiliary grid of buildAuxiliaryGrid
  // (src/ConnollySurface.cpp:3681-3870).  A point without a feasible projection keeps its own
  // coordinates (flag 1; the reference's sampled-circle retry for self-intersecting edges is not
  // restated), one in an empty cell too (flag 2).
  void boundary_points() {
    const int64_t NX = g.nx, NY = g.ny, NZ = g.nz;
    auto E = [&](int64_t i, int64_t j, int64_t k, int l) { return eps[3 * ((k * NY + j) * NX + i) + l]; };
    for (int64_t iz = 1; iz < NZ; iz++)
      for (int64_t iy = 1; iy < NY; iy++)
        for (int64_t ix = 1; ix < NX; ix++) {
          const int32_t k0 = E(ix, iy, iz, 0);
          if (k0 != E(ix, iy, iz, 1) || k0 != E(ix, iy, iz, 2) || k0 != E(ix - 1, iy, iz, 0) ||
              k0 != E(ix, iy - 1, iz, 1) || k0 != E(ix, iy, iz - 1, 2)) {
            ibgp.push_back((int32_t)ix);
            ibgp.push_back((int32_t)iy);
            ibgp.push_back((int32_t)iz);
            const bool ext = E(ix, iy, iz, 0) == 0 || E(ix, iy, iz, 1) == 0 || E(ix, iy, iz, 2) == 0 ||
                             E(ix - 1, iy, iz, 0) == 0 || E(ix, iy - 1, iz, 1) == 0 || E(ix, iy, iz - 1, 2) == 0;
            bgp_type.push_back(ext ? NS_EXTERNAL_BGP : NS_INTERNAL_BGP);
          }
        }
    // auxiliary grid
    int64_t igrid = NX, mul = 1;
    while (igrid > aux_max_dim) {
      mul += 2;
      int64_t digrid = NX;
      while (true) {
        const int64_t fp = (digrid + (mul - 1)) / mul;
        igrid = fp * mul;
        if (igrid % 2 == 0) digrid = igrid + 1;
        else { igrid = fp; break; }
      }
    }
    const double ascale = g.scale / (double)mul, aside = (double)mul / g.scale;
    const double amin[3] = {g.baricenter[0] - (igrid - 1) * 0.5 * aside, g.baricenter[1] - (igrid - 1) * 0.5 * aside,
                            g.baricenter[2] - (igrid - 1) * 0.5 * aside};
    std::vector<std::vector<int32_t>> cells((size_t)(igrid * igrid * igrid));
    for (int64_t it = 0; it < P.n; it++) {
      const double* f = P.f64 + NS_PATCH_F64 * it;
      int64_t lo[3], hi[3];
      if (P.i32[NS_PATCH_I32 * it] == NS_MESH_TRI) {
        // the triangle's vertex box (MeshSurface::buildAuxiliaryGrid, src/MeshSurface.cpp:867-929)
        for (int d = 0; d < 3; d++) {
          double dn = 1e20, up = -1e20;
          for (int v = 0; v < 3; v++) {
            dn = f[3 * v + d] < dn ? f[3 * v + d] : dn;
            up = f[3 * v + d] > up ? f[3 * v + d] : up;
          }
          lo[d] = std::min<int64_t>(std::max<int64_t>((int64_t)rintp((dn - amin[d]) * ascale), 0), igrid - 1);
          hi[d] = std::min<int64_t>(std::max<int64_t>((int64_t)rintp((up - amin[d]) * ascale), 0), igrid - 1);
        }
      } else
      for (int d = 0; d < 3; d++) {
        lo[d] = (int64_t)rintp(fmax(0., (f[d] - f[3]) - amin[d]) * ascale);
        hi[d] = (int64_t)rintp(fmax(0., (f[d] + f[3]) - amin[d]) * ascale);
        if (lo[d] >= igrid) lo[d] = igrid - 1;
        if (hi[d] >= igrid) hi[d] = igrid - 1;
      }
      for (int64_t iz = lo[2]; iz <= hi[2]; iz++)
        for (int64_t iy = lo[1]; iy <= hi[1]; iy++)
          for (int64_t ix = lo[0]; ix <= hi[0]; ix++) cells[(iz * igrid + iy) * igrid + ix].push_back((int32_t)it);
    }
    const size_t n = bgp_type.size();
    scspos.assign(3 * n, 0.0);
    scsnor.assign(3 * n, 0.0);
    bgp_flag.assign(n, 0);
    for (size_t q = 0; q < n; q++) {
      const double y[3] = {X(ibgp[3 * q]), Y(ibgp[3 * q + 1]), Z(ibgp[3 * q + 2])};
      for (int d = 0; d < 3; d++) scspos[3 * q + d] = y[d];
      if (bgp_type[q] != NS_EXTERNAL_BGP) { bgp_flag[q] = 3; continue; }
      int64_t ic[3];
      bool in = true;
      for (int d = 0; d < 3; d++) {
        ic[d] = (int64_t)rintp((y[d] - amin[d]) * ascale);
        in = in && ic[d] >= 0 && ic[d] < igrid;
      }
      if (!in || cells[(ic[2] * igrid + ic[1]) * igrid + ic[0]].empty()) { bgp_flag[q] = 2; continue; }
      double best = INFINITY;
      std::vector<int32_t> cand = cells[(ic[2] * igrid + ic[1]) * igrid + ic[0]];
      std::sort(cand.begin(), cand.end());
      bool inside_best = false;
      for (int32_t it : cand) {
        const double* f = P.f64 + NS_PATCH_F64 * (int64_t)it;
        const int kind = P.i32[NS_PATCH_I32 * (int64_t)it];
        double proj[3], dist;
        if (kind == NS_MESH_TRI) {
          double nrm[3];
          const bool in_tri = mesh_project(y, f, proj, &dist, nrm);
          if (dist < best) {
            best = dist;
            inside_best = in_tri;
            for (int d = 0; d < 3; d++) {
              scspos[3 * q + d] = proj[d];
              scsnor[3 * q + d] = nrm[d];
            }
          }
          continue;
        }
        if (kind == NS_POINT) dist = project_sphere(y, f, f[3], proj);
        else if (kind == NS_FACE_REG || kind == NS_FACE_SING) dist = project_sphere(y, f, P.probe, proj);
        else dist = project_torus(y, f, P.probe, proj);
        if (!feasible(P, it, proj)) continue;
        if (dist < best) {
          best = dist;
          for (int d = 0; d < 3; d++) scspos[3 * q + d] = proj[d];
        }
      }
      const bool mesh = P.i32[NS_PATCH_I32 * (int64_t)cand[0]] == NS_MESH_TRI;
      bgp_flag[q] = mesh ? (inside_best ? 0 : 1) : (best == INFINITY ? 1 : 0);
    }
  }

  std::vector<int32_t> idx[3];  // edge -> vertex index, dense per direction
  int64_t IX(int64_t i, int64_t j, int64_t k) const { return (k * g.ny + j) * g.nx + i; }

  // Dangling-vertex removal and first-vertex-per-edge wins (assembleVerticesList).
  void assemble() {
    vlist.clear();
    vkey.clear();
    int64_t tot = g.nx * g.ny * g.nz;
    for (int d = 0; d < 3; d++) idx[d].assign(tot, -1);
    size_t nv = vert_edge.size() / 4;
    for (size_t v = 0; v < nv; v++) {
      const int32_t* e = &vert_edge[4 * v];
      bool a = rbit(e[0], e[1], e[2]);
      bool b;
      if (e[3] == NS_X_DIR) b = rbit(e[0] + 1, e[1], e[2]);
      else if (e[3] == NS_Y_DIR) b = rbit(e[0], e[1] + 1, e[2]);
      else b = rbit(e[0], e[1], e[2] + 1);
      if (a == b) continue;
      int32_t& slot = idx[e[3]][IX(e[0], e[1], e[2])];
      if (slot != -1) continue;
      slot = (int32_t)(vlist.size() / 3);
      vlist.insert(vlist.end(), &vert[3 * v], &vert[3 * v] + 3);
      vkey.insert(vkey.end(), e, e + 4);
      vpid.push_back(vert_pid[v]);
    }
  }

  // Compute_Vertex_Normals: the patch normal at each analytic vertex (ConnollySurface::getNormal,
  // src/ConnollySurface.cpp:5736-5819, evaluated at the vertex; the skin quadric's gradient
  // times 2, -2 for reduced tetrahedra, src/SkinSurface.cpp:3684-3712), zero for the others, which
  // then get the mean of their triangles' plane3points normals, normalised (approximateNormals,
  // src/Surface.cpp:10420-10460, 10660-10735).
  void vertex_normals() {
    const int64_t nv = (int64_t)vlist.size() / 3, nan = (int64_t)vpid.size();
    normals.assign(3 * nv, 0.0);
    for (int64_t v = 0; v < nan; v++) {
      const int32_t pid = vpid[v];
      const double* f = P.f64 + NS_PATCH_F64 * (int64_t)pid;
      const int kind = P.i32[NS_PATCH_I32 * (int64_t)pid];
      const double* y = &vlist[3 * v];
      double* n = &normals[3 * v];
      if (kind == NS_FACE_REG || kind == NS_FACE_SING) {
        for (int d = 0; d < 3; d++) n[d] = (f[d] - y[d]) / P.probe;
      } else if (kind == NS_POINT) {
        for (int d = 0; d < 3; d++) n[d] = (y[d] - f[d]) / f[3];
      } else if (kind == NS_EDGE_REG || kind == NS_EDGE_SING) {
        const double* inv = f + 9;
        double t[3] = {y[0] - f[4], y[1] - f[5], y[2] - f[6]}, C[3];
        for (int i = 0; i < 3; i++) C[i] = inv[3 * i] * t[0] + inv[3 * i + 1] * t[1] + inv[3 * i + 2] * t[2];
        double d = C[0] * C[0] + C[1] * C[1];
        double rm1 = f[7] / sqrt(d) - 1.;
        d = sqrt(d * rm1 * rm1 + C[2] * C[2]);
        C[0] *= rm1 / d;
        C[1] *= rm1 / d;
        C[2] /= -d;
        for (int i = 0; i < 3; i++) n[i] = inv[i] * C[0] + inv[3 + i] * C[1] + inv[6 + i] * C[2];
      } else if (ns_is_skin(kind)) {
        const double* Q = f + NS_SKIN_Q;
        const double sg = kind == NS_SKIN_TETRA ? -2.0 : 2.0;
        n[0] = sg * (Q[0] * y[0] + Q[4] * y[1] + Q[7] * y[2] + Q[9]);
        n[1] = sg * (Q[4] * y[0] + Q[1] * y[1] + Q[5] * y[2] + Q[8]);
        n[2] = sg * (Q[7] * y[0] + Q[5] * y[1] + Q[2] * y[2] + Q[6]);
      }
    }
    std::vector<char> app(nv, 0);
    for (int64_t v = 0; v < nv; v++) app[v] = normals[3 * v] == 0 && normals[3 * v + 1] == 0 && normals[3 * v + 2] == 0;
    std::vector<double> mean(3 * nv, 0.0);
    const int64_t nt = (int64_t)tris.size() / 3;
    for (int64_t t = 0; t < nt; t++) {
      const double* p1 = &vlist[3 * (int64_t)tris[3 * t]];
      const double* p2 = &vlist[3 * (int64_t)tris[3 * t + 1]];
      const double* p3 = &vlist[3 * (int64_t)tris[3 * t + 2]];
      double w[3];
      w[0] = p1[1] * (p2[2] - p3[2]) + p2[1] * (p3[2] - p1[2]) + p3[1] * (p1[2] - p2[2]);
      w[1] = p1[2] * (p2[0] - p3[0]) + p2[2] * (p3[0] - p1[0]) + p3[2] * (p1[0] - p2[0]);
      w[2] = p1[0] * (p2[1] - p3[1]) + p2[0] * (p3[1] - p1[1]) + p3[0] * (p1[1] - p2[1]);
      for (int q = 0; q < 3; q++) {
        const int32_t v = tris[3 * t + q];
        if (!app[v]) continue;
        for (int d = 0; d < 3; d++) mean[3 * v + d] = mean[3 * v + d] + w[d];
      }
    }
    for (int64_t v = 0; v < nv; v++) {
      if (!app[v]) continue;
      double* m = &mean[3 * v];
      double len = sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
      for (int d = 0; d < 3; d++) normals[3 * v + d] = m[d] / len;
    }
  }

  void triangulate() {
    int64_t tot = g.nx * g.ny * g.nz;
    std::vector<char> active(tot, 0);
    auto cube = [&](int64_t i, int64_t j, int64_t k) {
      int c = 0;
      if (!rbit(i, j, k)) c |= 1;
      if (!rbit(i + 1, j, k)) c |= 2;
      if (!rbit(i + 1, j + 1, k)) c |= 4;
      if (!rbit(i, j + 1, k)) c |= 8;
      if (!rbit(i, j, k + 1)) c |= 16;
      if (!rbit(i + 1, j, k + 1)) c |= 32;
      if (!rbit(i + 1, j + 1, k + 1)) c |= 64;
      if (!rbit(i, j + 1, k + 1)) c |= 128;
      return c;
    };
    static const int ec[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6}, {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
    auto emask = [&](int c) {
      int m = 0;
      for (int e = 0; e < 12; e++)
        if (((c >> ec[e][0]) & 1) != ((c >> ec[e][1]) & 1)) m |= 1 << e;
      return m;
    };
    // pass 1: active cubes and midpoint vertices for own edges 5, 6, 10 (getVertices)
    for (int64_t k = 1; k < g.nz - 1; k++)
      for (int64_t j = 1; j < g.ny - 1; j++)
        for (int64_t i = 1; i < g.nx - 1; i++) {
          int c = cube(i, j, k);
          int m = emask(c);
          if (m == 0) continue;
          active[IX(i, j, k)] = 1;
          if (m & 32) {
            int32_t& s = idx[NS_Y_DIR][IX(i + 1, j, k + 1)];
            if (s == -1) {
              double p[3] = {X(i + 1) - g.hside, Y(j), Z(k + 1) - g.hside};
              s = (int32_t)(vlist.size() / 3);
              vlist.insert(vlist.end(), p, p + 3);
              int32_t e[4] = {(int32_t)(i + 1), (int32_t)j, (int32_t)(k + 1), NS_Y_DIR};
              vkey.insert(vkey.end(), e, e + 4);
            }
          }
          if (m & 64) {
            int32_t& s = idx[NS_X_DIR][IX(i, j + 1, k + 1)];
            if (s == -1) {
              double p[3] = {X(i), Y(j + 1) - g.hside, Z(k + 1) - g.hside};
              s = (int32_t)(vlist.size() / 3);
              vlist.insert(vlist.end(), p, p + 3);
              int32_t e[4] = {(int32_t)i, (int32_t)(j + 1), (int32_t)(k + 1), NS_X_DIR};
              vkey.insert(vkey.end(), e, e + 4);
            }
          }
          if (m & 1024) {
            int32_t& s = idx[NS_Z_DIR][IX(i + 1, j + 1, k)];
            if (s == -1) {
              double p[3] = {X(i + 1) - g.hside, Y(j + 1) - g.hside, Z(k)};
              s = (int32_t)(vlist.size() / 3);
              vlist.insert(vlist.end(), p, p + 3);
              int32_t e[4] = {(int32_t)(i + 1), (int32_t)(j + 1), (int32_t)k, NS_Z_DIR};
              vkey.insert(vkey.end(), e, e + 4);
            }
          }
        }
    // pass 2: triangles and Heron area (triangulationKernel / getTriangles)
    area = 0;
    for (int64_t k = 1; k < g.nz - 1; k++)
      for (int64_t j = 1; j < g.ny - 1; j++)
        for (int64_t i = 1; i < g.nx - 1; i++) {
          if (!active[IX(i, j, k)]) continue;
          int c = cube(i, j, k);
          int m = emask(c);
          int vl[12];
          for (int e = 0; e < 12; e++) vl[e] = -1;
          const int64_t ek[12][4] = {{i, j, k, 0}, {i + 1, j, k, 1}, {i, j + 1, k, 0}, {i, j, k, 1},
                                     {i, j, k + 1, 0}, {i + 1, j, k + 1, 1}, {i, j + 1, k + 1, 0}, {i, j, k + 1, 1},
                                     {i, j, k, 2}, {i + 1, j, k, 2}, {i + 1, j + 1, k, 2}, {i, j + 1, k, 2}};
          for (int e = 0; e < 12; e++)
            if (m & (1 << e)) vl[e] = idx[ek[e][3]][IX(ek[e][0], ek[e][1], ek[e][2])];
          const char* cs = kNsMcCases[c];
          for (int q = 0; cs[q]; q += 3) {
            int a = vl[cs[q] <= '9' ? cs[q] - '0' : cs[q] - 'a' + 10];
            int b = vl[cs[q + 1] <= '9' ? cs[q + 1] - '0' : cs[q + 1] - 'a' + 10];
            int cc = vl[cs[q + 2] <= '9' ? cs[q + 2] - '0' : cs[q + 2] - 'a' + 10];
            if (a == -1 || b == -1 || cc == -1) continue;
            const double* A = &vlist[3 * (int64_t)a];
            const double* B = &vlist[3 * (int64_t)b];
            const double* Cc = &vlist[3 * (int64_t)cc];
            double da = sqrt((A[0] - B[0]) * (A[0] - B[0]) + (A[1] - B[1]) * (A[1] - B[1]) + (A[2] - B[2]) * (A[2] - B[2]));
            double db = sqrt((A[0] - Cc[0]) * (A[0] - Cc[0]) + (A[1] - Cc[1]) * (A[1] - Cc[1]) + (A[2] - Cc[2]) * (A[2] - Cc[2]));
            double dc = sqrt((B[0] - Cc[0]) * (B[0] - Cc[0]) + (B[1] - Cc[1]) * (B[1] - Cc[1]) + (B[2] - Cc[2]) * (B[2] - Cc[2]));
            double ttt = (da + db + dc) * (db + dc - da) * (dc + da - db) * (da + db - dc);
            if (ttt > 0) area += 0.25 * sqrt(ttt);
            tris.push_back(cc);
            tris.push_back(b);
            tris.push_back(a);
          }
        }
  }

  void run() {
    for (int k = 0; k < kOpCount; k++) g_ops[k].store(0);
    NMAX = std::max(g.nx, std::max(g.ny, g.nz));
    panels[0] = eps_on() ? 3 : ((flags & 1) ? 1 : 0);
    panels[1] = (flags & 2) ? 3 : 0;
    numPanels = panels[0] + panels[1];
    if (flags & (1 | 32)) status.assign(g.nx * g.ny * g.nz, NS_STATUS_TEMPORARY_OUT);
    if (eps_on()) {
      eps.assign(3 * g.nx * g.ny * g.nz, 0);
      ideb.assign(g.nx * g.ny * g.nz, 1);
    }
    if (flags & 2) {
      int64_t cnx = (g.nx + 31) >> 5;
      bits.assign(cnx * g.ny * g.nz, ~0u);
    }
    if (P.n > 0 && numPanels > 0) trace();
    else {
      pix_off.assign(NMAX * NMAX * std::max(1, numPanels) + 1, 0);
    }
    int np = ((flags & 2) || eps_on()) ? 3 : ((flags & 1) ? 1 : 0);
    for (int panel = 0; panel < np; panel++) fill_panel(panel);
    volume = flagsum ? g.A * (volPanel[0] + volPanel[1] + volPanel[2]) / flagsum : 0;
    if ((flags & 4) && (flags & (1 | 32))) cavities();
    if (eps_on() && (flags & 64)) boundary_points();
    // vertex assembly and marching cubes (the dense edge-index grids are needed only here)
    if ((flags & 2) && (flags & 8)) {
      assemble();
      triangulate();
      if (flags & 16) vertex_normals();
    }
  }
};

// The blobby mesh: field, marching cubes at iso 1, smoothing, OFF round trip.
struct BlobbyMesh {
  std::vector<double> verts;  // 3 per vertex
  std::vector<int32_t> vkey;  // 4 per vertex: grid edge (x, y, z, axis)
  std::vector<int32_t> tris;  // 3 per triangle
};

BlobbyMesh blobby_mesh(const NsGrid& g, const double* atoms, int64_t na, double B, bool quantize) {
  const int64_t NX = g.nx, NY = g.ny, NZ = g.nz;
  auto X = [&](int64_t i) { return ns_coord(g.xmin, g.side, i); };
  auto Y = [&](int64_t j) { return ns_coord(g.ymin, g.side, j); };
  auto Z = [&](int64_t k) { return ns_coord(g.zmin, g.side, k); };
  auto IX = [&](int64_t i, int64_t j, int64_t k) { return (k * NY + j) * NX + i; };
  // BlobbySurface::build: atom by atom over its cube of +-numgrid nodes (cut-off 6 A)
  const int numgrid = (int)(6.0 / g.side + 0.5);
  std::vector<double> field(NX * NY * NZ, 0.0);
  for (int64_t a = 0; a < na; a++) {
    const double* pos = atoms + 4 * a;
    const double r = atoms[4 * a + 3];
    const double r2 = r * r;
    const int ix = (int)rintp((pos[0] - g.xmin) * g.scale);
    const int iy = (int)rintp((pos[1] - g.ymin) * g.scale);
    const int iz = (int)rintp((pos[2] - g.zmin) * g.scale);
    const int sx = std::max(0, ix - numgrid), sy = std::max(0, iy - numgrid), sz = std::max(0, iz - numgrid);
    const int ex = std::min((int)NX, ix + numgrid), ey = std::min((int)NY, iy + numgrid), ez = std::min((int)NZ, iz + numgrid);
    for (int kk = sz; kk < ez; kk++)
      for (int jj = sy; jj < ey; jj++)
        for (int ii = sx; ii < ex; ii++) {
          double p[3] = {X(ii) - g.hside, Y(jj) - g.hside, Z(kk) - g.hside};
          double dist2 = (p[0] - pos[0]) * (p[0] - pos[0]) + (p[1] - pos[1]) * (p[1] - pos[1]) +
                         (p[2] - pos[2]) * (p[2] - pos[2]);
          field[IX(ii, jj, kk)] += exp(B * (dist2 / r2 - 1));
        }
  }
  const double iso = 1.0;
  static const int ec[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6}, {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
  auto cube = [&](int64_t i, int64_t j, int64_t k, double* v) {
    v[0] = field[IX(i, j, k)]; v[1] = field[IX(i + 1, j, k)]; v[2] = field[IX(i + 1, j + 1, k)];
    v[3] = field[IX(i, j + 1, k)]; v[4] = field[IX(i, j, k + 1)]; v[5] = field[IX(i + 1, j, k + 1)];
    v[6] = field[IX(i + 1, j + 1, k + 1)]; v[7] = field[IX(i, j + 1, k + 1)];
    int c = 0;
    for (int q = 0; q < 8; q++)
      if (v[q] < iso) c |= 1 << q;
    return c;
  };
  auto emask = [&](int c) {
    int m = 0;
    for (int e = 0; e < 12; e++)
      if (((c >> ec[e][0]) & 1) != ((c >> ec[e][1]) & 1)) m |= 1 << e;
    return m;
  };
  BlobbyMesh M;
  std::vector<int32_t> idx[3];
  for (int d = 0; d < 3; d++) idx[d].assign(NX * NY * NZ, -1);
  // getVertices: the own edges 5, 6, 10 of every active cube, in (k, j, i) order
  for (int64_t k = 1; k < NZ - 1; k++)
    for (int64_t j = 1; j < NY - 1; j++)
      for (int64_t i = 1; i < NX - 1; i++) {
        double v[8];
        int c = cube(i, j, k, v);
        int m = emask(c);
        if (m == 0) continue;
        double xg = X(i), yg = Y(j), zg = Z(k);
        double tb[6] = {xg - g.hside, xg + g.hside, yg - g.hside, yg + g.hside, zg - g.hside, zg + g.hside};
        static const int mul[8][3] = {{0, 2, 4}, {1, 2, 4}, {1, 3, 4}, {0, 2, 4}, {0, 2, 5}, {1, 2, 5}, {1, 3, 5}, {0, 3, 5}};
        double pos[8][3];
        for (int q = 0; q < 8; q++)
          for (int d = 0; d < 3; d++) pos[q][d] = tb[mul[q][d]];
        auto interp = [&](int a, int b, double* p) {
          double mu = (iso - v[a]) / (v[b] - v[a]);
          for (int d = 0; d < 3; d++) {
            double tmp = pos[b][d] - pos[a][d];
            p[d] = pos[a][d] + mu * tmp;
          }
        };
        struct E { int bit, a, b, dir; int64_t x, y, z; };
        const E es[3] = {{32, 5, 6, NS_Y_DIR, i + 1, j, k + 1}, {64, 6, 7, NS_X_DIR, i, j + 1, k + 1},
                         {1024, 2, 6, NS_Z_DIR, i + 1, j + 1, k}};
        for (const E& e : es) {
          if (!(m & e.bit)) continue;
          double p[3];
          interp(e.a, e.b, p);
          idx[e.dir][IX(e.x, e.y, e.z)] = (int32_t)(M.verts.size() / 3);
          M.verts.insert(M.verts.end(), p, p + 3);
          int32_t key[4] = {(int32_t)e.x, (int32_t)e.y, (int32_t)e.z, e.dir};
          M.vkey.insert(M.vkey.end(), key, key + 4);
        }
      }
  // triangulationKernel: triangles in the case table's order and winding
  for (int64_t k = 1; k < NZ - 1; k++)
    for (int64_t j = 1; j < NY - 1; j++)
      for (int64_t i = 1; i < NX - 1; i++) {
        double v[8];
        int c = cube(i, j, k, v);
        int m = emask(c);
        if (m == 0) continue;
        const int64_t ek[12][4] = {{i, j, k, 0}, {i + 1, j, k, 1}, {i, j + 1, k, 0}, {i, j, k, 1},
                                   {i, j, k + 1, 0}, {i + 1, j, k + 1, 1}, {i, j + 1, k + 1, 0}, {i, j, k + 1, 1},
                                   {i, j, k, 2}, {i + 1, j, k, 2}, {i + 1, j + 1, k, 2}, {i, j + 1, k, 2}};
        int vl[12];
        for (int e = 0; e < 12; e++) vl[e] = (m & (1 << e)) ? idx[ek[e][3]][IX(ek[e][0], ek[e][1], ek[e][2])] : -1;
        const char* cs = kNsMcCases[c];
        for (int q = 0; cs[q]; q += 3) {
          int a = vl[cs[q] <= '9' ? cs[q] - '0' : cs[q] - 'a' + 10];
          int b = vl[cs[q + 1] <= '9' ? cs[q + 1] - '0' : cs[q + 1] - 'a' + 10];
          int cc = vl[cs[q + 2] <= '9' ? cs[q + 2] - '0' : cs[q + 2] - 'a' + 10];
          if (a == -1 || b == -1 || cc == -1) continue;
          M.tris.push_back(a);
          M.tris.push_back(b);
          M.tris.push_back(cc);
        }
      }
  // smoothSurface: one Laplacian pass
  const int64_t nv = (int64_t)M.verts.size() / 3, nt = (int64_t)M.tris.size() / 3;
  std::vector<double> temp(3 * nv, 0.0);
  std::vector<int> nn(nv, 0);
  for (int64_t t = 0; t < nt; t++) {
    int v1 = M.tris[3 * t], v2 = M.tris[3 * t + 1], v3 = M.tris[3 * t + 2];
    for (int d = 0; d < 3; d++) {
      temp[3 * v1 + d] += M.verts[3 * v2 + d] + M.verts[3 * v3 + d];
      temp[3 * v2 + d] += M.verts[3 * v1 + d] + M.verts[3 * v3 + d];
      temp[3 * v3 + d] += M.verts[3 * v1 + d] + M.verts[3 * v2 + d];
    }
    nn[v1] += 2;
    nn[v2] += 2;
    nn[v3] += 2;
  }
  for (int64_t v = 0; v < nv; v++) {
    double scale = 1.0 / (double)nn[v];
    for (int d = 0; d < 3; d++) M.verts[3 * v + d] = 0.5 * (M.verts[3 * v + d] + temp[3 * v + d] * scale);
  }
  // saveMesh writes "%.3f", loadOFF reads "%f" into floats
  if (quantize)
    for (auto& x : M.verts) {
      char buf[64];
      snprintf(buf, sizeof buf, "%.3f", x);
      float f;
      sscanf(buf, "%f", &f);
      x = f;
    }
  return M;
}

}  // namespace

extern "C" {

// Blobby mesh of atoms on a grid (test infrastructure); read back with nso_size / nso_copy on
// "verts", "vkeys", "tris", freed with nso_free_mesh.
void* nso_blobby(const NsGrid* g, const double* atoms, int64_t n_atoms, double blobbyness, int quantize) {
  return new BlobbyMesh(blobby_mesh(*g, atoms, n_atoms, blobbyness, quantize != 0));
}
int64_t nso_mesh_size(void* h, const char* what) {
  BlobbyMesh* m = (BlobbyMesh*)h;
  std::string w(what);
  if (w == "verts") return (int64_t)m->verts.size();
  if (w == "vkeys") return (int64_t)m->vkey.size();
  if (w == "tris") return (int64_t)m->tris.size();
  return -1;
}
int nso_mesh_copy(void* h, const char* what, void* dst) {
  BlobbyMesh* m = (BlobbyMesh*)h;
  std::string w(what);
  if (w == "verts") memcpy(dst, m->verts.data(), m->verts.size() * sizeof(double));
  else if (w == "vkeys") memcpy(dst, m->vkey.data(), m->vkey.size() * sizeof(int32_t));
  else if (w == "tris") memcpy(dst, m->tris.data(), m->tris.size() * sizeof(int32_t));
  else return -1;
  return 0;
}
void nso_free_mesh(void* h) { delete (BlobbyMesh*)h; }

}  // extern "C"

extern "C" {

// Water-shape filter of the kept cavities, Keep_Water_Shaped_Cavities
// (Surface::filterCavitiesWithBilevelStatusMap, src/Surface.cpp:3011-3290), restated loop for
// loop: cavity by cavity, each of its points marked SHAPE_UNDER_CHECK, then every point whose
// probe sphere (the rintp box, clamped, and dist^2 <= r^2 on the grid coordinates) holds no node
// outside {SHAPE_UNDER_CHECK, SHAPE_OK, -cavityId} becomes a support (-cavityId) and marks the
// sphere SHAPE_OK; the points left SHAPE_UNDER_CHECK are removed (epsilon, ideb and insideness
// entries as fillCavities writes them) and become STATUS_POINT_INSIDE when mod_status is set,
// the SHAPE_OK ones return to cavityId.  status holds the labels after cavity detection and is
// modified in place; filled (per cavity) is the fillCavities flag, updated as the reference
// updates cavitiesFlag.  The points of a cavity are taken in ascending node order rather than in
// the flood fill's order: the support test reads only membership of the set above, which the
// walk over one cavity does not change.  Returns the number of removed points.
int64_t nso_shape_filter(const NsGrid* gp, int32_t* status, int ncav, int32_t* filled, uint32_t* bits, int64_t nwords,
                         int32_t* eps, uint8_t* ideb, double probe, int mod_status) {
  const NsGrid& g = *gp;
  const int64_t NX = g.nx, NY = g.ny, NZ = g.nz, plane = NX * NY, n = plane * NZ;
  std::vector<std::vector<int64_t>> pts(ncav);
  for (int64_t f = 0; f < n; f++)
    if (status[f] >= NS_STATUS_FIRST_CAV && status[f] - NS_STATUS_FIRST_CAV < ncav)
      pts[status[f] - NS_STATUS_FIRST_CAV].push_back(f);
  std::vector<double> X(NX), Y(NY), Z(NZ);
  for (int64_t i = 0; i < NX; i++) X[i] = g.xmin + i * g.side;
  for (int64_t i = 0; i < NY; i++) Y[i] = g.ymin + i * g.side;
  for (int64_t i = 0; i < NZ; i++) Z[i] = g.zmin + i * g.side;
  auto box = [&](double c, double mn, int64_t N, int64_t& lo, int64_t& hi) {
    lo = (int64_t)floor(((c - probe) - mn) * g.scale + 0.5);
    hi = (int64_t)floor(((c + probe) - mn) * g.scale + 0.5);
    if (lo < 0) lo = 0;
    if (hi < 0) hi = 0;
    if (hi >= N) hi = N - 1;
    if (lo >= N) lo = N - 1;
  };
  const double dist2ref = probe * probe;
  int64_t total = 0;
  for (int c = 0; c < ncav; c++) {
    if (filled[c]) continue;
    const int cid = c + NS_STATUS_FIRST_CAV;
    for (int64_t f : pts[c]) status[f] = NS_STATUS_SHAPE_UNDER_CHECK;
    for (int64_t f : pts[c]) {
      const int64_t vk = f / plane, vj = (f % plane) / NX, vi = f % NX;
      int64_t x0, x1, y0, y1, z0, z1;
      box(X[vi], g.xmin, NX, x0, x1);
      box(Y[vj], g.ymin, NY, y0, y1);
      box(Z[vk], g.zmin, NZ, z0, z1);
      bool go_out = false;
      for (int64_t iz = z0; iz <= z1 && !go_out; iz++)
        for (int64_t iy = y0; iy <= y1 && !go_out; iy++)
          for (int64_t ix = x0; ix <= x1; ix++) {
            const double a = X[ix] - X[vi], b = Y[iy] - Y[vj], cc = Z[iz] - Z[vk];
            if (a * a + b * b + cc * cc > dist2ref) continue;
            const int32_t val = status[(iz * NY + iy) * NX + ix];
            if (val != NS_STATUS_SHAPE_UNDER_CHECK && val != NS_STATUS_SHAPE_OK && val != -cid) {
              go_out = true;
              break;
            }
          }
      if (go_out) continue;
      for (int64_t iz = z0; iz <= z1; iz++)
        for (int64_t iy = y0; iy <= y1; iy++)
          for (int64_t ix = x0; ix <= x1; ix++) {
            const double a = X[ix] - X[vi], b = Y[iy] - Y[vj], cc = Z[iz] - Z[vk];
            if (a * a + b * b + cc * cc > dist2ref) continue;
            int32_t& val = status[(iz * NY + iy) * NX + ix];
            if (val != -cid) val = NS_STATUS_SHAPE_OK;
          }
      status[f] = -cid;
    }
    int64_t removed = 0;
    for (int64_t f : pts[c]) {
      if (status[f] == NS_STATUS_SHAPE_UNDER_CHECK) {
        removed++;
        const int64_t vk = f / plane, vj = (f % plane) / NX;
        if (eps) {
          for (int a = 0; a < 3; a++) eps[3 * f + a] = NS_EPS_INSIDE;
          if (f % NX > 0) eps[3 * (f - 1)] = NS_EPS_INSIDE;
          if (vj > 0) eps[3 * (f - NX) + 1] = NS_EPS_INSIDE;
          if (vk > 0) eps[3 * (f - plane) + 2] = NS_EPS_INSIDE;
        }
        if (ideb) ideb[f] = 0;
        if (bits)
          for (int dk = 0; dk < 2; dk++)
            for (int dj = 0; dj < 2; dj++)
              for (int di = 0; di < 2; di++) {
                const int64_t q = f + dk * plane + dj * NX + di;
                if ((q >> 5) < nwords) bits[q >> 5] &= ~(1u << (q & 31));
              }
      }
      if (mod_status && status[f] == NS_STATUS_SHAPE_UNDER_CHECK)
        status[f] = NS_STATUS_INSIDE;
      else if (status[f] == NS_STATUS_SHAPE_OK)
        status[f] = cid;
    }
    if (removed && removed != (int64_t)pts[c].size())
      filled[c] = 0;
    else if (removed && removed == (int64_t)pts[c].size())
      filled[c] = 1;
    total += removed;
  }
  return total;
}


// Pocket detection by difference: Surface::difference (flat status map, src/Surface.cpp:11471-11717)
// loop for loop with its insideness writes, then operator-= (src/Surface.cpp:15556-15619): the
// water-shape filter of the one difference cavity with a 1.4 A probe and the status map modified,
// cav2out (src/Surface.cpp:2649-2689), getCavities(STATUS_POINT_OUT) (src/Surface.cpp:1877-1992:
// the seed scan alternates ascending and descending z; each seed's TEMPORARY_OUT region is the next
// pocket, here flooded breadth-first since only its node set matters), then fillCavities(fill_vol)
// (src/Surface.cpp:2355-2484) on the insideness bits.  st1 (fat probe) is modified in place; sizes
// and filled receive up to cap pockets.  Returns the number of pockets, -1 past cap.
// The mesh projection of one point onto one triangle (9 doubles: A, B, C), for tests.
int nso_mesh_project(const double* P, const double* tri, double* proj, double* dist, double* normal) {
  return Oracle::mesh_project(P, tri, proj, dist, normal) ? 1 : 0;
}

int nso_pocket_difference(const NsGrid* gp, int32_t* st1, const int32_t* st2, uint32_t* bits, int64_t nwords,
                          double fill_vol, double* sizes, int32_t* filled, int cap) {
  const NsGrid& g = *gp;
  const int64_t NX = g.nx, NY = g.ny, NZ = g.nz, plane = NX * NY, n = plane * NZ;
  auto setb = [&](int64_t i, int64_t j, int64_t k, bool v) {
    const int64_t f = k * plane + j * NX + i;
    if (!bits || (f >> 5) >= nwords) return;
    if (v) bits[f >> 5] |= 1u << (f & 31);
    else bits[f >> 5] &= ~(1u << (f & 31));
  };
  std::vector<int64_t> diff;
  for (int64_t k = 0; k < NZ; k++)
    for (int64_t j = 0; j < NY; j++)
      for (int64_t i = 0; i < NX; i++) {
        const int64_t f = k * plane + j * NX + i;
        const int32_t s1 = st1[f], s2 = st2[f];
        if ((s1 != NS_STATUS_TEMPORARY_OUT && s1 != NS_STATUS_OUT) &&
            (s2 == NS_STATUS_TEMPORARY_OUT || s2 == NS_STATUS_OUT)) {
          st1[f] = NS_STATUS_FIRST_CAV;
          diff.push_back(f);
          for (int dk = 0; dk < 2; dk++)
            for (int dj = 0; dj < 2; dj++)
              for (int di = 0; di < 2; di++) setb(i + di, j + dj, k + dk, true);
        } else {
          st1[f] = NS_STATUS_INSIDE;
          for (int dk = 0; dk < 2; dk++)
            for (int dj = 0; dj < 2; dj++)
              for (int di = 0; di < 2; di++)
                if (i + di < NX && j + dj < NY && k + dk < NZ) setb(i + di, j + dj, k + dk, false);
        }
      }
  if (!diff.empty()) {
    int32_t fl0 = 0;
    nso_shape_filter(gp, st1, 1, &fl0, bits, nwords, nullptr, nullptr, 1.4, 1);
    for (int64_t f : diff)
      if (st1[f] >= NS_STATUS_FIRST_CAV || st1[f] <= -NS_STATUS_FIRST_CAV) st1[f] = NS_STATUS_TEMPORARY_OUT;
  }
  int id = NS_STATUS_OUT, times = 0;
  std::vector<std::vector<int64_t>> regions;
  std::vector<int64_t> queue;
  while (true) {
    int64_t seed = -1;
    for (int64_t kk = 0; kk < NZ && seed < 0; kk++) {
      const int64_t k = (times % 2 == 0) ? kk : NZ - 1 - kk;
      for (int64_t q = k * plane; q < (k + 1) * plane; q++)
        if (st1[q] == NS_STATUS_TEMPORARY_OUT) { seed = q; break; }
    }
    times++;
    if (seed < 0) break;
    id++;
    std::vector<int64_t> nodes;
    queue.assign(1, seed);
    st1[seed] = id;
    for (size_t h = 0; h < queue.size(); h++) {
      const int64_t f = queue[h];
      nodes.push_back(f);
      const int64_t k = f / plane, j = (f % plane) / NX, i = f % NX;
      const int64_t nb[6][3] = {{i + 1, j, k}, {i - 1, j, k}, {i, j + 1, k}, {i, j - 1, k}, {i, j, k + 1}, {i, j, k - 1}};
      for (auto& b : nb) {
        if (b[0] < 0 || b[1] < 0 || b[2] < 0 || b[0] >= NX || b[1] >= NY || b[2] >= NZ) continue;
        const int64_t u = b[2] * plane + b[1] * NX + b[0];
        if (st1[u] != NS_STATUS_TEMPORARY_OUT) continue;
        st1[u] = id;
        queue.push_back(u);
      }
    }
    regions.push_back(std::move(nodes));
  }
  const int ncav = (int)regions.size();
  if (ncav > cap) return -1;
  const double cube = g.side * g.side * g.side;
  for (int c = 0; c < ncav; c++) {
    const double vol = regions[c].size() * cube;
    sizes[c] = vol;
    filled[c] = vol <= fill_vol ? 1 : 0;
    if (filled[c] && bits)
      for (int64_t f : regions[c]) {
        const int64_t k = f / plane, j = (f % plane) / NX, i = f % NX;
        for (int dk = 0; dk < 2; dk++)
          for (int dj = 0; dj < 2; dj++)
            for (int di = 0; di < 2; di++) setb(i + di, j + dj, k + dk, false);
      }
  }
  (void)n;
  return ncav;
}

}  // extern "C"

extern "C" {

// flags: 1 status map, 2 accurate-triangulation rays + insideness, 4 cavity detection/filling,
//        8 marching cubes, 16 vertex normals (Compute_Vertex_Normals), 32 epsilon and ideb maps
//        (Build_epsilon_maps), 64 boundary grid points and their projection (with 32).
void* nso_run_ex(const NsGrid* g, int64_t n_patches, const double* f64, const int32_t* i32, const double* pool,
                 const int8_t* pool_flag, double probe, int flags, double cav_vol, int nthreads, int aux_max_dim) {
  Oracle* o = new Oracle();
  o->g = *g;
  o->P = {n_patches, f64, i32, pool, pool_flag, probe};
  o->flags = flags;
  o->cav_vol = cav_vol;
  o->nthreads = nthreads;
  o->aux_max_dim = aux_max_dim;
  o->run();
  return o;
}

void* nso_run(const NsGrid* g, int64_t n_patches, const double* f64, const int32_t* i32, const double* pool,
              const int8_t* pool_flag, double probe, int flags, double cav_vol, int nthreads) {
  Oracle* o = new Oracle();
  o->g = *g;
  o->P = {n_patches, f64, i32, pool, pool_flag, probe};
  o->flags = flags;
  o->cav_vol = cav_vol;
  o->nthreads = nthreads;
  o->run();
  return o;
}

double nso_scalar(void* h, const char* what) {
  Oracle* o = (Oracle*)h;
  std::string w(what);
  if (w == "volume") return o->volume;
  if (w == "area") return o->area;
  if (w == "ncav") return o->ncav;
  if (w == "n_hits") return (double)o->n_hits;
  if (w == "rays_cast") return (double)o->rays_cast;
  if (w == "vol_panel0") return o->volPanel[0];
  if (w == "vol_panel1") return o->volPanel[1];
  if (w == "vol_panel2") return o->volPanel[2];
  static const char* kOpNames[kOpCount] = {"torus_cand", "torus_no_sphere", "quartic_none", "quartic_m0", "quartic_2",
                                           "quartic_4", "quartic_recip", "cubic_small_c", "cubic_ratio_sqrt",
                                           "cubic_ratio_eps", "cubic_cbrt", "cubic_acos", "sphere_cand",
                                           "sphere_miss", "root_test", "root_in", "feas_test", "plane_test",
                                           "clip_test", "sir_test"};
  for (int k = 0; k < kOpCount; k++)
    if (w == std::string("op_") + kOpNames[k]) return (double)g_ops[k].load();
  return NAN;
}

int64_t nso_size(void* h, const char* what) {
  Oracle* o = (Oracle*)h;
  std::string w(what);
  if (w == "status") return (int64_t)o->status.size();
  if (w == "bits") return (int64_t)o->bits.size();
  if (w == "verts") return (int64_t)o->vlist.size();
  if (w == "vkeys") return (int64_t)o->vkey.size();
  if (w == "tris") return (int64_t)o->tris.size();
  if (w == "cav_size") return (int64_t)o->cav_size.size();
  if (w == "pix_off") return (int64_t)o->pix_off.size();
  if (w == "pix_t") return (int64_t)o->pix_t.size();
  if (w == "pix_pid") return (int64_t)o->pix_pid.size();
  if (w == "normals") return (int64_t)o->normals.size();
  if (w == "eps") return (int64_t)o->eps.size();
  if (w == "ideb") return (int64_t)o->ideb.size();
  if (w == "bgp_type") return (int64_t)o->bgp_type.size();
  return -1;
}

int nso_copy(void* h, const char* what, void* dst) {
  Oracle* o = (Oracle*)h;
  std::string w(what);
  if (w == "status") memcpy(dst, o->status.data(), o->status.size() * 4);
  else if (w == "bits") memcpy(dst, o->bits.data(), o->bits.size() * 4);
  else if (w == "verts") memcpy(dst, o->vlist.data(), o->vlist.size() * 8);
  else if (w == "vkeys") memcpy(dst, o->vkey.data(), o->vkey.size() * 4);
  else if (w == "tris") memcpy(dst, o->tris.data(), o->tris.size() * 4);
  else if (w == "cav_size") memcpy(dst, o->cav_size.data(), o->cav_size.size() * 8);
  else if (w == "cav_filled") memcpy(dst, o->cav_filled.data(), o->cav_filled.size() * 4);
  else if (w == "pix_off") memcpy(dst, o->pix_off.data(), o->pix_off.size() * 8);
  else if (w == "pix_t") memcpy(dst, o->pix_t.data(), o->pix_t.size() * 8);
  else if (w == "pix_pid") memcpy(dst, o->pix_pid.data(), o->pix_pid.size() * 4);
  else if (w == "normals") memcpy(dst, o->normals.data(), o->normals.size() * 8);
  else if (w == "eps") memcpy(dst, o->eps.data(), o->eps.size() * 4);
  else if (w == "ideb") memcpy(dst, o->ideb.data(), o->ideb.size());
  else if (w == "ibgp") memcpy(dst, o->ibgp.data(), o->ibgp.size() * 4);
  else if (w == "bgp_type") memcpy(dst, o->bgp_type.data(), o->bgp_type.size() * 4);
  else if (w == "bgp_flag") memcpy(dst, o->bgp_flag.data(), o->bgp_flag.size() * 4);
  else if (w == "scspos") memcpy(dst, o->scspos.data(), o->scspos.size() * 8);
  else if (w == "scsnor") memcpy(dst, o->scsnor.data(), o->scsnor.size() * 8);
  else return -1;
  return 0;
}

void nso_free(void* h) { delete (Oracle*)h; }

// Ray casting of a slab of every ray set (rays whose second pixel index lies in
// [slab_lo, slab_hi) of its range), used to time a bounded sample of a large workload.
void* nso_run_slab(const NsGrid* g, int64_t n_patches, const double* f64, const int32_t* i32, const double* pool,
                   const int8_t* pool_flag, double probe, int flags, int nthreads, double slab_lo, double slab_hi) {
  Oracle* o = new Oracle();
  o->g = *g;
  o->P = {n_patches, f64, i32, pool, pool_flag, probe};
  o->flags = flags & 3;
  o->cav_vol = 0;
  o->nthreads = nthreads;
  o->slab_lo = slab_lo;
  o->slab_hi = slab_hi;
  o->run();
  return o;
}

// Individual math restatements, exposed for the known-answer tests.
int nso_ray_sphere(const double* orig, const double* dir, const double* c, double r, double* t) {
  return ray_sphere(orig, dir, c, r, &t[0], &t[1]) ? 1 : 0;
}
int nso_quartic(double b, double c, double d, double e, double* roots) {
  int n = 0;
  quartic(roots, b, c, d, e, &n);
  return n;
}
double nso_real_cubic(double b, double c, double d) { return real_cubic(b, c, d); }
// rayTorus restatement; t[0..1] hold the clipping-sphere hits on input.
int nso_ray_torus(const double* invrot9, const double* tc, const double* sc, double probe, double major,
                  double radius, int panel, const double* orig, const double* dir, double* t) {
  int vc = (panel == 0) ? 0 : ((panel == 1) ? 2 : 1);
  int n = 0;
  return ray_torus(invrot9, tc, sc, probe, major, radius, vc, orig, dir, t, n) ? n : 0;
}

}  // extern "C"
