// Host SES (Connolly surface) patch builder.
//
// The reference builds its patches from a CGAL Fixed_alpha_shape_3 (alpha = 0) over the regular
// triangulation of the atoms weighted by (r+probe)^2 (src/ConnollySurface.cpp:2038-2078), then
// turns REGULAR/SINGULAR vertices, facets and edges into PointCell, FacetCell and EdgeCell
// records (BuildPointCells :476, BuildFacetCells :787, BuildEdgeCells :1267,
// RemoveSelfIntersections :1928).  CGAL is not available here, so the same alpha-complex
// classification is derived directly from the geometry of the expanded spheres:
//
//  * a facet (i,j,k) is in the complex iff at least one of the two probe placements touching the
//    three expanded spheres lies outside every other expanded sphere; one free placement is a
//    REGULAR facet, two free placements a SINGULAR facet (mirror pair);
//  * an edge (i,j) is REGULAR iff the circle where the two expanded spheres meet is partially
//    free (its free arcs end at the incident facet probes), SINGULAR iff the whole circle is free
//    and INTERIOR iff the circle is fully buried while the power face of (i,j) still meets the
//    disc bounded by the circle;
//  * an atom gets a PointCell iff it has a REGULAR/SINGULAR edge or no neighbour at all.
//
// The cell records themselves (probe centre formula, trimming planes and their orientation, the
// torus frame, the clipping sphere, the cutting-plane circulator and its acute/obtuse flags,
// the self-intersection planes) follow the reference formulas line by line.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../ns_types.h"
#include "host_api.h"
#include "patchset.h"

namespace {

const double kPi = 3.14159265358979323846264338327950288;
const double kTwoPi = 2.0 * kPi;

inline double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
inline void sub3(double* d, const double* a, const double* b) {
  d[0] = a[0] - b[0]; d[1] = a[1] - b[1]; d[2] = a[2] - b[2];
}
inline void cross3(double* d, const double* a, const double* b) {
  d[0] = a[1] * b[2] - a[2] * b[1];
  d[1] = a[2] * b[0] - a[0] * b[2];
  d[2] = a[0] * b[1] - a[1] * b[0];
}
// NORMALIZE_S semantics: divide by (norm + 1e-20).
inline void normalize_s(double* w, const double* v) {
  double t = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  w[0] = v[0] / (t + 1e-20); w[1] = v[1] / (t + 1e-20); w[2] = v[2] / (t + 1e-20);
}
inline double dist2(const double* a, const double* b) {
  return (a[0] - b[0]) * (a[0] - b[0]) + (a[1] - b[1]) * (a[1] - b[1]) + (a[2] - b[2]) * (a[2] - b[2]);
}
// Plane through three points, normalised (plane3points, src/tools.cpp:257-273).
void plane3(const double* p1, const double* p2, const double* p3, double* w) {
  w[0] = p1[1] * (p2[2] - p3[2]) + p2[1] * (p3[2] - p1[2]) + p3[1] * (p1[2] - p2[2]);
  w[1] = p1[2] * (p2[0] - p3[0]) + p2[2] * (p3[0] - p1[0]) + p3[2] * (p1[0] - p2[0]);
  w[2] = p1[0] * (p2[1] - p3[1]) + p2[0] * (p3[1] - p1[1]) + p3[0] * (p1[1] - p2[1]);
  w[3] = -dot3(w, p1);
  double norm = sqrt(dot3(w, w));
  w[0] /= norm; w[1] /= norm; w[2] /= norm; w[3] /= norm;
}
// Distance of a point to a plane (point2plane, src/tools.cpp:276-286).
double point_plane_dist(const double* p, const double* w) {
  double den = dot3(w, w);
  double d = sqrt(den);
  double val = dot3(w, p) + w[3];
  return fabs(val / d);
}
// Sign test of the two bounding planes of a torus sector (ConnollySurface::orientation,
// src/ConnollySurface.cpp:6108-6131).
bool orientation(const double* c1, const double* c2, const double* w1, const double* w2) {
  double b = dot3(w1, w2);
  double c = dot3(w2, w2);
  double w0[3];
  sub3(w0, c1, c2);
  double d = dot3(w1, w0);
  double e = dot3(w2, w0);
  return b * e < c * d;
}

struct Facet {
  double center[3];
  double planes[4][4];
  int id[3];
  bool singular;
  int mirror;      // index of the mirror facet, -1 if none
  bool in_si_map;  // takes part in the self-intersection map
  std::vector<double> si_planes;  // 4 per plane, already signed for this facet
};

struct Edge {
  int kind;  // NS_EDGE_REG or NS_EDGE_SING
  int i, j;
  double tc[3], clip_c[3], clip_r, r2_clip, bigR, rcoi, sir;
  double invrot[9];
  std::vector<double> planes;  // 4 per plane, stored with the sign used by the feasibility test
  std::vector<int8_t> flags;   // one per plane (first of pair meaningful)
};

struct Buried {
  int i, j;
  double clip_c[3], r2_clip;
};

template <class F>
void parallel_for(int64_t n, int nthreads, F fn) {
  if (nthreads <= 1 || n < 64) {
    for (int64_t i = 0; i < n; i++) fn(i, 0);
    return;
  }
  std::atomic<int64_t> next(0);
  std::vector<std::thread> th;
  const int64_t chunk = 32;
  for (int t = 0; t < nthreads; t++) {
    th.emplace_back([&, t]() {
      while (true) {
        int64_t s = next.fetch_add(chunk);
        if (s >= n) break;
        int64_t e = std::min(n, s + chunk);
        for (int64_t i = s; i < e; i++) fn(i, t);
      }
    });
  }
  for (auto& x : th) x.join();
}

// Torus quantities shared by BuildPointCells (buried neighbours) and BuildEdgeCells
// (src/ConnollySurface.cpp:553-650, 1296-1420).
struct TorusGeom {
  double tc[3], rcoi, bigR, u[3], v[3], w[3], clip_c[3], r2_clip;
};
void torus_geom(const double* c1, double w1, double r1, const double* c2, double w2, TorusGeom* g) {
  double diff[3];
  sub3(diff, c2, c1);
  double dij2 = dot3(diff, diff);
  double ratio = (w1 + dij2 - w2) * 0.5;
  double tt2 = w1 - ratio * ratio / dij2;
  g->bigR = sqrt(tt2);
  double cof = ratio / dij2;
  double rj2[3] = {cof * diff[0], cof * diff[1], cof * diff[2]};
  for (int d = 0; d < 3; d++) g->tc[d] = rj2[d] + c1[d];
  double tcv1 = dot3(rj2, rj2);
  g->rcoi = sqrt(w1 - tcv1);
  normalize_s(g->w, diff);
  double va[3] = {0, g->w[2], -g->w[1]};
  double vb[3] = {g->w[2], 0, -g->w[0]};
  normalize_s(g->u, va);
  double ct[3], vv[3];
  cross3(ct, va, vb);
  cross3(vv, ct, va);
  normalize_s(g->v, vv);
  double rp[3];
  for (int d = 0; d < 3; d++) rp[d] = g->tc[d] + g->rcoi * g->u[d];
  double t1[3], t2[3];
  sub3(t1, rp, c1);
  double pai = sqrt(dot3(t1, t1));
  sub3(t2, rp, c2);
  double paj = sqrt(dot3(t2, t2));
  double xx[3] = {t1[0] * (r1 / pai), t1[1] * (r1 / pai), t1[2] * (r1 / pai)};
  double coeff = pai / (pai + paj);
  double ctemp[3] = {coeff * diff[0], coeff * diff[1], coeff * diff[2]};
  for (int d = 0; d < 3; d++) g->clip_c[d] = ctemp[d] + c1[d];
  double tt[3];
  sub3(tt, xx, ctemp);
  g->r2_clip = dot3(tt, tt);
}

// Inverse of a 3x3 matrix by adjugate / determinant (INVERT_3X3).
void invert3(const double a[3][3], double* b) {
  double det = a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1]);
  det -= a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0]);
  det += a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
  double s = 1.0 / det;
  b[0 * 3 + 0] = s * (a[1][1] * a[2][2] - a[1][2] * a[2][1]);
  b[1 * 3 + 0] = s * (a[1][2] * a[2][0] - a[1][0] * a[2][2]);
  b[2 * 3 + 0] = s * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
  b[0 * 3 + 1] = s * (a[0][2] * a[2][1] - a[0][1] * a[2][2]);
  b[1 * 3 + 1] = s * (a[0][0] * a[2][2] - a[0][2] * a[2][0]);
  b[2 * 3 + 1] = s * (a[0][1] * a[2][0] - a[0][0] * a[2][1]);
  b[0 * 3 + 2] = s * (a[0][1] * a[1][2] - a[0][2] * a[1][1]);
  b[1 * 3 + 2] = s * (a[0][2] * a[1][0] - a[0][0] * a[1][2]);
  b[2 * 3 + 2] = s * (a[0][0] * a[1][1] - a[0][1] * a[1][0]);
}

}  // namespace

namespace {

struct SesBuilder {
  const double* at;
  int64_t n;
  double probe;
  int nthreads;
  std::vector<double> W;  // (r+probe)^2
  std::vector<int64_t> nb_off;
  std::vector<int32_t> nb;  // neighbours (expanded spheres overlapping), sorted
  std::vector<Facet> facets;
  std::vector<Edge> edges;
  std::vector<Buried> buried;
  int64_t n_errors = 0;

  const double* C(int64_t i) const { return at + 4 * i; }
  double R(int64_t i) const { return at[4 * i + 3] + probe; }

  void neighbours() {
    W.resize(n);
    double rmax = 0;
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int64_t i = 0; i < n; i++) {
      double r = at[4 * i + 3] + probe;
      W[i] = r * r;
      rmax = std::max(rmax, r);
      for (int d = 0; d < 3; d++) { lo[d] = std::min(lo[d], at[4 * i + d]); hi[d] = std::max(hi[d], at[4 * i + d]); }
    }
    double cs = std::max(2 * rmax, 1e-3);
    int64_t dims[3];
    for (int d = 0; d < 3; d++) dims[d] = std::max<int64_t>(1, (int64_t)floor((hi[d] - lo[d]) / cs) + 1);
    std::vector<int64_t> cell(n), cnt(dims[0] * dims[1] * dims[2] + 1, 0);
    auto cid = [&](const double* p, int64_t* c3) {
      for (int d = 0; d < 3; d++) c3[d] = std::min(dims[d] - 1, std::max<int64_t>(0, (int64_t)floor((p[d] - lo[d]) / cs)));
      return (c3[2] * dims[1] + c3[1]) * dims[0] + c3[0];
    };
    for (int64_t i = 0; i < n; i++) { int64_t c3[3]; cell[i] = cid(C(i), c3); cnt[cell[i] + 1]++; }
    for (size_t c = 1; c < cnt.size(); c++) cnt[c] += cnt[c - 1];
    std::vector<int32_t> sorted(n);
    std::vector<int64_t> fill(cnt.begin(), cnt.end() - 1);
    for (int64_t i = 0; i < n; i++) sorted[fill[cell[i]]++] = (int32_t)i;
    std::vector<std::vector<int32_t>> lists(n);
    parallel_for(n, nthreads, [&](int64_t i, int) {
      int64_t c3[3];
      cid(C(i), c3);
      std::vector<int32_t>& L = lists[i];
      for (int64_t dz = -1; dz <= 1; dz++)
        for (int64_t dy = -1; dy <= 1; dy++)
          for (int64_t dx = -1; dx <= 1; dx++) {
            int64_t x = c3[0] + dx, y = c3[1] + dy, z = c3[2] + dz;
            if (x < 0 || y < 0 || z < 0 || x >= dims[0] || y >= dims[1] || z >= dims[2]) continue;
            int64_t c = (z * dims[1] + y) * dims[0] + x;
            for (int64_t s = cnt[c]; s < cnt[c + 1]; s++) {
              int32_t j = sorted[s];
              if (j == i) continue;
              double rr = R(i) + R(j);
              if (dist2(C(i), C(j)) < rr * rr) L.push_back(j);
            }
          }
      std::sort(L.begin(), L.end());
    });
    nb_off.assign(n + 1, 0);
    for (int64_t i = 0; i < n; i++) nb_off[i + 1] = nb_off[i] + (int64_t)lists[i].size();
    nb.resize(nb_off[n]);
    for (int64_t i = 0; i < n; i++) std::copy(lists[i].begin(), lists[i].end(), nb.begin() + nb_off[i]);
  }

  // Expanded spheres of i and j meet in a proper circle.
  bool proper(int64_t i, int64_t j) const {
    double d2 = dist2(C(i), C(j));
    double dr = R(i) - R(j);
    double rs = R(i) + R(j);
    return d2 > dr * dr && d2 < rs * rs;
  }

  // Whether point p (a probe placement touching the expanded spheres of i, j, k) lies inside the
  // expanded sphere of another neighbour of i.  *hint is the neighbour that buried the previous
  // placement tested from i; neighbouring placements are mostly buried by the same sphere, so it
  // is tried first (the answer does not depend on the order).
  bool buried_point(const double* p, int64_t i, int64_t j, int64_t k, int64_t* hint = nullptr) const {
    if (hint && *hint >= 0 && *hint != j && *hint != k && dist2(p, C(*hint)) < W[*hint]) return true;
    for (int64_t s = nb_off[i]; s < nb_off[i + 1]; s++) {
      int64_t l = nb[s];
      if (l == j || l == k) continue;
      if (dist2(p, C(l)) < W[l]) {
        if (hint) *hint = l;
        return true;
      }
    }
    return false;
  }

  // Builds one facet cell (BuildFacetCells, src/ConnollySurface.cpp:1060-1112).
  void make_facet(Facet& f, const double* probe_c, const double* P1, const double* P2, const double* P3,
                  bool singular, int i, int j, int k) {
    f.center[0] = probe_c[0]; f.center[1] = probe_c[1]; f.center[2] = probe_c[2];
    f.id[0] = i; f.id[1] = j; f.id[2] = k;
    f.singular = singular;
    f.mirror = -1;
    f.in_si_map = false;
    double PP1[3], PP2[3], PP3[3], YY[3];
    if (singular) {
      for (int d = 0; d < 3; d++) { PP1[d] = P1[d]; PP2[d] = P2[d]; PP3[d] = P3[d]; }
    } else {
      sub3(YY, P1, probe_c); for (int d = 0; d < 3; d++) PP1[d] = probe_c[d] + 50000. * YY[d];
      sub3(YY, P2, probe_c); for (int d = 0; d < 3; d++) PP2[d] = probe_c[d] + 50000. * YY[d];
      sub3(YY, P3, probe_c); for (int d = 0; d < 3; d++) PP3[d] = probe_c[d] + 50000. * YY[d];
    }
    plane3(PP1, PP2, PP3, f.planes[0]);
    plane3(PP1, PP2, probe_c, f.planes[1]);
    plane3(PP2, PP3, probe_c, f.planes[2]);
    plane3(PP1, PP3, probe_c, f.planes[3]);
    double inner[3];
    for (int d = 0; d < 3; d++) inner[d] = ((1. / 3.) * (PP1[d] + PP2[d] + PP3[d]) + probe_c[d]) * 0.5;
    for (int ff = 0; ff < 4; ff++) {
      double orient = dot3(inner, f.planes[ff]);
      if (!(orient < -(f.planes[ff][3])))
        for (int d = 0; d < 4; d++) f.planes[ff][d] = -f.planes[ff][d];
    }
  }

  // Probe placements of a triple (src/ConnollySurface.cpp:934-995).
  bool probe_pair(const double* P1, const double* P2, const double* P3, double w1, double w2, double w3,
                  double* Q, double* n, double* coeff) const {
    double P12[3], P13[3], P23[3];
    sub3(P12, P2, P1); sub3(P13, P3, P1); sub3(P23, P3, P2);
    cross3(n, P12, P13);
    const double A = dot3(P12, P12), B = dot3(P23, P23), Cc = dot3(P13, P13);
    const double D = w1, E = w2, F = w3;
    const double X = D + E - A, Y = E + F - B, Z = D + F - Cc;
    const double Varg = 4. * D * E * F - F * X * X - D * Y * Y - E * Z * Z + X * Y * Z;
    if (!(Varg >= 0.)) return false;
    const double V = 1. / 12. * sqrt(Varg);
    const double G = dot3(P12, P13);
    const double H = dot3(n, n);
    if (!(H > 0)) return false;
    const double I = dot3(P2, P2) - dot3(P1, P1);
    const double J = dot3(P3, P3) - dot3(P1, P1);
    const double K = dot3(n, P1);
    const double L = I - E + D;
    const double M = J - F + D;
    const double S = Cc * L - G * M;
    const double T = A * M - G * L;
    for (int d = 0; d < 3; d++) Q[d] = (K * n[d] + 0.5 * (S * P12[d] + T * P13[d])) / H;
    *coeff = (6.0 * V) / H;
    return true;
  }

  void build_facets() {
    std::vector<std::vector<Facet>> per_atom(n);
    parallel_for(n, nthreads, [&](int64_t i, int) {
      std::vector<Facet>& out = per_atom[i];
      int64_t hint = -1;
      const int32_t* ni = nb.data() + nb_off[i];
      int64_t nni = nb_off[i + 1] - nb_off[i];
      for (int64_t a = 0; a < nni; a++) {
        int64_t j = ni[a];
        if (j <= i || !proper(i, j)) continue;
        const int32_t* nj = nb.data() + nb_off[j];
        int64_t nnj = nb_off[j + 1] - nb_off[j];
        int64_t b = a + 1, c = 0;
        while (b < nni && c < nnj) {
          if (ni[b] < nj[c]) { b++; continue; }
          if (ni[b] > nj[c]) { c++; continue; }
          int64_t k = ni[b];
          b++; c++;
          if (k <= j || !proper(i, k) || !proper(j, k)) continue;
          double Q[3], nn[3], coeff;
          if (!probe_pair(C(i), C(j), C(k), W[i], W[j], W[k], Q, nn, &coeff)) continue;
          double pp[3], pm[3];
          for (int d = 0; d < 3; d++) { pp[d] = Q[d] + coeff * nn[d]; pm[d] = Q[d] - coeff * nn[d]; }
          bool fp = !buried_point(pp, i, j, k, &hint);
          bool fm = !buried_point(pm, i, j, k, &hint);
          if (fp && fm) {
            Facet f1, f2;
            make_facet(f1, pp, C(i), C(j), C(k), true, (int)i, (int)j, (int)k);
            make_facet(f2, pm, C(i), C(j), C(k), true, (int)i, (int)j, (int)k);
            f1.mirror = 1;  // relative: resolved after merge
            f2.mirror = -2;
            out.push_back(f1);
            out.push_back(f2);
          } else if (fp || fm) {
            Facet f1;
            make_facet(f1, fp ? pp : pm, C(i), C(j), C(k), false, (int)i, (int)j, (int)k);
            double plane[4];
            plane3(C(i), C(j), C(k), plane);
            f1.in_si_map = point_plane_dist(f1.center, plane) <= probe;
            out.push_back(f1);
          }
        }
      }
    });
    for (int64_t i = 0; i < n; i++)
      for (auto& f : per_atom[i]) {
        int idx = (int)facets.size();
        if (f.mirror == 1) f.mirror = idx + 1;
        else if (f.mirror == -2) f.mirror = idx - 1;
        facets.push_back(std::move(f));
      }
  }

  // Self-intersections between probe patches (RemoveSelfIntersections,
  // src/ConnollySurface.cpp:1928-2035): every facet is tested against the regular facets whose
  // probe centre is within one probe radius from the atoms' plane.
  void self_intersections() {
    const double p2 = probe * probe;
    std::vector<int> mapped;
    for (size_t f = 0; f < facets.size(); f++)
      if (facets[f].in_si_map) mapped.push_back((int)f);
    if (mapped.empty()) return;
    double cs = 2 * probe;
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (auto& f : facets)
      for (int d = 0; d < 3; d++) { lo[d] = std::min(lo[d], f.center[d]); hi[d] = std::max(hi[d], f.center[d]); }
    int64_t dims[3];
    for (int d = 0; d < 3; d++) dims[d] = std::max<int64_t>(1, (int64_t)floor((hi[d] - lo[d]) / cs) + 1);
    auto cid3 = [&](const double* p, int64_t* c3) {
      for (int d = 0; d < 3; d++) c3[d] = std::min(dims[d] - 1, std::max<int64_t>(0, (int64_t)floor((p[d] - lo[d]) / cs)));
    };
    std::unordered_map<int64_t, std::vector<int>> grid;
    for (int f : mapped) {
      int64_t c3[3];
      cid3(facets[f].center, c3);
      grid[(c3[2] * dims[1] + c3[1]) * dims[0] + c3[0]].push_back(f);
    }
    // Collect (fc1, fc2) pairs first, then apply in fc1 order so that the plane lists are
    // deterministic.
    std::vector<std::vector<int>> partner(facets.size());
    parallel_for((int64_t)facets.size(), nthreads, [&](int64_t f1, int) {
      int64_t c3[3];
      cid3(facets[f1].center, c3);
      for (int64_t dz = -1; dz <= 1; dz++)
        for (int64_t dy = -1; dy <= 1; dy++)
          for (int64_t dx = -1; dx <= 1; dx++) {
            int64_t x = c3[0] + dx, y = c3[1] + dy, z = c3[2] + dz;
            if (x < 0 || y < 0 || z < 0 || x >= dims[0] || y >= dims[1] || z >= dims[2]) continue;
            auto it = grid.find((z * dims[1] + y) * dims[0] + x);
            if (it == grid.end()) continue;
            for (int f2 : it->second) {
              if (f2 == f1) continue;
              if (dist2(facets[f1].center, facets[f2].center) < 4 * p2) partner[f1].push_back(f2);
            }
          }
      std::sort(partner[f1].begin(), partner[f1].end());
    });
    for (size_t f1 = 0; f1 < facets.size(); f1++)
      for (int f2 : partner[f1]) {
        const double* c1 = facets[f1].center;
        const double* c2 = facets[f2].center;
        double ref[3], dir[3], tmp[3];
        for (int d = 0; d < 3; d++) ref[d] = (c2[d] + c1[d]) * 0.5;
        sub3(tmp, c1, c2);
        normalize_s(dir, tmp);
        double bias = -dot3(dir, ref);
        double plane[4] = {dir[0], dir[1], dir[2], bias};
        double orient = dot3(c1, plane);
        if (!(orient < -plane[3])) { plane[0] = -dir[0]; plane[1] = -dir[1]; plane[2] = -dir[2]; plane[3] = -bias; }
        for (int d = 0; d < 4; d++) facets[f1].si_planes.push_back(plane[d]);
        for (int d = 0; d < 4; d++) facets[f2].si_planes.push_back(-plane[d]);
      }
  }

  // Index of the facet plane that contains the atom pair (a,b) (plane_indices lookup).
  static const double* edge_plane(const Facet& f, int a, int b) {
    static const int pi[3][2] = {{0, 1}, {1, 2}, {0, 2}};
    for (int ii = 0; ii < 3; ii++) {
      int i1 = f.id[pi[ii][0]], i2 = f.id[pi[ii][1]];
      if ((i1 == a && i2 == b) || (i1 == b && i2 == a)) return f.planes[ii + 1];
    }
    return nullptr;
  }

  // Power face of (i,j) meets the disc of the circle of intersection: the edge belongs to the
  // alpha complex.  Used for fully buried circles only.
  bool power_face_meets_disc(int64_t i, int64_t j, const TorusGeom& g) const {
    double r = g.rcoi;
    const int32_t* ni = nb.data() + nb_off[i];
    int64_t nni = nb_off[i + 1] - nb_off[i];
    const int32_t* nj = nb.data() + nb_off[j];
    int64_t nnj = nb_off[j + 1] - nb_off[j];
    {
      // the disc centre (the origin of the disc plane) inside every neighbour's half-plane, by a
      // margin well above rounding: it then lies inside the clipped polygon, which the full
      // clipping below would find too
      bool centre_in = true;
      int64_t b = 0, c = 0;
      while (centre_in && b < nni && c < nnj) {
        if (ni[b] < nj[c]) { b++; continue; }
        if (ni[b] > nj[c]) { c++; continue; }
        const int64_t k = ni[b];
        b++; c++;
        double e[3];
        sub3(e, g.tc, C(k));
        const double ee = dot3(e, e);
        const double ga = ee - W[k] + r * r;
        if (!(ga > 1e-9 * (ee + W[k] + r * r))) centre_in = false;
      }
      if (centre_in) return true;
    }
    // the clipped polygon: each clip adds at most one vertex, so 4 + (common neighbours) bound it;
    // two fixed buffers serve every call that fits, a heap pair the rest
    constexpr size_t kStack = 512;
    double sbuf[2][kStack];
    std::vector<double> hbuf[2];
    const int64_t nmax = 2 * (4 + std::min(nb_off[i + 1] - nb_off[i], nb_off[j + 1] - nb_off[j]) + 2);
    double* polyp = sbuf[0];
    double* nextp = sbuf[1];
    if (nmax > (int64_t)kStack) {
      hbuf[0].resize(nmax);
      hbuf[1].resize(nmax);
      polyp = hbuf[0].data();
      nextp = hbuf[1].data();
    }
    size_t plen = 8, nlen = 0;
    {
      const double init[8] = {-r, -r, r, -r, r, r, -r, r};
      for (int q = 0; q < 8; q++) polyp[q] = init[q];
    }
    int64_t b = 0, c = 0;
    while (b < nni && c < nnj) {
      if (ni[b] < nj[c]) { b++; continue; }
      if (ni[b] > nj[c]) { c++; continue; }
      int64_t k = ni[b];
      b++; c++;
      double e[3];
      sub3(e, g.tc, C(k));
      double al = -2 * dot3(g.u, e), be = -2 * dot3(g.v, e);
      double ga = dot3(e, e) - W[k] + r * r;
      nlen = 0;
      size_t m = plen / 2;
      for (size_t q = 0; q < m; q++) {
        double ax = polyp[2 * q], ay = polyp[2 * q + 1];
        double bx = polyp[2 * ((q + 1) % m)], by = polyp[2 * ((q + 1) % m) + 1];
        double fa = al * ax + be * ay - ga, fb = al * bx + be * by - ga;
        if (fa <= 0) { nextp[nlen++] = ax; nextp[nlen++] = ay; }
        if ((fa <= 0) != (fb <= 0)) {
          double t = fa / (fa - fb);
          nextp[nlen++] = ax + t * (bx - ax);
          nextp[nlen++] = ay + t * (by - ay);
        }
      }
      std::swap(polyp, nextp);
      plen = nlen;
      if (plen < 6) return false;
    }
    const double* poly = polyp;
    // distance from the disc centre to the clipped polygon
    size_t m = plen / 2;
    bool inside = true;
    double best = INFINITY;
    for (size_t q = 0; q < m; q++) {
      double ax = poly[2 * q], ay = poly[2 * q + 1];
      double bx = poly[2 * ((q + 1) % m)], by = poly[2 * ((q + 1) % m) + 1];
      double ex = bx - ax, ey = by - ay;
      if (ex * (-ay) - ey * (-ax) < 0) inside = false;
      double l2 = ex * ex + ey * ey;
      double t = l2 > 0 ? std::min(1.0, std::max(0.0, -(ax * ex + ay * ey) / l2)) : 0;
      double px = ax + t * ex, py = ay + t * ey;
      best = std::min(best, px * px + py * py);
    }
    // polygon orientation may be clockwise after clipping degenerate squares: test both windings
    if (!inside) {
      bool inside2 = true;
      for (size_t q = 0; q < m; q++) {
        double ax = poly[2 * q], ay = poly[2 * q + 1];
        double bx = poly[2 * ((q + 1) % m)], by = poly[2 * ((q + 1) % m) + 1];
        if ((bx - ax) * (-ay) - (by - ay) * (-ax) > 0) inside2 = false;
      }
      inside = inside2;
    }
    return inside || best < r * r;
  }

  void build_edges() {
    // incidence: (pair key, facet index) sorted by key, stable in facet order
    std::vector<std::pair<int64_t, int>> inc;
    inc.reserve(facets.size() * 3);
    for (size_t f = 0; f < facets.size(); f++) {
      const int* id = facets[f].id;
      int pr[3][2] = {{id[0], id[1]}, {id[0], id[2]}, {id[1], id[2]}};
      for (auto& p : pr) {
        int a = std::min(p[0], p[1]), b = std::max(p[0], p[1]);
        inc.push_back({(int64_t)a * n + b, (int)f});
      }
    }
    std::stable_sort(inc.begin(), inc.end(), [](const std::pair<int64_t, int>& x, const std::pair<int64_t, int>& y) {
      return x.first < y.first;
    });
    std::vector<std::vector<Edge>> per_atom(n);
    std::vector<std::vector<Buried>> per_atom_b(n);
    std::vector<int64_t> errs(std::max(1, nthreads), 0);
    parallel_for(n, nthreads, [&](int64_t i, int tid) {
      // the incidence entries of atom i's pairs (i, j > i) are contiguous and ascending in j, as
      // are i's neighbours: one search, then a forward walk
      auto it = std::lower_bound(inc.begin(), inc.end(), std::make_pair(i * n, -1));
      std::vector<int> fcv;
      for (int64_t s = nb_off[i]; s < nb_off[i + 1]; s++) {
        int64_t j = nb[s];
        if (j <= i) continue;
        const int64_t key = i * n + j;
        while (it != inc.end() && it->first < key) ++it;
        if (!proper(i, j)) continue;
        fcv.clear();
        for (auto jt = it; jt != inc.end() && jt->first == key; ++jt) fcv.push_back(jt->second);
        TorusGeom g;
        torus_geom(C(i), W[i], at[4 * i + 3], C(j), W[j], &g);
        if (fcv.empty()) {
          double rp[3];
          for (int d = 0; d < 3; d++) rp[d] = g.tc[d] + g.rcoi * g.u[d];
          if (buried_point(rp, i, j, j)) {
            if (power_face_meets_disc(i, j, g)) {
              Buried bb;
              bb.i = (int)i; bb.j = (int)j;
              for (int d = 0; d < 3; d++) bb.clip_c[d] = g.clip_c[d];
              bb.r2_clip = g.r2_clip;
              per_atom_b[i].push_back(bb);
            }
            continue;
          }
        } else if (fcv.size() % 2 != 0) {
          errs[tid]++;
          continue;
        }
        Edge e;
        e.kind = fcv.empty() ? NS_EDGE_SING : NS_EDGE_REG;
        e.i = (int)i; e.j = (int)j;
        for (int d = 0; d < 3; d++) { e.tc[d] = g.tc[d]; e.clip_c[d] = g.clip_c[d]; }
        e.r2_clip = g.r2_clip;
        e.clip_r = sqrt(g.r2_clip);
        e.bigR = g.bigR;
        e.rcoi = g.rcoi;
        e.sir = (g.bigR >= probe) ? -1.0 : sqrt(probe * probe - g.bigR * g.bigR);
        double Rot[3][3] = {{g.v[0], g.u[0], g.w[0]}, {g.v[1], g.u[1], g.w[1]}, {g.v[2], g.u[2], g.w[2]}};
        invert3(Rot, e.invrot);
        if (!fcv.empty() && !cutting_planes(e, fcv)) { errs[tid]++; continue; }
        per_atom[i].push_back(std::move(e));
      }
    });
    for (auto x : errs) n_errors += x;
    for (int64_t i = 0; i < n; i++) {
      for (auto& e : per_atom[i]) edges.push_back(std::move(e));
      for (auto& b : per_atom_b[i]) buried.push_back(b);
    }
  }

  void push_pair(Edge& e, const double* P1, const double* P2, bool flag) {
    // stored negated: the reference tests -(P.x + d) against the raw facet planes
    for (int d = 0; d < 4; d++) e.planes.push_back(-P1[d]);
    for (int d = 0; d < 4; d++) e.planes.push_back(-P2[d]);
    e.flags.push_back(flag ? 1 : 0);
    e.flags.push_back(0);
  }

  // Cutting planes of a REGULAR edge (src/ConnollySurface.cpp:1574-1850).
  bool cutting_planes(Edge& e, const std::vector<int>& fcv) {
    int index = (int)fcv.size();
    int a = e.i, b = e.j;
    if (index == 2) {
      const double* P0 = edge_plane(facets[fcv[0]], a, b);
      const double* P1 = edge_plane(facets[fcv[1]], a, b);
      if (!P0 || !P1) return false;
      bool acute = !orientation(facets[fcv[0]].center, facets[fcv[1]].center, P0, P1);
      push_pair(e, P0, P1, acute);
      return true;
    }
    // sort the probes along the circle of intersection (sortProbes, :6134-6169)
    std::vector<int> sorted(index);
    {
      double ref[3], temp[3], t0[3], vs[3], ws[3];
      sub3(t0, facets[fcv[0]].center, e.tc);
      normalize_s(ref, t0);
      sub3(t0, facets[fcv[1]].center, e.tc);
      normalize_s(temp, t0);
      cross3(vs, ref, temp);
      cross3(ws, vs, ref);
      std::vector<std::pair<double, int>> ang;
      for (int q = 1; q < index; q++) {
        sub3(t0, facets[fcv[q]].center, e.tc);
        normalize_s(temp, t0);
        double angle = atan2(dot3(ws, temp), dot3(ref, temp));
        if (angle < 0) angle = kTwoPi + angle;
        ang.push_back({angle, q});
      }
      std::stable_sort(ang.begin(), ang.end(), [](const std::pair<double, int>& x, const std::pair<double, int>& y) {
        return x.first < y.first;
      });
      sorted[0] = 0;
      for (int q = 1; q < index; q++) sorted[q] = ang[q - 1].second;
    }
    int start_index = 0, direction = 0;
    for (int u = 0; u < index; u++) {
      const Facet& f = facets[fcv[sorted[u]]];
      if (f.singular) {
        start_index = u;
        int nx = (u + 1) % index, pv = (index + u - 1) % index;
        if (f.mirror == fcv[sorted[nx]]) direction = -2;
        else if (f.mirror == fcv[sorted[pv]]) direction = +2;
        else return false;
        break;
      }
    }
    if (direction == 0) {
      const double* c1 = facets[fcv[sorted[0]]].center;
      const double* c2 = facets[fcv[sorted[1]]].center;
      double mid2[3];
      for (int d = 0; d < 3; d++) mid2[d] = (c1[d] + c2[d]) * 0.5 - e.tc[d];
      const double* P = edge_plane(facets[fcv[sorted[0]]], a, b);
      if (!P) return false;
      double plane[3] = {-P[0], -P[1], -P[2]};
      double test = -dot3(mid2, plane);
      start_index = 0;
      direction = (test > 0) ? +2 : -2;
    }
    int cp1 = start_index;
    int cp2 = (index + start_index + (direction >> 1)) % index;
    for (int guard = 0; guard <= index; guard++) {
      const Facet& f1 = facets[fcv[sorted[cp1]]];
      const Facet& f2 = facets[fcv[sorted[cp2]]];
      const double* P1 = edge_plane(f1, a, b);
      const double* P2 = edge_plane(f2, a, b);
      if (!P1 || !P2) return false;
      bool flag = !orientation(f1.center, f2.center, P1, P2);
      push_pair(e, P1, P2, flag);
      cp1 += direction;
      cp1 = (index + cp1) % index;
      cp2 = (index + cp1 + (direction >> 1)) % index;
      if (cp1 == start_index) return true;
    }
    return false;
  }

  void emit(NsPatchSet* ps) {
    // point cells first (atom order), then facets, then edges, as the reference sesComplex
    std::vector<std::vector<double>> clip(n);
    std::vector<char> exposed(n, 0);
    for (auto& e : edges) {
      exposed[e.i] = exposed[e.j] = 1;
      double s[4] = {e.clip_c[0], e.clip_c[1], e.clip_c[2], e.r2_clip};
      clip[e.i].insert(clip[e.i].end(), s, s + 4);
      clip[e.j].insert(clip[e.j].end(), s, s + 4);
    }
    for (int64_t i = 0; i < n; i++)
      if (nb_off[i + 1] == nb_off[i]) exposed[i] = 1;
    std::vector<std::vector<double>> bclip(n);
    for (auto& b : buried) {
      double s[4] = {b.clip_c[0], b.clip_c[1], b.clip_c[2], b.r2_clip};
      bclip[b.i].insert(bclip[b.i].end(), s, s + 4);
      bclip[b.j].insert(bclip[b.j].end(), s, s + 4);
    }
    double rec[NS_PATCH_F64];
    for (int64_t i = 0; i < n; i++) {
      if (!exposed[i]) continue;
      memset(rec, 0, sizeof rec);
      rec[0] = at[4 * i]; rec[1] = at[4 * i + 1]; rec[2] = at[4 * i + 2]; rec[3] = at[4 * i + 3];
      rec[8] = -1.0;
      std::vector<double> all = clip[i];
      all.insert(all.end(), bclip[i].begin(), bclip[i].end());
      ps->add_patch(NS_POINT, rec, all.data(), nullptr, (int64_t)all.size() / 4, (int32_t)i, -1, -1);
    }
    for (auto& f : facets) {
      memset(rec, 0, sizeof rec);
      rec[0] = f.center[0]; rec[1] = f.center[1]; rec[2] = f.center[2]; rec[3] = probe;
      rec[8] = -1.0;
      std::vector<double> pl;
      for (int q = f.singular ? 0 : 1; q < 4; q++) pl.insert(pl.end(), f.planes[q], f.planes[q] + 4);
      pl.insert(pl.end(), f.si_planes.begin(), f.si_planes.end());
      ps->add_patch(f.singular ? NS_FACE_SING : NS_FACE_REG, rec, pl.data(), nullptr, (int64_t)pl.size() / 4, f.id[0],
                    f.id[1], f.id[2]);
    }
    for (auto& e : edges) {
      memset(rec, 0, sizeof rec);
      rec[0] = e.clip_c[0]; rec[1] = e.clip_c[1]; rec[2] = e.clip_c[2]; rec[3] = e.clip_r;
      rec[4] = e.tc[0]; rec[5] = e.tc[1]; rec[6] = e.tc[2]; rec[7] = e.bigR; rec[8] = e.sir;
      for (int q = 0; q < 9; q++) rec[9 + q] = e.invrot[q];
      ps->add_patch(e.kind, rec, e.planes.data(), e.flags.data(), (int64_t)e.planes.size() / 4, e.i, e.j, -1);
    }
  }
};

}  // namespace

extern "C" {

int nsg_ses_build(const double* atoms_xyzr, int64_t n_atoms, double probe_radius, int n_threads,
                  NsPatchSet** out) {
  if (!atoms_xyzr || !out || probe_radius <= 0) return NSG_ERR_ARG;
  if (n_atoms <= 0) return NSG_ERR_EMPTY;
  if (n_threads <= 0) n_threads = (int)std::max(1u, std::thread::hardware_concurrency());
  SesBuilder b;
  b.at = atoms_xyzr;
  b.n = n_atoms;
  b.probe = probe_radius;
  b.nthreads = n_threads;
  b.neighbours();
  b.build_facets();
  b.self_intersections();
  b.build_edges();
  NsPatchSet* ps = new NsPatchSet();
  b.emit(ps);
  *out = ps;
  return b.n_errors ? NSG_ERR_GEOMETRY : NSG_OK;
}

int nsg_patchset_info(const NsPatchSet* ps, int64_t* n_patches, int64_t* n_pool, int64_t counts[5]) {
  if (!ps) return NSG_ERR_ARG;
  if (n_patches) *n_patches = (int64_t)ps->i32.size() / NS_PATCH_I32;
  if (n_pool) *n_pool = (int64_t)ps->pool_flag.size();
  if (counts)
    for (int k = 0; k < 5; k++) counts[k] = ps->counts[k];
  return NSG_OK;
}

int nsg_patchset_kind_counts(const NsPatchSet* ps, int64_t* counts, int n) {
  if (!ps || !counts || n < 0) return NSG_ERR_ARG;
  for (int k = 0; k < n; k++) counts[k] = k < NS_KIND_COUNT ? ps->counts[k] : 0;
  return NSG_OK;
}

int nsg_patchset_export(const NsPatchSet* ps, double* f64, int32_t* i32, double* pool, int8_t* pool_flag) {
  if (!ps) return NSG_ERR_ARG;
  if (f64) memcpy(f64, ps->f64.data(), ps->f64.size() * sizeof(double));
  if (i32) memcpy(i32, ps->i32.data(), ps->i32.size() * sizeof(int32_t));
  if (pool) memcpy(pool, ps->pool.data(), ps->pool.size() * sizeof(double));
  if (pool_flag) memcpy(pool_flag, ps->pool_flag.data(), ps->pool_flag.size());
  return NSG_OK;
}

int nsg_patchset_atoms(const NsPatchSet* ps, int32_t* out) {
  if (!ps || !out) return NSG_ERR_ARG;
  memcpy(out, ps->atoms.data(), ps->atoms.size() * sizeof(int32_t));
  return NSG_OK;
}

void nsg_patchset_free(NsPatchSet* ps) { delete ps; }

}  // extern "C"
