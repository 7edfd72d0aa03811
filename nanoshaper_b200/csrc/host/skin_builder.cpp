// Skin surface patch construction on the host: the mixed complex of the weighted atoms and one
// quadric patch per mixed cell.
//
// The reference (SkinSurface::buildSkinCGAL, src/SkinSurface.cpp:1271-1812) weights every atom by
// r^2/s, adds six dummy points of weight -1 on the axes of an enlarged bounding box, builds the
// CGAL regular triangulation, and derives four kinds of mixed cells:
//   Del3Cell per tetrahedron   (BuildDelaunayTetraCells, :348-480): reduced tetrahedron, sphere
//   Del0Cell per atom          (BuildDelaunayPointCells, :482-566): reduced Voronoi cell, atom sphere
//   Del1Cell per Delaunay edge (BuildDelaunayEdgeCells, :568-892): prism around the edge, hyperboloid
//   Del2Cell per Delaunay facet (BuildDelaunayFacetCells, :894-1208): triangular prism, hyperboloid
// with reduced points p + s (v - p) (p an atom of a tetrahedron, v the tetrahedron's weighted
// circumcentre), the cells' planes through reduced points oriented towards the cell's inside, and
// cells that touch a dummy point skipped (QUADRIC_CULLING).
//
// CGAL is not available here, so the regular triangulation is this file's own: incremental
// insertion (cavity of the tetrahedra whose orthosphere the new weighted point is in conflict
// with, re-starred from the point) with exact predicates.  The predicates decide on coordinates
// snapped to a power-of-two grid (2^-24 A for molecules within 1 km... of their centre) and on
// weights snapped to its square, evaluated exactly in 128/256-bit integer arithmetic; ties count
// as no conflict.  The geometry of the cells (circumcentres, reduced points, planes, quadrics) is
// computed in double precision from the original coordinates.  The quadrics are written from the
// closed forms of the reference's cell frames: sphere (|x - c|^2 - rho^2) for Del0 and Del3, and
// the surfaces of revolution -(o.y)^2/(1-s) + (|y|^2 - (o.y)^2)/s - R (Del1, o along the edge) and
// -(|y|^2 - (o.y)^2)/(1-s) + (o.y)^2/s - R (Del2, o normal to the facet), y = x - focus, which are
// the reference's Cinv^T M Cinv with M = diag(-1/(1-s), 1/s, 1/s, -R) and diag(-1/(1-s), -1/(1-s),
// 1/s, -R) in frames whose first (Del1) or last (Del2) axis is o.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <unordered_map>
#include <vector>

#include "../ns_types.h"
#include "host_api.h"
#include "patchset.h"

namespace {

typedef __int128 i128;
typedef unsigned __int128 u128;

// ---------------------------------------------------------------------------------------------
// Exact integer predicates.

// Signed 256-bit accumulator (two's complement, little-endian 64-bit limbs).
struct I256 {
  uint64_t w[4] = {0, 0, 0, 0};
};

I256 from_u128(u128 v) {
  I256 r;
  r.w[0] = (uint64_t)v;
  r.w[1] = (uint64_t)(v >> 64);
  return r;
}

I256 neg256(const I256& a) {
  I256 r;
  unsigned carry = 1;
  for (int i = 0; i < 4; i++) {
    uint64_t x = ~a.w[i];
    uint64_t y = x + carry;
    carry = (carry && y == 0) ? 1u : 0u;
    r.w[i] = y;
  }
  return r;
}

I256 add256(const I256& a, const I256& b) {
  I256 r;
  unsigned carry = 0;
  for (int i = 0; i < 4; i++) {
    u128 s = (u128)a.w[i] + b.w[i] + carry;
    r.w[i] = (uint64_t)s;
    carry = (unsigned)(s >> 64);
  }
  return r;
}

// a * b exactly, |a|, |b| < 2^127.
I256 mul128(i128 a, i128 b) {
  const bool neg = (a < 0) != (b < 0);
  const u128 ua = a < 0 ? (u128)(-a) : (u128)a;
  const u128 ub = b < 0 ? (u128)(-b) : (u128)b;
  const uint64_t a0 = (uint64_t)ua, a1 = (uint64_t)(ua >> 64);
  const uint64_t b0 = (uint64_t)ub, b1 = (uint64_t)(ub >> 64);
  const u128 p00 = (u128)a0 * b0, p01 = (u128)a0 * b1, p10 = (u128)a1 * b0, p11 = (u128)a1 * b1;
  I256 r = from_u128(p00);
  I256 mid = from_u128(p01);
  mid = add256(mid, from_u128(p10));  // < 2^129: fits in limbs 0..2
  // shift mid by 64 bits
  I256 ms;
  ms.w[1] = mid.w[0];
  ms.w[2] = mid.w[1];
  ms.w[3] = mid.w[2];
  r = add256(r, ms);
  I256 hs;
  hs.w[2] = (uint64_t)p11;
  hs.w[3] = (uint64_t)(p11 >> 64);
  r = add256(r, hs);
  return neg ? neg256(r) : r;
}

int sign256(const I256& a) {
  if ((int64_t)a.w[3] < 0) return -1;
  return (a.w[0] | a.w[1] | a.w[2] | a.w[3]) ? 1 : 0;
}

struct IPoint {
  int64_t x[3];
  int64_t w;  // weight in units of the squared snapping step
};

// 3x3 determinant of integer rows (entries below 2^36 in magnitude: exact in 128 bits).
i128 det3(const int64_t* a, const int64_t* b, const int64_t* c) {
  return (i128)a[0] * ((i128)b[1] * c[2] - (i128)b[2] * c[1]) - (i128)a[1] * ((i128)b[0] * c[2] - (i128)b[2] * c[0]) +
         (i128)a[2] * ((i128)b[0] * c[1] - (i128)b[1] * c[0]);
}

// Sign of det[b - a, c - a, d - a]: positive when d lies on the positive side of (a, b, c).
int orient3d(const IPoint& a, const IPoint& b, const IPoint& c, const IPoint& d) {
  int64_t u[3], v[3], w[3];
  for (int k = 0; k < 3; k++) {
    u[k] = b.x[k] - a.x[k];
    v[k] = c.x[k] - a.x[k];
    w[k] = d.x[k] - a.x[k];
  }
  i128 r = det3(u, v, w);
  return r > 0 ? 1 : (r < 0 ? -1 : 0);
}

// Conflict of weighted point p with the orthosphere of the positively oriented tetrahedron
// (a, b, c, d): the lifted determinant | q - p, |q - p|^2 - (w_q - w_p) | over q = a, b, c, d is
// negative exactly when p's power distance to the orthosphere is below its weight.
bool in_conflict(const IPoint& a, const IPoint& b, const IPoint& c, const IPoint& d, const IPoint& p) {
  const IPoint* q[4] = {&a, &b, &c, &d};
  int64_t r[4][3];
  i128 l[4];
  for (int i = 0; i < 4; i++) {
    i128 s = 0;
    for (int k = 0; k < 3; k++) {
      r[i][k] = q[i]->x[k] - p.x[k];
      s += (i128)r[i][k] * r[i][k];
    }
    l[i] = s - ((i128)q[i]->w - p.w);
  }
  // expansion along the lifted column: sum_i (-1)^(i+3) l_i M_i, M_i the minor without row i
  I256 acc;
  for (int i = 0; i < 4; i++) {
    const int64_t* rows[3];
    int n = 0;
    for (int j = 0; j < 4; j++)
      if (j != i) rows[n++] = r[j];
    i128 m = det3(rows[0], rows[1], rows[2]);
    I256 t = mul128(l[i], m);
    if (((i + 3) & 1) != 0) t = neg256(t);
    acc = add256(acc, t);
  }
  return sign256(acc) < 0;
}

// ---------------------------------------------------------------------------------------------
// Regular triangulation by incremental insertion.

struct Tet {
  int v[4];
  int n[4];  // neighbour across the face opposite v[i]; -1 on the hull
  bool alive;
};

struct RegularTriangulation {
  std::vector<IPoint> P;
  std::vector<Tet> T;
  std::vector<int> free_list;
  std::vector<int> mark;  // per tet: insertion stamp of the current cavity
  int stamp = 0;
  int last = 0;
  uint32_t rng = 12345u;
  int n_errors = 0;

  int orient_tet(const Tet& t) const { return orient3d(P[t.v[0]], P[t.v[1]], P[t.v[2]], P[t.v[3]]); }
  bool conflict(int ti, int pi) const {
    const Tet& t = T[ti];
    return in_conflict(P[t.v[0]], P[t.v[1]], P[t.v[2]], P[t.v[3]], P[pi]);
  }

  int new_tet(int a, int b, int c, int d) {
    int id;
    if (!free_list.empty()) {
      id = free_list.back();
      free_list.pop_back();
    } else {
      id = (int)T.size();
      T.push_back(Tet());
      mark.push_back(0);
    }
    Tet& t = T[id];
    t.v[0] = a; t.v[1] = b; t.v[2] = c; t.v[3] = d;
    t.n[0] = t.n[1] = t.n[2] = t.n[3] = -1;
    t.alive = true;
    mark[id] = 0;
    return id;
  }

  // The four tetrahedra of an octahedron around its diagonal (i, j); ring in cyclic order.
  void octahedron(int i, int j, const int ring[4]) {
    int ids[4];
    for (int k = 0; k < 4; k++) {
      int a = i, b = j, c = ring[k], d = ring[(k + 1) & 3];
      ids[k] = new_tet(a, b, c, d);
      if (orient_tet(T[ids[k]]) < 0) std::swap(T[ids[k]].v[0], T[ids[k]].v[1]);
    }
    link_all(ids, 4);
  }

  // Links the faces of the given tetrahedra that share three vertices.
  void link_all(const int* ids, int n) {
    for (int a = 0; a < n; a++)
      for (int fa = 0; fa < 4; fa++) {
        if (T[ids[a]].n[fa] >= 0) continue;
        for (int b = 0; b < n; b++) {
          if (b == a) continue;
          for (int fb = 0; fb < 4; fb++)
            if (same_face(T[ids[a]], fa, T[ids[b]], fb)) {
              T[ids[a]].n[fa] = ids[b];
              T[ids[b]].n[fb] = ids[a];
            }
        }
      }
  }

  static bool same_face(const Tet& a, int fa, const Tet& b, int fb) {
    int x[3], y[3], nx = 0, ny = 0;
    for (int k = 0; k < 4; k++) {
      if (k != fa) x[nx++] = a.v[k];
      if (k != fb) y[ny++] = b.v[k];
    }
    std::sort(x, x + 3);
    std::sort(y, y + 3);
    return x[0] == y[0] && x[1] == y[1] && x[2] == y[2];
  }

  // Walk from `start` to a tetrahedron containing point pi (all four faces see it inside or on).
  int locate(int pi, int start) {
    int t = start;
    const int64_t limit = 8 * (int64_t)T.size() + 1000;
    for (int64_t step = 0; step < limit; step++) {
      rng = rng * 1664525u + 1013904223u;
      const int off = (int)(rng >> 30);
      bool moved = false;
      for (int q = 0; q < 4; q++) {
        const int i = (q + off) & 3;
        const Tet& tt = T[t];
        const IPoint* v[4] = {&P[tt.v[0]], &P[tt.v[1]], &P[tt.v[2]], &P[tt.v[3]]};
        v[i] = &P[pi];
        if (orient3d(*v[0], *v[1], *v[2], *v[3]) < 0) {
          if (tt.n[i] < 0) return -1;  // outside the hull: cannot happen inside the dummy octahedron
          t = tt.n[i];
          moved = true;
          break;
        }
      }
      if (!moved) return t;
    }
    // fall back to a scan
    for (int t2 = 0; t2 < (int)T.size(); t2++) {
      if (!T[t2].alive) continue;
      bool in = true;
      for (int i = 0; i < 4 && in; i++) {
        const Tet& tt = T[t2];
        const IPoint* v[4] = {&P[tt.v[0]], &P[tt.v[1]], &P[tt.v[2]], &P[tt.v[3]]};
        v[i] = &P[pi];
        if (orient3d(*v[0], *v[1], *v[2], *v[3]) < 0) in = false;
      }
      if (in) return t2;
    }
    return -1;
  }

  // Inserts point pi; returns false when it is redundant (in conflict with no tetrahedron).
  bool insert(int pi) {
    int t0 = locate(pi, (last >= 0 && last < (int)T.size() && T[last].alive) ? last : first_alive());
    if (t0 < 0) {
      n_errors++;
      return false;
    }
    if (!conflict(t0, pi)) return false;
    stamp++;
    std::vector<int> cav{t0};
    mark[t0] = stamp;
    for (size_t q = 0; q < cav.size(); q++) {
      const Tet& t = T[cav[q]];
      for (int i = 0; i < 4; i++) {
        const int nb = t.n[i];
        if (nb < 0 || mark[nb] == stamp || mark[nb] == -stamp) continue;
        if (conflict(nb, pi)) {
          mark[nb] = stamp;
          cav.push_back(nb);
        } else {
          mark[nb] = -stamp;  // tested, outside the cavity
        }
      }
    }
    // boundary faces -> new tetrahedra
    struct EdgeSlot {
      int a, b, tet, face;
    };
    std::vector<EdgeSlot> open;
    std::vector<int> created;
    for (int ct : cav) {
      for (int i = 0; i < 4; i++) {
        const int nb = T[ct].n[i];
        if (nb >= 0 && mark[nb] == stamp) continue;
        int v[4] = {T[ct].v[0], T[ct].v[1], T[ct].v[2], T[ct].v[3]};
        v[i] = pi;
        const int k = new_tet(v[0], v[1], v[2], v[3]);
        if (orient_tet(T[k]) <= 0) n_errors++;
        created.push_back(k);
        // face opposite the new point: the outside neighbour
        T[k].n[i] = nb;
        if (nb >= 0)
          for (int j = 0; j < 4; j++)
            if (T[nb].n[j] == ct) T[nb].n[j] = k;
        // faces through the new point: matched by their edge among the new tetrahedra
        for (int j = 0; j < 4; j++) {
          if (j == i) continue;
          int e[2], ne = 0;
          for (int m = 0; m < 4; m++)
            if (m != i && m != j) e[ne++] = v[m];
          const int a = std::min(e[0], e[1]), b = std::max(e[0], e[1]);
          bool found = false;
          for (size_t s = 0; s < open.size(); s++)
            if (open[s].a == a && open[s].b == b) {
              T[k].n[j] = open[s].tet;
              T[open[s].tet].n[open[s].face] = k;
              open[s] = open.back();
              open.pop_back();
              found = true;
              break;
            }
          if (!found) open.push_back({a, b, k, j});
        }
      }
    }
    if (!open.empty()) n_errors++;
    for (int ct : cav) {
      T[ct].alive = false;
      free_list.push_back(ct);
    }
    // the freed slots may be reused by the next insertion only (new_tet above ran before)
    last = created.empty() ? first_alive() : created[0];
    return true;
  }

  int first_alive() const {
    for (int t = 0; t < (int)T.size(); t++)
      if (T[t].alive) return t;
    return -1;
  }
};

// ---------------------------------------------------------------------------------------------
// Geometry in double precision.

inline double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// Plane through three points (plane3points, src/tools.cpp:258-274), optionally normalised.
void plane3(const double* p1, const double* p2, const double* p3, double* w, bool normalize) {
  w[0] = p1[1] * (p2[2] - p3[2]) + p2[1] * (p3[2] - p1[2]) + p3[1] * (p1[2] - p2[2]);
  w[1] = p1[2] * (p2[0] - p3[0]) + p2[2] * (p3[0] - p1[0]) + p3[2] * (p1[0] - p2[0]);
  w[2] = p1[0] * (p2[1] - p3[1]) + p2[0] * (p3[1] - p1[1]) + p3[0] * (p1[1] - p2[1]);
  w[3] = -dot3(w, p1);
  if (normalize) {
    double norm = sqrt(dot3(w, w));
    w[0] /= norm; w[1] /= norm; w[2] /= norm; w[3] /= norm;
  }
}

// Orients a plane so that `inner` is on its non-positive side (negation is exact).
void orient_plane(double* w, const double* inner) {
  if (dot3(w, inner) + w[3] > 0)
    for (int k = 0; k < 4; k++) w[k] = -w[k];
}

// Weighted circumcentre (orthocentre) of four weighted points: the point of equal power distance
// |x - p_i|^2 - w_i to all four; solved relative to p0 by Cramer's rule.
bool orthocentre(const double* p[4], const double* w, double* out) {
  double a[3][3], r[3];
  for (int i = 0; i < 3; i++) {
    double d2 = 0;
    for (int k = 0; k < 3; k++) {
      a[i][k] = 2.0 * (p[i + 1][k] - p[0][k]);
      d2 += (p[i + 1][k] - p[0][k]) * (p[i + 1][k] - p[0][k]);
    }
    r[i] = d2 - (w[i + 1] - w[0]);
  }
  const double det = a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1]) - a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0]) +
                     a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
  if (det == 0.0) return false;
  double x[3];
  for (int c = 0; c < 3; c++) {
    double m[3][3];
    memcpy(m, a, sizeof m);
    for (int i = 0; i < 3; i++) m[i][c] = r[i];
    x[c] = (m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) - m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
            m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0])) / det;
  }
  for (int k = 0; k < 3; k++) out[k] = p[0][k] + x[k];
  return true;
}

// Quadric coding of the reference (q11, q22, q33, q44, q12, q23, q34, q13, q24, q14) of
// (x - f)^T A (x - f) - R for a symmetric 3x3 A.
void quadric_from(const double A[3][3], const double* f, double R, double* Q) {
  double Af[3];
  for (int i = 0; i < 3; i++) Af[i] = A[i][0] * f[0] + A[i][1] * f[1] + A[i][2] * f[2];
  Q[0] = A[0][0];
  Q[1] = A[1][1];
  Q[2] = A[2][2];
  Q[3] = (f[0] * Af[0] + f[1] * Af[1] + f[2] * Af[2]) - R;
  Q[4] = A[0][1];
  Q[5] = A[1][2];
  Q[6] = -Af[2];
  Q[7] = A[0][2];
  Q[8] = -Af[1];
  Q[9] = -Af[0];
}

// A = alpha I + beta o o^T (o unit): the surfaces of revolution of Del1 / Del2 cells.
void revolution(double alpha, double beta, const double* o, double A[3][3]) {
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) A[i][j] = (i == j ? alpha : 0.0) + beta * o[i] * o[j];
}

void unit(double* v) {
  const double n = sqrt(dot3(v, v));
  v[0] /= n; v[1] /= n; v[2] /= n;
}

struct Cell {
  int kind;
  double rec[NS_PATCH_F64];
  std::vector<double> planes;  // 4 per plane
  int atoms[3];
};

void set_box(Cell& c, const std::vector<const double*>& pts) {
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (const double* p : pts)
    for (int k = 0; k < 3; k++) {
      lo[k] = std::min(lo[k], p[k]);
      hi[k] = std::max(hi[k], p[k]);
    }
  double d2 = 0;
  for (int k = 0; k < 3; k++) {
    c.rec[NS_SKIN_LO + k] = lo[k];
    c.rec[NS_SKIN_HI + k] = hi[k];
    c.rec[k] = 0.5 * (lo[k] + hi[k]);
    d2 += (hi[k] - lo[k]) * (hi[k] - lo[k]);
  }
  c.rec[3] = 0.5 * sqrt(d2);
}

struct SkinBuilder {
  const double* at;  // atoms (x, y, z, r), already jittered
  int64_t na;
  double s;
  std::vector<double> X;  // 3 per point (atoms, then the 6 dummies)
  std::vector<double> W;  // weights
  RegularTriangulation rt;
  std::vector<int> alive;                // alive tetrahedra
  std::vector<double> vor;               // 3 per tetrahedron slot
  std::vector<double> psi;               // power of the orthocentre (the reference's radius2)
  std::vector<double> red;               // 12 per tetrahedron slot: reduced point of each vertex
  std::vector<Cell> del3, del0, del1, del2;
  std::vector<int> atom_cell;            // atom -> index into del0, -1 if none
  int n_errors = 0;

  bool is_dummy(int v) const { return v >= na; }
  const double* pt(int v) const { return &X[3 * (size_t)v]; }
  const double* reduced(int t, int v) const {
    const Tet& tt = rt.T[t];
    for (int k = 0; k < 4; k++)
      if (tt.v[k] == v) return &red[12 * (size_t)t + 3 * k];
    return nullptr;
  }

  void points() {
    X.resize(3 * (size_t)(na + 6));
    W.resize(na + 6);
    double mx[3] = {-1e6, -1e6, -1e6}, mn[3] = {1e6, 1e6, 1e6};
    for (int64_t i = 0; i < na; i++) {
      const double r = at[4 * i + 3];
      for (int k = 0; k < 3; k++) {
        X[3 * i + k] = at[4 * i + k];
        mx[k] = std::max(mx[k], at[4 * i + k] + r);
        mn[k] = std::min(mn[k], at[4 * i + k] - r);
      }
      W[i] = (r * r) / s;
    }
    // the six dummy points on the axes of the bounding box enlarged by twice its half extent
    // (src/SkinSurface.cpp:1330-1351), weight -1
    double mid[3];
    for (int k = 0; k < 3; k++) {
      mid[k] = (mx[k] + mn[k]) * 0.5;
      mn[k] -= fabs(mid[k] - mn[k]) * 2.;
      mx[k] += fabs(mid[k] - mx[k]) * 2.;
    }
    const double d[6][3] = {{mn[0], mid[1], mid[2]}, {mx[0], mid[1], mid[2]}, {mid[0], mn[1], mid[2]},
                            {mid[0], mx[1], mid[2]}, {mid[0], mid[1], mn[2]}, {mid[0], mid[1], mx[2]}};
    for (int i = 0; i < 6; i++) {
      for (int k = 0; k < 3; k++) X[3 * (na + i) + k] = d[i][k];
      W[na + i] = -1.0;
    }
    // snapped copies for the predicates, relative to the box centre
    double ext = 1.0;
    for (int64_t i = 0; i < na + 6; i++)
      for (int k = 0; k < 3; k++) ext = std::max(ext, fabs(X[3 * i + k] - mid[k]));
    int e = 0;
    frexp(ext, &e);                       // ext < 2^e
    const int sh = std::min(24, 33 - e);  // coordinates below 2^33 in snapped units
    const double sc = ldexp(1.0, sh), sc2 = ldexp(1.0, 2 * sh);
    rt.P.resize(na + 6);
    for (int64_t i = 0; i < na + 6; i++) {
      for (int k = 0; k < 3; k++) rt.P[i].x[k] = llround((X[3 * i + k] - mid[k]) * sc);
      rt.P[i].w = llround(W[i] * sc2);
    }
  }

  void triangulate() {
    const int d0 = (int)na;
    // the regular triangulation of the six dummies: four tetrahedra around one diagonal; the
    // diagonal whose tetrahedra are free of conflicts with the two remaining dummies
    const int diag[3][2] = {{0, 1}, {2, 3}, {4, 5}};
    const int ring[3][4] = {{2, 4, 3, 5}, {0, 4, 1, 5}, {0, 2, 1, 3}};
    int chosen = -1;
    for (int dgi = 0; dgi < 3 && chosen < 0; dgi++) {
      bool ok = true;
      for (int k = 0; k < 4 && ok; k++) {
        int v[4] = {d0 + diag[dgi][0], d0 + diag[dgi][1], d0 + ring[dgi][k], d0 + ring[dgi][(k + 1) & 3]};
        if (orient3d(rt.P[v[0]], rt.P[v[1]], rt.P[v[2]], rt.P[v[3]]) < 0) std::swap(v[0], v[1]);
        for (int o = 0; o < 6 && ok; o++) {
          const int q = d0 + o;
          if (q == v[0] || q == v[1] || q == v[2] || q == v[3]) continue;
          if (in_conflict(rt.P[v[0]], rt.P[v[1]], rt.P[v[2]], rt.P[v[3]], rt.P[q])) ok = false;
        }
      }
      if (ok) chosen = dgi;
    }
    if (chosen < 0) {
      n_errors++;
      chosen = 0;
    }
    int rg[4];
    for (int k = 0; k < 4; k++) rg[k] = d0 + ring[chosen][k];
    rt.octahedron(d0 + diag[chosen][0], d0 + diag[chosen][1], rg);
    // atoms in the order of a Morton curve over their snapped coordinates (short walks)
    std::vector<std::pair<uint64_t, int>> order(na);
    int64_t lo[3] = {INT64_MAX, INT64_MAX, INT64_MAX};
    for (int64_t i = 0; i < na; i++)
      for (int k = 0; k < 3; k++) lo[k] = std::min(lo[k], rt.P[i].x[k]);
    for (int64_t i = 0; i < na; i++) {
      uint64_t key = 0;
      uint64_t c[3];
      for (int k = 0; k < 3; k++) c[k] = (uint64_t)(rt.P[i].x[k] - lo[k]) >> 14;  // 2^-10 A cells
      for (int b = 20; b >= 0; b--)
        for (int k = 0; k < 3; k++) key = (key << 1) | ((c[k] >> b) & 1u);
      order[i] = {key, (int)i};
    }
    std::sort(order.begin(), order.end());
    for (auto& o : order) rt.insert(o.second);
    n_errors += rt.n_errors;
    for (int t = 0; t < (int)rt.T.size(); t++)
      if (rt.T[t].alive) alive.push_back(t);
  }

  void tetra_geometry() {
    vor.assign(3 * rt.T.size(), 0.0);
    psi.assign(rt.T.size(), 0.0);
    red.assign(12 * rt.T.size(), 0.0);
    for (int t : alive) {
      const Tet& tt = rt.T[t];
      const double* p[4] = {pt(tt.v[0]), pt(tt.v[1]), pt(tt.v[2]), pt(tt.v[3])};
      double w[4] = {W[tt.v[0]], W[tt.v[1]], W[tt.v[2]], W[tt.v[3]]};
      double* z = &vor[3 * (size_t)t];
      if (!orthocentre(p, w, z)) n_errors++;
      for (int i = 0; i < 4; i++) {
        double* rp = &red[12 * (size_t)t + 3 * i];
        double a[3];
        for (int k = 0; k < 3; k++) {
          a[k] = z[k] - p[i][k];
          rp[k] = p[i][k] + s * a[k];
        }
        if (i == 0) psi[t] = (a[0] * a[0] + a[1] * a[1] + a[2] * a[2]) - w[0];
      }
    }
  }

  // Del3: reduced tetrahedra (BuildDelaunayTetraCells)
  void build_del3() {
    for (int t : alive) {
      const Tet& tt = rt.T[t];
      bool dummy = false;
      for (int k = 0; k < 4; k++) dummy |= is_dummy(tt.v[k]);
      if (psi[t] < 0 || dummy) continue;
      Cell c{};
      c.kind = NS_SKIN_TETRA;
      const double* r[4];
      for (int k = 0; k < 4; k++) r[k] = &red[12 * (size_t)t + 3 * k];
      double inner[3] = {0, 0, 0};
      for (int k = 0; k < 4; k++)
        for (int q = 0; q < 3; q++) inner[q] += 0.25 * r[k][q];
      // the faces of the reduced tetrahedron, through the reference's vertex orders, oriented
      // towards the inside
      const int fo[4][3] = {{2, 1, 0}, {3, 2, 0}, {3, 1, 2}, {0, 1, 3}};
      c.planes.resize(16);
      for (int f = 0; f < 4; f++) {
        double* w = &c.planes[4 * f];
        plane3(r[fo[f][0]], r[fo[f][1]], r[fo[f][2]], w, false);
        orient_plane(w, inner);
      }
      const double* z = &vor[3 * (size_t)t];
      double* Q = c.rec + NS_SKIN_Q;
      Q[0] = 1; Q[1] = 1; Q[2] = 1;
      Q[3] = -psi[t] * (1 - s) + z[0] * z[0] + z[1] * z[1] + z[2] * z[2];
      Q[4] = 0; Q[7] = 0; Q[9] = -z[0];
      Q[5] = 0; Q[8] = -z[1]; Q[6] = -z[2];
      set_box(c, {r[0], r[1], r[2], r[3]});
      c.atoms[0] = tt.v[0]; c.atoms[1] = tt.v[1]; c.atoms[2] = tt.v[2];
      del3.push_back(std::move(c));
    }
  }

  // Del0: atom spheres inside reduced Voronoi cells (BuildDelaunayPointCells); planes added by
  // the edge cells.
  void build_del0() {
    std::vector<char> present(na, 0);
    for (int t : alive)
      for (int k = 0; k < 4; k++)
        if (!is_dummy(rt.T[t].v[k])) present[rt.T[t].v[k]] = 1;
    atom_cell.assign(na, -1);
    for (int64_t i = 0; i < na; i++) {
      if (!present[i]) continue;
      Cell c{};
      c.kind = NS_SKIN_POINT;
      const double* p = pt((int)i);
      const double r = at[4 * i + 3];
      double* Q = c.rec + NS_SKIN_Q;
      Q[0] = 1; Q[1] = 1; Q[2] = 1;
      Q[3] = -s * W[i] + p[0] * p[0] + p[1] * p[1] + p[2] * p[2];
      Q[4] = 0; Q[7] = 0; Q[9] = -p[0];
      Q[5] = 0; Q[8] = -p[1]; Q[6] = -p[2];
      for (int k = 0; k < 3; k++) {
        c.rec[k] = p[k];
        c.rec[NS_SKIN_LO + k] = p[k] - r;
        c.rec[NS_SKIN_HI + k] = p[k] + r;
      }
      c.rec[3] = r;
      c.atoms[0] = (int)i; c.atoms[1] = -1; c.atoms[2] = -1;
      atom_cell[i] = (int)del0.size();
      del0.push_back(std::move(c));
    }
  }

  // Del1: prisms around Delaunay edges between atoms (BuildDelaunayEdgeCells).
  void build_del1() {
    std::unordered_map<uint64_t, char> seen;
    seen.reserve(alive.size() * 8);
    for (int t0 : alive) {
      for (int e = 0; e < 6; e++) {
        static const int ep[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
        int a = rt.T[t0].v[ep[e][0]], b = rt.T[t0].v[ep[e][1]];
        if (a > b) std::swap(a, b);
        if (is_dummy(a) || is_dummy(b)) continue;
        const uint64_t key = (uint64_t)a * (uint64_t)(na + 6) + (uint64_t)b;
        if (!seen.emplace(key, 1).second) continue;
        // the tetrahedra around the edge in cyclic order
        std::vector<int> ring;
        int t = t0;
        int prev_other = -1;
        {
          int others[2], no = 0;
          for (int k = 0; k < 4; k++)
            if (rt.T[t].v[k] != a && rt.T[t].v[k] != b) others[no++] = rt.T[t].v[k];
          prev_other = others[0];
        }
        bool ok = true;
        for (int guard = 0; guard < 4096; guard++) {
          ring.push_back(t);
          // leave t through the face opposite prev_other (the face holding a, b and the other vertex)
          int fi = -1, nxt_other = -1;
          for (int k = 0; k < 4; k++) {
            const int v = rt.T[t].v[k];
            if (v == prev_other) fi = k;
            else if (v != a && v != b) nxt_other = v;
          }
          const int nt = rt.T[t].n[fi];
          if (nt < 0) {
            ok = false;
            break;
          }
          prev_other = nxt_other;
          t = nt;
          if (t == t0) break;
        }
        if (!ok || ring.size() < 3) {
          n_errors++;
          continue;
        }
        Cell c{};
        c.kind = NS_SKIN_EDGE;
        std::vector<const double*> up, lo, all;
        for (int rtet : ring) {
          const double* p1 = reduced(rtet, a);
          const double* p2 = reduced(rtet, b);
          up.push_back(p1);
          lo.push_back(p2);
          all.push_back(p1);
          all.push_back(p2);
        }
        double inner[3];
        for (int q = 0; q < 3; q++)
          inner[q] = (up[0][q] + up[1][q] + up[2][q] + lo[0][q] + lo[1][q] + lo[2][q]) / 6.;
        double upper[4], lower[4];
        plane3(up[0], up[1], up[2], upper, true);
        orient_plane(upper, inner);
        plane3(lo[0], lo[1], lo[2], lower, true);
        orient_plane(lower, inner);
        const size_t n = ring.size();
        for (size_t i = 0; i < n; i++) {
          double w[4];
          plane3(up[i], lo[i], up[(i + 1) % n], w, true);
          orient_plane(w, inner);
          c.planes.insert(c.planes.end(), w, w + 4);
        }
        c.planes.insert(c.planes.end(), upper, upper + 4);
        c.planes.insert(c.planes.end(), lower, lower + 4);
        // the reduced Voronoi faces bound the atoms' Del0 cells (stored negated: their test is
        // "outside when < 0")
        if (atom_cell[a] >= 0)
          for (int k = 0; k < 4; k++) del0[atom_cell[a]].planes.push_back(-upper[k]);
        if (atom_cell[b] >= 0)
          for (int k = 0; k < 4; k++) del0[atom_cell[b]].planes.push_back(-lower[k]);
        // focus: the edge's point of equal power to both atoms; R = w_a - |a - focus|^2
        const double* pa = pt(a);
        const double* pb = pt(b);
        double dv[3] = {pb[0] - pa[0], pb[1] - pa[1], pb[2] - pa[2]};
        const double d2 = dot3(dv, dv);
        const double mu = (d2 + W[a] - W[b]) / (2.0 * d2);
        double f[3];
        for (int k = 0; k < 3; k++) f[k] = pa[k] + mu * dv[k];
        double af[3] = {pa[0] - f[0], pa[1] - f[1], pa[2] - f[2]};
        const double R = W[a] - dot3(af, af);
        double o[3] = {dv[0], dv[1], dv[2]};
        unit(o);
        double A[3][3];
        revolution(1.0 / s, -(1.0 / s + 1.0 / (1.0 - s)), o, A);
        quadric_from(A, f, R, c.rec + NS_SKIN_Q);
        set_box(c, all);
        c.atoms[0] = a; c.atoms[1] = b; c.atoms[2] = -1;
        del1.push_back(std::move(c));
      }
    }
  }

  // Del2: prisms over Delaunay facets between atoms (BuildDelaunayFacetCells).
  void build_del2() {
    for (int t1 : alive) {
      for (int fi = 0; fi < 4; fi++) {
        const int t2 = rt.T[t1].n[fi];
        if (t2 < 0 || t2 < t1) continue;  // hull facet, or visited from the other side
        int ids[3], ni = 0;
        for (int k = 0; k < 4; k++)
          if (k != fi) ids[ni++] = rt.T[t1].v[k];
        if (is_dummy(ids[0]) || is_dummy(ids[1]) || is_dummy(ids[2])) continue;
        Cell c{};
        c.kind = NS_SKIN_FACET;
        const double* mp[6];
        for (int k = 0; k < 3; k++) {
          mp[2 * k] = reduced(t1, ids[k]);
          mp[2 * k + 1] = reduced(t2, ids[k]);
        }
        if (!mp[1] || !mp[3] || !mp[5]) {
          n_errors++;
          continue;
        }
        double inner[3];
        for (int q = 0; q < 3; q++) inner[q] = (mp[0][q] + mp[2][q] + mp[4][q] + mp[1][q] + mp[3][q] + mp[5][q]) / 6.;
        double w[4];
        const int lat[3][3] = {{0, 1, 2}, {2, 3, 4}, {4, 5, 0}};
        for (int l = 0; l < 3; l++) {
          plane3(mp[lat[l][0]], mp[lat[l][1]], mp[lat[l][2]], w, true);
          orient_plane(w, inner);
          c.planes.insert(c.planes.end(), w, w + 4);
        }
        plane3(mp[0], mp[2], mp[4], w, true);
        orient_plane(w, inner);
        c.planes.insert(c.planes.end(), w, w + 4);
        plane3(mp[1], mp[3], mp[5], w, true);
        orient_plane(w, inner);
        c.planes.insert(c.planes.end(), w, w + 4);
        // focus: the point of the facet's plane with equal power to its three atoms
        const double* p0 = pt(ids[0]);
        const double* p1 = pt(ids[1]);
        const double* p2 = pt(ids[2]);
        double u[3], v[3], nrm[3];
        for (int k = 0; k < 3; k++) {
          u[k] = p1[k] - p0[k];
          v[k] = p2[k] - p0[k];
        }
        nrm[0] = u[1] * v[2] - u[2] * v[1];
        nrm[1] = u[2] * v[0] - u[0] * v[2];
        nrm[2] = u[0] * v[1] - u[1] * v[0];
        // x = p0 + y with 2 u.y = |u|^2 - (w1 - w0), 2 v.y = |v|^2 - (w2 - w0), n.y = 0
        double M[3][3] = {{2 * u[0], 2 * u[1], 2 * u[2]}, {2 * v[0], 2 * v[1], 2 * v[2]}, {nrm[0], nrm[1], nrm[2]}};
        double rhs[3] = {dot3(u, u) - (W[ids[1]] - W[ids[0]]), dot3(v, v) - (W[ids[2]] - W[ids[0]]), 0.0};
        const double det = M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) -
                           M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0]) +
                           M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0]);
        if (det == 0.0) {
          n_errors++;
          continue;
        }
        double y[3];
        for (int col = 0; col < 3; col++) {
          double m[3][3];
          memcpy(m, M, sizeof m);
          for (int i = 0; i < 3; i++) m[i][col] = rhs[i];
          y[col] = (m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) - m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
                    m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0])) / det;
        }
        double f[3] = {p0[0] + y[0], p0[1] + y[1], p0[2] + y[2]};
        double af[3] = {p0[0] - f[0], p0[1] - f[1], p0[2] - f[2]};
        const double R = W[ids[0]] - dot3(af, af);
        unit(nrm);
        double A[3][3];
        revolution(-1.0 / (1.0 - s), 1.0 / s + 1.0 / (1.0 - s), nrm, A);
        quadric_from(A, f, R, c.rec + NS_SKIN_Q);
        set_box(c, {mp[0], mp[1], mp[2], mp[3], mp[4], mp[5]});
        c.atoms[0] = ids[0]; c.atoms[1] = ids[1]; c.atoms[2] = ids[2];
        del2.push_back(std::move(c));
      }
    }
  }

  void emit(NsPatchSet* ps) {
    for (auto* list : {&del3, &del0, &del1, &del2})
      for (const Cell& c : *list)
        ps->add_patch(c.kind, c.rec, c.planes.data(), nullptr, (int64_t)(c.planes.size() / 4), c.atoms[0],
                      c.atoms[1], c.atoms[2]);
  }
};

}  // namespace

extern "C" {

// Skin surface patch set of jittered atoms (SkinSurface::build / buildSkinCGAL,
// src/SkinSurface.cpp:329, 1271-1812) with shrink factor s.
int nsg_skin_build(const double* atoms_xyzr, int64_t n_atoms, double shrink, int n_threads, NsPatchSet** out) {
  (void)n_threads;
  if (!atoms_xyzr || n_atoms <= 0 || !out || !(shrink > 0.0 && shrink < 1.0)) return NSG_ERR_ARG;
  SkinBuilder b;
  b.at = atoms_xyzr;
  b.na = n_atoms;
  b.s = shrink;
  b.points();
  b.triangulate();
  b.tetra_geometry();
  b.build_del3();
  b.build_del0();
  b.build_del1();
  b.build_del2();
  NsPatchSet* ps = new NsPatchSet();
  b.emit(ps);
  *out = ps;
  return b.n_errors ? NSG_ERR_GEOMETRY : NSG_OK;
}

// Exact predicates of the skin builder's triangulation on integer coordinates, exposed for the
// tests: orientation of (a, b, c, d) and conflict of weighted point p with the orthosphere of
// (a, b, c, d); points are 4 int64 each (x, y, z, w).
int nsg_skin_predicates(const int64_t* pts, int* orient, int* conflict) {
  if (!pts || !orient || !conflict) return NSG_ERR_ARG;
  IPoint q[5];
  for (int i = 0; i < 5; i++) {
    for (int k = 0; k < 3; k++) q[i].x[k] = pts[4 * i + k];
    q[i].w = pts[4 * i + 3];
  }
  *orient = orient3d(q[0], q[1], q[2], q[3]);
  *conflict = in_conflict(q[0], q[1], q[2], q[3], q[4]) ? 1 : 0;
  return NSG_OK;
}

}  // extern "C"
