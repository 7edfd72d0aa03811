// C wrappers around the reference's own ray/solver math (src/tools.cpp, src/sturm), compiled
// from the reference sources into oracle/_ref/ to pin the oracle's restatement.  Test
// infrastructure only.
#include "tools.h"

// Globals the reference's tools.cpp refers to but that its main program defines.
fstream* errorStream = nullptr;
fstream* internals = nullptr;

extern "C" {
int ref_ray_sphere(const double* o, const double* d, const double* c, double r, double* t) {
  return raySphere(o, d, c, r, &t[0], &t[1]) ? 1 : 0;
}
int ref_ray_torus(int analytical, const double* invrot9, const double* tc, const double* sc, double probe,
                  double major, double radius, int panel, const double* orig, const double* dir, double* t) {
  double inv[3][3], tcc[3], scc[3], o[3], dd[3];
  for (int i = 0; i < 9; i++) inv[i / 3][i % 3] = invrot9[i];
  for (int i = 0; i < 3; i++) { tcc[i] = tc[i]; scc[i] = sc[i]; o[i] = orig[i]; dd[i] = dir[i]; }
  int n = 0;
  bool ok = rayTorus(analytical, inv, tcc, scc, probe, major, radius, panel, o, dd, t, n);
  return ok ? n : 0;
}
double ref_randnum_seq(int k) {
  double v = 0;
  for (int i = 0; i < k; i++) v = randnum();
  return v;
}
double ref_rintp(double x) { return rintp(x); }
void ref_plane3points(const double* a, const double* b, const double* c, double* w) { plane3points(a, b, c, w); }
int ref_sturm_roots(const double* poly5, double* roots) {
  int n = 4;
  getRealRootsSturm(poly5, 4, roots, n);
  return n;
}
}
