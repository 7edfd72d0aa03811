// Grid environment of the surface builder: grid construction, atom jitter and xyzr parsing.
//
// Follows DelPhiShared::getBounds / DelPhiShared::buildGrid (src/DelphiShared.cpp:775-798,
// 1038-1201), randnum (src/tools.cpp:64-81, SEED src/tools.h:1827) and the jitter loop of
// buildConnollyCGAL (src/ConnollySurface.cpp:2484-2488).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../ns_types.h"
#include "host_api.h"

extern "C" {

int nsg_grid_build(const double* atoms_xyzr, int64_t n_atoms, double scale, double perfil,
                   NsGrid* out) {
  if (!atoms_xyzr || !out) return NSG_ERR_ARG;
  if (n_atoms <= 0) return NSG_ERR_EMPTY;
  if (scale < 0) scale = 2.0;                 // DEFAULT_SCALE
  if (perfil < 0 || perfil > 100) perfil = 80; // DEFAULT_PERFIL
  double cmin[3] = {INFINITY, INFINITY, INFINITY};
  double cmax[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int64_t a = 0; a < n_atoms; a++) {
    const double* p = atoms_xyzr + 4 * a;
    for (int d = 0; d < 3; d++) {
      cmin[d] = std::min(cmin[d], p[d] - p[3]);
      cmax[d] = std::max(cmax[d], p[d] + p[3]);
    }
  }
  double mid[3];
  for (int d = 0; d < 3; d++) mid[d] = (cmax[d] + cmin[d]) / 2.;
  double v[6] = {fabs(cmax[0] - mid[0]), fabs(cmin[0] - mid[0]), fabs(cmax[1] - mid[1]),
                 fabs(cmin[1] - mid[1]), fabs(cmax[2] - mid[2]), fabs(cmin[2] - mid[2])};
  double rmaxdim = -INFINITY;
  for (int i = 0; i < 6; i++)
    if (rmaxdim < v[i]) rmaxdim = v[i];
  rmaxdim = 2 * rmaxdim;
  unsigned int igrid = (unsigned int)floor(scale * 100. / perfil * rmaxdim);
  if ((igrid % 2) == 0) igrid++;
  out->nx = out->ny = out->nz = igrid;
  out->scale = scale;
  out->side = 1. / scale;
  out->hside = 0.5 / scale;
  out->A = out->side * out->side;
  out->rmaxdim = rmaxdim;
  for (int d = 0; d < 3; d++) out->baricenter[d] = mid[d];
  out->xmin = mid[0] - (igrid - 1) / (2 * scale);
  out->ymin = mid[1] - (igrid - 1) / (2 * scale);
  out->zmin = mid[2] - (igrid - 1) / (2 * scale);
  out->xmax = mid[0] + (igrid - 1) / (2 * scale);
  out->ymax = mid[1] + (igrid - 1) / (2 * scale);
  out->zmax = mid[2] + (igrid - 1) / (2 * scale);
  return NSG_OK;
}

// Park-Miller minimal standard generator (multiplier 16807, modulus 2^31-1) evaluated with
// Schrage's decomposition, as the reference's randnum does; *seed is updated in place.
double nsg_randnum(int64_t* seed) {
  const int64_t aa = 16807, mm = 2147483647, qq = 127773, rr = 2836;
  int64_t s = *seed;
  int64_t hh = s / qq;
  int64_t lo = s - hh * qq;
  int64_t test = aa * lo - rr * hh;
  s = (test >= 0) ? test : test + mm;
  *seed = s;
  return s / (double)mm;
}

int nsg_jitter_atoms(double* atoms_xyzr, int64_t n_atoms, double displacement, int64_t* seed) {
  if (!atoms_xyzr || !seed) return NSG_ERR_ARG;
  for (int64_t a = 0; a < n_atoms; a++) {
    double* p = atoms_xyzr + 4 * a;
    p[0] += displacement * (nsg_randnum(seed) - 0.5);
    p[1] += displacement * (nsg_randnum(seed) - 0.5);
    p[2] += displacement * (nsg_randnum(seed) - 0.5);
  }
  return NSG_OK;
}

// Reads "x y z r" records (extra columns ignored, blank lines skipped), the xyzr format that
// DelPhiShared::loadAtoms accepts.  Returns the number of atoms, or a negative error code.
// When out is NULL only the count is returned.
int64_t nsg_read_xyzr(const char* path, double* out, int64_t capacity) {
  FILE* f = fopen(path, "r");
  if (!f) return NSG_ERR_IO;
  char line[4096];
  int64_t n = 0;
  while (fgets(line, sizeof line, f)) {
    double x, y, z, r;
    if (sscanf(line, "%lf %lf %lf %lf", &x, &y, &z, &r) != 4) continue;
    if (out) {
      if (n >= capacity) { fclose(f); return NSG_ERR_CAPACITY; }
      out[4 * n + 0] = x; out[4 * n + 1] = y; out[4 * n + 2] = z; out[4 * n + 3] = r;
    }
    n++;
  }
  fclose(f);
  return n;
}

// Reads the ATOM / HETATM records of a pqr file as DelPhiShared::loadAtoms does for a file name
// containing ".pqr" (src/DelphiShared.cpp:365-415, 520-545): whitespace-separated fields, 11 of
// them (serial, name, residue, chain, residue number, x, y, z, charge, radius) or 10 (no chain);
// every numeric field must parse completely; other records and empty lines are skipped, and so
// are atoms with a radius below 1e-20.  Returns the number of atoms (x, y, z, r into out unless
// NULL), or a negative error code: NSG_ERR_IO (unreadable), NSG_ERR_ARG (a malformed ATOM or
// HETATM record, where the reference exits), NSG_ERR_CAPACITY (more atoms than capacity).
int64_t nsg_read_pqr(const char* path, double* out, int64_t capacity) {
  FILE* f = fopen(path, "r");
  if (!f) return NSG_ERR_IO;
  char line[4096];
  int64_t n = 0;
  auto whole_int = [](const char* t) {
    char* e = nullptr;
    (void)strtol(t, &e, 10);
    return e != t && *e == '\0';
  };
  auto whole_double = [](const char* t, double* v) {
    char* e = nullptr;
    *v = strtod(t, &e);
    return e != t && *e == '\0';
  };
  while (fgets(line, sizeof line, f)) {
    if (strlen(line) <= 1) continue;
    char* fields[16];
    int nf = 0;
    for (char* tok = strtok(line, " \t\r\n"); tok; tok = strtok(nullptr, " \t\r\n")) {
      if (nf < 16) fields[nf] = tok;
      nf++;
    }
    if (nf == 0 || (strcmp(fields[0], "ATOM") != 0 && strcmp(fields[0], "HETATM") != 0)) continue;
    if (nf != 10 && nf != 11) {
      fclose(f);
      return NSG_ERR_ARG;
    }
    const int off = nf == 11 ? 1 : 0;  // the chain field
    double x, y, z, q, r;
    if (!whole_int(fields[1]) || !whole_int(fields[4 + off]) || !whole_double(fields[5 + off], &x) ||
        !whole_double(fields[6 + off], &y) || !whole_double(fields[7 + off], &z) ||
        !whole_double(fields[8 + off], &q) || !whole_double(fields[9 + off], &r)) {
      fclose(f);
      return NSG_ERR_ARG;
    }
    if (r < 1e-20) continue;
    if (out) {
      if (n >= capacity) {
        fclose(f);
        return NSG_ERR_CAPACITY;
      }
      out[4 * n + 0] = x;
      out[4 * n + 1] = y;
      out[4 * n + 2] = z;
      out[4 * n + 3] = r;
    }
    n++;
  }
  fclose(f);
  return n;
}

}  // extern "C"
