// On-disk outputs in the reference's text layouts, written from caller-owned host arrays:
//   status map      DelPhiShared::saveStatus (src/DelphiShared.cpp:1458-1502): "%d " per node,
//                   i outer, j, k inner; a newline after every k row and a blank line per i
//   cavities        DelPhiShared::saveCavities (src/DelphiShared.cpp:1889-1946): cavities.txt
//                   lists the nodes of every cavity ("\n %f %f %f", k, j, i scan); cavitiesSize.txt
//                   the count ("%f\n") then per cavity its node barycentre, volume and fill flag
//                   ("%lf %lf %lf %lf %d\n")
//   meshes          Surface::saveMesh (src/Surface.cpp:10857-11052): OFF ("%.3f" vertices,
//                   "3 %d %d %d" faces, winding reversed on request) with triangleAreas.txt
//                   (Heron area "%f" per triangle, "0." when degenerate); PLY as binary little
//                   endian (double x, y, z; int32 faces with a uchar count)
#include <cmath>
#include <cstdio>
#include <ctime>
#include <algorithm>
#include <string>
#include <vector>

#include "../ns_types.h"
#include "host_api.h"

namespace {

const char* kProg = "nanoshaper_b200";
const char* kVersion = "0.1.0";

double coord(double vmin, double side, int64_t i) { return vmin + (double)i * side; }

}  // namespace

extern "C" {

int nsg_write_status(const char* path, const int32_t* status, int64_t nx, int64_t ny, int64_t nz) {
  if (!path || !status || nx <= 0 || ny <= 0 || nz <= 0) return NSG_ERR_ARG;
  FILE* fp = fopen(path, "w");
  if (!fp) return NSG_ERR_IO;
  for (int64_t i = 0; i < nx; i++) {
    for (int64_t j = 0; j < ny; j++) {
      for (int64_t k = 0; k < nz; k++) fprintf(fp, "%d ", status[(k * ny + j) * nx + i]);
      fprintf(fp, "\n");
    }
    fprintf(fp, "\n");
  }
  return fclose(fp) == 0 ? NSG_OK : NSG_ERR_IO;
}

int nsg_write_cavities(const char* cavities_path, const char* sizes_path, const int32_t* status, const NsGrid* g,
                       int32_t n_cav, const double* sizes, const int32_t* filled) {
  if (!cavities_path || !sizes_path || !status || !g || n_cav < 0 || (n_cav > 0 && (!sizes || !filled)))
    return NSG_ERR_ARG;
  FILE* fp = fopen(cavities_path, "w");
  if (!fp) return NSG_ERR_IO;
  std::vector<double> bx(n_cav, 0.0), by(n_cav, 0.0), bz(n_cav, 0.0);
  std::vector<int64_t> cnt(n_cav, 0);
  for (int64_t k = 0; k < g->nz; k++)
    for (int64_t j = 0; j < g->ny; j++)
      for (int64_t i = 0; i < g->nx; i++) {
        const int32_t s = status[(k * g->ny + j) * g->nx + i];
        if (s <= NS_STATUS_OUT) continue;
        const double x = coord(g->xmin, g->side, i), y = coord(g->ymin, g->side, j), z = coord(g->zmin, g->side, k);
        fprintf(fp, "\n %f %f %f", x, y, z);
        const int c = s - NS_STATUS_FIRST_CAV;
        if (c >= 0 && c < n_cav) {
          bx[c] += x;
          by[c] += y;
          bz[c] += z;
          cnt[c]++;
        }
      }
  if (fclose(fp) != 0) return NSG_ERR_IO;
  fp = fopen(sizes_path, "w");
  if (!fp) return NSG_ERR_IO;
  fprintf(fp, "%f\n", (float)n_cav);
  for (int32_t c = 0; c < n_cav; c++) {
    const double n = cnt[c] ? (double)cnt[c] : 1.0;
    fprintf(fp, "%lf %lf %lf %lf %d\n", bx[c] / n, by[c] / n, bz[c] / n, sizes[c], filled[c] ? 1 : 0);
  }
  return fclose(fp) == 0 ? NSG_OK : NSG_ERR_IO;
}

// root + "triangleAreas.txt": the Heron area of every triangle, "0." for degenerate ones
// (Surface::saveMesh, src/Surface.cpp:11042-11062).
static int write_triangle_areas(const std::string& base, const double* vertices, const int32_t* triangles,
                                int64_t n_triangles) {
  FILE* fp = fopen((base + "triangleAreas.txt").c_str(), "w");
  if (!fp) return NSG_ERR_IO;
  for (int64_t t = 0; t < n_triangles; t++) {
    const double* p0 = vertices + 3 * (int64_t)triangles[3 * t];
    const double* p1 = vertices + 3 * (int64_t)triangles[3 * t + 1];
    const double* p2 = vertices + 3 * (int64_t)triangles[3 * t + 2];
    auto dist = [](const double* a, const double* b) {
      return sqrt((a[0] - b[0]) * (a[0] - b[0]) + (a[1] - b[1]) * (a[1] - b[1]) + (a[2] - b[2]) * (a[2] - b[2]));
    };
    const double a = dist(p0, p1), b = dist(p0, p2), c = dist(p1, p2);
    const double ttt = (a + b + c) * (b + c - a) * (c + a - b) * (a + b - c);
    if (ttt > 0)
      fprintf(fp, "%f\n", 0.25 * sqrt(ttt));
    else
      fprintf(fp, "0.\n");
  }
  return fclose(fp) == 0 ? NSG_OK : NSG_ERR_IO;
}

// format: 0 OFF (+ triangleAreas.txt), 1 PLY (binary little endian).  root is the path without
// extension; the reference's file names are root + ".off" / ".ply" and root + "triangleAreas.txt".
int nsg_write_cavity_atoms(const char* path, int32_t n_cav, const int32_t* offsets, const int32_t* atoms,
                           const int32_t* serials, int64_t n_atoms, const int32_t* skip) {
  if (!path || n_cav < 0 || (n_cav > 0 && (!offsets || !atoms))) return NSG_ERR_ARG;
  FILE* fp = fopen(path, "w");
  if (!fp) return NSG_ERR_IO;
  for (int32_t c = 0; c < n_cav; c++) {
    if (skip && skip[c]) continue;
    for (int32_t q = offsets[c]; q < offsets[c + 1]; q++) {
      const int32_t a = atoms[q];
      int32_t serial = a + 1;
      if (serials && a >= 0 && a < n_atoms && serials[a] > 0) serial = serials[a];
      fprintf(fp, "%d ", serial);
    }
    fprintf(fp, "\n");
  }
  return fclose(fp) == 0 ? NSG_OK : NSG_ERR_IO;
}

int nsg_write_mesh(const char* root, int format, const double* vertices, int64_t n_vertices, const int32_t* triangles,
                   int64_t n_triangles, int revert) {
  if (!root || n_vertices < 0 || n_triangles < 0 || (n_vertices && !vertices) || (n_triangles && !triangles))
    return NSG_ERR_ARG;
  std::string base(root);
  for (int64_t t = 0; t < 3 * n_triangles; t++)
    if (triangles[t] < 0 || triangles[t] >= n_vertices) return NSG_ERR_ARG;
  auto tri = [&](int64_t t, int q) { return triangles[3 * t + (revert ? 2 - q : q)]; };
  if (format == 0) {
    FILE* fp = fopen((base + ".off").c_str(), "w");
    if (!fp) return NSG_ERR_IO;
    time_t pt;
    time(&pt);
    fprintf(fp, "OFF\n");
    fprintf(fp, "# File created by %s version %s date %s\n", kProg, kVersion, ctime(&pt));
    fprintf(fp, "%d %d 0\n", (int)n_vertices, (int)n_triangles);
    for (int64_t v = 0; v < n_vertices; v++)
      fprintf(fp, "%.3f %.3f %.3f\n", vertices[3 * v], vertices[3 * v + 1], vertices[3 * v + 2]);
    for (int64_t t = 0; t < n_triangles; t++) fprintf(fp, "3 %d %d %d\n", tri(t, 0), tri(t, 1), tri(t, 2));
    if (fclose(fp) != 0) return NSG_ERR_IO;
  } else if (format == 1) {
    FILE* fp = fopen((base + ".ply").c_str(), "wb");
    if (!fp) return NSG_ERR_IO;
    fprintf(fp,
            "ply\nformat binary_little_endian 1.0\nelement vertex %lld\nproperty double x\nproperty double y\n"
            "property double z\nelement face %lld\nproperty list uchar int vertex_indices\nend_header\n",
            (long long)n_vertices, (long long)n_triangles);
    if (n_vertices) fwrite(vertices, sizeof(double), 3 * n_vertices, fp);
    for (int64_t t = 0; t < n_triangles; t++) {
      const unsigned char three = 3;
      const int32_t f[3] = {tri(t, 0), tri(t, 1), tri(t, 2)};
      fwrite(&three, 1, 1, fp);
      fwrite(f, sizeof(int32_t), 3, fp);
    }
    if (fclose(fp) != 0) return NSG_ERR_IO;
    return NSG_OK;
  } else {
    return NSG_ERR_ARG;
  }
  return write_triangle_areas(base, vertices, triangles, n_triangles);
}

// Vertex normals from the triangulation, as approximateNormals does for a surface without analytic
// normals (src/Surface.cpp:10588-10660, updateVertexTrianglesLists :10526-10566): per vertex, the
// sum over its triangles, in triangle order, of the unnormalised plane normal of plane3points
// (src/tools.cpp:258-274), divided by its length.  A vertex without triangles gets 0/0, as there.
int nsg_mesh_normals(const double* vertices, int64_t n_vertices, const int32_t* triangles, int64_t n_triangles,
                     double* normals) {
  if (n_vertices < 0 || n_triangles < 0 || (n_vertices && (!vertices || !normals)) || (n_triangles && !triangles))
    return NSG_ERR_ARG;
  for (int64_t t = 0; t < 3 * n_triangles; t++)
    if (triangles[t] < 0 || triangles[t] >= n_vertices) return NSG_ERR_ARG;
  for (int64_t k = 0; k < 3 * n_vertices; k++) normals[k] = 0.0;
  for (int64_t t = 0; t < n_triangles; t++) {
    const double* p1 = vertices + 3 * (int64_t)triangles[3 * t];
    const double* p2 = vertices + 3 * (int64_t)triangles[3 * t + 1];
    const double* p3 = vertices + 3 * (int64_t)triangles[3 * t + 2];
    const double w0 = p1[1] * (p2[2] - p3[2]) + p2[1] * (p3[2] - p1[2]) + p3[1] * (p1[2] - p2[2]);
    const double w1 = p1[2] * (p2[0] - p3[0]) + p2[2] * (p3[0] - p1[0]) + p3[2] * (p1[0] - p2[0]);
    const double w2 = p1[0] * (p2[1] - p3[1]) + p2[0] * (p3[1] - p1[1]) + p3[0] * (p1[1] - p2[1]);
    for (int q = 0; q < 3; q++) {
      double* nv = normals + 3 * (int64_t)triangles[3 * t + q];
      nv[0] = nv[0] + w0;
      nv[1] = nv[1] + w1;
      nv[2] = nv[2] + w2;
    }
  }
  for (int64_t v = 0; v < n_vertices; v++) {
    double* nv = normals + 3 * v;
    const double len = sqrt(nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2]);
    nv[0] = nv[0] / len;
    nv[1] = nv[1] / len;
    nv[2] = nv[2] / len;
  }
  return NSG_OK;
}

// The vertices whose normal is (0, 0, 0) get the triangle-averaged normal (approximateNormals for
// the listed vertices, src/Surface.cpp:10420-10460, 10660-10735); the others keep theirs.
int nsg_fill_zero_normals(const double* vertices, int64_t n_vertices, const int32_t* triangles, int64_t n_triangles,
                          double* normals) {
  if (n_vertices < 0 || (n_vertices && (!vertices || !normals))) return NSG_ERR_ARG;
  std::vector<double> avg(3 * (size_t)n_vertices);
  int rc = nsg_mesh_normals(vertices, n_vertices, triangles, n_triangles, avg.data());
  if (rc) return rc;
  for (int64_t v = 0; v < n_vertices; v++) {
    double* nv = normals + 3 * v;
    if (nv[0] == 0 && nv[1] == 0 && nv[2] == 0)
      for (int q = 0; q < 3; q++) nv[q] = avg[3 * v + q];
  }
  return NSG_OK;
}

// Nearest atom of every vertex, as vdwAccessible picks it (src/Surface.cpp:16663-16715): the atom of
// least power distance |p - c|^2 - r^2 (ties: the lower index).  The reference searches the atoms
// binned in the grid cells around the vertex; here a uniform grid of cells is searched in growing
// shells until no atom outside the searched cells can win, so the winner is the global one.
// atoms_xyzr: 4 doubles per atom; out: the 0-based atom index per vertex (-1 without atoms).
int nsg_vertex_atoms(const double* vertices, int64_t n_vertices, const double* atoms_xyzr, int64_t n_atoms,
                     int32_t* out) {
  if (n_vertices < 0 || n_atoms < 0 || (n_vertices && (!vertices || !out)) || (n_atoms && !atoms_xyzr))
    return NSG_ERR_ARG;
  if (n_atoms == 0) {
    for (int64_t v = 0; v < n_vertices; v++) out[v] = -1;
    return NSG_OK;
  }
  double lo[3] = {atoms_xyzr[0], atoms_xyzr[1], atoms_xyzr[2]}, hi[3] = {lo[0], lo[1], lo[2]}, rmax = 0.0;
  for (int64_t a = 0; a < n_atoms; a++) {
    for (int d = 0; d < 3; d++) {
      lo[d] = std::min(lo[d], atoms_xyzr[4 * a + d]);
      hi[d] = std::max(hi[d], atoms_xyzr[4 * a + d]);
    }
    rmax = std::max(rmax, atoms_xyzr[4 * a + 3]);
  }
  const double cell = std::max(2.0, rmax);
  int64_t dim[3];
  for (int d = 0; d < 3; d++) dim[d] = std::max<int64_t>(1, (int64_t)((hi[d] - lo[d]) / cell) + 1);
  const int64_t ncell = dim[0] * dim[1] * dim[2];
  std::vector<int64_t> start(ncell + 1, 0);
  std::vector<int32_t> items(n_atoms);
  auto cell_of = [&](const double* p, int d) {
    int64_t c = (int64_t)std::floor((p[d] - lo[d]) / cell);
    return std::min<int64_t>(std::max<int64_t>(c, 0), dim[d] - 1);
  };
  auto cid = [&](int64_t x, int64_t y, int64_t z) { return (z * dim[1] + y) * dim[0] + x; };
  for (int64_t a = 0; a < n_atoms; a++) {
    const double* p = atoms_xyzr + 4 * a;
    start[cid(cell_of(p, 0), cell_of(p, 1), cell_of(p, 2)) + 1]++;
  }
  for (int64_t c = 0; c < ncell; c++) start[c + 1] += start[c];
  std::vector<int64_t> fill(start.begin(), start.end() - 1);
  for (int64_t a = 0; a < n_atoms; a++) {
    const double* p = atoms_xyzr + 4 * a;
    items[fill[cid(cell_of(p, 0), cell_of(p, 1), cell_of(p, 2))]++] = (int32_t)a;
  }
  for (int64_t v = 0; v < n_vertices; v++) {
    const double* p = vertices + 3 * v;
    int64_t c0[3];
    for (int d = 0; d < 3; d++) c0[d] = cell_of(p, d);
    double best = INFINITY;
    int32_t winner = -1;
    // distance from p to the region outside the searched cube of cells [c0 - s, c0 + s]
    for (int64_t s = 0;; s++) {
      for (int64_t z = c0[2] - s; z <= c0[2] + s; z++)
        for (int64_t y = c0[1] - s; y <= c0[1] + s; y++)
          for (int64_t x = c0[0] - s; x <= c0[0] + s; x++) {
            if (x < 0 || y < 0 || z < 0 || x >= dim[0] || y >= dim[1] || z >= dim[2]) continue;
            if (std::max({std::llabs(x - c0[0]), std::llabs(y - c0[1]), std::llabs(z - c0[2])}) != s) continue;
            const int64_t c = cid(x, y, z);
            for (int64_t k = start[c]; k < start[c + 1]; k++) {
              const int32_t a = items[k];
              const double* q = atoms_xyzr + 4 * a;
              const double pd = (q[0] - p[0]) * (q[0] - p[0]) + (q[1] - p[1]) * (q[1] - p[1]) +
                                (q[2] - p[2]) * (q[2] - p[2]) - q[3] * q[3];
              if (pd < best || (pd == best && a < winner)) {
                best = pd;
                winner = a;
              }
            }
          }
      // every atom outside the searched cells is at least `gap` from p
      double gap = INFINITY;
      for (int d = 0; d < 3; d++) {
        if (c0[d] - s > 0) gap = std::min(gap, p[d] - (lo[d] + (double)(c0[d] - s) * cell));
        if (c0[d] + s < dim[d] - 1) gap = std::min(gap, (lo[d] + (double)(c0[d] + s + 1) * cell) - p[d]);
      }
      if (gap == INFINITY) break;  // the whole grid searched
      if (winner >= 0 && gap > 0 && gap * gap - rmax * rmax > best) break;
    }
    out[v] = winner;
  }
  return NSG_OK;
}

// Mesh with per-vertex normals and/or nearest atoms (Surface::saveMesh, src/Surface.cpp:10857-11062):
// format 0 = OFF+N, 1 = MSMS without nearest atoms (root.face, root.vert), 2 = OFF+A, 3 = OFF+N+A,
// 4 = MSMS (nearest atom + 1 in the .vert lines).  normals (3 doubles per vertex) are required by
// formats 0, 1, 3, 4 and atoms (0-based atom index per vertex) by formats 2, 3, 4.  Every format adds
// roottriangleAreas.txt.  revert writes every triangle in the opposite winding.
int nsg_write_mesh_attrs(const char* root, int format, const double* vertices, const double* normals,
                         const int32_t* atoms, int64_t n_vertices, const int32_t* triangles, int64_t n_triangles,
                         int revert) {
  const bool need_n = format == 0 || format == 1 || format == 3 || format == 4;
  const bool need_a = format >= 2;
  if (!root || n_vertices < 0 || n_triangles < 0 || format < 0 || format > 4 || (n_vertices && !vertices) ||
      (n_vertices && need_n && !normals) || (n_vertices && need_a && !atoms) || (n_triangles && !triangles))
    return NSG_ERR_ARG;
  for (int64_t t = 0; t < 3 * n_triangles; t++)
    if (triangles[t] < 0 || triangles[t] >= n_vertices) return NSG_ERR_ARG;
  const std::string base(root);
  auto tri = [&](int64_t t, int q) { return triangles[3 * t + (revert ? 2 - q : q)]; };
  time_t pt;
  time(&pt);
  if (format == 0 || format == 2 || format == 3) {
    FILE* fp = fopen((base + ".off").c_str(), "w");
    if (!fp) return NSG_ERR_IO;
    fprintf(fp, format == 0 ? "OFF+N\n" : (format == 2 ? "OFF+A\n" : "OFF+N+A\n"));
    fprintf(fp, "# File created by %s version %s date %s\n", kProg, kVersion, ctime(&pt));
    fprintf(fp, "%d %d 0\n", (int)n_vertices, (int)n_triangles);
    for (int64_t v = 0; v < n_vertices; v++) {
      const double* x = vertices + 3 * v;
      if (format == 2) {
        fprintf(fp, "%.3f %.3f %.3f %d\n", x[0], x[1], x[2], atoms[v]);
      } else {
        const double* nn = normals + 3 * v;
        if (format == 0)
          fprintf(fp, "%.3f %.3f %.3f %.3f %.3f %.3f\n", x[0], x[1], x[2], nn[0], nn[1], nn[2]);
        else
          fprintf(fp, "%.3f %.3f %.3f %.3f %.3f %.3f %d\n", x[0], x[1], x[2], nn[0], nn[1], nn[2], atoms[v]);
      }
    }
    for (int64_t t = 0; t < n_triangles; t++) fprintf(fp, "3 %d %d %d\n", tri(t, 0), tri(t, 1), tri(t, 2));
    if (fclose(fp) != 0) return NSG_ERR_IO;
  } else {
    FILE* ff = fopen((base + ".face").c_str(), "w");
    if (!ff) return NSG_ERR_IO;
    fprintf(ff, "# File created by %s version %s date %s", kProg, kVersion, ctime(&pt));
    fprintf(ff, "#faces\n");
    fprintf(ff, "%d\n", (int)n_triangles);
    for (int64_t t = 0; t < n_triangles; t++)
      fprintf(ff, "%6d %6d %6d %2d %6d\n", tri(t, 0) + 1, tri(t, 1) + 1, tri(t, 2) + 1, 1, 1);
    if (fclose(ff) != 0) return NSG_ERR_IO;
    FILE* fv = fopen((base + ".vert").c_str(), "w");
    if (!fv) return NSG_ERR_IO;
    fprintf(fv, "# File created by %s version %s date %s", kProg, kVersion, ctime(&pt));
    fprintf(fv, "#vertex\n");
    fprintf(fv, "%d\n", (int)n_vertices);
    for (int64_t v = 0; v < n_vertices; v++)
      fprintf(fv, "%9.3f %9.3f %9.3f %9.3f %9.3f %9.3f %7d %7d %2d \n", vertices[3 * v], vertices[3 * v + 1],
              vertices[3 * v + 2], normals[3 * v], normals[3 * v + 1], normals[3 * v + 2], 0,
              format == 4 ? atoms[v] + 1 : 1, 0);
    if (fclose(fv) != 0) return NSG_ERR_IO;
  }
  return write_triangle_areas(base, vertices, triangles, n_triangles);
}

}  // extern "C"
