// Blobby surface on the device: the Gaussian scalar field of the atoms, its marching-cubes mesh,
// one Laplacian smoothing pass and the reference's OFF round trip, as triangle patches for the
// ray caster; and the adjoint of that chain back to the atoms.
//
// The reference (BlobbySurface::build, src/BlobbySurface.cpp:83-229) sums exp(B (d^2/r^2 - 1))
// of every atom over the grid nodes of a cube of +-round(6 A / side) nodes around it, at the
// points (x_i - hside, y_j - hside, z_k - hside); runs the classical marching cubes on the field
// at iso level 1 (Surface::triangulateSurface with a scalar field, src/Surface.cpp:9909-10526:
// getVertices :8143-8327 interpolates the vertices of each cube's own edges 5, 6 and 10,
// triangulationKernel :9075-9318 keeps the case table's winding); smooths the mesh once
// (Surface::smoothSurface, src/Surface.cpp:13089-13354); writes it as blobby.off ("%.3f"
// vertices) and reloads it as a MeshSurface (MeshSurface::loadOFF, src/MeshSurface.cpp:2350-2479,
// float vertices).  Here each step is a kernel over the whole grid or mesh:
//   * field: one CTA per 16x4x4-node tile gathers, chunk by chunk in atom order, the atoms whose
//     cube reaches the tile into shared memory, so every node sums its atoms in the reference's
//     order (only exp's last bit can differ from the host's);
//   * marching cubes: cubes classified and counted, vertices and triangles numbered by prefix sums
//     in the reference's serial (k, j, i) order; an edge has a vertex when it is cut and its owner
//     cube lies in the cube range, which is what makes the reference skip boundary triangles;
//   * smoothing: each vertex sums its triangles' contributions in triangle order (a per-vertex
//     incidence list sorted by triangle), bit for bit the reference's accumulation;
//   * OFF round trip: the exact round-half-even of v * 1000 (an FMA gives the product's rounding
//     error), then the float nearest to n / 1000, as printf("%.3f") and sscanf("%f") produce.
#include <cub/cub.cuh>

#include "blobby.h"
#include "pipeline.h"
#include "../mc_cases.h"

namespace nsg {

namespace {

constexpr int kTX = 16, kTY = 4, kTZ = 4;
constexpr int kFieldThreads = kTX * kTY * kTZ;

__device__ __forceinline__ double rintp_d(double x) { return floor(x + 0.5); }

__device__ __forceinline__ void atom_window(const GridDev& g, const double* a, int ng, int lo[3], int hi[3]) {
  for (int d = 0; d < 3; d++) {
    const int ic = (int)rintp_d((a[d] - g.mn[d]) * g.scale);
    lo[d] = ic - ng > 0 ? ic - ng : 0;
    hi[d] = ic + ng < (int)g.n[d] ? ic + ng : (int)g.n[d];  // exclusive
  }
}

__global__ void __launch_bounds__(kFieldThreads) k_blobby_field(GridDev g, const double* __restrict__ atoms, int na,
                                                               double B, int ng, double* __restrict__ field) {
  __shared__ int s_list[kFieldThreads];
  __shared__ int s_warp[kFieldThreads / 32];
  const int tid = threadIdx.x;
  const int tx = tid % kTX, ty = (tid / kTX) % kTY, tz = tid / (kTX * kTY);
  const int tilesx = ((int)g.n[0] + kTX - 1) / kTX, tilesy = ((int)g.n[1] + kTY - 1) / kTY;
  const int bt = blockIdx.x;
  const int i0 = (bt % tilesx) * kTX, j0 = ((bt / tilesx) % tilesy) * kTY, k0 = (bt / (tilesx * tilesy)) * kTZ;
  const int i = i0 + tx, j = j0 + ty, k = k0 + tz;
  const bool valid = i < g.n[0] && j < g.n[1] && k < g.n[2];
  double p[3];
  p[0] = (g.mn[0] + (double)i * g.side) - g.hside;
  p[1] = (g.mn[1] + (double)j * g.side) - g.hside;
  p[2] = (g.mn[2] + (double)k * g.side) - g.hside;
  double acc = 0.0;
  const int lane = tid & 31, warp = tid >> 5;
  for (int base = 0; base < na; base += kFieldThreads) {
    const int a = base + tid;
    bool take = false;
    if (a < na) {
      int lo[3], hi[3];
      atom_window(g, atoms + 4 * (int64_t)a, ng, lo, hi);
      take = lo[0] < i0 + kTX && hi[0] > i0 && lo[1] < j0 + kTY && hi[1] > j0 && lo[2] < k0 + kTZ && hi[2] > k0;
    }
    // order-preserving compaction of the chunk's atoms that reach the tile
    const unsigned m = __ballot_sync(0xffffffffu, take);
    if (lane == 0) s_warp[warp] = __popc(m);
    __syncthreads();
    int before = 0, total = 0;
    for (int w = 0; w < kFieldThreads / 32; w++) {
      if (w < warp) before += s_warp[w];
      total += s_warp[w];
    }
    if (take) s_list[before + __popc(m & ((1u << lane) - 1u))] = a;
    __syncthreads();
    if (valid)
      for (int q = 0; q < total; q++) {
        const double* at = atoms + 4 * (int64_t)s_list[q];
        int lo[3], hi[3];
        atom_window(g, at, ng, lo, hi);
        if (i < lo[0] || i >= hi[0] || j < lo[1] || j >= hi[1] || k < lo[2] || k >= hi[2]) continue;
        const double r = at[3];
        const double r2 = r * r;
        const double dist2 = (p[0] - at[0]) * (p[0] - at[0]) + (p[1] - at[1]) * (p[1] - at[1]) +
                             (p[2] - at[2]) * (p[2] - at[2]);
        acc += exp(B * (dist2 / r2 - 1));
      }
    __syncthreads();
  }
  if (valid) field[((int64_t)k * g.n[1] + j) * g.n[0] + i] = acc;
}

__constant__ int8_t c_tri[256][16];
__constant__ int c_edge_mask[256];

__device__ __forceinline__ int64_t nidx(const GridDev& g, int64_t i, int64_t j, int64_t k) {
  return (k * g.n[1] + j) * g.n[0] + i;
}

// Cube (i, j, k), 1 <= i <= nx-2 etc., by linear index c over the cube range.
__device__ __forceinline__ void cube_of(const GridDev& g, int64_t c, int64_t* i, int64_t* j, int64_t* k) {
  const int64_t cx = g.n[0] - 2, cy = g.n[1] - 2;
  *i = 1 + c % cx;
  *j = 1 + (c / cx) % cy;
  *k = 1 + c / (cx * cy);
}

__device__ __forceinline__ int64_t cube_index(const GridDev& g, int64_t i, int64_t j, int64_t k) {
  return ((k - 1) * (g.n[1] - 2) + (j - 1)) * (g.n[0] - 2) + (i - 1);
}

// Case index of cube (i, j, k): bit v set when corner v's value is below the iso level
// (classifyCube, src/Surface.cpp:14526-14545).
__device__ __forceinline__ int classify(const GridDev& g, const double* f, int64_t i, int64_t j, int64_t k, double iso,
                                        double vals[8]) {
  vals[0] = f[nidx(g, i, j, k)];
  vals[1] = f[nidx(g, i + 1, j, k)];
  vals[2] = f[nidx(g, i + 1, j + 1, k)];
  vals[3] = f[nidx(g, i, j + 1, k)];
  vals[4] = f[nidx(g, i, j, k + 1)];
  vals[5] = f[nidx(g, i + 1, j, k + 1)];
  vals[6] = f[nidx(g, i + 1, j + 1, k + 1)];
  vals[7] = f[nidx(g, i, j + 1, k + 1)];
  int c = 0;
  for (int v = 0; v < 8; v++)
    if (vals[v] < iso) c |= 1 << v;
  return c;
}

// Grid edge of cube edge e: (x, y, z, dir) as getTriangles indexes its intersection matrices.
__device__ __forceinline__ int4 edge_key(int64_t i, int64_t j, int64_t k, int e) {
  switch (e) {
    case 0: return make_int4((int)i, (int)j, (int)k, 0);
    case 1: return make_int4((int)i + 1, (int)j, (int)k, 1);
    case 2: return make_int4((int)i, (int)j + 1, (int)k, 0);
    case 3: return make_int4((int)i, (int)j, (int)k, 1);
    case 4: return make_int4((int)i, (int)j, (int)k + 1, 0);
    case 5: return make_int4((int)i + 1, (int)j, (int)k + 1, 1);
    case 6: return make_int4((int)i, (int)j + 1, (int)k + 1, 0);
    case 7: return make_int4((int)i, (int)j, (int)k + 1, 1);
    case 8: return make_int4((int)i, (int)j, (int)k, 2);
    case 9: return make_int4((int)i + 1, (int)j, (int)k, 2);
    case 10: return make_int4((int)i + 1, (int)j + 1, (int)k, 2);
    default: return make_int4((int)i, (int)j + 1, (int)k, 2);
  }
}

// The cube that owns a grid edge (its edge 6 for x, 5 for y, 10 for z) and the slot of that edge
// among the owner's edges 5, 6, 10.
__device__ __forceinline__ void edge_owner(int4 key, int64_t* oi, int64_t* oj, int64_t* ok, int* slot) {
  if (key.w == 0) { *oi = key.x; *oj = key.y - 1; *ok = key.z - 1; *slot = 1; }
  else if (key.w == 1) { *oi = key.x - 1; *oj = key.y; *ok = key.z - 1; *slot = 0; }
  else { *oi = key.x - 1; *oj = key.y - 1; *ok = key.z; *slot = 2; }
}

__device__ __forceinline__ bool cube_in_range(const GridDev& g, int64_t i, int64_t j, int64_t k) {
  return i >= 1 && i <= g.n[0] - 2 && j >= 1 && j <= g.n[1] - 2 && k >= 1 && k <= g.n[2] - 2;
}

// Per cube: own-edge cut mask (bit 0 edge 5, bit 1 edge 6, bit 2 edge 10), vertex and triangle
// counts (triangles whose three edges all have a vertex).
__global__ void k_field_cubes(GridDev g, const double* __restrict__ f, double iso, int64_t ncubes, uint8_t* mask,
                              int32_t* nvert, int32_t* ntri) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ncubes; c += (int64_t)gridDim.x * blockDim.x) {
    int64_t i, j, k;
    cube_of(g, c, &i, &j, &k);
    double vals[8];
    const int ci = classify(g, f, i, j, k, iso, vals);
    const int em = c_edge_mask[ci];
    uint8_t m = 0;
    if (em & 32) m |= 1;
    if (em & 64) m |= 2;
    if (em & 1024) m |= 4;
    mask[c] = m;
    nvert[c] = __popc(m);
    int nt = 0;
    if (em)
      for (int q = 0; q < 16 && c_tri[ci][q] >= 0; q += 3) {
        bool ok = true;
        for (int r = 0; r < 3; r++) {
          int64_t oi, oj, ok2;
          int slot;
          edge_owner(edge_key(i, j, k, c_tri[ci][q + r]), &oi, &oj, &ok2, &slot);
          if (!cube_in_range(g, oi, oj, ok2)) ok = false;
        }
        nt += ok;
      }
    ntri[c] = nt;
  }
}

// Vertex of an own edge by vertexInterp (src/Surface.cpp:14516-14523) between the cube corner
// positions x +- hside etc. (the mulTable corners), and its grid edge.
__global__ void k_field_verts(GridDev g, const double* __restrict__ f, double iso, int64_t ncubes,
                              const uint8_t* __restrict__ mask, const int64_t* __restrict__ vbase, double* verts,
                              int4* vkey) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ncubes; c += (int64_t)gridDim.x * blockDim.x) {
    const uint8_t m = mask[c];
    if (!m) continue;
    int64_t i, j, k;
    cube_of(g, c, &i, &j, &k);
    double vals[8];
    classify(g, f, i, j, k, iso, vals);
    const double xg = g.mn[0] + (double)i * g.side, yg = g.mn[1] + (double)j * g.side, zg = g.mn[2] + (double)k * g.side;
    const double tb[6] = {xg - g.hside, xg + g.hside, yg - g.hside, yg + g.hside, zg - g.hside, zg + g.hside};
    // corners 2, 5, 6, 7 of the mulTable: (1,3,4), (1,2,5), (1,3,5), (0,3,5)
    const double c2[3] = {tb[1], tb[3], tb[4]}, c5[3] = {tb[1], tb[2], tb[5]}, c6[3] = {tb[1], tb[3], tb[5]},
                 c7[3] = {tb[0], tb[3], tb[5]};
    int64_t id = vbase[c];
    const int ed[3] = {5, 6, 10};
    for (int s = 0; s < 3; s++) {
      if (!((m >> s) & 1)) continue;
      const double *p1, *p2;
      double v1, v2;
      if (s == 0) { p1 = c5; p2 = c6; v1 = vals[5]; v2 = vals[6]; }
      else if (s == 1) { p1 = c6; p2 = c7; v1 = vals[6]; v2 = vals[7]; }
      else { p1 = c2; p2 = c6; v1 = vals[2]; v2 = vals[6]; }
      const double mu = (iso - v1) / (v2 - v1);
      double* o = verts + 3 * id;
      for (int d = 0; d < 3; d++) {
        const double tmp = p2[d] - p1[d];
        o[d] = p1[d] + mu * tmp;
      }
      vkey[id] = edge_key(i, j, k, ed[s]);
      id++;
    }
  }
}

__global__ void k_field_tris(GridDev g, const double* __restrict__ f, double iso, int64_t ncubes,
                             const uint8_t* __restrict__ mask, const int64_t* __restrict__ vbase,
                             const int64_t* __restrict__ tbase, const int32_t* __restrict__ ntri, int32_t* tris) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ncubes; c += (int64_t)gridDim.x * blockDim.x) {
    if (!ntri[c]) continue;
    int64_t i, j, k;
    cube_of(g, c, &i, &j, &k);
    double vals[8];
    const int ci = classify(g, f, i, j, k, iso, vals);
    int64_t t = tbase[c];
    for (int q = 0; q < 16 && c_tri[ci][q] >= 0; q += 3) {
      int32_t vid[3];
      bool ok = true;
      for (int r = 0; r < 3; r++) {
        int64_t oi, oj, ok2;
        int slot;
        edge_owner(edge_key(i, j, k, c_tri[ci][q + r]), &oi, &oj, &ok2, &slot);
        if (!cube_in_range(g, oi, oj, ok2)) {
          ok = false;
          break;
        }
        const int64_t oc = cube_index(g, oi, oj, ok2);
        const uint8_t om = mask[oc];
        vid[r] = (int32_t)(vbase[oc] + __popc(om & ((1u << slot) - 1u)));
      }
      if (!ok) continue;
      tris[3 * t] = vid[0];
      tris[3 * t + 1] = vid[1];
      tris[3 * t + 2] = vid[2];
      t++;
    }
  }
}

__global__ void k_incidence_count(const int32_t* __restrict__ tris, int64_t nt, int32_t* cnt) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nt; t += (int64_t)gridDim.x * blockDim.x)
    for (int r = 0; r < 3; r++) atomicAdd(cnt + tris[3 * t + r], 1);
}

__global__ void k_incidence_fill(const int32_t* __restrict__ tris, int64_t nt, const int64_t* __restrict__ off,
                                 int32_t* cursor, int32_t* inc) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nt; t += (int64_t)gridDim.x * blockDim.x)
    for (int r = 0; r < 3; r++) {
      const int32_t v = tris[3 * t + r];
      const int32_t pos = atomicAdd(cursor + v, 1);
      inc[off[v] + pos] = (int32_t)(t * 3 + r);  // triangle and corner
    }
}

// One Laplacian step (smoothSurface): every vertex adds, triangle by triangle in triangle order,
// the sum of the triangle's two other corners; v' = 0.5 (v + sum / (2 count)).
__global__ void k_smooth(const double* __restrict__ vin, int64_t nv, const int64_t* __restrict__ off,
                         int32_t* inc, const int32_t* __restrict__ tris, double* vout) {
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nv; v += (int64_t)gridDim.x * blockDim.x) {
    const int64_t a = off[v], b = off[v + 1];
    // the incidence list in triangle order (short lists: insertion sort)
    for (int64_t x = a + 1; x < b; x++) {
      const int32_t key = inc[x];
      int64_t y = x;
      while (y > a && inc[y - 1] > key) {
        inc[y] = inc[y - 1];
        y--;
      }
      inc[y] = key;
    }
    double acc[3] = {0.0, 0.0, 0.0};
    for (int64_t x = a; x < b; x++) {
      const int32_t t = inc[x] / 3, r = inc[x] % 3;
      const int32_t o1 = tris[3 * t + (r == 0 ? 1 : 0)], o2 = tris[3 * t + (r == 2 ? 1 : 2)];
      for (int d = 0; d < 3; d++) acc[d] += vin[3 * o1 + d] + vin[3 * o2 + d];
    }
    const double scale = 1.0 / (double)(int)(2 * (b - a));
    for (int d = 0; d < 3; d++) vout[3 * v + d] = 0.5 * (vin[3 * v + d] + acc[d] * scale);
  }
}

// printf("%.3f") then sscanf("%f"): n = the exact round-half-even of v * 1000, then the float
// nearest to n / 1000 (never a double-rounding case: n / 1000 is never within 2^-53 of a float
// midpoint).
__device__ __forceinline__ double off_round_trip(double v) {
  if (!(fabs(v) < 1e15)) return (double)(float)v;  // inf / nan pass through as the text does
  const double p = v * 1000.0;
  const double e = fma(v, 1000.0, -p);  // v * 1000 = p + e exactly
  const double fl = floor(p);
  const double d = p - fl;  // exact
  double n;
  if (d < 0.25) n = fl;
  else if (d > 0.75) n = fl + 1.0;
  else {
    const double s = (d - 0.5) + e;
    if (s < 0) n = fl;
    else if (s > 0) n = fl + 1.0;
    else n = fmod(fl, 2.0) == 0.0 ? fl : fl + 1.0;
  }
  return (double)(float)(n / 1000.0);
}

__global__ void k_quantize(double* v, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    v[i] = off_round_trip(v[i]);
}

__global__ void k_tri_patches(const double* __restrict__ verts, const int32_t* __restrict__ tris, int64_t nt,
                              double* f64, int32_t* i32, int32_t* patch_atoms) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nt; t += (int64_t)gridDim.x * blockDim.x) {
    double* r = f64 + (int64_t)NS_PATCH_F64 * t;
    const double* p[3];
    for (int q = 0; q < 3; q++) {
      const int32_t v = tris[3 * t + q];
      p[q] = verts + 3 * (int64_t)v;
      patch_atoms[3 * t + q] = v;
      for (int d = 0; d < 3; d++) r[3 * q + d] = p[q][d];
    }
    const double e1[3] = {p[1][0] - p[0][0], p[1][1] - p[0][1], p[1][2] - p[0][2]};
    const double e2[3] = {p[2][0] - p[0][0], p[2][1] - p[0][1], p[2][2] - p[0][2]};
    r[NS_TRI_N] = e1[1] * e2[2] - e1[2] * e2[1];
    r[NS_TRI_N + 1] = e1[2] * e2[0] - e1[0] * e2[2];
    r[NS_TRI_N + 2] = e1[0] * e2[1] - e1[1] * e2[0];
    r[12] = 0.0;
    r[13] = 0.0;
    for (int d = 0; d < 3; d++) {
      r[NS_SKIN_LO + d] = fmin(p[0][d], fmin(p[1][d], p[2][d]));
      r[NS_SKIN_HI + d] = fmax(p[0][d], fmax(p[1][d], p[2][d]));
    }
    int32_t* ir = i32 + NS_PATCH_I32 * t;
    ir[0] = NS_MESH_TRI;
    ir[1] = 0;
    ir[2] = 0;
    ir[3] = 0;
  }
}

// ---- adjoint ----

// d L / d mesh vertex (ray-cast mesh) from the per-triangle slots S_k (hit terms b_k / n_vc summed
// with their weights): corner k of triangle t gets n_t S_k.
__global__ void k_tri_chain(const double* __restrict__ f64, const int32_t* __restrict__ patch_atoms,
                            const double* __restrict__ gpatch, int64_t nt, double* gvert) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nt; t += (int64_t)gridDim.x * blockDim.x) {
    const double* n = f64 + (int64_t)NS_PATCH_F64 * t + NS_TRI_N;
    const double* s = gpatch + (int64_t)NS_GRAD_PER_PATCH * t;
    for (int q = 0; q < 3; q++) {
      if (s[q] == 0.0) continue;
      double* o = gvert + 3 * (int64_t)patch_atoms[3 * t + q];
      for (int d = 0; d < 3; d++) atomicAdd(o + d, n[d] * s[q]);
    }
  }
}

// Transpose of the smoothing step: g_pre = 0.5 g_post + sum over triangles of 0.5 / (2 count_u)
// g_post[u] for every other corner.
__global__ void k_smooth_adjoint_self(const double* __restrict__ gpost, int64_t nv, double* gpre) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < 3 * nv; i += (int64_t)gridDim.x * blockDim.x)
    gpre[i] = 0.5 * gpost[i];
}

__global__ void k_smooth_adjoint_tris(const int32_t* __restrict__ tris, int64_t nt, const int32_t* __restrict__ cnt,
                                      const double* __restrict__ gpost, double* gpre) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nt; t += (int64_t)gridDim.x * blockDim.x)
    for (int r = 0; r < 3; r++) {
      const int32_t u = tris[3 * t + r];
      const double w = 0.5 / (double)(2 * cnt[u]);
      for (int s = 1; s < 3; s++) {
        const int32_t o = tris[3 * t + (r + s) % 3];
        for (int d = 0; d < 3; d++) atomicAdd(gpre + 3 * (int64_t)o + d, w * gpost[3 * (int64_t)u + d]);
      }
    }
}

// Transpose of the interpolated vertices: p = p1 + mu (p2 - p1), mu = (iso - f1) / (f2 - f1).
__global__ void k_mc_adjoint(GridDev g, const double* __restrict__ f, double iso, const int4* __restrict__ vkey,
                             const double* __restrict__ gv, int64_t nv, double* gfield) {
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nv; v += (int64_t)gridDim.x * blockDim.x) {
    const int4 key = vkey[v];
    int64_t a[3] = {key.x, key.y, key.z}, b[3] = {key.x, key.y, key.z};
    b[key.w] += 1;
    const int64_t na = nidx(g, a[0], a[1], a[2]), nb = nidx(g, b[0], b[1], b[2]);
    const double f1 = f[na], f2 = f[nb];
    const double df = f2 - f1;
    // p2 - p1 is one grid step along the edge's axis
    const double dot = gv[3 * v + key.w] * g.side;
    const double inv2 = 1.0 / (df * df);
    atomicAdd(gfield + na, dot * (iso - f2) * inv2);
    atomicAdd(gfield + nb, -dot * (iso - f1) * inv2);
  }
}

// Transpose of the field: one warp per atom over its cube of nodes.
__global__ void k_field_adjoint(GridDev g, const double* __restrict__ atoms, int na, double B, int ng,
                                const double* __restrict__ gfield, double* gatoms) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t a = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; a < na; a += warps) {
    const double* at = atoms + 4 * a;
    int lo[3], hi[3];
    atom_window(g, at, ng, lo, hi);
    const int nxw = hi[0] - lo[0], nyw = hi[1] - lo[1], nzw = hi[2] - lo[2];
    const int64_t tot = (nxw > 0 && nyw > 0 && nzw > 0) ? (int64_t)nxw * nyw * nzw : 0;
    const double r = at[3], r2 = r * r;
    double gx = 0, gy = 0, gz = 0, gr = 0;
    for (int64_t q = lane; q < tot; q += 32) {
      const int i = lo[0] + (int)(q % nxw), j = lo[1] + (int)((q / nxw) % nyw), k = lo[2] + (int)(q / ((int64_t)nxw * nyw));
      const double gf = gfield[nidx(g, i, j, k)];
      if (gf == 0.0) continue;
      const double px = (g.mn[0] + (double)i * g.side) - g.hside;
      const double py = (g.mn[1] + (double)j * g.side) - g.hside;
      const double pz = (g.mn[2] + (double)k * g.side) - g.hside;
      const double dx = px - at[0], dy = py - at[1], dz = pz - at[2];
      const double d2 = dx * dx + dy * dy + dz * dz;
      const double e = exp(B * (d2 / r2 - 1)) * B * gf;
      gx += e * (-2.0 * dx / r2);
      gy += e * (-2.0 * dy / r2);
      gz += e * (-2.0 * dz / r2);
      gr += e * (-2.0 * d2 / (r2 * r));
    }
    for (int o = 16; o; o >>= 1) {
      gx += __shfl_xor_sync(0xffffffffu, gx, o);
      gy += __shfl_xor_sync(0xffffffffu, gy, o);
      gz += __shfl_xor_sync(0xffffffffu, gz, o);
      gr += __shfl_xor_sync(0xffffffffu, gr, o);
    }
    if (lane == 0) {
      gatoms[4 * a] += gx;
      gatoms[4 * a + 1] += gy;
      gatoms[4 * a + 2] += gz;
      gatoms[4 * a + 3] += gr;
    }
  }
}

int grid_for(int64_t n, int threads = 256) {
  int64_t b = (n + threads - 1) / threads;
  const int64_t cap = (int64_t)sm_count() * 32;
  return (int)(b < cap ? (b < 1 ? 1 : b) : cap);
}

}  // namespace

cudaError_t blobby_init_tables() {
  static bool done[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 64 && done[dev]) return cudaSuccess;
  int8_t tri[256][16];
  int em[256];
  static const int ec[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6}, {6, 7}, {7, 4},
                                {0, 4}, {1, 5}, {2, 6}, {3, 7}};
  for (int c = 0; c < 256; c++) {
    const char* s = kNsMcCases[c];
    int q = 0;
    for (; s[q]; q++) tri[c][q] = (int8_t)(s[q] <= '9' ? s[q] - '0' : s[q] - 'a' + 10);
    for (; q < 16; q++) tri[c][q] = -1;
    int m = 0;
    for (int e = 0; e < 12; e++)
      if (((c >> ec[e][0]) & 1) != ((c >> ec[e][1]) & 1)) m |= 1 << e;
    em[c] = m;
  }
  cudaError_t e = cudaMemcpyToSymbol(c_tri, tri, sizeof tri);
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_edge_mask, em, sizeof em);
  if (e == cudaSuccess && dev >= 0 && dev < 64) done[dev] = true;
  return e;
}

cudaError_t launch_blobby_field(const GridDev& g, const double* atoms, int na, double B, int ng, double* field,
                                cudaStream_t s) {
  const int64_t tiles = ((g.n[0] + kTX - 1) / kTX) * ((g.n[1] + kTY - 1) / kTY) * ((g.n[2] + kTZ - 1) / kTZ);
  k_blobby_field<<<(unsigned)tiles, kFieldThreads, 0, s>>>(g, atoms, na, B, ng, field);
  return cudaGetLastError();
}

cudaError_t launch_field_cubes(const GridDev& g, const double* f, double iso, int64_t ncubes, uint8_t* mask,
                               int32_t* nvert, int32_t* ntri, cudaStream_t s) {
  k_field_cubes<<<grid_for(ncubes), 256, 0, s>>>(g, f, iso, ncubes, mask, nvert, ntri);
  return cudaGetLastError();
}

cudaError_t launch_field_verts(const GridDev& g, const double* f, double iso, int64_t ncubes, const uint8_t* mask,
                               const int64_t* vbase, double* verts, int4* vkey, cudaStream_t s) {
  k_field_verts<<<grid_for(ncubes), 256, 0, s>>>(g, f, iso, ncubes, mask, vbase, verts, vkey);
  return cudaGetLastError();
}

cudaError_t launch_field_tris(const GridDev& g, const double* f, double iso, int64_t ncubes, const uint8_t* mask,
                              const int64_t* vbase, const int64_t* tbase, const int32_t* ntri, int32_t* tris,
                              cudaStream_t s) {
  k_field_tris<<<grid_for(ncubes), 256, 0, s>>>(g, f, iso, ncubes, mask, vbase, tbase, ntri, tris);
  return cudaGetLastError();
}

cudaError_t launch_incidence(const int32_t* tris, int64_t nt, int phase, const int64_t* off, int32_t* cnt_or_cursor,
                             int32_t* inc, cudaStream_t s) {
  if (nt <= 0) return cudaSuccess;
  if (phase == 0) k_incidence_count<<<grid_for(nt), 256, 0, s>>>(tris, nt, cnt_or_cursor);
  else k_incidence_fill<<<grid_for(nt), 256, 0, s>>>(tris, nt, off, cnt_or_cursor, inc);
  return cudaGetLastError();
}

cudaError_t launch_smooth(const double* vin, int64_t nv, const int64_t* off, int32_t* inc, const int32_t* tris,
                          double* vout, cudaStream_t s) {
  if (nv <= 0) return cudaSuccess;
  k_smooth<<<grid_for(nv), 256, 0, s>>>(vin, nv, off, inc, tris, vout);
  return cudaGetLastError();
}

cudaError_t launch_quantize(double* v, int64_t n, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_quantize<<<grid_for(n), 256, 0, s>>>(v, n);
  return cudaGetLastError();
}

cudaError_t launch_tri_patches(const double* verts, const int32_t* tris, int64_t nt, double* f64, int32_t* i32,
                               int32_t* patch_atoms, cudaStream_t s) {
  if (nt <= 0) return cudaSuccess;
  k_tri_patches<<<grid_for(nt), 256, 0, s>>>(verts, tris, nt, f64, i32, patch_atoms);
  return cudaGetLastError();
}

cudaError_t launch_blobby_adjoint(const GridDev& g, const double* atoms, int na, double B, int ng, const double* field,
                                  double iso, const BlobbyMeshDev& M, const double* gpatch, double* gvert_post,
                                  double* gvert_pre, double* gfield, double* gatoms, cudaStream_t s) {
  cudaError_t e;
  if ((e = cudaMemsetAsync(gvert_post, 0, 3 * std::max<int64_t>(M.nv, 1) * sizeof(double), s)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(gfield, 0, g.n[0] * g.n[1] * g.n[2] * sizeof(double), s)) != cudaSuccess) return e;
  if (M.nt > 0) k_tri_chain<<<grid_for(M.nt), 256, 0, s>>>(M.f64, M.patch_atoms, gpatch, M.nt, gvert_post);
  if (M.nv > 0) {
    k_smooth_adjoint_self<<<grid_for(3 * M.nv), 256, 0, s>>>(gvert_post, M.nv, gvert_pre);
    if (M.nt > 0) k_smooth_adjoint_tris<<<grid_for(M.nt), 256, 0, s>>>(M.tris, M.nt, M.inc_cnt, gvert_post, gvert_pre);
    k_mc_adjoint<<<grid_for(M.nv), 256, 0, s>>>(g, field, iso, M.vkey, gvert_pre, M.nv, gfield);
  }
  if (na > 0) k_field_adjoint<<<grid_for((int64_t)na * 32), 256, 0, s>>>(g, atoms, na, B, ng, gfield, gatoms);
  return cudaGetLastError();
}

}  // namespace nsg
