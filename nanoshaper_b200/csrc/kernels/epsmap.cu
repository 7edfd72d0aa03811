// Epsilon and ideb maps after the ray cast, boundary grid points and their projection onto the
// SES.
//
// The epsilon map itself is written by the fill kernels of the node rays (trace.cu: status rays
// for the x edges, ray sets 4 and 5 for the z and y edges); this file adds what follows the ray
// cast in Surface::getSurf: cavity filling on the map (fillCavities), the ideb map, the boundary
// grid points (nodes where the six edge codes differ, src/Surface.cpp:1488-1546) and the
// projection of the external ones (Surface::projector, src/Surface.cpp:4657-4676, with
// ConnollySurface::getProjection, src/ConnollySurface.cpp:5822-5912).
//
// Layout in HBM: the epsilon map in the reference's interleaved 4-D layout, 3 int32 per node
// (x, y, z edge), so that it downloads as is; the ideb map 1 byte per node.  Both are touched once
// per node by grid-stride kernels (HBM-bound); the projection is one warp per boundary point over
// the patch list of its auxiliary cell.
#include <cub/cub.cuh>

#include "epsmap.h"
#include "ray_math.cuh"

namespace nsg {

namespace {

int grid_for(int64_t n, int threads = 256) {
  int64_t b = (n + threads - 1) / threads;
  const int64_t cap = (int64_t)sm_count() * 32;
  return (int)(b < cap ? (b < 1 ? 1 : b) : cap);
}

__global__ void k_eps_fill_cavities(RunArgs A, const uint8_t* __restrict__ fill_of, int32_t* eps, int32_t inside) {
  for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < A.nruns; u += (int64_t)gridDim.x * blockDim.x) {
    if (!fill_of[A.L[u]]) continue;
    const int64_t r = A.frow[u];  // k*ny + j
    const int2 ru = A.fruns[u];
    const int64_t j = r % A.ny;
    const int64_t k = r / A.ny;
    for (int64_t i = ru.x; i <= ru.y; i++) {
      const int64_t f = r * A.nx + i;
      eps[3 * f] = inside;
      eps[3 * f + 1] = inside;
      eps[3 * f + 2] = inside;
      // the edges that end at the node (a cavity never touches the grid boundary; guarded anyway)
      if (i > 0) eps[3 * (f - 1)] = inside;
      if (j > 0) eps[3 * (f - A.nx) + 1] = inside;
      if (k > 0) eps[3 * (f - A.nx * A.ny) + 2] = inside;
    }
  }
}

// One warp per x-row: the inside segments between the free runs are 0, a free run is 1 unless its
// region is a filled cavity.
__global__ void k_ideb_write(RunArgs A, const uint8_t* __restrict__ fill_of, uint8_t* ideb) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t r = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); r < A.nrows; r += warps) {
    const int64_t b = A.fr_off[r], e = A.fr_off[r + 1];
    uint8_t* row = ideb + r * A.nx;
    int64_t next = 0;
    for (int64_t u = b; u <= e; u++) {
      int64_t x0 = A.nx, x1 = A.nx - 1;
      uint8_t v = 1;
      if (u < e) {
        const int2 ru = A.fruns[u];
        x0 = ru.x;
        x1 = ru.y;
        if (fill_of && fill_of[A.L[u]]) v = 0;
      }
      for (int64_t i = next + lane; i < x0; i += 32) row[i] = 0;
      for (int64_t i = x0 + lane; i <= x1; i += 32) row[i] = v;
      next = x1 + 1;
    }
  }
}

// The six edge codes around node f = (k*ny + j)*nx + i (i, j, k >= 1).
struct BgpPred {
  const int32_t* eps;
  int64_t nx, ny, nz;
  __device__ __forceinline__ bool operator()(const int32_t f) const {
    const int64_t i = f % nx, j = (f / nx) % ny, k = f / (nx * ny);
    if (i < 1 || j < 1 || k < 1) return false;
    const int32_t c = eps[3 * (int64_t)f];
    return c != eps[3 * (int64_t)f + 1] || c != eps[3 * (int64_t)f + 2] || c != eps[3 * ((int64_t)f - 1)] ||
           c != eps[3 * ((int64_t)f - nx) + 1] || c != eps[3 * ((int64_t)f - nx * ny) + 2];
  }
};

__global__ void k_bgp_expand(const int32_t* __restrict__ eps, int64_t nx, int64_t ny, const int32_t* __restrict__ nodes,
                             int32_t n, int32_t* ibgp, int32_t* type) {
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t f = nodes[q];
    ibgp[3 * q] = (int32_t)(f % nx);
    ibgp[3 * q + 1] = (int32_t)((f / nx) % ny);
    ibgp[3 * q + 2] = (int32_t)(f / (nx * ny));
    const bool ext = eps[3 * f] == 0 || eps[3 * f + 1] == 0 || eps[3 * f + 2] == 0 || eps[3 * (f - 1)] == 0 ||
                     eps[3 * (f - nx) + 1] == 0 || eps[3 * (f - nx * ny) + 2] == 0;
    type[q] = ext ? NS_EXTERNAL_BGP : NS_INTERNAL_BGP;
  }
}

// Cell range of a patch's bounding-sphere box on the auxiliary grid (src/ConnollySurface.cpp:3840-3870).
__device__ __forceinline__ void aux_box(const double* f, const AuxGrid& a, int64_t lo[3], int64_t hi[3]) {
  const double r = f[3];
  for (int d = 0; d < 3; d++) {
    lo[d] = (int64_t)rintp(fmax(0., (f[d] - r) - a.mn[d]) * a.scale);
    hi[d] = (int64_t)rintp(fmax(0., (f[d] + r) - a.mn[d]) * a.scale);
    if (lo[d] >= a.n) lo[d] = a.n - 1;
    if (hi[d] >= a.n) hi[d] = a.n - 1;
  }
}

// Cell range of a mesh triangle: its vertices' box (MeshSurface::buildAuxiliaryGrid,
// src/MeshSurface.cpp:867-929); the reference stops on a box outside the grid, here it is clamped.
__device__ __forceinline__ void aux_box_tri(const double* f, const AuxGrid& a, int64_t lo[3], int64_t hi[3]) {
  for (int d = 0; d < 3; d++) {
    double dn = 1e20, up = -1e20;
    for (int v = 0; v < 3; v++) {
      dn = f[3 * v + d] < dn ? f[3 * v + d] : dn;
      up = f[3 * v + d] > up ? f[3 * v + d] : up;
    }
    const int64_t l = (int64_t)rintp((dn - a.mn[d]) * a.scale), h = (int64_t)rintp((up - a.mn[d]) * a.scale);
    lo[d] = l < 0 ? 0 : (l >= a.n ? a.n - 1 : l);
    hi[d] = h < 0 ? 0 : (h >= a.n ? a.n - 1 : h);
  }
}

__global__ void k_aux_bin(PatchDev P, AuxGrid a, int32_t* cnt, const int64_t* __restrict__ off, int32_t* cursor,
                          int32_t* list) {
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < P.n; p += (int64_t)gridDim.x * blockDim.x) {
    int64_t lo[3], hi[3];
    if (P.i32[NS_PATCH_I32 * p] == NS_MESH_TRI) aux_box_tri(P.f64 + (int64_t)NS_PATCH_F64 * p, a, lo, hi);
    else aux_box(P.f64 + (int64_t)NS_PATCH_F64 * p, a, lo, hi);
    for (int64_t iz = lo[2]; iz <= hi[2]; iz++)
      for (int64_t iy = lo[1]; iy <= hi[1]; iy++)
        for (int64_t ix = lo[0]; ix <= hi[0]; ix++) {
          const int64_t c = (iz * a.n + iy) * a.n + ix;
          if (cnt) atomicAdd(cnt + c, 1);
          else list[off[c] + atomicAdd(cursor + c, 1)] = (int32_t)p;
        }
  }
}

// MeshSurface::point2triangle (src/MeshSurface.cpp:1864-2008) with the triangle's plane as
// preProcessTriangles stores it (plane3points, normalised, offset from the triple product,
// :674-684), point2plane (:2034-2044) and inTriangle (:2010-2032, whose barycentric test
// multiplies by the denominator).  Outside the triangle the nearest of the three clamped edge
// projections wins, with the reference's edge "normal" S + T t normalised.  Returns whether the
// plane projection fell inside the triangle.
__device__ __forceinline__ double dot3(const double* x, const double* y) { return x[0] * y[0] + x[1] * y[1] + x[2] * y[2]; }

__device__ bool project_tri(const double* P, const double* f, double* proj, double* dist, double* normal) {
  const double *A = f, *B = f + 3, *C = f + 6;
  double w[4];
  w[0] = A[1] * (B[2] - C[2]) + B[1] * (C[2] - A[2]) + C[1] * (A[2] - B[2]);
  w[1] = A[2] * (B[0] - C[0]) + B[2] * (C[0] - A[0]) + C[2] * (A[0] - B[0]);
  w[2] = A[0] * (B[1] - C[1]) + B[0] * (C[1] - A[1]) + C[0] * (A[1] - B[1]);
  const double norm = sqrt(dot3(w, w));
  for (int d = 0; d < 3; d++) w[d] /= norm;
  w[3] = -(A[0] * (B[1] * C[2] - C[1] * B[2]) + B[0] * (C[1] * A[2] - A[1] * C[2]) + C[0] * (A[1] * B[2] - B[1] * A[2]));
  w[3] /= norm;
  const double den = dot3(w, w);
  const double val = dot3(w, P) + w[3];
  for (int d = 0; d < 3; d++) proj[d] = P[d] - w[d] * (val / den);
  *dist = fabs(val / sqrt(den));
  double v0[3], v1[3], v2[3];
  for (int d = 0; d < 3; d++) {
    v0[d] = C[d] - A[d];
    v1[d] = B[d] - A[d];
    v2[d] = proj[d] - A[d];
  }
  const double d00 = dot3(v0, v0), d01 = dot3(v0, v1), d02 = dot3(v0, v2), d11 = dot3(v1, v1), d12 = dot3(v1, v2);
  const double den2 = d00 * d11 - d01 * d01;
  const double u = (d11 * d02 - d01 * d12) * den2, v = (d00 * d12 - d01 * d02) * den2;
  if (u > 0 && v > 0 && u + v < 1) {
    for (int d = 0; d < 3; d++) normal[d] = w[d];
    return true;
  }
  double bd = 0, bt = 0, bres[3] = {0, 0, 0};
  int be = -1;
  for (int e = 0; e < 3; e++) {
    const double* S = e == 2 ? B : A;
    const double* T = e == 0 ? B : C;
    double t2[3], t1[3], res[3], de;
    for (int d = 0; d < 3; d++) {
      t2[d] = T[d] - S[d];
      t1[d] = proj[d] - S[d];
    }
    const double l2 = dot3(t2, t2);
    double t = dot3(t1, t2);
    if (t < 0.0) {
      for (int d = 0; d < 3; d++) t1[d] = P[d] - S[d];
      de = sqrt(dot3(t1, t1));
      for (int d = 0; d < 3; d++) res[d] = S[d];
      t = 0.0;
    } else if (t > l2) {
      for (int d = 0; d < 3; d++) t1[d] = P[d] - T[d];
      de = sqrt(dot3(t1, t1));
      for (int d = 0; d < 3; d++) res[d] = T[d];
      t = 1.0;
    } else {
      t /= l2;
      for (int d = 0; d < 3; d++) res[d] = S[d] + t2[d] * t;
      for (int d = 0; d < 3; d++) t1[d] = res[d] - P[d];
      de = sqrt(dot3(t1, t1));
    }
    // the reference's choice (d0 <= d1 && d0 <= d2, then d1 <= d0 && d1 <= d2, else d2) is the
    // first smallest: keep an edge only when strictly nearer than the ones before it
    if (be < 0 || de < bd) {
      be = e;
      bd = de;
      bt = t;
      for (int d = 0; d < 3; d++) bres[d] = res[d];
    }
  }
  const double* S = be == 2 ? B : A;
  const double* T = be == 0 ? B : C;
  for (int d = 0; d < 3; d++) proj[d] = bres[d];
  *dist = bd;
  for (int d = 0; d < 3; d++) normal[d] = S[d] + T[d] * bt;
  const double nn = sqrt(dot3(normal, normal));
  for (int d = 0; d < 3; d++) normal[d] /= nn;
  return false;
}

// projectToSphere (src/tools.cpp:1112-1120), operation for operation.
__device__ __forceinline__ double project_sphere(const double* y, const double* c, double r, double* proj) {
  double dist = sqrt((y[0] - c[0]) * (y[0] - c[0]) + (y[1] - c[1]) * (y[1] - c[1]) + (y[2] - c[2]) * (y[2] - c[2]));
  dist = r / dist;
  for (int d = 0; d < 3; d++) proj[d] = y[d] - c[d];
  for (int d = 0; d < 3; d++) proj[d] = c[d] + dist * proj[d];
  return sqrt((proj[0] - y[0]) * (proj[0] - y[0]) + (proj[1] - y[1]) * (proj[1] - y[1]) +
              (proj[2] - y[2]) * (proj[2] - y[2]));
}

// projectToCircle (src/ConnollySurface.cpp:5693-5703) with point2plane (src/tools.cpp:277-287).
__device__ __forceinline__ void project_circle(const double* p, double radius, const double* c, const double* w,
                                               double* proj) {
  const double den = w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
  const double val = (w[0] * p[0] + w[1] * p[1] + w[2] * p[2]) + w[3];
  const double cc = val / den;
  for (int d = 0; d < 3; d++) proj[d] = p[d] - w[d] * cc;
  for (int d = 0; d < 3; d++) proj[d] = proj[d] - c[d];
  radius /= sqrt(proj[0] * proj[0] + proj[1] * proj[1] + proj[2] * proj[2]);
  for (int d = 0; d < 3; d++) proj[d] = c[d] + radius * proj[d];
}

// projectToTorus (src/ConnollySurface.cpp:5705-5733).  The torus frame is stored as its inverse;
// the rotation back uses its transpose (the frame is orthonormal, so this differs from the
// reference's separately stored matrix in the last bits only).
__device__ __forceinline__ double project_torus(const double* y, const double* f, double probe, double* proj) {
  const double* inv = f + 9;
  const double* tc = f + 4;
  double temp[3], pp[3];
  for (int d = 0; d < 3; d++) temp[d] = y[d] - tc[d];
  for (int i = 0; i < 3; i++) pp[i] = inv[3 * i] * temp[0] + inv[3 * i + 1] * temp[1] + inv[3 * i + 2] * temp[2];
  const double zero3[3] = {0., 0., 0.};
  const double torus_plane[4] = {0., 0., 1., 0.};
  double major[3];
  project_circle(pp, f[7], zero3, torus_plane, major);
  // plane3points(major, (0,0,1), (0,0,-1)) normalised (src/tools.cpp:258-274)
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

__global__ void k_bgp_project(PatchDev P, AuxGrid a, const int64_t* __restrict__ off, const int32_t* __restrict__ list,
                              GridDev g, const int32_t* __restrict__ ibgp, const int32_t* __restrict__ type, int32_t n,
                              double* pos, double* nor, int32_t* flag) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t q = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); q < n; q += warps) {
    double y[3];
    for (int d = 0; d < 3; d++) y[d] = g.mn[d] + (double)ibgp[3 * q + d] * g.side;
    if (type[q] != NS_EXTERNAL_BGP) {
      if (lane == 0) flag[q] = 3;
      continue;
    }
    int64_t ic[3];
    bool in = true;
    for (int d = 0; d < 3; d++) {
      ic[d] = (int64_t)rintp((y[d] - a.mn[d]) * a.scale);
      in = in && ic[d] >= 0 && ic[d] < a.n;
    }
    int64_t b = 0, e = 0;
    if (in) {
      const int64_t c = (ic[2] * a.n + ic[1]) * a.n + ic[0];
      b = off[c];
      e = off[c + 1];
    }
    double best = INFINITY;
    int32_t best_p = INT32_MAX;
    double bp[3] = {y[0], y[1], y[2]};
    double bn[3] = {0.0, 0.0, 0.0};
    int best_in = 0;
    for (int64_t u = b + lane; u < e; u += 32) {
      const int32_t p = list[u];
      const double* f = P.f64 + (int64_t)NS_PATCH_F64 * p;
      const int32_t* ir = P.i32 + NS_PATCH_I32 * (int64_t)p;
      const int kind = ir[0];
      double proj[3], dist;
      if (kind == NS_MESH_TRI) {
        double nrm[3];
        const bool in_tri = project_tri(y, f, proj, &dist, nrm);
        if (dist < best || (dist == best && p < best_p)) {
          best = dist;
          best_p = p;
          best_in = in_tri ? 1 : 0;
          for (int d = 0; d < 3; d++) {
            bp[d] = proj[d];
            bn[d] = nrm[d];
          }
        }
        continue;
      }
      if (kind == NS_POINT) dist = project_sphere(y, f, f[3], proj);
      else if (kind == NS_FACE_REG || kind == NS_FACE_SING) dist = project_sphere(y, f, P.probe, proj);
      else dist = project_torus(y, f, P.probe, proj);
      if (!feasible_f64(f, kind, ir[1], ir[2], P.pool, P.flag, proj)) continue;
      if (dist < best || (dist == best && p < best_p)) {
        best = dist;
        best_p = p;
        bp[0] = proj[0];
        bp[1] = proj[1];
        bp[2] = proj[2];
      }
    }
    // warp arg-min over (distance, patch)
    for (int o = 16; o > 0; o >>= 1) {
      const double od = __shfl_xor_sync(0xffffffffu, best, o);
      const int32_t op = __shfl_xor_sync(0xffffffffu, best_p, o);
      const double o0 = __shfl_xor_sync(0xffffffffu, bp[0], o);
      const double o1 = __shfl_xor_sync(0xffffffffu, bp[1], o);
      const double o2 = __shfl_xor_sync(0xffffffffu, bp[2], o);
      const double n0 = __shfl_xor_sync(0xffffffffu, bn[0], o);
      const double n1 = __shfl_xor_sync(0xffffffffu, bn[1], o);
      const double n2 = __shfl_xor_sync(0xffffffffu, bn[2], o);
      const int oi = __shfl_xor_sync(0xffffffffu, best_in, o);
      if (od < best || (od == best && op < best_p)) {
        best = od;
        best_p = op;
        bp[0] = o0;
        bp[1] = o1;
        bp[2] = o2;
        bn[0] = n0;
        bn[1] = n1;
        bn[2] = n2;
        best_in = oi;
      }
    }
    if (lane == 0) {
      const bool ok = best_p != INT32_MAX;
      const bool mesh = ok && P.i32[NS_PATCH_I32 * (int64_t)best_p] == NS_MESH_TRI;
      for (int d = 0; d < 3; d++) {
        pos[3 * q + d] = ok ? bp[d] : y[d];
        nor[3 * q + d] = mesh ? bn[d] : 0.0;
      }
      flag[q] = e == b ? 2 : (mesh ? (best_in ? 0 : 1) : (ok ? 0 : 1));
    }
  }
}

}  // namespace

cudaError_t eps_fill_cavities(const RunArgs& A, const uint8_t* fill_of, int32_t* eps, int32_t inside, cudaStream_t s) {
  if (A.nruns <= 0 || !eps) return cudaSuccess;
  k_eps_fill_cavities<<<grid_for(A.nruns), 256, 0, s>>>(A, fill_of, eps, inside);
  return cudaGetLastError();
}

cudaError_t ideb_write(const RunArgs& A, const uint8_t* fill_of, uint8_t* ideb, cudaStream_t s) {
  if (A.nrows <= 0) return cudaSuccess;
  k_ideb_write<<<grid_for(A.nrows * 32), 256, 0, s>>>(A, fill_of, ideb);
  return cudaGetLastError();
}

cudaError_t bgp_select(const int32_t* eps, int64_t nx, int64_t ny, int64_t nz, int32_t* nodes, int32_t* count,
                       void* temp, size_t* temp_bytes, cudaStream_t s) {
  cub::CountingInputIterator<int32_t> it(0);
  if (!nodes) {
    cub::DiscardOutputIterator<> none;
    return cub::DeviceSelect::If(temp, *temp_bytes, it, none, count, (int)(nx * ny * nz), BgpPred{eps, nx, ny, nz}, s);
  }
  return cub::DeviceSelect::If(temp, *temp_bytes, it, nodes, count, (int)(nx * ny * nz), BgpPred{eps, nx, ny, nz}, s);
}

cudaError_t sum_i32(const int32_t* in, int32_t n, int64_t* out, void* temp, size_t* temp_bytes, cudaStream_t s) {
  return cub::DeviceReduce::Sum(temp, *temp_bytes, in, out, n, s);
}

cudaError_t bgp_expand(const int32_t* eps, int64_t nx, int64_t ny, int64_t nz, const int32_t* nodes, int32_t n,
                       int32_t* ibgp, int32_t* type, cudaStream_t s) {
  (void)nz;
  if (n <= 0) return cudaSuccess;
  k_bgp_expand<<<grid_for(n), 256, 0, s>>>(eps, nx, ny, nodes, n, ibgp, type);
  return cudaGetLastError();
}

cudaError_t aux_count(const PatchDev& P, const AuxGrid& a, int32_t* cnt, cudaStream_t s) {
  if (P.n <= 0) return cudaSuccess;
  k_aux_bin<<<grid_for(P.n), 256, 0, s>>>(P, a, cnt, nullptr, nullptr, nullptr);
  return cudaGetLastError();
}

cudaError_t aux_fill(const PatchDev& P, const AuxGrid& a, const int64_t* off, int32_t* cursor, int32_t* list,
                     cudaStream_t s) {
  if (P.n <= 0) return cudaSuccess;
  k_aux_bin<<<grid_for(P.n), 256, 0, s>>>(P, a, nullptr, off, cursor, list);
  return cudaGetLastError();
}

cudaError_t bgp_project(const PatchDev& P, const AuxGrid& a, const int64_t* off, const int32_t* list,
                        const GridDev& g, const int32_t* ibgp, const int32_t* type, int32_t n, double* pos,
                        double* nor, int32_t* flag, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_bgp_project<<<grid_for((int64_t)n * 32), 256, 0, s>>>(P, a, off, list, g, ibgp, type, n, pos, nor, flag);
  return cudaGetLastError();
}

}  // namespace nsg
