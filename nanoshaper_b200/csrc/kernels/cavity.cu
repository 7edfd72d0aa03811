// Status map materialisation, cavity detection and conditional cavity filling.
//
// The reference labels the 6-connected regions of STATUS_POINT_TEMPORARY_OUT nodes one at a time
// with a scanline flood fill seeded at the first remaining node of a scan whose z direction
// alternates between ascending and descending (getCavitiesWithBilevelStatusMap
// src/Surface.cpp:1994-2126, floodFillWithBilevelStatusMap2 :4284-4554); the first region found
// becomes STATUS_POINT_OUT (3), the following ones cavities 4, 5, ...  Cavities whose node count
// times side^3 does not exceed the threshold get the insideness bits of the 8 corners of each of
// their nodes cleared (fillCavities :2355-2484).
//
// Here the status map is kept as runs: the status rays give, per x-row (j, k), the runs of
// inside nodes; their complement are the runs of free nodes.  Regions are found with a lock-free
// union-find over free runs (two runs are joined when they overlap in x in rows (j+1, k) or
// (j, k+1)), with each region's root being its smallest run index = its first node in ascending
// scan order.  Its first node in descending-z scan order is reduced per region.  The host
// replays the alternating seed selection over these two keys (nsg_cavity_order), which
// reproduces the reference labels; the dense status map is then written once, row by row.
#include <cub/cub.cuh>

#include "cavity.h"
#include "pipeline.h"

namespace nsg {

namespace {

__device__ __forceinline__ int32_t find_root(int32_t* L, int32_t v) {
  int32_t p = L[v];
  while (p != v) {
    int32_t gp = L[p];
    if (gp != p) L[v] = gp;  // path halving; only ever points a node to an ancestor
    v = p;
    p = gp;
  }
  return v;
}

__device__ __forceinline__ void unite(int32_t* L, int32_t a, int32_t b) {
  while (true) {
    a = find_root(L, a);
    b = find_root(L, b);
    if (a == b) return;
    if (a < b) { int32_t t = a; a = b; b = t; }
    int32_t old = atomicCAS(L + a, a, b);
    if (old == a) return;
    a = old;
  }
}

// Free runs of a status row: the gaps between its (sorted) inside runs.
__global__ void k_free_runs(RunArgs A, int emit) {
  const int64_t NX = A.nx;
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < A.nrows; r += (int64_t)gridDim.x * blockDim.x) {
    int cnt = A.srun_cnt[r];
    const int2* in = A.sruns + (cnt ? A.srun_off[r] : 0);
    int64_t prev = -1;
    int nf = 0;
    int64_t o = emit ? A.fr_off[r] : 0;
    for (int q = 0; q <= cnt; q++) {
      int64_t a = (q < cnt) ? in[q].x : NX;
      if (a > prev + 1) {
        if (emit) {
          A.fruns[o + nf] = make_int2((int)(prev + 1), (int)(a - 1));
          A.frow[o + nf] = (int32_t)r;
        }
        nf++;
      }
      if (q < cnt && in[q].y > prev) prev = in[q].y;
    }
    if (!emit) A.fr_cnt[r] = nf;
  }
}

__global__ void k_run_init(int32_t* L, int64_t n) {
  for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < n; u += (int64_t)gridDim.x * blockDim.x)
    L[u] = (int32_t)u;
}

__device__ __forceinline__ void hook_row(const RunArgs& A, int32_t u, int2 ru, int64_t s) {
  int64_t lo = A.fr_off[s], hi = A.fr_off[s + 1];
  // first run of row s ending at or after ru.x
  while (lo < hi) {
    int64_t mid = (lo + hi) >> 1;
    if (A.fruns[mid].y < ru.x) lo = mid + 1;
    else hi = mid;
  }
  for (int64_t v = lo; v < A.fr_off[s + 1] && A.fruns[v].x <= ru.y; v++) unite(A.L, u, (int32_t)v);
}

__global__ void k_run_hook(RunArgs A) {
  for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < A.nruns; u += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = A.frow[u];
    int64_t j = r % A.ny, k = r / A.ny;
    int2 ru = A.fruns[u];
    if (j + 1 < A.ny) hook_row(A, (int32_t)u, ru, r + 1);
    if (k + 1 < A.nz) hook_row(A, (int32_t)u, ru, r + A.ny);
  }
}

// Final root of every run.  The walk does not shorten paths: a halving write issued by one
// thread could otherwise overwrite a label another thread has already set to its root.
__global__ void k_run_compress(int32_t* L, int64_t n, uint8_t* is_root) {
  for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < n; u += (int64_t)gridDim.x * blockDim.x) {
    int32_t r = L[u];
    for (int32_t q = L[r]; q != r; q = L[r]) r = q;
    L[u] = r;
    is_root[u] = (r == u) ? 1 : 0;
  }
}

// Region index of every run (binary search in the sorted roots), region node counts and first
// node in descending-z scan order.  Lanes of a warp in the same region are combined before the
// atomics.
__global__ void k_run_stats(RunArgs A, const int32_t* __restrict__ roots, int32_t nroots, unsigned long long* count,
                            unsigned int* desc_key) {
  const int64_t plane = A.nx * A.ny;
  for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < A.nruns; u += (int64_t)gridDim.x * blockDim.x) {
    unsigned act = __activemask();
    int32_t l = A.L[u];
    int32_t lo = 0, hi = nroots - 1;
    if (roots[0] != l) {
      while (lo < hi) {
        int32_t mid = (lo + hi) >> 1;
        if (roots[mid] < l) lo = mid + 1;
        else hi = mid;
      }
    }
    A.L[u] = lo;
    int64_t r = A.frow[u];
    int64_t j = r % A.ny, k = r / A.ny;
    int2 ru = A.fruns[u];
    unsigned key = (unsigned)((A.nz - 1 - k) * plane + j * A.nx + ru.x);
    unsigned len = (unsigned)(ru.y - ru.x + 1);
    unsigned grp = __match_any_sync(act, lo);
    unsigned kmin = __reduce_min_sync(grp, key);
    unsigned sum = __reduce_add_sync(grp, len);
    if ((int)(threadIdx.x & 31) == __ffs(grp) - 1) {
      atomicAdd(count + lo, (unsigned long long)sum);
      atomicMin(desc_key + lo, kmin);
    }
  }
}

// Clears the 8 cube-corner insideness bits of every node of the filled cavities: for a run
// x0..x1 of row (j, k), bits x0..x1+1 of the rows (j, k), (j+1, k), (j, k+1), (j+1, k+1).
__global__ void k_run_fill(RunArgs A, const uint8_t* __restrict__ fill_of, uint32_t* bits, int64_t nwords) {
  for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < A.nruns; u += (int64_t)gridDim.x * blockDim.x) {
    int32_t c = A.L[u];
    if (!fill_of[c]) continue;
    int64_t r = A.frow[u];
    int2 ru = A.fruns[u];
    for (int dk = 0; dk < 2; dk++)
      for (int dj = 0; dj < 2; dj++) {
        int64_t base = (r + dj + dk * A.ny) * A.nx;
        int64_t f0 = base + ru.x, f1 = base + ru.y + 1;
        if (f0 < 0) f0 = 0;
        if (f1 > nwords * 32 - 1) f1 = nwords * 32 - 1;
        for (int64_t w = f0 >> 5; w <= (f1 >> 5); w++) {
          int64_t wl = w << 5;
          int s = (int)(f0 > wl ? f0 - wl : 0);
          int e = (int)(f1 < wl + 31 ? f1 - wl : 31);
          uint32_t mask = (e - s == 31) ? 0xffffffffu : (((1u << (e - s + 1)) - 1u) << s);
          atomicAnd(bits + w, ~mask);
        }
      }
  }
}

// Dense status map, one warp per x-row: the row is the sequence of its free runs (region label,
// or TEMPORARY_OUT before cavity detection) and the inside segments between them
// (STATUS_POINT_INSIDE); every segment is written by the whole warp with coalesced stores.
__global__ void k_status_write(RunArgs A, const int32_t* __restrict__ label_of, int32_t* status) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t r = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); r < A.nrows; r += warps) {
    const int64_t b = A.fr_off[r], e = A.fr_off[r + 1];
    int32_t* row = status + r * A.nx;
    int64_t next = 0;  // first node not yet written
    for (int64_t u = b; u <= e; u++) {
      int64_t x0 = A.nx, x1 = A.nx - 1;
      int32_t lab = NS_STATUS_TEMPORARY_OUT;
      if (u < e) {
        int2 ru = A.fruns[u];
        x0 = ru.x;
        x1 = ru.y;
        if (label_of) lab = label_of[A.L[u]];
      }
      for (int64_t i = next + lane; i < x0; i += 32) row[i] = NS_STATUS_INSIDE;
      for (int64_t i = x0 + lane; i <= x1; i += 32) row[i] = lab;
      next = x1 + 1;
    }
  }
}

// The 27 cells around a cell, in the reference's order (shift_map, src/tools.h:35-64).
__constant__ int8_t c_shift27[27][3] = {
    {0, 0, 0},   {0, 0, -1},  {0, 0, 1},   {0, 1, 0},   {0, 1, -1},  {0, 1, 1},   {0, -1, 0},  {0, -1, -1}, {0, -1, 1},
    {1, 0, 0},   {1, 0, -1},  {1, 0, 1},   {1, 1, 0},   {1, 1, -1},  {1, 1, 1},   {1, -1, 0},  {1, -1, -1}, {1, -1, 1},
    {-1, 0, 0},  {-1, 0, -1}, {-1, 0, 1},  {-1, 1, 0},  {-1, 1, -1}, {-1, 1, 1},  {-1, -1, 0}, {-1, -1, -1}, {-1, -1, 1}};

__device__ __forceinline__ int32_t status_at(const CavAtomArgs& A, int64_t i, int64_t j, int64_t k) {
  if (i < 0 || j < 0 || k < 0 || i >= A.nx || j >= A.ny || k >= A.nz) return NS_STATUS_TEMPORARY_OUT;
  return A.status[(k * A.ny + j) * A.nx + i];
}

// One thread per node (the status map is read once, coalesced); cavity boundary nodes search the
// atom grid and append their pair.
__global__ void k_cav_atoms(CavAtomArgs A) {
  const int64_t n = A.nx * A.ny * A.nz;
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
    const int32_t lab = A.label ? A.label[v] : A.status[v];
    if (lab < NS_STATUS_FIRST_CAV) continue;
    const int32_t s = A.status[v];
    const int64_t i = v % A.nx, j = (v / A.nx) % A.ny, k = v / (A.nx * A.ny);
    if (status_at(A, i + 1, j, k) == s && status_at(A, i - 1, j, k) == s && status_at(A, i, j + 1, k) == s &&
        status_at(A, i, j - 1, k) == s && status_at(A, i, j, k + 1) == s && status_at(A, i, j, k - 1) == s)
      continue;
    const double p[3] = {A.mn[0] + (double)i * A.side, A.mn[1] + (double)j * A.side, A.mn[2] + (double)k * A.side};
    int64_t c[3];
    for (int d = 0; d < 3; d++) c[d] = (int64_t)floor((p[d] - A.gmn[d]) * A.gscale + 0.5);
    double best = INFINITY;
    int32_t first = -1;
    for (int q = 0; q < 27; q++) {
      const int64_t cx = c[0] + c_shift27[q][0], cy = c[1] + c_shift27[q][1], cz = c[2] + c_shift27[q][2];
      if (cx >= A.gn || cy >= A.gn || cz >= A.gn || cx < 0 || cy < 0 || cz < 0) continue;
      const int64_t cell = (cz * A.gn + cy) * A.gn + cx;
      for (int32_t t = A.cell_off[cell]; t < A.cell_off[cell + 1]; t++) {
        const int32_t a = A.cell_atoms[t];
        const double* at = A.atoms + 4 * (int64_t)a;
        double d = (at[0] - p[0]) * (at[0] - p[0]) + (at[1] - p[1]) * (at[1] - p[1]) + (at[2] - p[2]) * (at[2] - p[2]);
        d -= at[3] * at[3];
        if (d < best) {
          best = d;
          first = a;
        }
      }
    }
    const unsigned long long slot = atomicAdd(A.count, 1ull);
    if ((int64_t)slot < A.cap)
      A.pairs[slot] = ((unsigned long long)(uint32_t)(lab - NS_STATUS_FIRST_CAV) << 32) | (uint32_t)(first + 1);
    else
      atomicExch(A.err, 1);
  }
}

// Water-shape filter.  The reference walks the kept cavities in order; within one cavity the
// support test reads only whether each node of the probe box is in the cavity's in-set
// (SHAPE_UNDER_CHECK, SHAPE_OK or -cavityId), a set that the walk does not change, so the supports
// do not depend on the order of the cavity's points.  Across cavities, the removed nodes of an
// earlier kept cavity stay SHAPE_UNDER_CHECK (or become SHAPE_OK inside a later support sphere)
// when the status map is not modified, and count as in-set nodes of every later cavity.  The
// passes below solve that lower-triangular dependency by fixed-point iteration: pass t takes the
// removed set of pass t-1 for the earlier cavities, so cavity t is exact after pass t and a pass
// that changes nothing is the reference's result.

// The reference's probe box around node q along one axis (rintp of the shifted coordinates,
// clamped to the grid).
__device__ __forceinline__ void shape_axis(double mn, double side, double scale, double r, int64_t n, int64_t q,
                                           int64_t* lo, int64_t* hi) {
  const double x = mn + (double)q * side;
  int64_t s = (int64_t)floor(((x - r) - mn) * scale + 0.5);
  int64_t e = (int64_t)floor(((x + r) - mn) * scale + 0.5);
  *lo = s < 0 ? 0 : (s >= n ? n - 1 : s);
  *hi = e < 0 ? 0 : (e >= n ? n - 1 : e);
}

// |x_u - x_v|^2 with the grid coordinates min + i*side, as the reference evaluates it.
__device__ __forceinline__ double shape_d2(const ShapeArgs& A, int64_t ui, int64_t uj, int64_t uk, int64_t vi,
                                           int64_t vj, int64_t vk) {
  const double a = (A.mn[0] + (double)ui * A.side) - (A.mn[0] + (double)vi * A.side);
  const double b = (A.mn[1] + (double)uj * A.side) - (A.mn[1] + (double)vj * A.side);
  const double c = (A.mn[2] + (double)uk * A.side) - (A.mn[2] + (double)vk * A.side);
  return a * a + b * b + c * c;
}

__device__ __forceinline__ bool shape_kept(const ShapeArgs& A, int32_t lab) {
  return lab >= NS_STATUS_FIRST_CAV && !A.filled[lab - NS_STATUS_FIRST_CAV];
}

// A node of a kept cavity is a support when no node of its probe sphere lies outside the in-set.
__global__ void k_shape_support(ShapeArgs A) {
  const int64_t n = A.nx * A.ny * A.nz;
  const double r2 = A.r * A.r;
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
    const int32_t lab = A.label[v];
    if (!shape_kept(A, lab)) continue;
    const int64_t i = v % A.nx, j = (v / A.nx) % A.ny, k = v / (A.nx * A.ny);
    int64_t lo[3], hi[3];
    shape_axis(A.mn[0], A.side, A.scale, A.r, A.nx, i, &lo[0], &hi[0]);
    shape_axis(A.mn[1], A.side, A.scale, A.r, A.ny, j, &lo[1], &hi[1]);
    shape_axis(A.mn[2], A.side, A.scale, A.r, A.nz, k, &lo[2], &hi[2]);
    bool ok = true;
    for (int64_t z = lo[2]; z <= hi[2] && ok; z++)
      for (int64_t y = lo[1]; y <= hi[1] && ok; y++)
        for (int64_t x = lo[0]; x <= hi[0]; x++) {
          if (shape_d2(A, x, y, z, i, j, k) > r2) continue;
          const int64_t u = (z * A.ny + y) * A.nx + x;
          const int32_t lu = A.label[u];
          if (lu == lab) continue;
          if (A.removed_prev && A.removed_prev[u] && lu >= NS_STATUS_FIRST_CAV && lu < lab) continue;
          ok = false;
          break;
        }
    A.support[v] = ok ? 1 : 0;
  }
}

// A node of a kept cavity is removed when no support of its own cavity has it in its probe
// sphere; `later` records a support sphere of a later cavity (which only reaches removed nodes).
// Gathered from the node's side: the supports whose probe box can hold it lie within its own box
// widened by one node, and each is tested with the support's own box and distance.
__global__ void k_shape_cover(ShapeArgs A) {
  const int64_t n = A.nx * A.ny * A.nz;
  const double r2 = A.r * A.r;
  for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < n; u += (int64_t)gridDim.x * blockDim.x) {
    const int32_t lab = A.label[u];
    if (!shape_kept(A, lab)) continue;
    const int64_t i = u % A.nx, j = (u / A.nx) % A.ny, k = u / (A.nx * A.ny);
    int64_t lo[3], hi[3];
    shape_axis(A.mn[0], A.side, A.scale, A.r, A.nx, i, &lo[0], &hi[0]);
    shape_axis(A.mn[1], A.side, A.scale, A.r, A.ny, j, &lo[1], &hi[1]);
    shape_axis(A.mn[2], A.side, A.scale, A.r, A.nz, k, &lo[2], &hi[2]);
    const int64_t nn[3] = {A.nx, A.ny, A.nz};
    for (int d = 0; d < 3; d++) {
      lo[d] = lo[d] > 0 ? lo[d] - 1 : 0;
      hi[d] = hi[d] < nn[d] - 1 ? hi[d] + 1 : nn[d] - 1;
    }
    bool own = false, later = false;
    for (int64_t z = lo[2]; z <= hi[2] && !own; z++)
      for (int64_t y = lo[1]; y <= hi[1] && !own; y++)
        for (int64_t x = lo[0]; x <= hi[0]; x++) {
          const int64_t v = (z * A.ny + y) * A.nx + x;
          if (!A.support[v]) continue;
          const int32_t lv = A.label[v];
          if (lv < lab || (lv > lab && later)) continue;
          int64_t a0, a1, b0, b1, c0, c1;
          shape_axis(A.mn[0], A.side, A.scale, A.r, A.nx, x, &a0, &a1);
          shape_axis(A.mn[1], A.side, A.scale, A.r, A.ny, y, &b0, &b1);
          shape_axis(A.mn[2], A.side, A.scale, A.r, A.nz, z, &c0, &c1);
          if (i < a0 || i > a1 || j < b0 || j > b1 || k < c0 || k > c1) continue;
          if (shape_d2(A, i, j, k, x, y, z) > r2) continue;
          if (lv == lab) {
            own = true;
            break;
          }
          later = true;
        }
    const uint8_t rm = own ? 0 : 1;
    A.removed[u] = rm;
    A.later[u] = later ? 1 : 0;
    if (A.removed_prev && A.removed_prev[u] != rm) atomicExch(A.changed, 1);
  }
}

__global__ void k_shape_apply(ShapeArgs A) {
  const int64_t n = A.nx * A.ny * A.nz;
  const int64_t plane = A.nx * A.ny;
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
    const int32_t lab = A.label[v];
    if (!shape_kept(A, lab)) continue;
    if (A.support[v]) {
      A.status[v] = -lab;
      continue;
    }
    if (!A.removed[v]) {
      A.status[v] = lab;
      continue;
    }
    A.status[v] = A.mod_status ? NS_STATUS_INSIDE : (A.later[v] ? NS_STATUS_SHAPE_OK : NS_STATUS_SHAPE_UNDER_CHECK);
    atomicAdd(A.n_removed + (lab - NS_STATUS_FIRST_CAV), 1ull);
    const int64_t i = v % A.nx, j = (v / A.nx) % A.ny, k = v / plane;
    if (A.bits) {
      // the 8 corners of the node's cube (a cavity never touches the grid's last planes)
      for (int dk = 0; dk < 2; dk++)
        for (int dj = 0; dj < 2; dj++)
          for (int di = 0; di < 2; di++) {
            const int64_t f = v + dk * plane + dj * A.nx + di;
            if ((f >> 5) < A.nwords) atomicAnd(A.bits + (f >> 5), ~(1u << (f & 31)));
          }
    }
    if (A.eps) {
      A.eps[3 * v] = NS_EPS_INSIDE;
      A.eps[3 * v + 1] = NS_EPS_INSIDE;
      A.eps[3 * v + 2] = NS_EPS_INSIDE;
      if (i > 0) A.eps[3 * (v - 1)] = NS_EPS_INSIDE;
      if (j > 0) A.eps[3 * (v - A.nx) + 1] = NS_EPS_INSIDE;
      if (k > 0) A.eps[3 * (v - plane) + 2] = NS_EPS_INSIDE;
    }
    if (A.ideb) A.ideb[v] = 0;
  }
}

// One warp per 32 consecutive nodes, so that each insideness word is formed by one ballot.
__global__ void k_pocket_diff(int32_t* st1, const int32_t* st2, int64_t n, uint32_t* bits,
                              unsigned long long* count) {
  const int lane = threadIdx.x & 31;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  unsigned long long mine = 0;
  for (int64_t f0 = blockIdx.x * (int64_t)blockDim.x + (threadIdx.x & ~31); f0 < n; f0 += stride) {
    const int64_t f = f0 + lane;
    bool pk = false;
    if (f < n) {
      const int32_t s1 = st1[f], s2 = st2[f];
      pk = (s1 != NS_STATUS_TEMPORARY_OUT && s1 != NS_STATUS_OUT) &&
           (s2 == NS_STATUS_TEMPORARY_OUT || s2 == NS_STATUS_OUT);
      st1[f] = pk ? NS_STATUS_FIRST_CAV : NS_STATUS_INSIDE;
    }
    const uint32_t m = __ballot_sync(0xffffffffu, pk);
    if (lane == 0) {
      mine += __popc(m);
      if (bits) {
        const int64_t valid = n - f0 < 32 ? n - f0 : 32;
        const uint32_t vm = valid == 32 ? 0xffffffffu : ((1u << valid) - 1u);
        uint32_t* w = bits + (f0 >> 5);
        *w = (*w & ~vm) | m;
      }
    }
  }
  if (lane == 0 && mine) atomicAdd(count, mine);
}

__global__ void k_pocket_cav2out(int32_t* status, const int32_t* __restrict__ label, int64_t n) {
  for (int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; f < n; f += (int64_t)gridDim.x * blockDim.x) {
    if (label[f] != NS_STATUS_FIRST_CAV) continue;
    const int32_t v = status[f];
    if (v >= NS_STATUS_FIRST_CAV || v <= -NS_STATUS_FIRST_CAV) status[f] = NS_STATUS_TEMPORARY_OUT;
  }
}

// One thread per x-row of the dense map.
__global__ void k_dense_free_runs(RunArgs A, const int32_t* __restrict__ status, int emit) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < A.nrows; r += (int64_t)gridDim.x * blockDim.x) {
    const int32_t* row = status + r * A.nx;
    int nf = 0;
    int64_t o = emit ? A.fr_off[r] : 0;
    int64_t start = -1;
    for (int64_t i = 0; i <= A.nx; i++) {
      const bool fr = i < A.nx && row[i] == NS_STATUS_TEMPORARY_OUT;
      if (fr && start < 0) start = i;
      if (!fr && start >= 0) {
        if (emit) {
          A.fruns[o + nf] = make_int2((int)start, (int)(i - 1));
          A.frow[o + nf] = (int32_t)r;
        }
        nf++;
        start = -1;
      }
    }
    if (!emit) A.fr_cnt[r] = nf;
  }
}

int grid_for(int64_t n, int threads = 256) {
  int64_t b = (n + threads - 1) / threads;
  const int64_t cap = (int64_t)sm_count() * 32;
  return (int)(b < cap ? (b < 1 ? 1 : b) : cap);
}

}  // namespace

cudaError_t launch_free_runs(const RunArgs& A, int emit, cudaStream_t s) {
  if (A.nrows <= 0) return cudaSuccess;
  k_free_runs<<<grid_for(A.nrows), 256, 0, s>>>(A, emit);
  return cudaGetLastError();
}

cudaError_t run_label(const RunArgs& A, uint8_t* is_root, cudaStream_t s) {
  if (A.nruns <= 0) return cudaSuccess;
  k_run_init<<<grid_for(A.nruns), 256, 0, s>>>(A.L, A.nruns);
  k_run_hook<<<grid_for(A.nruns), 256, 0, s>>>(A);
  k_run_compress<<<grid_for(A.nruns), 256, 0, s>>>(A.L, A.nruns, is_root);
  return cudaGetLastError();
}

cudaError_t run_select_roots(const uint8_t* is_root, int64_t n, int32_t* roots, int32_t* nroots, void* temp,
                             size_t* temp_bytes, cudaStream_t s) {
  cub::CountingInputIterator<int32_t> it(0);
  return cub::DeviceSelect::Flagged(temp, *temp_bytes, it, is_root, roots, nroots, n, s);
}

cudaError_t run_stats(const RunArgs& A, const int32_t* roots, int32_t nroots, unsigned long long* count,
                      unsigned int* desc_key, cudaStream_t s) {
  if (A.nruns <= 0 || nroots <= 0) return cudaSuccess;
  k_run_stats<<<grid_for(A.nruns), 256, 0, s>>>(A, roots, nroots, count, desc_key);
  return cudaGetLastError();
}

cudaError_t run_fill(const RunArgs& A, const uint8_t* fill_of, uint32_t* bits, int64_t nwords, cudaStream_t s) {
  if (A.nruns <= 0 || !bits) return cudaSuccess;
  k_run_fill<<<grid_for(A.nruns), 256, 0, s>>>(A, fill_of, bits, nwords);
  return cudaGetLastError();
}

cudaError_t status_write(const RunArgs& A, const int32_t* label_of, int32_t* status, cudaStream_t s) {
  if (A.nrows <= 0) return cudaSuccess;
  k_status_write<<<grid_for(A.nrows * 32), 256, 0, s>>>(A, label_of, status);
  return cudaGetLastError();
}

cudaError_t cavity_atom_pairs(const CavAtomArgs& A, cudaStream_t s) {
  const int64_t n = A.nx * A.ny * A.nz;
  if (n <= 0) return cudaSuccess;
  k_cav_atoms<<<grid_for(n), 256, 0, s>>>(A);
  return cudaGetLastError();
}

cudaError_t shape_pass(const ShapeArgs& A, cudaStream_t s) {
  const int64_t n = A.nx * A.ny * A.nz;
  if (n <= 0) return cudaSuccess;
  k_shape_support<<<grid_for(n), 256, 0, s>>>(A);
  k_shape_cover<<<grid_for(n), 256, 0, s>>>(A);
  return cudaGetLastError();
}

cudaError_t shape_apply(const ShapeArgs& A, cudaStream_t s) {
  const int64_t n = A.nx * A.ny * A.nz;
  if (n <= 0) return cudaSuccess;
  k_shape_apply<<<grid_for(n), 256, 0, s>>>(A);
  return cudaGetLastError();
}

cudaError_t pocket_difference(int32_t* st1, const int32_t* st2, int64_t n, uint32_t* bits, unsigned long long* count,
                              cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_pocket_diff<<<grid_for(n), 256, 0, s>>>(st1, st2, n, bits, count);
  return cudaGetLastError();
}

cudaError_t pocket_cav2out(int32_t* status, const int32_t* label, int64_t n, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_pocket_cav2out<<<grid_for(n), 256, 0, s>>>(status, label, n);
  return cudaGetLastError();
}

cudaError_t dense_free_runs(const RunArgs& A, const int32_t* status, int emit, cudaStream_t s) {
  if (A.nrows <= 0) return cudaSuccess;
  k_dense_free_runs<<<grid_for(A.nrows), 256, 0, s>>>(A, status, emit);
  return cudaGetLastError();
}

cudaError_t sort_unique_u64(unsigned long long* keys, unsigned long long* keys_alt, int64_t n, int64_t* n_unique,
                            void* temp, size_t* temp_bytes, cudaStream_t s) {
  // sorted keys land in keys_alt, the unique ones back in keys; n_unique is a device counter
  size_t t1 = 0, t2 = 0;
  cudaError_t e = cub::DeviceRadixSort::SortKeys(nullptr, t1, keys, keys_alt, (int)n, 0, 64, s);
  if (e != cudaSuccess) return e;
  e = cub::DeviceSelect::Unique(nullptr, t2, keys_alt, keys, n_unique, (int)n, s);
  if (e != cudaSuccess) return e;
  if (!temp) {
    *temp_bytes = t1 > t2 ? t1 : t2;
    return cudaSuccess;
  }
  e = cub::DeviceRadixSort::SortKeys(temp, t1, keys, keys_alt, (int)n, 0, 64, s);
  if (e != cudaSuccess) return e;
  return cub::DeviceSelect::Unique(temp, t2, keys_alt, keys, n_unique, (int)n, s);
}

}  // namespace nsg
