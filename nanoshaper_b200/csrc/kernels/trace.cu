// Patch windows, tile binning and the fused ray-trace + interval-fill kernel of the SES ray caster.
//
// The reference is patch-centric: every patch loops over the pixels of its bounding window,
// tests the rays and pushes hits into per-pixel heap lists that are then sorted
// (ConnollySurface::getPatchIntersectionData src/ConnollySurface.cpp:4319-4590,
// Surface::countPixelIntersections/copyPatchIntersections/reorderPatchIntersections
// src/Surface.cpp:4941-5095) and consumed by setVerticesAndGridsWithIntersectionData
// (src/Surface.cpp:5101-6251).  Here the work is ray-centric: patches are binned into 32x4-pixel
// tiles; a CTA owns one tile, stages its patch list through shared memory in chunks, every thread
// traces one ray, keeps its hits sorted in a shared-memory column, pairs them and the warp then
// writes the status rows / insideness bits of its 32 rays cooperatively (coalesced rows, ballot
// masks + atomicAnd on the 32x-packed bit grid).  The candidate set of a ray is the reference's:
// pixel inside the patch window, inside the bounding box, inside the equatorial disc.
#include <cub/cub.cuh>

#include "pipeline.h"
#include "ray_math.cuh"

namespace nsg {

namespace {

constexpr int kChunk = 32;  // patches staged per shared-memory chunk

__device__ __forceinline__ double gcoord(const GridDev& g, int d, int64_t i) { return g.mn[d] + (double)i * g.side; }

__global__ void k_windows(PatchDev P, int32_t* win, GridDev g) {
  int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p >= P.n) return;
  const double* f = P.f64 + (int64_t)NS_PATCH_F64 * p;
  double r = f[3];
  double down[3], up[3];
  bool cull = false;
  for (int d = 0; d < 3; d++) {
    down[d] = f[d] - r;
    up[d] = f[d] + r;
    if (down[d] > g.mx[d] + NS_EPS_INT) cull = true;
  }
  for (int d = 0; d < 3; d++)
    if (up[d] < g.mn[d] - (g.hside - NS_DELTA + NS_EPS_INT)) cull = true;
  int32_t* w = win + 6 * p;
  if (cull) {
    for (int d = 0; d < 6; d++) w[d] = -1;
    return;
  }
  for (int d = 0; d < 3; d++) {
    int64_t s = (int64_t)rintp(fmax(0., down[d] - g.mn[d]) * g.scale);
    int64_t e = (int64_t)rintp(fmax(0., up[d] - g.mn[d]) * g.scale);
    if (e >= g.n[d]) e = g.n[d] - 1;
    w[d] = (int32_t)s;
    w[3 + d] = (int32_t)e;
  }
}

__global__ void k_bin(PatchDev P, GridDev g, RaySet rs, int32_t* tile_cnt, const int64_t* tile_off,
                      int32_t* tile_cursor, int32_t* tile_list) {
  int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p >= P.n) return;
  const int32_t* w = P.win + 6 * p;
  if (w[0] < 0) return;
  int64_t ntm = (rs.nb + kTileM - 1) / kTileM;
  int m0 = w[rs.fd] / kTileM, m1 = w[3 + rs.fd] / kTileM;
  int n0 = w[rs.ld] / kTileN, n1 = w[3 + rs.ld] / kTileN;
  for (int tn = n0; tn <= n1; tn++)
    for (int tm = m0; tm <= m1; tm++) {
      int64_t t = (int64_t)tn * ntm + tm;
      if (tile_list == nullptr) {
        atomicAdd(tile_cnt + t, 1);
      } else {
        int pos = atomicAdd(tile_cursor + t, 1);
        tile_list[tile_off[t] + pos] = (int32_t)p;
      }
    }
}

// Tests one (ray, patch) candidate and reports the feasible hits in t[0..n-1].
__device__ __forceinline__ int ray_patch_f64(const double* f, int kind, int first, int cnt, const PatchDev& P,
                                             const RaySet& rs, const double* pa, const double* dir, double ray_dir,
                                             double* t) {
  int fd = rs.fd, ld = rs.ld, vc = rs.vc;
  double r = f[kR];
  if (pa[fd] < f[fd] - r || pa[fd] > f[fd] + r) return 0;
  if (pa[ld] < f[ld] - r || pa[ld] > f[ld] + r) return 0;
  double dx = f[fd] - pa[fd];
  double dy = f[ld] - pa[ld];
  if (dx * dx + dy * dy > r * r) return 0;
  if (!ray_sphere_f64(pa, dir, f, r, &t[0], &t[1])) return 0;
  int numInt = 2;
  if (kind == NS_EDGE_REG || kind == NS_EDGE_SING) numInt = ray_torus_f64(f, P.probe, vc, pa, ray_dir, t);
  int out = 0;
  for (int i = 0; i < numInt; i++) {
    double ip[3] = {pa[0], pa[1], pa[2]};
    ip[vc] += t[i] * ray_dir;
    if (feasible_f64(f, kind, first, cnt, P.pool, P.flag, ip)) t[out++] = t[i];
  }
  return out;
}

// Sorted insertion into a strided hit column; returns false when the column is full.
__device__ __forceinline__ bool insert_hit(double* col, int stride, int& nh, int cap, double t) {
  if (nh >= cap) return false;
  int pos = nh;
  while (pos > 0 && col[(pos - 1) * stride] > t) {
    col[pos * stride] = col[(pos - 1) * stride];
    pos--;
  }
  col[pos * stride] = t;
  nh++;
  return true;
}

// Pairs the sorted hits of one ray in place (NEW_INTERSECTION_FILTERING) and turns them into
// interval ends along the ray axis; returns the number of pairs and the interval length sum.
// When vertex_pairs is set, only pairs that clear at least one insideness node are kept.
__device__ __forceinline__ int make_pairs(double* col, int stride, int nh, double pa_vc, double dir, double vmin,
                                          double scale, bool vertex_pairs, double* vol) {
  double v = 0.0;
  int np = 0;
  if (nh > 0 && (nh & 1) == 0) {
    for (int q = 0; q < nh; q += 2) {
      double t1 = col[q * stride], t2 = col[(q + 1) * stride];
      if (fabs(t2 - t1) >= NS_EPS_INT) {
        double lim1 = pa_vc + dir * t1;
        double lim2 = pa_vc + dir * t2;
        v += lim2 - lim1;
        if (vertex_pairs) {
          int64_t a = (int64_t)rintp((lim1 - vmin) * scale);
          int64_t b = (int64_t)rintp((lim2 - vmin) * scale);
          if (b <= a) continue;
        }
        col[(2 * np) * stride] = lim1;
        col[(2 * np + 1) * stride] = lim2;
        np++;
      }
    }
  }
  *vol = v;
  return np;
}

// Nodes of a status row inside one interval: the reference loops over the clamped rintp range
// [i1, i2] and marks the nodes with lim1 <= x <= lim2 (src/Surface.cpp:5427-5552); that set is
// the contiguous range returned here (ia > ib when empty).
__device__ __forceinline__ void status_node_range(const GridDev& g, double lim1, double lim2, int64_t* ia, int64_t* ib) {
  const int64_t NX = g.n[0];
  int64_t i1 = (int64_t)rintp((lim1 - g.mn[0]) * g.scale);
  int64_t i2 = (int64_t)rintp((lim2 - g.mn[0]) * g.scale);
  i1 = i1 < 0 ? 0 : (i1 >= NX ? NX - 1 : i1);
  i2 = i2 < 0 ? 0 : (i2 >= NX ? NX - 1 : i2);
  int64_t a = i1, b = i2;
  while (a <= b && gcoord(g, 0, a) < lim1) a++;
  while (b >= a && gcoord(g, 0, b) > lim2) b--;
  *ia = a;
  *ib = b;
}

// Warp-aggregated append of this lane's `cnt` records to a shared store; returns the lane's first
// slot, or -1 when the store is full (the error flag is then set to `code`).
__device__ __forceinline__ int64_t warp_append(unsigned long long* cursor, int64_t cap, int cnt, int32_t* error_flag,
                                               int code) {
  const int lane = threadIdx.x & 31;
  int incl = cnt;
  for (int o = 1; o < 32; o <<= 1) {
    int v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  int total = __shfl_sync(0xffffffffu, incl, 31);
  unsigned long long base = 0;
  if (lane == 31 && total > 0) base = atomicAdd(cursor, (unsigned long long)total);
  base = __shfl_sync(0xffffffffu, base, 31);
  if ((int64_t)base + total > cap) {
    if (lane == 0 && total > 0) atomicExch(error_flag, code);
    return -1;
  }
  return (int64_t)base + incl - cnt;
}

__device__ __forceinline__ void clear_bits_range(uint32_t* bits, int64_t nwords, int64_t f0, int64_t f1) {
  // clears bits f0..f1 inclusive of the flat bit grid (bit = 0 means inside)
  if (f1 < f0) return;
  if (f0 < 0) f0 = 0;
  int64_t lim = nwords * 32 - 1;
  if (f1 > lim) f1 = lim;
  for (int64_t w = f0 >> 5; w <= (f1 >> 5); w++) {
    int64_t lo = w << 5;
    int s = (int)(f0 > lo ? f0 - lo : 0);
    int e = (int)(f1 < lo + 31 ? f1 - lo : 31);
    uint32_t mask = (e - s == 31) ? 0xffffffffu : (((1u << (e - s + 1)) - 1u) << s);
    atomicAnd(bits + w, ~mask);
  }
}

struct TraceCtx {
  PatchDev P;
  GridDev g;
  RaySet rs;
  TraceOut out;
  int64_t nwords;
};

template <int kThreads>
__global__ void __launch_bounds__(kTraceThreads) k_trace(TraceCtx C, const int64_t* __restrict__ tile_off,
                                                          const int32_t* __restrict__ tile_list) {
  const GridDev& g = C.g;
  const RaySet& rs = C.rs;
  __shared__ double s_f[kChunk * NS_PATCH_F64];
  __shared__ int s_i[kChunk * 3];
  __shared__ int s_w[kChunk * 4];
  __shared__ double s_hit[kHitCap * kThreads];

  const int64_t ntm = (rs.nb + kTileM - 1) / kTileM;
  const int64_t tile = blockIdx.x;
  const int64_t tm = tile % ntm, tn = tile / ntm;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t m = tm * kTileM + lane;
  const int64_t n = tn * kTileN + warp;
  const bool valid = (m < rs.nb) && (n < rs.na);
  const int tid = threadIdx.x;
  double* col = s_hit + tid;

  double pa[3], dir[3] = {0., 0., 0.};
  pa[rs.fd] = gcoord(g, rs.fd, valid ? m : 0) + rs.delta;
  pa[rs.ld] = gcoord(g, rs.ld, valid ? n : 0) + rs.delta;
  pa[rs.vc] = gcoord(g, rs.vc, 0) + rs.delta;
  const double ray_dir = gcoord(g, rs.vc, g.n[rs.vc] - 1) - gcoord(g, rs.vc, 0);
  dir[rs.vc] = ray_dir;

  int nh = 0;
  bool ovf = false;
  const int64_t beg = tile_off[tile], end = tile_off[tile + 1];
  for (int64_t base = beg; base < end; base += kChunk) {
    int cnt = (int)((end - base) < kChunk ? (end - base) : kChunk);
    __syncthreads();
    for (int e = tid; e < cnt * NS_PATCH_F64; e += kThreads) {
      int q = e / NS_PATCH_F64, k = e - q * NS_PATCH_F64;
      int64_t pid = tile_list[base + q];
      s_f[e] = __ldg(C.P.f64 + (int64_t)NS_PATCH_F64 * pid + k);
    }
    for (int q = tid; q < cnt; q += kThreads) {
      int64_t pid = tile_list[base + q];
      s_i[3 * q + 0] = C.P.i32[NS_PATCH_I32 * pid + 0];
      s_i[3 * q + 1] = C.P.i32[NS_PATCH_I32 * pid + 1];
      s_i[3 * q + 2] = C.P.i32[NS_PATCH_I32 * pid + 2];
      const int32_t* w = C.P.win + 6 * pid;
      s_w[4 * q + 0] = w[rs.fd];
      s_w[4 * q + 1] = w[3 + rs.fd];
      s_w[4 * q + 2] = w[rs.ld];
      s_w[4 * q + 3] = w[3 + rs.ld];
    }
    __syncthreads();
    if (!valid || ovf) continue;
    for (int q = 0; q < cnt; q++) {
      if (m < s_w[4 * q] || m > s_w[4 * q + 1] || n < s_w[4 * q + 2] || n > s_w[4 * q + 3]) continue;
      double t[4];
      int k = ray_patch_f64(s_f + q * NS_PATCH_F64, s_i[3 * q], s_i[3 * q + 1], s_i[3 * q + 2], C.P, rs, pa, dir,
                            ray_dir, t);
      for (int i = 0; i < k; i++)
        if (!insert_hit(col, kThreads, nh, kHitCap, t[i])) ovf = true;
    }
  }
  const int64_t rid = n * rs.nb + m;
  if (valid && ovf) {
    int slot = atomicAdd(C.out.ovf_count, 1);
    if (slot < C.out.ovf_cap) C.out.ovf_rays[slot] = (int32_t)rid;
    else atomicExch(C.out.error_flag, 1);
  }
  if (valid && !ovf && C.out.hits) {
    unsigned long long off = atomicAdd(C.out.hit_cursor, (unsigned long long)nh);
    if ((int64_t)(off + nh) <= C.out.hit_cap) {
      for (int i = 0; i < nh; i++) C.out.hits[off + i] = col[i * kThreads];
      C.out.ray_hit_off[rid] = (int64_t)off;
      C.out.ray_hit_cnt[rid] = nh;
    } else {
      atomicExch(C.out.error_flag, 2);
    }
  }
  // interval ends
  const bool mc = rs.set != 0;
  double pa_vc, dirl;
  if (!mc) {
    pa_vc = gcoord(g, 0, 0);
    dirl = gcoord(g, 0, g.n[0] - 1) - pa_vc;
  } else {
    pa_vc = gcoord(g, rs.vc, 0) + rs.delta;
    double pb = gcoord(g, rs.vc, g.n[rs.vc] - 1) + rs.delta;
    dirl = pb - pa_vc;
  }
  double vol = 0.0;
  int np = 0;
  if (valid && !ovf) np = make_pairs(col, kThreads, nh, pa_vc, dirl, g.mn[rs.vc], g.scale, mc, &vol);
  if (valid && !ovf) C.out.vol_ray[rid] = vol;
  __syncwarp();
  const int64_t NX = g.n[0], NY = g.n[1];
  if (!mc) {
    // status row (., j = m, k = n): runs of inside nodes
    int nr = 0;
    if (valid && !ovf)
      for (int q = 0; q < np; q++) {
        int64_t ia, ib;
        status_node_range(g, col[(2 * q) * kThreads], col[(2 * q + 1) * kThreads], &ia, &ib);
        if (ia > ib) continue;
        col[(2 * nr) * kThreads] = (double)ia;
        col[(2 * nr + 1) * kThreads] = (double)ib;
        nr++;
      }
    int64_t off = warp_append(C.out.srun_cursor, C.out.srun_cap, nr, C.out.error_flag, 5);
    if (valid && !ovf) {
      if (off >= 0) {
        for (int q = 0; q < nr; q++)
          C.out.sruns[off + q] = make_int2((int)col[(2 * q) * kThreads], (int)col[(2 * q + 1) * kThreads]);
        C.out.srun_off[rid] = off;
        C.out.srun_cnt[rid] = nr;
      } else {
        C.out.srun_cnt[rid] = 0;
      }
    }
    return;
  }
  // accurate-triangulation rays: pair store for the vertex assembly
  {
    int64_t off = warp_append(C.out.pair_cursor, C.out.pair_cap, np, C.out.error_flag, 3);
    if (valid && !ovf) {
      int64_t ord = rs.ordinal_base + rid;
      if (off >= 0) {
        for (int q = 0; q < np; q++) {
          C.out.pairs[2 * (off + q)] = col[(2 * q) * kThreads];
          C.out.pairs[2 * (off + q) + 1] = col[(2 * q + 1) * kThreads];
        }
        C.out.ray_pair_off[ord] = off;
        C.out.ray_pair_cnt[ord] = np;
      } else {
        C.out.ray_pair_cnt[ord] = 0;
      }
    }
  }
  const double vmin = g.mn[rs.vc];
  if (rs.panel == 0) {
    // row bits (i, j = m, k = n), i in (a, b]
    for (int r = 0; r < 32; r++) {
      int np_r = __shfl_sync(0xffffffffu, np, r);
      if (np_r == 0) continue;
      const double* cr = s_hit + warp * 32 + r;
      int64_t j = tm * kTileM + r;
      int64_t f0 = (n * NY + j) * NX;
      for (int q = 0; q < np_r; q++) {
        int64_t a = (int64_t)rintp((cr[(2 * q) * kThreads] - vmin) * g.scale);
        int64_t b = (int64_t)rintp((cr[(2 * q + 1) * kThreads] - vmin) * g.scale);
        int64_t lo = f0 + a + 1, hi = f0 + b;
        if (lo < 0) lo = 0;
        int64_t maxb = C.nwords * 32 - 1;
        if (hi > maxb) hi = maxb;
        if (hi < lo) continue;
        for (int64_t w = (lo >> 5) + lane; w <= (hi >> 5); w += 32) {
          int64_t wl = w << 5;
          int s = (int)(lo > wl ? lo - wl : 0);
          int e = (int)(hi < wl + 31 ? hi - wl : 31);
          uint32_t mask = (e - s == 31) ? 0xffffffffu : (((1u << (e - s + 1)) - 1u) << s);
          atomicAnd(C.out.bits + w, ~mask);
        }
      }
    }
    return;
  }
  // panels 1 and 2: lanes are consecutive i; one ballot per position along the ray axis
  int64_t first_a = INT64_MAX, last_b = INT64_MIN;
  if (np > 0) {
    first_a = (int64_t)rintp((col[0] - vmin) * g.scale) + 1;
    last_b = (int64_t)rintp((col[(2 * np - 1) * kThreads] - vmin) * g.scale);
  }
  int64_t vlo = first_a, vhi = last_b;
  for (int o = 16; o > 0; o >>= 1) {
    long long ol = __shfl_xor_sync(0xffffffffu, (long long)vlo, o);
    long long oh = __shfl_xor_sync(0xffffffffu, (long long)vhi, o);
    vlo = ol < vlo ? ol : vlo;
    vhi = oh > vhi ? oh : vhi;
  }
  if (vlo > vhi) return;
  int q = 0;
  int64_t qa = 0, qb = -1;
  if (np > 0) {
    qa = (int64_t)rintp((col[0] - vmin) * g.scale);
    qb = (int64_t)rintp((col[kThreads] - vmin) * g.scale);
  }
  const int64_t m0 = tm * kTileM;
  for (int64_t v = vlo; v <= vhi; v++) {
    while (q < np && qb < v) {
      q++;
      if (q < np) {
        qa = (int64_t)rintp((col[(2 * q) * kThreads] - vmin) * g.scale);
        qb = (int64_t)rintp((col[(2 * q + 1) * kThreads] - vmin) * g.scale);
      }
    }
    bool inside = q < np && qa < v && v <= qb;
    unsigned mask = __ballot_sync(0xffffffffu, inside);
    if (lane == 0 && mask) {
      int64_t f0 = (rs.panel == 1) ? ((v * NY + n) * NX + m0) : ((n * NY + v) * NX + m0);
      if (f0 >= 0) {
        int64_t w = f0 >> 5;
        int s = (int)(f0 & 31);
        if (w < C.nwords) atomicAnd(C.out.bits + w, ~(mask << s));
        if (s && w + 1 < C.nwords) atomicAnd(C.out.bits + w + 1, ~(mask >> (32 - s)));
      }
    }
  }
}

// One thread per overflow ray: the same candidate tests with the hits kept in a global column.
__global__ void k_trace_overflow(TraceCtx C, const int64_t* __restrict__ tile_off, const int32_t* __restrict__ tile_list,
                                 int n_ovf, double* scratch) {
  int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n_ovf) return;
  const GridDev& g = C.g;
  const RaySet& rs = C.rs;
  int64_t rid = C.out.ovf_rays[idx];
  int64_t m = rid % rs.nb, n = rid / rs.nb;
  int64_t ntm = (rs.nb + kTileM - 1) / kTileM;
  int64_t tile = (n / kTileN) * ntm + m / kTileM;
  double* col = scratch + (int64_t)idx * kOverflowCap;
  double pa[3], dir[3] = {0., 0., 0.};
  pa[rs.fd] = gcoord(g, rs.fd, m) + rs.delta;
  pa[rs.ld] = gcoord(g, rs.ld, n) + rs.delta;
  pa[rs.vc] = gcoord(g, rs.vc, 0) + rs.delta;
  const double ray_dir = gcoord(g, rs.vc, g.n[rs.vc] - 1) - gcoord(g, rs.vc, 0);
  dir[rs.vc] = ray_dir;
  int nh = 0;
  for (int64_t e = tile_off[tile]; e < tile_off[tile + 1]; e++) {
    int64_t pid = tile_list[e];
    const int32_t* w = C.P.win + 6 * pid;
    if (m < w[rs.fd] || m > w[3 + rs.fd] || n < w[rs.ld] || n > w[3 + rs.ld]) continue;
    double f[NS_PATCH_F64];
    for (int k = 0; k < NS_PATCH_F64; k++) f[k] = C.P.f64[(int64_t)NS_PATCH_F64 * pid + k];
    const int32_t* ir = C.P.i32 + NS_PATCH_I32 * pid;
    double t[4];
    int k = ray_patch_f64(f, ir[0], ir[1], ir[2], C.P, rs, pa, dir, ray_dir, t);
    for (int i = 0; i < k; i++)
      if (!insert_hit(col, 1, nh, kOverflowCap, t[i])) {
        atomicExch(C.out.error_flag, 4);
        return;
      }
  }
  if (C.out.hits) {
    unsigned long long off = atomicAdd(C.out.hit_cursor, (unsigned long long)nh);
    if ((int64_t)(off + nh) <= C.out.hit_cap) {
      for (int i = 0; i < nh; i++) C.out.hits[off + i] = col[i];
      C.out.ray_hit_off[rid] = (int64_t)off;
      C.out.ray_hit_cnt[rid] = nh;
    } else {
      atomicExch(C.out.error_flag, 2);
    }
  }
  const bool mc = rs.set != 0;
  double pa_vc, dirl;
  if (!mc) {
    pa_vc = gcoord(g, 0, 0);
    dirl = gcoord(g, 0, g.n[0] - 1) - pa_vc;
  } else {
    pa_vc = gcoord(g, rs.vc, 0) + rs.delta;
    dirl = (gcoord(g, rs.vc, g.n[rs.vc] - 1) + rs.delta) - pa_vc;
  }
  double vol = 0.0;
  int np = make_pairs(col, 1, nh, pa_vc, dirl, g.mn[rs.vc], g.scale, mc, &vol);
  C.out.vol_ray[rid] = vol;
  const int64_t NX = g.n[0], NY = g.n[1];
  if (!mc) {
    int nr = 0;
    for (int q = 0; q < np; q++) {
      int64_t ia, ib;
      status_node_range(g, col[2 * q], col[2 * q + 1], &ia, &ib);
      if (ia > ib) continue;
      col[2 * nr] = (double)ia;
      col[2 * nr + 1] = (double)ib;
      nr++;
    }
    unsigned long long off = nr ? atomicAdd(C.out.srun_cursor, (unsigned long long)nr) : 0;
    if ((int64_t)off + nr <= C.out.srun_cap) {
      for (int q = 0; q < nr; q++) C.out.sruns[off + q] = make_int2((int)col[2 * q], (int)col[2 * q + 1]);
      C.out.srun_off[rid] = (int64_t)off;
      C.out.srun_cnt[rid] = nr;
    } else {
      C.out.srun_cnt[rid] = 0;
      atomicExch(C.out.error_flag, 5);
    }
    return;
  }
  int64_t ord = rs.ordinal_base + rid;
  unsigned long long off = np ? atomicAdd(C.out.pair_cursor, (unsigned long long)np) : 0;
  if ((int64_t)off + np <= C.out.pair_cap) {
    for (int q = 0; q < np; q++) {
      C.out.pairs[2 * (off + q)] = col[2 * q];
      C.out.pairs[2 * (off + q) + 1] = col[2 * q + 1];
    }
    C.out.ray_pair_off[ord] = (int64_t)off;
    C.out.ray_pair_cnt[ord] = np;
  } else {
    C.out.ray_pair_cnt[ord] = 0;
    atomicExch(C.out.error_flag, 3);
  }
  const double vmin = g.mn[rs.vc];
  for (int q = 0; q < np; q++) {
    int64_t a = (int64_t)rintp((col[2 * q] - vmin) * g.scale);
    int64_t b = (int64_t)rintp((col[2 * q + 1] - vmin) * g.scale);
    if (rs.panel == 0) {
      int64_t f0 = (n * NY + m) * NX;
      clear_bits_range(C.out.bits, C.nwords, f0 + a + 1, f0 + b);
    } else {
      for (int64_t v = a + 1; v <= b; v++) {
        int64_t f = (rs.panel == 1) ? ((v * NY + n) * NX + m) : ((n * NY + v) * NX + m);
        clear_bits_range(C.out.bits, C.nwords, f, f);
      }
    }
  }
}

int64_t words_of(const GridDev& g) { return ((g.n[0] + 31) >> 5) * g.n[1] * g.n[2]; }

}  // namespace

cudaError_t launch_windows(const PatchDev& P, int32_t* win, const GridDev& g, cudaStream_t s) {
  if (P.n == 0) return cudaSuccess;
  k_windows<<<(unsigned)((P.n + 255) / 256), 256, 0, s>>>(P, win, g);
  return cudaGetLastError();
}

cudaError_t launch_bin_count(const PatchDev& P, const GridDev& g, const RaySet& rs, int32_t* tile_cnt,
                             cudaStream_t s) {
  if (P.n == 0) return cudaSuccess;
  k_bin<<<(unsigned)((P.n + 255) / 256), 256, 0, s>>>(P, g, rs, tile_cnt, nullptr, nullptr, nullptr);
  return cudaGetLastError();
}

cudaError_t launch_bin_fill(const PatchDev& P, const GridDev& g, const RaySet& rs, const int64_t* tile_off,
                            int32_t* tile_cursor, int32_t* tile_list, cudaStream_t s) {
  if (P.n == 0) return cudaSuccess;
  k_bin<<<(unsigned)((P.n + 255) / 256), 256, 0, s>>>(P, g, rs, nullptr, tile_off, tile_cursor, tile_list);
  return cudaGetLastError();
}

cudaError_t launch_trace(const PatchDev& P, const GridDev& g, const RaySet& rs, const int64_t* tile_off,
                         const int32_t* tile_list, const TraceOut& out, int precision, cudaStream_t s) {
  (void)precision;
  TraceCtx C{P, g, rs, out, words_of(g)};
  int64_t ntiles = ((rs.nb + kTileM - 1) / kTileM) * ((rs.na + kTileN - 1) / kTileN);
  k_trace<kTraceThreads><<<(unsigned)ntiles, kTraceThreads, 0, s>>>(C, tile_off, tile_list);
  return cudaGetLastError();
}

cudaError_t launch_trace_overflow(const PatchDev& P, const GridDev& g, const RaySet& rs, const int64_t* tile_off,
                                  const int32_t* tile_list, const TraceOut& out, int n_ovf, double* scratch,
                                  int precision, cudaStream_t s) {
  (void)precision;
  if (n_ovf <= 0) return cudaSuccess;
  TraceCtx C{P, g, rs, out, words_of(g)};
  k_trace_overflow<<<(n_ovf + 63) / 64, 64, 0, s>>>(C, tile_off, tile_list, n_ovf, scratch);
  return cudaGetLastError();
}

}  // namespace nsg
