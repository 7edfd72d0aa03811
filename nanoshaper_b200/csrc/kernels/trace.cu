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
#include "ray_math_mixed.cuh"
#include "grad.cuh"
#include "isect.cuh"

namespace nsg {

namespace {



__global__ void k_windows(PatchDev P, int32_t* win, BatchDev B) {
  int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p >= P.n) return;
  const GridDev& g = B.s[B.patch_struct[p]].g;
  const double* f = P.f64 + (int64_t)NS_PATCH_F64 * p;
  double r = f[3];
  double down[3], up[3];
  bool cull = false;
  const bool skin = ns_has_box(P.i32[NS_PATCH_I32 * p]);
  for (int d = 0; d < 3; d++) {
    // SES: the bounding sphere's box; skin cells and mesh triangles: their stored box
    // (src/SkinSurface.cpp:3470-3500, src/MeshSurface.cpp:447-472)
    down[d] = skin ? f[NS_SKIN_LO + d] : f[d] - r;
    up[d] = skin ? f[NS_SKIN_HI + d] : f[d] + r;
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

__global__ void k_pool32(PatchDev P, float4* out, float4* quad32, double4* quadl) {
  int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p >= P.n) return;
  const double* f = P.f64 + (int64_t)NS_PATCH_F64 * p;
  const int32_t* ir = P.i32 + NS_PATCH_I32 * p;
  const int kind = ir[0];
  const bool skin = ns_is_skin(kind);
  for (int q = ir[1]; q < ir[1] + ir[2]; q++) {
    double4 w = P.pool[q];
    if (kind == NS_POINT) {
      out[q] = make_float4((float)(w.x - f[0]), (float)(w.y - f[1]), (float)(w.z - f[2]), (float)w.w);
    } else {
      // planes about the local origin; the skin's (partly unnormalised) planes are scaled to unit
      // normals so that the FP32 value is a distance (the scale does not change a sign)
      const double inv = skin ? 1.0 / sqrt(w.x * w.x + w.y * w.y + w.z * w.z) : 1.0;
      out[q] = make_float4((float)(w.x * inv), (float)(w.y * inv), (float)(w.z * inv),
                           (float)((w.w + (w.x * f[0] + w.y * f[1] + w.z * f[2])) * inv));
    }
  }
  if (skin && quad32) {
    // the quadric about the local origin c: A, bl = A c + b, cl = f(c)
    const double* Q = f + NS_SKIN_Q;
    const double A[3][3] = {{Q[0], Q[4], Q[7]}, {Q[4], Q[1], Q[5]}, {Q[7], Q[5], Q[2]}};
    const double b[3] = {Q[9], Q[8], Q[6]};
    double bl[3];
    for (int i = 0; i < 3; i++) bl[i] = (A[i][0] * f[0] + A[i][1] * f[1] + A[i][2] * f[2]) + b[i];
    const double cl = (f[0] * (bl[0] + b[0]) + f[1] * (bl[1] + b[1]) + f[2] * (bl[2] + b[2])) + Q[3];
    quad32[3 * p] = make_float4((float)A[0][0], (float)A[1][1], (float)A[2][2], (float)A[0][1]);
    quad32[3 * p + 1] = make_float4((float)A[1][2], (float)A[0][2], (float)bl[0], (float)bl[1]);
    quad32[3 * p + 2] = make_float4((float)bl[2], (float)cl, 0.f, 0.f);
    quadl[p] = make_double4(bl[0], bl[1], bl[2], cl);
  }
}

__global__ void k_kind_mask(PatchDev P, int* mask) {
  int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int bit = p < P.n ? (1 << P.i32[NS_PATCH_I32 * p]) : 0;
  bit = __reduce_or_sync(0xffffffffu, bit);
  if ((threadIdx.x & 31) == 0 && bit) atomicOr(mask, bit);
}

__global__ void k_bin(PatchDev P, BatchDev B, int set, int32_t* tile_cnt, const int64_t* tile_off,
                      int32_t* tile_cursor, int32_t* tile_list, unsigned long long* area) {
  int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int32_t* w = P.win + 6 * (p < P.n ? p : 0);
  bool live = p < P.n && w[0] >= 0;
  const StructDev& S = B.s[p < P.n ? B.patch_struct[p] : 0];
  const RaySet rs = make_ray_set(set, S.g);
  if (area) {
    // pixel-window area: an upper bound of the patch's candidate rays in this panel
    const int ww = w[3 + rs.fd] - w[rs.fd] + 1, wh = w[3 + rs.ld] - w[rs.ld] + 1;
    unsigned a = (live && ww > 0 && wh > 0) ? (unsigned)(ww * wh) : 0u;
    unsigned sum = __reduce_add_sync(0xffffffffu, a);
    if ((threadIdx.x & 31) == 0 && sum) atomicAdd(area, (unsigned long long)sum);
  }
  if (!live || (tile_cnt == nullptr && tile_list == nullptr)) return;
  int64_t ntm = (rs.nb + kTileM - 1) / kTileM;
  int m0 = w[rs.fd] / kTileM, m1 = w[3 + rs.fd] / kTileM;
  int n0 = w[rs.ld] / kTileN, n1 = w[3 + rs.ld] / kTileN;
  for (int tn = n0; tn <= n1; tn++)
    for (int tm = m0; tm <= m1; tm++) {
      int64_t t = S.tile_base[rs.panel] + (int64_t)tn * ntm + tm;
      if (tile_list == nullptr) {
        atomicAdd(tile_cnt + t, 1);
      } else {
        int pos = atomicAdd(tile_cursor + t, 1);
        tile_list[tile_off[t] + pos] = (int32_t)p;
      }
    }
}

// Candidate test of the reference's pixel loop: the ray origin lies inside the patch's bounding
// box and equatorial disc (src/ConnollySurface.cpp:4469-4502); the pixel window test is done by
// the caller.
__device__ __forceinline__ bool candidate(const double* f, const RaySet& rs, const double* pa) {
  int fd = rs.fd, ld = rs.ld;
  double r = f[kR];
  if (pa[fd] < f[fd] - r || pa[fd] > f[fd] + r) return false;
  if (pa[ld] < f[ld] - r || pa[ld] > f[ld] + r) return false;
  double dx = f[fd] - pa[fd];
  double dy = f[ld] - pa[ld];
  return !(dx * dx + dy * dy > r * r);
}

// Double-precision intersection of a candidate: hits in t[0..n-1] (ray parameter units).
__device__ __forceinline__ int intersect_f64(const double* f, int kind, int first, int cnt, const PatchDev& P,
                                             const RaySet& rs, const double* pa, const double* dir, double ray_dir,
                                             double* t) {
  int vc = rs.vc;
  if (!ray_sphere_f64(pa, dir, f, f[kR], &t[0], &t[1])) return 0;
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

// Tests one (ray, patch) candidate and reports the feasible hits in t[0..n-1].
__device__ __forceinline__ int ray_patch_f64(const double* f, int kind, int first, int cnt, const PatchDev& P,
                                             const RaySet& rs, const double* pa, const double* dir, double ray_dir,
                                             double box_dir, double tri_dir, double* t) {
  if (kind == NS_MESH_TRI) {
    for (int a = 0; a < 2; a++) {
      const int d = a == 0 ? rs.fd : rs.ld;
      if (pa[d] < f[NS_SKIN_LO + d] || pa[d] > f[NS_SKIN_HI + d]) return 0;
    }
    double tdir[3] = {0.0, 0.0, 0.0}, u, v;
    tdir[rs.vc] = tri_dir;
    return ray_triangle_f64(pa, tdir, f, f + 3, f + 6, t, &u, &v) ? 1 : 0;
  }
  if (ns_is_skin(kind)) {
    // the cell's box in the pixel axes, the atom disc for Del0 cells, then the ray-quadric test
    for (int a = 0; a < 2; a++) {
      const int d = a == 0 ? rs.fd : rs.ld;
      if (pa[d] < f[NS_SKIN_LO + d] || pa[d] > f[NS_SKIN_HI + d]) return 0;
    }
    if (kind == NS_SKIN_POINT) {
      const double dx = f[rs.fd] - pa[rs.fd], dy = f[rs.ld] - pa[rs.ld];
      if (dx * dx + dy * dy > f[kR] * f[kR]) return 0;
    }
    double tt[2];
    bool hit = rs.vc == 0 ? ray_quadric_f64<0>(f + NS_SKIN_Q, pa, tt)
                          : (rs.vc == 1 ? ray_quadric_f64<1>(f + NS_SKIN_Q, pa, tt) : ray_quadric_f64<2>(f + NS_SKIN_Q, pa, tt));
    if (!hit) return 0;
    int out = 0;
    for (int i = 0; i < 2; i++) {
      double ip[3] = {pa[0], pa[1], pa[2]};
      ip[rs.vc] += tt[i];
      if (feasible_skin_f64(P.pool, first, cnt, ip)) t[out++] = tt[i] / box_dir;
    }
    return out;
  }
  if (!candidate(f, rs, pa)) return 0;
  return intersect_f64(f, kind, first, cnt, P, rs, pa, dir, ray_dir, t);
}

// Pairs the sorted hits of one ray in place (NEW_INTERSECTION_FILTERING) and turns them into
// interval ends along the ray axis; returns the number of pairs and the interval length sum.
// When vertex_pairs is set, only pairs that clear at least one insideness node are kept.
// With pcol (the hits' patches, gradient mode) the patch column is compacted alongside, and every
// interval end adds its term of d volume / d patch parameters (GradCtx).
struct GradCtx {
  const double* f64;
  const int32_t* i32;
  double probe;
  double w;          // volume weight of an interval length: A / number of ray sets
  double x[3];       // ray origin; x[vc] is replaced by the interval end
  int vc;
  double* gvol;
};

struct SamePid {
  __device__ __forceinline__ int32_t operator()(int32_t p) const { return p; }
};

// pcol holds, per hit, an id that pid_of turns into the hit's patch (the patch itself, or the
// hit's slot in the hit store).
template <class IdT = int32_t, class PidOf = SamePid>
__device__ __forceinline__ int make_pairs(double* col, int stride, int nh, double pa_vc, double dir, double vmin,
                                          double scale, bool vertex_pairs, double* vol, IdT* pcol = nullptr,
                                          GradCtx* gc = nullptr, PidOf pid_of = PidOf()) {
  double v = 0.0;
  int np = 0;
  if (nh > 0 && (nh & 1) == 0) {
    for (int q = 0; q < nh; q += 2) {
      double t1 = col[q * stride], t2 = col[(q + 1) * stride];
      if (fabs(t2 - t1) >= NS_EPS_INT) {
        double lim1 = pa_vc + dir * t1;
        double lim2 = pa_vc + dir * t2;
        v += lim2 - lim1;
        IdT p1 = 0, p2 = 0;
        if (pcol) {
          p1 = pcol[q * stride];
          p2 = pcol[(q + 1) * stride];
          if (gc) {
            double x[3] = {gc->x[0], gc->x[1], gc->x[2]};
            x[gc->vc] = lim1;
            add_hit_grad(gc->f64, gc->i32, gc->probe, pid_of(p1), x, gc->vc, -gc->w, gc->gvol);
            x[gc->vc] = lim2;
            add_hit_grad(gc->f64, gc->i32, gc->probe, pid_of(p2), x, gc->vc, gc->w, gc->gvol);
          }
        }
        if (vertex_pairs) {
          int64_t a = (int64_t)rintp((lim1 - vmin) * scale);
          int64_t b = (int64_t)rintp((lim2 - vmin) * scale);
          if (b <= a) continue;
        }
        col[(2 * np) * stride] = lim1;
        col[(2 * np + 1) * stride] = lim2;
        if (pcol) {
          pcol[(2 * np) * stride] = p1;
          pcol[(2 * np + 1) * stride] = p2;
        }
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

// Epsilon-map entries of one interval [lim1, lim2] of a node ray (sets 0, 4, 5): the reference takes
// the clamped rintp node range [c1, c2] of the interval and marks the grid edges that start at a
// node c with coord(c) <= lim2 - hside (src/Surface.cpp:6645-6680 for x, inclusive of c2;
// :6786-6795 for z and :6887-6896 for y, exclusive of c2).  m, n are the ray's pixel indices.
__device__ __forceinline__ void eps_fill(const GridDev& g, const RaySet& rs, int64_t m, int64_t n, double lim1,
                                         double lim2, int32_t* __restrict__ eps, int32_t inside) {
  const int vc = rs.vc;
  const int64_t N = g.n[vc];
  int64_t c1 = (int64_t)rintp((lim1 - g.mn[vc]) * g.scale);
  int64_t c2 = (int64_t)rintp((lim2 - g.mn[vc]) * g.scale);
  c1 = c1 < 0 ? 0 : (c1 >= N ? N - 1 : c1);
  c2 = c2 < 0 ? 0 : (c2 >= N ? N - 1 : c2);
  if (c2 < c1) return;
  int64_t e = vc == 0 ? c2 : c2 - 1;
  const double lim = lim2 - g.hside;
  while (e >= c1 && gcoord(g, vc, e) > lim) e--;
  const int64_t NX = g.n[0], NY = g.n[1];
  // node (i, j, k) of position c along the ray; l = the component of this ray set
  int64_t base, step;
  int l;
  if (vc == 0) { base = (n * NY + m) * NX; step = 1; l = 0; }
  else if (vc == 2) { base = n * NX + m; step = NX * NY; l = 2; }
  else { base = n * NY * NX + m; step = NX; l = 1; }
  for (int64_t c = c1; c <= e; c++) eps[(base + c * step) * 3 + l] = inside;
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


// Wavefront ray tracing of one ray set, three kernel kinds:
//  * k_cand: one warp per batch of 32 patches, whose records the lanes load together; then, patch
//    by patch, one lane per pixel row of the patch's pixel window (the reference's CELL_CULLING
//    window, k_windows): each row's rays that pass the bounding-box and equatorial-disc test form
//    an interval, found by binary search with the exact test.  One atomic per list and batch
//    reserves the slots; the (ray, patch) pairs follow in row-major order, in the sphere list
//    (atoms and probes) or the torus list; a patch's candidates stay contiguous, so the
//    intersection kernels read its record once per warp;
//  * k_isect<torus> (double precision) and k_isect_mixed<torus> (trace_mixed.cu): one thread per
//    candidate pair, sphere and torus pairs in separate launches so that both run converged with
//    their own register budget; hits are filed into the ray's slots of a slot-major hit store
//    through a per-ray atomic counter;
//  * k_fill: one CTA per 32x4 ray tile loads each ray's hits, sorts them and performs the
//    interval fill.
// A k_cand batch of 32 patches, staged in shared memory (structure of arrays, one entry per lane
// of the warp that loaded it): the operands of candidate() rounded as there, the pixel window
// and where the patch's rays start.
struct CandBatch {
  double cf[32], cl[32], lo_fd[32], hi_fd[32], lo_ld[32], hi_ld[32], r2[32], mn_fd[32], mn_ld[32], side[32],
      delta[32];
  int64_t nb[32], rbase[32], base[32];
  int m0[32], m1[32], n0[32], ty[32], pid[32], disc[32];
  int64_t gfirst[32], gend[32];
};

// Candidate count of pixel row `row` of batch patch p (its first candidate pixel in *a).  Along a
// row the pixel coordinate pa(m) is non-decreasing in m and dx = cf - pa(m) non-increasing;
// fl(fl(dx*dx) + fl(dy*dy)) is non-decreasing in |dx|.  So
//   Low(m)  = pa(m) >= lo_fd && (dx < 0 || disc(dx))   holds on an upper set of m,
//   High(m) = pa(m) <= hi_fd && (dx > 0 || disc(dx))   holds on a lower set of m,
// and candidate() (box in both axes, then disc) passes exactly when the row's box test holds and
// Low(m) && High(m).  The row's candidates are the interval [first Low, last High] of the
// window, found by two binary searches with the exact double-precision tests.
__device__ __forceinline__ int cand_row(const CandBatch& q, int p, int row, int* a) {
  *a = 0;
  const double pld = (q.mn_ld[p] + (double)(q.n0[p] + row) * q.side[p]) + q.delta[p];
  if (pld < q.lo_ld[p] || pld > q.hi_ld[p]) return 0;
  const double cl = q.cl[p], cf = q.cf[p], r2 = q.r2[p], mn = q.mn_fd[p], side = q.side[p], delta = q.delta[p];
  const double lo_fd = q.lo_fd[p], hi_fd = q.hi_fd[p];
  const double dy = cl - pld;
  const double dy2 = dy * dy;
  // skin cells other than Del0 have no equatorial-disc test (src/SkinSurface.cpp:3578-3587)
  const bool disc = q.disc[p];
  int lo = q.m0[p], hi = q.m1[p] + 1;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    const double pa = (mn + (double)mid * side) + delta;
    const double dx = cf - pa;
    const bool low = !(pa < lo_fd) && (!disc || dx < 0. || !(dx * dx + dy2 > r2));
    if (low) hi = mid;
    else lo = mid + 1;
  }
  *a = lo;
  hi = q.m1[p] + 1;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    const double pa = (mn + (double)mid * side) + delta;
    const double dx = cf - pa;
    const bool high = !(pa > hi_fd) && (!disc || dx > 0. || !(dx * dx + dy2 > r2));
    if (!high) hi = mid;
    else lo = mid + 1;
  }
  return lo - *a;
}

// Smallest lane whose inclusive prefix v exceeds k (k below the warp total).
__device__ __forceinline__ int owner_lane(int v, int k) {
  int rr = 0;
#pragma unroll
  for (int step = 16; step; step >>= 1) {
    const int x = __shfl_sync(0xffffffffu, v, rr + step - 1);
    if (x <= k) rr += step;
  }
  return rr;
}

__global__ void __launch_bounds__(256) k_cand(TraceCtx C, CandOut co) {
  __shared__ CandBatch s_batch[8];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  CandBatch& q = s_batch[wib];
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t base = (blockIdx.x * (int64_t)(blockDim.x >> 5) + wib) * 32; base < C.P.n; base += warps * 32) {
    // 1. the batch's 32 patches, one per lane
    int H = 0;
    {
      const int64_t pid = base + lane;
      q.ty[lane] = 0;
      q.pid[lane] = (int)pid;
      const int32_t* w = C.P.win + 6 * pid;
      if (pid < C.P.n && w[0] >= 0) {
        const StructDev& S = C.B.s[C.B.patch_struct[pid]];
        const GridDev& g = S.g;
        const RaySet rs = make_ray_set(C.set, g);
        const double* src = C.P.f64 + (int64_t)NS_PATCH_F64 * pid;
        const double cf = __ldg(src + rs.fd), cl = __ldg(src + rs.ld), r = __ldg(src + kR);
        const int kind0 = C.P.i32[NS_PATCH_I32 * pid];
        const bool skin = ns_has_box(kind0);
        q.cf[lane] = cf;
        q.cl[lane] = cl;
        q.lo_fd[lane] = skin ? __ldg(src + NS_SKIN_LO + rs.fd) : cf - r;
        q.hi_fd[lane] = skin ? __ldg(src + NS_SKIN_HI + rs.fd) : cf + r;
        q.lo_ld[lane] = skin ? __ldg(src + NS_SKIN_LO + rs.ld) : cl - r;
        q.hi_ld[lane] = skin ? __ldg(src + NS_SKIN_HI + rs.ld) : cl + r;
        q.disc[lane] = (!skin || kind0 == NS_SKIN_POINT) ? 1 : 0;
        q.r2[lane] = r * r;
        q.mn_fd[lane] = g.mn[rs.fd];
        q.mn_ld[lane] = g.mn[rs.ld];
        q.side[lane] = g.side;
        q.delta[lane] = rs.delta;
        q.nb[lane] = rs.nb;
        q.rbase[lane] = S.ray_base[C.set];
        q.m0[lane] = w[rs.fd];
        q.m1[lane] = w[3 + rs.fd];
        q.n0[lane] = w[rs.ld];
        const int h = w[3 + rs.ld] - w[rs.ld] + 1;
        H = (w[3 + rs.fd] >= w[rs.fd] && h > 0) ? h : 0;
        const int kind = C.P.i32[NS_PATCH_I32 * pid];
        q.ty[lane] = (kind == NS_EDGE_REG || kind == NS_EDGE_SING) ? 1 : 0;  // skin, triangles: sphere list
      }
      q.gfirst[lane] = 0;
      q.gend[lane] = 0;
    }
    // the batch's pixel rows, patch after patch, are processed 32 at a time
    int hincl = H;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, hincl, o);
      if (lane >= o) hincl += v;
    }
    const int hexcl = hincl - H;
    const int R = __shfl_sync(0xffffffffu, hincl, 31);
    __syncwarp();
    if (R == 0) continue;
    // 2. candidate counts: G = running exclusive prefix of the row counts in batch order; the
    //    lanes holding a patch's first and last rows record G there
    int64_t running = 0;
    for (int rb = 0; rb < R; rb += 32) {
      const int k = rb + lane;
      const int kk = k < R ? k : R - 1;
      const int p = owner_lane(hincl, kk);
      const int row = kk - __shfl_sync(0xffffffffu, hexcl, p);
      const int hp = __shfl_sync(0xffffffffu, H, p);
      int a, cnt = 0;
      if (k < R) cnt = cand_row(q, p, row, &a);
      int cincl = cnt;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, cincl, o);
        if (lane >= o) cincl += v;
      }
      if (k < R && row == 0) q.gfirst[p] = running + (cincl - cnt);
      if (k < R && row == hp - 1) q.gend[p] = running + cincl;
      running += __shfl_sync(0xffffffffu, cincl, 31);
    }
    __syncwarp();
    const int my_total = H > 0 ? (int)(q.gend[lane] - q.gfirst[lane]) : 0;
    // 3. one atomic per candidate list for the whole batch
    const int my_ty = q.ty[lane];
    int inc0 = my_ty == 0 ? my_total : 0, inc1 = my_ty == 1 ? my_total : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int v0 = __shfl_up_sync(0xffffffffu, inc0, o), v1 = __shfl_up_sync(0xffffffffu, inc1, o);
      if (lane >= o) {
        inc0 += v0;
        inc1 += v1;
      }
    }
    const int sum0 = __shfl_sync(0xffffffffu, inc0, 31), sum1 = __shfl_sync(0xffffffffu, inc1, 31);
    unsigned long long b0 = 0, b1 = 0;
    if (lane == 0 && sum0) b0 = atomicAdd(co.count + 0, (unsigned long long)sum0);
    if (lane == 0 && sum1) b1 = atomicAdd(co.count + 1, (unsigned long long)sum1);
    b0 = __shfl_sync(0xffffffffu, b0, 0);
    b1 = __shfl_sync(0xffffffffu, b1, 0);
    if ((int64_t)(b0 + sum0) > co.cap || (int64_t)(b1 + sum1) > co.cap) {
      if (lane == 0) atomicExch(C.out.error_flag, 6);
      __syncwarp();
      continue;
    }
    // a row's candidate j sits at base[p] + G(row) + j in its patch's list
    const int64_t my_slot = my_ty == 0 ? (int64_t)b0 + (inc0 - my_total) : (int64_t)b1 + (inc1 - my_total);
    q.base[lane] = my_slot - q.gfirst[lane];
    __syncwarp();
    // 4. the candidates, rows in batch order, stores coalesced
    running = 0;
    for (int rb = 0; rb < R; rb += 32) {
      const int k = rb + lane;
      const int kk = k < R ? k : R - 1;
      const int p = owner_lane(hincl, kk);
      const int row = kk - __shfl_sync(0xffffffffu, hexcl, p);
      int a = 0, cnt = 0;
      if (k < R) cnt = cand_row(q, p, row, &a);
      int cincl = cnt;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, cincl, o);
        if (lane >= o) cincl += v;
      }
      const int T = __shfl_sync(0xffffffffu, cincl, 31);
      const int cexcl = cincl - cnt;
      for (int kb = 0; kb < T; kb += 32) {
        const int j = kb + lane;
        const int jj = j < T ? j : T - 1;
        const int rr = owner_lane(cincl, jj);
        const int pr = __shfl_sync(0xffffffffu, p, rr), rowr = __shfl_sync(0xffffffffu, row, rr);
        const int ar = __shfl_sync(0xffffffffu, a, rr), er = __shfl_sync(0xffffffffu, cexcl, rr);
        if (j < T) {
          const int m = ar + (j - er);
          const int64_t n = q.n0[pr] + rowr;
          int2* dst = q.ty[pr] ? co.tor : co.sph;
          dst[q.base[pr] + running + j] = make_int2((int)(q.rbase[pr] + n * q.nb[pr] + m), q.pid[pr]);
        }
      }
      running += T;
    }
    __syncwarp();
  }
}

// Branch class of a torus candidate, from the operations of the double-precision path up to the
// resolvent cubic (ray_sphere_axis, torus_coeffs_f64, the head of quartic_f64 and of
// real_cubic_f64, the same operations in the same order): -1 when the path returns no hit there
// (no clipping-sphere hit, or no real quartic root), 1 for the resolvent's arccos branch, 0 for
// the cube-root branch and the rare others.
template <int PN>
__device__ __forceinline__ int torus_class(const double* f, double probe, const double* pa, double ray_dir) {
  constexpr int vc = Ax<PN>::vc;
  double t0, t1;
  if (!ray_sphere_axis<vc>(pa, ray_dir, f, f[kR], &t0, &t1)) return -1;
  double orig1[3] = {pa[0], pa[1], pa[2]};
  orig1[vc] += t0 * ray_dir;
  double b, c, d, e;
  torus_coeffs_f64(f, probe, vc, orig1, &b, &c, &d, &e);
  const double b_2 = 0.5 * b;
  const double b_4 = 0.25 * b;
  const double p = c - 1.5 * (b_2 * b_2);
  const double q = d + b_2 * (b_2 * b_2 - c);
  const double r = e + b_4 * (b_4 * (c - 3.0 * b_4 * b_4) - d);
  const double ff = p * p - 4. * r;
  const double delta =
      4. * ff * (4. * r * (p * p) - p * (q * q) - 16. * (r * r)) + (q * q) * (128. * p * r - 27. * (q * q));
  if (e != 0. && (fabs(p) > 3.E+3 || fabs(r) > 3.E+3 || fabs(q) > 3.E+3 || fabs(delta) > 1.E+14)) return 0;
  if (!(delta < 0. || (delta == 0. && (p >= 0. || ff < 0.))) && !((p < 0. && ff > 0.) || (delta == 0. && p == 0. && r == 0.)))
    return -1;
  // the resolvent cubic x^3 + cb x^2 + cc x + cd
  const double cb = p, cc = 0.25 * (p * p) - r, cd = (-0.125) * (q * q);
  if (fabs(cc) < cb * cb * 1.E-6 && fabs(cd) < fabs(cb) * 1.E-6) return 0;
  if (fabs(cd / cc) < 4.E-4) return 0;
  const double pc = -(1.0 / 3.0) * cb * cb + cc;
  const double qc = (2. / 27.) * cb * cb * cb - (1. / 3.) * cb * cc + cd;
  const double D3p = (1. / 27.) * pc * pc * pc;
  const double D3 = D3p + 0.25 * qc * qc;
  return D3 >= 0. ? 0 : 1;
}

// One thread per torus candidate: its branch class; candidates with no hit are dropped, the
// others appended (warp-aggregated) to the list of their class, so that each solve launch runs
// with the lanes of a warp on one branch of the solver.
template <int PN>
__global__ void __launch_bounds__(256) k_torus_split(TraceCtx C, CandOut co) {
  constexpr int fd = Ax<PN>::fd, ld = Ax<PN>::ld, vc = Ax<PN>::vc;
  const int64_t ncand = co.count[1];
  const int64_t nlim = ncand < co.cap ? ncand : co.cap;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int lane = threadIdx.x & 31;
  const int64_t c0 = blockIdx.x * (int64_t)blockDim.x + (threadIdx.x & ~31);
  for (int64_t cb = c0; cb < nlim; cb += stride) {
    const int64_t c = cb + lane;
    int cls = -1;
    int2 e = make_int2(0, 0);
    if (c < nlim) {
      e = co.tor[c];
      const int64_t rid = e.x, pid = e.y;
      const StructDev& S = C.B.s[C.B.patch_struct[pid]];
      const GridDev& g = S.g;
      const double delta = ray_set_shifted(C.set) ? NS_DELTA - g.hside : 0.0;
      const int64_t nb = g.n[fd];
      const int64_t lr = rid - S.ray_base[C.set];
      const int64_t m = lr % nb, n = lr / nb;
      double pa[3];
      pa[fd] = gcoord(g, fd, m) + delta;
      pa[ld] = gcoord(g, ld, n) + delta;
      pa[vc] = gcoord(g, vc, 0) + delta;
      double f[18];
      const double* src = C.P.f64 + (int64_t)NS_PATCH_F64 * pid;
#pragma unroll
      for (int k = 0; k < 18; k++) f[k] = __ldg(src + k);
      cls = torus_class<PN>(f, C.P.probe, pa, S.ray_dir[vc]);
    }
#pragma unroll
    for (int k = 0; k < 2; k++) {
      const unsigned m = __ballot_sync(0xffffffffu, cls == k);
      if (!m) continue;
      unsigned long long base = 0;
      if (lane == 0) base = atomicAdd(co.tscount + 1 + 2 * k, (unsigned long long)__popc(m));
      base = __shfl_sync(0xffffffffu, base, 0);
      if (cls == k) {
        const unsigned long long slot = base + __popc(m & ((1u << lane) - 1u));
        (k == 0 ? co.tsa : co.tsb)[slot] = e;
      }
    }
  }
}

template <int PN>
void launch_isect(const TraceCtx& C, const CandOut& co, const HitStore& hs, int precision, const TuneParams& tp,
                  cudaStream_t s) {
  const int ig = sm_count() * tp.isect_bpsm, it = tp.isect_threads;
  const bool ses = C.P.kind_mask & kSesKinds, skin = C.P.kind_mask & kBoxKinds;
  // the torus candidates, split by resolvent branch into two lists solved one after the other
  const bool split = tp.torus_split && co.tsa && co.tsb && co.tscount;
  CandOut ca = co, cb = co;
  if (split) {
    k_torus_split<PN><<<ig, 256, 0, s>>>(C, co);
    ca.tor = co.tsa;
    ca.count = co.tscount;
    cb.tor = co.tsb;
    cb.count = co.tscount + 2;
  }
  if (precision == 1) {
    if (ses) {
      launch_isect_mixed_sphere<PN>(C, co, hs, tp, s);
      launch_isect_mixed_torus<PN>(C, ca, hs, tp, s);
      if (split) launch_isect_mixed_torus<PN>(C, cb, hs, tp, s);
    }
    if (skin) launch_isect_quad_mixed<PN>(C, co, hs, tp, s);
    // the deferred candidates, in double precision (few: a small grid)
    const CandOut dco{co.dsph, co.dtor, co.dcap, co.dcount, nullptr, nullptr, 0, nullptr};
    if (ses) {
      k_isect<PN, false><<<sm_count(), 256, 0, s>>>(C, dco, hs);
      k_isect<PN, true><<<sm_count(), 256, 0, s>>>(C, dco, hs);
    }
    if (skin) k_isect_quad<PN><<<sm_count(), 256, 0, s>>>(C, dco, hs);
  } else {
    if (ses) {
      k_isect<PN, false><<<ig, it, 0, s>>>(C, co, hs);
      k_isect<PN, true><<<ig, it, 0, s>>>(C, ca, hs);
      if (split) k_isect<PN, true><<<ig, it, 0, s>>>(C, cb, hs);
    }
    if (skin) k_isect_quad<PN><<<ig, it, 0, s>>>(C, co, hs);
  }
}

// One CTA per 32x4 ray tile: loads, sorts and pairs the hits of its rays and performs the
// interval fill (status runs, insideness bits, pair store, volume).
// kGrad: the hits carry their patches (sorted along), and every interval end adds its term of
// d volume / d patch parameters; the stored pairs keep their patches for the area adjoint.
template <bool kGrad>
__global__ void __launch_bounds__(kTraceThreads, 6) k_fill(TraceCtx C, HitStore hs) {
  constexpr int kThreads = kTraceThreads;
  const int panel = ray_set_panel(C.set);
  const int64_t tile = blockIdx.x;
  const StructDev& S = C.B.s[C.B.tile_struct[panel][tile]];
  const GridDev g = S.g;
  const RaySet rs = make_ray_set(C.set, g);
  uint32_t* const bits = C.out.bits + S.word_base;
  const int64_t nwords = S.nwords;
  __shared__ double s_hit[kHitCap * kThreads];
  // gradient mode: each hit's slot in the hit store (its patch is read from there when needed),
  // one byte per hit to keep the shared-memory footprint and so the occupancy up
  __shared__ uint8_t s_slot[kGrad ? kHitCap * kThreads : 1];
  const int64_t ntm = (rs.nb + kTileM - 1) / kTileM;
  const int64_t lt = tile - S.tile_base[panel];
  const int64_t tm = lt % ntm, tn = lt / ntm;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t m = tm * kTileM + lane;
  const int64_t n = tn * kTileN + warp;
  const bool valid = (m < rs.nb) && (n < rs.na);
  const int tid = threadIdx.x;
  double* col = s_hit + tid;
  const int64_t lrid = n * rs.nb + m;
  const int64_t rid = S.ray_base[C.set] + lrid;
  int hc = valid ? hs.cnt[rid] : 0;
  bool ovf = hc > kHitCap;
  int nh = ovf ? 0 : hc;
  uint8_t* pcol = kGrad ? s_slot + tid : nullptr;
  for (int i = 0; i < nh; i++) col[i * kThreads] = hs.t[(int64_t)i * hs.nrays + rid];
  if (kGrad)
    for (int i = 0; i < nh; i++) pcol[i * kThreads] = (uint8_t)i;
  for (int i = 1; i < nh; i++) {
    double v = col[i * kThreads];
    uint8_t pv = kGrad ? pcol[i * kThreads] : 0;
    int j = i;
    while (j > 0 && col[(j - 1) * kThreads] > v) {
      col[j * kThreads] = col[(j - 1) * kThreads];
      if (kGrad) pcol[j * kThreads] = pcol[(j - 1) * kThreads];
      j--;
    }
    col[j * kThreads] = v;
    if (kGrad) pcol[j * kThreads] = pv;
  }
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
  const bool mc = ray_set_shifted(rs.set);
  double pa_vc, dirl;
  if (rs.set == 0) {
    pa_vc = gcoord(g, 0, 0);
    dirl = gcoord(g, 0, g.n[0] - 1) - pa_vc;
  } else {
    pa_vc = gcoord(g, rs.vc, 0) + rs.delta;
    double pb = gcoord(g, rs.vc, g.n[rs.vc] - 1) + rs.delta;
    dirl = pb - pa_vc;
  }
  double vol = 0.0;
  int np = 0;
  const auto slot_pid = [&](uint8_t sl) { return hs.pid[(int64_t)sl * hs.nrays + rid]; };
  if (kGrad && C.out.gvol) {
    // d volume / d patch parameters, interval end by interval end (the pairing rule of
    // make_pairs), summed over runs of lanes on the same patch before the atomics
    const double W = S.A * C.out.grad_scale;
    __syncwarp();  // the lanes read each other's sorted hit columns below
    const int nhw = (valid && !ovf && nh > 0 && (nh & 1) == 0) ? nh : 0;
    const int maxn = (int)__reduce_max_sync(0xffffffffu, (unsigned)nhw);
    // The warp's interval ends, 32 at a time: end q of every ray that has one (level q), levels in
    // order, so that neighbouring lanes hold neighbouring rays (which mostly hit the same patch).
    // Lane q keeps the ray mask of level q.
    unsigned lvl_mask = 0;
    for (int q = 0; q < maxn; q++) {
      const unsigned mq = __ballot_sync(0xffffffffu, nhw > q);
      if (lane == q) lvl_mask = mq;
    }
    const int lvl_size = __popc(lvl_mask);
    int lincl = lvl_size;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, lincl, o);
      if (lane >= o) lincl += v;
    }
    const int nends = __shfl_sync(0xffffffffu, lincl, 31);
    for (int kb = 0; kb < nends; kb += 32) {
      const int k = kb + lane;
      const int kk = k < nends ? k : nends - 1;
      int q = 0;
#pragma unroll
      for (int step = 16; step; step >>= 1) {
        const int x = __shfl_sync(0xffffffffu, lincl, q + step - 1);
        if (x <= kk) q += step;
      }
      const int idx = kk - __shfl_sync(0xffffffffu, lincl - lvl_size, q);
      unsigned mq = __shfl_sync(0xffffffffu, lvl_mask, q);
      for (int c2 = 0; c2 < idx; c2++) mq &= mq - 1;
      const int r = __ffs(mq) - 1;  // the ray (lane) of this end
      const int64_t rid_r = __shfl_sync(0xffffffffu, rid, r);
      double gk[NS_GRAD_PER_PATCH];
      int32_t pid = -1;
      if (k < nends) {
        const double* cr = s_hit + warp * 32 + r;
        const double t1 = cr[(q & ~1) * kThreads], t2 = cr[(q | 1) * kThreads];
        if (fabs(t2 - t1) >= NS_EPS_INT) {
          const uint8_t sl = s_slot[(q * kThreads) + warp * 32 + r];
          pid = hs.pid[(int64_t)sl * hs.nrays + rid_r];
          double x[3];
          x[rs.fd] = gcoord(g, rs.fd, tm * kTileM + r) + rs.delta;
          x[rs.ld] = gcoord(g, rs.ld, n) + rs.delta;
          x[rs.vc] = pa_vc + dirl * ((q & 1) ? t2 : t1);
          if (hit_grad(C.P.f64 + (int64_t)NS_PATCH_F64 * pid, C.P.i32[NS_PATCH_I32 * pid], C.P.probe, x, rs.vc, gk)) {
            const double w = (q & 1) ? W : -W;
#pragma unroll
            for (int c3 = 0; c3 < NS_GRAD_PER_PATCH; c3++) gk[c3] *= w;
          } else {
            pid = -1;
          }
        }
      }
      if (pid < 0)
#pragma unroll
        for (int c3 = 0; c3 < NS_GRAD_PER_PATCH; c3++) gk[c3] = 0.0;
      warp_add_grad(pid, gk, C.out.gvol);
    }
  }
  if (kGrad) {
    // the hits' patches follow their pairs (gradients, analytic normals)
    if (valid && !ovf)
      np = make_pairs(col, kThreads, nh, pa_vc, dirl, g.mn[rs.vc], g.scale, mc, &vol, pcol, (GradCtx*)nullptr,
                      slot_pid);
  } else {
    if (valid && !ovf) np = make_pairs(col, kThreads, nh, pa_vc, dirl, g.mn[rs.vc], g.scale, mc, &vol);
  }
  if (valid && !ovf) C.out.vol_ray[rid] = vol;
  __syncwarp();
  const int64_t NX = g.n[0], NY = g.n[1];
  if (rs.set >= 4) {
    // epsilon-map node rays of panels 1 and 2
    if (valid && !ovf && C.out.epsmap)
      for (int q = 0; q < np; q++)
        eps_fill(g, rs, m, n, col[(2 * q) * kThreads], col[(2 * q + 1) * kThreads], C.out.epsmap, C.out.eps_inside);
    return;
  }
  if (!mc) {
    // status row (., j = m, k = n): runs of inside nodes
    int nr = 0;
    if (valid && !ovf)
      for (int q = 0; q < np; q++) {
        if (C.out.epsmap)
          eps_fill(g, rs, m, n, col[(2 * q) * kThreads], col[(2 * q + 1) * kThreads], C.out.epsmap, C.out.eps_inside);
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
      int64_t ord = S.mc_base + rs.ordinal_base + lrid;
      if (off >= 0) {
        for (int q = 0; q < np; q++) {
          C.out.pairs[2 * (off + q)] = col[(2 * q) * kThreads];
          C.out.pairs[2 * (off + q) + 1] = col[(2 * q + 1) * kThreads];
          if (kGrad)
            C.out.pair_pid[off + q] = make_int2(slot_pid(pcol[(2 * q) * kThreads]), slot_pid(pcol[(2 * q + 1) * kThreads]));
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
    // row bits (i, j = m, k = n), i in (a, b]: every lane clears the runs of its own row
    if (valid && !ovf) {
      const int64_t f0 = (n * NY + m) * NX;
      const int64_t maxb = nwords * 32 - 1;
      for (int q = 0; q < np; q++) {
        const int64_t a = (int64_t)rintp((col[(2 * q) * kThreads] - vmin) * g.scale);
        const int64_t b = (int64_t)rintp((col[(2 * q + 1) * kThreads] - vmin) * g.scale);
        int64_t lo = f0 + a + 1, hi = f0 + b;
        if (lo < 0) lo = 0;
        if (hi > maxb) hi = maxb;
        for (int64_t w = lo >> 5; w <= (hi >> 5) && hi >= lo; w++) {
          const int64_t wl = w << 5;
          const int s0 = (int)(lo > wl ? lo - wl : 0);
          const int s1 = (int)(hi < wl + 31 ? hi - wl : 31);
          const uint32_t mask = (s1 - s0 == 31) ? 0xffffffffu : (((1u << (s1 - s0 + 1)) - 1u) << s0);
          atomicAnd(bits + w, ~mask);
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
  // 32 positions at a time: every lane builds the 32-bit membership word of its ray over
  // [v0, v0 + 31] from its intervals, 32 ballots transpose the words so that lane l holds the mask
  // of the 32 rays at position v0 + l, and the lanes clear their rows' bits in parallel
  int q = 0;
  int64_t qa = 0, qb = -1;
  if (np > 0) {
    qa = (int64_t)rintp((col[0] - vmin) * g.scale);
    qb = (int64_t)rintp((col[kThreads] - vmin) * g.scale);
  }
  const int64_t m0 = tm * kTileM;
  for (int64_t v0 = vlo; v0 <= vhi; v0 += 32) {
    const int64_t v1 = v0 + 31;
    unsigned mem = 0;
    while (q < np && qa < v1) {
      // positions qa < v <= qb of the current interval that fall in [v0, v1]
      const int64_t lo = qa + 1 > v0 ? qa + 1 : v0, hi = qb < v1 ? qb : v1;
      if (lo <= hi) {
        const int s0 = (int)(lo - v0), s1 = (int)(hi - v0);
        mem |= (s1 - s0 == 31) ? 0xffffffffu : (((1u << (s1 - s0 + 1)) - 1u) << s0);
      }
      if (qb > v1) break;  // the interval continues in the next window
      q++;
      if (q < np) {
        qa = (int64_t)rintp((col[(2 * q) * kThreads] - vmin) * g.scale);
        qb = (int64_t)rintp((col[(2 * q + 1) * kThreads] - vmin) * g.scale);
      }
    }
    unsigned mask = 0;
#pragma unroll
    for (int b = 0; b < 32; b++) {
      const unsigned mb = __ballot_sync(0xffffffffu, (mem >> b) & 1u);
      if (lane == b) mask = mb;
    }
    const int64_t v = v0 + lane;
    if (mask && v <= vhi) {
      const int64_t f0 = (rs.panel == 1) ? ((v * NY + n) * NX + m0) : ((n * NY + v) * NX + m0);
      if (f0 >= 0) {
        const int64_t w = f0 >> 5;
        const int sh = (int)(f0 & 31);
        if (w < nwords) atomicAnd(bits + w, ~(mask << sh));
        if (sh && w + 1 < nwords) atomicAnd(bits + w + 1, ~(mask >> (32 - sh)));
      }
    }
  }
}

// One thread per overflow ray: the same candidate tests with the hits kept in a global column.
__global__ void k_trace_overflow(TraceCtx C, const int64_t* __restrict__ tile_off, const int32_t* __restrict__ tile_list,
                                 int n_ovf, double* scratch, int32_t* pscratch) {
  int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n_ovf) return;
  int64_t rid = C.out.ovf_rays[idx];
  const StructDev& S = C.B.s[find_struct(C.B.ray_base[C.set], C.B.n, rid)];
  const GridDev g = S.g;
  const RaySet rs = make_ray_set(C.set, g);
  uint32_t* const bits = C.out.bits + S.word_base;
  const int64_t nwords = S.nwords;
  const int64_t lrid = rid - S.ray_base[C.set];
  int64_t m = lrid % rs.nb, n = lrid / rs.nb;
  int64_t ntm = (rs.nb + kTileM - 1) / kTileM;
  int64_t tile = S.tile_base[rs.panel] + (n / kTileN) * ntm + m / kTileM;
  double* col = scratch + (int64_t)idx * kOverflowCap;
  int32_t* pcol = pscratch ? pscratch + (int64_t)idx * kOverflowCap : nullptr;
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
    const double tri_dir = (gcoord(g, rs.vc, g.n[rs.vc] - 1) + rs.delta) - pa[rs.vc];
    int k = ray_patch_f64(f, ir[0], ir[1], ir[2], C.P, rs, pa, dir, ray_dir, S.box_dir[rs.vc], tri_dir, t);
    for (int i = 0; i < k; i++) {
      if (nh >= kOverflowCap) {
        atomicExch(C.out.error_flag, 4);
        return;
      }
      int pos = nh++;
      while (pos > 0 && col[pos - 1] > t[i]) {
        col[pos] = col[pos - 1];
        if (pcol) pcol[pos] = pcol[pos - 1];
        pos--;
      }
      col[pos] = t[i];
      if (pcol) pcol[pos] = (int32_t)pid;
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
  const bool mc = ray_set_shifted(rs.set);
  double pa_vc, dirl;
  if (rs.set == 0) {
    pa_vc = gcoord(g, 0, 0);
    dirl = gcoord(g, 0, g.n[0] - 1) - pa_vc;
  } else {
    pa_vc = gcoord(g, rs.vc, 0) + rs.delta;
    dirl = (gcoord(g, rs.vc, g.n[rs.vc] - 1) + rs.delta) - pa_vc;
  }
  double vol = 0.0;
  GradCtx gc;
  gc.f64 = C.P.f64;
  gc.i32 = C.P.i32;
  gc.probe = C.P.probe;
  gc.w = S.A * C.out.grad_scale;
  gc.x[rs.fd] = pa[rs.fd];
  gc.x[rs.ld] = pa[rs.ld];
  gc.x[rs.vc] = 0.0;
  gc.vc = rs.vc;
  gc.gvol = C.out.gvol;
  int np = make_pairs(col, 1, nh, pa_vc, dirl, g.mn[rs.vc], g.scale, mc, &vol, pcol, (pcol && gc.gvol) ? &gc : nullptr);
  C.out.vol_ray[rid] = vol;
  const int64_t NX = g.n[0], NY = g.n[1];
  if (rs.set >= 4) {
    if (C.out.epsmap)
      for (int q = 0; q < np; q++) eps_fill(g, rs, m, n, col[2 * q], col[2 * q + 1], C.out.epsmap, C.out.eps_inside);
    return;
  }
  if (!mc) {
    int nr = 0;
    for (int q = 0; q < np; q++) {
      if (C.out.epsmap) eps_fill(g, rs, m, n, col[2 * q], col[2 * q + 1], C.out.epsmap, C.out.eps_inside);
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
  int64_t ord = S.mc_base + rs.ordinal_base + lrid;
  unsigned long long off = np ? atomicAdd(C.out.pair_cursor, (unsigned long long)np) : 0;
  if ((int64_t)off + np <= C.out.pair_cap) {
    for (int q = 0; q < np; q++) {
      C.out.pairs[2 * (off + q)] = col[2 * q];
      C.out.pairs[2 * (off + q) + 1] = col[2 * q + 1];
      if (pcol) C.out.pair_pid[off + q] = make_int2(pcol[2 * q], pcol[2 * q + 1]);
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
      clear_bits_range(bits, nwords, f0 + a + 1, f0 + b);
    } else {
      for (int64_t v = a + 1; v <= b; v++) {
        int64_t f = (rs.panel == 1) ? ((v * NY + n) * NX + m) : ((n * NY + v) * NX + m);
        clear_bits_range(bits, nwords, f, f);
      }
    }
  }
}

}  // namespace

cudaError_t launch_windows(const PatchDev& P, int32_t* win, const BatchDev& B, cudaStream_t s) {
  if (P.n == 0) return cudaSuccess;
  k_windows<<<(unsigned)((P.n + 255) / 256), 256, 0, s>>>(P, win, B);
  return cudaGetLastError();
}

cudaError_t launch_pool32(const PatchDev& P, float4* pool32, float4* quad32, double4* quadl, cudaStream_t s) {
  if (P.n == 0) return cudaSuccess;
  k_pool32<<<(unsigned)((P.n + 255) / 256), 256, 0, s>>>(P, pool32, quad32, quadl);
  return cudaGetLastError();
}

cudaError_t launch_kind_mask(const PatchDev& P, int* mask, cudaStream_t s) {
  if (P.n == 0) return cudaSuccess;
  k_kind_mask<<<(unsigned)((P.n + 255) / 256), 256, 0, s>>>(P, mask);
  return cudaGetLastError();
}

cudaError_t launch_bin_count(const PatchDev& P, const BatchDev& B, int set, int32_t* tile_cnt,
                             unsigned long long* area, cudaStream_t s) {
  if (P.n == 0) return cudaSuccess;
  k_bin<<<(unsigned)((P.n + 255) / 256), 256, 0, s>>>(P, B, set, tile_cnt, nullptr, nullptr, nullptr, area);
  return cudaGetLastError();
}

cudaError_t launch_bin_fill(const PatchDev& P, const BatchDev& B, int set, const int64_t* tile_off,
                            int32_t* tile_cursor, int32_t* tile_list, cudaStream_t s) {
  if (P.n == 0) return cudaSuccess;
  k_bin<<<(unsigned)((P.n + 255) / 256), 256, 0, s>>>(P, B, set, nullptr, tile_off, tile_cursor, tile_list, nullptr);
  return cudaGetLastError();
}

cudaError_t launch_trace(const PatchDev& P, const BatchDev& B, int set, int64_t ntiles, const TraceOut& out,
                         const CandOut& co, const HitStore& hs, int precision, const TuneParams& tp, cudaStream_t s,
                         cudaEvent_t* ev) {
  if (ntiles <= 0) return cudaSuccess;
  TraceCtx C{P, B, set, out};
  const int panel = ray_set_panel(set);
  if (ev) cudaEventRecord(ev[0], s);
  if (P.n > 0) {
    const int wpb = tp.cand_threads / 32;
    int64_t blocks = (P.n + 32 * wpb - 1) / (32 * wpb);
    if (blocks > (int64_t)sm_count() * 64) blocks = (int64_t)sm_count() * 64;
    k_cand<<<(unsigned)blocks, tp.cand_threads, 0, s>>>(C, co);
  }
  if (ev) cudaEventRecord(ev[1], s);
  if (panel == 0) launch_isect<0>(C, co, hs, precision, tp, s);
  else if (panel == 1) launch_isect<1>(C, co, hs, precision, tp, s);
  else launch_isect<2>(C, co, hs, precision, tp, s);
  if (ev) cudaEventRecord(ev[2], s);
  if (hs.pid) k_fill<true><<<(unsigned)ntiles, kTraceThreads, 0, s>>>(C, hs);
  else k_fill<false><<<(unsigned)ntiles, kTraceThreads, 0, s>>>(C, hs);
  if (ev) cudaEventRecord(ev[3], s);
  return cudaGetLastError();
}

cudaError_t launch_trace_overflow(const PatchDev& P, const BatchDev& B, int set, const int64_t* tile_off,
                                  const int32_t* tile_list, const TraceOut& out, int n_ovf, double* scratch,
                                  int32_t* pscratch, int precision, cudaStream_t s) {
  (void)precision;
  if (n_ovf <= 0) return cudaSuccess;
  TraceCtx C{P, B, set, out};
  k_trace_overflow<<<(n_ovf + 63) / 64, 64, 0, s>>>(C, tile_off, tile_list, n_ovf, scratch, pscratch);
  return cudaGetLastError();
}

}  // namespace nsg
