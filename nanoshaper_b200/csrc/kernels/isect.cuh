// Ray-patch intersection kernels of the tracer, shared by two translation units:
//  * trace.cu compiles them without contraction of products and sums (--fmad=false), so the
//    double-precision path (k_isect<panel, torus, false>) rounds every operation as the host
//    restatement does;
//  * trace_mixed.cu compiles the mixed-precision instantiations (k_isect<panel, torus, true>)
//    with fused multiply-adds, which cut the double-precision instruction count of the torus
//    quartic; that path is held to a tolerance, not to bit equality, and its near-degenerate
//    decisions are deferred to the double-precision kernel by guards far wider than one rounding.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "pipeline.h"
#include "ray_math.cuh"
#include "ray_math_mixed.cuh"

namespace nsg {

struct TraceCtx {
  PatchDev P;
  BatchDev B;
  int set;
  TraceOut out;
};

// Mixed-precision intersection launches of one panel: the sphere candidate list of co
// (trace_mixed.cu) and the torus list (trace_mixed_torus.cu, built without fused multiply-adds),
// with the deferred candidates appended to co's deferred lists.
template <int PN>
void launch_isect_mixed_sphere(const TraceCtx& C, const CandOut& co, const HitStore& hs, const TuneParams& tp,
                               cudaStream_t s);
template <int PN>
void launch_isect_mixed_torus(const TraceCtx& C, const CandOut& co, const HitStore& hs, const TuneParams& tp,
                              cudaStream_t s);
// Mixed-precision skin cell launch of one panel (trace_mixed.cu).
template <int PN>
void launch_isect_quad_mixed(const TraceCtx& C, const CandOut& co, const HitStore& hs, const TuneParams& tp,
                             cudaStream_t s);

namespace {

// Node i of grid axis d.
__device__ __forceinline__ double gcoord(const GridDev& g, int d, int64_t i) { return g.mn[d] + (double)i * g.side; }

// Axes of a panel as compile-time constants: pixel axes (fd, ld) and ray axis vc.
template <int P>
struct Ax {
  static constexpr int fd = P == 0 ? 1 : 0;
  static constexpr int ld = P == 1 ? 1 : 2;
  static constexpr int vc = P == 0 ? 0 : (P == 1 ? 2 : 1);
};

// raySphere for a ray along axis VC with direction length d: the dot products of the generic
// routine reduce to single products (the other terms are zero), the rest keeps its operation order.
template <int VC>
__device__ __forceinline__ bool ray_sphere_axis(const double* orig, double d, const double* c, double r, double* t1,
                                                double* t2) {
  double temp0 = orig[0] - c[0], temp1 = orig[1] - c[1], temp2 = orig[2] - c[2];
  double tv = VC == 0 ? temp0 : (VC == 1 ? temp1 : temp2);
  double A = d * d;
  double B = tv * d;
  double C = temp0 * temp0 + temp1 * temp1 + temp2 * temp2 - r * r;
  double det = B * B - A * C;
  if (det < 0.) return false;
  det = sqrt(det);
  double a = (-B - det) / A;
  double b = (-B + det) / A;
  if (b < a) { double tt = a; a = b; b = tt; }
  *t1 = a;
  *t2 = b;
  return true;
}

template <int P, bool kTorus>
__device__ __forceinline__ int intersect_f64_p(const double* f, int kind, int first, int cnt, const PatchDev& Pd,
                                               const double* pa, double ray_dir, double* t) {
  constexpr int vc = Ax<P>::vc;
  if (!ray_sphere_axis<vc>(pa, ray_dir, f, f[kR], &t[0], &t[1])) return 0;
  int numInt = 2;
  if (kTorus) numInt = ray_torus_f64(f, Pd.probe, vc, pa, ray_dir, t);
  int out = 0;
  for (int i = 0; i < numInt; i++) {
    double ip[3] = {pa[0], pa[1], pa[2]};
    ip[vc] += t[i] * ray_dir;
    if (feasible_f64(f, kind, first, cnt, Pd.pool, Pd.flag, ip)) t[out++] = t[i];
  }
  return out;
}

// Result of the mixed-precision test for a candidate it cannot decide: the candidate goes to a
// deferred list that a double-precision pass takes afterwards, so that the mixed kernel's warps
// never wait on a double-precision path taken by one lane.
constexpr int kDefer = -1;

// Mixed-precision intersection of a candidate (see ray_math_mixed.cuh): the number of feasible
// hits, or kDefer when the single-precision bracket cannot decide the candidate.
template <int PN, bool kTorus>
__device__ __forceinline__ int intersect_mixed(const double* f, int kind, int first, int cnt, const PatchDev& P,
                                               const double* pa, double ray_dir, double inv_dir, double* t,
                                               unsigned long long* ctr) {
  constexpr int fd = Ax<PN>::fd, ld = Ax<PN>::ld, vc = Ax<PN>::vc;
  const double r = f[kR];
  const double dx64 = pa[fd] - f[fd], dy64 = pa[ld] - f[ld];
  const float dxf = (float)dx64, dyf = (float)dy64, rf = (float)r;
  float disc = rf * rf - dxf * dxf - dyf * dyf;
  if (disc < kDiscTol) {
    if (ctr) atomicAdd(ctr + kCntFbSphere, 1ull);
    return kDefer;
  }
  double xs[4], ts[4];
  int nx = 0;
  const double cv = f[vc];
  if (kTorus) {
    // the double-precision path's clipping-sphere entry and quartic, operation for operation (the
    // torus kernels are built without fused multiply-adds, trace_mixed_torus.cu), so that an
    // undeferred root is the FP64 path's to the bit: the reference's solver is ill-conditioned
    // for some rays (its resolvent approximations), where a different rounding moves a root by
    // up to 1e-4 A
    double tsph[2];
    if (!ray_sphere_axis<vc>(pa, ray_dir, f, r, &tsph[0], &tsph[1])) return 0;
    const double t0 = tsph[0];
    double orig1[3] = {pa[0], pa[1], pa[2]};
    orig1[vc] += t0 * ray_dir;
    double B, C, D, E;
    torus_coeffs_f64(f, P.probe, vc, orig1, &B, &C, &D, &E);
    double roots[4];
    int nr = quartic_guarded(roots, B, C, D, E);
    if (nr < 0) {
      if (ctr) atomicAdd(ctr + kCntFbQuartic, 1ull);
      return kDefer;
    }
    const double r2 = r * r;
    for (int i = 0; i < nr; i++) {
      double root = roots[i];
      if (fabs(root) < 1e-9) {
        if (ctr) atomicAdd(ctr + kCntFbRoot, 1ull);
        return kDefer;
      }
      if (root < 0) continue;
      double point[3] = {orig1[0], orig1[1], orig1[2]};
      point[vc] += root;
      double dd = (f[0] - point[0]) * (f[0] - point[0]) + (f[1] - point[1]) * (f[1] - point[1]) +
                  (f[2] - point[2]) * (f[2] - point[2]);
      if (fabs(dd - r2) < 1e-9) {
        if (ctr) atomicAdd(ctr + kCntFbRoot, 1ull);
        return kDefer;
      }
      if (dd < r2) {
        ts[nx] = t0 + root / ray_dir;
        xs[nx] = pa[vc] + ts[nx] * ray_dir;
        nx++;
      }
    }
  } else {
    // the chord half-length in FP32, one FP64 Newton correction against the FP64 discriminant
    const float s32 = sqrtf(disc);
    const double disc64 = r * r - dx64 * dx64 - dy64 * dy64;
    double sd = (double)s32;
    sd = sd + (disc64 - sd * sd) * (double)(0.5f / s32);
    xs[0] = cv - sd;
    xs[1] = cv + sd;
    ts[0] = (xs[0] - pa[vc]) * inv_dir;
    ts[1] = (xs[1] - pa[vc]) * inv_dir;
    nx = 2;
  }
  int out = 0;
  for (int i = 0; i < nx; i++) {
    float pl[3];
    pl[fd] = dxf;
    pl[ld] = dyf;
    pl[vc] = (float)(xs[i] - cv);
    double p64[3];
    p64[fd] = pa[fd];
    p64[ld] = pa[ld];
    p64[vc] = xs[i];
    if (feasible_mixed<kTorus>(f, kind, first, cnt, P.pool, P.pool32, P.flag, pl, p64)) t[out++] = ts[i];
  }
  return out;
}

// One thread per candidate pair of one type: intersection, feasibility, hit filing.
template <int PN, bool kTorus, bool kMixed>
__device__ __forceinline__ void isect_body(const TraceCtx& C, const CandOut& co, const HitStore& hs) {
  constexpr int fd = Ax<PN>::fd, ld = Ax<PN>::ld, vc = Ax<PN>::vc;
  const int64_t ncand = *(co.count + (kTorus ? 1 : 0));
  const int2* list = kTorus ? co.tor : co.sph;
  const int64_t nlim = ncand < co.cap ? ncand : co.cap;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  // the next candidate of this thread is loaded one iteration ahead
  int2 e_next = c < nlim ? list[c] : make_int2(0, 0);
  for (; c < nlim; c += stride) {
    const int2 e = e_next;
    if (c + stride < nlim) e_next = list[c + stride];
    const int64_t rid = e.x, pid = e.y;
    const StructDev& S = C.B.s[C.B.patch_struct[pid]];
    const GridDev& g = S.g;
    const double delta = ray_set_shifted(C.set) ? NS_DELTA - g.hside : 0.0;
    const double ray_dir = S.ray_dir[vc];
    const double inv_dir = S.inv_dir[vc];
    const int64_t nb = g.n[fd];
    const int64_t lr = rid - S.ray_base[C.set];
    const int64_t m = lr % nb, n = lr / nb;
    double pa[3];
    pa[fd] = gcoord(g, fd, m) + delta;
    pa[ld] = gcoord(g, ld, n) + delta;
    pa[vc] = gcoord(g, vc, 0) + delta;
    double f[NS_PATCH_F64];
    const double* src = C.P.f64 + (int64_t)NS_PATCH_F64 * pid;
    constexpr int nf = kTorus ? 18 : 4;
#pragma unroll
    for (int k = 0; k < nf; k++) f[k] = __ldg(src + k);
    const int32_t* ir = C.P.i32 + NS_PATCH_I32 * pid;
    const int kind = ir[0], first = ir[1], cnt = ir[2];
    if (!kTorus && ns_has_box(kind)) continue;  // skin cells and triangles share the list (k_isect_quad)
    double t[4];
    int k;
    if (kMixed) {
      k = intersect_mixed<PN, kTorus>(f, kind, first, cnt, C.P, pa, ray_dir, inv_dir, t, C.out.counters);
      // warp-aggregated append of the deferred candidates
      const bool defer = k == kDefer;
      const unsigned am = __activemask();
      const unsigned dm = __ballot_sync(am, defer);
      if (dm) {
        const int lane = threadIdx.x & 31;
        const int leader = __ffs(dm) - 1;
        unsigned long long base = 0;
        if (lane == leader) base = atomicAdd(co.dcount + (kTorus ? 1 : 0), (unsigned long long)__popc(dm));
        base = __shfl_sync(am, base, leader);
        if (defer) {
          unsigned long long slot = base + __popc(dm & ((1u << lane) - 1u));
          if ((int64_t)slot < co.dcap) (kTorus ? co.dtor : co.dsph)[slot] = e;
          else atomicExch(C.out.error_flag, 7);
        }
      }
    } else {
      k = intersect_f64_p<PN, kTorus>(f, kind, first, cnt, C.P, pa, ray_dir, t);
    }
    if (k <= 0) continue;
    int pos = atomicAdd(hs.cnt + rid, k);
    for (int i = 0; i < k; i++)
      if (pos + i < kHitCap) {
        hs.t[(int64_t)(pos + i) * hs.nrays + rid] = t[i];
        if (hs.pid) hs.pid[(int64_t)(pos + i) * hs.nrays + rid] = (int32_t)pid;
      }
  }
}

// ---- skin cells: ray-quadric tests inside the mixed cells ----

// Double-precision skin cell test (getPatchIntersectionData of the skin, src/SkinSurface.cpp:
// 3422-3760): the reference's rayQuadricIntersection along the panel's axis from the ray origin
// pa (pa[vc] = min + delta), the cell's plane tests at pa + t e_vc, and the hit stored as
// t / (max - min) of the axis.
template <int PN>
__device__ __forceinline__ int intersect_quadric_f64(const double* f, int first, int cnt, const PatchDev& Pd,
                                                     const double* pa, double box_dir, double* t) {
  constexpr int vc = Ax<PN>::vc;
  double tt[2];
  if (!ray_quadric_f64<vc>(f + NS_SKIN_Q, pa, tt)) return 0;
  int out = 0;
  for (int i = 0; i < 2; i++) {
    double ip[3] = {pa[0], pa[1], pa[2]};
    ip[vc] += tt[i];
    if (feasible_skin_f64(Pd.pool, first, cnt, ip)) t[out++] = tt[i] / box_dir;
  }
  return out;
}

// FP32 tolerance of the mixed-precision quadric: a discriminant within kQuadRel of the size of its
// terms leaves the candidate to the double-precision pass.
constexpr float kQuadRel = 1e-4f;

// Mixed-precision skin cell test: along the ray the quadric is a s^2 + 2 b s + c in s = x_vc -
// c_vc (c the cell's local origin), with b and c from the transverse offsets of the ray to c, all
// small numbers; the discriminant and roots are taken in FP32 (numerically stable form), each
// root is polished by one Newton step against the FP64 local quadric, and the plane tests run in
// FP32 on local coordinates with FP64 re-evaluation near zero.  Near-tangent rays (discriminant
// within rounding of zero) are deferred to the double-precision kernel.
template <int PN>
__device__ __forceinline__ int intersect_quadric_mixed(const double* f, int first, int cnt, const PatchDev& P,
                                                       int64_t pid, const double* pa, double box_dir, double* t,
                                                       unsigned long long* ctr) {
  constexpr int fd = Ax<PN>::fd, ld = Ax<PN>::ld, vc = Ax<PN>::vc;
  // quadric coefficients about the local origin: A (symmetric), bl = A c + b, cl = f(c)
  const float4 q0 = P.quad32[3 * pid], q1 = P.quad32[3 * pid + 1], q2 = P.quad32[3 * pid + 2];
  const double4 ql = P.quadl[pid];
  const float A00 = q0.x, A11 = q0.y, A22 = q0.z, A01 = q0.w, A12 = q1.x, A02 = q1.y;
  const float Af[3][3] = {{A00, A01, A02}, {A01, A11, A12}, {A02, A12, A22}};
  const float blf[3] = {q1.z, q1.w, q2.x};
  const double* Q = f + NS_SKIN_Q;
  const double A64[3][3] = {{Q[0], Q[4], Q[7]}, {Q[4], Q[1], Q[5]}, {Q[7], Q[5], Q[2]}};
  const double bl64[3] = {ql.x, ql.y, ql.z};
  const double a64 = A64[vc][vc];
  if (a64 == 0) return 0;
  const double u64f = pa[fd] - f[fd], u64l = pa[ld] - f[ld];
  const float uf = (float)u64f, ul = (float)u64l;
  const float a = Af[vc][vc];
  const float b = (Af[vc][fd] * uf + Af[vc][ld] * ul) + blf[vc];
  const float c = (Af[fd][fd] * uf * uf + Af[ld][ld] * ul * ul) + (2.f * Af[fd][ld] * uf * ul) +
                  (2.f * (blf[fd] * uf + blf[ld] * ul) + q2.y);
  const float bb = b * b, ac = a * c;
  const float disc = bb - ac;
  if (fabsf(disc) <= kQuadRel * (bb + fabsf(ac))) {
    if (ctr) atomicAdd(ctr + kCntFbSphere, 1ull);
    return kDefer;
  }
  if (disc < 0.f) return 0;
  const float sq = sqrtf(disc);
  const float qq = -(b + copysignf(sq, b));
  float sr[2];
  sr[0] = qq / a;
  sr[1] = qq != 0.f ? c / qq : -b / a;
  // the FP64 local quadratic along the ray: a s^2 + 2 b64 s + c64
  const double b64 = (A64[vc][fd] * u64f + A64[vc][ld] * u64l) + bl64[vc];
  const double c64 = (A64[fd][fd] * u64f * u64f + A64[ld][ld] * u64l * u64l) + (2.0 * A64[fd][ld] * u64f * u64l) +
                     (2.0 * (bl64[fd] * u64f + bl64[ld] * u64l) + ql.w);
  const double cv = f[vc];
  int out = 0;
  for (int i = 0; i < 2; i++) {
    double sd = (double)sr[i];
    const double res = (a64 * sd + 2.0 * b64) * sd + c64;
    const float der = 2.f * (a * sr[i] + b);
    sd -= res * (double)(1.f / der);
    float pl[3];
    pl[fd] = uf;
    pl[ld] = ul;
    pl[vc] = (float)sd;
    double p64[3];
    p64[fd] = pa[fd];
    p64[ld] = pa[ld];
    p64[vc] = cv + sd;
    const float4* lp = P.pool32 + first;
    const double4* dp = P.pool + first;
    bool ok = true;
    for (int q2i = 0; q2i < cnt && ok; q2i++)
      if (plane_value(lp[q2i], dp, q2i, pl, p64) > 0) ok = false;
    if (ok) t[out++] = (p64[vc] - pa[vc]) / box_dir;
  }
  return out;
}

// ---- mesh triangles: Moller-Trumbore ----

// Double-precision triangle test of the ray-based mesh caster (MeshSurface::getRayIntersection,
// src/MeshSurface.cpp:1756-1855): the reference's intersect_triangle with the ray from pa along
// axis vc of length dirl; the hit is the ray parameter t.
template <int PN>
__device__ __forceinline__ int intersect_tri_f64(const double* f, const double* pa, double dirl, double* t) {
  constexpr int vc = Ax<PN>::vc;
  double dir[3] = {0.0, 0.0, 0.0};
  dir[vc] = dirl;
  double u, v;
  return ray_triangle_f64(pa, dir, f, f + 3, f + 6, t, &u, &v) ? 1 : 0;
}

// Mixed-precision triangle test: the barycentric coordinates of the ray's foot in the triangle
// from the transverse offsets in FP32 (with the ray along an axis they need only the triangle's
// and the origin's transverse coordinates relative to v0) reject the candidates that miss by more
// than 1e-4 (in barycentric units); every other candidate, and every one with a determinant near
// the reference's EPS cut, is tested in double precision, so that no FP32 rounding reaches an
// accepted hit (which keeps the ray-cast volume and area smooth in the vertices).
template <int PN>
__device__ __forceinline__ int intersect_tri_mixed(const double* f, const double* pa, double dirl, double* t) {
  constexpr int vc = Ax<PN>::vc;
  constexpr int a = vc == 0 ? 1 : (vc == 1 ? 2 : 0), b = vc == 0 ? 2 : (vc == 1 ? 0 : 1);
  const float e1a = (float)(f[3 + a] - f[a]), e1b = (float)(f[3 + b] - f[b]);
  const float e2a = (float)(f[6 + a] - f[a]), e2b = (float)(f[6 + b] - f[b]);
  const float ta = (float)(pa[a] - f[a]), tb = (float)(pa[b] - f[b]);
  const float D = e1b * e2a - e1a * e2b;
  const float det = D * (float)dirl;
  constexpr float kBand = 1e-4f;
  if (fabsf(det) >= 4e-5f) {
    const float inv = 1.f / D;
    const float u = (tb * e2a - ta * e2b) * inv;
    const float v = (ta * e1b - tb * e1a) * inv;
    const float w = 1.f - u - v;
    // the reference's bounds: u <= 1 and u + v <= 1 as well (implied by w >= 0 and v >= 0)
    if (fminf(u, fminf(v, w)) < -kBand) return 0;
  }
  return intersect_tri_f64<PN>(f, pa, dirl, t);
}

// One thread per skin or triangle candidate (in the sphere list): intersection, feasibility, hit
// filing.
template <int PN, bool kMixed>
__device__ __forceinline__ void isect_quadric_body(const TraceCtx& C, const CandOut& co, const HitStore& hs) {
  constexpr int fd = Ax<PN>::fd, ld = Ax<PN>::ld, vc = Ax<PN>::vc;
  const int64_t ncand = *co.count;
  const int2* list = co.sph;
  const int64_t nlim = ncand < co.cap ? ncand : co.cap;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < nlim; c += stride) {
    const int2 e = list[c];
    const int64_t rid = e.x, pid = e.y;
    const int32_t* ir = C.P.i32 + NS_PATCH_I32 * pid;
    const int kind = ir[0], first = ir[1], cnt = ir[2];
    if (!ns_has_box(kind)) continue;
    const StructDev& S = C.B.s[C.B.patch_struct[pid]];
    const GridDev& g = S.g;
    const double delta = ray_set_shifted(C.set) ? NS_DELTA - g.hside : 0.0;
    const int64_t nb = g.n[fd];
    const int64_t lr = rid - S.ray_base[C.set];
    const int64_t m = lr % nb, n = lr / nb;
    double pa[3];
    pa[fd] = gcoord(g, fd, m) + delta;
    pa[ld] = gcoord(g, ld, n) + delta;
    pa[vc] = g.mn[vc] + delta;
    double f[NS_SKIN_Q + 10];
    const double* src = C.P.f64 + (int64_t)NS_PATCH_F64 * pid;
#pragma unroll
    for (int k = 0; k < NS_SKIN_Q + 10; k++) f[k] = __ldg(src + k);
    double t[2];
    int k;
    if (kind == NS_MESH_TRI) {
      // the ray of the mesh caster runs from pa to pb = the last node (+ delta) of the axis
      const double dirl = (gcoord(g, vc, g.n[vc] - 1) + delta) - (gcoord(g, vc, 0) + delta);
      pa[vc] = gcoord(g, vc, 0) + delta;
      k = kMixed ? intersect_tri_mixed<PN>(f, pa, dirl, t) : intersect_tri_f64<PN>(f, pa, dirl, t);
    } else if (kMixed) {
      k = intersect_quadric_mixed<PN>(f, first, cnt, C.P, pid, pa, S.box_dir[vc], t, C.out.counters);
      const bool defer = k == kDefer;
      const unsigned am = __activemask();
      const unsigned dm = __ballot_sync(am, defer);
      if (dm) {
        const int lane = threadIdx.x & 31;
        const int leader = __ffs(dm) - 1;
        unsigned long long base = 0;
        if (lane == leader) base = atomicAdd(co.dcount, (unsigned long long)__popc(dm));
        base = __shfl_sync(am, base, leader);
        if (defer) {
          unsigned long long slot = base + __popc(dm & ((1u << lane) - 1u));
          if ((int64_t)slot < co.dcap) co.dsph[slot] = e;
          else atomicExch(C.out.error_flag, 7);
        }
      }
    } else {
      k = intersect_quadric_f64<PN>(f, first, cnt, C.P, pa, S.box_dir[vc], t);
    }
    if (k <= 0) continue;
    int pos = atomicAdd(hs.cnt + rid, k);
    for (int i = 0; i < k; i++)
      if (pos + i < kHitCap) {
        hs.t[(int64_t)(pos + i) * hs.nrays + rid] = t[i];
        if (hs.pid) hs.pid[(int64_t)(pos + i) * hs.nrays + rid] = (int32_t)pid;
      }
  }
}

template <int PN>
__global__ void __launch_bounds__(256) k_isect_quad(TraceCtx C, CandOut co, HitStore hs) {
  isect_quadric_body<PN, false>(C, co, hs);
}

template <int PN>
__global__ void __launch_bounds__(256, 4) k_isect_quad_mixed(TraceCtx C, CandOut co, HitStore hs) {
  isect_quadric_body<PN, true>(C, co, hs);
}

// The double-precision kernels (the FP64 path and the deferred lists of the mixed path) and the
// mixed-precision ones; the latter ask for enough blocks per SM to keep the sphere kernel, which
// waits on its loads, and the torus kernel at full residency.
template <int PN, bool kTorus>
__global__ void __launch_bounds__(256) k_isect(TraceCtx C, CandOut co, HitStore hs) {
  isect_body<PN, kTorus, false>(C, co, hs);
}

template <int PN, bool kTorus>
__global__ void __launch_bounds__(256, kTorus ? 3 : 6) k_isect_mixed(TraceCtx C, CandOut co, HitStore hs) {
  isect_body<PN, kTorus, true>(C, co, hs);
}

}  // namespace

}  // namespace nsg
