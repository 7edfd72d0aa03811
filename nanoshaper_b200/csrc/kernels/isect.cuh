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

// Mixed-precision intersection launches of one panel (trace_mixed.cu): the sphere and torus
// candidate lists of co, with the deferred candidates appended to co's deferred lists.
template <int PN>
void launch_isect_mixed(const TraceCtx& C, const CandOut& co, const HitStore& hs, const TuneParams& tp,
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
  float s32 = sqrtf(disc);
  double disc64 = r * r - dx64 * dx64 - dy64 * dy64;
  double sd = (double)s32;
  sd = sd + (disc64 - sd * sd) * (double)(0.5f / s32);
  double xs[4];
  int nx = 0;
  const double cv = f[vc];
  if (kTorus) {
    const double x_in = cv - sd;
    double orig1[3];
    orig1[fd] = pa[fd];
    orig1[ld] = pa[ld];
    orig1[vc] = x_in;
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
      double px = x_in + root;
      double e0 = f[fd] - pa[fd], e1 = f[ld] - pa[ld], e2 = cv - px;
      double dd = e0 * e0 + e1 * e1 + e2 * e2;
      if (fabs(dd - r2) < 1e-9) {
        if (ctr) atomicAdd(ctr + kCntFbRoot, 1ull);
        return kDefer;
      }
      if (dd < r2) xs[nx++] = px;
    }
  } else {
    xs[0] = cv - sd;
    xs[1] = cv + sd;
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
    if (feasible_mixed<kTorus>(f, kind, first, cnt, P.pool, P.pool32, P.flag, pl, p64))
      t[out++] = (xs[i] - pa[vc]) * inv_dir;
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
    const double delta = C.set == 0 ? 0.0 : NS_DELTA - g.hside;
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
