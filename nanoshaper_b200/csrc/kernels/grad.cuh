// Adjoint of the ray-cast hit positions.
//
// A hit lies on the surface F(x; theta) = 0 of its patch at x = ray origin + s e (e the unit ray
// axis), so ds/dtheta = -(dF/dtheta) / (dF/dx . e).  The patch surfaces and their parameters:
//   sphere (atom or probe): F = |x - c|^2 - r^2,                 theta = (c, r)
//   torus:                  F = S^2 - 4 R^2 (|y|^2 - z^2),      theta = (tc, u, R)
//                           y = x - tc, z = u . y, S = |y|^2 + R^2 - probe^2
//   mesh triangle:          F = n . (x - v0), n = (v1 - v0) x (v2 - v0), theta = (v0, v1, v2)
// (the torus with the local z axis u = third row of the inverse frame, the surface rayTorus
// solves, src/tools.cpp:907-1098).  A probe sphere's radius is the fixed probe, so its slot 3
// stays 0.  Derivatives of the volume (interval ends) and of the marching-cubes area (analytic
// vertices) are sums of these terms.
#pragma once
#include "ray_math.cuh"

namespace nsg {

// ds/dtheta of a hit x on axis vc of patch record P into g[NS_GRAD_PER_PATCH]; returns false
// (g zero) when the ray is tangent to the surface there.
__device__ __forceinline__ bool hit_grad(const double* __restrict__ P, int kind, double probe, const double* x, int vc,
                                         double* g) {
#pragma unroll
  for (int k = 0; k < NS_GRAD_PER_PATCH; k++) g[k] = 0.0;
  if (kind == NS_EDGE_REG || kind == NS_EDGE_SING) {
    const double y0 = x[0] - P[kTC], y1 = x[1] - P[kTC + 1], y2 = x[2] - P[kTC + 2];
    const double u0 = P[kInv + 6], u1 = P[kInv + 7], u2 = P[kInv + 8];
    const double R = P[kMajor];
    const double yy = y0 * y0 + y1 * y1 + y2 * y2;
    const double z = u0 * y0 + u1 * y1 + u2 * y2;
    const double S = yy + R * R - probe * probe;
    const double R2 = R * R;
    const double G0 = 4.0 * S * y0 - 8.0 * R2 * (y0 - z * u0);
    const double G1 = 4.0 * S * y1 - 8.0 * R2 * (y1 - z * u1);
    const double G2 = 4.0 * S * y2 - 8.0 * R2 * (y2 - z * u2);
    const double den = vc == 0 ? G0 : (vc == 1 ? G1 : G2);
    if (!(fabs(den) > 1e-12 * (fabs(G0) + fabs(G1) + fabs(G2) + 1e-300))) return false;
    const double inv = 1.0 / den;
    g[0] = G0 * inv;
    g[1] = G1 * inv;
    g[2] = G2 * inv;
    const double cu = -8.0 * R2 * z * inv;
    g[3] = cu * y0;
    g[4] = cu * y1;
    g[5] = cu * y2;
    g[6] = -(4.0 * S * R - 8.0 * R * (yy - z * z)) * inv;
    return true;
  }
  if (kind == NS_MESH_TRI) {
    // F = n . (x - v0), n = (v1 - v0) x (v2 - v0): moving corner k by dv moves the hit along the
    // ray by b_k (n . dv) / n_vc (b the hit's barycentric weights); g[k] = b_k / n_vc, the factor n
    // is applied per triangle by the chain rule to the mesh vertices
    const double* n = P + NS_TRI_N;
    const double nn = n[0] * n[0] + n[1] * n[1] + n[2] * n[2];
    const double den = vc == 0 ? n[0] : (vc == 1 ? n[1] : n[2]);
    if (!(fabs(den) > 1e-12 * sqrt(nn))) return false;
    const double e1[3] = {P[3] - P[0], P[4] - P[1], P[5] - P[2]};
    const double e2[3] = {P[6] - P[0], P[7] - P[1], P[8] - P[2]};
    const double w[3] = {x[0] - P[0], x[1] - P[1], x[2] - P[2]};
    const double c1[3] = {w[1] * e2[2] - w[2] * e2[1], w[2] * e2[0] - w[0] * e2[2], w[0] * e2[1] - w[1] * e2[0]};
    const double c2[3] = {e1[1] * w[2] - e1[2] * w[1], e1[2] * w[0] - e1[0] * w[2], e1[0] * w[1] - e1[1] * w[0]};
    const double b1 = (c1[0] * n[0] + c1[1] * n[1] + c1[2] * n[2]) / nn;
    const double b2 = (c2[0] * n[0] + c2[1] * n[1] + c2[2] * n[2]) / nn;
    const double inv = 1.0 / den;
    g[0] = (1.0 - b1 - b2) * inv;
    g[1] = b1 * inv;
    g[2] = b2 * inv;
    return true;
  }
  const double d0 = x[0] - P[0], d1 = x[1] - P[1], d2 = x[2] - P[2];
  const double den = vc == 0 ? d0 : (vc == 1 ? d1 : d2);
  if (!(fabs(den) > 1e-12 * (fabs(d0) + fabs(d1) + fabs(d2) + 1e-300))) return false;
  const double inv = 1.0 / den;
  g[0] = d0 * inv;
  g[1] = d1 * inv;
  g[2] = d2 * inv;
  if (kind == NS_POINT) g[3] = P[kR] * inv;
  return true;
}

// gsum[8 * pid + k] += w * ds/dtheta_k for a hit of patch pid at x.
__device__ __forceinline__ void add_hit_grad(const double* __restrict__ f64, const int32_t* __restrict__ i32,
                                             double probe, int32_t pid, const double* x, int vc, double w,
                                             double* gsum) {
  if (pid < 0 || w == 0.0) return;
  double g[NS_GRAD_PER_PATCH];
  const double* P = f64 + (int64_t)NS_PATCH_F64 * pid;
  if (!hit_grad(P, i32[NS_PATCH_I32 * pid], probe, x, vc, g)) return;
  double* o = gsum + (int64_t)NS_GRAD_PER_PATCH * pid;
#pragma unroll
  for (int k = 0; k < NS_GRAD_PER_PATCH; k++)
    if (g[k] != 0.0) atomicAdd(o + k, w * g[k]);
}

// Warp-collective: lanes holding terms g (already weighted) for patch pid (-1: none) add them to
// gsum[8 * pid + k].  Consecutive lanes with the same patch (neighbouring rays or vertices usually
// hit the same patch) are summed with a segmented shuffle scan first, so each run of equal pids
// issues one atomic per component instead of one per lane.  All 32 lanes must call it.
__device__ __forceinline__ void warp_add_grad(int32_t pid, double* g, double* gsum) {
  // hit_grad fills at most the first kGradUsed components (a torus: centre, axis terms, major
  // radius); the last slot of a patch's record stays zero
  constexpr int kGradUsed = 7;
  static_assert(kGradUsed <= NS_GRAD_PER_PATCH, "gradient record too short");
  if (!__any_sync(0xffffffffu, pid >= 0)) return;
  const int lane = threadIdx.x & 31;
  const int32_t prev = __shfl_up_sync(0xffffffffu, pid, 1);
  const bool head = lane == 0 || prev != pid;
  const unsigned heads = __ballot_sync(0xffffffffu, head);
  const int start = 31 - __clz(heads & (0xffffffffu >> (31 - lane)));
  const bool tail = lane == 31 || ((heads >> (lane + 1)) & 1u);
#pragma unroll
  for (int k = 0; k < kGradUsed; k++) {
    double v = g[k];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const double u = __shfl_up_sync(0xffffffffu, v, o);
      if (lane - o >= start) v += u;
    }
    g[k] = v;
  }
  if (tail && pid >= 0) {
    double* o = gsum + (int64_t)NS_GRAD_PER_PATCH * pid;
#pragma unroll
    for (int k = 0; k < kGradUsed; k++)
      if (g[k] != 0.0) atomicAdd(o + k, g[k]);
  }
}

}  // namespace nsg
