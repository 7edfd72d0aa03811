// Allocation-free status ray cast: a variant of the per-ray tracer for callers that cannot
// allocate device memory (code running inside another framework's memory pool, inside a
// library whose allocator is locked down, or under a policy that forbids cudaMalloc after
// start-up).  The caller passes the patch set and the output status map in device memory it
// already owns; the per-ray hit columns, per-ray interval lengths, the error flag and the
// volume sum live in one file-scope __device__ array of fixed size.
//
// Limits: at most kMaxRays status rays (ny * nz) and kMaxHits hits per ray.  Larger inputs are
// rejected with NSG_ERR_CAPACITY before any launch.  The array is created with the module and
// stays resident on every GPU that loads the library until the process exits.
//
// Every call shares the array and leaves the previous call's contents in it; the parts that must
// start at zero are cleared by each call.  Calls whose work overlaps on the GPU (different
// streams, or different host threads on the same device) race on the array and must be
// serialised by the caller.
//
// Every call looks up the array's device address with cudaGetSymbolAddress on the current
// device, so the address stays valid across a cudaDeviceReset.  With lazy module loading (the
// CUDA default) the first call in a process loads the module and reserves the array; a caller
// whose device memory is fixed after start-up makes one call at start-up.  A call synchronises
// its stream and reads the result back to the host, so it cannot be made while any stream is
// being captured into a CUDA graph.
//
// A ray with more than kMaxHits hits makes the call return NSG_ERR_CAPACITY after its launches;
// the status map is then unspecified.
#include <cuda_runtime.h>

#include "host/host_api.h"
#include "kernels/ray_math.cuh"

namespace {

constexpr int64_t kMaxRays = 65536;  // status rays per call (ny * nz)
constexpr int kMaxHits = 32;         // hits per ray
// [hits: kMaxHits * kMaxRays][row lengths: kMaxRays][error flag][volume sum]
constexpr int64_t kScratch = (int64_t)kMaxHits * kMaxRays + kMaxRays + 2;
static __device__ __align__(256) double g_noalloc_scratch[kScratch];

struct Geo {
  int64_t n[3];
  double mn[3], mx[3];
  double scale, side, hside;
};

__device__ __forceinline__ double coord(const Geo& g, int d, int64_t i) { return g.mn[d] + (double)i * g.side; }

// Status ray (j, k) along x through grid nodes: every patch whose pixel window, bounding box and
// equatorial disc contain the ray is intersected in double precision (the arithmetic of the
// reference's raySphere / rayTorus / isFeasible); hits are sorted in the ray's scratch column,
// paired, and the row of the status map and the row's interval length are written.
__global__ void k_status_noalloc(Geo g, int64_t np, const double* __restrict__ f64, const int32_t* __restrict__ i32,
                                 const double4* __restrict__ pool, const int8_t* __restrict__ flag, double probe,
                                 int32_t* __restrict__ status, double* scratch) {
  const int64_t nrays = g.n[1] * g.n[2];
  double* hits = scratch;
  double* row_len = scratch + (int64_t)kMaxHits * kMaxRays;
  double* err = row_len + kMaxRays;
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < nrays; r += (int64_t)gridDim.x * blockDim.x) {
    const int64_t j = r % g.n[1], k = r / g.n[1];
    double pa[3] = {coord(g, 0, 0), coord(g, 1, j), coord(g, 2, k)};
    const double ray_dir = coord(g, 0, g.n[0] - 1) - coord(g, 0, 0);
    const double dir[3] = {ray_dir, 0., 0.};
    double* col = hits + r;  // slot q at col[q * kMaxRays]
    int nh = 0;
    bool ovf = false;
    for (int64_t p = 0; p < np && !ovf; p++) {
      const double* f = f64 + NS_PATCH_F64 * p;
      if (ns_has_box(i32[NS_PATCH_I32 * p])) {
        err[0] = 2.0;  // SES patch sets only
        ovf = true;
        break;
      }
      const double rad = f[3];
      double down[3], up[3];
      bool cull = false;
      for (int d = 0; d < 3; d++) {
        down[d] = f[d] - rad;
        up[d] = f[d] + rad;
        if (down[d] > g.mx[d] + NS_EPS_INT) cull = true;
        if (up[d] < g.mn[d] - (g.hside - NS_DELTA + NS_EPS_INT)) cull = true;
      }
      if (cull) continue;
      // pixel window over (y, z)
      int64_t ok = 1;
      for (int d = 1; d < 3; d++) {
        int64_t s = (int64_t)nsg::rintp(fmax(0., down[d] - g.mn[d]) * g.scale);
        int64_t e = (int64_t)nsg::rintp(fmax(0., up[d] - g.mn[d]) * g.scale);
        if (e >= g.n[d]) e = g.n[d] - 1;
        int64_t idx = d == 1 ? j : k;
        if (idx < s || idx > e) ok = 0;
      }
      if (!ok) continue;
      if (pa[1] < down[1] || pa[1] > up[1] || pa[2] < down[2] || pa[2] > up[2]) continue;
      double dx = f[1] - pa[1], dy = f[2] - pa[2];
      if (dx * dx + dy * dy > rad * rad) continue;
      double t[4];
      if (!nsg::ray_sphere_f64(pa, dir, f, rad, &t[0], &t[1])) continue;
      const int32_t* ir = i32 + NS_PATCH_I32 * p;
      if (ir[2] > 0 && (pool == nullptr || flag == nullptr)) {
        err[0] = 2.0;  // pool entries referenced but no pool given
        ovf = true;
        break;
      }
      int numInt = 2;
      if (ir[0] == NS_EDGE_REG || ir[0] == NS_EDGE_SING) numInt = nsg::ray_torus_f64(f, probe, 0, pa, ray_dir, t);
      for (int i = 0; i < numInt; i++) {
        double ip[3] = {pa[0] + t[i] * ray_dir, pa[1], pa[2]};
        if (!nsg::feasible_f64(f, ir[0], ir[1], ir[2], pool, flag, ip)) continue;
        if (nh >= kMaxHits) {
          ovf = true;
          break;
        }
        int pos = nh++;
        while (pos > 0 && col[(int64_t)(pos - 1) * kMaxRays] > t[i]) {
          col[(int64_t)pos * kMaxRays] = col[(int64_t)(pos - 1) * kMaxRays];
          pos--;
        }
        col[(int64_t)pos * kMaxRays] = t[i];
      }
    }
    if (ovf) {
      err[0] = 1.0;
      nh = 0;
    }
    // pairs (even hit counts only, intervals longer than EPS_INT) -> row of the status map
    int32_t* row = status + r * g.n[0];
    for (int64_t i = 0; i < g.n[0]; i++) row[i] = NS_STATUS_TEMPORARY_OUT;
    double len = 0.0;
    if (nh > 0 && (nh & 1) == 0) {
      const double x0 = coord(g, 0, 0);
      for (int q = 0; q < nh; q += 2) {
        double t1 = col[(int64_t)q * kMaxRays], t2 = col[(int64_t)(q + 1) * kMaxRays];
        if (!(fabs(t2 - t1) >= NS_EPS_INT)) continue;
        double lim1 = x0 + ray_dir * t1, lim2 = x0 + ray_dir * t2;
        len += lim2 - lim1;
        int64_t i1 = (int64_t)nsg::rintp((lim1 - g.mn[0]) * g.scale);
        int64_t i2 = (int64_t)nsg::rintp((lim2 - g.mn[0]) * g.scale);
        i1 = i1 < 0 ? 0 : (i1 >= g.n[0] ? g.n[0] - 1 : i1);
        i2 = i2 < 0 ? 0 : (i2 >= g.n[0] ? g.n[0] - 1 : i2);
        for (int64_t i = i1; i <= i2; i++) {
          double x = coord(g, 0, i);
          if (x <= lim2 && x >= lim1) row[i] = NS_STATUS_INSIDE;
        }
      }
    }
    row_len[r] = len;
  }
}

// Sum of the row interval lengths in a fixed order (one block), written to the scratch slot.
__global__ void k_noalloc_sum(int64_t nrays, double* scratch) {
  __shared__ double part[256];
  const double* row_len = scratch + (int64_t)kMaxHits * kMaxRays;
  double s = 0.0;
  for (int64_t r = threadIdx.x; r < nrays; r += blockDim.x) s += row_len[r];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) scratch[kScratch - 1] = part[0];
}

// Device address of the scratch array on the current device (host code cannot use the symbol
// itself: on the host it names a stand-in, not device memory).
int scratch_address(double** out) {
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p) return NSG_ERR_CUDA;
  *out = (double*)p;
  return NSG_OK;
}

}  // namespace

extern "C" {

// Status map (flat int32, k*ny*nx + j*nx + i) and status-ray volume of a grid from a patch set,
// without allocating device memory.  Patch arrays and the status map are device pointers owned
// by the caller; *volume is written on the host after the call's work completes on `stream`.
int nsg_status_noalloc(const NsGrid* grid, int64_t n_patches, const double* d_f64, const int32_t* d_i32,
                       const double* d_pool, const int8_t* d_pool_flag, double probe_radius, int32_t* d_status,
                       double* volume, void* stream) {
  if (!grid || !d_status || !volume || n_patches < 0 || (n_patches > 0 && (!d_f64 || !d_i32))) return NSG_ERR_ARG;
  if (grid->nx < 3 || grid->ny < 3 || grid->nz < 3) return NSG_ERR_ARG;
  if (grid->ny * grid->nz > kMaxRays) return NSG_ERR_CAPACITY;
  double* scratch = nullptr;
  int rc = scratch_address(&scratch);
  if (rc != NSG_OK) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  Geo g;
  g.n[0] = grid->nx; g.n[1] = grid->ny; g.n[2] = grid->nz;
  g.mn[0] = grid->xmin; g.mn[1] = grid->ymin; g.mn[2] = grid->zmin;
  g.mx[0] = grid->xmax; g.mx[1] = grid->ymax; g.mx[2] = grid->zmax;
  g.scale = grid->scale; g.side = grid->side; g.hside = grid->hside;
  double* err = scratch + (int64_t)kMaxHits * kMaxRays + kMaxRays;
  if (cudaMemsetAsync(err, 0, sizeof(double), s) != cudaSuccess) return NSG_ERR_CUDA;
  const int64_t nrays = grid->ny * grid->nz;
  int blocks = (int)((nrays + 127) / 128);
  k_status_noalloc<<<blocks, 128, 0, s>>>(g, n_patches, d_f64, d_i32, (const double4*)d_pool, d_pool_flag,
                                          probe_radius, d_status, scratch);
  k_noalloc_sum<<<1, 256, 0, s>>>(nrays, scratch);
  if (cudaGetLastError() != cudaSuccess) return NSG_ERR_CUDA;
  double out[2] = {0.0, 0.0};
  if (cudaMemcpyAsync(out, err, 2 * sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess) return NSG_ERR_CUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return NSG_ERR_CUDA;
  if (out[0] == 2.0) return NSG_ERR_ARG;
  if (out[0] != 0.0) return NSG_ERR_CAPACITY;
  *volume = grid->A * out[1];
  return NSG_OK;
}

}  // extern "C"
