// Cavity detection and conditional filling on the status map.
//
// The reference labels the 6-connected regions of STATUS_POINT_TEMPORARY_OUT nodes one at a time
// with a scanline flood fill seeded at the first remaining node of a scan whose z direction
// alternates between ascending and descending (getCavitiesWithBilevelStatusMap
// src/Surface.cpp:1994-2126, floodFillWithBilevelStatusMap2 :4284-4554); the first region found
// becomes STATUS_POINT_OUT (3), the following ones cavities 4, 5, ...  Cavities whose node count
// times side^3 does not exceed the threshold get the insideness bits of the 8 corners of each of
// their nodes cleared (fillCavities :2355-2484).
//
// On the GPU all regions are found at once with a lock-free union-find whose roots are the
// smallest node index of each region (= the region's first node in ascending scan order).  The
// region's first node in descending scan order is reduced with atomicMin.  The host then replays
// the alternating seed selection over these two keys, which reproduces the reference labels.
#include <cub/cub.cuh>

#include "cavity.h"

namespace nsg {

namespace {

__device__ __forceinline__ int32_t find_root(int32_t* L, int32_t v) {
  int32_t p = L[v];
  while (p != v) {
    int32_t gp = L[p];
    if (gp != p) L[v] = gp;  // path halving; benign race
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

__global__ void k_cc_init(const int32_t* __restrict__ status, int32_t* L, int64_t tot) {
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < tot; v += (int64_t)gridDim.x * blockDim.x)
    L[v] = (status[v] == NS_STATUS_TEMPORARY_OUT) ? (int32_t)v : -1;
}

// Hooks each free node to its +x, +y, +z free neighbours.
__global__ void k_cc_hook(const int32_t* __restrict__ status, int32_t* L, int64_t nx, int64_t ny, int64_t nz) {
  int64_t tot = nx * ny * nz;
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < tot; v += (int64_t)gridDim.x * blockDim.x) {
    if (status[v] != NS_STATUS_TEMPORARY_OUT) continue;
    int64_t i = v % nx;
    int64_t r = v / nx;
    int64_t j = r % ny;
    int64_t k = r / ny;
    if (i + 1 < nx && status[v + 1] == NS_STATUS_TEMPORARY_OUT) unite(L, (int32_t)v, (int32_t)(v + 1));
    if (j + 1 < ny && status[v + nx] == NS_STATUS_TEMPORARY_OUT) unite(L, (int32_t)v, (int32_t)(v + nx));
    if (k + 1 < nz && status[v + nx * ny] == NS_STATUS_TEMPORARY_OUT) unite(L, (int32_t)v, (int32_t)(v + nx * ny));
  }
}

// Final root of every node.  The walk does not shorten paths: a halving write issued by one
// thread could otherwise overwrite a label another thread has already set to its root.
__global__ void k_cc_compress(int32_t* L, int64_t tot, uint8_t* is_root) {
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < tot; v += (int64_t)gridDim.x * blockDim.x) {
    int32_t l = L[v];
    if (l < 0) { is_root[v] = 0; continue; }
    int32_t r = l;
    for (int32_t q = L[r]; q != r; q = L[r]) r = q;
    L[v] = r;
    is_root[v] = (r == v) ? 1 : 0;
  }
}

// Per node: component index by binary search in the sorted root list; size and descending-scan
// key reductions.  L[v] is replaced by the component index.  Lanes of a warp that fall into the
// same component (the common case: the outer region covers most of the grid) are combined
// before the atomics, so the hot counters see one update per warp instead of one per node.
__global__ void k_cc_stats(int32_t* L, const int32_t* __restrict__ roots, int32_t nroots, unsigned long long* count,
                           unsigned int* desc_key, int64_t nx, int64_t ny, int64_t nz) {
  int64_t tot = nx * ny * nz;
  int64_t plane = nx * ny;
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < tot; v += (int64_t)gridDim.x * blockDim.x) {
    unsigned act = __activemask();
    int32_t l = L[v];
    unsigned has = __ballot_sync(act, l >= 0);
    if (l < 0) continue;
    int32_t lo = 0, hi = nroots - 1;
    if (roots[0] != l) {
      while (lo < hi) {
        int32_t mid = (lo + hi) >> 1;
        if (roots[mid] < l) lo = mid + 1;
        else hi = mid;
      }
    }
    L[v] = lo;
    int64_t k = v / plane;
    unsigned key = (unsigned)((nz - 1 - k) * plane + (v - k * plane));
    unsigned grp = __match_any_sync(has, lo);
    unsigned kmin = __reduce_min_sync(grp, key);
    if ((int)(threadIdx.x & 31) == __ffs(grp) - 1) {
      atomicAdd(count + lo, (unsigned long long)__popc(grp));
      atomicMin(desc_key + lo, kmin);
    }
  }
}

// Writes region labels into the status map and clears the 8 cube-corner insideness bits of the
// nodes of filled cavities.
__global__ void k_cc_label_fill(int32_t* status, const int32_t* __restrict__ L, const int32_t* __restrict__ label_of,
                                const uint8_t* __restrict__ fill_of, uint32_t* bits, int64_t nwords, int64_t nx,
                                int64_t ny, int64_t nz) {
  int64_t tot = nx * ny * nz;
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < tot; v += (int64_t)gridDim.x * blockDim.x) {
    int32_t c = L[v];
    if (c < 0) continue;
    int32_t lab = label_of[c];
    status[v] = lab;
    if (bits && fill_of[c]) {
      for (int dk = 0; dk < 2; dk++)
        for (int dj = 0; dj < 2; dj++)
          for (int di = 0; di < 2; di++) {
            int64_t f = v + di + dj * nx + dk * nx * ny;
            if ((f >> 5) < nwords) atomicAnd(bits + (f >> 5), ~(1u << (f & 31)));
          }
    }
  }
}

int grid_for(int64_t tot) {
  int64_t b = (tot + 255) / 256;
  return (int)(b < 148 * 64 ? (b < 1 ? 1 : b) : 148 * 64);
}

}  // namespace

cudaError_t cc_label(const int32_t* status, int32_t* L, uint8_t* is_root, int64_t nx, int64_t ny, int64_t nz,
                     cudaStream_t s) {
  int64_t tot = nx * ny * nz;
  k_cc_init<<<grid_for(tot), 256, 0, s>>>(status, L, tot);
  k_cc_hook<<<grid_for(tot), 256, 0, s>>>(status, L, nx, ny, nz);
  k_cc_compress<<<grid_for(tot), 256, 0, s>>>(L, tot, is_root);
  return cudaGetLastError();
}

cudaError_t cc_select_roots(const uint8_t* is_root, int64_t tot, int32_t* roots, int32_t* nroots, void* temp,
                            size_t* temp_bytes, cudaStream_t s) {
  cub::CountingInputIterator<int32_t> it(0);
  return cub::DeviceSelect::Flagged(temp, *temp_bytes, it, is_root, roots, nroots, tot, s);
}

cudaError_t cc_stats(int32_t* L, const int32_t* roots, int32_t nroots, unsigned long long* count, unsigned int* desc_key,
                     int64_t nx, int64_t ny, int64_t nz, cudaStream_t s) {
  int64_t tot = nx * ny * nz;
  if (nroots <= 0) return cudaSuccess;
  k_cc_stats<<<grid_for(tot), 256, 0, s>>>(L, roots, nroots, count, desc_key, nx, ny, nz);
  return cudaGetLastError();
}

cudaError_t cc_label_fill(int32_t* status, const int32_t* L, const int32_t* label_of, const uint8_t* fill_of,
                          uint32_t* bits, int64_t nwords, int64_t nx, int64_t ny, int64_t nz, cudaStream_t s) {
  int64_t tot = nx * ny * nz;
  k_cc_label_fill<<<grid_for(tot), 256, 0, s>>>(status, L, label_of, fill_of, bits, nwords, nx, ny, nz);
  return cudaGetLastError();
}

}  // namespace nsg
