// Per-structure sums of a batch (interval lengths per ray, triangle areas per active cube) in an
// order fixed by the structure alone, so that the result depends neither on scheduling nor on the
// batch the structure is part of: kSegParts CTAs per structure sum interleaved blocks of its
// segment (by the element's index within the segment), and one thread per structure adds their
// partial sums in CTA order.
#include "pipeline.h"

namespace nsg {

namespace {

constexpr int kSumThreads = 256;

// part[b * kSegParts + k] = sum over the elements of segment b whose index i within the segment
// has (i / kSumThreads) % kSegParts == k; lo = base[idx ? idx[b] : b], hi = base[idx ? idx[b+1] : b+1].
__global__ void __launch_bounds__(kSumThreads) k_segment_parts(const double* __restrict__ v,
                                                                const int64_t* __restrict__ base,
                                                                const int64_t* __restrict__ idx, double* part) {
  __shared__ double red[kSumThreads];
  const int b = blockIdx.x / kSegParts, k = blockIdx.x % kSegParts;
  const int64_t lo = base[idx ? idx[b] : b], hi = base[idx ? idx[b + 1] : b + 1];
  double s = 0.0;
  for (int64_t i = lo + (int64_t)k * kSumThreads + threadIdx.x; i < hi; i += (int64_t)kSegParts * kSumThreads)
    s += v[i];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = kSumThreads / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// out[b] (+)= the partial sums of segment b in CTA order.
__global__ void k_segment_total(const double* __restrict__ part, int n, double* out, int accumulate) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  double s = 0.0;
  for (int k = 0; k < kSegParts; k++) s += part[(int64_t)b * kSegParts + k];
  out[b] = accumulate ? out[b] + s : s;
}

}  // namespace

cudaError_t launch_segment_sums(const double* v, const int64_t* base, const int64_t* idx, int n, double* out,
                                double* part, bool accumulate, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_segment_parts<<<(unsigned)(n * kSegParts), kSumThreads, 0, s>>>(v, base, idx, part);
  k_segment_total<<<(n + 127) / 128, 128, 0, s>>>(part, n, out, accumulate ? 1 : 0);
  return cudaGetLastError();
}

}  // namespace nsg

namespace nsg {

namespace {

// Batch upload fix-ups, one thread per patch: the structure of the patch (binary search in the
// patch offsets), its pool index made batch-wide, and the range checked against its structure's
// pool; its three atom indices made batch-wide and checked against its structure's atoms.
__global__ void k_batch_patches(int64_t np, const int64_t* __restrict__ patch_off, int n,
                                const int64_t* __restrict__ pool_off, int32_t* i32, int32_t* patch_struct,
                                int32_t* err) {
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < np; p += (int64_t)gridDim.x * blockDim.x) {
    const int b = find_struct(patch_off, n, p);
    int32_t* r = i32 + NS_PATCH_I32 * p;
    const int64_t first = r[1], cnt = r[2];
    if (first < 0 || cnt < 0 || first + cnt > pool_off[b + 1] - pool_off[b]) atomicExch(err, 1);
    r[1] = (int32_t)(first + pool_off[b]);
    patch_struct[p] = b;
  }
}

__global__ void k_batch_atoms(int64_t np, const int32_t* __restrict__ patch_struct,
                              const int64_t* __restrict__ atom_off, int32_t* patch_atoms, int32_t* err) {
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < np; p += (int64_t)gridDim.x * blockDim.x) {
    const int b = patch_struct[p];
    const int64_t base = atom_off[b], na = atom_off[b + 1] - base;
    for (int q = 0; q < 3; q++) {
      const int64_t a = patch_atoms[3 * p + q];
      if (a >= na) atomicExch(err, 1);
      patch_atoms[3 * p + q] = a < 0 ? -1 : (int32_t)(a + base);
    }
  }
}

int grid_of(int64_t n) {
  int64_t b = (n + 255) / 256;
  const int64_t cap = (int64_t)sm_count() * 32;
  return (int)(b < 1 ? 1 : (b > cap ? cap : b));
}

}  // namespace

int sm_count() {
  static int cache[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  if (cache[dev] == 0) {
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
    cache[dev] = n;
  }
  return cache[dev];
}

cudaError_t launch_batch_patches(int64_t np, const int64_t* patch_off, int n, const int64_t* pool_off, int32_t* i32,
                                 int32_t* patch_struct, int32_t* err, cudaStream_t s) {
  if (np <= 0) return cudaSuccess;
  k_batch_patches<<<grid_of(np), 256, 0, s>>>(np, patch_off, n, pool_off, i32, patch_struct, err);
  return cudaGetLastError();
}

cudaError_t launch_batch_atoms(int64_t np, const int32_t* patch_struct, const int64_t* atom_off, int32_t* patch_atoms,
                               int32_t* err, cudaStream_t s) {
  if (np <= 0) return cudaSuccess;
  k_batch_atoms<<<grid_of(np), 256, 0, s>>>(np, patch_struct, atom_off, patch_atoms, err);
  return cudaGetLastError();
}

namespace {

// 8 independent FMA chains per thread; the result is stored so that nothing is optimised away.
template <class T>
__global__ void k_fma_peak(int iters, T* out) {
  T a[8];
  const T m = (T)0.999999, c = (T)1e-7;
#pragma unroll
  for (int q = 0; q < 8; q++) a[q] = (T)(threadIdx.x + q);
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int q = 0; q < 8; q++) a[q] = fma(a[q], m, c);
  }
  T s = 0;
#pragma unroll
  for (int q = 0; q < 8; q++) s += a[q];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace

cudaError_t launch_fma_peak(int precision, int blocks, int threads, int iters, void* out, cudaStream_t s) {
  if (precision == 0) k_fma_peak<double><<<blocks, threads, 0, s>>>(iters, (double*)out);
  else k_fma_peak<float><<<blocks, threads, 0, s>>>(iters, (float*)out);
  return cudaGetLastError();
}

}  // namespace nsg
