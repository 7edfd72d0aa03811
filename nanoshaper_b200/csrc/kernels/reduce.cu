// Per-structure sums of a batch (interval lengths per ray, triangle areas per active cube): one
// CTA per structure sums its contiguous segment in a fixed order, so that the result does not
// depend on scheduling.
#include "pipeline.h"

namespace nsg {

namespace {

constexpr int kSumThreads = 256;

// out[b] (+)= sum of v[lo .. hi), lo = base[idx ? idx[b] : b], hi = base[idx ? idx[b+1] : b+1].
__global__ void __launch_bounds__(kSumThreads) k_segment_sums(const double* __restrict__ v,
                                                               const int64_t* __restrict__ base,
                                                               const int64_t* __restrict__ idx, double* out,
                                                               int accumulate) {
  __shared__ double part[kSumThreads];
  const int b = blockIdx.x;
  const int64_t lo = base[idx ? idx[b] : b], hi = base[idx ? idx[b + 1] : b + 1];
  double s = 0.0;
  for (int64_t i = lo + threadIdx.x; i < hi; i += kSumThreads) s += v[i];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int w = kSumThreads / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[b] = accumulate ? out[b] + part[0] : part[0];
}

}  // namespace

cudaError_t launch_segment_sums(const double* v, const int64_t* base, const int64_t* idx, int n, double* out,
                                bool accumulate, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_segment_sums<<<n, kSumThreads, 0, s>>>(v, base, idx, out, accumulate ? 1 : 0);
  return cudaGetLastError();
}

}  // namespace nsg
