// Device chain rule: atom derivatives of the volume and the area of every structure of a batch
// from the per-patch parameter derivatives (one thread per patch, chain_patch of chain.h,
// atomics into the atom arrays).
#include "../chain.h"
#include "pipeline.h"

namespace nsg {

namespace {

__global__ void k_chain(int64_t np, const int32_t* __restrict__ i32, const double* __restrict__ f64,
                        const int32_t* __restrict__ patch_atoms, const double* __restrict__ atoms, double probe,
                        const double* __restrict__ gpatch_vol, const double* __restrict__ gpatch_area,
                        double* gvol_atoms, double* garea_atoms, int32_t* n_bad) {
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < np; p += (int64_t)gridDim.x * blockDim.x) {
    const int kind = i32[NS_PATCH_I32 * p];
    const double* P = f64 + (int64_t)NS_PATCH_F64 * p;
    const int32_t* pa = patch_atoms + 3 * p;
    bool ok = chain_patch(kind, P, pa, atoms, probe, gpatch_vol + (int64_t)NS_GRAD_PER_PATCH * p,
                          [gvol_atoms](int32_t atom, int slot, double v) { atomicAdd(gvol_atoms + 4 * atom + slot, v); });
    if (gpatch_area)
      ok &= chain_patch(kind, P, pa, atoms, probe, gpatch_area + (int64_t)NS_GRAD_PER_PATCH * p,
                        [garea_atoms](int32_t atom, int slot, double v) { atomicAdd(garea_atoms + 4 * atom + slot, v); });
    if (!ok) atomicAdd(n_bad, 1);
  }
}

}  // namespace

cudaError_t launch_chain(int64_t np, const int32_t* i32, const double* f64, const int32_t* patch_atoms,
                         const double* atoms, double probe, const double* gpatch_vol, const double* gpatch_area,
                         double* gvol_atoms, double* garea_atoms, int32_t* n_bad, cudaStream_t s) {
  if (np <= 0) return cudaSuccess;
  int64_t blocks = (np + 255) / 256;
  if (blocks > (int64_t)sm_count() * 32) blocks = (int64_t)sm_count() * 32;
  k_chain<<<(unsigned)blocks, 256, 0, s>>>(np, i32, f64, patch_atoms, atoms, probe, gpatch_vol, gpatch_area,
                                           gvol_atoms, garea_atoms, n_bad);
  return cudaGetLastError();
}

}  // namespace nsg
