// Cavity kernels (cavity.cu).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "../ns_types.h"

namespace nsg {

// Union-find labelling of the TEMPORARY_OUT nodes; L[v] = smallest node index of v's region
// (-1 for other nodes), is_root[v] = 1 for region roots.
cudaError_t cc_label(const int32_t* status, int32_t* L, uint8_t* is_root, int64_t nx, int64_t ny, int64_t nz,
                     cudaStream_t s);
// Sorted list of region roots; pass roots == nullptr-free temp == nullptr to query temp_bytes.
cudaError_t cc_select_roots(const uint8_t* is_root, int64_t tot, int32_t* roots, int32_t* nroots, void* temp,
                            size_t* temp_bytes, cudaStream_t s);
// Region sizes and descending-scan keys; replaces L[v] by the region index.
cudaError_t cc_stats(int32_t* L, const int32_t* roots, int32_t nroots, unsigned long long* count, unsigned int* desc_key,
                     int64_t nx, int64_t ny, int64_t nz, cudaStream_t s);
// Final labels into the status map and cavity filling on the insideness bits.
cudaError_t cc_label_fill(int32_t* status, const int32_t* L, const int32_t* label_of, const uint8_t* fill_of,
                          uint32_t* bits, int64_t nwords, int64_t nx, int64_t ny, int64_t nz, cudaStream_t s);

}  // namespace nsg
