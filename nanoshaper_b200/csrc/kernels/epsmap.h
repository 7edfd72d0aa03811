// Epsilon and ideb maps after the ray cast, boundary grid points and their projection (epsmap.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "cavity.h"
#include "pipeline.h"

namespace nsg {

// Cavity filling on the epsilon map (fillCavities, src/Surface.cpp:2400-2417): every node of a
// filled cavity gets the inside code on its six grid edges (its three own, and those that end at it).
cudaError_t eps_fill_cavities(const RunArgs& A, const uint8_t* fill_of, int32_t* eps, int32_t inside, cudaStream_t s);

// ideb map, 1 byte per node in the reference's 3-D layout (k*ny + j)*nx + i: 0 at nodes that the
// status rays found inside (lim1 <= x <= lim2, src/Surface.cpp:6655-6663) and at nodes of filled
// cavities (fill_of, null before cavity detection), 1 elsewhere (the initial value,
// src/DelphiShared.cpp:990-997).
cudaError_t ideb_write(const RunArgs& A, const uint8_t* fill_of, uint8_t* ideb, cudaStream_t s);

// Boundary grid points (src/Surface.cpp:1488-1546): nodes with ix, iy, iz >= 1 whose six edge
// codes are not all equal, in the reference's scan order (z outer, x inner), as linear node
// indices (nodes == nullptr only counts them); pass temp == nullptr to query temp_bytes.
cudaError_t bgp_select(const int32_t* eps, int64_t nx, int64_t ny, int64_t nz, int32_t* nodes, int32_t* count,
                       void* temp, size_t* temp_bytes, cudaStream_t s);
// Sum of n int32 (the external points: EXTERNAL_BGP is 1); pass temp == nullptr to query temp_bytes.
cudaError_t sum_i32(const int32_t* in, int32_t n, int64_t* out, void* temp, size_t* temp_bytes, cudaStream_t s);
// ibgp (3 per point: ix, iy, iz) and the type of every selected node: EXTERNAL_BGP when one of
// the six codes is 0, else INTERNAL_BGP.
cudaError_t bgp_expand(const int32_t* eps, int64_t nx, int64_t ny, int64_t nz, const int32_t* nodes, int32_t n,
                       int32_t* ibgp, int32_t* type, cudaStream_t s);

// The SES auxiliary grid of the projection (ConnollySurface::buildAuxiliaryGrid,
// src/ConnollySurface.cpp:3666-3900): n^3 cells, node i of an axis at min + i*side.
struct AuxGrid {
  int64_t n;
  double mn[3];
  double scale;
};
// Per cell, the patches whose bounding-sphere box covers it: counts, then the lists (CSR).
cudaError_t aux_count(const PatchDev& P, const AuxGrid& a, int32_t* cnt, cudaStream_t s);
cudaError_t aux_fill(const PatchDev& P, const AuxGrid& a, const int64_t* off, int32_t* cursor, int32_t* list,
                     cudaStream_t s);

// Projection of the external boundary grid points onto the SES (ConnollySurface::getProjection,
// src/ConnollySurface.cpp:5822-5912): one warp per point, the nearest feasible projection over
// the patches of its auxiliary cell, ties to the smallest patch index.  pos / nor: 3 doubles per
// point (the reference leaves the normal of an external point at 0); flag: 0 projected, 1 no
// feasible projection (the point keeps its own coordinates), 2 empty auxiliary cell, 3 internal
// point (not projected here).
cudaError_t bgp_project(const PatchDev& P, const AuxGrid& a, const int64_t* off, const int32_t* list,
                        const GridDev& g, const int32_t* ibgp, const int32_t* type, int32_t n, double* pos,
                        double* nor, int32_t* flag, cudaStream_t s);

}  // namespace nsg
