// Blobby surface kernels (blobby.cu): the atoms' Gaussian field, its marching-cubes mesh, the
// smoothing pass and the OFF round trip, the mesh as triangle patches, and the adjoint chain.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "pipeline.h"

namespace nsg {

// The field's mesh on the device: vertices (3 doubles), their grid edges (x, y, z, axis),
// triangles (3 vertex ids), the triangle patch records, and per vertex its incident triangle count.
struct BlobbyMeshDev {
  int64_t nv, nt;
  const double* verts;
  const int4* vkey;
  const int32_t* tris;
  const double* f64;
  const int32_t* patch_atoms;
  const int32_t* inc_cnt;
};

cudaError_t blobby_init_tables();
// field[(k ny + j) nx + i] = sum over atoms of exp(B (d^2 / r^2 - 1)) at (x_i, y_j, z_k) - hside,
// each atom over its cube of +-ng nodes.
cudaError_t launch_blobby_field(const GridDev& g, const double* atoms, int na, double B, int ng, double* field,
                                cudaStream_t s);
// Marching cubes on the field over the cubes 1..n-2 of each axis (ncubes of them): per cube the
// own-edge cut mask and the vertex and triangle counts; then vertices (numbered by vbase) and
// triangles (numbered by tbase).
cudaError_t launch_field_cubes(const GridDev& g, const double* f, double iso, int64_t ncubes, uint8_t* mask,
                               int32_t* nvert, int32_t* ntri, cudaStream_t s);
cudaError_t launch_field_verts(const GridDev& g, const double* f, double iso, int64_t ncubes, const uint8_t* mask,
                               const int64_t* vbase, double* verts, int4* vkey, cudaStream_t s);
cudaError_t launch_field_tris(const GridDev& g, const double* f, double iso, int64_t ncubes, const uint8_t* mask,
                              const int64_t* vbase, const int64_t* tbase, const int32_t* ntri, int32_t* tris,
                              cudaStream_t s);
// Vertex -> (triangle, corner) incidence: phase 0 counts into cnt, phase 1 fills inc at off with
// cursor (zeroed) as the per-vertex fill count.
cudaError_t launch_incidence(const int32_t* tris, int64_t nt, int phase, const int64_t* off, int32_t* cnt_or_cursor,
                             int32_t* inc, cudaStream_t s);
cudaError_t launch_smooth(const double* vin, int64_t nv, const int64_t* off, int32_t* inc, const int32_t* tris,
                          double* vout, cudaStream_t s);
// Every coordinate through the OFF text round trip ("%.3f" written, "%f" read).
cudaError_t launch_quantize(double* v, int64_t n, cudaStream_t s);
cudaError_t launch_tri_patches(const double* verts, const int32_t* tris, int64_t nt, double* f64, int32_t* i32,
                               int32_t* patch_atoms, cudaStream_t s);
// d L / d atoms (x, y, z, r; added to gatoms) from the per-triangle slots gpatch of a ray cast of
// the unquantised mesh; gvert_post, gvert_pre (3 per vertex) and gfield (per node) are scratch.
cudaError_t launch_blobby_adjoint(const GridDev& g, const double* atoms, int na, double B, int ng, const double* field,
                                  double iso, const BlobbyMeshDev& M, const double* gpatch, double* gvert_post,
                                  double* gvert_pre, double* gfield, double* gatoms, cudaStream_t s);

}  // namespace nsg
