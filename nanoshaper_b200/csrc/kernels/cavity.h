// Status map, cavity detection and cavity filling kernels (cavity.cu).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "../ns_types.h"

namespace nsg {

// Status map in run form and the free-run union-find state.
struct RunArgs {
  int64_t nx, ny, nz;
  int64_t nrows;              // ny * nz status rows, row = k*ny + j
  const int2* sruns;          // inside runs (first, last node) per row
  const int64_t* srun_off;
  const int32_t* srun_cnt;
  int32_t* fr_cnt;            // free runs per row
  const int64_t* fr_off;      // nrows + 1 offsets
  int2* fruns;                // free runs (first, last node), row-major
  int32_t* frow;              // row of every free run
  int64_t nruns;
  int32_t* L;                 // union-find parents, then region index per run
};

cudaError_t launch_free_runs(const RunArgs& A, int emit, cudaStream_t s);
// Union-find over free runs; is_root[u] = 1 for region roots (smallest run of each region).
cudaError_t run_label(const RunArgs& A, uint8_t* is_root, cudaStream_t s);
// Sorted list of region roots; pass temp == nullptr to query temp_bytes.
cudaError_t run_select_roots(const uint8_t* is_root, int64_t n, int32_t* roots, int32_t* nroots, void* temp,
                             size_t* temp_bytes, cudaStream_t s);
// Region sizes (nodes) and first nodes in descending-z scan order; L becomes the region index.
cudaError_t run_stats(const RunArgs& A, const int32_t* roots, int32_t nroots, unsigned long long* count,
                      unsigned int* desc_key, cudaStream_t s);
// Cavity filling on the insideness bits.
cudaError_t run_fill(const RunArgs& A, const uint8_t* fill_of, uint32_t* bits, int64_t nwords, cudaStream_t s);
// Dense status map from the runs; label_of == nullptr writes TEMPORARY_OUT for free nodes.
cudaError_t status_write(const RunArgs& A, const int32_t* label_of, int32_t* status, cudaStream_t s);

// Atoms lining the cavities (getCavitiesAtomsWithBilevelStatusMap, src/Surface.cpp:2249-2346), on
// the dense status map after cavity detection and the reference's atom grid (buildAtomsMap,
// src/Surface.cpp:1695-1749): gn^3 cells of side 1/gscale from gmn, cell (x, y, z) at
// (z*gn + y)*gn + x, its atoms in ascending index order at cell_off.
struct CavAtomArgs {
  const int32_t* status;
  const int32_t* label;       // cavity membership (the labels before a shape filter); nullptr: status
  int64_t nx, ny, nz;
  double mn[3], side;
  int64_t gn;
  double gmn[3], gscale;
  const int32_t* cell_off;    // gn^3 + 1
  const int32_t* cell_atoms;
  const double* atoms;        // x, y, z, r per atom
  unsigned long long* pairs;  // (cavity << 32) | (atom + 1), one per cavity boundary node
  unsigned long long* count;
  int64_t cap;
  int32_t* err;               // set to 1 when the pairs overflow cap
};
// One pair per node of cavity c (status FIRST_CAV + c) that has a 6-neighbour of another status
// (TEMPORARY_OUT outside the grid): c and the atom of least |a - x|^2 - r^2 over the 27 cells
// around the node, in the reference's cell order, the first of equal ones; atom -1 when the cells
// hold no atom.
cudaError_t cavity_atom_pairs(const CavAtomArgs& A, cudaStream_t s);

// Water-shape filter of the cavities that filling kept (filterCavitiesWithBilevelStatusMap,
// src/Surface.cpp:3011-3290), on the dense status map after cavity detection.  A node of cavity c
// is a support when every grid node within the probe radius of it (inside the reference's
// rounded box) belongs to the filter's in-set of c: the nodes of c, and the removed nodes of the
// kept cavities before c, which the reference leaves as SHAPE_UNDER_CHECK / SHAPE_OK when the
// status map is not modified.  A node of c outside every support sphere of c is removed.
struct ShapeArgs {
  int32_t* status;              // labels in, filtered codes out
  const int32_t* label;         // the labels (FIRST_CAV + c for cavity c) before the filter
  int64_t nx, ny, nz;
  double mn[3], side, scale, r;
  const uint8_t* filled;        // per cavity: filled by the volume threshold (skipped)
  int mod_status;               // removed nodes become STATUS_POINT_INSIDE
  uint8_t* support;             // per node
  uint8_t* removed;             // per node, this pass
  const uint8_t* removed_prev;  // per node, the pass before; nullptr on the first pass
  uint8_t* later;               // per node: inside a support sphere of a later cavity
  int32_t* changed;             // set when removed differs from removed_prev
  uint32_t* bits;               // insideness bits or nullptr
  int64_t nwords;
  int32_t* eps;                 // epsilon map or nullptr
  uint8_t* ideb;                // ideb map or nullptr
  unsigned long long* n_removed;  // per cavity
};
// One pass: supports from the removed set of the pass before, then the removed set.
cudaError_t shape_pass(const ShapeArgs& A, cudaStream_t s);
// Filtered status codes; the removed nodes' insideness bits, epsilon and ideb entries.
cudaError_t shape_apply(const ShapeArgs& A, cudaStream_t s);

// Pocket difference (Surface::difference, src/Surface.cpp:11471-11717), on the dense maps of the
// fat-probe (st1, in/out) and small-probe (st2) surfaces: a node inside-or-cavity in st1 and
// TEMPORARY_OUT / OUT in st2 becomes FIRST_CAV, every other node STATUS_POINT_INSIDE; its
// insideness bit becomes the same predicate (the last of the reference's 8-corner writes to a
// node is the node's own).  count receives the number of difference nodes.
cudaError_t pocket_difference(int32_t* st1, const int32_t* st2, int64_t n, uint32_t* bits, unsigned long long* count,
                              cudaStream_t s);
// cav2outWithBilevelStatusMap (src/Surface.cpp:2691-2748) for the one difference cavity: its
// nodes (label FIRST_CAV) still at a cavity or support code return to TEMPORARY_OUT.
cudaError_t pocket_cav2out(int32_t* status, const int32_t* label, int64_t n, cudaStream_t s);
// Free runs (TEMPORARY_OUT runs per x-row) of a dense status map; count pass then emit pass.
cudaError_t dense_free_runs(const RunArgs& A, const int32_t* status, int emit, cudaStream_t s);

// Sorts the n pairs and keeps one of each; pass temp == nullptr to query temp_bytes.
cudaError_t sort_unique_u64(unsigned long long* keys, unsigned long long* keys_alt, int64_t n, int64_t* n_unique,
                            void* temp, size_t* temp_bytes, cudaStream_t s);

}  // namespace nsg
