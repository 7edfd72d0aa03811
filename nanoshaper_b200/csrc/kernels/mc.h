// Vertex assembly and marching-cubes kernels (mc.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "pipeline.h"

namespace nsg {

// Both argument blocks cover a whole batch: ray ordinals, cube rows, active cubes and vertices
// are batch-wide; every structure's bit grid starts at its word_base in `bits`.
struct VertArgs {
  BatchDev B;
  int64_t nrays;                 // accurate-triangulation rays of the three panels, all structures
  const int64_t* ray_pair_off;
  const int32_t* ray_pair_cnt;
  const double* pairs;
  const uint32_t* bits;
  int32_t* surv_cnt;             // surviving vertices per ray
  const int64_t* surv_off;       // exclusive scan of surv_cnt
  double* vpos;                  // 3 per vertex
  int4* vkey;                    // ix, iy, iz, dir per vertex
  int32_t* vstruct;              // structure of every vertex
  const int2* pair_pid;          // gradient mode: patches of the pair ends, else null
  int32_t* vpid;                 // gradient mode: patch of every analytic vertex
};

struct MCArgs {
  BatchDev B;
  const uint32_t* bits;
  const int32_t* surv_cnt;
  const int64_t* surv_off;
  int64_t n_analytic;
  double* vpos;
  int4* vkey;
  int32_t* vstruct;              // structure of every vertex
  int64_t nrows;                 // cube rows, (NY-2)*(NZ-2) per structure
  const int4* row_chunks;        // structure, first local row, row count (consecutive rows)
  int64_t nchunks;
  int64_t* row_act_cnt;
  const int64_t* row_act_off;    // nrows+1 entries
  int4* act_rec;                 // i, j, k, case | midpoint mask << 8 | structure << 11
  int32_t* mid_cnt;              // midpoint vertices per active cube
  const int64_t* mid_off;        // exclusive scan of mid_cnt
  int32_t* act_mid;              // index of the first midpoint vertex of the cube
  int64_t n_active;
  int32_t* tri_cnt;               // triangles per active cube (interior cubes: from the classification)
  int32_t* bnd_list;             // active cubes on the low faces of the cube range
  unsigned long long* bnd_cursor;
  // active-cube map, one entry per 32 cubes of a cube row (W = ceil((NX-2)/32) per row, rows of a
  // structure from its aword_base): the cubes' active bits and the active index of the first
  // active cube of the word
  int2* amap;
  int32_t* cube_vl;              // 12 per active cube: the vertex of each cut edge it reads
  const int64_t* tri_off;
  int32_t* tris;
  double* cube_area;
  // gradient mode (vgrad null otherwise): d area / d (analytic vertex position along its ray),
  // then d area / d patch parameters
  const int32_t* vpid;
  double* vgrad;
  double* garea;
  const double* f64;
  const int32_t* i32;
  double probe;
};

cudaError_t mc_init_tables();
cudaError_t launch_vert(const VertArgs& A, int emit, cudaStream_t s);
cudaError_t launch_mc_rows(const MCArgs& A, int emit, cudaStream_t s);
cudaError_t launch_mc_mid(const MCArgs& A, int emit, cudaStream_t s);
// blocks_per_sm: 4 (64 registers a thread) or 3 (80 registers).
cudaError_t launch_mc_tris(const MCArgs& A, int blocks_per_sm, cudaStream_t s);
// dst[q] = src[idx[q]] for q < n (per-structure offsets out of batch-wide prefix sums).
cudaError_t launch_gather_i64(const int64_t* src, const int64_t* idx, int64_t n, int64_t* dst, cudaStream_t s);
// Analytic vertices [v0, v1): the first vertex of each grid edge is written into the vertex slots
// of the (up to four) active cubes that share the edge.
cudaError_t launch_mc_push(const MCArgs& A, int64_t v0, int64_t v1, cudaStream_t s);
// Triangle counts of the listed low-face cubes, once the midpoint vertices are in place.
cudaError_t launch_mc_tris_bnd(const MCArgs& A, cudaStream_t s);
// Analytic normal of every analytic vertex v < n_analytic from its patch vpid[v] (zero for patch
// kinds without one, e.g. mesh triangles); 3 doubles per vertex.
cudaError_t launch_vertex_normals(const double* vpos, const int32_t* vpid, int64_t n_analytic, const double* f64,
                                  const int32_t* i32, double probe, double* normals, cudaStream_t s);
// d area / d patch parameters from the per-vertex derivatives (gradient mode).
cudaError_t launch_grad_vert(const MCArgs& A, cudaStream_t s);

}  // namespace nsg
