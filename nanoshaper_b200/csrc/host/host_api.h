// Host-side entry points of the surface builder library (grid environment and patch builders).
// Exported with C linkage from libnsgpu; the public declarations live in include/nsgpu.h.
#pragma once
#include <stdint.h>

#include "../ns_types.h"

#define NSG_OK 0
#define NSG_ERR_ARG (-1)
#define NSG_ERR_EMPTY (-2)
#define NSG_ERR_IO (-3)
#define NSG_ERR_CAPACITY (-4)
#define NSG_ERR_CUDA (-5)
#define NSG_ERR_NOMEM (-6)
#define NSG_ERR_STATE (-7)
#define NSG_ERR_GEOMETRY (-8)
#define NSG_ERR_TIMEOUT (-9)

#define NSG_PRECISION_FP64 0
#define NSG_PRECISION_MIXED 1

#define NSG_RAYCAST_EPSMAP 4

#ifdef __cplusplus
extern "C" {
#endif

int nsg_grid_build(const double* atoms_xyzr, int64_t n_atoms, double scale, double perfil, NsGrid* out);
double nsg_randnum(int64_t* seed);
int nsg_jitter_atoms(double* atoms_xyzr, int64_t n_atoms, double displacement, int64_t* seed);
int64_t nsg_read_xyzr(const char* path, double* out, int64_t capacity);
int64_t nsg_read_pqr(const char* path, double* out, int64_t capacity);

// Host-owned patch set produced by a patch builder.
typedef struct NsPatchSet NsPatchSet;

int nsg_ses_build(const double* atoms_xyzr, int64_t n_atoms, double probe_radius, int n_threads,
                  NsPatchSet** out);
int nsg_skin_build(const double* atoms_xyzr, int64_t n_atoms, double shrink, int n_threads, NsPatchSet** out);
int nsg_skin_predicates(const int64_t* points, int* orient, int* conflict);
int nsg_patchset_info(const NsPatchSet* ps, int64_t* n_patches, int64_t* n_pool, int64_t counts[5]);
int nsg_patchset_kind_counts(const NsPatchSet* ps, int64_t* counts, int n);
int nsg_patchset_export(const NsPatchSet* ps, double* f64, int32_t* i32, double* pool, int8_t* pool_flag);
int nsg_patchset_atoms(const NsPatchSet* ps, int32_t* out);
void nsg_patchset_free(NsPatchSet* ps);

int nsg_write_status(const char* path, const int32_t* status, int64_t nx, int64_t ny, int64_t nz);
int nsg_write_cavities(const char* cavities_path, const char* sizes_path, const int32_t* status, const NsGrid* g,
                       int32_t n_cav, const double* sizes, const int32_t* filled);
int nsg_write_mesh(const char* root, int format, const double* vertices, int64_t n_vertices, const int32_t* triangles,
                   int64_t n_triangles, int revert);

int nsg_mesh_normals(const double* vertices, int64_t n_vertices, const int32_t* triangles, int64_t n_triangles,
                     double* normals);
int nsg_fill_zero_normals(const double* vertices, int64_t n_vertices, const int32_t* triangles, int64_t n_triangles,
                          double* normals);

int nsg_ses_chain_grad(const double* atoms_xyzr, int64_t n_atoms, double probe, int64_t n_patches,
                       const int32_t* i32, const double* f64, const int32_t* patch_atoms, const double* gpatch,
                       double* grad_atoms);

#ifdef __cplusplus
}
#endif
