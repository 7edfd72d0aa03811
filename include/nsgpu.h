/* libnsgpu -- B200 grid ray-casting molecular surface builder, C ABI.
 *
 * Drop-in boundary for the part of NanoShaper that runs once a surface's patches exist:
 * Surface::getSurf (src/Surface.cpp:398-1692) and Surface::triangulateSurface
 * (src/Surface.cpp:9909-10526), behind the Surface plugin interface (src/Surface.h:835-990).
 * Plain pointers and sizes only.  Every call returns NSG_OK (0) or a negative NSG_ERR_* code and
 * never terminates the process (the reference exits on fatal errors).  Host buffers are always
 * owned by the caller; device buffers by the context.  One context per host thread.
 */
#ifndef NSGPU_H
#define NSGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

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

/* nsg_raycast flags */
#define NSG_RAYCAST_STATUS 1            /* status map: Build_status_map = true */
#define NSG_RAYCAST_TRIANGULATION 2     /* accurate-triangulation rays: Accurate_Triangulation = true */
#define NSG_RAYCAST_EPSMAP 4            /* epsilon and ideb maps: Build_epsilon_maps = true (node rays of all three panels) */
#define NSG_RAYCAST_KEEP_HITS 16        /* keep per-ray sorted hits for nsg_download_hits */
#define NSG_RAYCAST_GRAD 32             /* adjoint: d volume (and d area of the next nsg_triangulate) / d patch */
#define NSG_RAYCAST_NORMALS 64          /* keep the hits' patches for analytic vertex normals (Compute_Vertex_Normals) */

/* Gradient slots per patch (nsg_patch_grads): point (cx, cy, cz, r), facet (px, py, pz),
 * edge (tcx, tcy, tcz, ux, uy, uz, R); unused slots are 0. */
#define NSG_GRAD_PER_PATCH 8

/* precision of nsg_raycast */
#define NSG_PRECISION_FP64 0
#define NSG_PRECISION_MIXED 1

/* Grid environment; replaces the grid members of DelPhiShared (src/DelphiShared.h:151-213).
 * Node i of an axis sits at min + i*side. */
typedef struct NsGrid {
  int64_t nx, ny, nz;
  double xmin, ymin, zmin;
  double xmax, ymax, zmax;
  double scale, side, hside, A;
  double rmaxdim;
  double baricenter[3];
} NsGrid;

/* Patch set layout (host builder output, ray caster input).
 *   f64 : 20 doubles per patch: [0..2] bounding-sphere centre, [3] radius, [4..6] torus centre,
 *         [7] torus major radius, [8] spindle self-intersection radius (<0: none),
 *         [9..17] inverse torus frame (row major), [18..19] unused
 *   i32 : 4 ints per patch: kind (0 point, 1 regular edge, 2 singular edge, 3 regular facet,
 *         4 singular facet), first pool entry, pool entry count, unused
 *   pool: 4 doubles per entry: clipping sphere (x, y, z, r^2) for points, plane (a, b, c, d)
 *         for facets and edges (a point with a*x+b*y+c*z+d > 0 is cut away)
 *   pool_flag: 1 byte per entry; for edges, 1 on the first plane of an acute pair.
 * Mirrors the cell records of src/ConnollySurface.h:31-167.
 *
 * Skin cells (kinds 5 Del0 / reduced Voronoi cell, 6 Del1 / edge prism, 7 Del2 / facet prism,
 * 8 Del3 / reduced tetrahedron; the MixedCell records of src/SkinSurface.h:18-105):
 *   f64 : [0..2] local origin (Del0: the atom centre, else the centre of the cell's box),
 *         [3] Del0: atom radius (equatorial-disc culling), else half the box diagonal,
 *         [4..13] quadric q11, q22, q33, q44, q12, q23, q34, q13, q24, q14 (the reference's coding,
 *         src/SkinSurface.cpp:4461), [14..16] box low corner, [17..19] box high corner
 *   pool: the cell's planes (a, b, c, d); a point with a*x+b*y+c*z+d > 0 is outside the cell
 *         (Del0 planes are stored negated, which turns the reference's "< 0" test into this one). */

typedef struct nsg_ctx nsg_ctx;
typedef struct NsPatchSet NsPatchSet;

/* ---- grid environment (host) ---- */
/* DelPhiShared::buildGrid (src/DelphiShared.cpp:1038-1201). */
int nsg_grid_build(const double* atoms_xyzr, int64_t n_atoms, double scale, double perfil, NsGrid* out);
/* randnum (src/tools.cpp:64-81); *seed is the generator state (1234 initially, src/tools.h:1827). */
double nsg_randnum(int64_t* seed);
/* Atom jitter of buildConnollyCGAL (src/ConnollySurface.cpp:2484-2488). */
int nsg_jitter_atoms(double* atoms_xyzr, int64_t n_atoms, double displacement, int64_t* seed);
/* xyzr reading of DelPhiShared::loadAtoms (src/DelphiShared.cpp:309-704); out == NULL counts. */
int64_t nsg_read_xyzr(const char* path, double* out, int64_t capacity);
/* The ATOM / HETATM records of a pqr file (DelPhiShared::loadAtoms for ".pqr" names,
 * src/DelphiShared.cpp:365-415, 520-545): x, y, z, radius per atom, atoms with a radius below
 * 1e-20 skipped; NSG_ERR_ARG on a malformed record (where the reference exits). */
int64_t nsg_read_pqr(const char* path, double* out, int64_t capacity);

/* ---- patch construction (host) ---- */
/* ConnollySurface::build / buildConnollyCGAL (src/ConnollySurface.cpp:256, 2326-3316). */
int nsg_ses_build(const double* atoms_xyzr, int64_t n_atoms, double probe_radius, int n_threads, NsPatchSet** out);
/* SkinSurface::build / buildSkinCGAL (src/SkinSurface.cpp:329, 1271-1812): the mixed cells of
 * atoms weighted r^2/s (jittered beforehand, nsg_jitter_atoms) plus the reference's six dummy
 * points, with shrink factor s in (0, 1); the regular triangulation is this library's own (exact
 * predicates), not CGAL's.  NSG_ERR_GEOMETRY flags a degenerate configuration (patches are still
 * returned). */
int nsg_skin_build(const double* atoms_xyzr, int64_t n_atoms, double shrink, int n_threads, NsPatchSet** out);
/* Exact predicates of that triangulation on integer points (x, y, z, w; 5 points): orientation of
 * points 0..3 (+1, 0, -1) and whether point 4 conflicts with their orthosphere (tests). */
int nsg_skin_predicates(const int64_t* points, int* orient, int* conflict);
int nsg_patchset_info(const NsPatchSet* ps, int64_t* n_patches, int64_t* n_pool, int64_t counts[5]);
/* Patches per kind, counts[k] for k < n (kinds 0..8: the five SES kinds, then the four skin cells). */
int nsg_patchset_kind_counts(const NsPatchSet* ps, int64_t* counts, int n);
int nsg_patchset_export(const NsPatchSet* ps, double* f64, int32_t* i32, double* pool, int8_t* pool_flag);
/* The atoms every patch depends on, 3 per patch (-1 unused): point (i), facet (i, j, k), edge (i, j). */
int nsg_patchset_atoms(const NsPatchSet* ps, int32_t* out);
void nsg_patchset_free(NsPatchSet* ps);
/* Chain rule of the adjoint, no counterpart in the reference (which has no derivatives):
 * grad_atoms (n_atoms x 4: x, y, z, r) += d out / d atoms from per-patch parameter derivatives
 * gpatch (n_patches x NSG_GRAD_PER_PATCH), for patches built from atoms_xyzr (after jitter). */
int nsg_ses_chain_grad(const double* atoms_xyzr, int64_t n_atoms, double probe_radius, int64_t n_patches,
                       const int32_t* i32, const double* f64, const int32_t* patch_atoms, const double* gpatch,
                       double* grad_atoms);

/* ---- files in the reference's layouts (host) ---- */
/* DelPhiShared::saveStatus (src/DelphiShared.cpp:1458-1502): "%d " per node, i outer, k inner. */
int nsg_write_status(const char* path, const int32_t* status, int64_t nx, int64_t ny, int64_t nz);
/* DelPhiShared::saveCavities (src/DelphiShared.cpp:1889-1946): cavities.txt and cavitiesSize.txt. */
int nsg_write_cavities(const char* cavities_path, const char* sizes_path, const int32_t* status, const NsGrid* grid,
                       int32_t n_cavities, const double* sizes, const int32_t* filled);
/* DelPhiShared::saveCavities' cavAtomsSerials.txt (src/DelphiShared.cpp:1946-1962): one line per
 * cavity, its atoms' serials ("%d " each; the atom index + 1 unless serials gives a positive
 * serial), cavities with skip[c] != 0 left out (skip may be NULL: onlySaveNonFilled = false). */
int nsg_write_cavity_atoms(const char* path, int32_t n_cavities, const int32_t* offsets, const int32_t* atoms,
                           const int32_t* serials, int64_t n_atoms, const int32_t* skip);
/* Surface::saveMesh (src/Surface.cpp:10857-11052): format 0 = root.off + roottriangleAreas.txt,
 * 1 = root.ply (binary); revert writes every triangle in the opposite winding. */
int nsg_write_mesh(const char* root, int format, const double* vertices, int64_t n_vertices, const int32_t* triangles,
                   int64_t n_triangles, int revert);
/* Vertex normals of a mesh by triangle averaging: approximateNormals for a surface without analytic
 * normals (src/Surface.cpp:10588-10660): the normalised sum of the unnormalised plane normals
 * (plane3points, src/tools.cpp:258-274) of each vertex's triangles; 3 doubles per vertex. */
int nsg_mesh_normals(const double* vertices, int64_t n_vertices, const int32_t* triangles, int64_t n_triangles,
                     double* normals);
/* Nearest atom of every vertex (vdwAccessible, src/Surface.cpp:16663-16715): least power distance
 * |p - c|^2 - r^2 over all atoms (4 doubles each), ties to the lower index; 0-based, -1 without
 * atoms. */
int nsg_vertex_atoms(const double* vertices, int64_t n_vertices, const double* atoms_xyzr, int64_t n_atoms,
                     int32_t* vertex_atoms);
/* Surface::saveMesh with vertex attributes (src/Surface.cpp:10857-11062): format 0 = OFF+N,
 * 1 = MSMS without nearest atoms (root.face, root.vert), 2 = OFF+A, 3 = OFF+N+A, 4 = MSMS; normals
 * for 0, 1, 3, 4, vertex_atoms (0-based) for 2, 3, 4 (may be NULL otherwise); every format adds
 * roottriangleAreas.txt. */
int nsg_write_mesh_attrs(const char* root, int format, const double* vertices, const double* normals,
                         const int32_t* vertex_atoms, int64_t n_vertices, const int32_t* triangles,
                         int64_t n_triangles, int revert);

/* ---- device context ---- */
int nsg_version(void);
const char* nsg_last_error(void);
int nsg_ctx_create(int device, nsg_ctx** out);
int nsg_ctx_destroy(nsg_ctx* ctx);
int nsg_set_stream(nsg_ctx* ctx, void* cuda_stream);
void* nsg_get_stream(nsg_ctx* ctx);
/* Grid of the surface (the DelPhiShared* the reference Surface holds, src/Surface.h:572). */
int nsg_set_grid(nsg_ctx* ctx, const NsGrid* grid);
/* Patch set from host memory (the sesComplex of src/ConnollySurface.h). */
int nsg_upload_patches(nsg_ctx* ctx, int64_t n, const double* f64, const int32_t* i32, int64_t n_pool,
                       const double* pool, const int8_t* pool_flag, double probe_radius);
/* Patch set already resident in device memory (no copy). */
int nsg_bind_patches_device(nsg_ctx* ctx, int64_t n, const double* f64, const int32_t* i32, int64_t n_pool,
                            const double* pool, const int8_t* pool_flag, double probe_radius);

/* ---- batches (many structures, each on its own grid, in the same launches) ----
 * No single counterpart in the reference, which builds one Surface per structure; a batch of n
 * runs the same per-structure pipeline (one getSurf + triangulateSurface each) with every kernel
 * launch covering all n structures.  nsg_set_batch replaces the grid set by nsg_set_grid (which
 * is a batch of one).  Cavity detection and the dense status map stay single-structure calls;
 * insideness bits download concatenated (structure b's words follow those of b-1), and the mesh
 * arrays hold all structures' vertices (analytic ones of every structure, then the midpoint
 * ones) with batch-wide indices. */
int nsg_set_batch(nsg_ctx* ctx, int32_t n, const NsGrid* grids);
/* Concatenated patch sets: structure b owns patches [patch_off[b], patch_off[b+1]) and pool
 * entries [pool_off[b], pool_off[b+1]); pool indices inside each record are local to its
 * structure (as nsg_patchset_export writes them). */
int nsg_upload_batch(nsg_ctx* ctx, const int64_t* patch_off, const double* f64, const int32_t* i32,
                     const int64_t* pool_off, const double* pool, const int8_t* pool_flag, double probe_radius);
/* Per-structure volume (last nsg_raycast) and area (last nsg_triangulate); either may be NULL. */
int nsg_batch_results(nsg_ctx* ctx, double* volumes, double* areas);

/* ---- launch-shape tuning (no counterpart in the reference) ----
 * params: [intersection threads per block (64..256), intersection blocks per SM (1..64),
 * candidate-kernel threads per block (32..256), and optionally (n >= 4) the ray sets on concurrent
 * streams (1, default) or not, (n >= 5) the torus candidates split by resolvent branch before
 * the solve (1) or not (0, default: measured slower on the ensemble), and (n >= 6) the blocks per
 * SM of the marching-cubes triangle kernel (3, default, or 4); results do not depend on any of
 * them].  nsg_autotune times
 * `reps` ray casts of the current batch per candidate shape and keeps the fastest in the
 * context. */
int nsg_set_tuning(nsg_ctx* ctx, const int32_t* params, int n);
int nsg_get_tuning(nsg_ctx* ctx, int32_t* params, int n);
int nsg_autotune(nsg_ctx* ctx, int flags, int precision, int reps, double* best_ms);

/* ---- adjoint (no counterpart in the reference) ----
 * After nsg_raycast with NSG_RAYCAST_GRAD (and the nsg_triangulate that follows it): the
 * derivatives of the volume and of the area with respect to every patch's surface parameters,
 * NSG_GRAD_PER_PATCH doubles per patch in upload order (batch: all structures, concatenated).
 * Each hit x on its ray axis e moves by ds = -(dF/dtheta . dtheta) / (dF/dx . e) on the patch
 * surface F = 0; the volume sums them over interval ends, the area over analytic vertices. */
int nsg_patch_grads(nsg_ctx* ctx, double* d_volume, double* d_area);
/* The atoms behind the uploaded patches (after jitter; structure b owns [atom_off[b],
 * atom_off[b+1])) and the 3 structure-local atoms of every patch (nsg_patchset_atoms). */
int nsg_upload_atoms(nsg_ctx* ctx, const int64_t* atom_off, const double* atoms_xyzr, const int32_t* patch_atoms);
/* d volume and d area of every structure with respect to its atoms' x, y, z, r (n_atoms x 4 each),
 * chained from the patch derivatives on the device; either pointer may be NULL. */
int nsg_atom_grads(nsg_ctx* ctx, double* d_volume, double* d_area);

/* ---- blobby surface (BlobbySurface, src/BlobbySurface.cpp:83-229) ----
 * The atoms' Gaussian field sum exp(B (d^2/r^2 - 1)) (cut-off 6 A) on the context's grid, its
 * marching-cubes mesh at iso level 1 (src/Surface.cpp:8143-8327, 9075-9318), one Laplacian
 * smoothing pass (src/Surface.cpp:13089-13354) and the reference's OFF text round trip (vertices
 * written "%.3f", read back as floats, src/MeshSurface.cpp:2350-2479), all on the device; the
 * mesh's triangles (patch kind 9) become the context's patch set, ray cast like a MeshSurface
 * (src/MeshSurface.cpp:1487-1855).  blobbyness < 0.  flags: NSG_BLOBBY_DIFFERENTIABLE skips the
 * round trip (which is piecewise constant in the atoms) so that nsg_blobby_atom_grads applies. */
#define NSG_BLOBBY_DIFFERENTIABLE 1
int nsg_blobby_build(nsg_ctx* ctx, const double* atoms_xyzr, int64_t n_atoms, double blobbyness, int flags);
/* The mesh of the last nsg_blobby_build: vertex and triangle counts, vertices (3 doubles) and
 * triangles (3 ints); NULL buffers only report the counts. */
int nsg_blobby_mesh(nsg_ctx* ctx, int64_t* n_vertices, int64_t* n_triangles, double* vertices, int32_t* triangles);
/* d volume and d area of a NSG_BLOBBY_DIFFERENTIABLE blobby surface with respect to its atoms'
 * x, y, z, r (n_atoms x 4 each), after nsg_raycast with NSG_RAYCAST_GRAD (and nsg_triangulate for
 * the area): hit terms on the triangles, the smoothing, the interpolated vertices and the field,
 * chained on the device (no counterpart in the reference); either pointer may be NULL. */
int nsg_blobby_atom_grads(nsg_ctx* ctx, double* d_volume, double* d_area);

/* ---- the hot path ---- */
/* Ray casting of Surface::getSurf: getPatchIntersectionData (src/ConnollySurface.cpp:4319-4590),
 * pixel binning and sort (src/Surface.cpp:4766-5095), setVerticesAndGridsWithIntersectionData
 * (src/Surface.cpp:5101-6251) and the volume (src/Surface.cpp:1680-1684). */
int nsg_raycast(nsg_ctx* ctx, int flags, int precision, double* volume);
/* getCavitiesWithBilevelStatusMap + fillCavities (src/Surface.cpp:1994-2126, 2355-2484). */
int nsg_cavities(nsg_ctx* ctx, double cavity_volume, int* n_cavities);
/* Water-shape filter of the cavities that nsg_cavities kept, Keep_Water_Shaped_Cavities
 * (filterCavitiesWithBilevelStatusMap, src/Surface.cpp:3011-3290; called by getSurf at
 * src/Surface.cpp:1128-1139): the nodes of a cavity that no probe sphere of radius probe_radius
 * fitting inside the cavity covers are removed, i.e. their insideness bits, epsilon and ideb
 * entries filled as fillCavities does.  The status map takes the reference's codes: -(4 + c) for
 * the support nodes of cavity c, 4 + c for the covered ones, and for the removed ones
 * STATUS_POINT_INSIDE when modify_status is set, else -3 (SHAPE_UNDER_CHECK) or -2 (SHAPE_OK,
 * inside a support sphere of a later cavity).  A cavity whose nodes are all removed becomes
 * filled (nsg_download_cavities); nsg_cavity_atoms keeps the cavity membership from before the
 * filter.  Once per nsg_cavities; n_removed (may be NULL) receives the removed node count. */
int nsg_filter_cavities(nsg_ctx* ctx, double probe_radius, int modify_status, int64_t* n_removed);
/* Pocket detection by difference, the step `(*surf1) -= (*surf2)` of pocket mode followed by
 * fillCavities (src/main.cpp:1533, 1586; Surface::operator-= src/Surface.cpp:15556-15619).
 * ctx holds the fat-probe surface and small the small-probe one, both ray cast on the same grid
 * (cavity detection on either is optional: its cavities then count as inside, as the reference's
 * cavity codes do).  Surface::difference (src/Surface.cpp:11471-11717) marks the nodes inside the
 * fat surface and outside the small one as one cavity and every other node inside; the water-shape
 * filter with a 1.4 A probe and the status map modified (nsg_filter_cavities) keeps the part a
 * water molecule fits in; cav2out returns it to TEMPORARY_OUT, and its 6-connected regions become
 * the pockets 4, 5, ... in the reference's alternating-z seed order; pockets of at most
 * fill_volume A^3 are filled.  Afterwards ctx is in the state nsg_cavities leaves (pocket sizes and
 * flags from nsg_download_cavities, nsg_cavity_atoms, nsg_download_status, insideness bits).
 * The epsilon and ideb maps are left as the reference leaves them (not differenced).  Linking of
 * split pockets (linkCavities) is not part of this call. */
int nsg_pocket_difference(nsg_ctx* ctx, nsg_ctx* small, double fill_volume, int* n_pockets);
/* Label order of the alternating-z seed scan of getCavitiesWithBilevelStatusMap
 * (src/Surface.cpp:2044-2116) over regions sorted by first node; host only. */
int nsg_cavity_order(int32_t n_regions, const uint32_t* desc_key, int32_t* label_out);
/* assembleVerticesList + triangulateSurface (src/Surface.cpp:7415-7667, 9909-10526). */
int nsg_triangulate(nsg_ctx* ctx, double* area, int64_t* n_vertices, int64_t* n_triangles);

/* ---- results into caller-owned host buffers ---- */
/* Vertex normals of the last nsg_triangulate (after nsg_raycast with NSG_RAYCAST_NORMALS or
 * NSG_RAYCAST_GRAD), 3 doubles per vertex: analytic vertices get their patch's normal
 * (ConnollySurface::getNormal, src/ConnollySurface.cpp:5736-5819; the skin quadric's gradient,
 * src/SkinSurface.cpp:3684-3712), the others the triangle average of approximateNormals
 * (src/Surface.cpp:10420-10460, 10588-10735). */
int nsg_vertex_normals(nsg_ctx* ctx, double* normals);
/* Host: the vertices whose normal is (0, 0, 0) get the triangle-averaged normal (approximateNormals
 * for the listed vertices, src/Surface.cpp:10660-10735). */
int nsg_fill_zero_normals(const double* vertices, int64_t n_vertices, const int32_t* triangles, int64_t n_triangles,
                          double* normals);
/* Status map, flat int32 k*ny*nx + j*nx + i (read3DVector layout, src/tools.h:549-575). */
int nsg_download_status(nsg_ctx* ctx, int32_t* dst);
/* 32x-packed insideness bits, bit = 1 outside (src/tools.h:1324-1414); ceil(nx/32)*ny*nz words. */
int nsg_download_insideness(nsg_ctx* ctx, uint32_t* dst);
/* Vertices (3 doubles), their grid edges (ix, iy, iz, dir) and triangles (3 ints):
 * vertList / triList of Surface (src/Surface.h). */
int nsg_download_mesh(nsg_ctx* ctx, double* vertices, int32_t* vertex_edges, int32_t* triangles);
/* cavitiesSize / cavitiesFlag of DelPhiShared (src/DelphiShared.h:160-213). */
int nsg_download_cavities(nsg_ctx* ctx, double* sizes, int32_t* filled);
/* Atoms lining each cavity of the last nsg_cavities: DelPhiShared::cav2atoms as
 * Surface::getCavitiesAtomsWithBilevelStatusMap fills it (src/Surface.cpp:2249-2346).  Every node
 * of cavity c (status 4 + c) with a 6-neighbour of another status (outside the grid counts as
 * status 2) contributes the atom of least |a - x|^2 - r^2 among the atoms of the 27 cells around
 * it in the reference's atom grid (buildAtomsMap, src/Surface.cpp:1695-1749: side 2 r_max, halved
 * until it spans 1.3 rmaxdim in at most 100 cells, centred on the grid's barycentre), the first
 * of equal ones in cell order, or -1 when those cells hold no atom.  atoms_xyzr: the structure's
 * atoms (x, y, z, radius).  Per cavity, its distinct atoms ascending (std::set order, -1 first) at
 * offsets[c] .. offsets[c + 1] of atoms (n_cav + 1 offsets); with atoms == NULL only *n_total is
 * set.  The result is kept until the next cast or cavity detection. */
int nsg_cavity_atoms(nsg_ctx* ctx, const double* atoms_xyzr, int64_t n_atoms, int32_t* offsets, int32_t* atoms,
                     int64_t* n_total);
/* Sorted hit parameters per ray of one ray set (tests); sets 0 status, 1..3 accurate triangulation,
 * 4 and 5 the epsilon-map node rays along z and y. */
int nsg_download_hits(nsg_ctx* ctx, int ray_set, int32_t* counts, double* dst, int64_t dst_capacity);

/* ---- epsilon maps and boundary grid points (Build_epsilon_maps, Project_boundary_grid_points) ---- */
/* Epsilon map of the last nsg_raycast with NSG_RAYCAST_EPSMAP (single structure), cavity-filled
 * when nsg_cavities ran after it: DelPhiShared::epsmap, int32 ((k*ny + j)*nx + i)*3 + axis, the
 * code of the grid edge from node (i, j, k) to its neighbour along the axis: 0 outside, 5 inside
 * (the node-ray fill of src/Surface.cpp:6645-6680, 6786-6795, 6887-6896; fillCavities
 * src/Surface.cpp:2400-2417). */
int nsg_download_epsmap(nsg_ctx* ctx, int32_t* dst);
/* ideb map (DelPhiShared::idebmap), 1 byte per node, (k*ny + j)*nx + i: 0 inside the surface or in
 * a filled cavity, 1 elsewhere (src/Surface.cpp:6655-6663, 2416). */
int nsg_download_idebmap(nsg_ctx* ctx, uint8_t* dst);
/* Boundary grid points of the epsilon map (src/Surface.cpp:1488-1546: nodes whose six edge codes
 * differ, scan order z, y, x) and, with project != 0, the projection of the external ones onto an
 * SES (Surface::projector, src/Surface.cpp:4657-4676; ConnollySurface::getProjection,
 * src/ConnollySurface.cpp:5822-5912, over the auxiliary grid of buildAuxiliaryGrid,
 * src/ConnollySurface.cpp:3666-3900, aux_max_dim = Max_ses_patches_auxiliary_grid_size, 50 by
 * default), or onto a mesh surface (the blobby surface's triangles: MeshSurface::getProjection,
 * src/MeshSurface.cpp:2045-2141, point2triangle :1864-2008, over the triangles' vertex boxes on
 * the auxiliary grid of MeshSurface::buildAuxiliaryGrid :729-935, aux_max_dim =
 * Max_mesh_auxiliary_grid_size, 100 by default).  Skin cells are not projected (NSG_ERR_STATE).
 * Internal points (different dielectrics) do not arise with one inside code. */
int nsg_bgp(nsg_ctx* ctx, int project, int32_t aux_max_dim, int64_t* n_bgp, int64_t* n_external);
/* The points of the last nsg_bgp: ibgp (ix, iy, iz), type (1 external, 0 internal), scspos /
 * scsnor (3 doubles; the reference leaves an external SES point's normal at 0, a mesh point gets
 * its triangle's normal) and the projection flag (0 projected, 1 for the SES no feasible
 * projection among the cell's patches: the point is kept, for a mesh the nearest point lies on a
 * triangle's edge or corner (the reference's getProjection returns false; the point is still
 * projected), 2 empty auxiliary cell, 3 internal); any pointer may be NULL. */
int nsg_download_bgp(nsg_ctx* ctx, int32_t* ibgp, int32_t* type, double* scspos, double* scsnor, int32_t* flag);

/* ---- allocation-free status ray cast ----
 * No counterpart in the reference: an addition for callers that may not allocate device memory
 * (a host framework that owns every device allocation through its own pool, or a process whose
 * memory is fixed after start-up).  Status map (flat int32, k*ny*nx + j*nx + i; INSIDE /
 * TEMPORARY_OUT as nsg_raycast with NSG_RAYCAST_STATUS writes it) and status-ray volume of a grid
 * from a patch set, all in device memory the caller owns.  Scratch is one fixed file-scope device
 * array (16.5 MiB): at most 65536 status rays (ny * nz) and 32 hits per ray; larger grids return
 * NSG_ERR_CAPACITY before any launch, a ray with more hits returns NSG_ERR_CAPACITY after the
 * launches and leaves the status map unspecified.  SES patch sets only (a skin cell returns
 * NSG_ERR_ARG); d_pool and d_pool_flag may be NULL only when no patch has pool entries (else
 * NSG_ERR_ARG).  Allocates nothing.  Every call looks up the
 * scratch address on the current device; under lazy module loading the first call in a process
 * reserves the array, so a process with fixed device memory makes one call at start-up.  A call
 * synchronises `stream` and reads its result back, so it cannot be made while any stream is
 * being captured.  Calls that overlap on the GPU share the scratch and race: serialise them. */
int nsg_status_noalloc(const NsGrid* grid, int64_t n_patches, const double* d_f64, const int32_t* d_i32,
                       const double* d_pool, const int8_t* d_pool_flag, double probe_radius, int32_t* d_status,
                       double* volume, void* stream);

/* ---- instrumentation ---- */
int nsg_stats(nsg_ctx* ctx, int64_t* out, int n);
double nsg_volume(nsg_ctx* ctx);
double nsg_area(nsg_ctx* ctx);
int nsg_event_record(nsg_ctx* ctx, int slot);
int nsg_event_elapsed(nsg_ctx* ctx, int slot_a, int slot_b, double* ms);
int nsg_profile(nsg_ctx* ctx, int enable);
int nsg_stage_times(nsg_ctx* ctx, double* ms, int64_t* calls, int n);
int64_t nsg_launch_count(nsg_ctx* ctx);
/* Counters of the last profiled ray cast: candidates, torus candidates, mixed-precision fallbacks
 * (near-tangent sphere, quartic isolation, root polish), feasibility re-evaluations. */
int nsg_trace_counters(nsg_ctx* ctx, int64_t* out, int n);
/* Peak FP64 (precision 0) or FP32 (1) rate of the GPU, measured with FMA chains (flop/s). */
int nsg_fp_peak(nsg_ctx* ctx, int precision, double* flops_per_s);

#ifdef __cplusplus
}
#endif

#endif /* NSGPU_H */
