// Shared plain-old-data layouts of the grid-ray-casting surface builder.
// Included by the host patch builders, the C-ABI layer and the sm_100a kernels,
// so it must stay C/C++/CUDA neutral (no STL, no torch).
#pragma once
#include <stdint.h>

#ifdef __CUDACC__
#define NS_HD __host__ __device__ __forceinline__
#else
#define NS_HD inline
#endif

// Patch kinds.  They mirror the reference cell classes:
//   POINT      -> PointCell  (exposed atom sphere, clipped by neighbour spheres)
//   EDGE_REG   -> EdgeCell REGULAR_EDGE_CELL  (torus sector bounded by plane pairs)
//   EDGE_SING  -> EdgeCell SINGULAR_EDGE_CELL (full torus)
//   FACE_REG   -> FacetCell REGULAR_FACE_CELL (re-entrant probe patch, 3 trimming planes)
//   FACE_SING  -> FacetCell SINGULAR_FACE_CELL (probe patch, 4 trimming planes)
// (src/ConnollySurface.h:31-167, cell type tags src/Surface.h).
enum NsPatchKind {
  NS_POINT = 0,
  NS_EDGE_REG = 1,
  NS_EDGE_SING = 2,
  NS_FACE_REG = 3,
  NS_FACE_SING = 4,
  // Skin mixed cells (src/SkinSurface.h:18-105): a quadric patch inside a convex cell bounded by
  // planes.  Del0Cell (reduced Voronoi cell of an atom), Del1Cell (Delaunay edge x Voronoi face),
  // Del2Cell (Delaunay facet x Voronoi edge), Del3Cell (reduced tetrahedron).
  NS_SKIN_POINT = 5,
  NS_SKIN_EDGE = 6,
  NS_SKIN_FACET = 7,
  NS_SKIN_TETRA = 8,
  // Triangle of a mesh surface (MeshSurface, src/MeshSurface.h): the blobby surface is ray cast as
  // the triangle mesh of its scalar field (src/BlobbySurface.cpp:83-229).
  NS_MESH_TRI = 9
};
#define NS_KIND_COUNT 10

// Skin cell record (NS_PATCH_F64 doubles):
//   [0..2]  local origin: the atom centre (Del0), else the centre of the cell's bounding box
//   [3]     atom radius (Del0, equatorial-disc culling), else half the box diagonal
//   [4..13] quadric Q in the reference's coding (src/SkinSurface.cpp:4461):
//           q11, q22, q33, q44, q12, q23, q34, q13, q24, q14 (x^T Q x = 0, x homogeneous)
//   [14..16] bounding box low corner, [17..19] high corner (the reduced points' box, or the atom
//           sphere's box for Del0), as the reference's culling computes them
// Pool: the cell's planes (a, b, c, d); a point with a*x+b*y+c*z+d > 0 is outside the cell (the
// planes of Del0 cells are stored negated, which flips the reference's "< 0" test exactly).
#define NS_SKIN_Q 4
#define NS_SKIN_LO 14
#define NS_SKIN_HI 17
NS_HD bool ns_is_skin(int kind) { return kind >= NS_SKIN_POINT && kind <= NS_SKIN_TETRA; }

// Mesh triangle record (NS_PATCH_F64 doubles): [0..2] vertex 0, [3..5] vertex 1, [6..8] vertex 2,
// [9..11] the unnormalised normal (v1 - v0) x (v2 - v0), [14..16] / [17..19] the triangle's box
// (the NS_SKIN_LO / NS_SKIN_HI slots).  No pool entries.  The patch's three "atoms" are its mesh
// vertex indices.
#define NS_TRI_N 9
// Patches culled by a stored box (skin cells, mesh triangles) rather than their bounding sphere.
NS_HD bool ns_has_box(int kind) { return kind >= NS_SKIN_POINT; }

// Per-patch double record (NS_PATCH_F64 doubles per patch).
//   [0..2] bounding-sphere centre, [3] bounding-sphere radius
//          POINT: atom centre / radius; EDGE: clipping sphere; FACE: probe sphere
//   [4..6] torus centre (EDGE only)
//   [7]    torus major radius (EDGE only)
//   [8]    spindle self-intersection radius, < 0 when the torus is not spindle (EDGE)
//   [9..17] inverse torus frame rotation, row major (EDGE)
//   [18..19] unused
#define NS_PATCH_F64 20
// Per-patch int record (NS_PATCH_I32 ints per patch): kind, first pool entry, pool entry count, unused.
#define NS_PATCH_I32 4
// Per-patch surface-parameter gradient slots: point (cx, cy, cz, r), facet (px, py, pz),
// edge (tcx, tcy, tcz, ux, uy, uz, R).
#define NS_GRAD_PER_PATCH 8

// Pool entries are 4 doubles.
//   POINT: clipping sphere (cx, cy, cz, r^2); a point strictly inside any of them is infeasible.
//   FACE : plane (a, b, c, d); a point with a*x+b*y+c*z+d > 0 is infeasible.
//   EDGE : plane pairs (2 consecutive entries).  pool_flag[first entry of the pair] = 1 for an
//          acute pair (feasible iff both tests <= 0), 0 for an obtuse pair (feasible iff either
//          test <= 0).  A point is feasible if any pair accepts it; a pair-less EDGE accepts all.

// Status codes of the status map (src/DelphiShared.h:22-33).
#define NS_STATUS_INSIDE (-1)
#define NS_STATUS_TEMPORARY_OUT 2
#define NS_STATUS_OUT 3
#define NS_STATUS_FIRST_CAV 4
// water-shape filter codes (src/DelphiShared.h:22-23)
#define NS_STATUS_SHAPE_UNDER_CHECK (-3)
#define NS_STATUS_SHAPE_OK (-2)

// Epsilon-map code of the inside medium: every surface type sets inside = 5
// (src/ConnollySurface.cpp:214, src/SkinSurface.cpp:200, src/BlobbySurface.cpp:18,
// src/MeshSurface.cpp:188); outside edges keep 0.
#define NS_EPS_INSIDE 5
// Boundary grid point types (src/Surface.h:294-295).
#define NS_INTERNAL_BGP 0
#define NS_EXTERNAL_BGP 1

// Tolerances of the reference (src/Surface.h:285-291).
#define NS_EPS_INT 1e-8
#define NS_DELTA 1e-10

// Edge directions of marching-cubes vertices.
#define NS_X_DIR 0
#define NS_Y_DIR 1
#define NS_Z_DIR 2

typedef struct NsGrid {
  int64_t nx, ny, nz;
  double xmin, ymin, zmin;
  double xmax, ymax, zmax;
  double scale, side, hside, A;
  double rmaxdim;
  double baricenter[3];
} NsGrid;

// Grid coordinate of node i along an axis: min + i*side (src/DelphiShared.cpp:1155-1162).
NS_HD double ns_coord(double vmin, double side, int64_t i) { return vmin + (double)i * side; }
