// Device-side pipeline of the SES grid ray caster: shared parameter blocks and kernel launchers.
// Kernels live in trace.cu (patch windows, tile binning, ray tracing + interval fill),
// cavity.cu (connected components of the status map, cavity filling) and mc.cu (vertex
// assembly and marching cubes); capi.cu drives them.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../ns_types.h"

namespace nsg {

// Ray tile handled by one CTA: 32 consecutive pixels along the first panel axis (one per lane)
// times 4 rows along the second axis (one per warp).
constexpr int kTileM = 32;
constexpr int kTileN = 4;
constexpr int kTraceThreads = kTileM * kTileN;
// Hits kept on chip per ray; rays with more hits are re-traced by the overflow path.
constexpr int kHitCap = 32;
// Hits per ray on the overflow path.
constexpr int kOverflowCap = 2048;

// Ray sets: 0 = status rays along x (panel 0, through grid nodes); 1..3 = accurate
// triangulation rays of panels 0 (x), 1 (z), 2 (y), shifted by DELTA - hside; 4, 5 = the node rays
// of panels 1 (z) and 2 (y) that the epsilon maps add (the reference's node-ray pass over all
// three panels when Build_epsilon_maps is set, src/Surface.cpp:6318-6340).
constexpr int kRaySets = 6;
struct RaySet {
  int set;      // 0..5
  int panel;    // 0..2
  int fd, ld, vc;  // first pixel axis (m), second pixel axis (n), ray axis
  int64_t nb, na;  // pixel counts along m and n
  double delta;
  int64_t ordinal_base;  // first ray ordinal of this set in the accurate-triangulation order
};

struct GridDev {
  int64_t n[3];
  double mn[3];
  double mx[3];
  double scale, side, hside;
};

// One structure of a batch: its grid and where its tiles, rays, bits and cube rows start in the
// batch-wide arrays.  A single structure is a batch of one with every base 0.
struct StructDev {
  GridDev g;
  int64_t nwords;        // words of its 32x-packed insideness bit grid
  int64_t word_base;     // first word in the batch's bit array
  int64_t tile_base[3];  // first tile of each panel in the panel's tile arrays
  int64_t ray_base[kRaySets];  // first ray of each ray set in the set's ray arrays
  int64_t mc_base;       // first accurate-triangulation ray ordinal (its 3 panels are contiguous)
  int64_t row_base;      // first marching-cubes row ((NY-2)*(NZ-2) rows per structure)
  int64_t aword_base;    // first entry of its active-cube map (ceil((NX-2)/32) per cube row)
  double A;              // side^2: the area of one pixel, volume weight of an interval length
  double ray_dir[3];     // ray length along each axis: coordinate of the last node minus the first
  double inv_dir[3];     // 1 / ray_dir
  double box_dir[3];     // max - min of each axis: the skin tracer's ray-parameter unit
};

// Batch-wide lookup tables.  The *_base arrays hold n+1 entries (the last is the total), for a
// binary search from a batch-wide index to its structure.
struct BatchDev {
  int32_t n;
  const StructDev* s;
  const int32_t* patch_struct;    // structure of every patch
  const int32_t* tile_struct[3];  // structure of every tile of each panel
  const int64_t* ray_base[kRaySets];  // n+1 per ray set
  const int64_t* mc_base;         // n+1
  const int64_t* row_base;        // n+1
};

// Largest b with base[b] <= x (base ascending, base[0] = 0).
__device__ __forceinline__ int find_struct(const int64_t* __restrict__ base, int n, int64_t x) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (base[mid] <= x) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Panel of a ray set, and whether its origins are shifted off the grid nodes.
__host__ __device__ inline int ray_set_panel(int set) { return set == 0 ? 0 : (set <= 3 ? set - 1 : set - 3); }
__host__ __device__ inline bool ray_set_shifted(int set) { return set >= 1 && set <= 3; }

__host__ __device__ inline RaySet make_ray_set(int set, const GridDev& g) {
  RaySet r;
  r.set = set;
  r.panel = ray_set_panel(set);
  if (r.panel == 0) { r.fd = 1; r.ld = 2; r.vc = 0; }
  else if (r.panel == 1) { r.fd = 0; r.ld = 1; r.vc = 2; }
  else { r.fd = 0; r.ld = 2; r.vc = 1; }
  r.nb = g.n[r.fd];
  r.na = g.n[r.ld];
  r.delta = ray_set_shifted(set) ? NS_DELTA - g.hside : 0.0;
  // accurate triangulation ray order: panel 0 rays (n over z, m over y), panel 1 (n over y,
  // m over x), panel 2 (n over z, m over x)
  int64_t b = 0;
  if (r.panel >= 1) b += g.n[2] * g.n[1];
  if (r.panel >= 2) b += g.n[1] * g.n[0];
  r.ordinal_base = ray_set_shifted(set) ? b : 0;
  return r;
}

// Outputs of one trace launch.
struct TraceOut {
  // set 0: runs of inside nodes per status row (row = k*ny + j), the status map in run form
  int2* sruns;
  int64_t srun_cap;
  unsigned long long* srun_cursor;
  int64_t* srun_off;
  int32_t* srun_cnt;
  uint32_t* bits;          // sets 1..3: insideness bits (1 = outside), cleared with atomicAnd
  double* vol_ray;         // per ray interval length sum, indexed by n*nb+m
  // pair store (sets 1..3): lim1/lim2 of vertex-producing pairs
  double* pairs;           // 2 doubles per pair
  int64_t pair_cap;
  unsigned long long* pair_cursor;
  int64_t* ray_pair_off;   // per ray ordinal
  int32_t* ray_pair_cnt;   // per ray ordinal
  // overflow rays
  int32_t* ovf_rays;       // n*nb+m of rays whose hits exceeded kHitCap
  int32_t ovf_cap;
  int32_t* ovf_count;
  // optional per-ray hit dump (tests)
  double* hits;
  int64_t hit_cap;
  unsigned long long* hit_cursor;
  int64_t* ray_hit_off;    // indexed by n*nb+m
  int32_t* ray_hit_cnt;
  int32_t* error_flag;     // set when a device-side capacity is exceeded
  // gradient mode (null otherwise): d volume / d patch parameters (NS_GRAD_PER_PATCH per patch),
  // the patches of the stored pair ends, and 1 / (number of ray sets cast) of the volume formula
  double* gvol;
  int2* pair_pid;
  double grad_scale;
  // epsilon maps (null otherwise): the reference's 4-D layout ((k*ny + j)*nx + i)*3 + l, l the axis
  // of the grid edge from node (i, j, k) to its +1 neighbour; set 0 writes l = 0, set 4 l = 2,
  // set 5 l = 1; eps_inside is the code of the inside medium
  int32_t* epsmap;
  int32_t eps_inside;
  // optional event counters (profiling): candidates, torus candidates, mixed-precision fallbacks
  // (near-tangent sphere, quartic isolation, root polish / root boundary), FP64 re-evaluations of
  // feasibility tests
  unsigned long long* counters;
};

enum { kCntCandidates = 0, kCntTorus = 1, kCntFbSphere = 2, kCntFbQuartic = 3, kCntFbRoot = 4, kCntRecheck = 5,
       kCntN = 8 };

// Candidate (ray, patch) pairs of one ray set, by patch type (0 spheres, 1 tori), and the
// candidates the mixed-precision pass defers to the double-precision pass (same split).
struct CandOut {
  int2* sph;
  int2* tor;
  int64_t cap;
  unsigned long long* count;   // 2 counters
  int2* dsph;
  int2* dtor;
  int64_t dcap;
  unsigned long long* dcount;  // 2 counters
  // torus candidates split by the branch their resolvent cubic takes (null: no split): the
  // cube-root branch (and the rare approximate ones) in tsa, the arccos branch in tsb, each of
  // capacity cap; counts at tscount[1] and tscount[3]
  int2* tsa;
  int2* tsb;
  unsigned long long* tscount;
};

// Slot-major hit store of one ray set: hit i of ray r at t[i * nrays + r]; cnt[r] counts the
// hits filed (more than kHitCap sends the ray to the overflow path).
struct HitStore {
  double* t;
  int32_t* cnt;
  int64_t nrays;
  int32_t* pid;  // patch of every hit, same layout as t (gradient mode only, else null)
};

struct PatchDev {
  int64_t n;
  const double* f64;
  const int32_t* i32;
  const double4* pool;
  const float4* pool32;  // pool in patch-local FP32 form (mixed precision)
  const int8_t* flag;
  double probe;
  const int32_t* win;  // 6 per patch: start x,y,z, end x,y,z; start = -1 when culled
  int kind_mask;       // bit k set when some patch has kind k (host copy)
  const float4* quad32;  // skin cells in patch-local FP32 form, 3 per patch (mixed precision)
  const double4* quadl;  // skin cells: (A c + b, f(c)) about the local origin c, FP64 (mixed precision)
};

constexpr int kSesKinds = (1 << NS_POINT) | (1 << NS_EDGE_REG) | (1 << NS_EDGE_SING) | (1 << NS_FACE_REG) |
                          (1 << NS_FACE_SING);
constexpr int kSkinKinds = (1 << NS_SKIN_POINT) | (1 << NS_SKIN_EDGE) | (1 << NS_SKIN_FACET) | (1 << NS_SKIN_TETRA);
constexpr int kBoxKinds = kSkinKinds | (1 << NS_MESH_TRI);

// Streaming multiprocessors of the current device (queried once per device and cached); grids of
// the grid-stride kernels are sized as multiples of it.
int sm_count();

// Launch shapes of the tracer, picked per context by nsg_autotune (defaults below).
struct TuneParams {
  int isect_threads = 256;  // threads per block of the intersection kernels (64..256)
  int isect_bpsm = 16;      // their blocks per SM (grid = SMs * isect_bpsm, grid-stride)
  int cand_threads = 256;   // threads per block of the candidate kernel (one warp per patch)
  int torus_split = 0;      // torus candidates solved in two launches, one per resolvent branch
  int mc_tris_bpsm = 3;     // blocks per SM of the marching-cubes triangle kernel (3 or 4)
};

// trace.cu: every launch covers all structures of the batch; `set` is the ray set (0..3) and
// tile and ray indices are batch-wide.
cudaError_t launch_windows(const PatchDev& P, int32_t* win, const BatchDev& B, cudaStream_t s);
// Patch-local FP32 copy of the pool: planes (n, d + n.c), clipping spheres (s - c, r^2); with
// quad32, the skin cells' quadrics about their local origin (see k_pool32).
cudaError_t launch_pool32(const PatchDev& P, float4* pool32, float4* quad32, double4* quadl, cudaStream_t s);
// Bit mask of the patch kinds present (atomicOr into *mask, which the caller zeroes).
cudaError_t launch_kind_mask(const PatchDev& P, int* mask, cudaStream_t s);
// tile_cnt null: only the window-area sum (the candidate bound of the panel).
cudaError_t launch_bin_count(const PatchDev& P, const BatchDev& B, int set, int32_t* tile_cnt,
                             unsigned long long* area, cudaStream_t s);
cudaError_t launch_bin_fill(const PatchDev& P, const BatchDev& B, int set, const int64_t* tile_off,
                            int32_t* tile_cursor, int32_t* tile_list, cudaStream_t s);
// ev (optional, profiling): 4 events recorded before the candidate kernel and after the candidate,
// intersection and fill kernels.
cudaError_t launch_trace(const PatchDev& P, const BatchDev& B, int set, int64_t ntiles, const TraceOut& out,
                         const CandOut& co, const HitStore& hs, int precision, const TuneParams& tp, cudaStream_t s,
                         cudaEvent_t* ev = nullptr);
// pscratch: patch column of the overflow hits (gradient mode), else null.
cudaError_t launch_trace_overflow(const PatchDev& P, const BatchDev& B, int set, const int64_t* tile_off,
                                  const int32_t* tile_list, const TraceOut& out, int n_ovf, double* scratch,
                                  int32_t* pscratch, int precision, cudaStream_t s);

// reduce.cu: out[b] (+)= sum of v over structure b's segment [base[i(b)], base[i(b+1)]) with
// i(b) = idx[b] (idx given) or b, in a summation order fixed by the segment alone; part is scratch
// for n * kSegParts doubles.
constexpr int kSegParts = 64;
cudaError_t launch_segment_sums(const double* v, const int64_t* base, const int64_t* idx, int n, double* out,
                                double* part, bool accumulate, cudaStream_t s);

// reduce.cu, batch uploads: per-patch structure and batch-wide pool index (err set on a pool
// range outside the structure's pool); batch-wide patch atom indices (err on an index outside
// the structure's atoms).
cudaError_t launch_batch_patches(int64_t np, const int64_t* patch_off, int n, const int64_t* pool_off, int32_t* i32,
                                 int32_t* patch_struct, int32_t* err, cudaStream_t s);
cudaError_t launch_batch_atoms(int64_t np, const int32_t* patch_struct, const int64_t* atom_off, int32_t* patch_atoms,
                               int32_t* err, cudaStream_t s);

// reduce.cu: FMA-chain kernel timing the FP64 (precision 0) or FP32 (1) peak; out holds
// blocks * threads elements.
cudaError_t launch_fma_peak(int precision, int blocks, int threads, int iters, void* out, cudaStream_t s);

// chain.cu: atom derivatives (x, y, z, r per atom; atomics) of volume and area from the per-patch
// parameter derivatives; patch_atoms are batch-wide atom indices; n_bad counts singular facets.
cudaError_t launch_chain(int64_t np, const int32_t* i32, const double* f64, const int32_t* patch_atoms,
                         const double* atoms, double probe, const double* gpatch_vol, const double* gpatch_area,
                         double* gvol_atoms, double* garea_atoms, int32_t* n_bad, cudaStream_t s);

}  // namespace nsg
