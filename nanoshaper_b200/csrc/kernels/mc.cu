// Vertex assembly and marching cubes of the SES grid ray caster.
//
// Vertices: every vertex-producing pair of an accurate-triangulation ray yields two analytic
// vertices on the grid edges that contain the interval ends; a vertex is dropped when the two
// end nodes of its edge have the same final insideness, and the first vertex of an edge wins
// (assembleVerticesList src/Surface.cpp:7415-7667).  Vertices keep the reference order: panel 0
// rays (z-major), panel 1 rays (y-major), panel 2 rays (z-major), pairs in ray order.
//
// Marching cubes: cubes (i,j,k) in [1, N-2]^3 are classified from the 8 insideness bits; the
// classification writes the active cubes in (k, j, i) order and, per 32 cubes of a row, their
// active bits and the index of the first (the active-cube map, 8 bytes per 32 cubes, from which
// the active index of any active cube follows).  Every active cube has 12 vertex slots (cube_vl).
// The push pass (k_mc_push) writes each vertex that is the first of its grid edge into the slots
// of the (up to four) cubes that share the edge: a ray's vertices are sorted along it, so the
// vertices of an edge have consecutive ids, the first of them is the one whose predecessor has
// another edge key, and a slot is written once, with a plain store (the slots start at -1; the
// host clears and fills them structure chunk by structure chunk, so that a chunk's slots stay in
// L2 between the two).  Active cubes add an edge-midpoint vertex to their own edges 5, 6, 10
// that carry no analytic vertex, in (k, j, i, edge) order, appended after the analytic ones
// (getVertices :8002-8327), and write it into the slots in the same way.  The triangle pass emits
// the case-table triangles with reversed winding and sums their areas (the reference sums Heron
// areas; here |cross product| / 2, the same quantity) (triangulationKernel :9075-9318,
// getTriangles :14559-14780).  Triangles with an edge without a vertex are skipped, as the
// reference does.
#include <cub/cub.cuh>

#include "../mc_cases.h"
#include "grad.cuh"
#include "mc.h"

namespace nsg {

namespace {

__constant__ int8_t c_tri[256][16];  // triangle edge lists, -1 terminated
__constant__ uint16_t c_emask[256];  // cut-edge mask per case
__constant__ uint8_t c_ntri[256];    // case-table triangles per case

// Node coordinate, and the grid edge a point on a ray along axis d lies on: the nearest node after
// the half-side shift, floor((p - min) * scale + 0.5).  Each operation is rounded on its own (the
// file is built without contraction), so every kernel here that places or finds a vertex gets the
// same doubles.
__device__ __forceinline__ double gcoord(const GridDev& g, int d, int64_t i) { return g.mn[d] + (double)i * g.side; }
__device__ __forceinline__ int64_t edge_index(const GridDev& g, int d, double p) {
  return (int64_t)floor((p - g.mn[d]) * g.scale + 0.5);
}

__device__ __forceinline__ int rbit(const uint32_t* __restrict__ bits, int64_t nwords, int64_t f) {
  if (f < 0 || (f >> 5) >= nwords) return 1;
  return (bits[f >> 5] >> (f & 31)) & 1;
}

struct RayId {
  int panel;
  int64_t m, n;
};

__device__ __forceinline__ RayId ray_of(const GridDev& g, int64_t r) {
  const int64_t NX = g.n[0], NY = g.n[1], NZ = g.n[2];
  RayId id;
  int64_t R0 = NZ * NY, R1 = NY * NX;
  if (r < R0) { id.panel = 0; id.n = r / NY; id.m = r - id.n * NY; }
  else if (r < R0 + R1) { int64_t q = r - R0; id.panel = 1; id.n = q / NX; id.m = q - id.n * NX; }
  else { int64_t q = r - R0 - R1; id.panel = 2; id.n = q / NX; id.m = q - id.n * NX; }
  return id;
}

// Edge key (ix, iy, iz, dir) of the vertex at ray position index a.
__device__ __forceinline__ int4 edge_key(const RayId& id, int64_t a) {
  if (id.panel == 0) return make_int4((int)a, (int)id.m, (int)id.n, NS_X_DIR);
  if (id.panel == 1) return make_int4((int)id.m, (int)id.n, (int)a, NS_Z_DIR);
  return make_int4((int)id.m, (int)a, (int)id.n, NS_Y_DIR);
}

__device__ __forceinline__ bool keeps(const GridDev& g, const uint32_t* bits, int64_t nwords, int4 e) {
  const int64_t NX = g.n[0], NY = g.n[1];
  int64_t f = ((int64_t)e.z * NY + e.y) * NX + e.x;
  int64_t step = e.w == NS_X_DIR ? 1 : (e.w == NS_Y_DIR ? NX : NX * NY);
  return rbit(bits, nwords, f) != rbit(bits, nwords, f + step);
}

__device__ __forceinline__ int rec_struct(int w) { return (int)((unsigned)w >> 11); }

// vpid of an analytic vertex: its patch, and in bits 29-30 the axis of its ray (the gradient pass
// reads the axis from here rather than from the 16-byte edge key); -1 without a patch.
constexpr int kVpidAxisShift = 29;
constexpr int32_t kVpidPatchMask = (1 << kVpidAxisShift) - 1;
__device__ __forceinline__ int32_t vpid_pack(int32_t pid, int axis) {
  return pid < 0 ? -1 : (pid | (axis << kVpidAxisShift));
}

// Active index of the active cube (i, j, k) of structure S, from the active-cube map (a structure
// has fewer than 2^31 cubes, so the offsets within it fit 32 bits).
__device__ __forceinline__ int32_t active_index(const int2* __restrict__ amap, const StructDev& S, int i, int j,
                                                int k) {
  const int W = ((int)S.g.n[0] - 2 + 31) >> 5;
  const int b = i - 1;
  const int2 w = amap[S.aword_base + ((k - 1) * ((int)S.g.n[1] - 2) + (j - 1)) * W + (b >> 5)];
  return w.y + __popc((unsigned)w.x & ((1u << (b & 31)) - 1u));
}

// Writes vertex v into the slots of the active cubes (up to four, those inside the cube range)
// that share grid edge (axis, x, y, z).  An x edge at (x, y, z) is edge 0 of cube (x, y, z), 2 of
// (x, y-1, z), 4 of (x, y, z-1), 6 of (x, y-1, z-1); a y edge is 3 of (x, y, z), 1 of (x-1, y, z),
// 7 of (x, y, z-1), 5 of (x-1, y, z-1); a z edge 8 of (x, y, z), 9 of (x-1, y, z), 11 of
// (x, y-1, z), 10 of (x-1, y-1, z).  A cut edge's cubes are all active.
__device__ __forceinline__ void push_vertex(const int2* __restrict__ amap, int32_t* cube_vl, const StructDev& S,
                                            int axis, int x, int y, int z, int32_t v) {
  // per axis: the two offset axes of the four cubes and the slots of (0,0), (1,0), (0,1), (1,1)
  const int u = axis == NS_X_DIR ? 1 : 0, w = axis == NS_Z_DIR ? 1 : 2;
  const int s00 = axis == NS_X_DIR ? 0 : (axis == NS_Y_DIR ? 3 : 8);
  const int s10 = axis == NS_X_DIR ? 2 : (axis == NS_Y_DIR ? 1 : 9);
  const int s01 = axis == NS_X_DIR ? 4 : (axis == NS_Y_DIR ? 7 : 11);
  const int s11 = axis == NS_X_DIR ? 6 : (axis == NS_Y_DIR ? 5 : 10);
  const int nx = (int)S.g.n[0] - 2, ny = (int)S.g.n[1] - 2, nz = (int)S.g.n[2] - 2;
#pragma unroll
  for (int q = 0; q < 4; q++) {
    int c[3] = {x, y, z};
    if (q & 1) c[u]--;
    if (q & 2) c[w]--;
    if (c[0] < 1 || c[1] < 1 || c[2] < 1 || c[0] > nx || c[1] > ny || c[2] > nz) continue;
    const int slot = q == 0 ? s00 : (q == 1 ? s10 : (q == 2 ? s01 : s11));
    cube_vl[12 * (int64_t)active_index(amap, S, c[0], c[1], c[2]) + slot] = v;
  }
}

template <bool emit>
__global__ void k_vert(VertArgs A) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < A.nrays; r += (int64_t)gridDim.x * blockDim.x) {
    int np = A.ray_pair_cnt[r];
    if (!emit) {
      int cnt = 0;
      if (np > 0) {
        const StructDev& S = A.B.s[find_struct(A.B.mc_base, A.B.n, r)];
        const GridDev& g = S.g;
        const uint32_t* bits = A.bits + S.word_base;
        RayId id = ray_of(g, r - S.mc_base);
        int vc = id.panel == 0 ? 0 : (id.panel == 1 ? 2 : 1);
        const double* pr = A.pairs + 2 * A.ray_pair_off[r];
        for (int q = 0; q < 2 * np; q++)
          if (keeps(g, bits, S.nwords, edge_key(id, edge_index(g, vc, pr[q])))) cnt++;
      }
      A.surv_cnt[r] = cnt;
      continue;
    }
    if (np == 0 || A.surv_cnt[r] == 0) continue;
    const StructDev& S = A.B.s[find_struct(A.B.mc_base, A.B.n, r)];
    const GridDev& g = S.g;
    const uint32_t* bits = A.bits + S.word_base;
    RayId id = ray_of(g, r - S.mc_base);
    int vc = id.panel == 0 ? 0 : (id.panel == 1 ? 2 : 1);
    const double* pr = A.pairs + 2 * A.ray_pair_off[r];
    const double delta = NS_DELTA - g.hside;
    double base[3];
    if (id.panel == 0) { base[1] = gcoord(g, 1, id.m) + delta; base[2] = gcoord(g, 2, id.n) + delta; }
    else if (id.panel == 1) { base[0] = gcoord(g, 0, id.m) + delta; base[1] = gcoord(g, 1, id.n) + delta; }
    else { base[0] = gcoord(g, 0, id.m) + delta; base[2] = gcoord(g, 2, id.n) + delta; }
    int64_t o = A.surv_off[r];
    for (int q = 0; q < 2 * np; q++) {
      int4 e = edge_key(id, edge_index(g, vc, pr[q]));
      if (!keeps(g, bits, S.nwords, e)) continue;
      double p[3] = {base[0], base[1], base[2]};
      p[vc] = pr[q];
      A.vpos[3 * o + 0] = p[0];
      A.vpos[3 * o + 1] = p[1];
      A.vpos[3 * o + 2] = p[2];
      A.vkey[o] = e;
      A.vstruct[o] = (int32_t)(&S - A.B.s);
      if (A.vpid) {
        const int2 pp = A.pair_pid[A.ray_pair_off[r] + (q >> 1)];
        A.vpid[o] = vpid_pack((q & 1) ? pp.y : pp.x, e.w);
      }
      o++;
    }
  }
}

// The 32 bits of the flat bit grid starting at bit f (missing words read as outside), and in *next
// the 32 bits starting at f + 1, from the same two words.  A structure's grid has fewer than 2^31
// nodes, so its bit indices fit 32 bits.
__device__ __forceinline__ uint32_t bits32_pair(const uint32_t* __restrict__ bits, int32_t nwords, int32_t f,
                                                uint32_t* next) {
  const int32_t w = f >> 5;
  const int s = (int)(f & 31);
  const uint32_t lo = w < nwords ? bits[w] : 0xffffffffu;
  const uint32_t hi = (w + 1) < nwords ? bits[w + 1] : 0xffffffffu;
  const uint32_t x = s ? __funnelshift_r(lo, hi, s) : lo;
  *next = (x >> 1) | (((hi >> s) & 1u) << 31);  // bit f + 32 is bit s of the second word
  return x;
}

// Cube rows (j, k), one thread per row; a warp takes a chunk of consecutive rows of one structure.
// The thread walks its row 32 cubes at a time: the cubes' corners come from the four bit rows
// they touch (corner inside = bit 0), one pair of words per bit row, and a cube is active unless
// its 8 corners agree.  Pass 0 counts the active cubes of the row; pass 1 writes them in i order
// at the row's offset and the row's words of the active-cube map.
template <bool emit>
__global__ void k_mc_rows(MCArgs A) {
  __shared__ uint8_t s_ntri[256];
  for (int t = threadIdx.x; t < 256; t += blockDim.x) s_ntri[t] = c_ntri[t];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t ch = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); ch < A.nchunks; ch += warps) {
    const int4 C = A.row_chunks[ch];  // structure, first local row, row count
    const StructDev& S = A.B.s[C.x];
    const int NX = (int)S.g.n[0], NY = (int)S.g.n[1];
    const uint32_t* bits = A.bits + S.word_base;
    const int32_t nwords = (int32_t)S.nwords;
    const int W = (NX - 2 + 31) >> 5;
    for (int rr = lane; rr < C.z; rr += 32) {
      const int lr = C.y + rr;
      const int j = 1 + lr % (NY - 2), k = 1 + lr / (NY - 2);
      const int64_t grow = S.row_base + lr;
      const int32_t b00 = (k * NY + j) * NX, b10 = b00 + NX, b01 = b00 + NX * NY, b11 = b01 + NX;
      int64_t slot = emit ? A.row_act_off[grow] : 0;
      int32_t run = 0;
      for (int word = 0; word < W; word++) {
        const int32_t ic = 1 + 32 * word;
        const int32_t nvalid = NX - 1 - ic;
        const uint32_t vm = nvalid >= 32 ? 0xffffffffu : ((1u << nvalid) - 1u);
        // corners i and i + 1 of each of the four bit rows from one pair of words per row
        uint32_t c[8], n0, n1, n2, n3;
        c[0] = ~bits32_pair(bits, nwords, b00 + ic, &n0);
        c[1] = ~n0;
        c[3] = ~bits32_pair(bits, nwords, b10 + ic, &n1);
        c[2] = ~n1;
        c[4] = ~bits32_pair(bits, nwords, b01 + ic, &n2);
        c[5] = ~n2;
        c[7] = ~bits32_pair(bits, nwords, b11 + ic, &n3);
        c[6] = ~n3;
        uint32_t d = 0;
#pragma unroll
        for (int q = 1; q < 8; q++) d |= c[0] ^ c[q];
        const uint32_t act = d & vm;
        if (!emit) {
          run += __popc(act);
          continue;
        }
        A.amap[S.aword_base + (int64_t)lr * W + word] = make_int2((int)act, (int)slot);
        for (uint32_t m = act; m; m &= m - 1) {
          const int bit = __ffs(m) - 1;
          int cs = 0;
#pragma unroll
          for (int q = 0; q < 8; q++) cs |= ((c[q] >> bit) & 1u) << q;
          // every cut edge of a cube with i, j, k >= 2 has a vertex (an analytic one, or the
          // midpoint its owner cube adds), so its triangles are the case table's; a cube on the
          // low faces of the cube range may lack vertices on edges whose owner lies outside the
          // range, and is counted after the midpoint vertices are in place (k_mc_tris_bnd)
          if (ic + bit >= 2 && j >= 2 && k >= 2) {
            A.tri_cnt[slot] = s_ntri[cs];
          } else {
            A.tri_cnt[slot] = 0;
            const unsigned long long q = atomicAdd(A.bnd_cursor, 1ull);
            A.bnd_list[q] = (int32_t)slot;
          }
          A.act_rec[slot++] = make_int4(ic + bit, j, k, cs | (C.x << 11));
        }
      }
      if (!emit) A.row_act_cnt[grow] = run;
    }
  }
}

// One thread per active cube.  Pass 0: which of the cube's own edges 5, 6, 10 need a midpoint
// vertex (cut edge without an analytic vertex); the mask goes to bits 8..10 of the record and the
// count to mid_cnt.  Pass 1: writes those vertices at their final indices (act_mid) and into the
// slots of the cubes that share their edges.
template <bool emit>
__global__ void k_mc_mid(MCArgs A) {
  // case tables in shared memory: a constant-bank read with a different index per lane is
  // serialised across the warp
  __shared__ uint16_t s_emask[256];
  for (int t = threadIdx.x; t < 256; t += blockDim.x) s_emask[t] = c_emask[t];
  __syncthreads();
  for (int64_t a = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; a < A.n_active; a += (int64_t)gridDim.x * blockDim.x) {
    int4 rec = A.act_rec[a];
    const int i = rec.x, j = rec.y, k = rec.z;
    const StructDev& S = A.B.s[rec_struct(rec.w)];
    const GridDev& g = S.g;
    if (!emit) {
      // own edges 5 (y at (i+1, j, k+1)), 6 (x at (i, j+1, k+1)), 10 (z at (i+1, j+1, k)) that are
      // cut and carry no analytic vertex: their slots are still empty after the analytic push
      const int em = s_emask[rec.w & 255];
      const int4 s47 = reinterpret_cast<const int4*>(A.cube_vl + 12 * a)[1];
      const int s10 = A.cube_vl[12 * a + 10];
      int mm = 0;
      if ((em & 32) && s47.y < 0) mm |= 1;
      if ((em & 64) && s47.z < 0) mm |= 2;
      if ((em & 1024) && s10 < 0) mm |= 4;
      A.act_rec[a].w = (rec.w & ~(7 << 8)) | (mm << 8);
      A.mid_cnt[a] = __popc(mm);
      continue;
    }
    int mm = (rec.w >> 8) & 7;
    int64_t v = A.n_analytic + A.mid_off[a];
    A.act_mid[a] = (int32_t)v;
    for (int q = 0; q < __popc(mm); q++) A.vstruct[v + q] = rec_struct(rec.w);
    if (mm & 1) {
      A.vpos[3 * v] = gcoord(g, 0, i + 1) - g.hside; A.vpos[3 * v + 1] = gcoord(g, 1, j);
      A.vpos[3 * v + 2] = gcoord(g, 2, k + 1) - g.hside;
      A.vkey[v] = make_int4(i + 1, j, k + 1, NS_Y_DIR);
      push_vertex(A.amap, A.cube_vl, S, NS_Y_DIR, i + 1, j, k + 1, (int32_t)v);
      v++;
    }
    if (mm & 2) {
      A.vpos[3 * v] = gcoord(g, 0, i); A.vpos[3 * v + 1] = gcoord(g, 1, j + 1) - g.hside;
      A.vpos[3 * v + 2] = gcoord(g, 2, k + 1) - g.hside;
      A.vkey[v] = make_int4(i, j + 1, k + 1, NS_X_DIR);
      push_vertex(A.amap, A.cube_vl, S, NS_X_DIR, i, j + 1, k + 1, (int32_t)v);
      v++;
    }
    if (mm & 4) {
      A.vpos[3 * v] = gcoord(g, 0, i + 1) - g.hside; A.vpos[3 * v + 1] = gcoord(g, 1, j + 1) - g.hside;
      A.vpos[3 * v + 2] = gcoord(g, 2, k);
      A.vkey[v] = make_int4(i + 1, j + 1, k, NS_Z_DIR);
      push_vertex(A.amap, A.cube_vl, S, NS_Z_DIR, i + 1, j + 1, k, (int32_t)v);
    }
  }
}

// One thread per analytic vertex: the first vertex of each grid edge goes into the slots of the
// edge's cubes.  A ray's vertices are sorted along it and an edge's vertices all lie on one ray,
// so they have consecutive ids: vertex v is the first of its edge unless vertex v - 1 has the same
// edge key in the same structure.  Each slot is written once, with a plain store.
__global__ void k_mc_push(MCArgs A, int64_t v0, int64_t v1) {
  for (int64_t v = v0 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < v1; v += (int64_t)gridDim.x * blockDim.x) {
    const int4 e = A.vkey[v];
    const int32_t sv = A.vstruct[v];
    if (v > v0) {
      const int4 p = A.vkey[v - 1];
      if (p.x == e.x && p.y == e.y && p.z == e.z && p.w == e.w && A.vstruct[v - 1] == sv) continue;
    }
    push_vertex(A.amap, A.cube_vl, A.B.s[sv], e.w, e.x, e.y, e.z, (int32_t)v);
  }
}

// dst[q] = src[idx[q]]: per-structure offsets out of batch-wide prefix sums.
__global__ void k_gather_i64(const int64_t* __restrict__ src, const int64_t* __restrict__ idx, int64_t n,
                             int64_t* dst) {
  const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q < n) dst[q] = src[idx[q]];
}

// Triangle counts of the active cubes on the low faces of the cube range (listed by k_mc_rows): the
// case-table triangles whose three edges have vertices.
__global__ void k_mc_tris_bnd(MCArgs A) {
  const int64_t n = (int64_t)*A.bnd_cursor;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
    const int32_t a = A.bnd_list[q];
    const int c = A.act_rec[a].w & 255;
    const int32_t* cv = A.cube_vl + 12 * (int64_t)a;
    int cnt = 0;
    for (int t = 0; t < 16 && c_tri[c][t] >= 0; t += 3)
      if (cv[c_tri[c][t]] >= 0 && cv[c_tri[c][t + 1]] >= 0 && cv[c_tri[c][t + 2]] >= 0) cnt++;
    A.tri_cnt[a] = cnt;
  }
}

constexpr int kTrisThreads = 256;
constexpr int kTrisWarps = kTrisThreads / 32;
constexpr int kMaxCubeTris = 5;  // the most triangles of a case

// Triangles, 32 active cubes per warp: the lanes load their cubes' 12 vertex slots into shared
// memory, then the warp's triangles (tri_cnt per cube, at tri_off) are spread over the lanes, one
// per lane, whatever the cubes' cases.  Each writes its triangle with reversed winding (coalesced
// across the warp) and its area (and, in gradient mode, the area's derivatives with respect to its
// analytic vertices); each cube's area is the sum of its triangles' in case-table order.
template <int kMinBlocks>
__global__ void __launch_bounds__(kTrisThreads, kMinBlocks) k_mc_tris(MCArgs A) {
  __shared__ int8_t s_tri[256][16];
  __shared__ uint8_t s_ntri[256];
  // per warp: each cube's vertex slots ([slot][lane]) and the areas of the warp's triangles
  __shared__ int32_t s_vid[kTrisWarps][12][32];
  __shared__ double s_area[kTrisWarps][kMaxCubeTris * 32];
  for (int t = threadIdx.x; t < 256 * 16; t += blockDim.x) (&s_tri[0][0])[t] = (&c_tri[0][0])[t];
  for (int t = threadIdx.x; t < 256; t += blockDim.x) s_ntri[t] = c_ntri[t];
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int64_t base = ((int64_t)blockIdx.x * kTrisWarps + w) * 32; base < A.n_active;
       base += (int64_t)gridDim.x * kTrisThreads) {
    const int64_t a = base + lane;
    const bool valid = a < A.n_active;
    const int cw = valid ? A.act_rec[a].w : 0;
    if (valid) {
      const int4* cv = reinterpret_cast<const int4*>(A.cube_vl + 12 * a);
      const int4 v0 = cv[0], v1 = cv[1], v2 = cv[2];
      s_vid[w][0][lane] = v0.x; s_vid[w][1][lane] = v0.y; s_vid[w][2][lane] = v0.z; s_vid[w][3][lane] = v0.w;
      s_vid[w][4][lane] = v1.x; s_vid[w][5][lane] = v1.y; s_vid[w][6][lane] = v1.z; s_vid[w][7][lane] = v1.w;
      s_vid[w][8][lane] = v2.x; s_vid[w][9][lane] = v2.y; s_vid[w][10][lane] = v2.z; s_vid[w][11][lane] = v2.w;
    }
    const int cnt = valid ? A.tri_cnt[a] : 0;
    int incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int x = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += x;
    }
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    const int64_t tbase = A.tri_off[base];
    __syncwarp();
    for (int t0 = 0; t0 < total; t0 += 32) {
      const int t = t0 + lane;
      // the cube of triangle t: the first lane whose inclusive count exceeds t
      int l = 0;
#pragma unroll
      for (int step = 16; step; step >>= 1) {
        const int x = __shfl_sync(0xffffffffu, incl, l + step - 1);
        if (x <= t) l += step;
      }
      const int ll = l < 31 ? l : 31;
      const int first = __shfl_sync(0xffffffffu, incl - cnt, ll);
      const int lcnt = __shfl_sync(0xffffffffu, cnt, ll);
      const int lw = __shfl_sync(0xffffffffu, cw, ll);
      if (t >= total) continue;
      const int q = t - first;
      const int c = lw & 255;
      const int32_t* lv = &s_vid[w][0][ll];
      // the q-th case triangle whose three edges have vertices: the q-th of the case when the cube
      // keeps all of them (every cube off the low faces), else found by a scan
      int e0 = s_tri[c][3 * q], e1 = s_tri[c][3 * q + 1], e2 = s_tri[c][3 * q + 2];
      if (lcnt != s_ntri[c]) {
        for (int qq = 0, seen = 0; qq < 15 && s_tri[c][qq] >= 0; qq += 3) {
          e0 = s_tri[c][qq];
          e1 = s_tri[c][qq + 1];
          e2 = s_tri[c][qq + 2];
          if (lv[32 * e0] >= 0 && lv[32 * e1] >= 0 && lv[32 * e2] >= 0) {
            if (seen == q) break;
            seen++;
          }
        }
      }
      const int32_t v0 = lv[32 * e0], v1 = lv[32 * e1], v2 = lv[32 * e2];
      A.tris[3 * (tbase + t) + 0] = v2;
      A.tris[3 * (tbase + t) + 1] = v1;
      A.tris[3 * (tbase + t) + 2] = v0;
      const double* P0 = A.vpos + 3 * (int64_t)v0;
      const double* P1 = A.vpos + 3 * (int64_t)v1;
      const double* P2 = A.vpos + 3 * (int64_t)v2;
      const double p0[3] = {P0[0], P0[1], P0[2]}, p1[3] = {P1[0], P1[1], P1[2]}, p2[3] = {P2[0], P2[1], P2[2]};
      // area = |n| / 2, n = (P1 - P0) x (P2 - P0): the area the reference computes with Heron's
      // formula (getTriangles, src/Surface.cpp:14559-14780), with one square root instead of four
      const double f1[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]};
      const double f2[3] = {p2[0] - p0[0], p2[1] - p0[1], p2[2] - p0[2]};
      double nn[3] = {f1[1] * f2[2] - f1[2] * f2[1], f1[2] * f2[0] - f1[0] * f2[2], f1[0] * f2[1] - f1[1] * f2[0]};
      const double nl = sqrt(nn[0] * nn[0] + nn[1] * nn[1] + nn[2] * nn[2]);
      s_area[w][t] = nl > 0 ? 0.5 * nl : 0.0;
      if (nl > 0 && A.vgrad) {
        // d area / d (position of vertex vv along the axis of its cube edge ev, which is the ray
        // an analytic vertex moves on): ((Pa - Pb) x n / (2 |n|)) along that axis
        const double h = 0.5 / nl;
        nn[0] *= h;
        nn[1] *= h;
        nn[2] *= h;
        const auto add = [&](int32_t vv, int ev, double dx, double dy, double dz) {
          if (vv >= A.n_analytic) return;
          double comp;
          if (ev >= 8) comp = dx * nn[1] - dy * nn[0];        // z
          else if (ev & 1) comp = dz * nn[0] - dx * nn[2];    // y
          else comp = dy * nn[2] - dz * nn[1];                // x
          if (comp != 0.0) atomicAdd(A.vgrad + vv, comp);
        };
        add(v0, e0, p1[0] - p2[0], p1[1] - p2[1], p1[2] - p2[2]);
        add(v1, e1, p2[0] - p0[0], p2[1] - p0[1], p2[2] - p0[2]);
        add(v2, e2, p0[0] - p1[0], p0[1] - p1[1], p0[2] - p1[2]);
      }
    }
    __syncwarp();
    if (valid) {
      double area = 0.0;
      for (int q = 0; q < cnt; q++) area += s_area[w][incl - cnt + q];
      A.cube_area[a] = area;
    }
    __syncwarp();
  }
}

// One thread per analytic vertex: d area / d patch parameters += (d area / d s) * ds / d theta.
// Consecutive vertices (along a ray, and of neighbouring rays) mostly lie on the same patch, so the
// per-patch sums go through warp_add_grad.
__global__ void k_grad_vert(MCArgs A) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t base = (int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < A.n_analytic; base += stride) {
    const int64_t v = base + (threadIdx.x & 31);
    double g[NS_GRAD_PER_PATCH];
    int32_t pid = -1;
    const double gv = v < A.n_analytic ? A.vgrad[v] : 0.0;
    if (gv != 0.0) {
      const double x[3] = {A.vpos[3 * v], A.vpos[3 * v + 1], A.vpos[3 * v + 2]};
      const int32_t vp = A.vpid[v];
      pid = vp & kVpidPatchMask;
      if (vp >= 0 &&
          hit_grad(A.f64 + (int64_t)NS_PATCH_F64 * pid, A.i32[NS_PATCH_I32 * pid], A.probe, x, vp >> kVpidAxisShift, g)) {
#pragma unroll
        for (int k = 0; k < NS_GRAD_PER_PATCH; k++) g[k] *= gv;
      } else {
        pid = -1;
      }
    }
    if (pid < 0)
#pragma unroll
      for (int k = 0; k < NS_GRAD_PER_PATCH; k++) g[k] = 0.0;
    warp_add_grad(pid, g, A.garea);
  }
}

// The patch normal at a vertex: ConnollySurface::getNormal (src/ConnollySurface.cpp:5736-5819) for
// atom spheres (y - c) / r, probe spheres (c - y) / probe and tori (getNormalToTorus, with the
// frame's transpose for Rot); for skin cells the quadric's gradient times 2 (-2 for reduced
// tetrahedra), as SkinSurface::getPatchIntersectionData stores it (src/SkinSurface.cpp:3684-3712).
__global__ void k_vertex_normals(const double* __restrict__ vpos, const int32_t* __restrict__ vpid, int64_t n,
                                 const double* __restrict__ f64, const int32_t* __restrict__ i32, double probe,
                                 double* out) {
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
    const int32_t vp = vpid[v];
    if (vp < 0) continue;
    const int32_t pid = vp & kVpidPatchMask;
    const double* f = f64 + (int64_t)NS_PATCH_F64 * pid;
    const int kind = i32[NS_PATCH_I32 * pid];
    const double y[3] = {vpos[3 * v], vpos[3 * v + 1], vpos[3 * v + 2]};
    double nrm[3] = {0.0, 0.0, 0.0};
    if (kind == NS_FACE_REG || kind == NS_FACE_SING) {
      for (int d = 0; d < 3; d++) nrm[d] = (f[d] - y[d]) / probe;
    } else if (kind == NS_POINT) {
      for (int d = 0; d < 3; d++) nrm[d] = (y[d] - f[d]) / f[3];
    } else if (kind == NS_EDGE_REG || kind == NS_EDGE_SING) {
      const double* inv = f + 9;
      const double t[3] = {y[0] - f[4], y[1] - f[5], y[2] - f[6]};
      double C[3];
      for (int i = 0; i < 3; i++) C[i] = inv[3 * i] * t[0] + inv[3 * i + 1] * t[1] + inv[3 * i + 2] * t[2];
      double dd = C[0] * C[0] + C[1] * C[1];
      const double rm1 = f[7] / sqrt(dd) - 1.;
      dd = sqrt(dd * rm1 * rm1 + C[2] * C[2]);
      C[0] *= rm1 / dd;
      C[1] *= rm1 / dd;
      C[2] /= -dd;
      for (int i = 0; i < 3; i++) nrm[i] = inv[i] * C[0] + inv[3 + i] * C[1] + inv[6 + i] * C[2];
    } else if (ns_is_skin(kind)) {
      const double* Q = f + NS_SKIN_Q;
      const double sg = kind == NS_SKIN_TETRA ? -2.0 : 2.0;
      nrm[0] = sg * (Q[0] * y[0] + Q[4] * y[1] + Q[7] * y[2] + Q[9]);
      nrm[1] = sg * (Q[4] * y[0] + Q[1] * y[1] + Q[5] * y[2] + Q[8]);
      nrm[2] = sg * (Q[7] * y[0] + Q[5] * y[1] + Q[2] * y[2] + Q[6]);
    }
    for (int d = 0; d < 3; d++) out[3 * v + d] = nrm[d];
  }
}

int grid_for(int64_t n, int threads) {
  int64_t b = (n + threads - 1) / threads;
  const int64_t cap = (int64_t)sm_count() * 32;
  return (int)(b < cap ? (b < 1 ? 1 : b) : cap);
}

}  // namespace

cudaError_t mc_init_tables() {
  int8_t tri[256][16];
  uint16_t em[256];
  uint8_t nt[256];
  static const int ec[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6}, {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
  for (int c = 0; c < 256; c++) {
    int m = 0;
    for (int e = 0; e < 12; e++)
      if (((c >> ec[e][0]) & 1) != ((c >> ec[e][1]) & 1)) m |= 1 << e;
    em[c] = (uint16_t)m;
    const char* s = kNsMcCases[c];
    int q = 0;
    for (; s[q] && q < 16; q++) tri[c][q] = (int8_t)(s[q] <= '9' ? s[q] - '0' : s[q] - 'a' + 10);
    nt[c] = (uint8_t)(q / 3);
    for (; q < 16; q++) tri[c][q] = -1;
  }
  cudaError_t err = cudaMemcpyToSymbol(c_tri, tri, sizeof tri);
  if (err == cudaSuccess) err = cudaMemcpyToSymbol(c_ntri, nt, sizeof nt);
  if (err != cudaSuccess) return err;
  return cudaMemcpyToSymbol(c_emask, em, sizeof em);
}

cudaError_t launch_vert(const VertArgs& A, int emit, cudaStream_t s) {
  if (A.nrays == 0) return cudaSuccess;
  if (emit) k_vert<true><<<grid_for(A.nrays, 256), 256, 0, s>>>(A);
  else k_vert<false><<<grid_for(A.nrays, 256), 256, 0, s>>>(A);
  return cudaGetLastError();
}

cudaError_t launch_mc_rows(const MCArgs& A, int emit, cudaStream_t s) {
  if (A.nchunks <= 0) return cudaSuccess;
  if (emit) k_mc_rows<true><<<grid_for(A.nchunks * 32, 256), 256, 0, s>>>(A);
  else k_mc_rows<false><<<grid_for(A.nchunks * 32, 256), 256, 0, s>>>(A);
  return cudaGetLastError();
}

cudaError_t launch_mc_mid(const MCArgs& A, int emit, cudaStream_t s) {
  if (A.n_active <= 0) return cudaSuccess;
  if (emit) k_mc_mid<true><<<grid_for(A.n_active, 256), 256, 0, s>>>(A);
  else k_mc_mid<false><<<grid_for(A.n_active, 256), 256, 0, s>>>(A);
  return cudaGetLastError();
}

template <int kMinBlocks>
cudaError_t launch_tris(const MCArgs& A, cudaStream_t s) {
  int64_t b = (A.n_active + kTrisThreads - 1) / kTrisThreads;
  const int64_t cap = (int64_t)sm_count() * kMinBlocks * 8;
  k_mc_tris<kMinBlocks><<<(unsigned)(b < cap ? b : cap), kTrisThreads, 0, s>>>(A);
  return cudaGetLastError();
}

cudaError_t launch_mc_tris(const MCArgs& A, int blocks_per_sm, cudaStream_t s) {
  if (A.n_active <= 0) return cudaSuccess;
  return blocks_per_sm >= 4 ? launch_tris<4>(A, s) : launch_tris<3>(A, s);
}

cudaError_t launch_vertex_normals(const double* vpos, const int32_t* vpid, int64_t n_analytic, const double* f64,
                                  const int32_t* i32, double probe, double* normals, cudaStream_t s) {
  if (n_analytic <= 0) return cudaSuccess;
  k_vertex_normals<<<grid_for(n_analytic, 256), 256, 0, s>>>(vpos, vpid, n_analytic, f64, i32, probe, normals);
  return cudaGetLastError();
}

cudaError_t launch_gather_i64(const int64_t* src, const int64_t* idx, int64_t n, int64_t* dst, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_gather_i64<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(src, idx, n, dst);
  return cudaGetLastError();
}

cudaError_t launch_mc_push(const MCArgs& A, int64_t v0, int64_t v1, cudaStream_t s) {
  if (v1 <= v0) return cudaSuccess;
  k_mc_push<<<grid_for(v1 - v0, 256), 256, 0, s>>>(A, v0, v1);
  return cudaGetLastError();
}

cudaError_t launch_mc_tris_bnd(const MCArgs& A, cudaStream_t s) {
  if (A.n_active <= 0) return cudaSuccess;
  k_mc_tris_bnd<<<sm_count() * 4, 256, 0, s>>>(A);
  return cudaGetLastError();
}

cudaError_t launch_grad_vert(const MCArgs& A, cudaStream_t s) {
  if (A.n_analytic <= 0 || !A.vgrad) return cudaSuccess;
  k_grad_vert<<<grid_for(A.n_analytic, 256), 256, 0, s>>>(A);
  return cudaGetLastError();
}

}  // namespace nsg
