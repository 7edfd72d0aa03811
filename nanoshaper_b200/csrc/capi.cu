// C-ABI of the B200 grid ray-casting surface builder (libnsgpu).
//
// One context per host thread: it owns a CUDA stream and grow-only device buffers; host buffers
// are always caller-owned.  Calls return NSG_OK or a negative NSG_ERR_* code, never exit.  The
// entry points mirror the pieces of Surface::getSurf (src/Surface.cpp:398-1692) and
// Surface::triangulateSurface (src/Surface.cpp:9909-10526) that run once the surface patches
// exist: ray casting with status/insideness fill and volume, cavity detection and filling, vertex
// assembly and marching cubes.  Declarations and the reference interface each one replaces are
// in include/nsgpu.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <cub/cub.cuh>

#include "host/host_api.h"
#include "kernels/blobby.h"
#include "kernels/cavity.h"
#include "kernels/epsmap.h"
#include "kernels/mc.h"
#include "kernels/pipeline.h"

namespace {

thread_local char g_last_error[512] = "";

int fail(int code, const char* what, cudaError_t e = cudaSuccess) {
  if (e != cudaSuccess)
    snprintf(g_last_error, sizeof g_last_error, "%s: %s", what, cudaGetErrorString(e));
  else
    snprintf(g_last_error, sizeof g_last_error, "%s", what);
  return code;
}

#define CK(call)                                              \
  do {                                                        \
    cudaError_t e_ = (call);                                  \
    if (e_ != cudaSuccess) return fail(NSG_ERR_CUDA, #call, e_); \
  } while (0)

struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
  cudaError_t ensure(size_t bytes) {
    if (bytes <= cap) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    size_t want = std::max<size_t>(bytes, 256);
    cudaError_t e = cudaMalloc(&p, want);
    if (e == cudaSuccess) cap = want;
    return e;
  }
  template <class T>
  T* as() const { return (T*)p; }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
};

}  // namespace

struct nsg_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  NsGrid grid{};  // first structure's grid
  bool has_grid = false;
  // batch layout: one StructDev per structure (a single structure is a batch of one)
  int32_t nstruct = 0;
  std::vector<NsGrid> grids;
  std::vector<nsg::StructDev> sd;
  DevBuf d_sd, d_patch_struct, d_tile_struct[3], d_ray_base[nsg::kRaySets], d_mc_base, d_row_base, d_row_chunks;
  int64_t nchunks = 0;
  int64_t tiles_tot[3] = {0, 0, 0}, rays_tot[nsg::kRaySets] = {0, 0, 0, 0, 0, 0}, mc_tot = 0, rows_tot = 0, words_tot = 0, awords_tot = 0;
  int32_t patch_nstruct = 0;  // structures the uploaded patches belong to
  bool patch_struct_valid = false;
  std::vector<double> volumes, areas;
  DevBuf vol_struct, area_struct, seg_part;
  // patches
  int64_t np = 0, npool = 0;
  double probe = 1.4;
  DevBuf f64, i32, pool, flag, win, pool32, quad32, quadl, kind_mask_d;
  bool pool32_valid = false;
  int kind_mask = 0;  // patch kinds present (bit per kind), valid when kind_mask_valid
  bool kind_mask_valid = false;
  const double* ext_f64 = nullptr;  // device-resident patch arrays bound by the caller
  const int32_t* ext_i32 = nullptr;
  const double* ext_pool = nullptr;
  const int8_t* ext_flag = nullptr;
  bool has_patches = false;
  // binning per panel
  DevBuf tile_cnt[3], tile_off[3], tile_list[3], bin_area;
  int64_t win_area[3] = {0, 0, 0};
  // wavefront tracing: candidate lists and the slot-major hit store
  // per ray set (slot s when the ray sets run on their own streams, slot 0 otherwise)
  DevBuf cand_sph[nsg::kRaySets], cand_tor[nsg::kRaySets], hit_t[nsg::kRaySets], hit_cnt[nsg::kRaySets],
      def_sph[nsg::kRaySets], def_tor[nsg::kRaySets], hit_pid[nsg::kRaySets], tsplit_a[nsg::kRaySets],
      tsplit_b[nsg::kRaySets];
  bool concurrent_sets = true;
  cudaStream_t set_stream[nsg::kRaySets] = {};
  cudaEvent_t fork_ev = nullptr, join_ev[nsg::kRaySets] = {};
  // gradient mode: hit / pair / vertex patches and the per-patch derivatives of volume and area
  DevBuf pair_pid, ovf_pscratch, gvol, garea, vpid, vgrad;
  // atoms behind the patches (for the device chain rule) and the atom derivatives
  std::vector<int64_t> patch_off{0, 0};
  DevBuf d_atoms, d_patch_atoms, d_gatoms_vol, d_gatoms_area, d_bad, d_patch_off, d_pool_off, d_atom_off;
  int64_t n_atoms = 0;
  bool have_atoms = false;
  bool grad_mode = false, have_gvol = false, have_garea = false, have_pids = false;
  int64_t cand_cap = 0, def_cap = 0;
  // trace outputs
  DevBuf status, bits, vol_ray[nsg::kRaySets], epsmap;
  DevBuf pairs, ray_pair_off, ray_pair_cnt, cursors, ovf_rays[nsg::kRaySets], ovf_scratch, err;
  DevBuf hits, ray_hit_off[nsg::kRaySets], ray_hit_cnt[nsg::kRaySets];
  int64_t pair_cap = 0, hit_cap = 0;
  int flags = 0;
  int precision = 0;
  double volume = 0;
  bool have_status = false, have_bits = false;
  // status map in run form (inside runs per row) and its free runs; the dense map is written
  // on demand (download, cavity labelling)
  DevBuf sruns, srun_off, srun_cnt, fr_cnt, fr_off, fruns, frow;
  int64_t srun_cap = 0, n_fruns = 0;
  bool status_dense = false;
  bool have_eps = false;     // the last ray cast built the epsilon maps
  bool eps_filled = false;   // cavity filling has been applied to them
  // ideb map and boundary grid points (node index, ibgp, type, projection, projection flag), the
  // auxiliary grid of the projection
  DevBuf ideb, bgp_node, bgp_ibgp, bgp_type, bgp_pos, bgp_nor, bgp_flag, bgp_n, aux_cnt, aux_off, aux_list;
  int64_t n_bgp = 0, n_bgp_ext = 0;
  bool have_bgp = false, bgp_projected = false;
  // cavities
  DevBuf labels, is_root, roots, cc_count, cc_desc, cc_label_of, cc_fill_of, nroots_d;
  int ncav = 0;
  std::vector<double> cav_size;
  std::vector<int32_t> cav_filled;
  int64_t cav_nodes = 0;                       // nodes of all cavities (labels >= 4)
  bool cav_detected = false;                   // nsg_cavities ran on the last cast
  bool have_cav_atoms = false;
  std::vector<int64_t> cav_count;              // nodes per cavity
  // water-shape filter: the labels before it, per-node support / removed / later flags
  DevBuf cav_label, sh_support, sh_removed[2], sh_later, sh_filled, sh_nrem, sh_changed;
  bool shape_filtered = false;
  bool ideb_ready = false;                     // ideb holds the map (after a shape filter)
  std::vector<int32_t> cav_atom_off, cav_atom_list;
  DevBuf ca_atoms, ca_cell_off, ca_cell_atoms, ca_pairs, ca_alt, ca_count;
  // mesh
  DevBuf amap, cube_vl, vstruct, chunk_off;
  nsg::TuneParams tune;
  DevBuf surv_cnt, surv_off, vpos, vkey, row_act_cnt, row_mid_cnt, row_act_off, row_mid_off, act_rec, act_mid,
      tri_cnt, tri_off, tris, cube_area, red_out, bnd_list, bnd_cursor;
  int64_t n_vert = 0, n_analytic = 0, n_tri = 0, n_active = 0;
  double area = 0;
  DevBuf temp;  // cub temporary storage
  // blobby surface: atoms, field, the field's marching-cubes mesh and its patches, adjoint scratch
  DevBuf b_atoms, b_field, b_mask, b_nv, b_nt, b_voff, b_toff, b_vraw, b_verts, b_vkey, b_tris, b_inc_cnt, b_inc_off,
      b_inc_cur, b_inc, b_patch_atoms, b_gpost, b_gpre, b_gfield, b_gatoms;
  int64_t b_natoms = 0, b_nv_n = 0, b_nt_n = 0;
  double b_B = -2.5;
  int b_ng = 0;
  bool b_valid = false, b_quantized = true;
  int64_t last_overflow_rays = 0;
  // timing: user events and per-stage kernel times (milliseconds, summed over calls)
  cudaEvent_t user_ev[8] = {};
  bool profile = false;
  cudaEvent_t st_ev[2 * 12] = {};
  double stage_ms[12] = {};
  int64_t stage_calls[12] = {};
  cudaEvent_t sub_ev[nsg::kRaySets][4] = {};  // per ray set: before candidates, after candidates / intersections / fill
  int64_t launches = 0;
  DevBuf counters;
  unsigned long long counter_host[8] = {};
};

namespace {

nsg::PatchDev patch_dev(nsg_ctx* c) {
  nsg::PatchDev P;
  P.n = c->np;
  P.f64 = c->ext_f64 ? c->ext_f64 : c->f64.as<double>();
  P.i32 = c->ext_i32 ? c->ext_i32 : c->i32.as<int32_t>();
  P.pool = (const double4*)(c->ext_pool ? c->ext_pool : c->pool.as<double>());
  P.flag = c->ext_flag ? c->ext_flag : c->flag.as<int8_t>();
  P.pool32 = c->pool32.as<float4>();
  P.quad32 = c->quad32.as<float4>();
  P.quadl = c->quadl.as<double4>();
  P.probe = c->probe;
  P.win = c->win.as<int32_t>();
  P.kind_mask = c->kind_mask;
  return P;
}

int64_t nwords_of(const NsGrid& g) { return ((g.nx + 31) >> 5) * g.ny * g.nz; }

nsg::GridDev grid_dev(const NsGrid& g) {
  nsg::GridDev d{};
  d.n[0] = g.nx; d.n[1] = g.ny; d.n[2] = g.nz;
  d.mn[0] = g.xmin; d.mn[1] = g.ymin; d.mn[2] = g.zmin;
  d.mx[0] = g.xmax; d.mx[1] = g.ymax; d.mx[2] = g.zmax;
  d.scale = g.scale; d.side = g.side; d.hside = g.hside;
  return d;
}

nsg::BatchDev batch_dev(nsg_ctx* c) {
  nsg::BatchDev B{};
  B.n = c->nstruct;
  B.s = c->d_sd.as<nsg::StructDev>();
  B.patch_struct = c->d_patch_struct.as<int32_t>();
  for (int i = 0; i < 3; i++) B.tile_struct[i] = c->d_tile_struct[i].as<int32_t>();
  for (int i = 0; i < nsg::kRaySets; i++) B.ray_base[i] = c->d_ray_base[i].as<int64_t>();
  B.mc_base = c->d_mc_base.as<int64_t>();
  B.row_base = c->d_row_base.as<int64_t>();
  return B;
}

template <class T>
cudaError_t upload_vec(DevBuf& d, const std::vector<T>& h, cudaStream_t s) {
  cudaError_t e = d.ensure(std::max<size_t>(h.size(), 1) * sizeof(T));
  if (e != cudaSuccess || h.empty()) return e;
  return cudaMemcpyAsync(d.p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, s);
}

// Host and device layout of the batch: per-structure bases of tiles, rays, MC ray ordinals, cube
// rows and bit words, and the reverse maps tile -> structure.
int batch_layout(nsg_ctx* c, const NsGrid* grids, int32_t n) {
  std::vector<nsg::StructDev> sd(n);
  std::vector<int64_t> rb[nsg::kRaySets], mcb(n + 1), rowb(n + 1);
  std::vector<int32_t> ts[3];
  std::vector<int4> chunks;  // marching-cubes row chunks: structure, first row, row count
  constexpr int32_t kRowChunk = 32;  // cube rows per chunk: one warp, one row per lane
  for (int i = 0; i < nsg::kRaySets; i++) rb[i].resize(n + 1);
  int64_t tiles[3] = {0, 0, 0}, rays[nsg::kRaySets] = {0, 0, 0, 0, 0, 0}, mc = 0, rows = 0, words = 0, awords = 0;
  for (int32_t b = 0; b < n; b++) {
    const NsGrid& G = grids[b];
    if (G.nx < 3 || G.ny < 3 || G.nz < 3) return fail(NSG_ERR_ARG, "grid must have at least 3 nodes per axis");
    if (G.nx * G.ny * G.nz >= (int64_t)1 << 31) return fail(NSG_ERR_ARG, "grid larger than 2^31 nodes");
    nsg::StructDev& S = sd[b];
    S.g = grid_dev(G);
    S.A = G.A;
    S.nwords = nwords_of(G);
    S.word_base = words;
    words += S.nwords;
    for (int panel = 0; panel < 3; panel++) {
      nsg::RaySet rs = nsg::make_ray_set(panel == 0 ? 0 : panel + 1, S.g);
      int64_t nt = ((rs.nb + nsg::kTileM - 1) / nsg::kTileM) * ((rs.na + nsg::kTileN - 1) / nsg::kTileN);
      S.tile_base[panel] = tiles[panel];
      ts[panel].insert(ts[panel].end(), nt, b);
      tiles[panel] += nt;
    }
    for (int set = 0; set < nsg::kRaySets; set++) {
      nsg::RaySet rs = nsg::make_ray_set(set, S.g);
      S.ray_base[set] = rb[set][b] = rays[set];
      rays[set] += rs.nb * rs.na;
    }
    S.mc_base = mcb[b] = mc;
    mc += G.nz * G.ny + G.ny * G.nx + G.nz * G.nx;
    S.row_base = rowb[b] = rows;
    S.aword_base = awords;
    awords += ((G.nx - 2 + 31) / 32) * (G.ny - 2) * (G.nz - 2);
    const int64_t srows = (G.ny - 2) * (G.nz - 2);
    for (int64_t r = 0; r < srows; r += kRowChunk)
      chunks.push_back(make_int4(b, (int32_t)r, (int32_t)std::min<int64_t>(kRowChunk, srows - r), 0));
    rows += srows;
    for (int d = 0; d < 3; d++) {
      S.ray_dir[d] = (S.g.mn[d] + (double)(S.g.n[d] - 1) * S.g.side) - (S.g.mn[d] + 0.0 * S.g.side);
      S.inv_dir[d] = 1.0 / S.ray_dir[d];
      S.box_dir[d] = S.g.mx[d] - S.g.mn[d];
    }
  }
  for (int i = 0; i < nsg::kRaySets; i++) {
    rb[i][n] = rays[i];
    if (rays[i] >= (int64_t)1 << 31) return fail(NSG_ERR_CAPACITY, "more than 2^31 rays in one ray set of a batch");
  }
  mcb[n] = mc;
  rowb[n] = rows;
  CK(upload_vec(c->d_sd, sd, c->stream));
  for (int i = 0; i < 3; i++) CK(upload_vec(c->d_tile_struct[i], ts[i], c->stream));
  for (int i = 0; i < nsg::kRaySets; i++) CK(upload_vec(c->d_ray_base[i], rb[i], c->stream));
  CK(upload_vec(c->d_mc_base, mcb, c->stream));
  CK(upload_vec(c->d_row_base, rowb, c->stream));
  CK(upload_vec(c->d_row_chunks, chunks, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->nchunks = (int64_t)chunks.size();
  c->nstruct = n;
  c->grids.assign(grids, grids + n);
  c->sd = sd;
  c->grid = grids[0];
  for (int i = 0; i < 3; i++) c->tiles_tot[i] = tiles[i];
  for (int i = 0; i < nsg::kRaySets; i++) c->rays_tot[i] = rays[i];
  c->mc_tot = mc;
  c->rows_tot = rows;
  c->words_tot = words;
  c->awords_tot = awords;
  c->has_grid = true;
  c->have_status = c->have_bits = false;
  c->volumes.assign(n, 0.0);
  c->areas.assign(n, 0.0);
  return NSG_OK;
}

// Structure index of every patch: all 0 for a single structure.
int ensure_patch_struct(nsg_ctx* c) {
  if (c->patch_struct_valid) return NSG_OK;
  CK(c->d_patch_struct.ensure(std::max<int64_t>(c->np, 1) * sizeof(int32_t)));
  CK(cudaMemsetAsync(c->d_patch_struct.p, 0, std::max<int64_t>(c->np, 1) * sizeof(int32_t), c->stream));
  c->patch_struct_valid = true;
  return NSG_OK;
}

// Stage ids of the per-stage kernel timers.
enum { kStageBin = 0, kStageTrace = 1, kStageOverflow = 2, kStageCavity = 3, kStageVertex = 4, kStageMC = 5,
       kStageCand = 6, kStageIsect = 7, kStageFill = 8, kStageCount = 9 };

void stage_begin(nsg_ctx* c, int id) {
  if (!c->profile) return;
  if (!c->st_ev[2 * id]) {
    cudaEventCreate(&c->st_ev[2 * id]);
    cudaEventCreate(&c->st_ev[2 * id + 1]);
  }
  cudaEventRecord(c->st_ev[2 * id], c->stream);
}

// A stage may be timed in several intervals per call; the last one passes count = true.
void stage_end(nsg_ctx* c, int id, bool count = true) {
  if (!c->profile) return;
  cudaEventRecord(c->st_ev[2 * id + 1], c->stream);
  cudaEventSynchronize(c->st_ev[2 * id + 1]);
  float ms = 0;
  cudaEventElapsedTime(&ms, c->st_ev[2 * id], c->st_ev[2 * id + 1]);
  c->stage_ms[id] += ms;
  if (count) c->stage_calls[id]++;
}

#define LAUNCH(call)  \
  do {                \
    c->launches++;    \
    CK(call);         \
  } while (0)

// Exclusive scan of n int32 (or int64) counts into n+1 int64 offsets; returns the total.
template <class In>
int scan_counts(nsg_ctx* c, const In* in, int64_t n, int64_t* out, int64_t* total) {
  size_t tb = 0;
  CK(cub::DeviceScan::ExclusiveScan(nullptr, tb, in, out, cub::Sum(), (int64_t)0, n, c->stream));
  CK(c->temp.ensure(tb));
  tb = c->temp.cap;
  CK(cub::DeviceScan::ExclusiveScan(c->temp.p, tb, in, out, cub::Sum(), (int64_t)0, n, c->stream));
  if (total) {
    int64_t last_off = 0;
    In last_cnt = 0;
    if (n > 0) {
      CK(cudaMemcpyAsync(&last_off, out + n - 1, sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream));
      CK(cudaMemcpyAsync(&last_cnt, in + n - 1, sizeof(In), cudaMemcpyDeviceToHost, c->stream));
    }
    CK(cudaStreamSynchronize(c->stream));
    *total = last_off + (int64_t)last_cnt;
    CK(cudaMemcpyAsync(out + n, total, sizeof(int64_t), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
  }
  return NSG_OK;
}


// Window-area sum of a panel (the bound of its candidate count).
int panel_area(nsg_ctx* c, int panel) {
  const int set = panel == 0 ? 0 : panel + 1;
  const nsg::BatchDev B = batch_dev(c);
  nsg::PatchDev P = patch_dev(c);
  CK(c->bin_area.ensure(3 * sizeof(unsigned long long)));
  unsigned long long* area = c->bin_area.as<unsigned long long>() + panel;
  CK(cudaMemsetAsync(area, 0, sizeof(unsigned long long), c->stream));
  LAUNCH(nsg::launch_bin_count(P, B, set, nullptr, area, c->stream));
  unsigned long long a_host = 0;
  CK(cudaMemcpyAsync(&a_host, area, sizeof(a_host), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->win_area[panel] = (int64_t)a_host;
  return NSG_OK;
}

// Patch lists of every 32x4 ray tile of a panel (CSR), for the per-ray overflow path.
int bin_panel(nsg_ctx* c, int panel) {
  const int set = panel == 0 ? 0 : panel + 1;
  const int64_t ntiles = c->tiles_tot[panel];
  const nsg::BatchDev B = batch_dev(c);
  CK(c->tile_cnt[panel].ensure((ntiles + 1) * sizeof(int32_t)));
  CK(c->tile_off[panel].ensure((ntiles + 1) * sizeof(int64_t)));
  CK(cudaMemsetAsync(c->tile_cnt[panel].p, 0, (ntiles + 1) * sizeof(int32_t), c->stream));
  nsg::PatchDev P = patch_dev(c);
  LAUNCH(nsg::launch_bin_count(P, B, set, c->tile_cnt[panel].as<int32_t>(), nullptr, c->stream));
  int64_t total = 0;
  int rc = scan_counts(c, c->tile_cnt[panel].as<int32_t>(), ntiles, c->tile_off[panel].as<int64_t>(), &total);
  if (rc) return rc;
  CK(c->tile_list[panel].ensure(std::max<int64_t>(total, 1) * sizeof(int32_t)));
  CK(cudaMemsetAsync(c->tile_cnt[panel].p, 0, (ntiles + 1) * sizeof(int32_t), c->stream));
  LAUNCH(nsg::launch_bin_fill(P, B, set, c->tile_off[panel].as<int64_t>(), c->tile_cnt[panel].as<int32_t>(),
                          c->tile_list[panel].as<int32_t>(), c->stream));
  return NSG_OK;
}

nsg::RunArgs run_args(nsg_ctx* c) {
  nsg::RunArgs A{};
  const NsGrid& g = c->grid;
  A.nx = g.nx; A.ny = g.ny; A.nz = g.nz;
  A.nrows = g.ny * g.nz;
  A.sruns = c->sruns.as<int2>();
  A.srun_off = c->srun_off.as<int64_t>();
  A.srun_cnt = c->srun_cnt.as<int32_t>();
  A.fr_cnt = c->fr_cnt.as<int32_t>();
  A.fr_off = c->fr_off.as<int64_t>();
  A.fruns = c->fruns.as<int2>();
  A.frow = c->frow.as<int32_t>();
  A.nruns = c->n_fruns;
  A.L = c->labels.as<int32_t>();
  return A;
}

// Free runs of every status row (complement of the inside runs).
int build_free_runs(nsg_ctx* c) {
  const int64_t nrows = c->grid.ny * c->grid.nz;
  CK(c->fr_cnt.ensure(nrows * sizeof(int32_t)));
  CK(c->fr_off.ensure((nrows + 1) * sizeof(int64_t)));
  nsg::RunArgs A = run_args(c);
  LAUNCH(nsg::launch_free_runs(A, 0, c->stream));
  int64_t n = 0;
  int rc = scan_counts(c, c->fr_cnt.as<int32_t>(), nrows, c->fr_off.as<int64_t>(), &n);
  if (rc) return rc;
  CK(c->fruns.ensure(std::max<int64_t>(n, 1) * sizeof(int2)));
  CK(c->frow.ensure(std::max<int64_t>(n, 1) * sizeof(int32_t)));
  c->n_fruns = n;
  A = run_args(c);
  LAUNCH(nsg::launch_free_runs(A, 1, c->stream));
  return NSG_OK;
}

// Dense status map from the runs (labels when cavity detection ran).
int materialize_status(nsg_ctx* c, const int32_t* label_of_dev) {
  const NsGrid& g = c->grid;
  CK(c->status.ensure(g.nx * g.ny * g.nz * sizeof(int32_t)));
  nsg::RunArgs A = run_args(c);
  LAUNCH(nsg::status_write(A, label_of_dev, c->status.as<int32_t>(), c->stream));
  c->status_dense = true;
  return NSG_OK;
}

}  // namespace

extern "C" {

const char* nsg_last_error(void) { return g_last_error; }

int nsg_version(void) { return 1; }

int nsg_ctx_create(int device, nsg_ctx** out) {
  if (!out) return NSG_ERR_ARG;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) return fail(NSG_ERR_CUDA, "no CUDA device", e);
  if (device < 0 || device >= ndev) return fail(NSG_ERR_ARG, "device index out of range");
  CK(cudaSetDevice(device));
  nsg_ctx* c = new nsg_ctx();
  c->device = device;
  e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) { delete c; return fail(NSG_ERR_CUDA, "cudaStreamCreate", e); }
  c->own_stream = true;
  e = nsg::mc_init_tables();
  if (e != cudaSuccess) { cudaStreamDestroy(c->stream); delete c; return fail(NSG_ERR_CUDA, "mc tables", e); }
  *out = c;
  return NSG_OK;
}

int nsg_ctx_destroy(nsg_ctx* c) {
  if (!c) return NSG_ERR_ARG;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  DevBuf* bufs[] = {&c->f64, &c->i32, &c->pool, &c->flag, &c->win, &c->pool32, &c->quad32, &c->quadl, &c->kind_mask_d, &c->b_atoms, &c->b_field, &c->b_mask, &c->b_nv, &c->b_nt, &c->b_voff, &c->b_toff, &c->b_vraw, &c->b_verts, &c->b_vkey, &c->b_tris, &c->b_inc_cnt, &c->b_inc_off, &c->b_inc_cur, &c->b_inc, &c->b_patch_atoms, &c->b_gpost, &c->b_gpre, &c->b_gfield, &c->b_gatoms, &c->counters, &c->bin_area,
                    &c->status, &c->bits, &c->epsmap, &c->ideb, &c->bgp_node, &c->bgp_ibgp, &c->bgp_type,
                    &c->bgp_pos, &c->bgp_nor, &c->bgp_flag, &c->bgp_n, &c->aux_cnt, &c->aux_off, &c->aux_list, &c->pairs,
                    &c->ray_pair_off, &c->ray_pair_cnt, &c->cursors, &c->ovf_scratch, &c->err, &c->hits,
                    &c->pair_pid, &c->ovf_pscratch, &c->gvol, &c->garea, &c->vpid, &c->vgrad,
                    &c->d_atoms, &c->d_patch_atoms, &c->d_gatoms_vol, &c->d_gatoms_area, &c->d_bad, &c->amap, &c->cube_vl, &c->vstruct, &c->chunk_off, &c->ca_atoms, &c->ca_cell_off, &c->ca_cell_atoms, &c->ca_pairs, &c->ca_alt, &c->ca_count,
                    &c->d_patch_off, &c->d_pool_off, &c->d_atom_off,
                    &c->labels, &c->is_root, &c->sruns, &c->srun_off, &c->srun_cnt, &c->fr_cnt, &c->fr_off,
                    &c->fruns, &c->frow, &c->roots, &c->cc_count, &c->cc_desc, &c->cc_label_of,
                    &c->cc_fill_of, &c->nroots_d, &c->surv_cnt, &c->surv_off, &c->vpos, &c->vkey,
                    &c->row_act_cnt, &c->row_mid_cnt, &c->row_act_off, &c->row_mid_off, &c->act_rec,
                    &c->act_mid, &c->tri_cnt, &c->tri_off, &c->tris, &c->cube_area, &c->red_out, &c->bnd_list,
                    &c->bnd_cursor, &c->temp};
  for (DevBuf* b : bufs) b->release();
  for (int i = 0; i < 3; i++) { c->tile_cnt[i].release(); c->tile_off[i].release(); c->tile_list[i].release(); }
  c->d_sd.release(); c->d_patch_struct.release(); c->d_mc_base.release(); c->d_row_base.release();
  c->d_row_chunks.release();
  c->vol_struct.release(); c->area_struct.release(); c->seg_part.release();
  for (int i = 0; i < 3; i++) c->d_tile_struct[i].release();
  for (int i = 0; i < nsg::kRaySets; i++) c->d_ray_base[i].release();
  for (int i = 0; i < nsg::kRaySets; i++) {
    c->vol_ray[i].release(); c->ovf_rays[i].release(); c->ray_hit_off[i].release(); c->ray_hit_cnt[i].release();
    c->cand_sph[i].release(); c->cand_tor[i].release(); c->def_sph[i].release(); c->def_tor[i].release();
    c->hit_t[i].release(); c->hit_cnt[i].release(); c->hit_pid[i].release();
    c->tsplit_a[i].release(); c->tsplit_b[i].release();
    if (c->set_stream[i]) cudaStreamDestroy(c->set_stream[i]);
    if (c->join_ev[i]) cudaEventDestroy(c->join_ev[i]);
  }
  for (int i = 0; i < 8; i++)
    if (c->user_ev[i]) cudaEventDestroy(c->user_ev[i]);
  for (int i = 0; i < 24; i++)
    if (c->st_ev[i]) cudaEventDestroy(c->st_ev[i]);
  for (int i = 0; i < nsg::kRaySets; i++)
    for (int q = 0; q < 4; q++)
      if (c->sub_ev[i][q]) cudaEventDestroy(c->sub_ev[i][q]);
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return NSG_OK;
}

// Use a caller-provided stream (e.g. a framework's current stream) instead of the context's own.
int nsg_set_stream(nsg_ctx* c, void* stream) {
  if (!c) return NSG_ERR_ARG;
  CK(cudaSetDevice(c->device));
  if (c->stream) CK(cudaStreamSynchronize(c->stream));
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
  c->stream = (cudaStream_t)stream;
  c->own_stream = false;
  return NSG_OK;
}

int nsg_set_grid(nsg_ctx* c, const NsGrid* g) {
  if (!c || !g) return NSG_ERR_ARG;
  CK(cudaSetDevice(c->device));
  return batch_layout(c, g, 1);
}

// A batch of structures, each on its own grid; patches follow with nsg_upload_batch.
int nsg_set_batch(nsg_ctx* c, int32_t n, const NsGrid* grids) {
  if (!c || n < 1 || !grids) return NSG_ERR_ARG;
  CK(cudaSetDevice(c->device));
  return batch_layout(c, grids, n);
}

static int upload_common(nsg_ctx* c, int64_t n, int64_t npool, double probe) {
  c->np = n;
  c->npool = npool;
  c->probe = probe;
  CK(c->win.ensure(std::max<int64_t>(n, 1) * 6 * sizeof(int32_t)));
  c->has_patches = true;
  c->pool32_valid = false;
  c->kind_mask_valid = false;
  c->b_valid = false;
  c->patch_nstruct = 1;
  c->patch_struct_valid = false;
  c->patch_off.assign({0, n});
  c->have_atoms = false;
  return NSG_OK;
}

int nsg_upload_patches(nsg_ctx* c, int64_t n, const double* f64, const int32_t* i32, int64_t npool,
                       const double* pool, const int8_t* pool_flag, double probe) {
  if (!c || n < 0 || npool < 0 || (n > 0 && (!f64 || !i32)) || (npool > 0 && (!pool || !pool_flag)))
    return NSG_ERR_ARG;
  CK(cudaSetDevice(c->device));
  CK(c->f64.ensure(std::max<int64_t>(n, 1) * NS_PATCH_F64 * sizeof(double)));
  CK(c->i32.ensure(std::max<int64_t>(n, 1) * NS_PATCH_I32 * sizeof(int32_t)));
  CK(c->pool.ensure(std::max<int64_t>(npool, 1) * 4 * sizeof(double)));
  CK(c->flag.ensure(std::max<int64_t>(npool, 1)));
  if (n) {
    CK(cudaMemcpyAsync(c->f64.p, f64, n * NS_PATCH_F64 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->i32.p, i32, n * NS_PATCH_I32 * sizeof(int32_t), cudaMemcpyHostToDevice, c->stream));
  }
  if (npool) {
    CK(cudaMemcpyAsync(c->pool.p, pool, npool * 4 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->flag.p, pool_flag, npool, cudaMemcpyHostToDevice, c->stream));
  }
  c->ext_f64 = nullptr; c->ext_i32 = nullptr; c->ext_pool = nullptr; c->ext_flag = nullptr;
  return upload_common(c, n, npool, probe);
}

// Patch sets of the structures of a batch, concatenated: structure b owns patches
// [patch_off[b], patch_off[b+1]) and pool entries [pool_off[b], pool_off[b+1]); the pool indices in
// each patch record are local to its structure's pool.
int nsg_upload_batch(nsg_ctx* c, const int64_t* patch_off, const double* f64, const int32_t* i32,
                     const int64_t* pool_off, const double* pool, const int8_t* pool_flag, double probe) {
  if (!c || !patch_off || !pool_off) return NSG_ERR_ARG;
  if (c->nstruct < 1) return fail(NSG_ERR_STATE, "nsg_set_batch must come first");
  const int32_t nb = c->nstruct;
  if (patch_off[0] != 0 || pool_off[0] != 0) return fail(NSG_ERR_ARG, "offsets must start at 0");
  for (int32_t b = 0; b < nb; b++)
    if (patch_off[b + 1] < patch_off[b] || pool_off[b + 1] < pool_off[b])
      return fail(NSG_ERR_ARG, "offsets must be non-decreasing");
  const int64_t n = patch_off[nb], npool = pool_off[nb];
  if ((n > 0 && (!f64 || !i32)) || (npool > 0 && (!pool || !pool_flag))) return NSG_ERR_ARG;
  if (n >= (int64_t)1 << 31 || npool >= (int64_t)1 << 31) return fail(NSG_ERR_CAPACITY, "more than 2^31 patches");
  CK(cudaSetDevice(c->device));
  CK(c->f64.ensure(std::max<int64_t>(n, 1) * NS_PATCH_F64 * sizeof(double)));
  CK(c->i32.ensure(std::max<int64_t>(n, 1) * NS_PATCH_I32 * sizeof(int32_t)));
  CK(c->pool.ensure(std::max<int64_t>(npool, 1) * 4 * sizeof(double)));
  CK(c->flag.ensure(std::max<int64_t>(npool, 1)));
  CK(c->d_patch_struct.ensure(std::max<int64_t>(n, 1) * sizeof(int32_t)));
  // straight copies of the caller's arrays (pinned buffers copy at full link speed); the pool
  // indices are made batch-wide and the patch -> structure map is built on the device
  if (n) {
    CK(cudaMemcpyAsync(c->f64.p, f64, n * NS_PATCH_F64 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->i32.p, i32, n * NS_PATCH_I32 * sizeof(int32_t), cudaMemcpyHostToDevice, c->stream));
  }
  if (npool) {
    CK(cudaMemcpyAsync(c->pool.p, pool, npool * 4 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->flag.p, pool_flag, npool, cudaMemcpyHostToDevice, c->stream));
  }
  std::vector<int64_t> po(patch_off, patch_off + nb + 1), qo(pool_off, pool_off + nb + 1);
  CK(upload_vec(c->d_patch_off, po, c->stream));
  CK(upload_vec(c->d_pool_off, qo, c->stream));
  CK(c->d_bad.ensure(sizeof(int32_t)));
  CK(cudaMemsetAsync(c->d_bad.p, 0, sizeof(int32_t), c->stream));
  LAUNCH(nsg::launch_batch_patches(n, c->d_patch_off.as<int64_t>(), nb, c->d_pool_off.as<int64_t>(),
                                   c->i32.as<int32_t>(), c->d_patch_struct.as<int32_t>(), c->d_bad.as<int32_t>(),
                                   c->stream));
  int32_t bad = 0;
  CK(cudaMemcpyAsync(&bad, c->d_bad.p, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (bad) {
    c->has_patches = false;
    return fail(NSG_ERR_ARG, "patch pool range outside its structure's pool");
  }
  c->ext_f64 = nullptr; c->ext_i32 = nullptr; c->ext_pool = nullptr; c->ext_flag = nullptr;
  int rc = upload_common(c, n, npool, probe);
  if (rc) return rc;
  c->patch_nstruct = nb;
  c->patch_struct_valid = true;
  c->patch_off.assign(patch_off, patch_off + nb + 1);
  return NSG_OK;
}

// The atoms the uploaded patches were built from (after jitter), concatenated over the batch
// (structure b owns atoms [atom_off[b], atom_off[b+1])), and the 3 atoms of every patch with
// indices local to its structure (nsg_patchset_atoms); needed by nsg_atom_grads.
int nsg_upload_atoms(nsg_ctx* c, const int64_t* atom_off, const double* atoms_xyzr, const int32_t* patch_atoms) {
  if (!c || !atom_off || !atoms_xyzr || !patch_atoms) return NSG_ERR_ARG;
  if (!c->has_patches || c->patch_nstruct != c->nstruct || (int32_t)c->patch_off.size() != c->nstruct + 1)
    return fail(NSG_ERR_STATE, "patches of the current batch must be uploaded first");
  const int32_t nb = c->nstruct;
  if (atom_off[0] != 0) return fail(NSG_ERR_ARG, "atom offsets must start at 0");
  for (int32_t b = 0; b < nb; b++)
    if (atom_off[b + 1] < atom_off[b]) return fail(NSG_ERR_ARG, "atom offsets must be non-decreasing");
  const int64_t n = atom_off[nb];
  if (n >= ((int64_t)1 << 31)) return fail(NSG_ERR_CAPACITY, "more than 2^31 atoms");
  CK(cudaSetDevice(c->device));
  int rc = ensure_patch_struct(c);
  if (rc) return rc;
  CK(c->d_atoms.ensure(std::max<int64_t>(n, 1) * 4 * sizeof(double)));
  CK(c->d_patch_atoms.ensure(std::max<int64_t>(3 * c->np, 1) * sizeof(int32_t)));
  if (n) CK(cudaMemcpyAsync(c->d_atoms.p, atoms_xyzr, n * 4 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  if (c->np)
    CK(cudaMemcpyAsync(c->d_patch_atoms.p, patch_atoms, 3 * c->np * sizeof(int32_t), cudaMemcpyHostToDevice,
                       c->stream));
  std::vector<int64_t> ao(atom_off, atom_off + nb + 1);
  CK(upload_vec(c->d_atom_off, ao, c->stream));
  CK(c->d_bad.ensure(sizeof(int32_t)));
  CK(cudaMemsetAsync(c->d_bad.p, 0, sizeof(int32_t), c->stream));
  LAUNCH(nsg::launch_batch_atoms(c->np, c->d_patch_struct.as<int32_t>(), c->d_atom_off.as<int64_t>(),
                                 c->d_patch_atoms.as<int32_t>(), c->d_bad.as<int32_t>(), c->stream));
  int32_t bad = 0;
  CK(cudaMemcpyAsync(&bad, c->d_bad.p, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (bad) return fail(NSG_ERR_ARG, "patch atom index outside its structure");
  c->n_atoms = n;
  c->have_atoms = true;
  return NSG_OK;
}

// Derivatives of every structure's volume and area (last gradient-mode nsg_raycast /
// nsg_triangulate) with respect to its atoms' x, y, z, r (n_atoms x 4 each, batch atom order),
// chained on the device; either host pointer may be NULL.
int nsg_atom_grads(nsg_ctx* c, double* d_volume, double* d_area) {
  if (!c) return NSG_ERR_ARG;
  if (!c->have_gvol || !c->have_atoms) return fail(NSG_ERR_STATE, "needs a gradient-mode ray cast and the atoms");
  CK(cudaSetDevice(c->device));
  const int64_t n = std::max<int64_t>(c->n_atoms, 1) * 4;
  CK(c->d_gatoms_vol.ensure(n * sizeof(double)));
  CK(c->d_gatoms_area.ensure(n * sizeof(double)));
  CK(c->d_bad.ensure(sizeof(int32_t)));
  CK(cudaMemsetAsync(c->d_gatoms_vol.p, 0, n * sizeof(double), c->stream));
  CK(cudaMemsetAsync(c->d_gatoms_area.p, 0, n * sizeof(double), c->stream));
  CK(cudaMemsetAsync(c->d_bad.p, 0, sizeof(int32_t), c->stream));
  const nsg::PatchDev P = patch_dev(c);
  LAUNCH(nsg::launch_chain(c->np, P.i32, P.f64, c->d_patch_atoms.as<int32_t>(), c->d_atoms.as<double>(), c->probe,
                           c->gvol.as<double>(), c->have_garea ? c->garea.as<double>() : nullptr,
                           c->d_gatoms_vol.as<double>(), c->d_gatoms_area.as<double>(), c->d_bad.as<int32_t>(),
                           c->stream));
  int32_t bad = 0;
  CK(cudaMemcpyAsync(&bad, c->d_bad.p, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
  if (d_volume && c->n_atoms)
    CK(cudaMemcpyAsync(d_volume, c->d_gatoms_vol.p, c->n_atoms * 4 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  if (d_area && c->n_atoms)
    CK(cudaMemcpyAsync(d_area, c->d_gatoms_area.p, c->n_atoms * 4 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (bad) return fail(NSG_ERR_GEOMETRY, "a probe patch with a singular placement system was skipped");
  return NSG_OK;
}

// Derivatives of the volume (last nsg_raycast with NSG_RAYCAST_GRAD) and of the area (the
// nsg_triangulate that followed it) with respect to the patch surface parameters,
// NS_GRAD_PER_PATCH doubles per patch in upload order; either pointer may be NULL.
int nsg_patch_grads(nsg_ctx* c, double* gvol, double* garea) {
  if (!c) return NSG_ERR_ARG;
  if ((gvol && !c->have_gvol) || (garea && !c->have_garea))
    return fail(NSG_ERR_STATE, "no gradient-mode ray cast / triangulation to read");
  CK(cudaSetDevice(c->device));
  const size_t bytes = (size_t)c->np * NS_GRAD_PER_PATCH * sizeof(double);
  if (gvol && c->np) CK(cudaMemcpyAsync(gvol, c->gvol.p, bytes, cudaMemcpyDeviceToHost, c->stream));
  if (garea && c->np) CK(cudaMemcpyAsync(garea, c->garea.p, bytes, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return NSG_OK;
}

int nsg_raycast(nsg_ctx* c, int flags, int precision, double* volume);

// Peak floating-point rate of this GPU measured live: independent fused multiply-add chains
// (8 per thread, 8 blocks of 256 threads per SM), 2 flops per FMA; precision 0 = FP64, 1 = FP32.
int nsg_fp_peak(nsg_ctx* c, int precision, double* flops_per_s) {
  if (!c || !flops_per_s || (precision != 0 && precision != 1)) return NSG_ERR_ARG;
  CK(cudaSetDevice(c->device));
  const int blocks = nsg::sm_count() * 8, threads = 256, iters = 4096;
  CK(c->red_out.ensure(blocks * threads * sizeof(double)));
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  float best = 1e30f;
  for (int rep = 0; rep < 4; rep++) {
    cudaEventRecord(e0, c->stream);
    cudaError_t e = nsg::launch_fma_peak(precision, blocks, threads, iters, c->red_out.p, c->stream);
    cudaEventRecord(e1, c->stream);
    if (e != cudaSuccess) {
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      return fail(NSG_ERR_CUDA, "fma peak", e);
    }
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (rep > 0 && ms < best) best = ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *flops_per_s = 2.0 * 8.0 * (double)blocks * threads * iters / (best * 1e-3);
  return NSG_OK;
}

// Launch shapes of the tracer: [isect threads per block, isect blocks per SM, candidate threads
// per block].
int nsg_set_tuning(nsg_ctx* c, const int32_t* params, int n) {
  if (!c || !params || n < 3) return NSG_ERR_ARG;
  const int it = params[0], bpsm = params[1], ct = params[2];
  if (it < 64 || it > 256 || it % 32 || bpsm < 1 || bpsm > 64 || ct < 32 || ct > 256 || ct % 32)
    return fail(NSG_ERR_ARG, "tuning parameters out of range");
  c->tune.isect_threads = it;
  c->tune.isect_bpsm = bpsm;
  c->tune.cand_threads = ct;
  if (n >= 4) c->concurrent_sets = params[3] != 0;
  if (n >= 5) c->tune.torus_split = params[4] != 0;
  if (n >= 6) {
    if (params[5] != 3 && params[5] != 4) return fail(NSG_ERR_ARG, "tuning parameter 5 is 3 or 4");
    c->tune.mc_tris_bpsm = params[5];
  }
  return NSG_OK;
}

int nsg_get_tuning(nsg_ctx* c, int32_t* params, int n) {
  if (!c || !params || n < 3) return NSG_ERR_ARG;
  params[0] = c->tune.isect_threads;
  params[1] = c->tune.isect_bpsm;
  params[2] = c->tune.cand_threads;
  if (n >= 4) params[3] = c->concurrent_sets ? 1 : 0;
  if (n >= 5) params[4] = c->tune.torus_split;
  if (n >= 6) params[5] = c->tune.mc_tris_bpsm;
  return NSG_OK;
}

// Picks the tracer's launch shapes for the current batch and precision: every candidate shape
// runs `reps` timed ray casts (after one untimed) and the fastest is kept in the context.
// best_ms (optional) receives its time per ray cast.
int nsg_autotune(nsg_ctx* c, int flags, int precision, int reps, double* best_ms) {
  if (!c || reps < 1) return NSG_ERR_ARG;
  static const int kThreads[] = {128, 256};
  static const int kBpsm[] = {4, 8, 16, 32};
  static const int kCand[] = {128, 256};
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  nsg::TuneParams best = c->tune;
  double best_t = 1e300;
  int rc = NSG_OK;
  for (int it : kThreads)
    for (int bp : kBpsm)
      for (int ct : kCand) {
        c->tune.isect_threads = it;
        c->tune.isect_bpsm = bp;
        c->tune.cand_threads = ct;
        double v = 0;
        rc = nsg_raycast(c, flags, precision, &v);
        if (rc) break;
        cudaEventRecord(e0, c->stream);
        for (int r = 0; r < reps && !rc; r++) rc = nsg_raycast(c, flags, precision, &v);
        cudaEventRecord(e1, c->stream);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rc) break;
        if (ms / reps < best_t) {
          best_t = ms / reps;
          best = c->tune;
        }
      }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  c->tune = best;
  if (rc) return rc;
  if (best_ms) *best_ms = best_t;
  return NSG_OK;
}

// Per-structure volume and area of the last ray cast / triangulation of the batch.
int nsg_batch_results(nsg_ctx* c, double* volumes, double* areas) {
  if (!c || c->nstruct < 1) return NSG_ERR_ARG;
  for (int32_t b = 0; b < c->nstruct; b++) {
    if (volumes) volumes[b] = c->volumes[b];
    if (areas) areas[b] = c->areas[b];
  }
  return NSG_OK;
}

// Binds patch arrays that already live in device memory (no copy); they must stay valid until
// the next bind/upload or the context's destruction.
int nsg_bind_patches_device(nsg_ctx* c, int64_t n, const double* f64, const int32_t* i32, int64_t npool,
                            const double* pool, const int8_t* pool_flag, double probe) {
  if (!c || n < 0 || npool < 0) return NSG_ERR_ARG;
  CK(cudaSetDevice(c->device));
  c->ext_f64 = f64; c->ext_i32 = i32; c->ext_pool = pool; c->ext_flag = pool_flag;
  return upload_common(c, n, npool, probe);
}

// Blobby surface of the context's grid (BlobbySurface::build, src/BlobbySurface.cpp:83-229): the
// atoms' Gaussian field, its marching-cubes mesh at iso level 1, one smoothing pass and (unless
// NSG_BLOBBY_DIFFERENTIABLE) the OFF text round trip; the mesh's triangles become the context's
// patch set.
int nsg_blobby_build(nsg_ctx* c, const double* atoms_xyzr, int64_t n_atoms, double blobbyness, int flags) {
  if (!c || !atoms_xyzr || n_atoms <= 0 || n_atoms >= ((int64_t)1 << 31) || !(blobbyness < 0))
    return NSG_ERR_ARG;
  if (!c->has_grid || c->nstruct != 1) return fail(NSG_ERR_STATE, "a single-structure grid must be set first");
  CK(cudaSetDevice(c->device));
  CK(nsg::blobby_init_tables());
  const NsGrid& G = c->grid;
  const nsg::GridDev g = grid_dev(G);
  const int64_t nodes = G.nx * G.ny * G.nz;
  const int64_t ncubes = (G.nx - 2) * (G.ny - 2) * (G.nz - 2);
  cudaStream_t s = c->stream;
  CK(c->b_atoms.ensure(n_atoms * 4 * sizeof(double)));
  CK(cudaMemcpyAsync(c->b_atoms.p, atoms_xyzr, n_atoms * 4 * sizeof(double), cudaMemcpyHostToDevice, s));
  // cut-off of 6 A in whole grid steps (DEFAULT_CUTOFF, src/BlobbySurface.h)
  const int ng = (int)(6.0 / G.side + 0.5);
  CK(c->b_field.ensure(nodes * sizeof(double)));
  LAUNCH(nsg::launch_blobby_field(g, c->b_atoms.as<double>(), (int)n_atoms, blobbyness, ng, c->b_field.as<double>(), s));
  const double iso = 1.0;
  CK(c->b_mask.ensure(std::max<int64_t>(ncubes, 1)));
  CK(c->b_nv.ensure(std::max<int64_t>(ncubes, 1) * sizeof(int32_t)));
  CK(c->b_nt.ensure(std::max<int64_t>(ncubes, 1) * sizeof(int32_t)));
  CK(c->b_voff.ensure((ncubes + 1) * sizeof(int64_t)));
  CK(c->b_toff.ensure((ncubes + 1) * sizeof(int64_t)));
  LAUNCH(nsg::launch_field_cubes(g, c->b_field.as<double>(), iso, ncubes, c->b_mask.as<uint8_t>(), c->b_nv.as<int32_t>(),
                                 c->b_nt.as<int32_t>(), s));
  int64_t nv = 0, nt = 0;
  int rc = scan_counts(c, c->b_nv.as<int32_t>(), ncubes, c->b_voff.as<int64_t>(), &nv);
  if (rc) return rc;
  rc = scan_counts(c, c->b_nt.as<int32_t>(), ncubes, c->b_toff.as<int64_t>(), &nt);
  if (rc) return rc;
  if (nv >= ((int64_t)1 << 31) || nt >= ((int64_t)1 << 31)) return fail(NSG_ERR_CAPACITY, "mesh too large");
  CK(c->b_vraw.ensure(std::max<int64_t>(nv, 1) * 3 * sizeof(double)));
  CK(c->b_verts.ensure(std::max<int64_t>(nv, 1) * 3 * sizeof(double)));
  CK(c->b_vkey.ensure(std::max<int64_t>(nv, 1) * sizeof(int4)));
  CK(c->b_tris.ensure(std::max<int64_t>(nt, 1) * 3 * sizeof(int32_t)));
  LAUNCH(nsg::launch_field_verts(g, c->b_field.as<double>(), iso, ncubes, c->b_mask.as<uint8_t>(),
                                 c->b_voff.as<int64_t>(), c->b_vraw.as<double>(), c->b_vkey.as<int4>(), s));
  LAUNCH(nsg::launch_field_tris(g, c->b_field.as<double>(), iso, ncubes, c->b_mask.as<uint8_t>(), c->b_voff.as<int64_t>(),
                                c->b_toff.as<int64_t>(), c->b_nt.as<int32_t>(), c->b_tris.as<int32_t>(), s));
  // smoothing: per-vertex incidence lists, then the triangle-ordered sums
  CK(c->b_inc_cnt.ensure(std::max<int64_t>(nv, 1) * sizeof(int32_t)));
  CK(c->b_inc_cur.ensure(std::max<int64_t>(nv, 1) * sizeof(int32_t)));
  CK(c->b_inc_off.ensure((nv + 1) * sizeof(int64_t)));
  CK(c->b_inc.ensure(std::max<int64_t>(3 * nt, 1) * sizeof(int32_t)));
  CK(cudaMemsetAsync(c->b_inc_cnt.p, 0, std::max<int64_t>(nv, 1) * sizeof(int32_t), s));
  CK(cudaMemsetAsync(c->b_inc_cur.p, 0, std::max<int64_t>(nv, 1) * sizeof(int32_t), s));
  LAUNCH(nsg::launch_incidence(c->b_tris.as<int32_t>(), nt, 0, nullptr, c->b_inc_cnt.as<int32_t>(), nullptr, s));
  int64_t ninc = 0;
  if (nv > 0) {
    rc = scan_counts(c, c->b_inc_cnt.as<int32_t>(), nv, c->b_inc_off.as<int64_t>(), &ninc);
    if (rc) return rc;
  }
  LAUNCH(nsg::launch_incidence(c->b_tris.as<int32_t>(), nt, 1, c->b_inc_off.as<int64_t>(), c->b_inc_cur.as<int32_t>(),
                               c->b_inc.as<int32_t>(), s));
  LAUNCH(nsg::launch_smooth(c->b_vraw.as<double>(), nv, c->b_inc_off.as<int64_t>(), c->b_inc.as<int32_t>(),
                            c->b_tris.as<int32_t>(), c->b_verts.as<double>(), s));
  const bool quantize = !(flags & 1);
  if (quantize) LAUNCH(nsg::launch_quantize(c->b_verts.as<double>(), 3 * nv, s));
  // the triangles as the context's patch set
  CK(c->f64.ensure(std::max<int64_t>(nt, 1) * NS_PATCH_F64 * sizeof(double)));
  CK(c->i32.ensure(std::max<int64_t>(nt, 1) * NS_PATCH_I32 * sizeof(int32_t)));
  CK(c->pool.ensure(4 * sizeof(double)));
  CK(c->flag.ensure(1));
  CK(c->b_patch_atoms.ensure(std::max<int64_t>(nt, 1) * 3 * sizeof(int32_t)));
  LAUNCH(nsg::launch_tri_patches(c->b_verts.as<double>(), c->b_tris.as<int32_t>(), nt, c->f64.as<double>(),
                                 c->i32.as<int32_t>(), c->b_patch_atoms.as<int32_t>(), s));
  CK(cudaStreamSynchronize(s));
  c->ext_f64 = nullptr; c->ext_i32 = nullptr; c->ext_pool = nullptr; c->ext_flag = nullptr;
  rc = upload_common(c, nt, 0, 0.0);
  if (rc) return rc;
  c->b_natoms = n_atoms;
  c->b_nv_n = nv;
  c->b_nt_n = nt;
  c->b_B = blobbyness;
  c->b_ng = ng;
  c->b_quantized = quantize;
  c->b_valid = true;
  return NSG_OK;
}

// The blobby mesh of the last nsg_blobby_build (vertices after smoothing and the OFF round trip,
// triangles with the field's marching-cubes winding); NULL buffers only report the sizes.
int nsg_blobby_mesh(nsg_ctx* c, int64_t* n_vertices, int64_t* n_triangles, double* vertices, int32_t* triangles) {
  if (!c) return NSG_ERR_ARG;
  if (!c->b_valid) return fail(NSG_ERR_STATE, "no blobby mesh built");
  if (n_vertices) *n_vertices = c->b_nv_n;
  if (n_triangles) *n_triangles = c->b_nt_n;
  if (vertices && c->b_nv_n)
    CK(cudaMemcpyAsync(vertices, c->b_verts.p, c->b_nv_n * 3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  if (triangles && c->b_nt_n)
    CK(cudaMemcpyAsync(triangles, c->b_tris.p, c->b_nt_n * 3 * sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return NSG_OK;
}

// d volume and d area of a differentiable blobby surface with respect to its atoms (x, y, z, r per
// atom, in the order given to nsg_blobby_build), after a gradient-mode nsg_raycast (and the
// nsg_triangulate that followed it, for the area); either pointer may be NULL.
int nsg_blobby_atom_grads(nsg_ctx* c, double* d_volume, double* d_area) {
  if (!c) return NSG_ERR_ARG;
  if (!c->b_valid) return fail(NSG_ERR_STATE, "no blobby mesh built");
  if (c->b_quantized)
    return fail(NSG_ERR_STATE, "the OFF round trip is piecewise constant: build with NSG_BLOBBY_DIFFERENTIABLE");
  if ((d_volume && !c->have_gvol) || (d_area && !c->have_garea))
    return fail(NSG_ERR_STATE, "no gradient-mode ray cast / triangulation to read");
  CK(cudaSetDevice(c->device));
  const NsGrid& G = c->grid;
  const nsg::GridDev g = grid_dev(G);
  CK(c->b_gpost.ensure(std::max<int64_t>(c->b_nv_n, 1) * 3 * sizeof(double)));
  CK(c->b_gpre.ensure(std::max<int64_t>(c->b_nv_n, 1) * 3 * sizeof(double)));
  CK(c->b_gfield.ensure(G.nx * G.ny * G.nz * sizeof(double)));
  CK(c->b_gatoms.ensure(c->b_natoms * 4 * sizeof(double)));
  nsg::BlobbyMeshDev M{c->b_nv_n, c->b_nt_n, c->b_verts.as<double>(), c->b_vkey.as<int4>(), c->b_tris.as<int32_t>(),
                       c->f64.as<double>(), c->b_patch_atoms.as<int32_t>(), c->b_inc_cnt.as<int32_t>()};
  for (int which = 0; which < 2; which++) {
    double* dst = which == 0 ? d_volume : d_area;
    if (!dst) continue;
    CK(cudaMemsetAsync(c->b_gatoms.p, 0, c->b_natoms * 4 * sizeof(double), c->stream));
    LAUNCH(nsg::launch_blobby_adjoint(g, c->b_atoms.as<double>(), (int)c->b_natoms, c->b_B, c->b_ng,
                                      c->b_field.as<double>(), 1.0, M,
                                      which == 0 ? c->gvol.as<double>() : c->garea.as<double>(), c->b_gpost.as<double>(),
                                      c->b_gpre.as<double>(), c->b_gfield.as<double>(), c->b_gatoms.as<double>(),
                                      c->stream));
    CK(cudaMemcpyAsync(dst, c->b_gatoms.p, c->b_natoms * 4 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
  }
  return NSG_OK;
}

int nsg_raycast(nsg_ctx* c, int flags, int precision, double* volume) {
  if (!c || !c->has_grid || !c->has_patches) return fail(NSG_ERR_STATE, "grid and patches must be set first");
  if (c->patch_nstruct != c->nstruct) return fail(NSG_ERR_STATE, "patches were uploaded for another batch layout");
  if (precision != NSG_PRECISION_FP64 && precision != NSG_PRECISION_MIXED)
    return fail(NSG_ERR_ARG, "unsupported precision");
  CK(cudaSetDevice(c->device));
  {
    int rc = ensure_patch_struct(c);
    if (rc) return rc;
  }
  const nsg::BatchDev B = batch_dev(c);
  const bool do_status = flags & 1;
  const bool do_mc = flags & 2;
  const bool keep_hits = flags & 16;
  const bool grad = flags & 32;
  // epsilon maps: the node rays of panels 1 and 2 besides the status rays (Build_epsilon_maps)
  const bool do_eps = flags & NSG_RAYCAST_EPSMAP;
  if (do_eps && c->nstruct != 1) return fail(NSG_ERR_STATE, "epsilon maps are built for a single structure");
  const auto cast = [&](int set) { return set == 0 ? (do_status || do_eps) : (set <= 3 ? do_mc : do_eps); };
  // the patches of the hits are kept for the gradients and for the analytic vertex normals
  const bool pids = grad || (flags & 64);
  // the marching-cubes vertices carry their patch index in 29 bits (vpid_pack, mc.cu)
  if (pids && c->np >= ((int64_t)1 << 29)) return fail(NSG_ERR_CAPACITY, "more than 2^29 patches with patch ids");
  if (!c->kind_mask_valid) {
    // which patch kinds are present (SES and / or skin cells) selects the intersection kernels
    CK(c->kind_mask_d.ensure(sizeof(int)));
    CK(cudaMemsetAsync(c->kind_mask_d.p, 0, sizeof(int), c->stream));
    nsg::PatchDev P0 = patch_dev(c);
    LAUNCH(nsg::launch_kind_mask(P0, c->kind_mask_d.as<int>(), c->stream));
    CK(cudaMemcpyAsync(&c->kind_mask, c->kind_mask_d.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->kind_mask_valid = true;
  }
  if (grad && (c->kind_mask & nsg::kSkinKinds))
    return fail(NSG_ERR_STATE, "gradients are provided for SES and mesh patch sets, not for skin cells");
  c->grad_mode = grad;
  c->have_gvol = c->have_garea = false;
  c->flags = flags;
  c->precision = precision;
  if (precision == NSG_PRECISION_MIXED && !c->pool32_valid) {
    CK(c->pool32.ensure(std::max<int64_t>(c->npool, 1) * sizeof(float4)));
    const bool skin = c->kind_mask & nsg::kSkinKinds;
    if (skin) {
      CK(c->quad32.ensure(std::max<int64_t>(c->np, 1) * 3 * sizeof(float4)));
      CK(c->quadl.ensure(std::max<int64_t>(c->np, 1) * sizeof(double4)));
    }
    nsg::PatchDev P0 = patch_dev(c);
    LAUNCH(nsg::launch_pool32(P0, c->pool32.as<float4>(), skin ? c->quad32.as<float4>() : nullptr,
                              skin ? c->quadl.as<double4>() : nullptr, c->stream));
    c->pool32_valid = true;
  }
  nsg::PatchDev P = patch_dev(c);
  stage_begin(c, kStageBin);
  LAUNCH(nsg::launch_windows(P, c->win.as<int32_t>(), B, c->stream));
  for (int panel = 0; panel < 3; panel++) {
    if (panel == 0 && !(do_status || do_eps || do_mc)) continue;
    if (panel > 0 && !(do_mc || do_eps)) continue;
    int rc = panel_area(c, panel);
    if (rc) return rc;
  }
  stage_end(c, kStageBin);
  const int64_t nwords = c->words_tot;
  const int64_t nrays_mc = c->mc_tot;
  const int64_t nrows = c->rays_tot[0];
  if (do_status || do_eps) {
    CK(c->srun_off.ensure(nrows * sizeof(int64_t)));
    CK(c->srun_cnt.ensure(nrows * sizeof(int32_t)));
    if (c->srun_cap == 0) c->srun_cap = std::max<int64_t>(4 * nrows, 1 << 16);
  }
  if (do_mc) {
    CK(c->bits.ensure(nwords * sizeof(uint32_t)));
    CK(cudaMemsetAsync(c->bits.p, 0xff, nwords * sizeof(uint32_t), c->stream));
    CK(c->ray_pair_off.ensure(nrays_mc * sizeof(int64_t)));
    CK(c->ray_pair_cnt.ensure(nrays_mc * sizeof(int32_t)));
    CK(cudaMemsetAsync(c->ray_pair_cnt.p, 0, nrays_mc * sizeof(int32_t), c->stream));
    if (c->pair_cap == 0) c->pair_cap = std::max<int64_t>(4 * nrays_mc, 1 << 16);
  }
  CK(c->cursors.ensure(64 * sizeof(unsigned long long)));
  // the ray sets run on their own streams (each with its own candidate lists and hit store) so
  // that the double-precision intersection launches of one set overlap the integer-bound candidate
  // and fill launches of another; or, with concurrent_sets off, one after another on the context's
  // stream through slot 0
  const bool conc = c->concurrent_sets && (do_mc ? 3 : 0) + ((do_status || do_eps) ? 1 : 0) + (do_eps ? 2 : 0) > 1;
  // torus candidates split by resolvent branch (SES patch sets)
  const bool split = c->tune.torus_split && (c->kind_mask & nsg::kSesKinds);
  const auto slot_of = [&](int set) { return conc ? set : 0; };
  {
    int64_t amax = std::max(c->win_area[0], std::max(c->win_area[1], c->win_area[2]));
    c->cand_cap = std::max<int64_t>(c->cand_cap, amax + 1024);
    int64_t nr_all = 0;
    for (int set = 0; set < nsg::kRaySets; set++)
      if (cast(set)) nr_all = std::max(nr_all, c->rays_tot[set]);
    for (int set = 0; set < nsg::kRaySets; set++) {
      if (!cast(set)) continue;
      const int sl = slot_of(set);
      const int64_t nr = conc ? c->rays_tot[set] : nr_all;
      CK(c->hit_t[sl].ensure((size_t)nr * nsg::kHitCap * sizeof(double)));
      CK(c->hit_cnt[sl].ensure(nr * sizeof(int32_t)));
      if (pids) CK(c->hit_pid[sl].ensure((size_t)nr * nsg::kHitCap * sizeof(int32_t)));
    }
    if (grad) CK(c->gvol.ensure(std::max<int64_t>(c->np, 1) * NS_GRAD_PER_PATCH * sizeof(double)));
    if (conc) {
      if (!c->fork_ev) CK(cudaEventCreateWithFlags(&c->fork_ev, cudaEventDisableTiming));
      for (int set = 0; set < nsg::kRaySets; set++) {
        if (!c->set_stream[set]) CK(cudaStreamCreateWithFlags(&c->set_stream[set], cudaStreamNonBlocking));
        if (!c->join_ev[set]) CK(cudaEventCreateWithFlags(&c->join_ev[set], cudaEventDisableTiming));
      }
    }
  }
  CK(c->err.ensure(sizeof(int32_t)));
  const int ovf_cap = 1 << 16;
  for (int attempt = 0; attempt < 4; attempt++) {
    if (do_mc) CK(c->pairs.ensure(c->pair_cap * 2 * sizeof(double)));
    if (do_mc && pids) CK(c->pair_pid.ensure(c->pair_cap * sizeof(int2)));
    if (grad)
      CK(cudaMemsetAsync(c->gvol.p, 0, std::max<int64_t>(c->np, 1) * NS_GRAD_PER_PATCH * sizeof(double), c->stream));
    if (precision == NSG_PRECISION_MIXED) c->def_cap = std::max<int64_t>(c->def_cap, c->cand_cap / 16 + (1 << 16));
    for (int set = 0; set < nsg::kRaySets; set++) {
      if (!cast(set)) continue;
      const int sl = slot_of(set);
      CK(c->cand_sph[sl].ensure(c->cand_cap * sizeof(int2)));
      CK(c->cand_tor[sl].ensure(c->cand_cap * sizeof(int2)));
      if (split) {
        CK(c->tsplit_a[sl].ensure(c->cand_cap * sizeof(int2)));
        CK(c->tsplit_b[sl].ensure(c->cand_cap * sizeof(int2)));
      }
      if (precision == NSG_PRECISION_MIXED) {
        CK(c->def_sph[sl].ensure(c->def_cap * sizeof(int2)));
        CK(c->def_tor[sl].ensure(c->def_cap * sizeof(int2)));
      }
    }
    if (do_status || do_eps) {
      CK(c->sruns.ensure(c->srun_cap * sizeof(int2)));
      CK(cudaMemsetAsync(c->srun_cnt.p, 0, nrows * sizeof(int32_t), c->stream));
    }
    if (keep_hits) {
      if (c->hit_cap == 0)
        c->hit_cap = std::max<int64_t>(8 * (nrays_mc + c->rays_tot[0] + (do_eps ? c->rays_tot[4] + c->rays_tot[5] : 0)),
                                       1 << 16);
      CK(c->hits.ensure(c->hit_cap * sizeof(double)));
    }
    CK(cudaMemsetAsync(c->cursors.p, 0, 64 * sizeof(unsigned long long), c->stream));
    CK(cudaMemsetAsync(c->err.p, 0, sizeof(int32_t), c->stream));
    if (do_mc) CK(cudaMemsetAsync(c->bits.p, 0xff, nwords * sizeof(uint32_t), c->stream));
    // cursors: 0 pairs, 1 kept hits, 2 status runs, 4..6 the overflow counts of the six ray sets
    // (int32), 8 + 2 s the candidate counts of set s (spheres, tori), 20 + 2 s its deferred counts,
    // 32 + 4 s its split torus counts (at +1 and +3)
    unsigned long long* cur = c->cursors.as<unsigned long long>();
    int32_t* ovf_count = (int32_t*)(cur + 4);
    int sets[nsg::kRaySets], nsets = 0;
    for (int set = 0; set < nsg::kRaySets; set++)
      if (cast(set)) sets[nsets++] = set;
    nsg::TraceOut outs[nsg::kRaySets];
    if (do_eps) {
      const size_t eb = (size_t)c->grid.nx * c->grid.ny * c->grid.nz * 3 * sizeof(int32_t);
      CK(c->epsmap.ensure(eb));
      CK(cudaMemsetAsync(c->epsmap.p, 0, eb, c->stream));
    }
    if (c->profile) {
      CK(c->counters.ensure(8 * sizeof(unsigned long long)));
      CK(cudaMemsetAsync(c->counters.p, 0, 8 * sizeof(unsigned long long), c->stream));
    }
    stage_begin(c, kStageTrace);
    if (conc) CK(cudaEventRecord(c->fork_ev, c->stream));
    for (int si = 0; si < nsets; si++) {
      int s = sets[si];
      cudaStream_t st = c->stream;
      if (conc) {
        st = c->set_stream[s];
        CK(cudaStreamWaitEvent(st, c->fork_ev, 0));
      }
      int panel = nsg::ray_set_panel(s);
      int64_t nr = c->rays_tot[s];
      CK(c->vol_ray[s].ensure(nr * sizeof(double)));
      CK(c->ovf_rays[s].ensure(ovf_cap * sizeof(int32_t)));
      nsg::TraceOut o{};
      o.sruns = c->sruns.as<int2>();
      o.srun_cap = c->srun_cap;
      o.srun_cursor = cur + 2;
      o.srun_off = c->srun_off.as<int64_t>();
      o.srun_cnt = c->srun_cnt.as<int32_t>();
      o.bits = c->bits.as<uint32_t>();
      o.vol_ray = c->vol_ray[s].as<double>();
      o.pairs = c->pairs.as<double>();
      o.pair_cap = c->pair_cap;
      o.pair_cursor = cur + 0;
      o.ray_pair_off = c->ray_pair_off.as<int64_t>();
      o.ray_pair_cnt = c->ray_pair_cnt.as<int32_t>();
      o.ovf_rays = c->ovf_rays[s].as<int32_t>();
      o.ovf_cap = ovf_cap;
      o.ovf_count = ovf_count + s;
      o.error_flag = c->err.as<int32_t>();
      o.counters = c->profile ? c->counters.as<unsigned long long>() : nullptr;
      if (do_eps && (s == 0 || s >= 4)) {
        o.epsmap = c->epsmap.as<int32_t>();
        o.eps_inside = NS_EPS_INSIDE;
      }
      if (pids) o.pair_pid = c->pair_pid.as<int2>();
      if (grad) {
        o.gvol = c->gvol.as<double>();
        o.grad_scale = 1.0 / (double)nsets;
      }
      if (keep_hits) {
        CK(c->ray_hit_off[s].ensure(nr * sizeof(int64_t)));
        CK(c->ray_hit_cnt[s].ensure(nr * sizeof(int32_t)));
        CK(cudaMemsetAsync(c->ray_hit_cnt[s].p, 0, nr * sizeof(int32_t), st));
        o.hits = c->hits.as<double>();
        o.hit_cap = c->hit_cap;
        o.hit_cursor = cur + 1;
        o.ray_hit_off = c->ray_hit_off[s].as<int64_t>();
        o.ray_hit_cnt = c->ray_hit_cnt[s].as<int32_t>();
      }
      outs[s] = o;
      const int sl = slot_of(s);
      nsg::CandOut co{c->cand_sph[sl].as<int2>(), c->cand_tor[sl].as<int2>(), c->cand_cap, cur + 8 + 2 * s,
                      c->def_sph[sl].as<int2>(), c->def_tor[sl].as<int2>(), c->def_cap, cur + 20 + 2 * s,
                      split ? c->tsplit_a[sl].as<int2>() : nullptr, split ? c->tsplit_b[sl].as<int2>() : nullptr,
                      split ? cur + 32 + 4 * s : nullptr};
      nsg::HitStore hs{c->hit_t[sl].as<double>(), c->hit_cnt[sl].as<int32_t>(), nr,
                       pids ? c->hit_pid[sl].as<int32_t>() : nullptr};
      CK(cudaMemsetAsync(c->hit_cnt[sl].p, 0, nr * sizeof(int32_t), st));
      c->launches += precision == NSG_PRECISION_MIXED ? 6 : 4;
      cudaEvent_t* ev = nullptr;
      if (c->profile) {
        for (int q = 0; q < 4; q++)
          if (!c->sub_ev[s][q]) CK(cudaEventCreate(&c->sub_ev[s][q]));
        ev = c->sub_ev[s];
      }
      CK(nsg::launch_trace(P, B, s, c->tiles_tot[panel], o, co, hs, precision, c->tune, st, ev));
      if (conc) CK(cudaEventRecord(c->join_ev[s], st));
    }
    if (conc)
      for (int si = 0; si < nsets; si++) CK(cudaStreamWaitEvent(c->stream, c->join_ev[sets[si]], 0));
    stage_end(c, kStageTrace);
    if (c->profile) {
      // candidate, intersection and fill kernels of every ray set (stage_end synchronised the stream)
      for (int si = 0; si < nsets; si++) {
        const int s = sets[si];
        for (int q = 0; q < 3; q++) {
          float ms = 0;
          CK(cudaEventElapsedTime(&ms, c->sub_ev[s][q], c->sub_ev[s][q + 1]));
          c->stage_ms[kStageCand + q] += ms;
          c->stage_calls[kStageCand + q]++;
        }
      }
    }
    int32_t novf[nsg::kRaySets] = {0, 0, 0, 0, 0, 0};
    CK(cudaMemcpyAsync(novf, ovf_count, nsg::kRaySets * sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    int64_t tot_ovf = 0;
    bool tiles_built[3] = {false, false, false};
    stage_begin(c, kStageOverflow);
    for (int si = 0; si < nsets; si++) {
      int s = sets[si];
      int n = std::min(novf[s], ovf_cap);
      tot_ovf += n;
      if (n == 0) continue;
      const int panel = nsg::ray_set_panel(s);
      if (!tiles_built[panel]) {
        int rc = bin_panel(c, panel);
        if (rc) return rc;
        tiles_built[panel] = true;
      }
      CK(c->ovf_scratch.ensure((size_t)n * nsg::kOverflowCap * sizeof(double)));
      if (pids) CK(c->ovf_pscratch.ensure((size_t)n * nsg::kOverflowCap * sizeof(int32_t)));
      LAUNCH(nsg::launch_trace_overflow(P, B, s, c->tile_off[panel].as<int64_t>(), c->tile_list[panel].as<int32_t>(),
                                        outs[s], n, c->ovf_scratch.as<double>(),
                                        pids ? c->ovf_pscratch.as<int32_t>() : nullptr, precision, c->stream));
      CK(cudaStreamSynchronize(c->stream));
    }
    stage_end(c, kStageOverflow);
    c->last_overflow_rays = tot_ovf;
    if (c->profile) {
      CK(cudaMemcpyAsync(c->counter_host, c->counters.p, 8 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                         c->stream));
      unsigned long long cand[2 * nsg::kRaySets];
      CK(cudaMemcpyAsync(cand, cur + 8, 2 * nsg::kRaySets * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                         c->stream));
      CK(cudaStreamSynchronize(c->stream));
      // candidate pairs (spheres + tori) and torus pairs of all ray sets
      c->counter_host[nsg::kCntCandidates] = 0;
      c->counter_host[nsg::kCntTorus] = 0;
      for (int si = 0; si < nsets; si++) {
        c->counter_host[nsg::kCntCandidates] += cand[2 * sets[si]] + cand[2 * sets[si] + 1];
        c->counter_host[nsg::kCntTorus] += cand[2 * sets[si] + 1];
      }
    }
    int32_t errflag = 0;
    unsigned long long used[3] = {0, 0, 0};
    CK(cudaMemcpyAsync(&errflag, c->err.p, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(used, cur, 3 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (errflag == 0) break;
    if (errflag == 3) { c->pair_cap = std::max<int64_t>(2 * c->pair_cap, (int64_t)used[0] + 1024); continue; }
    if (errflag == 2) { c->hit_cap = std::max<int64_t>(2 * c->hit_cap, (int64_t)used[1] + 1024); continue; }
    if (errflag == 5) { c->srun_cap = std::max<int64_t>(2 * c->srun_cap, (int64_t)used[2] + 1024); continue; }
    if (errflag == 6) { c->cand_cap *= 2; continue; }
    if (errflag == 7) { c->def_cap *= 2; continue; }
    return fail(NSG_ERR_CAPACITY, errflag == 1 ? "too many overflow rays" : "ray hit capacity exceeded");
  }
  // volume: A * sum of interval lengths over the ray sets / number of ray sets, per structure; the
  // per-structure sums run in an order fixed by the structure alone, so a structure's volume does
  // not depend on the batch it is part of
  const int32_t nb = c->nstruct;
  std::vector<double> vsum(nb, 0.0);
  int flag_sum = 0;
  CK(c->vol_struct.ensure(nb * sizeof(double)));
  CK(c->seg_part.ensure((size_t)nb * nsg::kSegParts * sizeof(double)));
  for (int s = 0; s < nsg::kRaySets; s++) {
    if (!cast(s)) continue;
    LAUNCH(nsg::launch_segment_sums(c->vol_ray[s].as<double>(), B.ray_base[s], nullptr, nb,
                                    c->vol_struct.as<double>(), c->seg_part.as<double>(), flag_sum > 0, c->stream));
    flag_sum++;
  }
  if (flag_sum) {
    CK(cudaMemcpyAsync(vsum.data(), c->vol_struct.p, nb * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
  }
  for (int32_t b = 0; b < nb; b++) c->volumes[b] = flag_sum ? c->grids[b].A * vsum[b] / flag_sum : 0.0;
  c->volume = c->volumes[0];
  if (volume) *volume = c->volume;
  if ((do_status || do_eps) && nb == 1) {
    int rc = build_free_runs(c);
    if (rc) return rc;
  }
  c->status_dense = false;
  c->cav_detected = c->have_cav_atoms = false;
  c->shape_filtered = c->ideb_ready = false;
  c->have_gvol = grad;
  c->have_pids = pids && do_mc;
  c->have_status = do_status || do_eps;
  c->have_eps = do_eps;
  c->eps_filled = false;
  c->have_bgp = c->bgp_projected = false;
  c->have_bits = do_mc;
  c->n_vert = c->n_tri = 0;
  return NSG_OK;
}

// Labels of the free regions in the order the reference's alternating scan discovers them
// (getCavitiesWithBilevelStatusMap, src/Surface.cpp:2044-2116): regions are given sorted by
// their first node in ascending scan order (k, j, i); desc_key[r] is region r's first node in
// the descending-z scan.  Even rounds take the first remaining region of the ascending scan, odd
// rounds that of the descending scan; the first region found is STATUS_POINT_OUT (3), the next
// ones 4, 5, ...  Host-only; needs no device.
int nsg_cavity_order(int32_t n, const uint32_t* desc_key, int32_t* label_out) {
  if (n < 0 || (n > 0 && (!desc_key || !label_out))) return NSG_ERR_ARG;
  std::vector<int32_t> by_desc(n);
  for (int32_t i = 0; i < n; i++) by_desc[i] = i;
  std::sort(by_desc.begin(), by_desc.end(), [&](int32_t a, int32_t b) { return desc_key[a] < desc_key[b]; });
  std::vector<char> taken(n, 0);
  int32_t pa = 0, pd = 0, id = NS_STATUS_TEMPORARY_OUT;
  for (int32_t t = 0; t < n; t++) {
    int32_t pick;
    if ((t & 1) == 0) {
      while (taken[pa]) pa++;
      pick = pa;
    } else {
      while (taken[by_desc[pd]]) pd++;
      pick = by_desc[pd];
    }
    taken[pick] = 1;
    label_out[pick] = ++id;
  }
  return NSG_OK;
}

}  // extern "C"

namespace {

// Region labelling of the context's free runs and conditional filling.  With `pockets` every
// region is a cavity (getCavitiesWithBilevelStatusMap with idStart = STATUS_POINT_OUT, as the
// difference map is labelled), else the first region found is the outside.
int detect_cavities(nsg_ctx* c, double cav_vol, bool pockets, int* ncav_out) {
  const NsGrid& g = c->grid;
  const int64_t nr = c->n_fruns;
  c->cav_size.clear();
  c->cav_filled.clear();
  c->cav_count.clear();
  c->cav_nodes = 0;
  c->cav_detected = c->have_cav_atoms = false;
  c->shape_filtered = c->ideb_ready = false;
  stage_begin(c, kStageCavity);
  CK(c->labels.ensure(std::max<int64_t>(nr, 1) * sizeof(int32_t)));
  CK(c->is_root.ensure(std::max<int64_t>(nr, 1)));
  CK(c->roots.ensure(std::max<int64_t>(nr, 1) * sizeof(int32_t)));
  CK(c->nroots_d.ensure(sizeof(int32_t)));
  nsg::RunArgs A = run_args(c);
  c->launches += 3;
  CK(nsg::run_label(A, c->is_root.as<uint8_t>(), c->stream));
  int32_t nroots = 0;
  if (nr > 0) {
    size_t tb = 0;
    CK(nsg::run_select_roots(c->is_root.as<uint8_t>(), nr, nullptr, nullptr, nullptr, &tb, c->stream));
    CK(c->temp.ensure(tb));
    tb = c->temp.cap;
    CK(nsg::run_select_roots(c->is_root.as<uint8_t>(), nr, c->roots.as<int32_t>(), c->nroots_d.as<int32_t>(),
                             c->temp.p, &tb, c->stream));
    CK(cudaMemcpyAsync(&nroots, c->nroots_d.p, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
  }
  if (nroots == 0) {
    c->ncav = 0;
    int rc = materialize_status(c, nullptr);
    if (rc) return rc;
    stage_end(c, kStageCavity);
    c->cav_detected = true;
    if (ncav_out) *ncav_out = 0;
    return NSG_OK;
  }
  CK(c->cc_count.ensure(nroots * sizeof(unsigned long long)));
  CK(c->cc_desc.ensure(nroots * sizeof(unsigned int)));
  CK(cudaMemsetAsync(c->cc_count.p, 0, nroots * sizeof(unsigned long long), c->stream));
  CK(cudaMemsetAsync(c->cc_desc.p, 0xff, nroots * sizeof(unsigned int), c->stream));
  LAUNCH(nsg::run_stats(A, c->roots.as<int32_t>(), nroots, c->cc_count.as<unsigned long long>(),
                        c->cc_desc.as<unsigned int>(), c->stream));
  std::vector<unsigned long long> cnt(nroots);
  std::vector<unsigned int> desc(nroots);
  CK(cudaMemcpyAsync(cnt.data(), c->cc_count.p, nroots * sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(desc.data(), c->cc_desc.p, nroots * sizeof(unsigned int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  std::vector<int32_t> label_of(nroots, 0);
  std::vector<uint8_t> fill_of(nroots, 0);
  nsg_cavity_order(nroots, desc.data(), label_of.data());
  if (pockets)
    for (auto& l : label_of) l++;
  const int32_t id = NS_STATUS_TEMPORARY_OUT + nroots + (pockets ? 1 : 0);
  const double cube = g.side * g.side * g.side;
  c->ncav = id - NS_STATUS_OUT;
  c->cav_size.assign(c->ncav, 0.0);
  c->cav_filled.assign(c->ncav, 0);
  c->cav_count.assign(c->ncav, 0);
  for (int32_t r = 0; r < nroots; r++) {
    int lab = label_of[r];
    if (lab < NS_STATUS_FIRST_CAV) continue;
    double v = (double)cnt[r] * cube;
    c->cav_nodes += (int64_t)cnt[r];
    c->cav_count[lab - NS_STATUS_FIRST_CAV] = (int64_t)cnt[r];
    c->cav_size[lab - NS_STATUS_FIRST_CAV] = v;
    if (v <= cav_vol) {
      c->cav_filled[lab - NS_STATUS_FIRST_CAV] = 1;
      fill_of[r] = 1;
    }
  }
  CK(c->cc_label_of.ensure(nroots * sizeof(int32_t)));
  CK(c->cc_fill_of.ensure(nroots));
  CK(cudaMemcpyAsync(c->cc_label_of.p, label_of.data(), nroots * sizeof(int32_t), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->cc_fill_of.p, fill_of.data(), nroots, cudaMemcpyHostToDevice, c->stream));
  if (c->have_bits)
    LAUNCH(nsg::run_fill(A, c->cc_fill_of.as<uint8_t>(), c->bits.as<uint32_t>(), nwords_of(g), c->stream));
  if (c->have_eps) {
    LAUNCH(nsg::eps_fill_cavities(A, c->cc_fill_of.as<uint8_t>(), c->epsmap.as<int32_t>(), NS_EPS_INSIDE, c->stream));
    c->eps_filled = true;
    c->have_bgp = false;
  }
  int rc = materialize_status(c, c->cc_label_of.as<int32_t>());
  if (rc) return rc;
  stage_end(c, kStageCavity);
  CK(cudaStreamSynchronize(c->stream));
  c->cav_detected = true;
  if (ncav_out) *ncav_out = c->ncav;
  c->n_vert = c->n_tri = 0;
  return NSG_OK;
}

}  // namespace

extern "C" {

int nsg_cavities(nsg_ctx* c, double cav_vol, int* ncav_out) {
  if (!c || !c->have_status) return fail(NSG_ERR_STATE, "cavity detection needs the status map");
  if (c->nstruct != 1) return fail(NSG_ERR_STATE, "cavity detection runs on a single structure");
  CK(cudaSetDevice(c->device));
  return detect_cavities(c, cav_vol, false, ncav_out);
}

int nsg_filter_cavities(nsg_ctx* c, double probe_radius, int modify_status, int64_t* n_removed);

int nsg_pocket_difference(nsg_ctx* c, nsg_ctx* small, double fill_volume, int* n_pockets) {
  if (!c || !small || c == small) return NSG_ERR_ARG;
  if (!c->have_status || !small->have_status) return fail(NSG_ERR_STATE, "the difference needs both status maps");
  if (c->nstruct != 1 || small->nstruct != 1) return fail(NSG_ERR_STATE, "the difference runs on single structures");
  if (c->device != small->device) return fail(NSG_ERR_ARG, "both surfaces must live on one device");
  const NsGrid& g = c->grid;
  const NsGrid& h = small->grid;
  if (g.nx != h.nx || g.ny != h.ny || g.nz != h.nz) return fail(NSG_ERR_ARG, "the two grids differ");
  CK(cudaSetDevice(c->device));
  const int64_t nn = g.nx * g.ny * g.nz;
  if (!c->status_dense) {
    int rc = materialize_status(c, nullptr);
    if (rc) return rc;
  }
  if (!small->status_dense) {
    int rc = materialize_status(small, nullptr);
    if (rc) return rc;
  }
  CK(cudaStreamSynchronize(small->stream));
  stage_begin(c, kStageCavity);
  CK(c->ca_count.ensure(2 * sizeof(unsigned long long)));
  CK(cudaMemsetAsync(c->ca_count.p, 0, sizeof(unsigned long long), c->stream));
  LAUNCH(nsg::pocket_difference(c->status.as<int32_t>(), small->status.as<int32_t>(), nn,
                                c->have_bits ? c->bits.as<uint32_t>() : nullptr, c->ca_count.as<unsigned long long>(),
                                c->stream));
  unsigned long long ndiff = 0;
  CK(cudaMemcpyAsync(&ndiff, c->ca_count.p, sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  // the difference is one cavity, kept, for the Connolly filter with a 1.4 A probe
  c->ncav = 1;
  c->cav_count.assign(1, (int64_t)ndiff);
  c->cav_size.assign(1, (double)ndiff * g.side * g.side * g.side);
  c->cav_filled.assign(1, 0);
  c->cav_nodes = (int64_t)ndiff;
  c->status_dense = c->cav_detected = true;
  c->shape_filtered = c->have_cav_atoms = false;
  c->eps_filled = false;
  int rc = ndiff ? nsg_filter_cavities(c, 1.4, 1, nullptr) : NSG_OK;
  if (rc) return rc;
  if (ndiff) LAUNCH(nsg::pocket_cav2out(c->status.as<int32_t>(), c->cav_label.as<int32_t>(), nn, c->stream));
  // the filtered map's free runs replace the cast's, then the regions are labelled as pockets
  const int64_t nrows = g.ny * g.nz;
  CK(c->fr_cnt.ensure(nrows * sizeof(int32_t)));
  CK(c->fr_off.ensure((nrows + 1) * sizeof(int64_t)));
  nsg::RunArgs A = run_args(c);
  LAUNCH(nsg::dense_free_runs(A, c->status.as<int32_t>(), 0, c->stream));
  int64_t nr = 0;
  rc = scan_counts(c, c->fr_cnt.as<int32_t>(), nrows, c->fr_off.as<int64_t>(), &nr);
  if (rc) return rc;
  CK(c->fruns.ensure(std::max<int64_t>(nr, 1) * sizeof(int2)));
  CK(c->frow.ensure(std::max<int64_t>(nr, 1) * sizeof(int32_t)));
  c->n_fruns = nr;
  A = run_args(c);
  LAUNCH(nsg::dense_free_runs(A, c->status.as<int32_t>(), 1, c->stream));
  stage_end(c, kStageCavity);
  return detect_cavities(c, fill_volume, true, n_pockets);
}

int nsg_filter_cavities(nsg_ctx* c, double probe_radius, int modify_status, int64_t* n_removed) {
  if (!c || !(probe_radius > 0)) return NSG_ERR_ARG;
  if (!c->cav_detected || !c->status_dense || c->nstruct != 1)
    return fail(NSG_ERR_STATE, "the shape filter needs nsg_cavities after the cast");
  if (c->shape_filtered) return fail(NSG_ERR_STATE, "the shape filter runs once per cavity detection");
  if (n_removed) *n_removed = 0;
  if (c->ncav == 0) return NSG_OK;
  CK(cudaSetDevice(c->device));
  const NsGrid& g = c->grid;
  const int64_t nn = g.nx * g.ny * g.nz;
  const int ncav = c->ncav;
  CK(c->cav_label.ensure(nn * sizeof(int32_t)));
  CK(c->sh_support.ensure(nn));
  CK(c->sh_removed[0].ensure(nn));
  CK(c->sh_removed[1].ensure(nn));
  CK(c->sh_later.ensure(nn));
  CK(c->sh_filled.ensure(ncav));
  CK(c->sh_nrem.ensure(ncav * sizeof(unsigned long long)));
  CK(c->sh_changed.ensure(sizeof(int32_t)));
  std::vector<uint8_t> filled(ncav);
  for (int q = 0; q < ncav; q++) filled[q] = c->cav_filled[q] ? 1 : 0;
  CK(cudaMemcpyAsync(c->cav_label.p, c->status.p, nn * sizeof(int32_t), cudaMemcpyDeviceToDevice, c->stream));
  CK(cudaMemcpyAsync(c->sh_filled.p, filled.data(), ncav, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemsetAsync(c->sh_nrem.p, 0, ncav * sizeof(unsigned long long), c->stream));
  if (c->have_eps && !c->ideb_ready) {
    CK(c->ideb.ensure(nn));
    nsg::RunArgs R = run_args(c);
    LAUNCH(nsg::ideb_write(R, c->eps_filled ? c->cc_fill_of.as<uint8_t>() : nullptr, c->ideb.as<uint8_t>(),
                           c->stream));
  }
  nsg::ShapeArgs A{};
  A.status = c->status.as<int32_t>();
  A.label = c->cav_label.as<int32_t>();
  A.nx = g.nx;
  A.ny = g.ny;
  A.nz = g.nz;
  A.mn[0] = g.xmin;
  A.mn[1] = g.ymin;
  A.mn[2] = g.zmin;
  A.side = g.side;
  A.scale = g.scale;
  A.r = probe_radius;
  A.filled = c->sh_filled.as<uint8_t>();
  A.mod_status = modify_status ? 1 : 0;
  A.support = c->sh_support.as<uint8_t>();
  A.later = c->sh_later.as<uint8_t>();
  A.changed = c->sh_changed.as<int32_t>();
  A.bits = c->have_bits ? c->bits.as<uint32_t>() : nullptr;
  A.nwords = nwords_of(g);
  A.eps = c->have_eps ? c->epsmap.as<int32_t>() : nullptr;
  A.ideb = c->have_eps ? c->ideb.as<uint8_t>() : nullptr;
  A.n_removed = c->sh_nrem.as<unsigned long long>();
  // pass t is exact for cavities 0..t; a pass that changes no removed flag is the fixed point
  // (a modified status map turns removed nodes inside at once: one pass)
  int cur = 0;
  for (int pass = 0; pass <= ncav; pass++) {
    A.removed = c->sh_removed[cur].as<uint8_t>();
    A.removed_prev = pass ? c->sh_removed[cur ^ 1].as<uint8_t>() : nullptr;
    CK(cudaMemsetAsync(c->sh_changed.p, 0, sizeof(int32_t), c->stream));
    c->launches += 2;
    CK(nsg::shape_pass(A, c->stream));
    if (modify_status) break;
    int32_t changed = 0;
    CK(cudaMemcpyAsync(&changed, c->sh_changed.p, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (pass && !changed) break;
    if (pass == ncav) return fail(NSG_ERR_STATE, "the shape filter did not settle");
    cur ^= 1;
  }
  LAUNCH(nsg::shape_apply(A, c->stream));
  std::vector<unsigned long long> nrem(ncav);
  CK(cudaMemcpyAsync(nrem.data(), c->sh_nrem.p, ncav * sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  int64_t tot = 0;
  for (int q = 0; q < ncav; q++) {
    tot += (int64_t)nrem[q];
    // partially filled cavities stay open; completely filled ones are flagged
    if (!c->cav_filled[q] && nrem[q] > 0 && (int64_t)nrem[q] == c->cav_count[q]) c->cav_filled[q] = 1;
  }
  c->shape_filtered = true;
  c->ideb_ready = c->have_eps;
  c->have_cav_atoms = false;
  if (c->have_eps) c->have_bgp = c->bgp_projected = false;
  c->n_vert = c->n_tri = 0;
  if (n_removed) *n_removed = tot;
  return NSG_OK;
}

int nsg_triangulate(nsg_ctx* c, double* area_out, int64_t* nverts, int64_t* ntris) {
  if (!c || !c->have_bits) return fail(NSG_ERR_STATE, "triangulation needs the accurate-triangulation rays");
  CK(cudaSetDevice(c->device));
  const nsg::BatchDev B = batch_dev(c);
  const int64_t nrays = c->mc_tot;
  CK(c->surv_cnt.ensure(nrays * sizeof(int32_t)));
  CK(c->surv_off.ensure((nrays + 1) * sizeof(int64_t)));
  nsg::VertArgs V{};
  V.B = B;
  V.nrays = nrays;
  V.ray_pair_off = c->ray_pair_off.as<int64_t>();
  V.ray_pair_cnt = c->ray_pair_cnt.as<int32_t>();
  V.pairs = c->pairs.as<double>();
  V.bits = c->bits.as<uint32_t>();
  V.surv_cnt = c->surv_cnt.as<int32_t>();
  V.surv_off = c->surv_off.as<int64_t>();
  stage_begin(c, kStageVertex);
  LAUNCH(nsg::launch_vert(V, 0, c->stream));
  int64_t n_an = 0;
  int rc = scan_counts(c, c->surv_cnt.as<int32_t>(), nrays, c->surv_off.as<int64_t>(), &n_an);
  if (rc) return rc;
  // rows of cubes
  const int64_t nrows = c->rows_tot;
  CK(c->row_act_cnt.ensure((nrows + 1) * sizeof(int64_t)));
  CK(c->row_act_off.ensure((nrows + 1) * sizeof(int64_t)));
  nsg::MCArgs M{};
  M.B = B;
  M.row_chunks = c->d_row_chunks.as<int4>();
  M.nchunks = c->nchunks;
  M.bits = c->bits.as<uint32_t>();
  M.surv_cnt = c->surv_cnt.as<int32_t>();
  M.surv_off = c->surv_off.as<int64_t>();
  M.n_analytic = n_an;
  M.nrows = nrows;
  M.row_act_cnt = c->row_act_cnt.as<int64_t>();
  stage_end(c, kStageVertex, false);
  stage_begin(c, kStageMC);
  // active cubes, their map and vertex slots (the vertex pass writes into the slots)
  LAUNCH(nsg::launch_mc_rows(M, 0, c->stream));
  int64_t n_act = 0, n_mid = 0;
  rc = scan_counts(c, c->row_act_cnt.as<int64_t>(), nrows, c->row_act_off.as<int64_t>(), &n_act);
  if (rc) return rc;
  if (n_act >= ((int64_t)1 << 31) / 12) return fail(NSG_ERR_CAPACITY, "too many active cubes in one batch");
  M.row_act_off = c->row_act_off.as<int64_t>();
  CK(c->act_rec.ensure(std::max<int64_t>(n_act, 1) * sizeof(int4)));
  CK(c->act_mid.ensure(std::max<int64_t>(n_act, 1) * sizeof(int32_t)));
  CK(c->row_mid_cnt.ensure(std::max<int64_t>(n_act, 1) * sizeof(int32_t)));
  CK(c->row_mid_off.ensure((n_act + 1) * sizeof(int64_t)));
  M.act_rec = c->act_rec.as<int4>();
  M.act_mid = c->act_mid.as<int32_t>();
  M.mid_cnt = c->row_mid_cnt.as<int32_t>();
  M.mid_off = c->row_mid_off.as<int64_t>();
  M.n_active = n_act;
  // the active-cube map (per 32 cubes of a row: their active bits and the first one's index) and
  // 12 vertex slots per active cube, all -1 until the vertices are written into them
  CK(c->amap.ensure(std::max<int64_t>(c->awords_tot, 1) * sizeof(int2)));
  CK(c->cube_vl.ensure(std::max<int64_t>(n_act, 1) * 12 * sizeof(int32_t)));
  M.amap = c->amap.as<int2>();
  M.cube_vl = c->cube_vl.as<int32_t>();
  // triangle counts per active cube: the case table's for interior cubes (written by the
  // classification), a count over the vertex slots for the listed low-face cubes
  CK(c->tri_cnt.ensure(std::max<int64_t>(n_act, 1) * sizeof(int32_t)));
  CK(c->bnd_list.ensure(std::max<int64_t>(n_act, 1) * sizeof(int32_t)));
  CK(c->bnd_cursor.ensure(sizeof(unsigned long long)));
  CK(cudaMemsetAsync(c->bnd_cursor.p, 0, sizeof(unsigned long long), c->stream));
  M.tri_cnt = c->tri_cnt.as<int32_t>();
  M.bnd_list = c->bnd_list.as<int32_t>();
  M.bnd_cursor = c->bnd_cursor.as<unsigned long long>();
  LAUNCH(nsg::launch_mc_rows(M, 1, c->stream));
  stage_end(c, kStageMC, false);
  // analytic vertices, then each first vertex of an edge into the slots of the edge's cubes
  stage_begin(c, kStageVertex);
  CK(c->vkey.ensure(std::max<int64_t>(n_an, 1) * sizeof(int4)));
  CK(c->vpos.ensure(std::max<int64_t>(n_an, 1) * 3 * sizeof(double)));
  V.vpos = c->vpos.as<double>();
  V.vkey = c->vkey.as<int4>();
  CK(c->vstruct.ensure(std::max<int64_t>(n_an, 1) * sizeof(int32_t)));
  V.vstruct = c->vstruct.as<int32_t>();
  const bool grad = c->grad_mode && c->have_gvol;
  if (c->have_pids) {
    CK(c->vpid.ensure(std::max<int64_t>(n_an, 1) * sizeof(int32_t)));
    V.pair_pid = c->pair_pid.as<int2>();
    V.vpid = c->vpid.as<int32_t>();
  }
  LAUNCH(nsg::launch_vert(V, 1, c->stream));
  stage_end(c, kStageVertex);
  stage_begin(c, kStageMC);
  M.vpos = c->vpos.as<double>();
  M.vkey = c->vkey.as<int4>();
  M.vstruct = c->vstruct.as<int32_t>();
  {
    // The slots are cleared to -1 and the analytic vertices written into them structure chunk by
    // structure chunk, each chunk's slots small enough to stay in L2 between the two: the push's
    // 4-byte stores then complete sectors in L2 instead of making DRAM read every sector back.
    const int32_t nb = c->nstruct;
    CK(c->chunk_off.ensure(2 * (size_t)(nb + 1) * sizeof(int64_t)));
    int64_t* d_off = c->chunk_off.as<int64_t>();
    LAUNCH(nsg::launch_gather_i64(c->surv_off.as<int64_t>(), B.mc_base, nb + 1, d_off, c->stream));
    LAUNCH(nsg::launch_gather_i64(c->row_act_off.as<int64_t>(), B.row_base, nb + 1, d_off + nb + 1, c->stream));
    std::vector<int64_t> off(2 * (size_t)(nb + 1));
    CK(cudaMemcpyAsync(off.data(), d_off, off.size() * sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    const int64_t* voff = off.data();
    const int64_t* aoff = off.data() + nb + 1;
    constexpr int64_t kChunkCubes = (int64_t)1 << 20;  // 48 MB of slots
    for (int32_t b0 = 0; b0 < nb;) {
      int32_t b1 = b0 + 1;
      while (b1 < nb && aoff[b1 + 1] - aoff[b0] <= kChunkCubes) b1++;
      const int64_t a0 = aoff[b0], a1 = aoff[b1];
      if (a1 > a0) CK(cudaMemsetAsync(c->cube_vl.as<int32_t>() + 12 * a0, 0xff, (a1 - a0) * 12 * sizeof(int32_t),
                                      c->stream));
      LAUNCH(nsg::launch_mc_push(M, voff[b0], voff[b1], c->stream));
      b0 = b1;
    }
  }
  // midpoint vertices of cut edges without an analytic vertex
  LAUNCH(nsg::launch_mc_mid(M, 0, c->stream));
  rc = scan_counts(c, c->row_mid_cnt.as<int32_t>(), n_act, c->row_mid_off.as<int64_t>(), &n_mid);
  if (rc) return rc;
  const int64_t n_v = n_an + n_mid;
  if ((size_t)n_v * sizeof(int4) > c->vkey.cap || (size_t)n_v * 3 * sizeof(double) > c->vpos.cap) {
    DevBuf nk, np_;
    CK(nk.ensure(n_v * sizeof(int4)));
    CK(np_.ensure(n_v * 3 * sizeof(double)));
    if (n_an) {
      CK(cudaMemcpyAsync(nk.p, c->vkey.p, n_an * sizeof(int4), cudaMemcpyDeviceToDevice, c->stream));
      CK(cudaMemcpyAsync(np_.p, c->vpos.p, n_an * 3 * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    }
    CK(cudaStreamSynchronize(c->stream));
    c->vkey.release();
    c->vpos.release();
    c->vkey = nk;
    c->vpos = np_;
  }
  if ((size_t)n_v * sizeof(int32_t) > c->vstruct.cap) {
    DevBuf ns;
    CK(ns.ensure(n_v * sizeof(int32_t)));
    if (n_an) CK(cudaMemcpyAsync(ns.p, c->vstruct.p, n_an * sizeof(int32_t), cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->vstruct.release();
    c->vstruct = ns;
  }
  M.vpos = c->vpos.as<double>();
  M.vkey = c->vkey.as<int4>();
  M.vstruct = c->vstruct.as<int32_t>();
  LAUNCH(nsg::launch_mc_mid(M, 1, c->stream));
  M.n_active = n_act;
  CK(c->tri_off.ensure((n_act + 1) * sizeof(int64_t)));
  CK(c->cube_area.ensure(std::max<int64_t>(n_act, 1) * sizeof(double)));
  M.tri_cnt = c->tri_cnt.as<int32_t>();
  M.cube_area = c->cube_area.as<double>();
  if (grad) {
    const nsg::PatchDev P = patch_dev(c);
    CK(c->vgrad.ensure(std::max<int64_t>(n_an, 1) * sizeof(double)));
    CK(c->garea.ensure(std::max<int64_t>(c->np, 1) * NS_GRAD_PER_PATCH * sizeof(double)));
    CK(cudaMemsetAsync(c->vgrad.p, 0, std::max<int64_t>(n_an, 1) * sizeof(double), c->stream));
    CK(cudaMemsetAsync(c->garea.p, 0, std::max<int64_t>(c->np, 1) * NS_GRAD_PER_PATCH * sizeof(double), c->stream));
    M.vpid = c->vpid.as<int32_t>();
    M.vgrad = c->vgrad.as<double>();
    M.garea = c->garea.as<double>();
    M.f64 = P.f64;
    M.i32 = P.i32;
    M.probe = P.probe;
  }
  LAUNCH(nsg::launch_mc_tris_bnd(M, c->stream));
  int64_t n_tri = 0;
  rc = scan_counts(c, c->tri_cnt.as<int32_t>(), n_act, c->tri_off.as<int64_t>(), &n_tri);
  if (rc) return rc;
  CK(c->tris.ensure(std::max<int64_t>(n_tri, 1) * 3 * sizeof(int32_t)));
  M.tri_off = c->tri_off.as<int64_t>();
  M.tris = c->tris.as<int32_t>();
  LAUNCH(nsg::launch_mc_tris(M, c->tune.mc_tris_bpsm, c->stream));
  if (grad) LAUNCH(nsg::launch_grad_vert(M, c->stream));
  c->have_garea = grad;
  // per-structure areas in an order fixed by the structure alone (independent of the batch)
  CK(c->area_struct.ensure(c->nstruct * sizeof(double)));
  CK(c->seg_part.ensure((size_t)c->nstruct * nsg::kSegParts * sizeof(double)));
  LAUNCH(nsg::launch_segment_sums(c->cube_area.as<double>(), c->row_act_off.as<int64_t>(), B.row_base, c->nstruct,
                                  c->area_struct.as<double>(), c->seg_part.as<double>(), false, c->stream));
  CK(cudaMemcpyAsync(c->areas.data(), c->area_struct.p, c->nstruct * sizeof(double), cudaMemcpyDeviceToHost,
                     c->stream));
  CK(cudaStreamSynchronize(c->stream));
  const double area = c->areas[0];
  stage_end(c, kStageMC);
  c->n_analytic = n_an;
  c->n_vert = n_v;
  c->n_tri = n_tri;
  c->n_active = n_act;
  c->area = area;
  if (area_out) *area_out = area;
  if (nverts) *nverts = n_v;
  if (ntris) *ntris = n_tri;
  return NSG_OK;
}

// Vertex normals of the last triangulation (Compute_Vertex_Normals): for a surface with analytic
// normals the normal of each analytic vertex's patch at the vertex (ConnollySurface::getNormal,
// src/ConnollySurface.cpp:5736-5819; the skin quadric's gradient, src/SkinSurface.cpp:3684-3712),
// the others (midpoint vertices, mesh surfaces) by triangle averaging as approximateNormals does
// for the vertices whose normal is zero (src/Surface.cpp:10420-10460, 10588-10735).
int nsg_vertex_normals(nsg_ctx* c, double* normals) {
  if (!c || !normals) return NSG_ERR_ARG;
  if (!c->have_pids) return fail(NSG_ERR_STATE, "ray cast with NSG_RAYCAST_NORMALS (or NSG_RAYCAST_GRAD) first");
  const int64_t nv = c->n_vert, nt = c->n_tri;
  if (nv == 0) return NSG_OK;
  CK(cudaSetDevice(c->device));
  DevBuf dn;
  CK(dn.ensure(nv * 3 * sizeof(double)));
  CK(cudaMemsetAsync(dn.p, 0, nv * 3 * sizeof(double), c->stream));
  const nsg::PatchDev P = patch_dev(c);
  LAUNCH(nsg::launch_vertex_normals(c->vpos.as<double>(), c->vpid.as<int32_t>(), c->n_analytic, P.f64, P.i32, P.probe,
                                    dn.as<double>(), c->stream));
  std::vector<double> verts(nv * 3);
  std::vector<int32_t> tris(std::max<int64_t>(nt, 1) * 3);
  CK(cudaMemcpyAsync(normals, dn.p, nv * 3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(verts.data(), c->vpos.p, nv * 3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  if (nt) CK(cudaMemcpyAsync(tris.data(), c->tris.p, nt * 3 * sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  dn.release();
  return nsg_fill_zero_normals(verts.data(), nv, tris.data(), nt, normals);
}

int nsg_download_status(nsg_ctx* c, int32_t* dst) {
  if (!c || !dst || !c->have_status) return NSG_ERR_STATE;
  if (c->nstruct != 1) return fail(NSG_ERR_STATE, "the dense status map is kept for a single structure");
  CK(cudaSetDevice(c->device));
  if (!c->status_dense) {
    int rc = materialize_status(c, nullptr);
    if (rc) return rc;
  }
  const NsGrid& g = c->grid;
  CK(cudaMemcpyAsync(dst, c->status.p, g.nx * g.ny * g.nz * sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return NSG_OK;
}

int nsg_download_insideness(nsg_ctx* c, uint32_t* dst) {
  if (!c || !dst || !c->have_bits) return NSG_ERR_STATE;
  CK(cudaMemcpyAsync(dst, c->bits.p, c->words_tot * sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return NSG_OK;
}

int nsg_download_mesh(nsg_ctx* c, double* verts, int32_t* vkeys, int32_t* tris) {
  if (!c) return NSG_ERR_ARG;
  if (verts && c->n_vert)
    CK(cudaMemcpyAsync(verts, c->vpos.p, c->n_vert * 3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  if (vkeys && c->n_vert)
    CK(cudaMemcpyAsync(vkeys, c->vkey.p, c->n_vert * sizeof(int4), cudaMemcpyDeviceToHost, c->stream));
  if (tris && c->n_tri)
    CK(cudaMemcpyAsync(tris, c->tris.p, c->n_tri * 3 * sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return NSG_OK;
}

int nsg_download_cavities(nsg_ctx* c, double* sizes, int32_t* filled) {
  if (!c) return NSG_ERR_ARG;
  if (sizes && !c->cav_size.empty()) memcpy(sizes, c->cav_size.data(), c->cav_size.size() * sizeof(double));
  if (filled && !c->cav_filled.empty()) memcpy(filled, c->cav_filled.data(), c->cav_filled.size() * sizeof(int32_t));
  return NSG_OK;
}

int nsg_cavity_atoms(nsg_ctx* c, const double* atoms_xyzr, int64_t n_atoms, int32_t* offsets, int32_t* atoms,
                     int64_t* n_total) {
  if (!c || (n_atoms > 0 && !atoms_xyzr) || n_atoms < 0 || (atoms && !offsets)) return NSG_ERR_ARG;
  if (!c->cav_detected || !c->status_dense || c->nstruct != 1)
    return fail(NSG_ERR_STATE, "cavity atoms need nsg_cavities after the cast");
  if (!c->have_cav_atoms) {
    CK(cudaSetDevice(c->device));
    const NsGrid& g = c->grid;
    c->cav_atom_off.assign(c->ncav + 1, 0);
    c->cav_atom_list.clear();
    if (c->ncav > 0 && c->cav_nodes > 0) {
      if (c->cav_nodes >= ((int64_t)1 << 31)) return fail(NSG_ERR_CAPACITY, "more than 2^31 cavity nodes");
      // the reference's atom grid (buildAtomsMap)
      double rmax = 0;
      for (int64_t a = 0; a < n_atoms; a++) rmax = std::max(atoms_xyzr[4 * a + 3], rmax);
      if (!(rmax > 0)) return fail(NSG_ERR_ARG, "cavity atoms need atoms of positive radius");
      double gscale = 0.5 / rmax;
      unsigned int ggrid = 1;
      for (int it = 0; it < 4096; it++) {
        ggrid = (unsigned int)floor(gscale * 1.3 * g.rmaxdim);
        if (ggrid <= 100) {
          if (ggrid <= 0) gscale *= 2.0;
          else break;
        } else {
          gscale *= 0.5;
        }
      }
      if (ggrid == 0 || ggrid > 100) return fail(NSG_ERR_ARG, "atom grid size out of range");
      const double gside = 1. / gscale;
      const int64_t gn = ggrid, ncell = gn * gn * gn;
      double gmn[3];
      for (int d = 0; d < 3; d++) gmn[d] = g.baricenter[d] - (ggrid - 1) * 0.5 * gside;
      std::vector<int32_t> cell_of(n_atoms), cell_off(ncell + 1, 0), cell_atoms(n_atoms);
      for (int64_t a = 0; a < n_atoms; a++) {
        int64_t ix[3];
        for (int d = 0; d < 3; d++) ix[d] = (int64_t)floor((atoms_xyzr[4 * a + d] - gmn[d]) * gscale + 0.5);
        if (ix[0] < 0 || ix[1] < 0 || ix[2] < 0 || ix[0] >= gn || ix[1] >= gn || ix[2] >= gn)
          return fail(NSG_ERR_ARG, "an atom lies outside the atom grid (atoms of another structure?)");
        cell_of[a] = (int32_t)((ix[2] * gn + ix[1]) * gn + ix[0]);
        cell_off[cell_of[a] + 1]++;
      }
      for (int64_t q = 0; q < ncell; q++) cell_off[q + 1] += cell_off[q];
      {
        std::vector<int32_t> cur(cell_off.begin(), cell_off.end() - 1);
        for (int64_t a = 0; a < n_atoms; a++) cell_atoms[cur[cell_of[a]]++] = (int32_t)a;
      }
      const int64_t cap = c->cav_nodes;
      CK(c->ca_atoms.ensure(std::max<int64_t>(n_atoms, 1) * 4 * sizeof(double)));
      CK(c->ca_cell_off.ensure((ncell + 1) * sizeof(int32_t)));
      CK(c->ca_cell_atoms.ensure(std::max<int64_t>(n_atoms, 1) * sizeof(int32_t)));
      CK(c->ca_pairs.ensure(cap * sizeof(unsigned long long)));
      CK(c->ca_alt.ensure(cap * sizeof(unsigned long long)));
      CK(c->ca_count.ensure(2 * sizeof(unsigned long long)));
      if (n_atoms)
        CK(cudaMemcpyAsync(c->ca_atoms.p, atoms_xyzr, n_atoms * 4 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
      CK(cudaMemcpyAsync(c->ca_cell_off.p, cell_off.data(), (ncell + 1) * sizeof(int32_t), cudaMemcpyHostToDevice,
                         c->stream));
      if (n_atoms)
        CK(cudaMemcpyAsync(c->ca_cell_atoms.p, cell_atoms.data(), n_atoms * sizeof(int32_t), cudaMemcpyHostToDevice,
                           c->stream));
      CK(cudaMemsetAsync(c->ca_count.p, 0, 2 * sizeof(unsigned long long), c->stream));
      CK(cudaMemsetAsync(c->err.p, 0, sizeof(int32_t), c->stream));
      nsg::CavAtomArgs A{};
      A.status = c->status.as<int32_t>();
      A.label = c->shape_filtered ? c->cav_label.as<int32_t>() : nullptr;
      A.nx = g.nx;
      A.ny = g.ny;
      A.nz = g.nz;
      A.mn[0] = g.xmin;
      A.mn[1] = g.ymin;
      A.mn[2] = g.zmin;
      A.side = g.side;
      A.gn = gn;
      for (int d = 0; d < 3; d++) A.gmn[d] = gmn[d];
      A.gscale = gscale;
      A.cell_off = c->ca_cell_off.as<int32_t>();
      A.cell_atoms = c->ca_cell_atoms.as<int32_t>();
      A.atoms = c->ca_atoms.as<double>();
      A.pairs = c->ca_pairs.as<unsigned long long>();
      A.count = c->ca_count.as<unsigned long long>();
      A.cap = cap;
      A.err = c->err.as<int32_t>();
      LAUNCH(nsg::cavity_atom_pairs(A, c->stream));
      unsigned long long npairs = 0;
      int32_t errflag = 0;
      CK(cudaMemcpyAsync(&npairs, c->ca_count.p, sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->stream));
      CK(cudaMemcpyAsync(&errflag, c->err.p, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
      CK(cudaStreamSynchronize(c->stream));
      if (errflag) return fail(NSG_ERR_CAPACITY, "cavity boundary nodes exceed the cavity node count");
      int64_t nu = 0;
      if (npairs > 0) {
        size_t tb = 0;
        int64_t* d_nu = reinterpret_cast<int64_t*>(c->ca_count.as<unsigned long long>() + 1);
        CK(nsg::sort_unique_u64(A.pairs, c->ca_alt.as<unsigned long long>(), (int64_t)npairs, d_nu, nullptr, &tb,
                                c->stream));
        CK(c->temp.ensure(tb));
        tb = c->temp.cap;
        c->launches += 2;
        CK(nsg::sort_unique_u64(A.pairs, c->ca_alt.as<unsigned long long>(), (int64_t)npairs, d_nu, c->temp.p, &tb,
                                c->stream));
        CK(cudaMemcpyAsync(&nu, d_nu, sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
      }
      std::vector<unsigned long long> keys(nu);
      if (nu) {
        CK(cudaMemcpyAsync(keys.data(), c->ca_pairs.p, nu * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                           c->stream));
        CK(cudaStreamSynchronize(c->stream));
      }
      c->cav_atom_list.resize(nu);
      for (int64_t q = 0; q < nu; q++) {
        const int64_t cav = (int64_t)(keys[q] >> 32);
        if (cav < 0 || cav >= c->ncav) return fail(NSG_ERR_STATE, "cavity index out of range");
        c->cav_atom_list[q] = (int32_t)(uint32_t)(keys[q] & 0xffffffffu) - 1;
        c->cav_atom_off[cav + 1]++;
      }
      for (int q = 0; q < c->ncav; q++) c->cav_atom_off[q + 1] += c->cav_atom_off[q];
    }
    c->have_cav_atoms = true;
  }
  if (n_total) *n_total = (int64_t)c->cav_atom_list.size();
  if (atoms) {
    memcpy(offsets, c->cav_atom_off.data(), c->cav_atom_off.size() * sizeof(int32_t));
    if (!c->cav_atom_list.empty())
      memcpy(atoms, c->cav_atom_list.data(), c->cav_atom_list.size() * sizeof(int32_t));
  }
  return NSG_OK;
}

// Epsilon map in the reference's layout ((k*ny + j)*nx + i)*3 + axis (DelPhiShared::epsmap), after
// cavity filling when nsg_cavities ran on this ray cast.
int nsg_download_epsmap(nsg_ctx* c, int32_t* dst) {
  if (!c || !dst) return NSG_ERR_ARG;
  if (!c->have_eps) return fail(NSG_ERR_STATE, "no epsilon maps: ray cast with NSG_RAYCAST_EPSMAP");
  CK(cudaSetDevice(c->device));
  const NsGrid& g = c->grid;
  CK(cudaMemcpyAsync(dst, c->epsmap.p, (size_t)g.nx * g.ny * g.nz * 3 * sizeof(int32_t), cudaMemcpyDeviceToHost,
                     c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return NSG_OK;
}

// ideb map (DelPhiShared::idebmap), 1 byte per node, (k*ny + j)*nx + i.
int nsg_download_idebmap(nsg_ctx* c, uint8_t* dst) {
  if (!c || !dst) return NSG_ERR_ARG;
  if (!c->have_eps) return fail(NSG_ERR_STATE, "no ideb map: ray cast with NSG_RAYCAST_EPSMAP");
  CK(cudaSetDevice(c->device));
  const NsGrid& g = c->grid;
  const size_t nn = (size_t)g.nx * g.ny * g.nz;
  if (!c->ideb_ready) {
    CK(c->ideb.ensure(nn));
    nsg::RunArgs A = run_args(c);
    LAUNCH(nsg::ideb_write(A, c->eps_filled ? c->cc_fill_of.as<uint8_t>() : nullptr, c->ideb.as<uint8_t>(),
                           c->stream));
  }
  CK(cudaMemcpyAsync(dst, c->ideb.p, nn, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return NSG_OK;
}

// Auxiliary grid of the SES projection (ConnollySurface::buildAuxiliaryGrid,
// src/ConnollySurface.cpp:3681-3726): the smallest odd multiplier gridMul >= 1 that brings the
// node count igrid (an odd count of gridMul-wide cells covering nx nodes) to at most max_dim,
// centred on the grid's barycentre.
nsg::AuxGrid aux_grid_of(const NsGrid& g, int64_t max_dim) {
  int64_t igrid = g.nx, mul = 1;
  while (igrid > max_dim) {
    mul += 2;
    int64_t digrid = g.nx;
    while (true) {
      const int64_t fixed_point = (digrid + (mul - 1)) / mul;
      igrid = fixed_point * mul;
      if (igrid % 2 == 0) {
        digrid = igrid + 1;
      } else {
        igrid = fixed_point;
        break;
      }
    }
  }
  nsg::AuxGrid a;
  a.n = igrid;
  a.scale = g.scale / (double)mul;
  const double side = (double)mul / g.scale;
  a.mn[0] = g.baricenter[0] - (igrid - 1) * 0.5 * side;
  a.mn[1] = g.baricenter[1] - (igrid - 1) * 0.5 * side;
  a.mn[2] = g.baricenter[2] - (igrid - 1) * 0.5 * side;
  return a;
}

// Boundary grid points of the epsilon map (src/Surface.cpp:1488-1546) and, with project != 0,
// the projection of the external ones onto the SES (Surface::projector with
// ConnollySurface::getProjection); aux_max_dim is Max_ses_patches_auxiliary_grid_size (50).
int nsg_bgp(nsg_ctx* c, int project, int32_t aux_max_dim, int64_t* n_bgp, int64_t* n_external) {
  if (!c) return NSG_ERR_ARG;
  if (!c->have_eps) return fail(NSG_ERR_STATE, "boundary grid points need the epsilon maps (NSG_RAYCAST_EPSMAP)");
  if (project && (c->kind_mask & ~nsg::kSesKinds) && c->kind_mask != (1 << NS_MESH_TRI))
    return fail(NSG_ERR_STATE, "boundary grid point projection is provided for SES and mesh patch sets");
  if (project && aux_max_dim < 1) return fail(NSG_ERR_ARG, "auxiliary grid size must be positive");
  CK(cudaSetDevice(c->device));
  const NsGrid& g = c->grid;
  const int32_t* eps = c->epsmap.as<int32_t>();
  CK(c->bgp_n.ensure(2 * sizeof(int64_t)));
  int32_t* cnt_d = c->bgp_n.as<int32_t>();
  size_t tb = 0;
  CK(nsg::bgp_select(eps, g.nx, g.ny, g.nz, nullptr, cnt_d, nullptr, &tb, c->stream));
  CK(c->temp.ensure(tb));
  tb = c->temp.cap;
  c->launches++;
  CK(nsg::bgp_select(eps, g.nx, g.ny, g.nz, nullptr, cnt_d, c->temp.p, &tb, c->stream));
  int32_t n = 0;
  CK(cudaMemcpyAsync(&n, cnt_d, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  const size_t ncap = std::max<int32_t>(n, 1);
  CK(c->bgp_node.ensure(ncap * sizeof(int32_t)));
  CK(c->bgp_ibgp.ensure(3 * ncap * sizeof(int32_t)));
  CK(c->bgp_type.ensure(ncap * sizeof(int32_t)));
  tb = 0;
  CK(nsg::bgp_select(eps, g.nx, g.ny, g.nz, c->bgp_node.as<int32_t>(), cnt_d, nullptr, &tb, c->stream));
  CK(c->temp.ensure(tb));
  tb = c->temp.cap;
  c->launches++;
  CK(nsg::bgp_select(eps, g.nx, g.ny, g.nz, c->bgp_node.as<int32_t>(), cnt_d, c->temp.p, &tb, c->stream));
  LAUNCH(nsg::bgp_expand(eps, g.nx, g.ny, g.nz, c->bgp_node.as<int32_t>(), n, c->bgp_ibgp.as<int32_t>(),
                         c->bgp_type.as<int32_t>(), c->stream));
  int64_t n_ext = 0;
  if (n > 0) {
    int64_t* ext_d = c->bgp_n.as<int64_t>() + 1;
    tb = 0;
    CK(nsg::sum_i32(c->bgp_type.as<int32_t>(), n, ext_d, nullptr, &tb, c->stream));
    CK(c->temp.ensure(tb));
    tb = c->temp.cap;
    c->launches++;
    CK(nsg::sum_i32(c->bgp_type.as<int32_t>(), n, ext_d, c->temp.p, &tb, c->stream));
    CK(cudaMemcpyAsync(&n_ext, ext_d, sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream));
  }
  CK(cudaStreamSynchronize(c->stream));
  c->n_bgp = n;
  c->n_bgp_ext = n_ext;
  c->have_bgp = true;
  c->bgp_projected = false;
  if (project && n > 0) {
    const nsg::AuxGrid a = aux_grid_of(g, aux_max_dim);
    const int64_t ncell = a.n * a.n * a.n;
    CK(c->aux_cnt.ensure(ncell * sizeof(int32_t)));
    CK(c->aux_off.ensure((ncell + 1) * sizeof(int64_t)));
    CK(cudaMemsetAsync(c->aux_cnt.p, 0, ncell * sizeof(int32_t), c->stream));
    nsg::PatchDev P = patch_dev(c);
    LAUNCH(nsg::aux_count(P, a, c->aux_cnt.as<int32_t>(), c->stream));
    int64_t total = 0;
    int rc = scan_counts(c, c->aux_cnt.as<int32_t>(), ncell, c->aux_off.as<int64_t>(), &total);
    if (rc) return rc;
    CK(c->aux_list.ensure(std::max<int64_t>(total, 1) * sizeof(int32_t)));
    CK(cudaMemsetAsync(c->aux_cnt.p, 0, ncell * sizeof(int32_t), c->stream));
    LAUNCH(nsg::aux_fill(P, a, c->aux_off.as<int64_t>(), c->aux_cnt.as<int32_t>(), c->aux_list.as<int32_t>(),
                         c->stream));
    CK(c->bgp_pos.ensure(3 * ncap * sizeof(double)));
    CK(c->bgp_nor.ensure(3 * ncap * sizeof(double)));
    CK(c->bgp_flag.ensure(ncap * sizeof(int32_t)));
    LAUNCH(nsg::bgp_project(P, a, c->aux_off.as<int64_t>(), c->aux_list.as<int32_t>(), grid_dev(g), c->bgp_ibgp.as<int32_t>(),
                            c->bgp_type.as<int32_t>(), n, c->bgp_pos.as<double>(), c->bgp_nor.as<double>(),
                            c->bgp_flag.as<int32_t>(), c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->bgp_projected = true;
  }
  if (n_bgp) *n_bgp = n;
  if (n_external) *n_external = n_ext;
  return NSG_OK;
}

// The boundary grid points of the last nsg_bgp: ibgp (3 int32 per point), type (EXTERNAL 1 /
// INTERNAL 0), and when projected scspos / scsnor (3 doubles per point) and the projection flag
// (0 projected, 1 no feasible projection, 2 empty auxiliary cell, 3 internal point); any pointer
// may be NULL.
int nsg_download_bgp(nsg_ctx* c, int32_t* ibgp, int32_t* type, double* scspos, double* scsnor, int32_t* flag) {
  if (!c) return NSG_ERR_ARG;
  if (!c->have_bgp) return fail(NSG_ERR_STATE, "no boundary grid points: call nsg_bgp first");
  if ((scspos || scsnor || flag) && !c->bgp_projected) return fail(NSG_ERR_STATE, "boundary grid points not projected");
  CK(cudaSetDevice(c->device));
  const size_t n = (size_t)c->n_bgp;
  if (n) {
    if (ibgp) CK(cudaMemcpyAsync(ibgp, c->bgp_ibgp.p, 3 * n * sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
    if (type) CK(cudaMemcpyAsync(type, c->bgp_type.p, n * sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
    if (scspos) CK(cudaMemcpyAsync(scspos, c->bgp_pos.p, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (scsnor) CK(cudaMemcpyAsync(scsnor, c->bgp_nor.p, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (flag) CK(cudaMemcpyAsync(flag, c->bgp_flag.p, n * sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
  }
  CK(cudaStreamSynchronize(c->stream));
  return NSG_OK;
}

// Per-ray sorted hit parameters of one ray set (raycast with flag 16): counts are indexed by
// n*nb + m of the set; hits are gathered in that order into dst.
int nsg_download_hits(nsg_ctx* c, int set, int32_t* counts, double* dst, int64_t dst_cap) {
  if (!c || set < 0 || set >= nsg::kRaySets || !(c->flags & 16)) return NSG_ERR_STATE;
  int64_t nr = c->rays_tot[set];
  std::vector<int64_t> off(nr);
  std::vector<int32_t> cnt(nr);
  CK(cudaMemcpyAsync(off.data(), c->ray_hit_off[set].p, nr * sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(cnt.data(), c->ray_hit_cnt[set].p, nr * sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  int64_t total = 0;
  for (int64_t r = 0; r < nr; r++) total += cnt[r];
  if (counts) memcpy(counts, cnt.data(), nr * sizeof(int32_t));
  if (!dst) return (int)std::min<int64_t>(total, INT32_MAX);
  if (total > dst_cap) return NSG_ERR_CAPACITY;
  std::vector<double> all(c->hit_cap);
  CK(cudaMemcpyAsync(all.data(), c->hits.p, c->hit_cap * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  int64_t o = 0;
  for (int64_t r = 0; r < nr; r++)
    for (int32_t q = 0; q < cnt[r]; q++) dst[o++] = all[off[r] + q];
  return NSG_OK;
}

// Records user event `slot` (0..7) on the context's stream.
int nsg_event_record(nsg_ctx* c, int slot) {
  if (!c || slot < 0 || slot >= 8) return NSG_ERR_ARG;
  CK(cudaSetDevice(c->device));
  if (!c->user_ev[slot]) CK(cudaEventCreate(&c->user_ev[slot]));
  CK(cudaEventRecord(c->user_ev[slot], c->stream));
  return NSG_OK;
}

// Milliseconds between two recorded user events (waits for the second one).
int nsg_event_elapsed(nsg_ctx* c, int slot_a, int slot_b, double* ms) {
  if (!c || !ms || slot_a < 0 || slot_a >= 8 || slot_b < 0 || slot_b >= 8) return NSG_ERR_ARG;
  if (!c->user_ev[slot_a] || !c->user_ev[slot_b]) return NSG_ERR_STATE;
  CK(cudaEventSynchronize(c->user_ev[slot_b]));
  float f = 0;
  CK(cudaEventElapsedTime(&f, c->user_ev[slot_a], c->user_ev[slot_b]));
  *ms = f;
  return NSG_OK;
}

// Enables (1) / disables (0) per-stage kernel timing; enabling resets the accumulated times.
int nsg_profile(nsg_ctx* c, int enable) {
  if (!c) return NSG_ERR_ARG;
  c->profile = enable != 0;
  if (c->profile)
    for (int i = 0; i < 12; i++) { c->stage_ms[i] = 0; c->stage_calls[i] = 0; }
  return NSG_OK;
}

// Accumulated per-stage milliseconds and call counts: bin, trace, overflow, cavity, vertex, mc, and
// within the trace the candidate, intersection and fill kernels.
int nsg_stage_times(nsg_ctx* c, double* ms, int64_t* calls, int n) {
  if (!c) return NSG_ERR_ARG;
  for (int i = 0; i < n && i < 12; i++) {
    if (ms) ms[i] = c->stage_ms[i];
    if (calls) calls[i] = c->stage_calls[i];
  }
  return NSG_OK;
}

// Event counters of the last profiled ray cast: candidates, torus candidates, mixed-precision
// fallbacks (near-tangent sphere, quartic isolation, root polish), feasibility re-evaluations.
int nsg_trace_counters(nsg_ctx* c, int64_t* out, int n) {
  if (!c || !out) return NSG_ERR_ARG;
  for (int i = 0; i < n && i < 8; i++) out[i] = (int64_t)c->counter_host[i];
  return NSG_OK;
}

// Number of this library's kernels launched since the context was created.
int64_t nsg_launch_count(nsg_ctx* c) { return c ? c->launches : -1; }

void* nsg_get_stream(nsg_ctx* c) { return c ? (void*)c->stream : nullptr; }

int nsg_stats(nsg_ctx* c, int64_t* out, int n) {
  if (!c || !out) return NSG_ERR_ARG;
  int64_t v[8] = {c->np, c->n_vert, c->n_analytic, c->n_tri, c->n_active, c->ncav, c->last_overflow_rays, c->pair_cap};
  for (int i = 0; i < n && i < 8; i++) out[i] = v[i];
  return NSG_OK;
}

double nsg_volume(nsg_ctx* c) { return c ? c->volume : 0.0; }
double nsg_area(nsg_ctx* c) { return c ? c->area : 0.0; }

}  // extern "C"
