"""ORACLE — test infrastructure only.  Python access to the CPU restatement in ns_oracle.cpp.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this module, as the
checker; the product library never imports it.
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "libnsoracle.so"

STATUS = 1
ACCURATE_TRIANGULATION = 2
CAVITIES = 4
TRIANGULATE = 8
NORMALS = 16
EPSMAP = 32
BGP = 64

_lib = None


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = ctypes.CDLL(str(LIB))
        P = ctypes.c_void_p
        L.nso_run.restype = P
        L.nso_run.argtypes = [P, ctypes.c_int64, P, P, P, P, ctypes.c_double, ctypes.c_int, ctypes.c_double,
                              ctypes.c_int]
        L.nso_run_ex.restype = P
        L.nso_run_ex.argtypes = [P, ctypes.c_int64, P, P, P, P, ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                 ctypes.c_int, ctypes.c_int]
        L.nso_scalar.restype = ctypes.c_double
        L.nso_scalar.argtypes = [P, ctypes.c_char_p]
        L.nso_size.restype = ctypes.c_int64
        L.nso_size.argtypes = [P, ctypes.c_char_p]
        L.nso_copy.restype = ctypes.c_int
        L.nso_copy.argtypes = [P, ctypes.c_char_p, P]
        L.nso_free.argtypes = [P]
        L.nso_ray_sphere.restype = ctypes.c_int
        L.nso_ray_sphere.argtypes = [P, P, P, ctypes.c_double, P]
        L.nso_quartic.restype = ctypes.c_int
        L.nso_quartic.argtypes = [ctypes.c_double] * 4 + [P]
        L.nso_real_cubic.restype = ctypes.c_double
        L.nso_real_cubic.argtypes = [ctypes.c_double] * 3
        L.nso_run_slab.restype = P
        L.nso_run_slab.argtypes = [P, ctypes.c_int64, P, P, P, P, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_double, ctypes.c_double]
        L.nso_blobby.restype = P
        L.nso_blobby.argtypes = [P, P, ctypes.c_int64, ctypes.c_double, ctypes.c_int]
        L.nso_mesh_size.restype = ctypes.c_int64
        L.nso_mesh_size.argtypes = [P, ctypes.c_char_p]
        L.nso_mesh_copy.restype = ctypes.c_int
        L.nso_mesh_copy.argtypes = [P, ctypes.c_char_p, P]
        L.nso_free_mesh.argtypes = [P]
        L.nso_shape_filter.restype = ctypes.c_int64
        L.nso_shape_filter.argtypes = [P, P, ctypes.c_int, P, P, ctypes.c_int64, P, P, ctypes.c_double, ctypes.c_int]
        L.nso_pocket_difference.restype = ctypes.c_int
        L.nso_pocket_difference.argtypes = [P, P, P, P, ctypes.c_int64, ctypes.c_double, P, P, ctypes.c_int]
        L.nso_mesh_project.restype = ctypes.c_int
        L.nso_mesh_project.argtypes = [P, P, P, P, P]
        L.nso_ray_torus.restype = ctypes.c_int
        L.nso_ray_torus.argtypes = [P, P, P, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int, P, P, P]
        _lib = L
    return _lib


class OracleResult:
    """Products of one oracle run (arrays copied out, native handle freed)."""

    def __init__(self, handle, grid, flags: int = 0):
        L = lib()
        self.grid = grid
        self.flags = flags

        def arr(name, dtype):
            n = L.nso_size(handle, name.encode())
            a = np.zeros(max(n, 0), dtype)
            if n > 0:
                L.nso_copy(handle, name.encode(), a.ctypes.data)
            return a

        self.volume = L.nso_scalar(handle, b"volume")
        self.area = L.nso_scalar(handle, b"area")
        self.ncav = int(L.nso_scalar(handle, b"ncav"))
        self.n_hits = int(L.nso_scalar(handle, b"n_hits"))
        self.status = arr("status", np.int32)
        if len(self.status):
            self.status = self.status.reshape(grid.nz, grid.ny, grid.nx)
        self.bits = arr("bits", np.uint32)
        self.vertices = arr("verts", np.float64).reshape(-1, 3)
        self.vertex_edges = arr("vkeys", np.int32).reshape(-1, 4)
        self.triangles = arr("tris", np.int32).reshape(-1, 3)
        self.cav_size = arr("cav_size", np.float64)
        n = L.nso_size(handle, b"cav_size")
        fl = np.zeros(max(n, 0), np.int32)
        if n > 0:
            L.nso_copy(handle, b"cav_filled", fl.ctypes.data)
        self.cav_filled = fl
        self.normals = arr("normals", np.float64).reshape(-1, 3)
        self.pix_off = arr("pix_off", np.int64)
        self.pix_t = arr("pix_t", np.float64)
        self.pix_pid = arr("pix_pid", np.int32)
        # epsilon / ideb maps and boundary grid points
        self.epsmap = arr("eps", np.int32)
        if len(self.epsmap):
            self.epsmap = self.epsmap.reshape(grid.nz, grid.ny, grid.nx, 3)
        ideb = arr("ideb", np.uint8)
        self.idebmap = ideb.reshape(grid.nz, grid.ny, grid.nx).astype(bool) if len(ideb) else ideb
        nb = max(L.nso_size(handle, b"bgp_type"), 0)
        self.nbgp = nb

        def fixed(name, dtype, k):
            a = np.zeros(nb * k, dtype)
            if nb:
                L.nso_copy(handle, name.encode(), a.ctypes.data)
            return a.reshape(nb, k) if k > 1 else a

        self.ibgp = fixed("ibgp", np.int32, 3)
        self.bgp_type = fixed("bgp_type", np.int32, 1)
        if flags & BGP:
            self.scspos = fixed("scspos", np.float64, 3)
            self.scsnor = fixed("scsnor", np.float64, 3)
            self.bgp_flag = fixed("bgp_flag", np.int32, 1)


def run(grid, patches, flags: int = STATUS | ACCURATE_TRIANGULATION | CAVITIES | TRIANGULATE, cav_vol: float = 0.0,
        threads: int = 1, aux_grid_dim: int = 50) -> OracleResult:
    """Runs the CPU restatement on a grid (NsGrid ctypes struct) and a PatchSet; aux_grid_dim is
    Max_ses_patches_auxiliary_grid_size of the boundary-point projection."""
    L = lib()
    p = patches
    h = L.nso_run_ex(ctypes.byref(grid), p.n, p.f64.ctypes.data, p.i32.ctypes.data, p.pool.ctypes.data,
                     p.pool_flag.ctypes.data, p.probe, flags, cav_vol, threads, aux_grid_dim)
    try:
        return OracleResult(h, grid, flags)
    finally:
        L.nso_free(h)


def ray_hits(res: OracleResult, ray_set: int) -> tuple[np.ndarray, np.ndarray]:
    """Per-ray sorted hits of one ray set, laid out like the GPU dump: (counts[na, nb], values)."""
    g = res.grid
    nmax = max(g.nx, g.ny, g.nz)
    nb, na = ((g.ny, g.nz), (g.ny, g.nz), (g.nx, g.ny), (g.nx, g.nz), (g.nx, g.ny), (g.nx, g.nz))[ray_set]
    npan = (len(res.pix_off) - 1) // (nmax * nmax)
    # oracle panel order: the node-ray panels (1, or 3 with the epsilon maps), then the three
    # accurate-triangulation panels
    node_panels = 3 if res.flags & EPSMAP else (1 if res.flags & STATUS else 0)
    panel_idx = {0: 0, 4: 1, 5: 2}[ray_set] if ray_set in (0, 4, 5) else node_panels + ray_set - 1
    assert panel_idx < npan, "ray set not cast by this oracle run"
    n_idx = np.arange(na)[:, None]
    m_idx = np.arange(nb)[None, :]
    pid = (n_idx * nmax + m_idx) * npan + panel_idx
    off = res.pix_off[pid]
    cnt = res.pix_off[pid + 1] - off
    vals = np.concatenate([res.pix_t[o:o + c] for o, c in zip(off.ravel(), cnt.ravel())]) if cnt.sum() else np.zeros(0)
    return cnt.astype(np.int32), vals


def time_slab(grid, patches, threads: int, slab_lo: float, slab_hi: float,
              flags: int = STATUS | ACCURATE_TRIANGULATION) -> tuple[float, int]:
    """Wall time (s) and number of rays of the oracle's ray casting of a slab of every ray set."""
    import time
    L = lib()
    p = patches
    t0 = time.perf_counter()
    h = L.nso_run_slab(ctypes.byref(grid), p.n, p.f64.ctypes.data, p.i32.ctypes.data, p.pool.ctypes.data,
                       p.pool_flag.ctypes.data, p.probe, flags, threads, slab_lo, slab_hi)
    dt = time.perf_counter() - t0
    rays = int(L.nso_scalar(h, b"rays_cast"))
    L.nso_free(h)
    return dt, rays


def blobby_mesh(grid, atoms: np.ndarray, blobbyness: float = -2.5, quantize: bool = True):
    """The oracle's blobby mesh (field, marching cubes, smoothing, OFF round trip): vertices (n, 3),
    their grid edges (n, 4) and triangles (m, 3)."""
    L = lib()
    atoms = np.ascontiguousarray(atoms, np.float64)
    h = L.nso_blobby(ctypes.byref(grid), atoms.ctypes.data, len(atoms), blobbyness, int(quantize))
    try:
        out = []
        for name, dt, w in (("verts", np.float64, 3), ("vkeys", np.int32, 4), ("tris", np.int32, 3)):
            n = L.nso_mesh_size(h, name.encode())
            a = np.zeros(max(n, 0), dt)
            if n > 0:
                L.nso_mesh_copy(h, name.encode(), a.ctypes.data)
            out.append(a.reshape(-1, w))
        return tuple(out)
    finally:
        L.nso_free_mesh(h)


class TrianglePatches:
    """A mesh as the oracle's triangle patch set (kind 9): vertices, normal, box per triangle."""

    def __init__(self, verts: np.ndarray, tris: np.ndarray):
        p = verts[tris]  # (m, 3, 3)
        self.n = len(tris)
        f = np.zeros((self.n, 20))
        f[:, 0:9] = p.reshape(-1, 9)
        f[:, 9:12] = np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0])
        f[:, 14:17] = p.min(axis=1)
        f[:, 17:20] = p.max(axis=1)
        self.f64 = np.ascontiguousarray(f)
        self.i32 = np.zeros((self.n, 4), np.int32)
        self.i32[:, 0] = 9
        self.pool = np.zeros((1, 4))
        self.pool_flag = np.zeros(1, np.int8)
        self.probe = 0.0


OP_NAMES = ("torus_cand", "torus_no_sphere", "quartic_none", "quartic_m0", "quartic_2", "quartic_4", "quartic_recip",
            "cubic_small_c", "cubic_ratio_sqrt", "cubic_ratio_eps", "cubic_cbrt", "cubic_acos", "sphere_cand",
            "sphere_miss", "root_test", "root_in", "feas_test", "plane_test", "clip_test", "sir_test")

# Operation model of the ray-patch tests (adds, subtractions and multiplications of doubles counted
# as one flop each, so a fused multiply-add is two; square roots, divisions, cube roots, arccos and
# cos counted apart), per executed block of the restated code:
#   ray-sphere (raySphere on an axis ray): 15 flops, +2 flops, 1 sqrt and 2 divisions on a hit
#   torus: the entry point 2, the coefficients 53, the quartic head 38, then (with roots) the
#     resolvent's arguments 5 and head 19 + 1 division; the resolvent branch: cube roots 7 + 1 sqrt
#     + 2 cbrt; arccos 7 + 2 sqrt + 1 division + acos + cos; the two approximations 9 + 1 sqrt and
#     10 + 1 division; the small-coefficient one 3 + 2 divisions; the quartic tail 16 + 1 division
#     + 3 sqrt for 2 roots, 25 + 1 division + 4 sqrt for 4; per non-negative root 10, per root in
#     the clipping sphere 1 + 1 division
#   feasibility: 2 per tested point, a plane 6, a clipping sphere 9, the spindle sphere 9
OP_MODEL = {
    "sphere_cand": {"flops": 15}, "sphere_hit": {"flops": 2, "sqrt": 1, "div": 2},
    "torus_entry": {"flops": 2 + 53 + 38},
    "cubic_head": {"flops": 5 + 19, "div": 1},
    "cubic_cbrt": {"flops": 7, "sqrt": 1, "cbrt": 2},
    "cubic_acos": {"flops": 7, "sqrt": 2, "div": 1, "acos": 1, "cos": 1},
    "cubic_ratio_sqrt": {"flops": 9, "sqrt": 1},
    "cubic_ratio_eps": {"flops": 10, "div": 1},
    "cubic_small_c": {"flops": 3, "div": 2},
    "quartic_2": {"flops": 16, "div": 1, "sqrt": 3},
    "quartic_4": {"flops": 25, "div": 1, "sqrt": 4},
    "root_test": {"flops": 10}, "root_in": {"flops": 1, "div": 1},
    "feas_test": {"flops": 2}, "plane_test": {"flops": 6}, "clip_test": {"flops": 9}, "sir_test": {"flops": 9},
}


def op_counts(handle) -> dict:
    """The branch counters of the last oracle run (a native handle of nso_run*)."""
    L = lib()
    return {n: L.nso_scalar(handle, ("op_" + n).encode()) for n in OP_NAMES}


def op_model(c: dict) -> dict:
    """Operations of a run's ray-patch tests from its branch counters (OP_MODEL)."""
    blocks = {
        "sphere_cand": c["sphere_cand"] + c["torus_cand"],
        "sphere_hit": c["sphere_cand"] - c["sphere_miss"] + c["torus_cand"] - c["torus_no_sphere"],
        "torus_entry": c["torus_cand"] - c["torus_no_sphere"],
        "cubic_head": c["quartic_2"] + c["quartic_4"],
        "cubic_cbrt": c["cubic_cbrt"], "cubic_acos": c["cubic_acos"], "cubic_ratio_sqrt": c["cubic_ratio_sqrt"],
        "cubic_ratio_eps": c["cubic_ratio_eps"], "cubic_small_c": c["cubic_small_c"],
        "quartic_2": c["quartic_2"], "quartic_4": c["quartic_4"],
        "root_test": c["root_test"], "root_in": c["root_in"], "feas_test": c["feas_test"],
        "plane_test": c["plane_test"], "clip_test": c["clip_test"], "sir_test": c["sir_test"],
    }
    out = {}
    for b, n in blocks.items():
        for k, v in OP_MODEL[b].items():
            out[k] = out.get(k, 0.0) + n * v
    return out


# The 27 cells around a cell in the reference's order (shift_map, src/tools.h:35-64).
SHIFT27 = ((0, 0, 0), (0, 0, -1), (0, 0, 1), (0, 1, 0), (0, 1, -1), (0, 1, 1), (0, -1, 0), (0, -1, -1), (0, -1, 1),
           (1, 0, 0), (1, 0, -1), (1, 0, 1), (1, 1, 0), (1, 1, -1), (1, 1, 1), (1, -1, 0), (1, -1, -1), (1, -1, 1),
           (-1, 0, 0), (-1, 0, -1), (-1, 0, 1), (-1, 1, 0), (-1, 1, -1), (-1, 1, 1), (-1, -1, 0), (-1, -1, -1),
           (-1, -1, 1))


def atom_grid(grid, atoms: np.ndarray):
    """The reference's atom grid (Surface::buildAtomsMap, src/Surface.cpp:1695-1749): cell side
    2 r_max, halved or doubled until 1.3 rmaxdim spans 1..100 cells, centred on the grid's
    barycentre; the atoms of each cell in ascending index order.  Returns (ggrid, gmin, gscale,
    cells: dict flat cell index -> atom indices)."""
    rmax = 0.0
    for r in atoms[:, 3]:
        rmax = max(float(r), rmax)
    gscale = 0.5 / rmax
    while True:
        ggrid = int(np.floor(gscale * 1.3 * grid.rmaxdim))
        if ggrid <= 100:
            if ggrid <= 0:
                gscale *= 2.0
            else:
                break
        else:
            gscale *= 0.5
    gside = 1. / gscale
    gmin = np.array([grid.baricenter[d] - (ggrid - 1) * 0.5 * gside for d in range(3)])
    idx = np.floor((atoms[:, :3] - gmin) * gscale + 0.5).astype(np.int64)
    flat = (idx[:, 2] * ggrid + idx[:, 1]) * ggrid + idx[:, 0]
    cells: dict[int, list[int]] = {}
    for a, f in enumerate(flat.tolist()):
        cells.setdefault(f, []).append(a)
    return ggrid, gmin, gscale, cells


def shape_filter(grid, status: np.ndarray, ncav: int, filled, bits=None, eps=None, ideb=None, probe: float = 1.4,
                 mod_status: bool = False):
    """Keep_Water_Shaped_Cavities on copies of the maps after cavity detection
    (nso_shape_filter in ns_oracle.cpp).  Returns (status, filled, bits, eps, ideb, removed)."""
    L = lib()
    st = np.ascontiguousarray(status, np.int32).copy()
    fl = np.ascontiguousarray(filled, np.int32).copy()
    b = None if bits is None else np.ascontiguousarray(bits, np.uint32).copy()
    e = None if eps is None else np.ascontiguousarray(eps, np.int32).copy()
    d = None if ideb is None else np.ascontiguousarray(ideb, np.uint8).copy()

    def ptr(a):
        return None if a is None else a.ctypes.data
    n = L.nso_shape_filter(ctypes.byref(grid), st.ctypes.data, int(ncav), ptr(fl), ptr(b), 0 if b is None else b.size,
                           ptr(e), ptr(d), float(probe), int(bool(mod_status)))
    return st, fl, b, e, None if d is None else d.astype(bool), int(n)


def mesh_project(point, tri):
    """MeshSurface::point2triangle of one point onto one triangle (nso_mesh_project):
    (inside the triangle, projection, distance, normal)."""
    L = lib()
    p = np.ascontiguousarray(point, np.float64)
    t = np.ascontiguousarray(tri, np.float64).reshape(9)
    proj = np.zeros(3)
    nrm = np.zeros(3)
    dist = ctypes.c_double()
    ins = L.nso_mesh_project(p.ctypes.data, t.ctypes.data, proj.ctypes.data, ctypes.byref(dist), nrm.ctypes.data)
    return bool(ins), proj, dist.value, nrm


def pocket_difference(grid, status_fat: np.ndarray, status_small: np.ndarray, bits=None, fill_volume: float = 0.0):
    """Pocket mode's difference step on copies of two status maps after their casts
    (nso_pocket_difference in ns_oracle.cpp).  Returns (status, bits, sizes, filled)."""
    L = lib()
    st = np.ascontiguousarray(status_fat, np.int32).copy()
    s2 = np.ascontiguousarray(status_small, np.int32)
    b = None if bits is None else np.ascontiguousarray(bits, np.uint32).copy()
    cap = st.size
    sizes = np.zeros(cap)
    filled = np.zeros(cap, np.int32)
    n = L.nso_pocket_difference(ctypes.byref(grid), st.ctypes.data, s2.ctypes.data, None if b is None else b.ctypes.data,
                                0 if b is None else b.size, float(fill_volume), sizes.ctypes.data, filled.ctypes.data,
                                cap)
    assert n >= 0
    return st, b, sizes[:n].copy(), filled[:n].copy()


def cavity_atoms(grid, status: np.ndarray, ncav: int, atoms: np.ndarray, label: np.ndarray | None = None) -> list[list[int]]:
    """cav2atoms as Surface::getCavitiesAtomsWithBilevelStatusMap fills it
    (src/Surface.cpp:2249-2346): for every node of cavity c (status 4 + c) with a 6-neighbour of
    another status (TEMPORARY_OUT = 2 outside the grid), the atom of least |a - x|^2 - r^2 over the
    27 atom-grid cells around the node, scanned in shift_map order and ascending atom order with a
    strict comparison (the first of equal ones wins), -1 when those cells are empty; per cavity the
    distinct atoms ascending (std::set order).  After a shape filter the cavities' points are
    those of ``label`` (the labels before it) and the comparisons read the filtered ``status``.
    Vectorised over the boundary nodes: one pass per
    (cell shift, slot within the cell) keeps the scan order of the reference's loops."""
    nz, ny, nx = status.shape
    pad = np.pad(status, 1, constant_values=2)
    s = pad[1:-1, 1:-1, 1:-1]
    same = ((pad[1:-1, 1:-1, 2:] == s) & (pad[1:-1, 1:-1, :-2] == s) & (pad[1:-1, 2:, 1:-1] == s) &
            (pad[1:-1, :-2, 1:-1] == s) & (pad[2:, 1:-1, 1:-1] == s) & (pad[:-2, 1:-1, 1:-1] == s))
    lab = status if label is None else np.asarray(label).reshape(status.shape)
    k, j, i = np.nonzero((lab >= 4) & ~same)
    out: list[set] = [set() for _ in range(ncav)]
    if len(i) == 0:
        return [sorted(x) for x in out]
    ggrid, gmin, gscale, cells = atom_grid(grid, atoms)
    p = np.stack([grid.xmin + i * grid.side, grid.ymin + j * grid.side, grid.zmin + k * grid.side], 1)
    c = np.floor((p - gmin) * gscale + 0.5).astype(np.int64)
    maxper = max(len(v) for v in cells.values())
    table = np.full((ggrid ** 3, maxper), -1, np.int64)
    for f, lst in cells.items():
        table[f, :len(lst)] = lst
    best = np.full(len(i), np.inf)
    first = np.full(len(i), -1, np.int64)
    for sx, sy, sz in SHIFT27:
        cx, cy, cz = c[:, 0] + sx, c[:, 1] + sy, c[:, 2] + sz
        ok = (cx >= 0) & (cy >= 0) & (cz >= 0) & (cx < ggrid) & (cy < ggrid) & (cz < ggrid)
        f = np.where(ok, (cz * ggrid + cy) * ggrid + cx, 0)
        for slot in range(maxper):
            a = np.where(ok, table[f, slot], -1)
            has = a >= 0
            at = atoms[np.maximum(a, 0)]
            d = ((at[:, 0] - p[:, 0]) * (at[:, 0] - p[:, 0]) + (at[:, 1] - p[:, 1]) * (at[:, 1] - p[:, 1]) +
                 (at[:, 2] - p[:, 2]) * (at[:, 2] - p[:, 2]))
            d = d - at[:, 3] * at[:, 3]
            better = has & (d < best)
            best = np.where(better, d, best)
            first = np.where(better, a, first)
    cav = lab[k, j, i] - 4
    for cc, a in zip(cav.tolist(), first.tolist()):
        out[cc].add(a)
    return [sorted(x) for x in out]
