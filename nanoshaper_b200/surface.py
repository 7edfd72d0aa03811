"""Host-side mirror of the reference's surface plugin interface, backed by libnsgpu.

Mirrors, with the same names and argument meanings:
  * ``ConfigFile``      -- the .prm ``key = value`` reader (src/ConfigFile/ConfigFile.{h,cpp})
  * ``DelPhiShared``    -- the grid environment: atoms, grid construction, maps
                           (src/DelphiShared.cpp:309-704, 1038-1201)
  * ``Surface``         -- ``build()``, ``getSurf()``, ``triangulateSurface()`` (src/Surface.h:835-990)
  * ``ConnollySurface`` -- the "ses" surface (src/ConnollySurface.h)
  * ``SurfaceFactory``  -- name -> surface registry keyed by the .prm ``Surface`` key
                           (src/SurfaceFactory.h:15-65)
  * ``NanoShaper``      -- the library facade (src/nanoshaper.h:294-423)

The ray casting, cavity detection and marching cubes run on the GPU through the C-ABI; the
patch construction runs in host C++ inside the same library.  Errors raise instead of calling
``exit``.
"""
from __future__ import annotations

import ctypes
from pathlib import Path
from typing import Callable

import numpy as np

from . import _native as N

DEFAULT_PERFIL = 80.0
DEFAULT_SCALE = 2.0
DEFAULT_PROBE = 1.4
RAND_DISPLACEMENT = 1e-4
SEED = 1234

STATUS_POINT_INSIDE = -1
STATUS_POINT_TEMPORARY_OUT = 2
STATUS_POINT_OUT = 3
STATUS_FIRST_CAV = 4

PRECISIONS = {"fp64": 0, "mixed": 1}

# Process-wide generator state of the atom jitter, like the reference's static SEED.
_seed = ctypes.c_int64(SEED)


def reset_seed(value: int = SEED) -> None:
    _seed.value = value


# --------------------------------------------------------------------------------------------
class ConfigFile:
    """``key = value`` configuration with ``#`` comments and an optional ``EndConfigFile`` sentry.

    A value continues on the following lines until a blank line or a line holding a delimiter.
    Unknown keys are kept and ignored by the surfaces, as in the reference.
    """

    def __init__(self, path: str | Path | None = None, text: str | None = None):
        self.contents: dict[str, str] = {}
        self.path = Path(path) if path is not None else None
        if path is not None:
            text = Path(path).read_text()
        if text:
            self._parse(text)

    def _parse(self, text: str) -> None:
        lines = text.splitlines()
        i = 0
        while i < len(lines):
            line = lines[i].split("#", 1)[0]
            i += 1
            if "EndConfigFile" in line:
                return
            if "=" not in line:
                continue
            key, value = line.split("=", 1)
            key = key.strip()
            while i < len(lines):
                nxt = lines[i].split("#", 1)[0]
                if "EndConfigFile" in nxt or "=" in nxt or not nxt.strip():
                    break
                value += "\n" + nxt
                i += 1
            self.contents[key] = value.strip()

    def keyExists(self, key: str) -> bool:
        return key in self.contents

    def add(self, key: str, value) -> None:
        self.contents[key] = str(value).lower() if isinstance(value, bool) else str(value)

    def read(self, key: str, default=None, type_: type | None = None):
        if key not in self.contents:
            if default is None:
                raise KeyError(key)
            return default
        raw = self.contents[key]
        t = type_ or (type(default) if default is not None else str)
        if t is bool:
            return raw.strip().upper() not in ("FALSE", "F", "NO", "N", "0", "NONE")
        if t is int:
            return int(float(raw.split()[0]))
        if t is float:
            return float(raw.split()[0])
        return raw


# --------------------------------------------------------------------------------------------
def read_xyzr(path: str | Path) -> np.ndarray:
    """Atoms of an xyzr file as an (N, 4) float64 array (x, y, z, radius)."""
    L = N.lib()
    n = L.nsg_read_xyzr(str(path).encode(), None, 0)
    if n < 0:
        raise N.NativeError(f"cannot read {path}: {N.ERRORS.get(n, n)}")
    out = np.zeros((n, 4), np.float64)
    n2 = L.nsg_read_xyzr(str(path).encode(), N.ptr(out), n)
    if n2 != n:
        raise N.NativeError(f"cannot read {path}")
    return out


def read_pqr(path: str | Path) -> np.ndarray:
    """Atoms of the ATOM / HETATM records of a pqr file as an (N, 4) float64 array (x, y, z,
    radius); atoms with a zero radius are skipped, as DelPhiShared::loadAtoms does."""
    L = N.lib()
    n = L.nsg_read_pqr(str(path).encode(), None, 0)
    if n < 0:
        raise N.NativeError(f"cannot read {path}: {N.ERRORS.get(n, n)}")
    out = np.zeros((n, 4), np.float64)
    n2 = L.nsg_read_pqr(str(path).encode(), N.ptr(out), n)
    if n2 != n:
        raise N.NativeError(f"cannot read {path}")
    return out


def read_atoms(path: str | Path) -> np.ndarray:
    """Atoms of a molecule file, pqr when its name contains ".pqr" and xyzr otherwise (the choice
    DelPhiShared::loadAtoms makes, src/DelphiShared.cpp:338-342)."""
    return read_pqr(path) if ".pqr" in str(path) else read_xyzr(path)


class DelPhiShared:
    """Grid environment: the atoms, the cubic grid and the maps produced on it."""

    def __init__(self, atoms: np.ndarray, scale: float = DEFAULT_SCALE, perfil: float = DEFAULT_PERFIL,
                 build_status: bool = True, build_eps_map: bool = False, grid: "N.NsGrid | None" = None):
        self.atoms = np.ascontiguousarray(np.asarray(atoms, np.float64).reshape(-1, 4)).copy()
        if len(self.atoms) == 0:
            raise ValueError("Cannot build grid with no atoms!")
        self.buildStatus = build_status
        self.buildEpsMap = build_eps_map
        self.grid = N.NsGrid()
        if grid is None:
            self.buildGrid(scale, perfil)
        else:
            # a given grid (e.g. kept fixed while the atoms move by finite differences)
            ctypes.pointer(self.grid)[0] = grid
            self._grid_fields()
        self.status: np.ndarray | None = None
        self.cavitiesSize: list[float] = []
        self.cavitiesFlag: list[bool] = []
        # atoms lining each cavity (cav2atoms), ascending atom indices, -1 for a boundary node with
        # no atom in its 27 atom-grid cells
        self.cav2atoms: list[list[int]] = []
        # epsilon and ideb maps (Build_epsilon_maps): epsmap[k, j, i, axis] is the code of the grid
        # edge from node (i, j, k) along the axis (0 outside, 5 inside), idebmap[k, j, i] is False
        # inside the surface and in filled cavities
        self.epsmap: np.ndarray | None = None
        self.idebmap: np.ndarray | None = None
        # boundary grid points (Project_boundary_grid_points): nodes (ix, iy, iz), their type
        # (1 external, 0 internal), projections onto the surface and normals
        self.nbgp = 0
        self.ibgp: np.ndarray | None = None
        self.bgp_type: np.ndarray | None = None
        self.scspos: np.ndarray | None = None
        self.scsnor: np.ndarray | None = None
        self.bgp_flag: np.ndarray | None = None

    def saveStatus(self, fname: str | Path = "") -> None:
        """``fname.status.txt`` and the cavity files (DelPhiShared::saveStatus / saveCavities)."""
        if self.status is None:
            raise RuntimeError("Cannot save null status!")
        st = np.ascontiguousarray(self.status, np.int32).reshape(-1)
        N.check(N.lib().nsg_write_status(f"{fname}.status.txt".encode(), N.ptr(st), self.nx, self.ny, self.nz),
                "saveStatus")
        self.saveCavities(Path(str(fname)).parent if str(fname) else Path("."))

    def saveCavities(self, directory: str | Path = ".") -> None:
        """``cavities.txt`` (cavity nodes) and ``cavitiesSize.txt`` (barycentre, volume, filled)."""
        if self.status is None:
            raise RuntimeError("Cannot save cavities with null status!")
        st = np.ascontiguousarray(self.status, np.int32).reshape(-1)
        sizes = np.ascontiguousarray(self.cavitiesSize, np.float64)
        flags = np.ascontiguousarray([1 if f else 0 for f in self.cavitiesFlag], np.int32)
        d = Path(directory)
        N.check(N.lib().nsg_write_cavities(str(d / "cavities.txt").encode(), str(d / "cavitiesSize.txt").encode(),
                                           N.ptr(st), ctypes.byref(self.grid), len(sizes),
                                           N.ptr(sizes) if len(sizes) else None, N.ptr(flags) if len(flags) else None),
                "saveCavities")
        # cavAtomsSerials.txt: every cavity's atoms (onlySaveNonFilled = false)
        off = np.zeros(len(self.cav2atoms) + 1, np.int32)
        off[1:] = np.cumsum([len(a) for a in self.cav2atoms]) if self.cav2atoms else []
        lst = np.ascontiguousarray([a for cav in self.cav2atoms for a in cav] or [0], np.int32)
        N.check(N.lib().nsg_write_cavity_atoms(str(d / "cavAtomsSerials.txt").encode(), len(self.cav2atoms),
                                               N.ptr(off), N.ptr(lst), None, len(self.atoms), None),
                "saveCavities (atoms)")

    def buildGrid(self, scale: float, perfil: float) -> bool:
        N.check(N.lib().nsg_grid_build(N.ptr(self.atoms), len(self.atoms), scale, perfil, ctypes.byref(self.grid)),
                "buildGrid")
        self._grid_fields()
        return True

    def _grid_fields(self) -> None:
        g = self.grid
        self.nx, self.ny, self.nz = g.nx, g.ny, g.nz
        self.scale, self.side, self.hside, self.A = g.scale, g.side, g.hside, g.A
        self.xmin, self.ymin, self.zmin = g.xmin, g.ymin, g.zmin
        self.xmax, self.ymax, self.zmax = g.xmax, g.ymax, g.zmax
        self.rmaxdim = g.rmaxdim
        self.x = g.xmin + np.arange(g.nx) * g.side
        self.y = g.ymin + np.arange(g.ny) * g.side
        self.z = g.zmin + np.arange(g.nz) * g.side


class PatchSet:
    """Host copy of a patch set in the C-ABI layout (see include/nsgpu.h)."""

    KINDS = ("point", "regular_edge", "singular_edge", "regular_facet", "singular_facet",
             "skin_point", "skin_edge", "skin_facet", "skin_tetra")

    def __init__(self, f64: np.ndarray, i32: np.ndarray, pool: np.ndarray, pool_flag: np.ndarray, probe: float,
                 counts: tuple[int, ...] = (), atoms_of: np.ndarray | None = None,
                 built_from: np.ndarray | None = None):
        self.f64 = np.ascontiguousarray(f64, np.float64).reshape(-1, 20)
        self.i32 = np.ascontiguousarray(i32, np.int32).reshape(-1, 4)
        self.pool = np.ascontiguousarray(pool, np.float64).reshape(-1, 4)
        self.pool_flag = np.ascontiguousarray(pool_flag, np.int8).reshape(-1)
        self.probe = float(probe)
        self.counts = tuple(counts) or tuple(int((self.i32[:, 0] == k).sum()) for k in range(len(self.KINDS)))
        # atoms each patch depends on (3 per patch, -1 unused) and the atoms the set was built
        # from (after jitter): the chain rule from patch parameters to atoms needs both
        self.atoms_of = None if atoms_of is None else np.ascontiguousarray(atoms_of, np.int32).reshape(-1, 3)
        self.built_from = built_from

    @property
    def n(self) -> int:
        return len(self.i32)

    @classmethod
    def from_native(cls, handle: ctypes.c_void_p, probe: float) -> "PatchSet":
        L = N.lib()
        n = ctypes.c_int64()
        npool = ctypes.c_int64()
        counts = (ctypes.c_int64 * 5)()
        N.check(L.nsg_patchset_info(handle, ctypes.byref(n), ctypes.byref(npool), counts), "patchset_info")
        counts = (ctypes.c_int64 * len(cls.KINDS))()
        N.check(L.nsg_patchset_kind_counts(handle, counts, len(cls.KINDS)), "patchset_kind_counts")
        f64 = np.zeros((n.value, 20))
        i32 = np.zeros((n.value, 4), np.int32)
        pool = np.zeros((npool.value, 4))
        flag = np.zeros(npool.value, np.int8)
        N.check(L.nsg_patchset_export(handle, N.ptr(f64), N.ptr(i32), N.ptr(pool), N.ptr(flag)), "patchset_export")
        atoms_of = np.zeros((n.value, 3), np.int32)
        if n.value:
            N.check(L.nsg_patchset_atoms(handle, N.ptr(atoms_of)), "patchset_atoms")
        return cls(f64, i32, pool, flag, probe, tuple(counts), atoms_of)

    def chain_to_atoms(self, gpatch: np.ndarray, atoms: np.ndarray | None = None) -> np.ndarray:
        """(n_atoms, 4) derivative with respect to atom x, y, z, r from per-patch parameter
        derivatives (n_patches x 8)."""
        atoms = self.built_from if atoms is None else atoms
        if atoms is None or self.atoms_of is None:
            raise RuntimeError("patch set has no atom map")
        atoms = np.ascontiguousarray(atoms, np.float64)
        gpatch = np.ascontiguousarray(gpatch, np.float64)
        out = np.zeros((len(atoms), 4))
        rc = N.lib().nsg_ses_chain_grad(N.ptr(atoms), len(atoms), self.probe, self.n, N.ptr(self.i32), N.ptr(self.f64),
                                        N.ptr(self.atoms_of), N.ptr(gpatch), N.ptr(out))
        if rc not in (N.NSG_OK, -8):
            N.check(rc, "gradient chain rule")
        return out


def build_ses_patches(atoms: np.ndarray, probe: float, threads: int = 0) -> PatchSet:
    """SES patch set (points, tori, probe patches) of jittered atoms, built on the host."""
    atoms = np.ascontiguousarray(atoms, np.float64)
    h = ctypes.c_void_p()
    rc = N.lib().nsg_ses_build(N.ptr(atoms), len(atoms), probe, threads, ctypes.byref(h))
    if rc not in (N.NSG_OK, -8):
        N.check(rc, "SES patch construction")
    try:
        ps = PatchSet.from_native(h, probe)
        ps.degenerate = rc == -8
        ps.built_from = atoms.copy()
        return ps
    finally:
        N.lib().nsg_patchset_free(h)


def build_skin_patches(atoms: np.ndarray, shrink: float) -> PatchSet:
    """Skin patch set (mixed cells of the weighted atoms: reduced Voronoi cells, edge and facet
    prisms, reduced tetrahedra) of jittered atoms with shrink factor ``shrink``, built on the host."""
    atoms = np.ascontiguousarray(atoms, np.float64)
    h = ctypes.c_void_p()
    rc = N.lib().nsg_skin_build(N.ptr(atoms), len(atoms), float(shrink), 0, ctypes.byref(h))
    if rc not in (N.NSG_OK, -8):
        N.check(rc, "skin patch construction")
    try:
        ps = PatchSet.from_native(h, 0.0)
        ps.degenerate = rc == -8
        ps.built_from = atoms.copy()
        ps.shrink = float(shrink)
        return ps
    finally:
        N.lib().nsg_patchset_free(h)


# --------------------------------------------------------------------------------------------
class Context:
    """A libnsgpu context: a CUDA stream plus device-resident buffers on one GPU."""

    def __init__(self, device: int = 0):
        self.handle = ctypes.c_void_p()
        N.check(N.lib().nsg_ctx_create(device, ctypes.byref(self.handle)), "context creation")

    def close(self) -> None:
        if self.handle:
            N.lib().nsg_ctx_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Surface:
    """Base of the GPU-backed surfaces (the reference's ``Surface`` plugin interface)."""

    name = "surface"

    def __init__(self, cf: ConfigFile | None = None, delphi: DelPhiShared | None = None, device: int = 0):
        self.delphi = delphi
        cf = cf or ConfigFile()
        self.accurateTriangulation = cf.read("Accurate_Triangulation", False, bool)
        self.triangulation = cf.read("Triangulation", False, bool)
        self.probe_radius = cf.read("Probe_Radius", DEFAULT_PROBE, float)
        self.patchBasedAlgorithm = cf.read("Patch_Based_Algorithm", True, bool)
        self.analyticalTorus = cf.read("Analytical_Ray_Vs_Torus_Intersection", True, bool)
        self.computeNormals = cf.read("Compute_Vertex_Normals", False, bool)
        self.forceSerialBuild = cf.read("Force_Serial_Build", False, bool)
        self.numThreads = cf.read("Number_thread", 0, int)
        self.precision = cf.read("Gpu_Precision", "fp64", str).strip().lower()
        self.projBGP = cf.read("Project_boundary_grid_points", False, bool)
        self.auxGridDim = cf.read("Max_ses_patches_auxiliary_grid_size", 50, int)
        self.keepWellShapedCavities = cf.read("Keep_Water_Shaped_Cavities", False, bool)
        self.randDisplacement = RAND_DISPLACEMENT
        self.device = device
        self.ctx: Context | None = None
        self.patches: PatchSet | None = None
        self.volume = None
        self.area = None
        self.insideness: np.ndarray | None = None
        self.vertices: np.ndarray | None = None
        self.vertex_edges: np.ndarray | None = None
        self.triangles: np.ndarray | None = None
        self.ncav = 0

    # -- reference interface ---------------------------------------------------------------
    def build(self) -> bool:
        raise NotImplementedError

    def getNumPatches(self) -> int:
        return 0 if self.patches is None else self.patches.n

    def isPatchBasedRayTracingSupported(self) -> bool:
        return True

    def _context(self) -> Context:
        if self.ctx is None:
            self.ctx = Context(self.device)
        return self.ctx

    def upload(self) -> None:
        if self.patches is None or self.delphi is None:
            raise RuntimeError("Cannot get surface without DelPhi environment and patches")
        c = self._context().handle
        p = self.patches
        N.check(N.lib().nsg_set_grid(c, ctypes.byref(self.delphi.grid)), "set_grid")
        N.check(N.lib().nsg_upload_patches(c, p.n, N.ptr(p.f64), N.ptr(p.i32), len(p.pool), N.ptr(p.pool),
                                           N.ptr(p.pool_flag), p.probe), "upload_patches")

    def setKeepWellShapedCavities(self, flag: bool) -> None:
        self.keepWellShapedCavities = bool(flag)

    def filterCavities(self, modStatus: bool = False) -> int:
        """Water-shape filter of the cavities kept by the last cavity detection
        (filterCavitiesWithBilevelStatusMap, src/Surface.cpp:3011-3290) with a probe of
        ``probe_radius``: the nodes of a cavity that no probe sphere inside the cavity covers are
        filled; a cavity filled completely is flagged in ``delphi.cavitiesFlag``.  Returns the
        number of filled nodes."""
        c = self._context().handle
        nrem = ctypes.c_int64()
        N.check(N.lib().nsg_filter_cavities(c, float(self.probe_radius), int(bool(modStatus)), ctypes.byref(nrem)),
                "cavity shape filter")
        flagv = np.zeros(max(self.ncav, 0), np.int32)
        if self.ncav > 0:
            N.check(N.lib().nsg_download_cavities(c, None, N.ptr(flagv)), "download cavities")
        self.delphi.cavitiesFlag = [bool(f) for f in flagv]
        return nrem.value

    def difference(self, small: "Surface", fill_volume: float = 0.0) -> int:
        """Pocket detection by difference, pocket mode's ``(*surf1) -= (*surf2)`` followed by
        ``fillCavities`` (src/main.cpp:1533, 1586; Surface::operator-=, src/Surface.cpp:15556-15619):
        this surface holds the fat-probe cast and ``small`` the small-probe cast of the same grid.
        The nodes inside this surface and outside ``small`` that a 1.4 A water probe fits in become
        the pockets (``ncav``, ``delphi.cavitiesSize`` / ``cavitiesFlag``, the status map with the
        pocket labels); pockets of at most ``fill_volume`` A^3 are filled.  Returns the pocket
        count."""
        c = self._context().handle
        n = ctypes.c_int()
        N.check(N.lib().nsg_pocket_difference(c, small._context().handle, float(fill_volume), ctypes.byref(n)),
                "pocket difference")
        self.ncav = n.value
        sizes = np.zeros(max(self.ncav, 0))
        flagv = np.zeros(max(self.ncav, 0), np.int32)
        if self.ncav > 0:
            N.check(N.lib().nsg_download_cavities(c, N.ptr(sizes), N.ptr(flagv)), "download cavities")
        self.delphi.cavitiesSize = sizes.tolist()
        self.delphi.cavitiesFlag = [bool(f) for f in flagv]
        g = self.delphi.grid
        if self.delphi.buildStatus:
            st = np.empty(g.nx * g.ny * g.nz, np.int32)
            N.check(N.lib().nsg_download_status(c, N.ptr(st)), "download status")
            self.delphi.status = st.reshape(g.nz, g.ny, g.nx)
        if self.accurateTriangulation:
            bits = np.empty(((g.nx + 31) >> 5) * g.ny * g.nz, np.uint32)
            N.check(N.lib().nsg_download_insideness(c, N.ptr(bits)), "download insideness")
            self.insideness = bits
        return self.ncav

    def getCavitiesAtoms(self) -> list[list[int]]:
        """Atoms lining each cavity of the last cavity detection (getCavitiesAtomsWithBilevelStatusMap,
        src/Surface.cpp:2249-2346), into ``delphi.cav2atoms``: per cavity the ascending indices of
        the atoms nearest (least power distance, in the reference's atom grid) to the cavity's
        boundary nodes; -1 where a boundary node has no atom in its 27 grid cells."""
        c = self._context().handle
        atoms = np.ascontiguousarray(self.delphi.atoms, np.float64)
        n = ctypes.c_int64()
        N.check(N.lib().nsg_cavity_atoms(c, N.ptr(atoms), len(atoms), None, None, ctypes.byref(n)), "cavity atoms")
        off = np.zeros(max(self.ncav, 0) + 1, np.int32)
        lst = np.zeros(max(n.value, 1), np.int32)
        N.check(N.lib().nsg_cavity_atoms(c, N.ptr(atoms), len(atoms), N.ptr(off), N.ptr(lst), ctypes.byref(n)),
                "cavity atoms")
        self.delphi.cav2atoms = [lst[off[i]:off[i + 1]].tolist() for i in range(max(self.ncav, 0))]
        return self.delphi.cav2atoms

    def getSurf(self, optimize_grids: bool = True, fill: bool = False, cav_vol: float = 0.0,
                keep_hits: bool = False, download: bool = True, grad: bool = False) -> float:
        """Ray casts the grid: status map, insideness bits, volume; optional cavity filling.
        With ``grad`` the derivatives of the volume (and of the area of the following
        ``triangulateSurface``) with respect to the atoms become available from ``gradients``."""
        if self.delphi is None:
            raise RuntimeError("Cannot get surface without DelPhi environment!")
        self.upload()
        c = self._context().handle
        flags = 0
        if self.delphi.buildStatus:
            flags |= N.STATUS
        if self.accurateTriangulation:
            flags |= N.ACCURATE_TRIANGULATION
        if self.delphi.buildEpsMap:
            flags |= N.EPSMAP
        elif self.projBGP:
            raise RuntimeError("Cannot project boundary grid points without an epsilon map (Build_epsilon_maps = true)")
        if keep_hits:
            flags |= N.KEEP_HITS
        if grad:
            flags |= N.GRAD
        if self.computeNormals and self.providesAnalyticalNormals and self.accurateTriangulation:
            flags |= N.NORMALS
        prec = PRECISIONS.get(self.precision)
        if prec is None:
            raise ValueError(f"unknown Gpu_Precision {self.precision}")
        vol = ctypes.c_double()
        N.check(N.lib().nsg_raycast(c, flags, prec, ctypes.byref(vol)), "ray casting")
        self.volume = vol.value
        self._analytic_normals = bool(flags & (N.NORMALS | N.GRAD))
        if fill:
            if not self.delphi.buildStatus:
                raise RuntimeError("Cannot do cavity detection without a status map (Build_status_map = true)")
            ncav = ctypes.c_int()
            N.check(N.lib().nsg_cavities(c, float(cav_vol), ctypes.byref(ncav)), "cavity detection")
            self.ncav = ncav.value
            sizes = np.zeros(max(self.ncav, 0))
            flagv = np.zeros(max(self.ncav, 0), np.int32)
            if self.ncav > 0:
                N.check(N.lib().nsg_download_cavities(c, N.ptr(sizes), N.ptr(flagv)), "download cavities")
            self.delphi.cavitiesSize = sizes.tolist()
            self.delphi.cavitiesFlag = [bool(f) for f in flagv]
            if self.keepWellShapedCavities:
                self.filterCavities()
            self.getCavitiesAtoms()
        if download:
            g = self.delphi.grid
            if self.delphi.buildStatus:
                st = np.empty(g.nx * g.ny * g.nz, np.int32)
                N.check(N.lib().nsg_download_status(c, N.ptr(st)), "download status")
                self.delphi.status = st.reshape(g.nz, g.ny, g.nx)
            if self.accurateTriangulation:
                words = ((g.nx + 31) >> 5) * g.ny * g.nz
                bits = np.empty(words, np.uint32)
                N.check(N.lib().nsg_download_insideness(c, N.ptr(bits)), "download insideness")
                self.insideness = bits
            if self.delphi.buildEpsMap:
                eps = np.empty(g.nx * g.ny * g.nz * 3, np.int32)
                N.check(N.lib().nsg_download_epsmap(c, N.ptr(eps)), "download epsilon map")
                self.delphi.epsmap = eps.reshape(g.nz, g.ny, g.nx, 3)
                ideb = np.empty(g.nx * g.ny * g.nz, np.uint8)
                N.check(N.lib().nsg_download_idebmap(c, N.ptr(ideb)), "download ideb map")
                self.delphi.idebmap = ideb.reshape(g.nz, g.ny, g.nx).astype(bool)
        if self.projBGP:
            self.projectBoundaryGridPoints()
        return self.volume

    def projectBoundaryGridPoints(self) -> int:
        """Boundary grid points of the epsilon map and their projection onto the surface (the
        projBGP phase of Surface::getSurf, src/Surface.cpp:1473-1678); fills the DelPhiShared's
        ibgp, bgp_type, scspos, scsnor (and bgp_flag: 0 projected; 1 for the SES no feasible
        projection among the auxiliary cell's patches, the point kept, for the blobby mesh the
        nearest point on a triangle's edge or corner; 2 empty cell).  The blobby surface projects
        onto its triangles as MeshSurface::getProjection (src/MeshSurface.cpp:2045-2141) does.
        Returns the point count."""
        if self.name not in ("ses", "blobby"):
            raise NotImplementedError("boundary grid point projection is provided for the SES and blobby surfaces")
        c = self._context().handle
        n = ctypes.c_int64()
        ne = ctypes.c_int64()
        N.check(N.lib().nsg_bgp(c, 1, int(self.auxGridDim), ctypes.byref(n), ctypes.byref(ne)), "boundary grid points")
        d = self.delphi
        d.nbgp = n.value
        d.ibgp = np.zeros((d.nbgp, 3), np.int32)
        d.bgp_type = np.zeros(d.nbgp, np.int32)
        d.scspos = np.zeros((d.nbgp, 3))
        d.scsnor = np.zeros((d.nbgp, 3))
        d.bgp_flag = np.zeros(d.nbgp, np.int32)
        if d.nbgp:
            N.check(N.lib().nsg_download_bgp(c, N.ptr(d.ibgp), N.ptr(d.bgp_type), N.ptr(d.scspos), N.ptr(d.scsnor),
                                             N.ptr(d.bgp_flag)), "download boundary grid points")
        return d.nbgp

    def triangulateSurface(self, outputMesh: bool = False, fileName: str = "triangulatedSurf",
                           download: bool = True) -> float:
        """Analytical marching cubes on the insideness grid; returns the mesh area."""
        c = self._context().handle
        area = ctypes.c_double()
        nv = ctypes.c_int64()
        nt = ctypes.c_int64()
        N.check(N.lib().nsg_triangulate(c, ctypes.byref(area), ctypes.byref(nv), ctypes.byref(nt)), "triangulation")
        self.area = area.value
        if download:
            self.vertices = np.empty((nv.value, 3))
            self.vertex_edges = np.empty((nv.value, 4), np.int32)
            self.triangles = np.empty((nt.value, 3), np.int32)
            N.check(N.lib().nsg_download_mesh(c, N.ptr(self.vertices), N.ptr(self.vertex_edges),
                                              N.ptr(self.triangles)), "download mesh")
        if outputMesh:
            self.saveMesh("off", False, fileName)
        return self.area

    MESH_FORMATS = {"off": 0, "ply": 1}
    # formats with vertex normals and/or nearest atoms (nsg_write_mesh_attrs)
    ATTR_MESH_FORMATS = {"off_n": 0, "msms_no_a": 1, "off_a": 2, "off_n_a": 3, "msms": 4}

    def vertexAtoms(self) -> np.ndarray:
        """Nearest atom (0-based, least power distance as vdwAccessible, src/Surface.cpp:16663-16715)
        of every vertex of the last triangulation."""
        if self.vertices is None:
            raise RuntimeError("no mesh: call triangulateSurface() first")
        v = np.ascontiguousarray(self.vertices, np.float64)
        a = np.ascontiguousarray(self.delphi.atoms, np.float64)
        out = np.zeros(len(v), np.int32)
        N.check(N.lib().nsg_vertex_atoms(N.ptr(v), len(v), N.ptr(a), len(a), N.ptr(out)), "vertex atoms")
        return out

    # surfaces whose patches give a normal at every hit (the reference's providesAnalyticalNormals)
    providesAnalyticalNormals = True

    def vertexNormals(self) -> np.ndarray:
        """Vertex normals of the last triangulation, as the reference outputs them with
        Compute_Vertex_Normals: the patch normal at each analytic vertex and the triangle average for
        the others (nsg_vertex_normals); by triangle averaging alone when the surface has no analytic
        normals or the ray cast did not keep its hits' patches."""
        if self.vertices is None:
            raise RuntimeError("no mesh: call triangulateSurface() first")
        if not (self.providesAnalyticalNormals and getattr(self, "_analytic_normals", False)):
            return self.approximateNormals()
        out = np.zeros((len(self.vertices), 3))
        N.check(N.lib().nsg_vertex_normals(self._context().handle, N.ptr(out)), "vertex normals")
        return out

    def approximateNormals(self) -> np.ndarray:
        """Vertex normals of the last triangulation by triangle averaging (the reference's
        approximateNormals for surfaces without analytic normals, src/Surface.cpp:10588-10660);
        (n_vertices, 3)."""
        if self.vertices is None or self.triangles is None:
            raise RuntimeError("no mesh: call triangulateSurface() first")
        v = np.ascontiguousarray(self.vertices, np.float64)
        t = np.ascontiguousarray(self.triangles, np.int32)
        out = np.zeros((len(v), 3))
        N.check(N.lib().nsg_mesh_normals(N.ptr(v), len(v), N.ptr(t), len(t), N.ptr(out)), "mesh normals")
        return out

    def saveMesh(self, format: str = "off", revert: bool = False, fileName: str | Path = "triangulatedSurf") -> None:
        """Mesh file in the reference's layout: ``fileName.off`` (+ ``fileNametriangleAreas.txt``),
        ``fileName.ply``, or with vertex normals from approximateNormals() and nearest atoms from
        vertexAtoms(): ``off_n``, ``off_a``, ``off_n_a``, ``msms_no_a`` and ``msms``
        (``fileName.face`` / ``fileName.vert``) (Surface::saveMesh, src/Surface.cpp:10857-11062)."""
        if self.vertices is None or self.triangles is None:
            raise RuntimeError("no mesh: call triangulateSurface() first")
        name = str(format).lower()
        v = np.ascontiguousarray(self.vertices, np.float64)
        t = np.ascontiguousarray(self.triangles, np.int32)
        if name in self.ATTR_MESH_FORMATS:
            fmt = self.ATTR_MESH_FORMATS[name]
            nrm = np.ascontiguousarray(self.vertexNormals(), np.float64) if fmt != 2 else None
            ato = self.vertexAtoms() if fmt >= 2 else None
            N.check(N.lib().nsg_write_mesh_attrs(str(fileName).encode(), fmt, N.ptr(v),
                                                 None if nrm is None else N.ptr(nrm),
                                                 None if ato is None else N.ptr(ato), len(v), N.ptr(t), len(t),
                                                 int(revert)), "saveMesh")
            return
        fmt = self.MESH_FORMATS.get(name)
        if fmt is None:
            raise ValueError(f"unsupported mesh format {format}; available: "
                             f"{sorted(self.MESH_FORMATS) + sorted(self.ATTR_MESH_FORMATS)}")
        N.check(N.lib().nsg_write_mesh(str(fileName).encode(), fmt, N.ptr(v), len(v), N.ptr(t), len(t), int(revert)),
                "saveMesh")

    def hits(self, ray_set: int) -> tuple[np.ndarray, np.ndarray]:
        """Per-ray sorted hit parameters of one ray set from the last keep_hits ray cast."""
        c = self._context().handle
        g = self.delphi.grid
        nb, na = ((g.ny, g.nz), (g.ny, g.nz), (g.nx, g.ny), (g.nx, g.nz), (g.nx, g.ny), (g.nx, g.nz))[ray_set]
        counts = np.zeros(nb * na, np.int32)
        total = N.lib().nsg_download_hits(c, ray_set, N.ptr(counts), None, 0)
        if total < 0:
            N.check(total, "download hits")
        vals = np.zeros(int(counts.sum()))
        N.check(N.lib().nsg_download_hits(c, ray_set, N.ptr(counts), N.ptr(vals), len(vals)), "download hits")
        return counts.reshape(na, nb), vals

    def patch_gradients(self, area: bool = True) -> tuple[np.ndarray, np.ndarray | None]:
        """Per-patch derivatives (n_patches x 8) of the volume and, when the triangulation ran in
        gradient mode, of the area."""
        c = self._context().handle
        gv = np.zeros((self.patches.n, 8))
        ga = np.zeros((self.patches.n, 8)) if area else None
        N.check(N.lib().nsg_patch_grads(c, N.ptr(gv), N.ptr(ga)), "patch gradients")
        return gv, ga

    def gradients(self, dvol: float = 1.0, darea: float = 0.0) -> np.ndarray:
        """(n_atoms, 4) derivative of dvol * volume + darea * area with respect to the atoms'
        x, y, z and radius, on the fixed grid of the last gradient-mode getSurf (and
        triangulateSurface when darea is nonzero)."""
        gv, ga = self.patch_gradients(area=darea != 0.0)
        g = dvol * gv if ga is None else dvol * gv + darea * ga
        return self.patches.chain_to_atoms(g)

    def stats(self) -> dict:
        out = np.zeros(8, np.int64)
        N.check(N.lib().nsg_stats(self._context().handle, N.ptr(out), 8), "stats")
        keys = ("patches", "vertices", "analytic_vertices", "triangles", "active_cubes", "cavities",
                "overflow_rays", "pair_capacity")
        return dict(zip(keys, out.tolist()))

    # snake_case aliases
    get_surf = getSurf
    triangulate_surface = triangulateSurface


class ConnollySurface(Surface):
    """Solvent-excluded (Connolly) surface, ``Surface = ses``."""

    name = "ses"

    def build(self) -> bool:
        atoms = self.delphi.atoms
        # jitter the atoms after the grid was built (src/ConnollySurface.cpp:2484-2488)
        if self.randDisplacement > 0:
            N.check(N.lib().nsg_jitter_atoms(N.ptr(atoms), len(atoms), self.randDisplacement, ctypes.byref(_seed)),
                    "jitter")
        threads = 1 if self.forceSerialBuild else self.numThreads
        self.patches = build_ses_patches(atoms, self.probe_radius, threads)
        return True


class SkinSurface(Surface):
    """Skin surface of the weighted atoms, ``Surface = skin`` (src/SkinSurface.h): quadric patches
    in the cells of the mixed complex, shrink factor ``Skin_Surface_Parameter``."""

    name = "skin"
    DEFAULT_S = 0.45

    def __init__(self, cf: ConfigFile | None = None, delphi: DelPhiShared | None = None, device: int = 0):
        super().__init__(cf, delphi, device)
        cf = cf or ConfigFile()
        self.setShrinking(cf.read("Skin_Surface_Parameter", self.DEFAULT_S, float))

    def setShrinking(self, ss: float) -> None:
        """The shrink factor s, accepted in [0.05, 0.95]; otherwise the default 0.45 is kept with a
        warning, as SkinSurface::setShrinking does (src/SkinSurface.h)."""
        e = 0.05
        if e <= ss <= 1.0 - e:
            self.s = float(ss)
        else:
            import warnings
            warnings.warn(f"Cannot set {ss}. s parameter is in (0+e,1-e], where e is {e}. Setting {self.DEFAULT_S}")
            self.s = self.DEFAULT_S

    def getShrinking(self) -> float:
        return self.s

    def build(self) -> bool:
        atoms = self.delphi.atoms
        # the reference jitters the atoms inside its build (src/SkinSurface.cpp:1303-1311)
        if self.randDisplacement > 0:
            N.check(N.lib().nsg_jitter_atoms(N.ptr(atoms), len(atoms), self.randDisplacement, ctypes.byref(_seed)),
                    "jitter")
        self.patches = build_skin_patches(atoms, self.s)
        return True

    def getSurf(self, optimize_grids: bool = True, fill: bool = False, cav_vol: float = 0.0,
                keep_hits: bool = False, download: bool = True, grad: bool = False) -> float:
        if grad:
            raise NotImplementedError("gradients are provided for the SES (and blobby) surfaces, not for skin")
        return super().getSurf(optimize_grids, fill, cav_vol, keep_hits, download, grad)


class BlobbySurface(Surface):
    """Blobby surface, ``Surface = blobby`` (src/BlobbySurface.h): the triangle mesh of the atoms'
    Gaussian field (blobbyness ``Blobbyness``, cut-off 6 A) at iso level 1, smoothed once and
    passed through the reference's OFF text round trip, then ray cast as a mesh surface.  The
    field, its marching cubes, the smoothing and the round trip run on the GPU (nsg_blobby_build);
    the mesh stays in device memory as the context's patch set.

    ``differentiable = True`` skips the OFF round trip (a rounding of every coordinate to 1e-3 A,
    piecewise constant in the atoms) so that ``gradients`` can chain the ray-cast volume and area
    back to the atoms."""

    name = "blobby"
    DEFAULT_BLOBBYNESS = -2.5
    providesAnalyticalNormals = False

    def __init__(self, cf: ConfigFile | None = None, delphi: DelPhiShared | None = None, device: int = 0):
        super().__init__(cf, delphi, device)
        cf = cf or ConfigFile()
        self.setBlobbyness(cf.read("Blobbyness", self.DEFAULT_BLOBBYNESS, float))
        # the projection runs on the mesh's auxiliary grid (MeshSurface::init, src/MeshSurface.cpp:179)
        self.auxGridDim = cf.read("Max_mesh_auxiliary_grid_size", 100, int)
        self.differentiable = False
        self.n_mesh_vertices = 0
        self.n_mesh_triangles = 0

    def setBlobbyness(self, b: float) -> None:
        """B < 0; a non-negative value keeps the default -2.5 with a warning (setBlobbyness)."""
        if b >= 0:
            import warnings
            warnings.warn(f"Blobbyness is always a stricly negative real: setting {self.DEFAULT_BLOBBYNESS}")
            b = self.DEFAULT_BLOBBYNESS
        self.B = float(b)

    def getBlobbyness(self) -> float:
        return self.B

    def isPatchBasedRayTracingSupported(self) -> bool:
        # the reference ray casts the blobby mesh ray by ray (BlobbySurface overrides this to false)
        return False

    def getNumPatches(self) -> int:
        return 0

    def build(self) -> bool:
        if self.delphi is None:
            raise RuntimeError("Cannot build without DelPhi environment")
        c = self._context().handle
        N.check(N.lib().nsg_set_grid(c, ctypes.byref(self.delphi.grid)), "set_grid")
        atoms = np.ascontiguousarray(self.delphi.atoms, np.float64)
        flags = 1 if self.differentiable else 0
        N.check(N.lib().nsg_blobby_build(c, N.ptr(atoms), len(atoms), self.B, flags), "blobby build")
        nv, nt = ctypes.c_int64(), ctypes.c_int64()
        N.check(N.lib().nsg_blobby_mesh(c, ctypes.byref(nv), ctypes.byref(nt), None, None), "blobby mesh")
        self.n_mesh_vertices, self.n_mesh_triangles = nv.value, nt.value
        self.built_from = atoms.copy()
        return True

    def upload(self) -> None:
        # the mesh patches are built in the context's device memory by build()
        if self.ctx is None or self.n_mesh_triangles is None:
            raise RuntimeError("Cannot get surface before build()")

    def mesh(self) -> tuple[np.ndarray, np.ndarray]:
        """The blobby mesh that is ray cast: vertices (n, 3) and triangles (m, 3)."""
        c = self._context().handle
        v = np.zeros((self.n_mesh_vertices, 3))
        t = np.zeros((self.n_mesh_triangles, 3), np.int32)
        N.check(N.lib().nsg_blobby_mesh(c, None, None, N.ptr(v), N.ptr(t)), "blobby mesh")
        return v, t

    def gradients(self, dvol: float = 1.0, darea: float = 0.0) -> np.ndarray:
        """(n_atoms, 4) derivative of dvol * volume + darea * area with respect to the atoms' x, y,
        z and radius, after a gradient-mode getSurf (and triangulateSurface when darea is nonzero)
        of a differentiable blobby surface."""
        c = self._context().handle
        n = len(self.built_from)
        gv = np.zeros((n, 4))
        ga = np.zeros((n, 4)) if darea != 0.0 else None
        N.check(N.lib().nsg_blobby_atom_grads(c, N.ptr(gv), None if ga is None else N.ptr(ga)), "blobby gradients")
        return dvol * gv if ga is None else dvol * gv + darea * ga


class SurfaceBatch:
    """Many built surfaces, each with its own grid and patch set, ray cast and triangulated in the
    same kernel launches: one ``getSurf`` + ``triangulateSurface`` per structure, batched.

    Per-structure results are the volumes and areas; the insideness bits come back concatenated.
    Cavity detection and the dense status map stay with the single-structure ``Surface``.
    """

    def __init__(self, surfaces: list[Surface], device: int = 0, precision: str | None = None):
        if not surfaces:
            raise ValueError("empty batch")
        for s in surfaces:
            if s.patches is None or s.delphi is None:
                raise RuntimeError("every surface of a batch must be built first")
        self.surfaces = surfaces
        self.device = device
        self.precision = (precision or surfaces[0].precision).strip().lower()
        self.ctx: Context | None = None
        self.volumes: np.ndarray | None = None
        self.areas: np.ndarray | None = None
        self.n_vertices = 0
        self.n_triangles = 0
        self.insideness: list[np.ndarray] | None = None

    def __len__(self) -> int:
        return len(self.surfaces)

    def _context(self) -> Context:
        if self.ctx is None:
            self.ctx = Context(self.device)
        return self.ctx

    def packed(self) -> tuple:
        """Concatenated patch arrays and their per-structure offsets (host)."""
        ps = [s.patches for s in self.surfaces]
        patch_off = np.zeros(len(ps) + 1, np.int64)
        pool_off = np.zeros(len(ps) + 1, np.int64)
        patch_off[1:] = np.cumsum([p.n for p in ps])
        pool_off[1:] = np.cumsum([len(p.pool) for p in ps])
        f64 = np.ascontiguousarray(np.concatenate([p.f64 for p in ps]))
        i32 = np.ascontiguousarray(np.concatenate([p.i32 for p in ps]))
        pool = np.ascontiguousarray(np.concatenate([p.pool for p in ps])) if pool_off[-1] else np.zeros((1, 4))
        flag = np.ascontiguousarray(np.concatenate([p.pool_flag for p in ps])) if pool_off[-1] else np.zeros(1, np.int8)
        return patch_off, pool_off, f64, i32, pool, flag

    def upload(self) -> None:
        c = self._context().handle
        n = len(self.surfaces)
        grids = (N.NsGrid * n)(*[s.delphi.grid for s in self.surfaces])
        N.check(N.lib().nsg_set_batch(c, n, grids), "set_batch")
        patch_off, pool_off, f64, i32, pool, flag = self.packed()
        probe = self.surfaces[0].patches.probe
        N.check(N.lib().nsg_upload_batch(c, N.ptr(patch_off), N.ptr(f64), N.ptr(i32), N.ptr(pool_off), N.ptr(pool),
                                         N.ptr(flag), probe), "upload_batch")

    def getSurf(self, download: bool = False, grad: bool = False) -> np.ndarray:
        """Ray casts every structure's grid; returns the per-structure volumes.  With ``grad`` the
        atom derivatives of the volumes (and of the areas of the following triangulateSurface)
        become available from ``atom_gradients``."""
        self.upload()
        c = self._context().handle
        s0 = self.surfaces[0]
        flags = 0
        if s0.delphi.buildStatus:
            flags |= N.STATUS
        if s0.accurateTriangulation:
            flags |= N.ACCURATE_TRIANGULATION
        if grad:
            flags |= N.GRAD
        prec = PRECISIONS.get(self.precision)
        if prec is None:
            raise ValueError(f"unknown Gpu_Precision {self.precision}")
        vol = ctypes.c_double()
        N.check(N.lib().nsg_raycast(c, flags, prec, ctypes.byref(vol)), "ray casting")
        self.volumes = np.zeros(len(self))
        N.check(N.lib().nsg_batch_results(c, N.ptr(self.volumes), None), "batch results")
        if download and s0.accurateTriangulation:
            words = [((s.delphi.grid.nx + 31) >> 5) * s.delphi.grid.ny * s.delphi.grid.nz for s in self.surfaces]
            bits = np.empty(sum(words), np.uint32)
            N.check(N.lib().nsg_download_insideness(c, N.ptr(bits)), "download insideness")
            self.insideness = np.split(bits, np.cumsum(words)[:-1])
        return self.volumes

    def triangulateSurface(self) -> np.ndarray:
        """Marching cubes on every structure; returns the per-structure areas."""
        c = self._context().handle
        area = ctypes.c_double()
        nv = ctypes.c_int64()
        nt = ctypes.c_int64()
        N.check(N.lib().nsg_triangulate(c, ctypes.byref(area), ctypes.byref(nv), ctypes.byref(nt)), "triangulation")
        self.n_vertices, self.n_triangles = nv.value, nt.value
        self.areas = np.zeros(len(self))
        N.check(N.lib().nsg_batch_results(c, None, N.ptr(self.areas)), "batch results")
        return self.areas

    def set_tuning(self, params) -> None:
        """Sets the tracer's launch shapes: [intersection threads per block, intersection blocks
        per SM, candidate threads per block] (the ranges of ``nsg_set_tuning``)."""
        p = np.ascontiguousarray(params, np.int32)
        N.check(N.lib().nsg_set_tuning(self._context().handle, N.ptr(p), len(p)), "set tuning")

    def autotune(self, grad: bool = False, reps: int = 2) -> tuple[list[int], float]:
        """Picks the tracer's launch shapes (intersection block size and blocks per SM, candidate
        block size) for this batch by timing ray casts; returns the shape and its ms per cast."""
        self.upload()
        c = self._context().handle
        s0 = self.surfaces[0]
        flags = (N.STATUS if s0.delphi.buildStatus else 0) | (N.ACCURATE_TRIANGULATION if s0.accurateTriangulation else 0)
        if grad:
            flags |= N.GRAD
        ms = ctypes.c_double()
        N.check(N.lib().nsg_autotune(c, flags, PRECISIONS[self.precision], reps, ctypes.byref(ms)), "autotune")
        p = np.zeros(3, np.int32)
        N.check(N.lib().nsg_get_tuning(c, N.ptr(p), 3), "get tuning")
        return p.tolist(), ms.value

    def packed_atoms(self) -> tuple:
        """Concatenated atoms the patch sets were built from, their offsets and the patch atom map."""
        ps = [s.patches for s in self.surfaces]
        atom_off = np.zeros(len(ps) + 1, np.int64)
        atom_off[1:] = np.cumsum([len(p.built_from) for p in ps])
        atoms = np.ascontiguousarray(np.concatenate([p.built_from for p in ps]))
        patch_atoms = np.ascontiguousarray(np.concatenate([p.atoms_of for p in ps]))
        return atom_off, atoms, patch_atoms

    def atom_gradients(self) -> list[tuple[np.ndarray, np.ndarray]]:
        """Per structure: (d volume / d atoms, d area / d atoms), each (n_atoms, 4) for x, y, z, r,
        after a gradient-mode getSurf and triangulateSurface (chained on the device)."""
        c = self._context().handle
        atom_off, atoms, patch_atoms = self.packed_atoms()
        N.check(N.lib().nsg_upload_atoms(c, N.ptr(atom_off), N.ptr(atoms), N.ptr(patch_atoms)), "upload atoms")
        gv = np.zeros((len(atoms), 4))
        ga = np.zeros((len(atoms), 4))
        rc = N.lib().nsg_atom_grads(c, N.ptr(gv), N.ptr(ga))
        if rc not in (N.NSG_OK, -8):
            N.check(rc, "atom gradients")
        return [(gv[atom_off[b]:atom_off[b + 1]], ga[atom_off[b]:atom_off[b + 1]]) for b in range(len(self))]

    def close(self) -> None:
        if self.ctx is not None:
            self.ctx.close()
            self.ctx = None


class SurfaceFactory:
    """Surface registry keyed by the .prm ``Surface`` value."""

    def __init__(self):
        self.surfRegister: dict[str, Callable[..., Surface]] = {}

    def add(self, name: str, ctor: Callable[..., Surface]) -> None:
        self.surfRegister[name] = ctor

    def create(self, conf: ConfigFile, ds: DelPhiShared, device: int = 0) -> Surface:
        name = conf.read("Surface", "ses", str).strip()
        if name not in self.surfRegister:
            raise KeyError(f"{name} type is not registered!")
        return self.surfRegister[name](conf, ds, device)

    def available(self) -> list[str]:
        return sorted(self.surfRegister)


_factory = SurfaceFactory()
_factory.add("ses", lambda cf, ds, dev=0: ConnollySurface(cf, ds, dev))
_factory.add("skin", lambda cf, ds, dev=0: SkinSurface(cf, ds, dev))
_factory.add("blobby", lambda cf, ds, dev=0: BlobbySurface(cf, ds, dev))


def surfaceFactory() -> SurfaceFactory:
    return _factory


# --------------------------------------------------------------------------------------------
class NanoShaper:
    """Library facade: atoms + configuration in, surface volume / area / maps out."""

    def __init__(self, atoms: "np.ndarray | str | Path | None" = None, surface: str = "ses",
                 probe: float = DEFAULT_PROBE, scale: float = DEFAULT_SCALE, perfil: float = DEFAULT_PERFIL,
                 config: ConfigFile | None = None, device: int = 0, precision: str = "fp64"):
        cf = config or ConfigFile()
        # atoms: an (N, 4) array, a molecule file (xyzr, or pqr by name), or, when None, the
        # configuration's XYZR_FileName as in a .prm file
        if atoms is None:
            if not cf.keyExists("XYZR_FileName"):
                raise ValueError("no atoms: pass an array or a file, or set XYZR_FileName")
            atoms = cf.read("XYZR_FileName", "", str).strip()
            # the reference runs in the directory of its .prm file: a relative name is read there
            if cf.path is not None and not Path(atoms).is_absolute() and not Path(atoms).exists():
                atoms = str(cf.path.parent / atoms)
        if isinstance(atoms, (str, Path)):
            atoms = read_atoms(atoms)
        if not cf.keyExists("Surface"):
            cf.add("Surface", surface)
        if not cf.keyExists("Probe_Radius"):
            cf.add("Probe_Radius", probe)
        if not cf.keyExists("Accurate_Triangulation"):
            cf.add("Accurate_Triangulation", True)
        if not cf.keyExists("Gpu_Precision"):
            cf.add("Gpu_Precision", precision)
        self.cf = cf
        self.scale = cf.read("Grid_scale", scale, float)
        self.perfil = cf.read("Grid_perfil", perfil, float)
        self.ds = DelPhiShared(atoms, self.scale, self.perfil, build_status=cf.read("Build_status_map", True, bool),
                               build_eps_map=cf.read("Build_epsilon_maps", False, bool))
        self.surf = surfaceFactory().create(cf, self.ds, device)

    def buildAnalyticalSurface(self, randDisplacement: float = -1) -> bool:
        if randDisplacement >= 0:
            self.surf.randDisplacement = randDisplacement
        return self.surf.build()

    def colourGrid(self, fill_cavities: bool | None = None, cav_vol: float | None = None) -> float:
        fill = self.cf.read("Cavity_Detection_Filling", False, bool) if fill_cavities is None else fill_cavities
        vol = self.cf.read("Conditional_Volume_Filling_Value", 11.4, float) if cav_vol is None else cav_vol
        return self.surf.getSurf(True, fill, vol)

    def triangulate(self) -> float:
        return self.surf.triangulateSurface()

    def getGridSize(self) -> list[int]:
        return [self.ds.nx, self.ds.ny, self.ds.nz]

    def getGridPointStatus(self, ix: int, iy: int, iz: int) -> int:
        """+1 outside, -1 inside, 0 unknown (grid not computed)."""
        if self.ds.status is None:
            return 0
        return -1 if self.ds.status[iz, iy, ix] == STATUS_POINT_INSIDE else 1
