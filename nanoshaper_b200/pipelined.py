"""Pipelined batches: host-resident ensembles with transfers overlapped with compute.

An ensemble whose patch sets live in host memory spends a large share of its time in the
host-to-device copy (about 0.9 GB per 1,000 structures of ~4,000 atoms).  ``PipelinedBatches``
splits the ensemble into chunks, keeps every chunk's inputs in pinned host buffers, and drives
several libnsgpu contexts (two by default, each with its own CUDA stream) from as many host threads.
While one context computes a chunk, another copies the next, so the copy engines and the SMs work
at the same time.  Each chunk is
one batch (``nsg_set_batch`` / ``nsg_upload_batch`` / ``nsg_upload_atoms``, then the ray cast,
the triangulation and the atom derivatives).  The results are the same as one batch of the whole
ensemble.

Two details shorten the start of the pipeline, when no kernel has work yet: the first chunk is half
the size of the others, and one upload is in flight at a time (a lock), so that each copy has the
whole host link and the first chunk's kernels start as early as possible.
"""
from __future__ import annotations

import ctypes
import threading

import numpy as np
import torch

from . import _native as N
from . import surface as S


def chunk_bounds(n: int, n_chunks: int) -> np.ndarray:
    """Boundaries of the chunks of an ensemble of n structures: chunk weights 1/2, 1, 1, ... (a
    short first chunk starts the kernels early), no empty chunk; returns n_chunks' + 1 increasing
    offsets from 0 to n with n_chunks' <= n_chunks."""
    n_chunks = max(1, min(n_chunks, n))
    weights = np.array([0.5] + [1.0] * (n_chunks - 1))
    bounds = np.round(np.concatenate([[0.0], np.cumsum(weights)]) / weights.sum() * n).astype(int)
    bounds = np.maximum.accumulate(bounds)
    keep = [0] + [i for i in range(1, len(bounds)) if bounds[i] > bounds[i - 1]]
    return bounds[keep]


class _Chunk:
    def __init__(self, surfs: list, lo: int, hi: int):
        self.lo, self.hi = lo, hi
        batch = S.SurfaceBatch(surfs[lo:hi])
        self.patch_off, self.pool_off, f64, i32, pool, flag = batch.packed()
        self.atom_off, atoms, patch_atoms = batch.packed_atoms()
        self.pin = {}
        for name, a in (("f64", f64), ("i32", i32), ("pool", pool), ("flag", flag), ("atoms", atoms),
                        ("patch_atoms", patch_atoms)):
            t = torch.empty(a.nbytes, dtype=torch.uint8, pin_memory=True)
            t.numpy()[:] = a.view(np.uint8).ravel()
            self.pin[name] = t
        self.grids = (N.NsGrid * (hi - lo))(*[s.delphi.grid for s in surfs[lo:hi]])
        self.probe = surfs[lo].patches.probe
        n_atoms = int(self.atom_off[-1])
        self.gvol = torch.empty(n_atoms * 4, dtype=torch.float64, pin_memory=True)
        self.garea = torch.empty(n_atoms * 4, dtype=torch.float64, pin_memory=True)
        self.volumes = np.zeros(hi - lo)
        self.areas = np.zeros(hi - lo)

    @property
    def h2d_bytes(self) -> int:
        return sum(t.numel() for t in self.pin.values())


class PipelinedBatches:
    """Volume, area and their atom derivatives of every structure of an ensemble, chunk by chunk
    on two contexts with overlapped transfers."""

    def __init__(self, surfaces: list, n_chunks: int = 4, device: int = 0, precision: str = "mixed",
                 tuning: list[int] | None = None, n_contexts: int = 2):
        if not surfaces:
            raise ValueError("empty ensemble")
        bounds = chunk_bounds(len(surfaces), n_chunks)
        n_chunks = len(bounds) - 1
        self.chunks = [_Chunk(surfaces, int(bounds[i]), int(bounds[i + 1])) for i in range(n_chunks)]
        self.n = len(surfaces)
        self.prec = S.PRECISIONS[precision]
        s0 = surfaces[0]
        self.flags = (N.STATUS if s0.delphi.buildStatus else 0) | N.ACCURATE_TRIANGULATION | N.GRAD
        self.ctxs = [S.Context(device) for _ in range(max(1, n_contexts))]
        self._upload_lock = threading.Lock()
        if tuning is not None:
            p = np.ascontiguousarray(tuning, np.int32)
            for c in self.ctxs:
                N.check(N.lib().nsg_set_tuning(c.handle, N.ptr(p), len(p)), "set tuning")

    @property
    def h2d_bytes(self) -> int:
        return sum(ch.h2d_bytes for ch in self.chunks)

    @property
    def d2h_bytes(self) -> int:
        return sum(16 * (ch.hi - ch.lo) + 8 * (ch.gvol.numel() + ch.garea.numel()) for ch in self.chunks)

    def _run_chunk(self, c, ch: _Chunk) -> None:
        L = N.lib()
        with self._upload_lock:
            N.check(L.nsg_set_batch(c, ch.hi - ch.lo, ch.grids), "set_batch")
            N.check(L.nsg_upload_batch(c, N.ptr(ch.patch_off), ch.pin["f64"].data_ptr(), ch.pin["i32"].data_ptr(),
                                       N.ptr(ch.pool_off), ch.pin["pool"].data_ptr(), ch.pin["flag"].data_ptr(),
                                       ch.probe), "upload_batch")
            N.check(L.nsg_upload_atoms(c, N.ptr(ch.atom_off), ch.pin["atoms"].data_ptr(),
                                       ch.pin["patch_atoms"].data_ptr()), "upload atoms")
        v = ctypes.c_double()
        N.check(L.nsg_raycast(c, self.flags, self.prec, ctypes.byref(v)), "raycast")
        a = ctypes.c_double()
        nv = ctypes.c_int64()
        nt = ctypes.c_int64()
        N.check(L.nsg_triangulate(c, ctypes.byref(a), ctypes.byref(nv), ctypes.byref(nt)), "triangulate")
        rc = L.nsg_atom_grads(c, ch.gvol.data_ptr(), ch.garea.data_ptr())
        if rc not in (N.NSG_OK, -8):
            N.check(rc, "atom gradients")
        N.check(L.nsg_batch_results(c, N.ptr(ch.volumes), N.ptr(ch.areas)), "batch results")

    def run(self) -> tuple[np.ndarray, np.ndarray]:
        """One pass over the ensemble; returns the per-structure volumes and areas (the atom
        derivatives are in ``gradients()``)."""
        errors: list[BaseException] = []

        nw = len(self.ctxs)

        def worker(w: int) -> None:
            try:
                for ch in self.chunks[w::nw]:
                    self._run_chunk(self.ctxs[w].handle, ch)
            except BaseException as e:  # reported after all workers joined
                errors.append(e)

        threads = [threading.Thread(target=worker, args=(w,)) for w in range(nw)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        if errors:
            raise errors[0]
        return (np.concatenate([ch.volumes for ch in self.chunks]), np.concatenate([ch.areas for ch in self.chunks]))

    def gradients(self) -> list[tuple[np.ndarray, np.ndarray]]:
        """Per structure (d volume / d atoms, d area / d atoms), each (n_atoms, 4)."""
        out = []
        for ch in self.chunks:
            gv = ch.gvol.numpy().reshape(-1, 4)
            ga = ch.garea.numpy().reshape(-1, 4)
            for b in range(ch.hi - ch.lo):
                lo, hi = int(ch.atom_off[b]), int(ch.atom_off[b + 1])
                out.append((gv[lo:hi], ga[lo:hi]))
        return out

    def close(self) -> None:
        for c in self.ctxs:
            c.close()


class AtomsPipeline:
    """Volume, area and their atom derivatives of every structure of an ensemble, starting from
    the atoms: per step each structure's grid is built (buildGrid), its atoms jittered with the
    process-wide generator in structure order (as one ConnollySurface::build per structure would),
    its SES patches built on the host, and the chunks ray cast, triangulated and differentiated
    on two contexts as in PipelinedBatches.  The host work overlaps the device work: structures are
    built on a pool of host threads (one single-threaded patch build per structure), each chunk's
    patch sets are exported straight into its pinned buffers, and a chunk goes to the GPU as soon
    as it is complete while the pool builds the next."""

    def __init__(self, atoms: list, probe: float = 1.4, scale: float = 2.0, perfil: float = 80.0, n_chunks: int = 8,
                 device: int = 0, precision: str = "mixed", tuning: list[int] | None = None, threads: int = 0):
        import os
        if not atoms:
            raise ValueError("empty ensemble")
        self.atoms = [np.ascontiguousarray(a, np.float64) for a in atoms]
        self.probe, self.scale, self.perfil = probe, scale, perfil
        self.bounds = chunk_bounds(len(atoms), n_chunks)
        self.prec = S.PRECISIONS[precision]
        self.flags = N.STATUS | N.ACCURATE_TRIANGULATION | N.GRAD
        self.threads = threads or (os.cpu_count() or 1)
        self.ctxs = [S.Context(device), S.Context(device)]
        self._upload_lock = threading.Lock()
        if tuning is not None:
            p = np.ascontiguousarray(tuning, np.int32)
            for c in self.ctxs:
                N.check(N.lib().nsg_set_tuning(c.handle, N.ptr(p), len(p)), "set tuning")
        self._pinned: dict = {}
        self.h2d_bytes = 0
        self.d2h_bytes = 0
        self.volumes = np.zeros(len(atoms))
        self.areas = np.zeros(len(atoms))

    def _pin(self, key, nbytes: int) -> torch.Tensor:
        t = self._pinned.get(key)
        if t is None or t.numel() < nbytes:
            t = torch.empty(max(nbytes, 64), dtype=torch.uint8, pin_memory=True)
            self._pinned[key] = t
        return t

    def _build_one(self, b: int, jittered: np.ndarray):
        h = ctypes.c_void_p()
        rc = N.lib().nsg_ses_build(N.ptr(jittered), len(jittered), self.probe, 1, ctypes.byref(h))
        if rc not in (N.NSG_OK, -8):
            N.check(rc, "SES patch construction")
        n = ctypes.c_int64()
        npool = ctypes.c_int64()
        N.check(N.lib().nsg_patchset_info(h, ctypes.byref(n), ctypes.byref(npool), None), "patchset_info")
        return h, n.value, npool.value

    def _host_chunk(self, ci: int, pool, grids, jittered):
        """Builds chunk ci's patch sets on the pool and exports them into its pinned buffers."""
        lo, hi = int(self.bounds[ci]), int(self.bounds[ci + 1])
        built = list(pool.map(lambda b: self._build_one(b, jittered[b]), range(lo, hi)))
        m = hi - lo
        patch_off = np.zeros(m + 1, np.int64)
        pool_off = np.zeros(m + 1, np.int64)
        atom_off = np.zeros(m + 1, np.int64)
        patch_off[1:] = np.cumsum([x[1] for x in built])
        pool_off[1:] = np.cumsum([x[2] for x in built])
        atom_off[1:] = np.cumsum([len(jittered[b]) for b in range(lo, hi)])
        npat, npool, nat = int(patch_off[-1]), int(pool_off[-1]), int(atom_off[-1])
        pin = {"f64": self._pin((ci, "f64"), npat * 160), "i32": self._pin((ci, "i32"), npat * 16),
               "pool": self._pin((ci, "pool"), max(npool, 1) * 32), "flag": self._pin((ci, "flag"), max(npool, 1)),
               "atoms": self._pin((ci, "atoms"), nat * 32), "patch_atoms": self._pin((ci, "pa"), npat * 12),
               "gvol": self._pin((ci, "gvol"), nat * 32), "garea": self._pin((ci, "garea"), nat * 32)}
        L = N.lib()

        def export(q: int) -> None:
            h = built[q][0]
            try:
                po, qo, ao = int(patch_off[q]), int(pool_off[q]), int(atom_off[q])
                N.check(L.nsg_patchset_export(h, pin["f64"].data_ptr() + po * 160, pin["i32"].data_ptr() + po * 16,
                                              pin["pool"].data_ptr() + qo * 32, pin["flag"].data_ptr() + qo),
                        "patchset_export")
                N.check(L.nsg_patchset_atoms(h, pin["patch_atoms"].data_ptr() + po * 12), "patchset_atoms")
                a = jittered[lo + q]
                ctypes.memmove(pin["atoms"].data_ptr() + ao * 32, a.ctypes.data, a.nbytes)
            finally:
                L.nsg_patchset_free(h)

        list(pool.map(export, range(m)))
        if npool == 0:
            pin["flag"].zero_()
        g = (N.NsGrid * m)(*grids[lo:hi])
        return dict(lo=lo, hi=hi, patch_off=patch_off, pool_off=pool_off, atom_off=atom_off, pin=pin, grids=g,
                    h2d=npat * 188 + max(npool, 1) * 33 + nat * 32, d2h=16 * m + 64 * nat)

    def _gpu_chunk(self, c, ch) -> None:
        L = N.lib()
        pin = ch["pin"]
        m = ch["hi"] - ch["lo"]
        with self._upload_lock:
            N.check(L.nsg_set_batch(c, m, ch["grids"]), "set_batch")
            N.check(L.nsg_upload_batch(c, N.ptr(ch["patch_off"]), pin["f64"].data_ptr(), pin["i32"].data_ptr(),
                                       N.ptr(ch["pool_off"]), pin["pool"].data_ptr(), pin["flag"].data_ptr(),
                                       self.probe), "upload_batch")
            N.check(L.nsg_upload_atoms(c, N.ptr(ch["atom_off"]), pin["atoms"].data_ptr(), pin["patch_atoms"].data_ptr()),
                    "upload atoms")
        v = ctypes.c_double()
        N.check(L.nsg_raycast(c, self.flags, self.prec, ctypes.byref(v)), "raycast")
        a = ctypes.c_double()
        nv = ctypes.c_int64()
        nt = ctypes.c_int64()
        N.check(L.nsg_triangulate(c, ctypes.byref(a), ctypes.byref(nv), ctypes.byref(nt)), "triangulate")
        rc = L.nsg_atom_grads(c, pin["gvol"].data_ptr(), pin["garea"].data_ptr())
        if rc not in (N.NSG_OK, -8):
            N.check(rc, "atom gradients")
        vols = np.zeros(m)
        areas = np.zeros(m)
        N.check(L.nsg_batch_results(c, N.ptr(vols), N.ptr(areas)), "batch results")
        self.volumes[ch["lo"]:ch["hi"]] = vols
        self.areas[ch["lo"]:ch["hi"]] = areas

    def run(self) -> tuple[np.ndarray, np.ndarray]:
        """One pass over the ensemble from its atoms; returns the per-structure volumes and areas."""
        import queue
        from concurrent.futures import ThreadPoolExecutor
        L = N.lib()
        # grids from the loaded atoms, then the jitter in structure order (process-wide generator)
        grids = []
        jittered = []
        S.reset_seed()
        for a in self.atoms:
            g = N.NsGrid()
            N.check(L.nsg_grid_build(N.ptr(a), len(a), self.scale, self.perfil, ctypes.byref(g)), "buildGrid")
            grids.append(g)
            j = a.copy()
            N.check(L.nsg_jitter_atoms(N.ptr(j), len(j), S.RAND_DISPLACEMENT, ctypes.byref(S._seed)), "jitter")
            jittered.append(j)
        ready: "queue.Queue" = queue.Queue()
        errors: list[BaseException] = []
        n_chunks = len(self.bounds) - 1
        h2d = [0]
        d2h = [0]

        def producer() -> None:
            try:
                with ThreadPoolExecutor(self.threads) as pool:
                    for ci in range(n_chunks):
                        ch = self._host_chunk(ci, pool, grids, jittered)
                        h2d[0] += ch["h2d"]
                        d2h[0] += ch["d2h"]
                        ready.put(ch)
            except BaseException as e:
                errors.append(e)
            finally:
                for _ in range(2):
                    ready.put(None)

        def worker(w: int) -> None:
            try:
                while True:
                    ch = ready.get()
                    if ch is None:
                        return
                    self._gpu_chunk(self.ctxs[w].handle, ch)
            except BaseException as e:
                errors.append(e)

        threads = [threading.Thread(target=producer)] + [threading.Thread(target=worker, args=(w,)) for w in range(2)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        if errors:
            raise errors[0]
        self.h2d_bytes, self.d2h_bytes = h2d[0], d2h[0]
        return self.volumes.copy(), self.areas.copy()

    def close(self) -> None:
        for c in self.ctxs:
            c.close()
