"""Pipelined batches: host-resident ensembles with transfers overlapped with compute.

An ensemble whose patch sets live in host memory spends a large share of its time in the
host-to-device copy (about 0.9 GB per 1,000 structures of ~4,000 atoms).  ``PipelinedBatches``
splits the ensemble into chunks, keeps every chunk's inputs in pinned host buffers, and drives two
libnsgpu contexts (two CUDA streams) from two host threads.  While one context computes a chunk,
the other copies the next, so the copy engines and the SMs work at the same time.  Each chunk is
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
                 tuning: list[int] | None = None):
        if not surfaces:
            raise ValueError("empty ensemble")
        bounds = chunk_bounds(len(surfaces), n_chunks)
        n_chunks = len(bounds) - 1
        self.chunks = [_Chunk(surfaces, int(bounds[i]), int(bounds[i + 1])) for i in range(n_chunks)]
        self.n = len(surfaces)
        self.prec = S.PRECISIONS[precision]
        s0 = surfaces[0]
        self.flags = (N.STATUS if s0.delphi.buildStatus else 0) | N.ACCURATE_TRIANGULATION | N.GRAD
        self.ctxs = [S.Context(device), S.Context(device)]
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

        def worker(w: int) -> None:
            try:
                for ch in self.chunks[w::2]:
                    self._run_chunk(self.ctxs[w].handle, ch)
            except BaseException as e:  # reported after both workers joined
                errors.append(e)

        threads = [threading.Thread(target=worker, args=(w,)) for w in range(2)]
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
