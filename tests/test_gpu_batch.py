"""Batched pipeline (nsg_set_batch / nsg_upload_batch): every structure of a batch must give the
same result as the same structure run alone.  Insideness bits, vertex and triangle counts equal;
volumes and areas within 1e-12 relative (the per-structure sums are taken in another order).
The single-structure path is itself checked against the oracle in test_gpu_parity.py.
"""
import numpy as np
import pytest

import nanoshaper_b200 as nb
from nanoshaper_b200 import generator

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def _structures(specs):
    out = []
    nb.reset_seed()
    for n_atoms, seed, scale, perfil in specs:
        atoms = generator.rsa_globule(n_atoms, seed)
        cf = nb.ConfigFile()
        cf.add("Surface", "ses")
        cf.add("Probe_Radius", 1.4)
        cf.add("Accurate_Triangulation", True)
        cf.add("Triangulation", True)
        ds = nb.DelPhiShared(atoms, scale, perfil)
        s = nb.surfaceFactory().create(cf, ds)
        s.build()
        out.append(s)
    return out


SPECS = [(60, 11, 2.0, 80.0), (327, 1, 2.0, 80.0), (150, 5, 2.5, 70.0), (800, 7, 2.0, 80.0), (40, 2, 3.0, 60.0),
         (500, 9, 2.0, 80.0)]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_matches_single(precision, native_lib):
    surfs = _structures(SPECS)
    vols, areas, bits, nv, nt = [], [], [], 0, 0
    for s in surfs:
        s.precision = precision
        vols.append(s.getSurf(True, False, 0.0))
        areas.append(s.triangulateSurface())
        bits.append(s.insideness.copy())
        nv += len(s.vertices)
        nt += len(s.triangles)
        s.ctx.close()
        s.ctx = None
    batch = nb.SurfaceBatch(surfs, precision=precision)
    bvol = batch.getSurf(download=True)
    barea = batch.triangulateSurface()
    for b in range(len(surfs)):
        assert np.array_equal(batch.insideness[b], bits[b]), f"structure {b}: insideness bits differ"
        assert abs(bvol[b] - vols[b]) <= RTOL * abs(vols[b]), f"structure {b}: volume {bvol[b]} vs {vols[b]}"
        assert abs(barea[b] - areas[b]) <= RTOL * abs(areas[b]), f"structure {b}: area {barea[b]} vs {areas[b]}"
    assert batch.n_vertices == nv
    assert batch.n_triangles == nt
    # a second pass over the same batch gives the same numbers
    bvol2 = batch.getSurf()
    barea2 = batch.triangulateSurface()
    assert np.array_equal(bvol, bvol2) and np.array_equal(barea, barea2)
    batch.close()


def test_batch_gradients_match_single(native_lib):
    """Atom derivatives of volume and area from the batched device chain rule equal those of each
    structure run alone through the host chain rule (1e-10 relative: atomics sum in any order)."""
    surfs = _structures(SPECS[:4])
    single = []
    for s in surfs:
        s.getSurf(True, False, 0.0, download=False, grad=True)
        s.triangulateSurface(download=False)
        single.append((s.gradients(1.0, 0.0), s.gradients(0.0, 1.0)))
        s.ctx.close()
        s.ctx = None
    batch = nb.SurfaceBatch(surfs)
    batch.getSurf(grad=True)
    batch.triangulateSurface()
    for b, (gv, ga) in enumerate(batch.atom_gradients()):
        sv, sa = single[b]
        assert np.abs(gv - sv).max() <= 1e-10 * np.abs(sv).max(), f"structure {b}: volume gradient"
        assert np.abs(ga - sa).max() <= 1e-10 * np.abs(sa).max(), f"structure {b}: area gradient"
    batch.close()


def test_autotune_keeps_results(native_lib):
    """The autotuner only changes launch shapes: volumes and areas are unchanged."""
    surfs = _structures(SPECS[:3])
    batch = nb.SurfaceBatch(surfs, precision="mixed")
    v0 = batch.getSurf().copy()
    a0 = batch.triangulateSurface().copy()
    shape, ms = batch.autotune(reps=1)
    assert 64 <= shape[0] <= 256 and 1 <= shape[1] <= 64 and 32 <= shape[2] <= 1024 and ms > 0
    v1 = batch.getSurf()
    a1 = batch.triangulateSurface()
    assert np.array_equal(v0, v1) and np.array_equal(a0, a1)
    batch.close()


def test_pipelined_batches_match_one_batch(native_lib):
    """Chunked processing on two and on three contexts, with overlapped copies, gives the same
    per-structure volumes and areas as one batch, and the same atom derivatives (1e-10 relative)."""
    from nanoshaper_b200.pipelined import PipelinedBatches
    surfs = _structures(SPECS)
    batch = nb.SurfaceBatch(surfs, precision="mixed")
    v = batch.getSurf(grad=True).copy()
    a = batch.triangulateSurface().copy()
    g = batch.atom_gradients()
    batch.close()
    for n_chunks, n_contexts in ((3, 2), (4, 3)):
        runner = PipelinedBatches(surfs, n_chunks=n_chunks, precision="mixed", n_contexts=n_contexts)
        for _ in range(2):
            pv, pa = runner.run()
            assert np.array_equal(pv, v) and np.array_equal(pa, a)
        for (gv, ga), (rv, ra) in zip(g, runner.gradients()):
            assert np.abs(gv - rv).max() <= 1e-10 * np.abs(gv).max()
            assert np.abs(ga - ra).max() <= 1e-10 * np.abs(ga).max()
        runner.close()


def test_atoms_pipeline_matches_batch(native_lib):
    """AtomsPipeline (grids, jitter and patch builds on host threads, overlapped with the device)
    gives the per-structure volumes and areas of the same ensemble built structure by structure
    and run as one batch."""
    from nanoshaper_b200.pipelined import AtomsPipeline
    atoms = generator.ensemble(2, 4, 300, 900, 0.3, 3)
    nb.reset_seed()
    surfs = []
    for a in atoms:
        ds = nb.DelPhiShared(a, 2.0, 80.0)
        cf = nb.ConfigFile(text="Surface = ses\nProbe_Radius = 1.4\nAccurate_Triangulation = true\n"
                                "Gpu_Precision = mixed\n")
        sf = nb.surfaceFactory().create(cf, ds)
        sf.build()
        surfs.append(sf)
    batch = nb.SurfaceBatch(surfs, precision="mixed")
    vol = batch.getSurf(grad=True)
    area = batch.triangulateSurface()
    batch.close()
    ap = AtomsPipeline(atoms, n_chunks=3, precision="mixed", threads=4)
    for _ in range(2):
        v2, a2 = ap.run()
        np.testing.assert_allclose(v2, vol, rtol=1e-12, atol=0)
        np.testing.assert_allclose(a2, area, rtol=1e-12, atol=0)
    ap.close()
