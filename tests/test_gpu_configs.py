"""GPU parity at the benchmark configurations and on the reference's own fixture.

* The reference's 1crn SES fixture (tests/1crn_ses of the reference: 327 atoms, Grid_scale 2.0,
  Grid_perfil 90, Cavity_Detection_Filling false), configured by parsing its .prm through
  ConfigFile and run through the NanoShaper facade: every ray's hits, the status map, the
  insideness bits, the vertices, the triangles, volume and area against the oracle.
* The large SES structure (100,000 atoms, probe 1.4, scale 4.0, perfil 70, 1049^3 nodes) in double
  precision with cavity detection and filling: status map (cavity labels included), insideness
  bits, cavity count, sizes and fill flags bit-exact against the oracle except at grid nodes whose
  oracle hit lies within 1e-6 A of the node (counted and printed); volume within 1e-12 relative.
  The oracle fills the status rows on its threads but sums the volume in the reference's serial
  ray order.
* Eight seeded structures of the 512-structure conformer ensemble, taken out of the full batch
  (every structure on its own grid, one launch per kernel for all 512): per-ray hits, insideness
  bits, volume and area against the oracle, in double precision and in mixed precision (hits
  within 1e-5 A, same hit counts and bits).
"""
import os
from pathlib import Path

import numpy as np
import pytest

import nanoshaper_b200 as nb
from nanoshaper_b200 import generator

pytestmark = pytest.mark.gpu

FIXTURES = Path(__file__).resolve().parent / "golden" / "fixtures"
HIT_TOL = 1e-12     # double precision, ray-parameter units
MIXED_HIT_A = 1e-5  # mixed precision, Angstrom


def _ray_len(g, s):
    return ((g.nx - 1) * g.side, (g.nx - 1) * g.side, (g.nz - 1) * g.side, (g.ny - 1) * g.side)[s]


def test_reference_fixture_1crn_ses(native_lib, oracle_mod):
    import compare
    cf = nb.ConfigFile(FIXTURES / "1crn_ses_conf.prm")
    nb.reset_seed()
    ns = nb.NanoShaper(config=cf)
    assert ns.buildAnalyticalSurface()
    fill = cf.read("Cavity_Detection_Filling", False, bool)
    cav_vol = cf.read("Conditional_Volume_Filling_Value", 11.4, float)
    surf, ds = ns.surf, ns.ds
    surf.getSurf(True, fill, cav_vol, keep_hits=True)
    surf.triangulateSurface()
    assert surf.computeNormals  # the fixture asks for Compute_Vertex_Normals
    ref = oracle_mod.run(ds.grid, surf.patches, cav_vol=cav_vol if fill else 0.0,
                         flags=oracle_mod.STATUS | oracle_mod.ACCURATE_TRIANGULATION | oracle_mod.TRIANGULATE |
                         oracle_mod.NORMALS | (oracle_mod.CAVITIES if fill else 0))
    worst = 0.0
    for s in range(4):
        cnt_g, val_g = surf.hits(s)
        cnt_o, val_o = oracle_mod.ray_hits(ref, s)
        assert np.array_equal(cnt_g, cnt_o), f"ray set {s}: {(cnt_g != cnt_o).sum()} rays with other hit counts"
        if len(val_o):
            worst = max(worst, float(np.abs(val_g - val_o).max()))
    assert worst <= HIT_TOL
    figs = compare.compare_surface(surf, ds, ref)
    # analytic vertex normals (patch normal at every analytic vertex, triangle average elsewhere)
    nrm = surf.vertexNormals()
    dn = float(np.abs(nrm - ref.normals).max())
    assert dn <= 1e-9, f"vertex normals differ by {dn}"
    print(f"1crn ses (grid {ds.nx}x{ds.ny}x{ds.nz}, {surf.patches.n} patches): worst hit diff {worst:.2e}, "
          f"normals within {dn:.1e}, {figs}")


def test_ses_100k_maps_match_oracle(native_lib, oracle_mod):
    import compare
    atoms = generator.rsa_globule(100000, 3)
    nb.reset_seed()
    cf = nb.ConfigFile(text="Surface = ses\nProbe_Radius = 1.4\nAccurate_Triangulation = true\n")
    ds = nb.DelPhiShared(atoms, 4.0, 70.0)
    surf = nb.surfaceFactory().create(cf, ds)
    surf.build()
    vol = surf.getSurf(True, True, 10.0)
    ref = oracle_mod.run(ds.grid, surf.patches, flags=oracle_mod.STATUS | oracle_mod.ACCURATE_TRIANGULATION |
                         oracle_mod.CAVITIES, cav_vol=10.0, threads=os.cpu_count() or 1)
    n_mis, n_near = compare.near_node_status(ds.status, ref, ds.grid)
    bits_mis = int(np.unpackbits((surf.insideness ^ ref.bits).view(np.uint8)).sum())
    print(f"ses_100k grid {ds.nx}^3, {surf.patches.n} patches: status mismatches {n_mis} (near-node {n_near}), "
          f"insideness bit mismatches {bits_mis}, cavities {surf.ncav}/{ref.ncav}, "
          f"volume {vol:.9f} vs {ref.volume:.9f}")
    assert n_mis == n_near, f"{n_mis - n_near} status nodes differ away from any hit"
    assert bits_mis == 0
    assert surf.ncav == ref.ncav
    np.testing.assert_array_equal(np.array(ds.cavitiesSize), ref.cav_size)
    np.testing.assert_array_equal(np.array(ds.cavitiesFlag, np.int32), ref.cav_filled)
    assert abs(vol - ref.volume) <= 1e-12 * abs(ref.volume)


@pytest.fixture(scope="module")
def ensemble_512():
    """The benchmark's conformer ensemble (32 globules x 16 perturbations) and its patch sets."""
    atoms = generator.ensemble(32, 16, 500, 8000, 0.3, 5)
    nb.reset_seed()
    surfs = []
    for a in atoms:
        ds = nb.DelPhiShared(a, 2.0, 80.0)
        cf = nb.ConfigFile(text="Surface = ses\nProbe_Radius = 1.4\nAccurate_Triangulation = true\n"
                                "Triangulation = true\n")
        sf = nb.surfaceFactory().create(cf, ds)
        sf.build()
        surfs.append(sf)
    return surfs


def _batch_hits(batch, surfs, picks):
    """Per picked structure and ray set: (counts (na, nb), sorted hits) out of the batch."""
    from nanoshaper_b200 import _native as N
    import ctypes
    c = batch._context().handle
    out = {b: [None] * 4 for b in picks}
    for s in range(4):
        dims = []
        for sf in surfs:
            g = sf.delphi.grid
            dims.append(((g.ny, g.nz), (g.ny, g.nz), (g.nx, g.ny), (g.nx, g.nz))[s])
        nrays = np.array([nb_ * na for nb_, na in dims], np.int64)
        base = np.concatenate([[0], np.cumsum(nrays)])
        counts = np.zeros(int(base[-1]), np.int32)
        total = N.lib().nsg_download_hits(c, s, N.ptr(counts), None, 0)
        assert total >= 0
        vals = np.zeros(int(counts.sum()))
        N.check(N.lib().nsg_download_hits(c, s, N.ptr(counts), N.ptr(vals), len(vals)), "download hits")
        hoff = np.concatenate([[0], np.cumsum(counts.astype(np.int64))])
        for b in picks:
            nb_, na = dims[b]
            cnt = counts[base[b]:base[b + 1]]
            out[b][s] = (cnt.reshape(na, nb_), vals[hoff[base[b]]:hoff[base[b + 1]]])
    return out


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_ensemble_structures_match_oracle(precision, ensemble_512, native_lib, oracle_mod):
    from nanoshaper_b200 import _native as N
    import ctypes
    surfs = ensemble_512
    picks = sorted(np.random.default_rng(2024).choice(len(surfs), 8, replace=False).tolist())
    batch = nb.SurfaceBatch(surfs, precision=precision)
    batch.upload()
    c = batch._context().handle
    vol = ctypes.c_double()
    N.check(N.lib().nsg_raycast(c, N.STATUS | N.ACCURATE_TRIANGULATION | N.KEEP_HITS, 0 if precision == "fp64" else 1,
                                ctypes.byref(vol)), "raycast")
    vols = np.zeros(len(surfs))
    N.check(N.lib().nsg_batch_results(c, N.ptr(vols), None), "results")
    words = [((s.delphi.grid.nx + 31) >> 5) * s.delphi.grid.ny * s.delphi.grid.nz for s in surfs]
    bits = np.empty(sum(words), np.uint32)
    N.check(N.lib().nsg_download_insideness(c, N.ptr(bits)), "download insideness")
    bits = np.split(bits, np.cumsum(words)[:-1])
    hits = _batch_hits(batch, surfs, picks)
    areas = batch.triangulateSurface()
    batch.close()
    worst = 0.0
    for b in picks:
        sf = surfs[b]
        g = sf.delphi.grid
        ref = oracle_mod.run(g, sf.patches)
        for s in range(4):
            cnt_g, val_g = hits[b][s]
            cnt_o, val_o = oracle_mod.ray_hits(ref, s)
            assert np.array_equal(cnt_g, cnt_o), f"structure {b} set {s}: {(cnt_g != cnt_o).sum()} rays differ"
            if len(val_o):
                d = float(np.abs(val_g - val_o).max())
                worst = max(worst, d * _ray_len(g, s) if precision == "mixed" else d)
        assert np.array_equal(bits[b], ref.bits), f"structure {b}: insideness bits differ"
        tol = 1e-12 if precision == "fp64" else 1e-9
        assert abs(vols[b] - ref.volume) <= tol * abs(ref.volume), f"structure {b}: volume {vols[b]} vs {ref.volume}"
        assert abs(areas[b] - ref.area) <= tol * abs(ref.area), f"structure {b}: area {areas[b]} vs {ref.area}"
    assert worst <= (HIT_TOL if precision == "fp64" else MIXED_HIT_A)
    print(f"ensemble_512 {precision}: structures {picks} match the oracle; worst hit diff {worst:.3e}")
