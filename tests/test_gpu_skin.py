"""GPU parity of the skin surface (mixed cells, ray-quadric tests) against the oracle.

* The reference's 1crn skin fixture (its .prm through ConfigFile, s = 0.45, scale 2, perfil 90) in
  double precision: every ray's hits, status map, insideness bits, vertices, triangles, volume and
  area.
* The skin configuration of the benchmark set: 10,000 atoms, s = 0.45, grid scale 3.0, perfil 80,
  marching cubes; in double precision (hits, maps, mesh, volume and area as above) and in mixed
  precision (FP32 ray-quadric and plane tests with FP64 refinement): every ray's hit count equal,
  hits within 1e-5 A, status map and insideness bits equal except at nodes whose oracle hit lies
  within 1e-6 A of the node (counted).
* The reference's 6xm4 skin fixture (48,519 atoms, scale 2, perfil 90, Build_epsilon_maps on) in
  double precision: every ray's hits over all six ray sets (the epsilon map's node rays included),
  status map, insideness bits, epsilon and ideb maps, and the volume averaged over the six sets.
"""
import gzip
import shutil
from pathlib import Path

import numpy as np
import pytest

import nanoshaper_b200 as nb
from nanoshaper_b200 import generator

pytestmark = pytest.mark.gpu

FIXTURES = Path(__file__).resolve().parent / "golden" / "fixtures"
HIT_TOL = 1e-12


def _ray_len(g, s):
    return ((g.nx - 1) * g.side, (g.nx - 1) * g.side, (g.nz - 1) * g.side, (g.ny - 1) * g.side,
            (g.nz - 1) * g.side, (g.ny - 1) * g.side)[s]


def _compare_hits(surf, ref, oracle_mod, angstrom=False, sets=range(4)):
    worst = 0.0
    g = surf.delphi.grid
    for s in sets:
        cnt_g, val_g = surf.hits(s)
        cnt_o, val_o = oracle_mod.ray_hits(ref, s)
        if not np.array_equal(cnt_g, cnt_o):
            bad = np.argwhere(cnt_g != cnt_o)[:4]
            og = np.concatenate([[0], np.cumsum(cnt_g.ravel())])
            oo = np.concatenate([[0], np.cumsum(cnt_o.ravel())])
            det = []
            for n, m in bad:
                r = n * cnt_g.shape[1] + m
                det.append((int(n), int(m), val_g[og[r]:og[r + 1]].tolist(), val_o[oo[r]:oo[r + 1]].tolist()))
            raise AssertionError(f"ray set {s}: {(cnt_g != cnt_o).sum()} rays with other hit counts: {det}")
        if len(val_o):
            d = np.abs(val_g - val_o)
            k = int(d.argmax())
            if d[k] > HIT_TOL:
                print(f"ray set {s}: largest hit difference {d[k]:.3e} at hit {k}: {val_g[k]!r} vs {val_o[k]!r}")
            worst = max(worst, float(d[k]) * _ray_len(g, s) if angstrom else float(d[k]))
    return worst


def _skin(atoms, scale, perfil, precision="fp64"):
    nb.reset_seed()
    ds = nb.DelPhiShared(atoms, scale, perfil)
    cf = nb.ConfigFile(text="Surface = skin\nSkin_Surface_Parameter = 0.45\nAccurate_Triangulation = true\n"
                            f"Triangulation = true\nGpu_Precision = {precision}\n")
    surf = nb.surfaceFactory().create(cf, ds)
    surf.build()
    return ds, surf


def test_skin_fixture_1crn_fp64(native_lib, oracle_mod):
    import compare
    cf = nb.ConfigFile(FIXTURES / "1crn_skin_conf.prm")
    nb.reset_seed()
    ns = nb.NanoShaper(config=cf)
    ns.buildAnalyticalSurface()
    surf, ds = ns.surf, ns.ds
    surf.getSurf(True, False, 0.0, keep_hits=True)
    surf.triangulateSurface()
    ref = oracle_mod.run(ds.grid, surf.patches, flags=oracle_mod.STATUS | oracle_mod.ACCURATE_TRIANGULATION |
                         oracle_mod.TRIANGULATE | oracle_mod.NORMALS)
    worst = _compare_hits(surf, ref, oracle_mod)
    assert worst <= HIT_TOL
    figs = compare.compare_surface(surf, ds, ref)
    nrm = surf.vertexNormals()
    dn = float(np.abs(nrm - ref.normals).max() / max(np.abs(ref.normals).max(), 1.0))
    assert dn <= 1e-9, f"vertex normals differ by {dn} (relative)"
    print(f"1crn skin ({surf.patches.n} cells, grid {ds.nx}^3): worst hit diff {worst:.2e}, normals {dn:.1e}, {figs}")


@pytest.fixture(scope="module")
def skin_10k():
    return generator.rsa_globule(10000, 2)


def test_skin_10k_fp64_matches_oracle(skin_10k, native_lib, oracle_mod):
    import compare
    ds, surf = _skin(skin_10k, 3.0, 80.0)
    surf.getSurf(True, True, 10.0, keep_hits=True)
    surf.triangulateSurface()
    ref = oracle_mod.run(ds.grid, surf.patches, cav_vol=10.0, threads=8)
    worst = _compare_hits(surf, ref, oracle_mod)
    assert worst <= HIT_TOL
    figs = compare.compare_surface(surf, ds, ref)
    print(f"skin 10k fp64 ({surf.patches.n} cells, grid {ds.nx}^3): worst hit diff {worst:.2e}, {figs}")


def test_skin_10k_mixed_matches_oracle(skin_10k, native_lib, oracle_mod):
    import compare
    ds, surf = _skin(skin_10k, 3.0, 80.0, precision="mixed")
    surf.getSurf(True, True, 10.0, keep_hits=True)
    surf.triangulateSurface()
    ref = oracle_mod.run(ds.grid, surf.patches, cav_vol=10.0, threads=8)
    worst = _compare_hits(surf, ref, oracle_mod, angstrom=True)
    assert worst <= 1e-5, f"max hit error {worst} A"
    figs = compare.compare_surface(surf, ds, ref, rel_tol=1e-9, vert_tol=1e-5)
    print(f"skin 10k mixed: max hit error {worst:.3e} A, {figs}")


def test_skin_fixture_6xm4_maps(native_lib, oracle_mod, tmp_path):
    import compare
    with gzip.open(FIXTURES / "6xm4.xyzr.gz", "rb") as f, open(tmp_path / "6xm4.xyzr", "wb") as g:
        shutil.copyfileobj(f, g)
    shutil.copyfile(FIXTURES / "6xm4_skin_conf.prm", tmp_path / "6xm4_skin_conf.prm")
    cf = nb.ConfigFile(tmp_path / "6xm4_skin_conf.prm")
    nb.reset_seed()
    ns = nb.NanoShaper(config=cf)
    assert len(ns.ds.atoms) == 48519
    ns.buildAnalyticalSurface()
    surf, ds = ns.surf, ns.ds
    # the fixture builds the epsilon map: six ray sets, the volume averaged over all six
    assert ds.buildEpsMap
    vol = surf.getSurf(True, False, 0.0, keep_hits=True)
    ref = oracle_mod.run(ds.grid, surf.patches, threads=8,
                         flags=oracle_mod.STATUS | oracle_mod.ACCURATE_TRIANGULATION | oracle_mod.EPSMAP)
    worst = _compare_hits(surf, ref, oracle_mod, sets=range(6))
    assert worst <= HIT_TOL
    n_mis, n_near = compare.near_node_status(ds.status, ref, ds.grid)
    assert n_mis == n_near
    assert np.array_equal(surf.insideness, ref.bits)
    e_mis, e_near = compare.near_threshold_eps(ds.epsmap, ref, ds.grid)
    assert e_mis == 0, f"{e_mis} epsilon-map entries differ ({e_near} near a threshold)"
    assert np.array_equal(ds.idebmap, ref.idebmap)
    assert abs(vol - ref.volume) <= 1e-12 * abs(ref.volume), f"volume {vol} vs {ref.volume}"
    print(f"6xm4 skin ({surf.patches.n} cells, grid {ds.nx}^3): status mismatches {n_mis} (near-node {n_near}), "
          f"worst hit diff {worst:.2e}, epsilon map exact")
