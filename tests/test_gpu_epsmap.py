"""GPU parity of the epsilon and ideb maps, the boundary grid points and their projection.

* The reference's 1crn SES fixture (its .prm through ConfigFile) with Build_epsilon_maps and
  Project_boundary_grid_points switched on, cavity detection and filling at 30 A^3, in double
  precision: the epsilon map (every edge code), the ideb map, the boundary grid point list, types
  and projection flags equal the oracle's; projections within 1e-12 A; volume (now over six ray
  sets) within 1e-12 relative.  The fixture's Max_ses_patches_auxiliary_grid_size = 1000 makes
  the auxiliary grid the DelPhi grid itself.
* A 2,000-atom SES at scale 2.0 with the default auxiliary grid (50 cells per axis, coarser than
  the DelPhi grid), in double and mixed precision; in mixed precision edge codes may differ only
  where an oracle interval end lies within 1e-6 A of the edge's threshold (counted).
"""
from pathlib import Path

import numpy as np
import pytest

import nanoshaper_b200 as nb
from nanoshaper_b200 import generator

pytestmark = pytest.mark.gpu

FIXTURES = Path(__file__).resolve().parent / "golden" / "fixtures"


def _check(surf, ds, ref, exact=True):
    import compare
    n_mis, n_near = compare.near_threshold_eps(ds.epsmap, ref, ds.grid)
    if exact:
        assert n_mis == 0, f"{n_mis} epsilon-map entries differ ({n_near} near a threshold)"
    else:
        assert n_mis == n_near, f"{n_mis - n_near} epsilon-map entries differ away from any threshold"
    n_st, n_st_near = compare.near_node_status(ds.status, ref, ds.grid)
    assert n_st == n_st_near
    ideb_mis = int((ds.idebmap != ref.idebmap).sum())
    assert ideb_mis <= n_st, f"ideb map: {ideb_mis} nodes differ"
    out = {"eps_mismatch": n_mis, "eps_near": n_near, "ideb_mismatch": ideb_mis, "nbgp": ds.nbgp}
    if n_mis == 0:
        np.testing.assert_array_equal(ds.ibgp, ref.ibgp)
        np.testing.assert_array_equal(ds.bgp_type, ref.bgp_type)
        np.testing.assert_array_equal(ds.bgp_flag, ref.bgp_flag)
        d = float(np.abs(ds.scspos - ref.scspos).max()) if ds.nbgp else 0.0
        assert d <= 1e-12, f"projections differ by {d} A"
        assert not ds.scsnor.any() and not ref.scsnor.any()
        out["proj_max_abs"] = d
    out["unprojected"] = int((ds.bgp_flag != 0).sum())
    out["volume_rel"] = abs(surf.volume - ref.volume) / abs(ref.volume)
    return out


def test_epsmap_fixture_1crn_fp64(native_lib, oracle_mod):
    cf = nb.ConfigFile(FIXTURES / "1crn_ses_conf.prm")
    cf.add("Build_epsilon_maps", True)
    cf.add("Project_boundary_grid_points", True)
    nb.reset_seed()
    ns = nb.NanoShaper(config=cf)
    assert ns.ds.buildEpsMap
    ns.buildAnalyticalSurface()
    surf, ds = ns.surf, ns.ds
    assert surf.auxGridDim == 1000
    surf.getSurf(True, True, 30.0)
    ref = oracle_mod.run(ds.grid, surf.patches, cav_vol=30.0, aux_grid_dim=1000,
                         flags=oracle_mod.STATUS | oracle_mod.ACCURATE_TRIANGULATION | oracle_mod.CAVITIES |
                         oracle_mod.EPSMAP | oracle_mod.BGP)
    figs = _check(surf, ds, ref)
    assert figs["volume_rel"] <= 1e-12
    assert ds.nbgp > 0 and (ds.bgp_type == 1).all()
    assert int((ds.epsmap == 5).sum()) > 0
    print(f"1crn eps (grid {ds.nx}^3, cavities {surf.ncav}, filled {sum(ds.cavitiesFlag)}): {figs}")


@pytest.fixture(scope="module")
def atoms_2000():
    return generator.rsa_globule(2000, 5)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_epsmap_2000_matches_oracle(precision, atoms_2000, native_lib, oracle_mod):
    nb.reset_seed()
    ds = nb.DelPhiShared(atoms_2000, 2.0, 80.0, build_eps_map=True)
    cf = nb.ConfigFile(text="Surface = ses\nProbe_Radius = 1.4\nAccurate_Triangulation = true\n"
                            f"Project_boundary_grid_points = true\nGpu_Precision = {precision}\n")
    surf = nb.surfaceFactory().create(cf, ds)
    surf.build()
    assert surf.auxGridDim == 50
    surf.getSurf(True, True, 10.0, keep_hits=True)
    ref = oracle_mod.run(ds.grid, surf.patches, cav_vol=10.0, threads=8, aux_grid_dim=50,
                         flags=oracle_mod.STATUS | oracle_mod.ACCURATE_TRIANGULATION | oracle_mod.CAVITIES |
                         oracle_mod.EPSMAP | oracle_mod.BGP)
    # the node rays of the epsilon map (ray sets 4, 5): same hit counts as the oracle
    g = ds.grid
    for s, ln in ((4, (g.nz - 1) * g.side), (5, (g.ny - 1) * g.side)):
        cnt_g, val_g = surf.hits(s)
        cnt_o, val_o = oracle_mod.ray_hits(ref, s)
        assert np.array_equal(cnt_g, cnt_o), f"ray set {s}: {(cnt_g != cnt_o).sum()} rays with other hit counts"
        if len(val_o):
            d = float(np.abs(val_g - val_o).max()) * (ln if precision == "mixed" else 1.0)
            assert d <= (1e-5 if precision == "mixed" else 1e-12), f"ray set {s}: hits differ by {d}"
    figs = _check(surf, ds, ref, exact=precision == "fp64")
    assert figs["volume_rel"] <= (1e-12 if precision == "fp64" else 1e-9)
    print(f"ses 2000 eps {precision} (grid {ds.nx}^3): {figs}")
