"""GPU parity of the atoms lining each cavity (cav2atoms, Surface::getCavitiesAtomsWithBilevelStatusMap)
against the oracle's restatement, on status maps that first equal the oracle's node for node.

* A 2,000-atom SES at scale 2.0 with cavity detection (cavities up to 10 A^3 filled): every
  cavity's atom set equals the oracle's.
* The reference's 1crn SES fixture (its .prm through ConfigFile) with Cavity_Detection_Filling
  switched on, and the cavAtomsSerials.txt it writes.
"""
from pathlib import Path

import numpy as np
import pytest

import nanoshaper_b200 as nb
from nanoshaper_b200 import generator

pytestmark = pytest.mark.gpu

FIXTURES = Path(__file__).resolve().parent / "golden" / "fixtures"


def _check(surf, ds, oracle_mod, cav_vol):
    ref = oracle_mod.run(ds.grid, surf.patches, cav_vol=cav_vol, threads=8,
                         flags=oracle_mod.STATUS | oracle_mod.CAVITIES)
    assert surf.ncav == ref.ncav
    np.testing.assert_array_equal(ds.status, ref.status)
    want = oracle_mod.cavity_atoms(ds.grid, ref.status, ref.ncav, ds.atoms)
    assert ds.cav2atoms == want
    return ref


def test_cavity_atoms_2000(native_lib, oracle_mod):
    atoms = generator.rsa_globule(2000, 5)
    nb.reset_seed()
    ds = nb.DelPhiShared(atoms, 2.0, 80.0)
    cf = nb.ConfigFile(text="Surface = ses\nProbe_Radius = 1.4\n")
    surf = nb.surfaceFactory().create(cf, ds)
    surf.build()
    surf.getSurf(True, True, 10.0)
    _check(surf, ds, oracle_mod, 10.0)
    assert surf.ncav > 0 and all(len(a) > 0 for a in ds.cav2atoms)
    n = sum(len(a) for a in ds.cav2atoms)
    print(f"ses 2000: {surf.ncav} cavities, {n} cavity atoms")


def test_cavity_atoms_fixture_1crn(native_lib, oracle_mod, tmp_path):
    cf = nb.ConfigFile(FIXTURES / "1crn_ses_conf.prm")
    cf.add("Cavity_Detection_Filling", True)
    nb.reset_seed()
    ns = nb.NanoShaper(config=cf)
    ns.buildAnalyticalSurface()
    surf, ds = ns.surf, ns.ds
    surf.getSurf(True, True, 11.4)
    _check(surf, ds, oracle_mod, 11.4)
    ds.saveCavities(tmp_path)
    lines = (tmp_path / "cavAtomsSerials.txt").read_text().split("\n")
    assert len(lines) == surf.ncav + 1 and lines[-1] == ""
    for line, cav in zip(lines, ds.cav2atoms):
        assert line == "".join(f"{a + 1} " for a in cav)
    print(f"1crn: {surf.ncav} cavities, atoms {ds.cav2atoms}")
