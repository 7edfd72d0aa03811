"""GPU parity of pocket detection by difference (pocket mode's ``(*surf1) -= (*surf2)`` and
``fillCavities``, src/main.cpp:1411-1586) against the oracle's loop-for-loop restatement applied
to the oracle's own status maps and insideness bits of the two casts.

SES of 2,000 atoms (pockets of at most 22.8 A^3, two water molecules, filled) and of 10,000 atoms
(no pocket filled) at scale 2.0: the fat surface with a 3.0 A probe and the small one with 1.4 A,
both with cavity detection and every cavity filled (as pocket mode casts them).  Status map with
the pocket labels, insideness bits, pocket sizes and flags, and the pockets' atoms equal the
oracle's.
"""
import math

import numpy as np
import pytest

import nanoshaper_b200 as nb
from nanoshaper_b200 import generator

pytestmark = pytest.mark.gpu


def _cast(atoms, probe):
    nb.reset_seed()
    ds = nb.DelPhiShared(atoms, 2.0, 80.0)
    cf = nb.ConfigFile(text=f"Surface = ses\nProbe_Radius = {probe}\nAccurate_Triangulation = true\n")
    surf = nb.surfaceFactory().create(cf, ds)
    surf.build()
    surf.getSurf(True, True, math.inf)
    return ds, surf


@pytest.mark.parametrize("n_atoms,seed,fill", [(2000, 5, 22.8), (10000, 2, 0.0)])
def test_pocket_difference(n_atoms, seed, fill, native_lib, oracle_mod):
    atoms = generator.rsa_globule(n_atoms, seed)
    ds1, fat = _cast(atoms, 3.0)
    ds2, small = _cast(atoms, 1.4)
    flags = oracle_mod.STATUS | oracle_mod.ACCURATE_TRIANGULATION | oracle_mod.CAVITIES
    r1 = oracle_mod.run(ds1.grid, fat.patches, flags=flags, cav_vol=math.inf, threads=8)
    r2 = oracle_mod.run(ds2.grid, small.patches, flags=flags, cav_vol=math.inf, threads=8)
    np.testing.assert_array_equal(ds1.status, r1.status)
    np.testing.assert_array_equal(ds2.status, r2.status)
    n = fat.difference(small, fill)
    st, bits, sizes, filled = oracle_mod.pocket_difference(ds1.grid, r1.status, r2.status, r1.bits, fill)
    assert n == len(sizes) and n > 0
    np.testing.assert_array_equal(ds1.status.reshape(-1), st.reshape(-1))
    np.testing.assert_array_equal(fat.insideness, bits)
    np.testing.assert_allclose(ds1.cavitiesSize, sizes, rtol=0, atol=0)
    assert ds1.cavitiesFlag == [bool(f) for f in filled]
    got = fat.getCavitiesAtoms()
    assert got == oracle_mod.cavity_atoms(ds1.grid, st.reshape(r1.status.shape), n, ds1.atoms)
    print(f"ses {n_atoms} pockets (probes 3.0 / 1.4): {n} pockets, {int(sum(filled))} filled, "
          f"largest {max(sizes):.2f} A^3")
