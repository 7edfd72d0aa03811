"""GPU parity of the water-shape cavity filter, Keep_Water_Shaped_Cavities
(Surface::filterCavitiesWithBilevelStatusMap, src/Surface.cpp:3011-3290), against the oracle's
loop-for-loop restatement applied to the oracle's own maps after cavity detection.

* A 2,000-atom SES at scale 2.0 with cavities up to 10 A^3 filled and the epsilon maps on, through
  the Python getSurf (the status map left unmodified, as getSurf runs the filter): status codes,
  insideness bits, epsilon and ideb maps, cavity flags and the cavity atoms equal the oracle's.
* The same surface with the status map modified (removed nodes inside), through the C-ABI.
"""
import ctypes

import numpy as np
import pytest

import nanoshaper_b200 as nb
from nanoshaper_b200 import _native as N
from nanoshaper_b200 import generator

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def atoms_2000():
    return generator.rsa_globule(2000, 5)


def _surface(atoms, shape: bool):
    nb.reset_seed()
    ds = nb.DelPhiShared(atoms, 2.0, 80.0, build_eps_map=True)
    cf = nb.ConfigFile(text="Surface = ses\nProbe_Radius = 1.4\nAccurate_Triangulation = true\n"
                            f"Keep_Water_Shaped_Cavities = {'true' if shape else 'false'}\n")
    surf = nb.surfaceFactory().create(cf, ds)
    surf.build()
    return ds, surf


def _oracle(ds, surf, oracle_mod, mod_status):
    ref = oracle_mod.run(ds.grid, surf.patches, cav_vol=10.0, threads=8,
                         flags=oracle_mod.STATUS | oracle_mod.ACCURATE_TRIANGULATION | oracle_mod.CAVITIES |
                         oracle_mod.EPSMAP)
    out = oracle_mod.shape_filter(ds.grid, ref.status, ref.ncav, ref.cav_filled, bits=ref.bits,
                                  eps=ref.epsmap, ideb=ref.idebmap, probe=1.4, mod_status=mod_status)
    return ref, out


def test_shape_filter_getsurf(atoms_2000, native_lib, oracle_mod):
    ds, surf = _surface(atoms_2000, True)
    surf.getSurf(True, True, 10.0)
    ref, (st, fl, bits, eps, ideb, nrem) = _oracle(ds, surf, oracle_mod, False)
    assert surf.ncav == ref.ncav
    np.testing.assert_array_equal(ds.status.reshape(-1), st.reshape(-1))
    np.testing.assert_array_equal(surf.insideness, bits)
    np.testing.assert_array_equal(ds.epsmap.reshape(-1), eps.reshape(-1))
    np.testing.assert_array_equal(ds.idebmap.reshape(-1), ideb.reshape(-1))
    assert ds.cavitiesFlag == [bool(f) for f in fl]
    assert nrem > 0, "the case should remove nodes"
    want = oracle_mod.cavity_atoms(ds.grid, st.reshape(ref.status.shape), ref.ncav, ds.atoms, label=ref.status)
    assert ds.cav2atoms == want
    n_sup = int((st < -3).sum())
    print(f"ses 2000 shape filter: {surf.ncav} cavities, {nrem} nodes removed, {n_sup} supports, "
          f"{sum(fl) - sum(ref.cav_filled)} cavities filled by the filter")


def test_shape_filter_modify_status(atoms_2000, native_lib, oracle_mod):
    ds, surf = _surface(atoms_2000, False)
    surf.getSurf(True, True, 10.0, download=False)
    c = surf._context().handle
    nrem = ctypes.c_int64()
    N.check(N.lib().nsg_filter_cavities(c, 1.4, 1, ctypes.byref(nrem)), "shape filter")
    # a second filter on the same detection is refused
    assert N.lib().nsg_filter_cavities(c, 1.4, 1, None) != 0
    g = ds.grid
    st = np.empty(g.nx * g.ny * g.nz, np.int32)
    N.check(N.lib().nsg_download_status(c, N.ptr(st)), "status")
    words = ((g.nx + 31) >> 5) * g.ny * g.nz
    bits = np.empty(words, np.uint32)
    N.check(N.lib().nsg_download_insideness(c, N.ptr(bits)), "bits")
    fl = np.zeros(surf.ncav, np.int32)
    N.check(N.lib().nsg_download_cavities(c, None, N.ptr(fl)), "flags")
    ref, (st_o, fl_o, bits_o, _eps, _ideb, nrem_o) = _oracle(ds, surf, oracle_mod, True)
    assert nrem.value == nrem_o
    np.testing.assert_array_equal(st, st_o.reshape(-1))
    np.testing.assert_array_equal(bits, bits_o)
    np.testing.assert_array_equal(fl, fl_o)
    assert not np.isin(st, [-3, -2]).any()
    print(f"ses 2000 shape filter (status modified): {nrem.value} nodes removed")
