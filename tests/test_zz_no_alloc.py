"""The allocation-free status ray cast (nsg_status_noalloc) against the context pipeline
(nsg_raycast with the status flag) on the same patch set: status maps equal node for node and
volumes within 1e-12 relative (the interval-length sums are reduced in a different order), on two
calls in a row so that state left in the shared scratch array by the first call cannot leak
into the second.  The file name keeps it last in collection order; it also passes alone.
"""
import ctypes

import numpy as np
import pytest

import nanoshaper_b200 as nb
from nanoshaper_b200 import _native as N
from nanoshaper_b200 import generator

pytestmark = pytest.mark.gpu

VOL_RTOL = 1e-12
MAX_RAYS = 65536
ERR_CAPACITY = -4


def _bind(L):
    fn = L.nsg_status_noalloc
    fn.argtypes = [ctypes.POINTER(N.NsGrid), ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                   ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                   ctypes.c_void_p]
    fn.restype = ctypes.c_int
    return fn


def _surface(n_atoms, seed, scale, perfil):
    atoms = generator.rsa_globule(n_atoms, seed)
    nb.reset_seed()
    cf = nb.ConfigFile()
    cf.add("Surface", "ses")
    cf.add("Probe_Radius", 1.4)
    ds = nb.DelPhiShared(atoms, scale, perfil)
    surf = nb.surfaceFactory().create(cf, ds)
    surf.build()
    return ds, surf


@pytest.mark.parametrize("n_atoms,seed,scale,perfil", [(60, 11, 2.0, 70.0), (327, 1, 2.0, 70.0)])
def test_noalloc_status_matches_pipeline(n_atoms, seed, scale, perfil, native_lib):
    import torch

    fn = _bind(native_lib)
    ds, surf = _surface(n_atoms, seed, scale, perfil)
    g = ds.grid
    assert g.ny * g.nz <= MAX_RAYS
    vol_ref = surf.getSurf(True, False, 0.0)
    st_ref = ds.status.reshape(-1).copy()

    p = surf.patches
    dev = torch.device("cuda:0")
    f64 = torch.from_numpy(p.f64).to(dev)
    i32 = torch.from_numpy(p.i32).to(dev)
    pool = torch.from_numpy(p.pool).to(dev)
    flag = torch.from_numpy(p.pool_flag).to(dev)
    status = torch.full((g.nx * g.ny * g.nz,), 7, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    for call in range(2):
        vol = ctypes.c_double(-1.0)
        rc = fn(ctypes.byref(g), p.n, f64.data_ptr(), i32.data_ptr(), pool.data_ptr() if len(p.pool) else None,
                flag.data_ptr() if len(p.pool) else None, p.probe, status.data_ptr(), ctypes.byref(vol),
                stream.cuda_stream)
        assert rc == N.NSG_OK, f"call {call}: rc {rc}"
        st = status.cpu().numpy()
        diff = int((st != st_ref).sum())
        assert diff == 0, f"call {call}: {diff} status nodes differ"
        assert abs(vol.value - vol_ref) <= VOL_RTOL * abs(vol_ref), f"call {call}: volume {vol.value} vs {vol_ref}"
        status.fill_(7)


def test_noalloc_rejects_oversize_grid(native_lib):
    fn = _bind(native_lib)
    g = N.NsGrid()
    g.nx, g.ny, g.nz = 4, 300, 300  # 90000 status rays > 65536
    vol = ctypes.c_double()
    rc = fn(ctypes.byref(g), 0, None, None, None, None, 1.4, ctypes.c_void_p(16), ctypes.byref(vol), None)
    assert rc == ERR_CAPACITY


def test_noalloc_reports_hit_overflow(native_lib):
    """A status ray with more than 32 hits: 17 disjoint spheres strung along the x axis give 34
    hits on the ray through their centres; the call returns NSG_ERR_CAPACITY after its launches."""
    import torch

    fn = _bind(native_lib)
    n = 17
    atoms = np.zeros((n, 4))
    atoms[:, 0] = np.arange(n) * 3.0
    atoms[:, 3] = 1.0
    ds = nb.DelPhiShared(atoms, 2.0, 50.0)
    g = ds.grid
    f64 = np.zeros((n, 20))
    f64[:, 0:4] = atoms
    i32 = np.zeros((n, 4), np.int32)  # point patches without clipping spheres
    # put the atom centres on the grid's middle status ray (j, k) so that it crosses all of them
    jm, km = g.ny // 2, g.nz // 2
    f64[:, 1] = g.ymin + jm * g.side
    f64[:, 2] = g.zmin + km * g.side
    dev = torch.device("cuda:0")
    d_f64 = torch.from_numpy(f64).to(dev)
    d_i32 = torch.from_numpy(i32).to(dev)
    status = torch.zeros(g.nx * g.ny * g.nz, dtype=torch.int32, device=dev)
    vol = ctypes.c_double()
    stream = torch.cuda.current_stream(dev)
    rc = fn(ctypes.byref(g), n, d_f64.data_ptr(), d_i32.data_ptr(), None, None, 1.4, status.data_ptr(),
            ctypes.byref(vol), stream.cuda_stream)
    assert rc == ERR_CAPACITY
