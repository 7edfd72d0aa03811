"""Generates tests/golden/ref_math.npz: golden vectors of the reference's own ray/solver math.

Needs the reference sources: NANOSHAPER_REFERENCE names the root of a NanoShaper source checkout,
compiled into oracle/_ref/libnsref.so by oracle/ref.mk.  Inputs are
seeded: rays of the status and triangulation panels of a synthetic globule against its sphere
and torus patches (the patch set comes from this package's host builder), plus the jitter
generator sequence, rintp and plane-through-three-points values.  Outputs are evaluated by the
reference functions raySphere, rayTorus (analytical and Sturm), randnum, rintp and plane3points
(src/tools.cpp).  Run:  NANOSHAPER_REFERENCE=<checkout> python tests/golden/make_golden.py
"""
from __future__ import annotations

import ctypes
import subprocess
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))


def ref_lib() -> ctypes.CDLL:
    subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "-f", "ref.mk"], check=True)
    L = ctypes.CDLL(str(ROOT / "oracle" / "_ref" / "libnsref.so"))
    P = ctypes.c_void_p
    D = ctypes.c_double
    L.ref_ray_sphere.argtypes = [P, P, P, D, P]
    L.ref_ray_sphere.restype = ctypes.c_int
    L.ref_ray_torus.argtypes = [ctypes.c_int, P, P, P, D, D, D, ctypes.c_int, P, P, P]
    L.ref_ray_torus.restype = ctypes.c_int
    L.ref_randnum_seq.argtypes = [ctypes.c_int]
    L.ref_randnum_seq.restype = D
    L.ref_rintp.argtypes = [D]
    L.ref_rintp.restype = D
    L.ref_plane3points.argtypes = [P, P, P, P]
    return L


def main() -> None:
    import nanoshaper_b200 as nb
    from nanoshaper_b200 import generator

    L = ref_lib()
    rng = np.random.default_rng(2024)
    atoms = generator.rsa_globule(200, seed=21)
    ds = nb.DelPhiShared(atoms, 3.0, 70.0)
    nb.reset_seed()
    cf = nb.ConfigFile(text="Surface = ses\n")
    surf = nb.ConnollySurface(cf, ds)
    surf.build()
    p = surf.patches
    g = ds.grid
    mins = np.array([g.xmin, g.ymin, g.zmin])
    n_axis = np.array([g.nx, g.ny, g.nz])
    dims = {0: (1, 2, 0), 1: (0, 1, 2), 2: (0, 2, 1)}  # panel -> (first, second, ray axis)

    sph_in, sph_out, tor_in, tor_out = [], [], [], []
    for it in range(p.n):
        kind = p.i32[it, 0]
        c = p.f64[it, :3]
        r = p.f64[it, 3]
        for panel in range(3):
            fd, ld, vc = dims[panel]
            for delta in (0.0, 1e-10 - g.hside):
                for _ in range(1):
                    pa = np.zeros(3)
                    # pixel centres near the patch
                    m = int(round((c[fd] - mins[fd]) * g.scale + rng.uniform(-r, r) * g.scale))
                    n = int(round((c[ld] - mins[ld]) * g.scale + rng.uniform(-r, r) * g.scale))
                    m = min(max(m, 0), n_axis[fd] - 1)
                    n = min(max(n, 0), n_axis[ld] - 1)
                    pa[fd] = mins[fd] + m * g.side + delta
                    pa[ld] = mins[ld] + n * g.side + delta
                    pa[vc] = mins[vc] + delta
                    d = np.zeros(3)
                    d[vc] = (mins[vc] + (n_axis[vc] - 1) * g.side) - mins[vc]
                    t = np.zeros(2)
                    ok = L.ref_ray_sphere(pa.ctypes.data, d.ctypes.data, c.ctypes.data, r, t.ctypes.data)
                    sph_in.append(np.concatenate([pa, d, c, [r]]))
                    sph_out.append([ok, t[0], t[1]])
                    if ok and kind in (1, 2):
                        tt = np.zeros(4)
                        tt[:2] = t
                        inv = np.ascontiguousarray(p.f64[it, 9:18])
                        tc = np.ascontiguousarray(p.f64[it, 4:7])
                        cc = np.ascontiguousarray(c)
                        nn = L.ref_ray_torus(1, inv.ctypes.data, tc.ctypes.data, cc.ctypes.data, p.probe,
                                             p.f64[it, 7], r, panel, pa.ctypes.data, d.ctypes.data, tt.ctypes.data)
                        tor_in.append(np.concatenate([inv, tc, cc, [p.probe, p.f64[it, 7], r, panel], pa, d, t]))
                        tor_out.append(np.concatenate([[nn], tt]))
    seq = np.array([L.ref_randnum_seq(1) for _ in range(64)])
    xs = rng.uniform(-50, 50, 256)
    xs = np.concatenate([xs, np.arange(-4, 4) + 0.5, np.arange(-4, 4) - 1e-12])
    rint = np.array([L.ref_rintp(float(x)) for x in xs])
    pts = rng.uniform(-10, 10, size=(64, 3, 3))
    planes = np.zeros((64, 4))
    for i in range(64):
        a, b, c3 = (np.ascontiguousarray(pts[i, k]) for k in range(3))
        L.ref_plane3points(a.ctypes.data, b.ctypes.data, c3.ctypes.data, planes[i].ctypes.data)
    out = Path(__file__).resolve().parent / "ref_math.npz"
    np.savez_compressed(out, sphere_in=np.array(sph_in), sphere_out=np.array(sph_out), torus_in=np.array(tor_in),
                        torus_out=np.array(tor_out), randnum=seq, rint_in=xs, rint_out=rint, plane_pts=pts,
                        plane_out=planes)
    print(out, len(sph_in), "sphere cases,", len(tor_in), "torus cases")


if __name__ == "__main__":
    main()
