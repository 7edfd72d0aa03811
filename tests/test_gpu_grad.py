"""Adjoint of the ray-cast volume and the marching-cubes area against central finite differences.

Each checked component is d(volume) or d(area) / d(atom x, y, z or r), on a fixed grid.
Central differences use h = 1e-4 A. A component is compared with h = 1e-4; where the volume
or area is not smooth on that scale, the two central differences at h and h/10 disagree by
more than the tolerance, and the comparison uses h/10 instead. Area components whose ±h
runs change an insideness bit are discontinuous there and are skipped. The skipped share is
bounded. The bar is 1e-4 relative (with an absolute floor of 1e-6 of the gradient's
largest component).
"""
import numpy as np
import pytest
import torch

import nanoshaper_b200 as nb
from nanoshaper_b200 import autograd as AG
from nanoshaper_b200 import generator

pytestmark = pytest.mark.gpu

H = 1e-4
RTOL = 1e-4


class FixedGridRunner:
    """Volume / area / insideness of perturbed atoms on one fixed grid, one GPU context."""

    def __init__(self, grid, precision):
        self.grid = grid
        self.cf = nb.ConfigFile()
        self.cf.add("Surface", "ses")
        self.cf.add("Probe_Radius", 1.4)
        self.cf.add("Accurate_Triangulation", True)
        self.cf.add("Gpu_Precision", precision)
        self.surf = None

    def __call__(self, atoms):
        nb.reset_seed()
        ds = nb.DelPhiShared(atoms, grid=self.grid)
        if self.surf is None:
            self.surf = nb.ConnollySurface(self.cf, ds)
        self.surf.delphi = ds
        self.surf.build()
        v = self.surf.getSurf(True, False, 0.0, download=True)
        a = self.surf.triangulateSurface(download=False)
        return v, a, self.surf.insideness.copy()


def _fd(run, atoms, i, d, h):
    a1 = atoms.copy()
    a1[i, d] += h
    a2 = atoms.copy()
    a2[i, d] -= h
    v1, ar1, b1 = run(a1)
    v2, ar2, b2 = run(a2)
    return (v1 - v2) / (2 * h), (ar1 - ar2) / (2 * h), bool((b1 != b2).any())


def _check(n_atoms, seed, scale, n_pick, precision, max_skip_frac):
    atoms = generator.rsa_globule(n_atoms, seed)
    grid = AG.grid_for(atoms, scale, 80.0)
    x = torch.tensor(atoms, dtype=torch.float64, requires_grad=True)
    out = AG.ses_volume_area(x, 1.4, grid, precision=precision)
    gv = torch.autograd.grad(out[0], x, retain_graph=True)[0].numpy()
    ga = torch.autograd.grad(out[1], x)[0].numpy()
    run = FixedGridRunner(grid, precision)
    v0, a0, _ = run(atoms)
    assert abs(v0 - out[0].item()) <= 1e-12 * abs(v0) and abs(a0 - out[1].item()) <= 1e-12 * abs(a0)
    pick = np.random.default_rng(7).choice(n_atoms, size=n_pick, replace=False)
    floor_v, floor_a = 1e-6 * np.abs(gv).max(), 1e-6 * np.abs(ga).max()
    bad, skipped, total = [], 0, 0
    for i in pick:
        for d in range(4):
            fv, fa, jump = _fd(run, atoms, i, d, H)
            fv2, fa2, jump2 = _fd(run, atoms, i, d, H / 10)
            for name, g, f, f2, fl, disc in (("vol", gv[i, d], fv, fv2, floor_v, False),
                                             ("area", ga[i, d], fa, fa2, floor_a, jump or jump2)):
                total += 1
                if disc:
                    skipped += 1
                    continue
                tol = lambda ref: RTOL * abs(ref) + fl  # noqa: E731
                if abs(g - f) <= tol(f):
                    continue
                if abs(f - f2) > tol(f2) and abs(g - f2) <= tol(f2):
                    continue  # not smooth at scale h; the finer difference agrees
                bad.append((name, int(i), d, g, f, f2))
    assert skipped <= max_skip_frac * total, f"{skipped} of {total} components skipped as discontinuous"
    assert not bad, f"{len(bad)} of {total} components off: {bad[:6]}"
    return total, skipped


def test_gradients_match_fd_300(native_lib):
    _check(300, 4, 3.0, 16, "fp64", 0.1)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_gradients_match_fd_2000(precision, native_lib):
    """Differentiation configuration: 2,000 atoms, grid scale 3.0, 64 atoms checked."""
    total, skipped = _check(2000, 11, 3.0, 64, precision, 0.1)
    print(f"{precision}: {total} components, {skipped} skipped as discontinuous")


def test_mixed_gradients_match_fp64(native_lib):
    """The adjoint of the mixed-precision forward against that of the double-precision forward."""
    atoms = generator.rsa_globule(800, 5)
    grid = AG.grid_for(atoms, 3.0, 80.0)
    g = {}
    for prec in ("fp64", "mixed"):
        x = torch.tensor(atoms, dtype=torch.float64, requires_grad=True)
        out = AG.ses_volume_area(x, 1.4, grid, precision=prec)
        (out[0] + 0.5 * out[1]).backward()
        g[prec] = x.grad.numpy().copy()
    scale = np.abs(g["fp64"]).max()
    assert np.abs(g["mixed"] - g["fp64"]).max() <= 1e-6 * scale


def test_surface_gradients_api(native_lib):
    """Surface.gradients (the non-torch path) equals the autograd backward."""
    atoms = generator.rsa_globule(120, 9)
    grid = AG.grid_for(atoms, 3.0, 80.0)
    x = torch.tensor(atoms, dtype=torch.float64, requires_grad=True)
    out = AG.ses_volume_area(x, 1.4, grid)
    (2.0 * out[0] - 3.0 * out[1]).backward()
    run = FixedGridRunner(grid, "fp64")
    nb.reset_seed()
    ds = nb.DelPhiShared(atoms, grid=grid)
    s = nb.ConnollySurface(run.cf, ds)
    s.build()
    s.getSurf(True, False, 0.0, download=False, grad=True)
    s.triangulateSurface(download=False)
    g = s.gradients(2.0, -3.0)
    assert np.allclose(g, x.grad.numpy(), rtol=1e-12, atol=1e-12)
