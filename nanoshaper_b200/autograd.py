"""torch.autograd bindings of the ray-cast volume and marching-cubes area (SES and blobby).

``ses_volume_area(atoms)`` returns a tensor ``[volume, area]`` whose backward gives
d/d(atom x, y, z, radius).  The forward builds the SES patches on the host, ray casts and
triangulates on the GPU in gradient mode, and keeps the per-patch derivatives of both outputs
(the adjoint kernels: ``kernels/grad.cuh``); the backward combines them with the incoming
gradient and applies the chain rule from patch parameters to atoms on the host.

The grid is an input: by default it is built once from the atoms passed in, and it can be given
explicitly so that it stays fixed while the atoms move (the derivative is taken on a fixed grid,
which is also what central finite differences with a fixed grid measure).  The atom jitter
generator is reset before every build, so the output is a deterministic function of the atoms.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _native as N
from . import surface as S


def _surface(atoms: np.ndarray, probe: float, grid, precision: str, device: int) -> S.ConnollySurface:
    cf = S.ConfigFile()
    cf.add("Surface", "ses")
    cf.add("Probe_Radius", probe)
    cf.add("Accurate_Triangulation", True)
    cf.add("Triangulation", True)
    cf.add("Gpu_Precision", precision)
    S.reset_seed()
    ds = S.DelPhiShared(atoms, grid=grid)
    surf = S.ConnollySurface(cf, ds, device)
    surf.build()
    return surf


class SesVolumeArea(torch.autograd.Function):
    """[volume, area] of the ray-cast SES of ``atoms`` (n, 4: x, y, z, r) on a given grid."""

    @staticmethod
    def forward(ctx, atoms: torch.Tensor, probe: float, grid: N.NsGrid, precision: str, device: int) -> torch.Tensor:
        a = atoms.detach().to("cpu", torch.float64).numpy()
        surf = _surface(a, probe, grid, precision, device)
        try:
            vol = surf.getSurf(True, False, 0.0, download=False, grad=True)
            area = surf.triangulateSurface(download=False)
            gv, ga = surf.patch_gradients(area=True)
        finally:
            surf.ctx.close()
        ctx.patches = surf.patches
        ctx.gv, ctx.ga = gv, ga
        ctx.out_dtype, ctx.out_device = atoms.dtype, atoms.device
        return torch.tensor([vol, area], dtype=atoms.dtype, device=atoms.device)

    @staticmethod
    def backward(ctx, g: torch.Tensor):
        gg = g.detach().to("cpu", torch.float64).numpy()
        gpatch = gg[0] * ctx.gv + gg[1] * ctx.ga
        grad = ctx.patches.chain_to_atoms(gpatch)
        return torch.from_numpy(grad).to(ctx.out_device, ctx.out_dtype), None, None, None, None


class BlobbyVolumeArea(torch.autograd.Function):
    """[volume, area] of the ray-cast blobby surface of ``atoms`` (n, 4) on a given grid.  The
    blobby mesh is built without the OFF text round trip (whose 1e-3 A rounding is piecewise
    constant in the atoms); the backward chains the per-triangle hit terms through the smoothing,
    the interpolated marching-cubes vertices and the Gaussian field to the atoms, on the device."""

    @staticmethod
    def forward(ctx, atoms: torch.Tensor, blobbyness: float, grid: N.NsGrid, precision: str,
                device: int) -> torch.Tensor:
        a = atoms.detach().to("cpu", torch.float64).numpy()
        cf = S.ConfigFile()
        cf.add("Surface", "blobby")
        cf.add("Blobbyness", blobbyness)
        cf.add("Accurate_Triangulation", True)
        cf.add("Triangulation", True)
        cf.add("Gpu_Precision", precision)
        ds = S.DelPhiShared(a, grid=grid)
        surf = S.BlobbySurface(cf, ds, device)
        surf.differentiable = True
        try:
            surf.build()
            vol = surf.getSurf(True, False, 0.0, download=False, grad=True)
            area = surf.triangulateSurface(download=False)
            gv = surf.gradients(1.0, 0.0)
            ga = surf.gradients(0.0, 1.0)
        finally:
            surf.ctx.close()
        ctx.gv, ctx.ga = gv, ga
        ctx.out_dtype, ctx.out_device = atoms.dtype, atoms.device
        return torch.tensor([vol, area], dtype=atoms.dtype, device=atoms.device)

    @staticmethod
    def backward(ctx, g: torch.Tensor):
        gg = g.detach().to("cpu", torch.float64).numpy()
        grad = gg[0] * ctx.gv + gg[1] * ctx.ga
        return torch.from_numpy(grad).to(ctx.out_device, ctx.out_dtype), None, None, None, None


def blobby_volume_area(atoms: torch.Tensor, blobbyness: float = -2.5, grid: N.NsGrid | None = None,
                       scale: float = S.DEFAULT_SCALE, perfil: float = S.DEFAULT_PERFIL, precision: str = "fp64",
                       device: int = 0) -> torch.Tensor:
    """Differentiable [volume, area] of the blobby surface of ``atoms``; see BlobbyVolumeArea."""
    if grid is None:
        grid = grid_for(atoms, scale, perfil)
    return BlobbyVolumeArea.apply(atoms, blobbyness, grid, precision, device)


def grid_for(atoms, scale: float = S.DEFAULT_SCALE, perfil: float = S.DEFAULT_PERFIL) -> N.NsGrid:
    """The reference's grid (buildGrid) for a set of atoms."""
    a = atoms.detach().to("cpu", torch.float64).numpy() if isinstance(atoms, torch.Tensor) else np.asarray(atoms)
    return S.DelPhiShared(a, scale, perfil).grid


def ses_volume_area(atoms: torch.Tensor, probe: float = S.DEFAULT_PROBE, grid: N.NsGrid | None = None,
                    scale: float = S.DEFAULT_SCALE, perfil: float = S.DEFAULT_PERFIL, precision: str = "fp64",
                    device: int = 0) -> torch.Tensor:
    """Differentiable [volume, area] of the SES of ``atoms``; see the module docstring."""
    if grid is None:
        grid = grid_for(atoms, scale, perfil)
    return SesVolumeArea.apply(atoms, probe, grid, precision, device)
