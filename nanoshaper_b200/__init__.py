"""B200-native grid ray-casting molecular surface builder (NanoShaper-compatible interface)."""
from .surface import (  # noqa: F401
    BlobbySurface,
    ConfigFile,
    ConnollySurface,
    Context,
    DelPhiShared,
    NanoShaper,
    PatchSet,
    Surface,
    SurfaceBatch,
    SkinSurface,
    SurfaceFactory,
    build_ses_patches,
    build_skin_patches,
    read_atoms,
    read_pqr,
    read_xyzr,
    reset_seed,
    surfaceFactory,
)

__version__ = "0.1.0"
