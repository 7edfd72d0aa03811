"""Builds libnsgpu.so in-tree (nanoshaper_b200/lib/) for sm_100a.

Device code is compiled with ``--fmad=false`` so that grid coordinates and the double-precision
ray tests round exactly as the host restatement does; kernels that want fused multiply-adds
request them explicitly.  The one exception is ``kernels/trace_mixed.cu`` (the mixed-precision
intersection kernels, held to a tolerance rather than to bit equality), compiled with
``--fmad=true``.  Host code is compiled with ``-ffp-contract=off``.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIB_DIR = PKG / "lib"
BUILD_DIR = PKG / "_build"
LIB = LIB_DIR / "libnsgpu.so"

CU_SOURCES = ["capi.cu", "kernels/trace.cu", "kernels/trace_mixed.cu", "kernels/trace_mixed_torus.cu", "kernels/cavity.cu", "kernels/mc.cu", "kernels/reduce.cu", "kernels/chain.cu", "kernels/blobby.cu", "kernels/epsmap.cu", "noalloc.cu"]
CPP_SOURCES = ["host/grid.cpp", "host/ses_builder.cpp", "host/skin_builder.cpp", "host/grad.cpp", "host/formats.cpp"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-std=c++17", "-lineinfo", "--fmad=false",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
]
# Files whose device code may contract products and sums into fused multiply-adds (flag replaced).
FMAD_FILES = {"kernels/trace_mixed.cu": {"--fmad=false": "--fmad=true"}}
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-Wall"]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _run(cmd: list[str]) -> None:
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd))


def _stale(out: Path, deps: list[Path]) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compiles the CUDA and host sources and links libnsgpu.so; returns its path."""
    LIB_DIR.mkdir(exist_ok=True)
    BUILD_DIR.mkdir(exist_ok=True)
    headers = list(CSRC.rglob("*.h")) + list(CSRC.rglob("*.cuh"))
    objs = []
    nvcc = _nvcc()
    for src in CU_SOURCES:
        s = CSRC / src
        o = BUILD_DIR / (src.replace("/", "_") + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            flags = [f for f in NVCC_FLAGS if f not in FMAD_FILES.get(src, {})] + list(FMAD_FILES.get(src, {}).values())
            cmd = [nvcc, *flags, "-I", str(CSRC), "-c", str(s), "-o", str(o)]
            if verbose:
                print(" ".join(cmd))
            _run(cmd)
    for src in CPP_SOURCES:
        s = CSRC / src
        o = BUILD_DIR / (src.replace("/", "_") + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            cmd = ["g++", *CXX_FLAGS, "-I", str(CSRC), "-c", str(s), "-o", str(o)]
            if verbose:
                print(" ".join(cmd))
            _run(cmd)
    if force or _stale(LIB, objs):
        cmd = [nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", str(LIB), *map(str, objs),
               "-Xcompiler", "-pthread", "--cudart", "static"]
        if verbose:
            print(" ".join(cmd))
        _run(cmd)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
