"""ctypes binding of libnsgpu.so (the C-ABI declared in include/nsgpu.h).

The library is loaded from the package's ``lib/`` directory.  There is no CPU fallback: when the
library or a CUDA device is missing, the calls fail loudly.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libnsgpu.so"

NSG_OK = 0
ERRORS = {
    -1: "invalid argument",
    -2: "empty input",
    -3: "I/O error",
    -4: "capacity exceeded",
    -5: "CUDA error",
    -6: "out of memory",
    -7: "invalid state",
    -8: "degenerate geometry",
    -9: "device wait timed out",
}

# raycast flags
STATUS = 1
ACCURATE_TRIANGULATION = 2
EPSMAP = 4
KEEP_HITS = 16
GRAD = 32
NORMALS = 64


class NsGrid(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int64), ("ny", ctypes.c_int64), ("nz", ctypes.c_int64),
        ("xmin", ctypes.c_double), ("ymin", ctypes.c_double), ("zmin", ctypes.c_double),
        ("xmax", ctypes.c_double), ("ymax", ctypes.c_double), ("zmax", ctypes.c_double),
        ("scale", ctypes.c_double), ("side", ctypes.c_double), ("hside", ctypes.c_double),
        ("A", ctypes.c_double), ("rmaxdim", ctypes.c_double), ("baricenter", ctypes.c_double * 3),
    ]


class NativeError(RuntimeError):
    pass


_P = ctypes.c_void_p
_I64 = ctypes.c_int64
_D = ctypes.c_double
_INT = ctypes.c_int

_SIGNATURES = {
    "nsg_last_error": ([], ctypes.c_char_p),
    "nsg_version": ([], _INT),
    "nsg_ctx_create": ([_INT, ctypes.POINTER(_P)], _INT),
    "nsg_ctx_destroy": ([_P], _INT),
    "nsg_set_stream": ([_P, _P], _INT),
    "nsg_set_grid": ([_P, ctypes.POINTER(NsGrid)], _INT),
    "nsg_upload_patches": ([_P, _I64, _P, _P, _I64, _P, _P, _D], _INT),
    "nsg_bind_patches_device": ([_P, _I64, _P, _P, _I64, _P, _P, _D], _INT),
    "nsg_raycast": ([_P, _INT, _INT, ctypes.POINTER(_D)], _INT),
    "nsg_set_batch": ([_P, ctypes.c_int32, _P], _INT),
    "nsg_upload_batch": ([_P, _P, _P, _P, _P, _P, _P, _D], _INT),
    "nsg_batch_results": ([_P, _P, _P], _INT),
    "nsg_set_tuning": ([_P, _P, _INT], _INT),
    "nsg_get_tuning": ([_P, _P, _INT], _INT),
    "nsg_autotune": ([_P, _INT, _INT, _INT, ctypes.POINTER(_D)], _INT),
    "nsg_fp_peak": ([_P, _INT, ctypes.POINTER(_D)], _INT),
    "nsg_cavities": ([_P, _D, ctypes.POINTER(_INT)], _INT),
    "nsg_filter_cavities": ([_P, _D, _INT, ctypes.POINTER(ctypes.c_int64)], _INT),
    "nsg_pocket_difference": ([_P, _P, _D, ctypes.POINTER(_INT)], _INT),
    "nsg_cavity_order": ([ctypes.c_int32, _P, _P], _INT),
    "nsg_triangulate": ([_P, ctypes.POINTER(_D), ctypes.POINTER(_I64), ctypes.POINTER(_I64)], _INT),
    "nsg_download_status": ([_P, _P], _INT),
    "nsg_download_insideness": ([_P, _P], _INT),
    "nsg_download_mesh": ([_P, _P, _P, _P], _INT),
    "nsg_download_cavities": ([_P, _P, _P], _INT),
    "nsg_cavity_atoms": ([_P, _P, _I64, _P, _P, ctypes.POINTER(_I64)], _INT),
    "nsg_download_hits": ([_P, _INT, _P, _P, _I64], _INT),
    "nsg_download_epsmap": ([_P, _P], _INT),
    "nsg_download_idebmap": ([_P, _P], _INT),
    "nsg_bgp": ([_P, _INT, ctypes.c_int32, _P, _P], _INT),
    "nsg_download_bgp": ([_P, _P, _P, _P, _P, _P], _INT),
    "nsg_stats": ([_P, _P, _INT], _INT),
    "nsg_event_record": ([_P, _INT], _INT),
    "nsg_event_elapsed": ([_P, _INT, _INT, ctypes.POINTER(_D)], _INT),
    "nsg_profile": ([_P, _INT], _INT),
    "nsg_stage_times": ([_P, _P, _P, _INT], _INT),
    "nsg_launch_count": ([_P], _I64),
    "nsg_trace_counters": ([_P, _P, _INT], _INT),
    "nsg_get_stream": ([_P], _P),
    "nsg_volume": ([_P], _D),
    "nsg_area": ([_P], _D),
    "nsg_grid_build": ([_P, _I64, _D, _D, ctypes.POINTER(NsGrid)], _INT),
    "nsg_randnum": ([ctypes.POINTER(_I64)], _D),
    "nsg_jitter_atoms": ([_P, _I64, _D, ctypes.POINTER(_I64)], _INT),
    "nsg_read_xyzr": ([ctypes.c_char_p, _P, _I64], _I64),
    "nsg_read_pqr": ([ctypes.c_char_p, _P, _I64], _I64),
    "nsg_ses_build": ([_P, _I64, _D, _INT, ctypes.POINTER(_P)], _INT),
    "nsg_patchset_info": ([_P, ctypes.POINTER(_I64), ctypes.POINTER(_I64), _P], _INT),
    "nsg_patchset_kind_counts": ([_P, _P, _INT], _INT),
    "nsg_skin_build": ([_P, _I64, _D, _INT, ctypes.POINTER(_P)], _INT),
    "nsg_skin_predicates": ([_P, _P, _P], _INT),
    "nsg_blobby_build": ([_P, _P, _I64, _D, _INT], _INT),
    "nsg_blobby_mesh": ([_P, ctypes.POINTER(_I64), ctypes.POINTER(_I64), _P, _P], _INT),
    "nsg_blobby_atom_grads": ([_P, _P, _P], _INT),
    "nsg_vertex_normals": ([_P, _P], _INT),
    "nsg_fill_zero_normals": ([_P, _I64, _P, _I64, _P], _INT),
    "nsg_patchset_export": ([_P, _P, _P, _P, _P], _INT),
    "nsg_patchset_free": ([_P], None),
    "nsg_patchset_atoms": ([_P, _P], _INT),
    "nsg_write_status": ([ctypes.c_char_p, _P, _I64, _I64, _I64], _INT),
    "nsg_write_cavities": ([ctypes.c_char_p, ctypes.c_char_p, _P, ctypes.POINTER(NsGrid), ctypes.c_int32, _P, _P],
                           _INT),
    "nsg_write_cavity_atoms": ([ctypes.c_char_p, ctypes.c_int32, _P, _P, _P, _I64, _P], _INT),
    "nsg_write_mesh": ([ctypes.c_char_p, _INT, _P, _I64, _P, _I64, _INT], _INT),
    "nsg_mesh_normals": ([_P, _I64, _P, _I64, _P], _INT),
    "nsg_vertex_atoms": ([_P, _I64, _P, _I64, _P], _INT),
    "nsg_write_mesh_attrs": ([ctypes.c_char_p, _INT, _P, _P, _P, _I64, _P, _I64, _INT], _INT),
    "nsg_patch_grads": ([_P, _P, _P], _INT),
    "nsg_upload_atoms": ([_P, _P, _P, _P], _INT),
    "nsg_atom_grads": ([_P, _P, _P], _INT),
    "nsg_ses_chain_grad": ([_P, _I64, _D, _I64, _P, _P, _P, _P, _P], _INT),
}

_lib = None


def lib() -> ctypes.CDLL:
    """Loads libnsgpu.so once; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise NativeError(f"{LIB_PATH} is missing: run nanoshaper_b200.build.build() first")
        L = ctypes.CDLL(str(LIB_PATH))
        for name, (args, res) in _SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def check(rc: int, what: str) -> None:
    if rc != NSG_OK:
        msg = lib().nsg_last_error().decode(errors="replace")
        raise NativeError(f"{what} failed: {ERRORS.get(rc, rc)} ({msg})")


def ptr(a: np.ndarray | None) -> int | None:
    if a is None:
        return None
    return a.ctypes.data


def exported_symbols() -> list[str]:
    return list(_SIGNATURES)
