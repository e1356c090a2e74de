"""ctypes binding of the C-ABI library ``lib/librkb200.so`` (include/rkb200.h).

The engine has no CPU fallback: loading fails loudly when the library is
missing or the current CUDA device is not an sm_100 part, and every entry
point's status is turned into the exception atomx raises for the same
condition (ValueError, FloatingPointError, MemoryError, TimeoutError).
"""
from __future__ import annotations

import ctypes
import os
import threading

from . import build as _build

__all__ = ["lib", "check", "RkbError", "ptr", "stream_handle", "load"]

_c = ctypes
_vp, _l, _i, _d = _c.c_void_p, _c.c_long, _c.c_int, _c.c_double

# name -> argument types (all return int status unless listed in _RESTYPE)
_SIGNATURES = {
    "rkb_last_error": [],
    "rkb_version": [],
    "rkb_device_supported": [],
    "rkb_yk_flat": [_vp, _vp, _vp, _l, _i, _i, _i, _vp, _vp, _vp, _vp],
    "rkb_yk_rows": [_vp, _l, _vp, _l, _vp, _vp, _i, _i, _vp, _vp, _vp, _l, _vp],
    "rkb_eval_orbitals": [_vp, _l, _l, _vp, _i, _i, _i, _i, _vp, _l, _vp],
    "rkb_pair_density": [_vp, _vp, _l, _vp, _l, _l, _vp, _l, _vp],
    "rkb_pack_upper": [_vp, _l, _vp, _vp],
    "rkb_weighted_dots": [_vp, _l, _vp, _l, _vp, _l, _vp, _vp, _l, _vp, _vp],
    "rkb_slater_direct": [_vp, _vp, _vp, _vp, _i, _i, _i, _i, _d, _vp, _vp, _vp, _vp, _vp, _vp],
    "rkb_grid_yk_rows": [_vp, _l, _vp, _l, _vp, _l, _vp, _vp, _vp, _l, _vp, _l, _l, _vp, _l, _vp],
    "rkb_grid_pair_dot_batch": [_vp, _vp, _vp, _vp, _l, _vp, _vp, _vp, _vp, _l, _vp, _l, _vp, _vp, _vp, _l, _vp,
                                _vp, _vp, _l, _vp, _l, _l, _vp, _vp, _l, _vp],
    "rkb_table_rows_fp64": [_vp, _vp, _l, _vp, _vp, _vp, _l, _vp, _vp, _i, _i, _vp, _vp, _vp, _vp, _l, _vp],
    "rkb_table_contract_fp64": [_vp, _vp, _l, _l, _vp, _vp, _vp, _vp, _l, _vp, _vp],
    "rkb_table_contract_fp64_groups": [_vp, _vp, _l, _l, _vp, _vp, _vp, _vp, _vp, _l, _vp, _vp],
    "rkb_split_rows": [_vp, _vp, _l, _vp, _vp, _vp, _l, _vp, _i, _i, _vp, _vp, _i, _i, _vp, _vp, _vp, _l, _l,
                       _l, _vp, _vp, _vp, _vp, _i, _vp, _vp, _vp],
    "rkb_split_rows_noalloc": [_vp, _vp, _l, _vp, _vp, _vp, _l, _vp, _i, _i, _vp, _vp, _i, _i, _vp, _vp, _vp, _l,
                               _l, _l, _vp, _vp, _vp, _vp, _i, _vp, _vp],
    "rkb_split_rows_fused": [_vp, _vp, _l, _vp, _vp, _vp, _l, _vp, _i, _i, _vp, _vp, _i, _i, _i, _vp, _vp, _vp, _l,
                             _l, _l, _vp, _vp, _vp, _vp, _i, _vp],
    "rkb_split_rows_cells": [_vp, _vp, _l, _vp, _vp, _vp, _l, _vp, _i, _i, _vp, _vp, _vp, _vp, _i, _i, _i, _vp, _vp,
                             _vp, _l, _l, _l, _vp, _vp, _vp, _vp, _i, _vp],
    "rkb_split_fused_body_width": [_i, _i],
    "rkb_green_factor": [_vp, _i, _i, _i, _d, _vp, _vp, _vp, _l],
    "rkb_green_tables": [_vp, _i, _i, _vp, _i, _d, _vp, _vp, _i, _i, _vp, _l, _vp, _vp, _l, _vp, _vp],
    "rkb_table_plan": [_vp, _vp, _i, _vp, _i, _l, _l, _vp, _vp, _vp, _vp],
    "rkb_split_certify": [_vp, _vp, _l, _vp, _vp, _d, _vp, _vp, _vp],
    "rkb_occupied_density": [_vp, _vp, _l, _l, _vp, _l, _l, _vp, _vp],
    "rkb_bspline_sym_matrix": [_vp, _i, _vp, _i, _i, _i, _vp, _vp, _l, _vp, _vp],
    "rkb_exchange_matrix": [_vp, _vp, _vp, _vp, _i, _i, _i, _i, _i, _vp, _vp],
    "rkb_gauss_legendre_01": [_i, _vp, _vp],
    "rkb_cell_moments": [_vp, _vp, _vp, _i, _i, _i, _i, _vp, _vp],
    "rkb_cell_diag": [_vp, _vp, _vp, _vp, _vp, _vp, _i, _i, _i, _i, _i, _i, _vp, _vp, _i, _vp, _vp],
    "rkb_cell_assemble": [_vp, _vp, _vp, _vp, _vp, _i, _i, _i, _i, _vp, _l, _l, _l, _vp],
    "rkb_cell_densities": [_vp, _vp, _l, _vp, _l, _i, _i, _i, _i, _i, _vp, _l, _l, _vp],
    "rkb_gemm_nt_fp64": [_vp, _l, _vp, _l, _vp, _l, _l, _l, _l, _i, _vp],
    "rkb_cell_dots": [_vp, _l, _vp, _l, _l, _vp, _vp, _l, _vp, _vp],
    "rkb_cell_exchange": [_vp, _l, _vp, _vp, _l, _i, _i, _i, _i, _i, _vp, _vp],
    "rkb_cell_bilinear": [_vp, _l, _i, _vp, _vp, _i, _i, _i, _i, _i, _vp, _vp, _vp],
    "rkb_cell_direct_density": [_vp, _l, _i, _vp, _l, _vp, _l, _i, _i, _vp, _l, _vp],
    "rkb_cell_exchange_density": [_vp, _vp, _l, _i, _vp, _l, _l, _i, _vp, _vp],
    "rkb_cell_banded_to_full": [_vp, _i, _i, _l, _vp, _vp],
    "rkb_cell_fock_finish": [_vp, _vp, _i, _i, _l, _vp, _vp],
    "rkb_split_contract": [_vp, _vp, _l, _l, _i, _vp, _vp, _vp, _vp, _d, _vp, _vp, _vp, _vp, _d, _i, _i, _vp, _vp,
                           _vp, _vp, _vp, _l, _vp, _vp, _vp],
}
_RESTYPE = {"rkb_last_error": _c.c_char_p, "rkb_version": _c.c_char_p, "rkb_split_fused_body_width": _c.c_long,
            "rkb_green_factor": _c.c_long, "rkb_green_tables": _c.c_long, "rkb_table_plan": _c.c_long, "rkb_gauss_legendre_01": None}

_lock = threading.Lock()
_lib = None


class RkbError(RuntimeError):
    """CUDA runtime failure or unsupported device inside the engine."""


def load():
    """Load (building first if stale) and bind the library; raise if unusable."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        path = _build.LIB_PATH
        if not os.path.exists(path) or os.environ.get("RKB_AUTOBUILD", "1") == "1":
            try:
                path = _build.build()
            except Exception as exc:  # pragma: no cover - toolchain missing
                if not os.path.exists(path):
                    raise RkbError(f"librkb200.so is missing and could not be built: {exc}") from exc
        lib = _c.CDLL(path)
        for name, args in _SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = _RESTYPE.get(name, _c.c_int)
        _lib = lib
        return lib


def lib():
    return load()


def require_device():
    """Raise unless torch sees a CUDA device that the library supports."""
    import torch
    if not torch.cuda.is_available():
        raise RkbError("the rkb200 engine needs a CUDA device (B200, sm_100a); none is visible")
    L = load()
    torch.cuda.current_device()
    if not L.rkb_device_supported():
        raise RkbError("the current CUDA device is not sm_100; librkb200 is built for sm_100a only")
    return L


def check(status: int, what: str = "") -> None:
    if status == 0:
        return
    msg = (load().rkb_last_error() or b"").decode(errors="replace")
    where = f"{what}: " if what else ""
    if status == 1:
        raise ValueError(where + msg)
    if status == 2:
        raise FloatingPointError(where + msg)
    if status == 3:
        raise MemoryError(where + msg)
    if status == 4:
        raise TimeoutError(where + msg)
    raise RkbError(f"{where}status {status}: {msg}")


def ptr(t) -> int:
    """Device (or host) address of a torch tensor, or 0 for None."""
    return 0 if t is None else int(t.data_ptr())


def stream_handle(stream=None) -> int:
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return int(s.cuda_stream)
