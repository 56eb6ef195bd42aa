"""ctypes binding of ``libtopo_b200.so`` (the C ABI in ``include/topo_b200.h``).

The library is the only compute path: if it is missing or a call fails,
this module raises; there is no CPU fallback.
"""

from __future__ import annotations

import ctypes as C
from pathlib import Path

import os

# TOPO_B200_LIB=dbg loads the range-checked build (python -m topogpu_b200.build --debug-bounds)
_LIB_PATH = Path(__file__).resolve().parent / (
    "libtopo_b200_dbg.so" if os.environ.get("TOPO_B200_LIB") == "dbg" else "libtopo_b200.so")
_lib = None

F64, F32, BF16, BF16_F32IN = 0, 1, 2, 3
EPI_STORE, EPI_RESIDUAL, EPI_CHEB, EPI_RUPD = 0, 1, 2, 4
MODE_FP64, MODE_FP32, MODE_MIXED = 0, 1, 2
MODES = {"fp64": MODE_FP64, "fp32": MODE_FP32, "mixed": MODE_MIXED}

_vp = C.c_void_p
_i = C.c_int
_d = C.c_double
_ll = C.c_longlong

# name -> (restype, argtypes); mirrors include/topo_b200.h
SIGNATURES = {
    "topo_version": (_i, []),
    "topo_ctx_create": (_i, [_i, _i, _i, _i, _i, _i, _i, _d, _i, _vp, C.POINTER(_vp)]),
    "topo_ctx_destroy": (_i, [_vp]),
    "topo_set_smoother": (_i, [_vp, _i, _d]),
    "topo_last_error": (_i, [_vp, C.c_char_p, _i]),
    "topo_set_problem": (_i, [_vp, _vp, _vp, _vp]),
    "topo_modulus": (_i, [_vp, _vp, _d, _d, _d, _vp, _vp]),
    "topo_matvec": (_i, [_vp, _i, _vp, _vp, _vp, _vp]),
    "topo_level0_apply": (_i, [_vp, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _d, _d, _d, _d, _vp]),
    "topo_wait_status": (_i, [_vp, _vp]),
    "topo_debug_tc_wait": (_i, [_i, _i]),
    "topo_debug_bounds": (_i, [C.POINTER(_i)]),
    "topo_diag": (_i, [_vp, _vp, _vp, _vp]),
    "topo_gmg_setup": (_i, [_vp, _vp, _vp]),
    "topo_gmg_apply": (_i, [_vp, _vp, _vp, _vp]),
    "topo_pcg": (_i, [_vp, _vp, _vp, _d, _i, C.POINTER(_i), C.POINTER(_d), _vp]),
    "topo_fgmres": (_i, [_vp, _vp, _vp, _d, _i, _i, C.POINTER(_i), C.POINTER(_d), _vp]),
    "topo_set_coarse_lag": (_i, [_vp, _i]),
    "topo_set_tc": (_i, [_vp, _i]),
    "topo_set_cycle": (_i, [_vp, _i]),
    "topo_block_pcg": (_i, [_vp, _vp, _vp, _i, _d, _i, C.POINTER(_i), C.POINTER(_d), _vp]),
    "topo_sensitivity": (_i, [_vp, _vp, _i, _vp, _d, _d, _d, _vp, _vp]),
    "topo_sensitivity_adjoint": (_i, [_vp, _vp, _vp, _i, _vp, _d, _d, _d, _vp, _vp]),
    "topo_dot": (_i, [_vp, _i, _vp, _vp, _ll, C.POINTER(_d), _vp]),
    "topo_filter": (_i, [_vp, _d, _vp, _vp, _i, _vp]),
    "topo_oc": (_i, [_vp, _vp, _vp, _d, _d, _d, _vp, C.POINTER(_i), _vp]),
    "topo_oc_filtered": (_i, [_vp, _vp, _vp, _vp, _vp, _d, _d, _d, _vp, C.POINTER(_i), _vp]),
    "topo_heaviside": (_i, [_vp, _vp, _d, _d, _vp, _vp, _vp]),
    "topo_oc_projected": (_i, [_vp, _d, _vp, _vp, _vp, _d, _d, _d, _d, _d, _vp, C.POINTER(_i), _vp]),
    "topo_oc_noalloc": (_i, [_vp, _vp, _ll, _d, _d, _d, _vp, C.POINTER(_i), _vp]),
    "topo_field_stats": (_i, [_vp, _vp, _ll, C.POINTER(_d), _vp]),
    "topo_gmg_info": (_i, [_vp, C.POINTER(_ll), C.POINTER(_d), C.POINTER(_i)]),
    "topo_setup_phases": (_i, [_vp, C.POINTER(_d)]),
    "topo_gmg_level_operator": (_i, [_vp, _i, _vp, _vp]),
    "topo_workspace_bytes": (_ll, [_vp]),
    "topo_launch_count": (_ll, []),
}


def lib_path() -> Path:
    return _LIB_PATH


def load():
    """Load the shared library (once) and declare every entry point."""
    global _lib
    if _lib is not None:
        return _lib
    if not _LIB_PATH.exists():
        raise RuntimeError(
            f"{_LIB_PATH.name} is not built; run `python -m topogpu_b200.build` (nvcc, sm_100a)."
        )
    lib = C.CDLL(str(_LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def last_error(ctx=None) -> str:
    lib = load()
    buf = C.create_string_buffer(4096)
    lib.topo_last_error(ctx, buf, 4096)
    return buf.value.decode(errors="replace")


def check(rc: int, ctx=None, what: str = "call") -> int:
    """Raise on a negative status; return non-negative statuses to the caller."""
    if rc < 0:
        raise RuntimeError(f"libtopo_b200 {what} failed: {last_error(ctx)}")
    return rc
