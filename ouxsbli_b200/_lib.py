"""ctypes binding of liboux.so (include/oux.h).

The library is required: importing this module raises if liboux.so has not been
built (``python -m ouxsbli_b200.build``).  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import pathlib

import os

# OUX_LIB may point at another build of the same library (e.g. a tuning variant)
LIB_PATH = pathlib.Path(os.environ.get("OUX_LIB") or (pathlib.Path(__file__).resolve().parent / "liboux.so"))

from .abi import *  # noqa: F401,F403  (enum tables, structures, SYMBOLS)
from .abi import OuxBatchTuning, OuxConfig, OuxLayout


class OuxError(RuntimeError):
    """A liboux call returned a negative status."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"liboux error {code}: {msg}")
        self.code = code


def _load() -> C.CDLL:
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is missing: build the CUDA library with `python -m ouxsbli_b200.build` "
            "(there is no CPU fallback)")
    lib = C.CDLL(str(LIB_PATH))
    vp, i32, i64, dp = C.c_void_p, C.c_int32, C.c_int64, C.POINTER(C.c_double)
    cfgp = C.POINTER(OuxConfig)
    sig = {
        "oux_create": (C.c_int, [cfgp, C.POINTER(vp)]),
        "oux_destroy": (C.c_int, [vp]),
        "oux_last_error": (C.c_char_p, []),
        "oux_abi_version": (C.c_int, []),
        "oux_state_bytes": (C.c_int, [cfgp, C.POINTER(C.c_size_t)]),
        "oux_scratch_bytes": (C.c_int, [cfgp, C.POINTER(C.c_size_t)]),
        "oux_layout_of": (C.c_int, [vp, C.POINTER(OuxLayout)]),
        "oux_bind": (C.c_int, [vp, vp, vp, C.c_size_t, vp]),
        "oux_set_state": (C.c_int, [vp, dp, vp]),
        "oux_get_state": (C.c_int, [vp, dp, vp]),
        "oux_get_state_async": (C.c_int, [vp, dp, vp]),
        "oux_pack_state": (C.c_int, [vp, dp, vp]),
        "oux_unpack_state": (C.c_int, [vp, vp, dp]),
        "oux_set_boundary": (C.c_int, [vp, C.c_int32, C.c_int32, vp]),
        "oux_set_boundary_farfield": (C.c_int, [vp, C.c_int32, C.c_double, C.c_double, C.c_double, C.c_double]),
        "oux_set_boundary_cells": (C.c_int, [vp, C.c_int32, vp]),
        "oux_set_boundary_order": (C.c_int, [vp, C.c_int32]),
        "oux_stage": (C.c_int, [vp, C.c_int32, vp]),
        "oux_stage_part": (C.c_int, [vp, C.c_int32, C.c_int32, vp]),
        "oux_halo_bytes": (C.c_int, [vp, C.c_int32, C.POINTER(C.c_size_t)]),
        "oux_halo_pack": (C.c_int, [vp, C.c_int32, vp, vp, vp]),
        "oux_halo_unpack": (C.c_int, [vp, C.c_int32, vp, vp, vp]),
        "oux_fill_ghosts": (C.c_int, [vp, vp]),
        "oux_rhs": (C.c_int, [vp, vp, vp]),
        "oux_step": (C.c_int, [vp, i32, vp]),
        "oux_diagnostics": (C.c_int, [vp, dp, vp]),
        "oux_check_state": (C.c_int, [vp, C.POINTER(i32), vp]),
        "oux_status": (C.c_int, [vp, C.POINTER(i32)]),
        "oux_profile": (C.c_int, [vp, i32]),
        "oux_profile_read": (C.c_int, [vp, dp, C.POINTER(i64), i32]),
        "oux_host_ref_diagnostics": (C.c_int, [i32, i32, i32, i32, C.c_double, C.POINTER(C.c_float),
                                               C.POINTER(C.c_float), C.POINTER(C.c_float), dp]),
        "oux_launch_count": (C.c_int, [vp, C.POINTER(i64)]),
        "oux_rhs_noalloc": (C.c_int, [cfgp, vp, vp, vp]),
        "oux_batch_create": (C.c_int, [C.POINTER(vp), i32, C.POINTER(OuxBatchTuning), C.POINTER(vp)]),
        "oux_batch_workspace_bytes": (C.c_int, [vp, C.POINTER(C.c_size_t)]),
        "oux_batch_bind": (C.c_int, [vp, vp, C.c_size_t, vp]),
        "oux_batch_step": (C.c_int, [vp, i32, vp]),
        "oux_batch_status": (C.c_int, [vp, C.POINTER(i32)]),
        "oux_batch_info": (C.c_int, [vp, C.POINTER(i64), C.POINTER(i32), C.POINTER(i32)]),
        "oux_batch_set_spin_limit": (C.c_int, [vp, i32]),
        "oux_batch_dep_offset": (C.c_int, [vp, i32, i32, C.POINTER(C.c_size_t)]),
        "oux_batch_destroy": (C.c_int, [vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


LIB = _load()


def check(rc: int) -> int:
    if rc != OUX_OK:
        msg = LIB.oux_last_error()
        raise OuxError(rc, msg.decode() if msg else "")
    return rc
