"""Constants and ctypes structures of the C ABI (include/oux.h).

Importing this module does not load liboux.so, so configurations can be built
and validated by code that must not map the CUDA library (the CPU-only parts of
the benchmark); ``ouxsbli_b200._lib`` re-exports every name and loads the library.
"""
from __future__ import annotations

import ctypes as C

OUX_OK = 0
OUX_E_INVALID = -1
OUX_E_CUDA = -2
OUX_E_UNBOUND = -3
OUX_E_TOO_SMALL = -4
OUX_E_DEVICE_FAULT = -5

SCHEMES = {"KEEP": 0, "SLAU": 1, "Roe": 2, "Hybrid": 3}
VISC = {"Euler": 0, "NS": 1, "LES": 2}
STENCILS = {"Central": 0, "ME4Base": 1}
TVD = {"none": 0, "tvd": 1, "hybrid": 2}
SLAU_VARIANTS = {"SLAU": 0, "HRSLAU2": 1}
PRECISION = {"fp64": 0, "mixed": 1}

FAULT_NAN = 1
FAULT_NONPOSITIVE = 2
FAULT_TIMEOUT = 4

# exported symbols, in include/oux.h order
SYMBOLS = [
    "oux_create", "oux_destroy", "oux_last_error", "oux_abi_version", "oux_state_bytes",
    "oux_scratch_bytes", "oux_layout_of", "oux_bind", "oux_set_state", "oux_get_state",
    "oux_pack_state", "oux_unpack_state", "oux_set_boundary", "oux_fill_ghosts", "oux_rhs",
    "oux_stage", "oux_stage_part", "oux_halo_bytes", "oux_halo_pack", "oux_halo_unpack",
    "oux_set_boundary_farfield", "oux_set_boundary_cells", "oux_set_boundary_order", "oux_step", "oux_get_state_async",
    "oux_diagnostics", "oux_check_state", "oux_status", "oux_profile", "oux_profile_read",
    "oux_host_ref_diagnostics", "oux_launch_count", "oux_rhs_noalloc",
    "oux_batch_create", "oux_batch_workspace_bytes", "oux_batch_bind", "oux_batch_step",
    "oux_batch_status", "oux_batch_info", "oux_batch_set_spin_limit", "oux_batch_dep_offset",
    "oux_batch_destroy",
]
NOALLOC_SCRATCH_BYTES = 32 << 20  # OUX_NOALLOC_SCRATCH_BYTES
FACES = {"x_lo": 0, "x_hi": 1, "y_lo": 2, "y_hi": 3, "z_lo": 4, "z_hi": 5}  # enum oux_face
BC_KINDS = {"zero_gradient": 0, "slip_wall": 1, "fixed": 2, "noslip_wall": 3, "farfield": 4,
            "neumann": 5}  # enum oux_bc_kind


class OuxConfig(C.Structure):
    _fields_ = [
        ("dim", C.c_int32), ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
        ("order", C.c_int32), ("scheme", C.c_int32), ("visc", C.c_int32), ("visc_order", C.c_int32),
        ("visc_stencil", C.c_int32), ("tvd", C.c_int32), ("slau", C.c_int32), ("rk", C.c_int32),
        ("bc_x", C.c_int32), ("bc_y", C.c_int32), ("bc_z", C.c_int32), ("precision", C.c_int32),
        ("gamma", C.c_double), ("R", C.c_double), ("Pr", C.c_double), ("Prt", C.c_double),
        ("threshold", C.c_double), ("dt", C.c_double),
        ("dx", C.POINTER(C.c_double)), ("dy", C.POINTER(C.c_double)), ("dz", C.POINTER(C.c_double)),
    ]


class OuxLayout(C.Structure):
    _fields_ = [("nv", C.c_int32), ("row_stride", C.c_int64), ("plane_stride", C.c_int64),
                ("var_stride", C.c_int64), ("elem_bytes", C.c_int64)]


class OuxBatchTuning(C.Structure):
    _fields_ = [("pencil", C.c_int32), ("chunk", C.c_int32), ("blocks_per_sm", C.c_int32),
                ("use_graph", C.c_int32), ("mode", C.c_int32)]


BATCH_MODES = {"persistent": 0, "graph": 1}
