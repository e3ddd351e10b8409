"""B200-native (sm_100a) explicit compressible-flow time step with the ouxsbli Case API.

Public names mirror the reference package (`ouxsbli/__init__.py`): Case, patch,
UniformIC, TaylorGreenIC, RiemannIC, PeriodicBC.  The solver itself lives in
liboux.so (C ABI, include/oux.h); this package is its host-side driver.
Attributes are imported lazily so that `ouxsbli_b200.build` works before the
CUDA library exists.
"""
from __future__ import annotations

import importlib

__all__ = ["Case", "patch", "UniformIC", "TaylorGreenIC", "RiemannIC", "PeriodicBC",
           "Solver", "SolverConfig", "build"]

_LAZY = {
    "Case": ("ouxsbli_b200.case", "Case"),
    "patch": ("ouxsbli_b200.patcher", "patch"),
    "UniformIC": ("ouxsbli_b200.ic", "UniformIC"),
    "TaylorGreenIC": ("ouxsbli_b200.ic", "TaylorGreenIC"),
    "RiemannIC": ("ouxsbli_b200.ic", "RiemannIC"),
    "PeriodicBC": ("ouxsbli_b200.ic", "PeriodicBC"),
    "Solver": ("ouxsbli_b200.solver", "Solver"),
    "SolverConfig": ("ouxsbli_b200.config", "SolverConfig"),
    "build": ("ouxsbli_b200.build", "build"),
}


def __getattr__(name):
    if name in _LAZY:
        mod, attr = _LAZY[name]
        return getattr(importlib.import_module(mod), attr)
    raise AttributeError(name)
