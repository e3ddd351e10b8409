"""Initial- and boundary-condition specifications accepted by ``Case(ic=..., bc=...)``.

Same names, fields and parameter mapping as the reference's ouxsbli/ic.py:20-215.
In the reference these map to mod_globals.f90 parameters that no set.f90 reads
(the case's own set_init decides the field); here ``TaylorGreenIC`` and
``UniformIC`` do select the initial field of the periodic 3D cases, and
``RiemannIC`` is accepted but needs a non-periodic case (not built).
"""
from __future__ import annotations

from dataclasses import dataclass

_IC_UNIFORM = 1
_IC_TAYLOR_GREEN = 2
_IC_RIEMANN = 3


@dataclass
class UniformIC:
    rho: float = 1.0
    u: float = 0.0
    v: float = 0.0
    w: float = 0.0
    p: float = 0.71429

    def to_params(self) -> dict:
        return {"ic_type": _IC_UNIFORM, "rho0": self.rho, "u0": self.u, "v0": self.v, "w0": self.w, "p0": self.p}


@dataclass
class TaylorGreenIC:
    Ma: float = 0.1
    rho0: float = 1.0
    p0: float = 0.71429

    def to_params(self) -> dict:
        return {"ic_type": _IC_TAYLOR_GREEN, "Ma": self.Ma, "rho0": self.rho0, "p0": self.p0}


@dataclass
class RiemannIC:
    rho_l: float = 1.0
    u_l: float = 0.0
    p_l: float = 1.0
    rho_r: float = 0.125
    u_r: float = 0.0
    p_r: float = 0.1
    x0: float = 0.5

    def to_params(self) -> dict:
        return {"ic_type": _IC_RIEMANN, "rho_l": self.rho_l, "u_l": self.u_l, "p_l": self.p_l,
                "rho_r": self.rho_r, "u_r": self.u_r, "p_r": self.p_r, "x0_frac": self.x0}


@dataclass
class PeriodicBC:
    """Fully periodic boundaries (BC_X = BC_Y = BC_Z = False)."""

    def to_params(self) -> dict:
        return {"BC_X": False, "BC_Y": False, "BC_Z": False}


def _ic_from_dict(d: dict):
    d = dict(d)
    kind = str(d.pop("type", "uniform")).lower()
    table = {"uniform": UniformIC, "tgv": TaylorGreenIC, "taylor_green": TaylorGreenIC, "riemann": RiemannIC}
    if kind not in table:
        raise ValueError(f"Unknown IC type: {kind!r}.  Supported: 'uniform', 'tgv', 'riemann'.")
    cls = table[kind]
    return cls(**{k: v for k, v in d.items() if k in cls.__dataclass_fields__})


def ic_to_params(ic) -> dict:
    if isinstance(ic, dict):
        ic = _ic_from_dict(ic)
    if hasattr(ic, "to_params"):
        return ic.to_params()
    raise TypeError(f"Unsupported IC specification: {type(ic)!r}")


def bc_to_params(bc) -> dict:
    if isinstance(bc, str):
        if bc.lower() == "periodic":
            return PeriodicBC().to_params()
        raise ValueError(f"Unknown BC type string: {bc!r}.  Supported: 'periodic'.")
    if isinstance(bc, dict):
        kind = str(bc.get("type", "periodic")).lower()
        if kind == "periodic":
            return PeriodicBC().to_params()
        raise ValueError(f"Unknown BC type: {kind!r}.")
    if hasattr(bc, "to_params"):
        return bc.to_params()
    raise TypeError(f"Unsupported BC specification: {type(bc)!r}")
