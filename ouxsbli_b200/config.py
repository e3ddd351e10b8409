"""SolverConfig: the numerical configuration of one solve (the config.fypp macros
and mod_globals parameters) and its C form (struct oux_config).

This module does not load liboux.so: building a configuration, converting it and
handing it to the CPU oracle need no GPU library.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import abi
from .abi import OuxConfig


@dataclass
class SolverConfig:
    """Numerical configuration (the config.fypp macros + mod_globals parameters)."""

    dim: int = 3
    nx: int = 70
    ny: int = 70
    nz: int = 70
    order: int = 6                 # ORDER
    scheme: str = "SLAU"           # SCHEME: KEEP | SLAU | Roe | Hybrid
    visc: str = "NS"               # VISC: Euler | NS | LES
    visc_order: int = 0            # VISC_ORDER (0 -> ORDER)
    visc_stencil: str = "Central"  # VISC_STENCIL: Central | ME4Base
    tvd: str = "hybrid"            # TVD: none | tvd | hybrid
    slau: str = "HRSLAU2"          # SLAU_VARIANT
    rk: int = 3
    precision: str = "fp64"        # fp64 | mixed (FP32 stage states/fluxes, FP64 Q^n + accumulation)
    bc_x: int = 0                  # 0 periodic; 1 non-periodic x (boundary flux kernels, boundary cells)
    bc_y: int = 0                  # the same for y
    bc_z: int = 0                  # 0 periodic; 1 non-periodic; 2-4 z slab of a larger grid (enum oux_bc_z)
    # rules of the non-periodic faces ("x_lo", "x_hi", "y_lo", "y_hi", "z_lo", "z_hi"):
    # "zero_gradient" (the default), "slip_wall", "noslip_wall", "neumann" or the forms
    # boundary_rules() lists (fixed values, far field, a split face)
    boundary: dict = field(default=None, repr=False)
    boundary_order: str = "x_last"   # x_last: corners take their x rule (OS); y_last: their y rule (BL0)
    gamma: float = 1.4
    R: float = 287.03
    Pr: float = 0.71
    Prt: float = 0.9
    threshold: float = 0.4
    dt: float = 1.0e-3
    dx: np.ndarray = field(default=None, repr=False)
    dy: np.ndarray = field(default=None, repr=False)
    dz: np.ndarray = field(default=None, repr=False)

    @property
    def nv(self) -> int:
        return self.dim + 2

    @property
    def g(self) -> int:
        return self.order // 2

    def interior_cells(self) -> int:
        g = self.g
        gx, gy = (1 if self.bc_x else g), (1 if self.bc_y else g)
        gz = 1 if self.bc_z in (1, 3, 4) else g
        n = (self.nx - 2 * gx) * (self.ny - 2 * gy)
        return n * (self.nz - 2 * gz if self.dim == 3 else 1)

    def boundary_rules(self) -> list[dict]:
        """The non-periodic faces' rules, normalised: per given face a dict with
        face, kind, fixed ((nv, len) values or None), farfield ((rho, u_t, u_n, c) or
        None) and cells (int8 kind per position or None).

        Rule forms: "zero_gradient", "slip_wall", "noslip_wall", "neumann"; ("fixed", values of
        shape (nv, ny) for x faces / (nv, nx) for y faces, of Q/J); ("farfield", rho,
        u_tangential, u_normal, c) on a high face; ("split", at, rule_lo, rule_hi):
        positions below `at` follow rule_lo, the others rule_hi (two of the plain
        names)."""
        out = []
        for name, rule in (self.boundary or {}).items():
            face = abi.FACES[name]
            if self.dim == 3:
                n = (self.ny * self.nz, self.nx * self.nz, self.nx * self.ny)[face // 2]
            else:
                n = self.ny if face < 2 else self.nx
            r = {"face": face, "kind": None, "fixed": None, "farfield": None, "cells": None}
            if isinstance(rule, str):
                r["kind"] = abi.BC_KINDS[rule]
            elif rule[0] == "fixed":
                v = np.ascontiguousarray(rule[1], dtype=np.float64)
                if v.shape != (self.nv, n):
                    raise ValueError(f"fixed values of face {name} must have shape {(self.nv, n)}, got {v.shape}")
                r["kind"], r["fixed"] = abi.BC_KINDS["fixed"], v
            elif rule[0] == "farfield":
                if face not in (abi.FACES["x_hi"], abi.FACES["y_hi"]):
                    raise ValueError("the far-field rule is built for the high faces")
                r["kind"], r["farfield"] = abi.BC_KINDS["farfield"], tuple(float(x) for x in rule[1:5])
            elif rule[0] == "split":
                at, lo, hi = int(rule[1]), abi.BC_KINDS[rule[2]], abi.BC_KINDS[rule[3]]
                cells = np.full(n, hi, dtype=np.int8)
                cells[:max(0, min(at, n))] = lo
                r["kind"], r["cells"] = hi, cells
            else:
                raise ValueError(f"unknown boundary rule {rule!r}")
            out.append(r)
        return out

    def to_c(self) -> tuple[OuxConfig, list]:
        keep = []

        def arr(a):
            a = np.ascontiguousarray(a, dtype=np.float64)
            keep.append(a)
            return a.ctypes.data_as(C.POINTER(C.c_double))

        c = OuxConfig()
        c.dim, c.nx, c.ny = self.dim, self.nx, self.ny
        c.nz = self.nz if self.dim == 3 else 1
        c.order = self.order
        c.scheme = abi.SCHEMES[self.scheme]
        c.visc = abi.VISC[self.visc]
        c.visc_order = self.visc_order
        c.visc_stencil = abi.STENCILS[self.visc_stencil]
        c.tvd = abi.TVD[self.tvd]
        c.slau = abi.SLAU_VARIANTS[self.slau]
        c.rk = self.rk
        c.bc_x = self.bc_x
        c.bc_y = self.bc_y
        c.bc_z = self.bc_z if self.dim == 3 else 0
        c.precision = abi.PRECISION[self.precision]
        c.gamma, c.R, c.Pr, c.Prt, c.threshold, c.dt = (self.gamma, self.R, self.Pr, self.Prt,
                                                         self.threshold, self.dt)
        c.dx = arr(self.dx)
        c.dy = arr(self.dy)
        c.dz = arr(self.dz) if self.dim == 3 else arr(np.zeros(1))
        return c, keep
