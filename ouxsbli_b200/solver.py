"""Solver: one periodic solve driven through liboux's C ABI.

Device memory is PyTorch-owned (torch is the allocator and stream provider, the
library never calls cudaMalloc for a solve).  The hot path is entirely inside
liboux; this class only carries pointers and sizes across the boundary.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from ._lib import LIB, OuxConfig, check


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
            face = _lib.FACES[name]
            if self.dim == 3:
                n = (self.ny * self.nz, self.nx * self.nz, self.nx * self.ny)[face // 2]
            else:
                n = self.ny if face < 2 else self.nx
            r = {"face": face, "kind": None, "fixed": None, "farfield": None, "cells": None}
            if isinstance(rule, str):
                r["kind"] = _lib.BC_KINDS[rule]
            elif rule[0] == "fixed":
                v = np.ascontiguousarray(rule[1], dtype=np.float64)
                if v.shape != (self.nv, n):
                    raise ValueError(f"fixed values of face {name} must have shape {(self.nv, n)}, got {v.shape}")
                r["kind"], r["fixed"] = _lib.BC_KINDS["fixed"], v
            elif rule[0] == "farfield":
                if face not in (_lib.FACES["x_hi"], _lib.FACES["y_hi"]):
                    raise ValueError("the far-field rule is built for the high faces")
                r["kind"], r["farfield"] = _lib.BC_KINDS["farfield"], tuple(float(x) for x in rule[1:5])
            elif rule[0] == "split":
                at, lo, hi = int(rule[1]), _lib.BC_KINDS[rule[2]], _lib.BC_KINDS[rule[3]]
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
        c.scheme = _lib.SCHEMES[self.scheme]
        c.visc = _lib.VISC[self.visc]
        c.visc_order = self.visc_order
        c.visc_stencil = _lib.STENCILS[self.visc_stencil]
        c.tvd = _lib.TVD[self.tvd]
        c.slau = _lib.SLAU_VARIANTS[self.slau]
        c.rk = self.rk
        c.bc_x = self.bc_x
        c.bc_y = self.bc_y
        c.bc_z = self.bc_z if self.dim == 3 else 0
        c.precision = _lib.PRECISION[self.precision]
        c.gamma, c.R, c.Pr, c.Prt, c.threshold, c.dt = (self.gamma, self.R, self.Pr, self.Prt,
                                                         self.threshold, self.dt)
        c.dx = arr(self.dx)
        c.dy = arr(self.dy)
        c.dz = arr(self.dz) if self.dim == 3 else arr(np.zeros(1))
        return c, keep


class Solver:
    """A bound liboux handle with its device state and scratch.

    `device` must be a CUDA device; the CUDA library is the only implementation.
    """

    def __init__(self, cfg: SolverConfig, device: str | torch.device = "cuda:0"):
        self.cfg = cfg
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise RuntimeError("liboux runs on a CUDA device only (no CPU fallback)")
        c, keep = cfg.to_c()
        h = C.c_void_p()
        check(LIB.oux_create(C.byref(c), C.byref(h)))
        self._h = h
        sb, kb = C.c_size_t(), C.c_size_t()
        check(LIB.oux_state_bytes(C.byref(c), C.byref(sb)))
        check(LIB.oux_scratch_bytes(C.byref(c), C.byref(kb)))
        del keep
        self.state = torch.empty(sb.value // 8, dtype=torch.float64, device=self.device)
        self.scratch = torch.empty((kb.value + 7) // 8, dtype=torch.float64, device=self.device)
        self.stream = torch.cuda.current_stream(self.device)
        with torch.cuda.device(self.device):
            check(LIB.oux_bind(self._h, C.c_void_p(self.state.data_ptr()), C.c_void_p(self.scratch.data_ptr()),
                               C.c_size_t(self.scratch.numel() * 8), C.c_void_p(self.stream.cuda_stream)))
        lay = _lib.OuxLayout()
        check(LIB.oux_layout_of(self._h, C.byref(lay)))
        self.layout = lay
        self._bfix = {}  # device copies of boundary values / kinds (the library reads them every fill)
        for r in cfg.boundary_rules():
            face = r["face"]
            if r["farfield"] is not None:
                check(LIB.oux_set_boundary_farfield(self._h, face, *r["farfield"]))
            else:
                ptr = None
                if r["fixed"] is not None:
                    t = torch.from_numpy(r["fixed"].ravel()).to(self.device)
                    self._bfix[face] = t
                    ptr = C.c_void_p(t.data_ptr())
                check(LIB.oux_set_boundary(self._h, face, r["kind"], ptr))
            if r["cells"] is not None:
                t = torch.from_numpy(r["cells"]).to(self.device)
                self._bfix[("cells", face)] = t
                check(LIB.oux_set_boundary_cells(self._h, face, C.c_void_p(t.data_ptr())))
        check(LIB.oux_set_boundary_order(self._h, 1 if cfg.boundary_order == "y_last" else 0))

    # -- lifetime --
    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            LIB.oux_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _s(self) -> C.c_void_p:
        return C.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    # -- state transfer (reference layout QJ(nx,nv,ny[,nz]), Fortran order) --
    def set_state(self, qj: np.ndarray) -> None:
        a = np.asfortranarray(qj, dtype=np.float64)
        self._keep = a  # the copy is asynchronous: keep the host buffer alive
        with torch.cuda.device(self.device):
            check(LIB.oux_set_state(self._h, a.ctypes.data_as(C.POINTER(C.c_double)), self._s()))
            torch.cuda.current_stream(self.device).synchronize()
        self._keep = None

    def get_state(self) -> np.ndarray:
        c = self.cfg
        shape = (c.nx, c.nv, c.ny, c.nz) if c.dim == 3 else (c.nx, c.nv, c.ny)
        out = np.empty(shape, dtype=np.float64, order="F")
        with torch.cuda.device(self.device):
            check(LIB.oux_get_state(self._h, out.ctypes.data_as(C.POINTER(C.c_double)), self._s()))
        return out

    # -- hot path --
    def step(self, nsteps: int = 1) -> None:
        with torch.cuda.device(self.device):
            check(LIB.oux_step(self._h, int(nsteps), self._s()))

    def fill_ghosts(self) -> None:
        with torch.cuda.device(self.device):
            check(LIB.oux_fill_ghosts(self._h, self._s()))

    def rhs(self) -> np.ndarray:
        """The stage residual of the current state in the reference's Rs order."""
        c = self.cfg
        n = c.nv * (c.nx - 2) * (c.ny - 2) * ((c.nz - 2) if c.dim == 3 else 1)
        out = torch.zeros(n, dtype=torch.float64, device=self.device)
        with torch.cuda.device(self.device):
            check(LIB.oux_rhs(self._h, C.c_void_p(out.data_ptr()), self._s()))
        shape = (c.nx - 2, c.nv, c.ny - 2, c.nz - 2) if c.dim == 3 else (c.nx - 2, c.nv, c.ny - 2)
        return out.cpu().numpy().reshape(shape[::-1]).transpose(tuple(range(len(shape)))[::-1])

    def diagnostics(self) -> tuple[float, float, float]:
        out = (C.c_double * 3)()
        with torch.cuda.device(self.device):
            check(LIB.oux_diagnostics(self._h, out, self._s()))
        return out[0], out[1], out[2]

    def check_state(self) -> int:
        bits = C.c_int32()
        with torch.cuda.device(self.device):
            rc = LIB.oux_check_state(self._h, C.byref(bits), self._s())
        if rc not in (_lib.OUX_OK, _lib.OUX_E_DEVICE_FAULT):
            check(rc)
        return bits.value

    def launches(self) -> int:
        n = C.c_int64()
        check(LIB.oux_launch_count(self._h, C.byref(n)))
        return n.value
