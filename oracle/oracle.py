"""ctypes wrapper of the CPU oracle (oracle.cpp) -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs import
this module; the product package never does.  See oracle.cpp for what the
restatement follows and its parity status.
"""
from __future__ import annotations

import ctypes as C
import os
import pathlib
import subprocess

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
SRC = HERE / "oracle.cpp"
LIB_PATH = HERE / "liboracle.so"
# -ffp-contract=off: no fused multiply-add, so the oracle evaluates exactly the
# operations written; x86-64-v3 keeps the shared object portable to other hosts.
CFLAGS = ["-O3", "-march=x86-64-v3", "-ffp-contract=off", "-fopenmp", "-std=c++17", "-fPIC", "-shared"]

SCHEMES = {"KEEP": 0, "SLAU": 1, "Roe": 2, "Hybrid": 3}
VISC = {"Euler": 0, "NS": 1, "LES": 2}
STENCILS = {"Central": 0, "ME4Base": 1}
TVD = {"none": 0, "tvd": 1, "hybrid": 2}
SLAU_VARIANTS = {"SLAU": 0, "HRSLAU2": 1}


def build(force: bool = False) -> pathlib.Path:
    if force or not LIB_PATH.exists() or LIB_PATH.stat().st_mtime < SRC.stat().st_mtime:
        cmd = ["g++", *CFLAGS, "-o", str(LIB_PATH), str(SRC)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"oracle build failed:\n{r.stderr}")
    return LIB_PATH


class _Cfg(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("dim", "nx", "ny", "nz", "order", "scheme", "visc", "visc_order",
                                       "visc_stencil", "tvd", "slau", "rk", "bc_x")] + \
               [(n, C.c_double) for n in ("gamma", "R", "Pr", "Prt", "threshold", "dt")] + \
               [("bc_y", C.c_int), ("bkind", C.c_int * 4), ("bfix", C.POINTER(C.c_double) * 4), ("bc_z", C.c_int),
                ("ylast", C.c_int), ("bkinds", C.POINTER(C.c_int8) * 4), ("bpar", (C.c_double * 4) * 4),
                ("bkindz", C.c_int * 2), ("bfix3", C.POINTER(C.c_double) * 6)]


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(str(LIB_PATH))
        dp = C.POINTER(C.c_double)
        cp = C.POINTER(_Cfg)
        _lib.orc_step.argtypes = [cp, dp, dp, dp, dp, C.c_int]
        _lib.orc_rhs.argtypes = [cp, dp, dp, dp, dp, dp]
        _lib.orc_fields.argtypes = [cp, dp, dp, dp, dp, dp]
        _lib.orc_jacobian.argtypes = [cp, dp, dp, dp, dp]
        _lib.orc_fill_ghosts.argtypes = [cp, dp, dp, dp, dp]
        _lib.orc_stage.argtypes = [cp, dp, dp, dp, dp, dp, dp, C.c_int]
        _lib.orc_diag_f32.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_double,
                                      C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float), dp]
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def make_cfg(cfg) -> _Cfg:
    """Build the oracle config from an object with the SolverConfig attributes."""
    c = _Cfg()
    c.dim, c.nx, c.ny = cfg.dim, cfg.nx, cfg.ny
    c.nz = cfg.nz if cfg.dim == 3 else 1
    c.order = cfg.order
    c.scheme = SCHEMES[cfg.scheme]
    c.visc = VISC[cfg.visc]
    # unset: the order in 3D, 4 if the order is at least 4 else 2 in 2D (as the library)
    c.visc_order = cfg.visc_order or (cfg.order if cfg.dim == 3 else (4 if cfg.order >= 4 else 2))
    c.visc_stencil = STENCILS[cfg.visc_stencil]
    c.tvd = TVD[cfg.tvd]
    c.slau = SLAU_VARIANTS[cfg.slau]
    c.rk = cfg.rk
    c.bc_x = getattr(cfg, "bc_x", 0)
    c.bc_y = getattr(cfg, "bc_y", 0)
    c.bc_z = getattr(cfg, "bc_z", 0)
    c._keep = []
    rules = cfg.boundary_rules() if hasattr(cfg, "boundary_rules") else []
    for r in rules:
        face = r["face"]
        if face < 4:
            c.bkind[face] = r["kind"]
        else:
            c.bkindz[face - 4] = r["kind"]
        if r["fixed"] is not None:
            c._keep.append(r["fixed"])
            if cfg.dim == 3:
                c.bfix3[face] = _ptr(r["fixed"])
            else:
                c.bfix[face] = _ptr(r["fixed"])
        if r["farfield"] is not None:
            for q in range(4):
                c.bpar[face][q] = r["farfield"][q]
        if r["cells"] is not None:
            c._keep.append(r["cells"])
            c.bkinds[face] = r["cells"].ctypes.data_as(C.POINTER(C.c_int8))
    c.ylast = 1 if getattr(cfg, "boundary_order", "x_last") == "y_last" else 0
    c.gamma, c.R, c.Pr, c.Prt, c.threshold, c.dt = cfg.gamma, cfg.R, cfg.Pr, cfg.Prt, cfg.threshold, cfg.dt
    return c


def _axes(cfg):
    dx = np.ascontiguousarray(cfg.dx, dtype=np.float64)
    dy = np.ascontiguousarray(cfg.dy, dtype=np.float64)
    dz = np.ascontiguousarray(cfg.dz if cfg.dim == 3 else np.zeros(1), dtype=np.float64)
    return dx, dy, dz


def step(cfg, qj: np.ndarray, nsteps: int, threads: int | None = None) -> np.ndarray:
    """Advance a copy of qj (reference layout, Fortran order) by nsteps."""
    if threads is not None:
        os.environ["OMP_NUM_THREADS"] = str(threads)
    q = np.asfortranarray(qj, dtype=np.float64).copy(order="F")
    dx, dy, dz = _axes(cfg)
    c = make_cfg(cfg)
    rc = lib().orc_step(C.byref(c), _ptr(dx), _ptr(dy), _ptr(dz), _ptr(q), int(nsteps))
    assert rc == 0
    return q


def rhs(cfg, qj: np.ndarray) -> np.ndarray:
    """Stage residual (coef 1) in the reference's Rs(nx-2,nv,ny-2[,nz-2]) order."""
    q = np.asfortranarray(qj, dtype=np.float64)
    dx, dy, dz = _axes(cfg)
    nv = cfg.dim + 2
    shape = (cfg.nx - 2, nv, cfg.ny - 2, cfg.nz - 2) if cfg.dim == 3 else (cfg.nx - 2, nv, cfg.ny - 2)
    out = np.zeros(shape, dtype=np.float64, order="F")
    c = make_cfg(cfg)
    lib().orc_rhs(C.byref(c), _ptr(dx), _ptr(dy), _ptr(dz), _ptr(q), _ptr(out))
    return out


def fields(cfg, qj: np.ndarray) -> dict:
    q = np.asfortranarray(qj, dtype=np.float64)
    dx, dy, dz = _axes(cfg)
    n = cfg.nx * cfg.ny * (cfg.nz if cfg.dim == 3 else 1)
    out = np.zeros(10 * n)
    c = make_cfg(cfg)
    lib().orc_fields(C.byref(c), _ptr(dx), _ptr(dy), _ptr(dz), _ptr(q), _ptr(out))
    names = ["rho", "u", "v", "w", "p", "T", "mu", "sensor", "mut", "qc2"]
    shp = (cfg.nx, cfg.ny, cfg.nz) if cfg.dim == 3 else (cfg.nx, cfg.ny)
    return {nm: out[i * n:(i + 1) * n].reshape(shp, order="F") for i, nm in enumerate(names)}


class Stepper:
    """Stage-by-stage stepping of one state (orc_stage), for z slabs that exchange
    halo planes between stages.  q (Q^n) and q2 (the stage state) are Fortran-order
    arrays in the reference layout; rs is the RK4 accumulator."""

    def __init__(self, cfg, qj: np.ndarray):
        self.cfg = cfg
        self.c = make_cfg(cfg)
        self.dx, self.dy, self.dz = _axes(cfg)
        self.q = np.asfortranarray(qj, dtype=np.float64).copy(order="F")
        self.q2 = self.q.copy(order="F")
        nv = cfg.dim + 2
        shape = (cfg.nx - 2, nv, cfg.ny - 2, cfg.nz - 2) if cfg.dim == 3 else (cfg.nx - 2, nv, cfg.ny - 2)
        self.rs = np.zeros(shape, order="F")

    @property
    def stages(self) -> int:
        return 3 if self.cfg.rk == 3 else 4

    def written(self, stage: int) -> np.ndarray:
        """The array stage `stage` writes (Q^{n+1} after the last stage)."""
        return self.q if stage == self.stages - 1 else self.q2

    def stage(self, st: int) -> None:
        rc = lib().orc_stage(C.byref(self.c), _ptr(self.dx), _ptr(self.dy), _ptr(self.dz), _ptr(self.q),
                             _ptr(self.q2), _ptr(self.rs), int(st))
        assert rc == 0


def fill_ghosts(cfg, qj: np.ndarray) -> np.ndarray:
    """A copy of qj with its ghost / boundary cells set (periodic images and the
    boundary-cell rules of the non-periodic faces)."""
    q = np.asfortranarray(qj, dtype=np.float64).copy(order="F")
    c = make_cfg(cfg)
    dx, dy, dz = _axes(cfg)
    assert lib().orc_fill_ghosts(C.byref(c), _ptr(dx), _ptr(dy), _ptr(dz), _ptr(q)) == 0
    return q


def diag_f32(nx, ny, nz, order, gamma, rho, p, vel) -> tuple[float, float]:
    """Reference-form KE / entropy (float32 fields, float32 running sum)."""
    r = np.ascontiguousarray(rho, dtype=np.float32)
    pp = np.ascontiguousarray(p, dtype=np.float32)
    v = np.ascontiguousarray(vel, dtype=np.float32)
    out = np.zeros(2)
    fp = C.POINTER(C.c_float)
    lib().orc_diag_f32(nx, ny, nz, order, gamma, r.ctypes.data_as(fp), pp.ctypes.data_as(fp),
                       v.ctypes.data_as(fp), _ptr(out))
    return float(out[0]), float(out[1])
