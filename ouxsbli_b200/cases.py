"""Case definitions: default parameters and initial fields of the periodic cases.

Each case mirrors a reference case directory (``3D_solver/<CASE>`` or
``2D_solver/<CASE>``): its config.fypp macros, its mod_globals.f90 parameters
and its ``set_init``.  Initial fields are built on the host in the reference's
layout Q(nx, nv, ny[, nz]) (conservative variables, Fortran order), ghosts
filled periodically.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Callable

import numpy as np

from .grid import cyclic_axis, fill_periodic


def sutherland_mu(T: float) -> float:
    """mu0 of NSTGV/mod_globals.f90:46 (Sutherland with S = 111 K)."""
    S = 111.0
    return 1.716e-5 * (273.2 + S) / (T + S) * (T / 273.2) ** 1.5


@dataclass
class CaseDef:
    name: str
    dim: int
    config: dict            # config.fypp macros
    params: dict            # mod_globals.f90 parameters
    init: Callable          # (params, xc, yc, zc) -> Q interior-filled
    derived: Callable = None  # (params) -> params with derived quantities (V0, dt, ...)
    doc: str = ""
    grid: Callable = None     # (params) -> (x, dx, y, dy) for node-based grids; default: periodic cell centres
    bc_x: bool = False        # the case's x boundaries are non-periodic (BC_X = True)
    bc_y: bool = False        # the case's y boundaries are non-periodic (BC_Y = True)
    boundary: Callable = None  # (params, J) -> rules of the non-periodic faces (SolverConfig.boundary)
    boundary_order: str = "x_last"  # which rules the corners take last (SolverConfig.boundary_order)
    x_periodic_copy: bool = False  # BC_X = True, but set_bc copies the x ghosts periodically: periodic x
    bc_z: bool = False        # 3D: the case's z boundaries are non-periodic (BC_Z = True)
    slabs: int = 0            # COMMZ: the number of z slabs the reference's run splits the grid into


# ---------------------------------------------------------------------------
# Taylor-Green vortex, dimensional form of 3D_solver/NSTGV (mod_globals.f90:42-57,
# set.f90:16-47).  `rho_mode` = "isothermal" reproduces NSTGV (rho = p / (R T));
# "uniform" gives rho = rho0 everywhere (the ETGV-style field).
# ---------------------------------------------------------------------------
def _tgv_derived(p: dict) -> dict:
    p = dict(p)
    T0 = p["T"]
    p["mu0"] = sutherland_mu(T0)
    p["V0"] = p["M0"] * math.sqrt(p["gamma"] * p["R"] * T0)
    p["RHO0"] = p["mu0"] * p["Re"] / (p["V0"] * p["L0"])
    p["p0"] = p["RHO0"] * p["R"] * T0
    n = p["nx"]
    g = p["order"] // 2
    L = p.get("Lx", 2.0 * math.pi * p["L0"])
    p.setdefault("Lx", L)
    p.setdefault("Ly", 2.0 * math.pi * p["L0"])
    p.setdefault("Lz", 2.0 * math.pi * p["L0"])
    if p.get("dt") is None:
        if p.get("cfl_mode", "reference") == "acoustic":
            # acoustic CFL: dt = CFL * delta / (V0 + c), c = V0 / M0
            delta = p["Lx"] / (n - 2 * g)
            p["dt"] = p["CFL"] * delta / (p["V0"] + p["V0"] / p["M0"])
        else:
            # NSTGV/mod_globals.f90:53: dt = CFL * (Lx/(nx-1)) / V0
            p["dt"] = p["CFL"] * (p["Lx"] / float(n - 1)) / p["V0"]
    p["dtn"] = p["V0"] * p["dt"] / p["L0"]
    if p.get("nt") is None:
        p["nt"] = int(20.0 / (float(p["np"]) * p["dtn"]))
    return p


def _tgv_init(p: dict, x, y, z, fill: bool = True) -> np.ndarray:
    """The field on cell centres x, y, z (ghosts included).  fill=False keeps the
    analytic values in the ghost cells instead of periodic images, for a block of z
    planes cut out of a larger grid (its ghost planes then hold the neighbouring
    planes' values, as a z slab's halo does)."""
    nx, ny, nz = x.size, y.size, z.size
    g = p["order"] // 2
    L0, V0, RHO0, p0, R, T0, gam = p["L0"], p["V0"], p["RHO0"], p["p0"], p["R"], p["T"], p["gamma"]
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    pr = p0 + RHO0 * (V0 ** 2) * (np.cos(2.0 * X / L0) + np.cos(2.0 * Y / L0)) * (np.cos(2.0 * Z / L0) + 2.0) / 16.0
    if p.get("rho_mode", "isothermal") == "isothermal":
        rho = pr / (R * T0)
    else:
        rho = np.full_like(pr, RHO0)
    Q = np.zeros((nx, 5, ny, nz), order="F")
    ru = rho * V0 * np.sin(X / L0) * np.cos(Y / L0) * np.cos(Z / L0)
    rv = -rho * V0 * np.cos(X / L0) * np.sin(Y / L0) * np.cos(Z / L0)
    Q[:, 0] = rho
    Q[:, 1] = ru
    Q[:, 2] = rv
    Q[:, 3] = 0.0
    Q[:, 4] = pr / (gam - 1.0) + 0.5 * (ru ** 2 + rv ** 2) / rho
    if fill:
        fill_periodic(Q, g)
    return Q


def tgv_planes(p: dict, xc, yc, zc, k0: int, k1: int) -> np.ndarray:
    """Q of the Taylor-Green grid `p` (derived parameters, cell centres of the whole
    grid) on its z planes k0 .. k1-1 only, with analytic ghost values."""
    return _tgv_init(p, xc, yc, zc[k0:k1], fill=False)


# ---------------------------------------------------------------------------
# Inviscid Taylor-Green vortex, nondimensional: 3D_solver/ETGV (set.f90:16-45)
# ---------------------------------------------------------------------------
def _etgv_init(p: dict, x, y, z) -> np.ndarray:
    g = p["order"] // 2
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    R0, M0, gam = p["RHO0"], p["M0"], p["gamma"]
    Q = np.zeros((x.size, 5, y.size, z.size), order="F")
    ru = R0 * M0 * np.sin(X) * np.cos(Y) * np.cos(Z)
    rv = -R0 * M0 * np.cos(X) * np.sin(Y) * np.cos(Z)
    Q[:, 0] = R0
    Q[:, 1] = ru
    Q[:, 2] = rv
    Q[:, 3] = 0.0
    Q[:, 4] = (1.0 / gam + 0.0625 * R0 * (M0 ** 2) * (np.cos(2.0 * X) + np.cos(2.0 * Y)) * (np.cos(2.0 * Z) + 2.0)) / \
        (gam - 1.0) + 0.5 * (ru ** 2 + rv ** 2) / R0
    fill_periodic(Q, g)
    return Q


def _etgv_derived(p: dict) -> dict:
    p = dict(p)
    p.setdefault("Lx", 2.0 * math.pi)
    p.setdefault("Ly", 2.0 * math.pi)
    p.setdefault("Lz", 2.0 * math.pi)
    return p


# ---------------------------------------------------------------------------
# Euler vortex convection: 2D_solver/EVC (mod_globals.f90:24-46, set.f90:24-41)
# ---------------------------------------------------------------------------
def _evc_derived(p: dict) -> dict:
    p = dict(p)
    p["u0"] = p.get("u0") or p["M0"] * math.sqrt(p["gamma"] * p["R"] * p["T0"])
    p["rho0"] = p["p0"] / (p["R"] * p["T0"])
    if p.get("dt") is None:
        p["dt"] = p["CFL"] * p["Lx"] / (float(p["nx"] - 1) * p["u0"])
    if p.get("nt") is None:
        T = 2.0 * p["Lx"] / p["u0"]
        p["nt"] = int(T / (float(p["np"]) * abs(p["dt"])))
    return p


def _evc_init(p: dict, x, y, z=None) -> np.ndarray:
    nx, ny = x.size, y.size
    gam, R, T0, u0, beta, Rc, theta = p["gamma"], p["R"], p["T0"], p["u0"], p["beta"], p["Rc"], p["theta"]
    Cp = R * gam / (gam - 1.0)
    xc = x[int(nx / 2) - 1]
    yc = y[int(ny / 2) - 1]
    X, Y = np.meshgrid(x, y, indexing="ij")
    ex = np.exp(-0.5 * ((X - xc) ** 2 + (Y - yc) ** 2) / (Rc ** 2))
    T = T0 - 0.5 * (u0 * beta) ** 2 / Cp * ex ** 2
    rho = p["rho0"] * (T / T0) ** (1.0 / (gam - 1.0))
    du = -u0 * beta * (Y - yc) / Rc * ex
    dv = u0 * beta * (X - xc) / Rc * ex
    u = u0 * math.cos(theta) + du * math.cos(theta) - dv * math.sin(theta)
    v = u0 * math.sin(theta) + du * math.sin(theta) + dv * math.cos(theta)
    pr = rho * R * T
    Q = np.zeros((nx, 4, ny), order="F")
    Q[:, 0] = rho
    Q[:, 1] = rho * u
    Q[:, 2] = rho * v
    Q[:, 3] = pr / (gam - 1.0) + 0.5 * rho * (u ** 2 + v ** 2)
    return Q


# ---------------------------------------------------------------------------
# Isentropic vortex (beta form) for the batched 2D ensemble: nondimensional
# free stream (rho = 1, p = 1/gamma, c = 1), u_inf = Ma; exact solution = the
# initial field translated by u_inf * t (periodic).
# ---------------------------------------------------------------------------
def isentropic_vortex(nx: int, ny: int, order: int, L: float, beta: float, mach: float,
                      gamma: float = 1.4, R: float = 1.0, t: float = 0.0) -> np.ndarray:
    g = order // 2
    x, _ = cyclic_axis(nx, L, order)
    y, _ = cyclic_axis(ny, L, order)
    uinf, vinf = mach, 0.0
    X, Y = np.meshgrid(x, y, indexing="ij")
    x0 = 0.5 * L + uinf * t
    y0 = 0.5 * L + vinf * t
    dxr = (X - x0 + 0.5 * L) % L - 0.5 * L
    dyr = (Y - y0 + 0.5 * L) % L - 0.5 * L
    r2 = dxr ** 2 + dyr ** 2
    f = np.exp(0.5 * (1.0 - r2))
    du = -beta / (2.0 * math.pi) * dyr * f
    dv = beta / (2.0 * math.pi) * dxr * f
    Tn = 1.0 - (gamma - 1.0) * beta ** 2 / (8.0 * gamma * math.pi ** 2) * np.exp(1.0 - r2)
    rho = Tn ** (1.0 / (gamma - 1.0))
    pr = rho ** gamma / gamma
    u, v = uinf + du, vinf + dv
    Q = np.zeros((nx, 4, ny), order="F")
    Q[:, 0] = rho
    Q[:, 1] = rho * u
    Q[:, 2] = rho * v
    Q[:, 3] = pr / (gamma - 1.0) + 0.5 * rho * (u ** 2 + v ** 2)
    fill_periodic(Q, g)
    return Q


# ---------------------------------------------------------------------------
# Inviscid shock tube (Sod): 2D_solver/ST (mod_globals.f90:22-45, set.f90:9-46).
# x is non-periodic with zero-gradient boundary cells; y is periodic here (the
# reference's y-wall / symmetry rows leave the 1D flow unchanged).
# ---------------------------------------------------------------------------
def _st_derived(p: dict) -> dict:
    p = dict(p)
    p["mu0"] = p["C"] * p["T0"] ** 1.5 / (p["T0"] + p["S"])
    p["p0"] = p["rho0"] * p["R"] * p["T0"]
    p["rho1"] = 0.125 * p["rho0"]
    p["p1"] = 0.1 * p["p0"]
    p.setdefault("Lx", p["Re"] * p["mu0"] / math.sqrt(p["rho0"] * p["p0"]))
    p.setdefault("Ly", 0.1 * p["Lx"])
    c0 = math.sqrt(p["p0"] / p["rho0"])
    if p.get("dt") is None:
        p["dt"] = p["CFL"] * p["Lx"] / (float(p["nx"] - 1) * c0)
    p["endT"] = 0.2136 * p["Lx"] / c0
    if p.get("nt") is None:
        p["nt"] = int(p["endT"] / (float(p["np"]) * p["dt"]))
    return p


def _st_grid(p: dict):
    """set_grid: nodes x(1) = 0, x(i+1) = x(i) + Lx / (nx-1); same in y."""
    nx, ny = p["nx"], p["ny"]
    dx0, dy0 = p["Lx"] / (nx - 1), p["Ly"] / (ny - 1)
    x = np.zeros(nx)
    for i in range(nx - 1):
        x[i + 1] = x[i] + dx0
    y = np.zeros(ny)
    for j in range(ny - 1):
        y[j + 1] = y[j] + dy0
    return x, np.full(nx - 1, dx0), y, np.full(ny - 1, dy0)


def _st_init(p: dict, x, y, z=None) -> np.ndarray:
    """set_init: the left state in cells 1..nx/2 (1-based), the right state after."""
    nx, ny, gam = x.size, y.size, p["gamma"]
    Q = np.zeros((nx, 4, ny), order="F")
    half = nx // 2
    Q[:half, 0] = p["rho0"]
    Q[:half, 3] = p["p0"] / (gam - 1.0)
    Q[half:, 0] = p["rho1"]
    Q[half:, 3] = p["p1"] / (gam - 1.0)
    return Q


# ---------------------------------------------------------------------------
# Kelvin-Helmholtz instability: 3D_solver/KHI (mod_globals.f90, set.f90 set_init):
# a supersonic stream (T2, 3 c2) in 0.25 L <= y <= 0.75 L inside a Mach-2 stream
# (T1), equal pressure, perturbed by v = amp u1 sin(2 pi x / Lx), w = amp u1 sin(2 pi z / Lz).
# ---------------------------------------------------------------------------
def _khi_derived(p: dict) -> dict:
    p = dict(p)
    g, R = p["gamma"], p["R"]
    p["rho1"] = p["p"] / (R * p["T1"])
    p["u1"] = 2.0 * math.sqrt(g * R * p["T1"])
    p["rho2"] = p["p"] / (R * p["T2"])
    p["u2"] = 3.0 * math.sqrt(g * R * p["T2"])
    if p.get("dt") is None:
        p["dt"] = p["CFL"] * p["Lx"] / (float(p["nx"] - 1) * abs(p["u1"]))
    p.setdefault("endT", 10.0 * p["Lx"] / p["u2"])
    if p.get("nt") is None:
        p["nt"] = int(p["endT"] / (float(p["np"]) * p["dt"]))
    return p


def _khi_init(p: dict, x, y, z) -> np.ndarray:
    """set_init on the interior cells (offset g), then the periodic fill."""
    g = p["order"] // 2
    gam = p["gamma"]
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    v = p["amp"] * p["u1"] * np.sin(2.0 * math.pi * X / p["Lx"])
    w = p["amp"] * p["u1"] * np.sin(2.0 * math.pi * Z / p["Lz"])
    outer = (Y > 0.75 * p["Lx"]) | (Y < 0.25 * p["Lx"])
    rho = np.where(outer, p["rho1"], p["rho2"])
    u = np.where(outer, p["u1"], p["u2"])
    Q = np.zeros((x.size, 5, y.size, z.size), order="F")
    Q[:, 0] = rho
    Q[:, 1] = rho * u
    Q[:, 2] = rho * v
    Q[:, 3] = rho * w
    Q[:, 4] = p["p"] / (gam - 1.0) + 0.5 * rho * (u ** 2 + v ** 2 + w ** 2)
    fill_periodic(Q, g)
    return Q


# ---------------------------------------------------------------------------
# Double shear layer: 2D_solver/DSL (mod_globals.f90, set.f90 set_init): two tanh
# shear layers at y = pi/2 and 3 pi/2 on [0, 2 pi)^2 with a sinusoidal v
# perturbation; set_init writes every point, ghosts included.
# ---------------------------------------------------------------------------
def _dsl_derived(p: dict) -> dict:
    p = dict(p)
    p.setdefault("Lx", 2.0 * math.pi)
    p.setdefault("Ly", 2.0 * math.pi)
    p["d1"] = math.pi / 15.0 if p.get("d1") is None else p["d1"]
    if p.get("nt") is None:
        p["nt"] = int(p["endT"] / (float(p["np"]) * p["dt"]))
    return p


def _dsl_init(p: dict, x, y, z=None) -> np.ndarray:
    gam, rho0, u0, M0, d1, d2 = p["gamma"], p["rho0"], p["u0"], p["M0"], p["d1"], p["d2"]
    pr = rho0 * u0 ** 2 / (gam * M0 ** 2)
    X, Y = np.meshgrid(x, y, indexing="ij")
    lower = Y <= math.pi
    ru = np.where(lower, rho0 * u0 * np.tanh((Y - 0.5 * math.pi) / d1), rho0 * u0 * np.tanh((1.5 * math.pi - Y) / d1))
    rv = rho0 * u0 * d2 * np.sin(X)
    Q = np.zeros((x.size, 4, y.size), order="F")
    Q[:, 0] = rho0
    Q[:, 1] = ru
    Q[:, 2] = rv
    Q[:, 3] = pr / (gam - 1.0) + 0.5 * (ru ** 2 + rv ** 2) / rho0
    return Q


# ---------------------------------------------------------------------------
# Reflection of an oblique shock from a slip wall: 2D_solver/OS (mod_globals.f90,
# set.f90).  Supersonic inflow at x low, zero-gradient outflow at x high, a slip wall
# at y low and, at y high, the free stream up to 0.1 Lx and the state behind an
# incident shock of angle beta after it (that shock enters the domain there).
# ---------------------------------------------------------------------------
def _os_derived(p: dict) -> dict:
    """The free-stream and post-incident-shock states of mod_globals.f90 (the
    oblique-shock relations for the angle beta)."""
    p = dict(p)
    g, R, M0 = p["gamma"], p["R"], p["M0"]
    p.setdefault("Lx", 5.0 * p["blt"])
    p.setdefault("Ly", 2.0 * p["blt"])
    p["p0"] = p["p_tot"] / ((1.0 + 0.5 * (g - 1.0) * M0 ** 2) ** (g / (g - 1.0)))
    p["T0"] = p["T_tot"] / (1.0 + 0.5 * (g - 1.0) * M0 ** 2)
    p["u0"] = M0 * math.sqrt(g * R * p["T0"])
    p["rho0"] = p["p0"] / (R * p["T0"])
    beta = p["beta"]
    Ms = M0 * math.sin(beta)
    Ms2 = Ms ** 2
    p["theta"] = math.atan(2.0 * (1.0 / math.tan(beta)) * (Ms2 - 1.0) / (M0 ** 2 * (g + math.cos(2.0 * beta)) + 2.0))
    p["T2"] = p["T0"] * (1.0 + 2.0 * (g - 1.0) * (Ms2 - 1.0) * (1.0 + g * Ms2) / (Ms2 * (g + 1.0) ** 2))
    p["p2"] = p["p0"] * (1.0 + 2.0 * g * (Ms2 - 1.0) / (g + 1.0))
    p["rho2"] = p["p2"] / (R * p["T2"])
    u1 = p["u0"] * math.sin(beta)
    a1 = p["u0"] / M0
    u2 = u1 - 2.0 * a1 * (Ms - 1.0 / Ms) / (g + 1.0)
    v2 = p["u0"] * math.cos(beta)
    umag = math.sqrt(u2 ** 2 + v2 ** 2)
    p["ux"] = umag * math.cos(p["theta"])
    p["uy"] = -umag * math.sin(p["theta"])
    if p.get("nt") is None:
        p["nt"] = int(p["endT"] / (float(p["np"]) * p["dt"]))
    return p


def _os_states(p: dict) -> tuple[np.ndarray, np.ndarray]:
    """Conservative (rho, rho u, rho v, E) of the free stream and of the post-shock state."""
    og1 = 1.0 / (p["gamma"] - 1.0)
    free = np.array([p["rho0"], p["rho0"] * p["u0"], 0.0, p["p0"] * og1 + 0.5 * p["rho0"] * p["u0"] ** 2])
    r2, ux, uy = p["rho2"], p["ux"], p["uy"]
    post = np.array([r2, r2 * ux, r2 * uy, p["p2"] * og1 + 0.5 * r2 * (ux ** 2 + uy ** 2)])
    return free, post


def _os_first_post(nx: int) -> int:
    """0-based first column of the post-shock part of the top row (1-based int(0.1 nx))."""
    return int(0.1 * nx) - 1


def _os_init(p: dict, x, y, z=None) -> np.ndarray:
    """set_init: the free stream everywhere, the post-shock state on the top row from
    column int(0.1 nx) (1-based) on."""
    nx, ny = x.size, y.size
    free, post = _os_states(p)
    Q = np.zeros((nx, 4, ny), order="F")
    Q[:] = free[None, :, None]
    Q[_os_first_post(nx):, :, ny - 1] = post
    return Q


def _os_boundary(p: dict, J: np.ndarray) -> dict:
    """set_bc: inflow (fixed free stream) at x low, zero gradient at x high, a slip
    wall at y low, the fixed top row at y high (values of Q/J)."""
    nx, ny = J.shape
    free, post = _os_states(p)
    top = np.empty((4, nx))
    top[:] = free[:, None]
    top[:, _os_first_post(nx):] = post[:, None]
    top = top * (1.0 / J[0, ny - 2])
    inflow = free[:, None] * (1.0 / J[0, :])[None, :]
    return {"x_lo": ("fixed", inflow), "x_hi": "zero_gradient", "y_lo": "slip_wall", "y_hi": ("fixed", top)}


# ---------------------------------------------------------------------------
# Laminar boundary layer on a flat plate at Mach 2: 2D_solver/BL0 (mod_globals.f90,
# set.f90).  Inflow at x low, zero gradient at x high; along y low a copy of the
# neighbour ahead of the plate (the first nx/10 columns) and an adiabatic no-slip
# wall after; a characteristic far field at y high; corners take their y rule (the
# y rows are written after the x columns).
# ---------------------------------------------------------------------------
def _bl_derived(p: dict) -> dict:
    p = dict(p)
    g, R, M0 = p["gamma"], p["R"], p["M0"]
    p.setdefault("Lx", 80.0 * p["blt"])
    p.setdefault("Ly", 5.0 * p["blt"])
    f = 1.0 + 0.5 * (g - 1.0) * M0 ** 2
    p["p0"] = p["p_tot"] / f ** (g / (g - 1.0))
    p["T0"] = p["T_tot"] / f
    p["rho0"] = p["p0"] / (R * p["T0"])
    p["u0"] = M0 * math.sqrt(g * R * p["T0"])
    p["Cp"] = g * R / (g - 1.0)
    p["Taw"] = p["T0"] * (1.0 + p["rf"] * 0.5 * (g - 1.0) * M0 ** 2)
    # set_bc's inflow / far-field temperature and density (equal to T0, rho0 up to rounding)
    p["T_bc"] = p["Taw"] - p["rf"] * p["u0"] ** 2 / (2.0 * p["Cp"])
    p["rho_bc"] = p["p0"] / (R * p["T_bc"])
    p["c_bc"] = math.sqrt(g * p["p0"] / p["rho_bc"])
    if p.get("nt") is None:
        p["nt"] = int(p["endT"] / (float(p["np"]) * p["dt"]))
    return p


def _bl_grid(p: dict):
    """set_grid: uniform x nodes from 0; y nodes refined at the wall up to 3 blt
    (dy = min(1, max(0.07, j / 128)) dx), then stretched by up to 1.75 dx."""
    nx, ny, blt = p["nx"], p["ny"], p["blt"]
    dx1 = p["Lx"] / (nx - 1)
    dy1 = dx1
    x = np.zeros(nx)
    dx = np.full(nx - 1, dx1)
    for i in range(nx - 1):
        x[i + 1] = x[i] + dx[i]
    y = np.zeros(ny)
    dy = np.zeros(ny - 1)
    ny_b = 0
    for j in range(1, ny):  # Fortran j = 1 .. ny-1
        if y[j - 1] <= 3.0 * blt:
            dy[j - 1] = min(1.0, max(0.07, float(j) / 128.0)) * dy1
            ny_b = j
        else:
            dy[j - 1] = dy1 * (1.0 + 0.75 * float(j - ny_b) / float(ny - ny_b))
        y[j] = y[j - 1] + dy[j - 1]
    return x, dx, y, dy


def _bl_init(p: dict, x, y, z=None) -> np.ndarray:
    nx, ny, gam = x.size, y.size, p["gamma"]
    Q = np.zeros((nx, 4, ny), order="F")
    Q[:, 0] = p["rho0"]
    Q[:, 1] = p["rho0"] * p["u0"]
    Q[:, 3] = p["p0"] / (gam - 1.0) + 0.5 * p["rho0"] * p["u0"] ** 2
    return Q


def _bl_boundary(p: dict, J: np.ndarray) -> dict:
    nx, ny = J.shape
    gam, rho, u0 = p["gamma"], p["rho_bc"], p["u0"]
    free = np.array([rho, rho * u0, 0.0, p["p0"] / (gam - 1.0) + 0.5 * rho * u0 ** 2])
    inflow = free[:, None] * (1.0 / J[0, :])[None, :]
    return {"x_lo": ("fixed", inflow), "x_hi": "zero_gradient",
            "y_lo": ("split", nx // 10 - 1, "zero_gradient", "noslip_wall"),
            "y_hi": ("farfield", rho, u0, 0.0, p["c_bc"])}


# ---------------------------------------------------------------------------
# Boundary layer from an inflow profile: 2D_solver/BL (mod_globals.f90, set.f90).  The
# flat-plate grid and Mach-2 constants of BL0 with blt = 1 mm, Lx = 20 blt and a 4th-order
# viscous stencil on the 2nd-order grid.  set_init reads the profile file (`inflow`;
# the reference reads ./Qin.dat): nyi rows of 5 float64 values (y, rho, u, v, p), the
# rows one after another; it interpolates them linearly onto the grid's y nodes (held
# at the end rows outside the profile's range), takes one pressure, the mean of the
# interpolated p over the first nyi grid rows, and fills every column with the
# result.  set_bc: the inflow column keeps its initial values, zero gradient at x high
# and at y high (Neumann), an adiabatic no-slip wall along all of y low; corners take
# their y rule.
# ---------------------------------------------------------------------------
def read_inflow_profile(path) -> np.ndarray:
    """The (nyi, 5) rows (y, rho, u, v, p) of a BL inflow profile file (little-endian
    float64, written row after row as the reference's Qi(5, nyi) lies in memory)."""
    a = np.fromfile(path, dtype="<f8")
    if a.size == 0 or a.size % 5:
        raise ValueError(f"{path}: an inflow profile holds rows of 5 float64 values, found {a.size} values")
    return a.reshape(-1, 5)


def interpolate_inflow(y: np.ndarray, prof: np.ndarray) -> np.ndarray:
    """interpolate_Q (2D_solver/BL/set.f90:39-63): (ny, 4) rho, u, v, p at the nodes y."""
    out = np.empty((y.size, 4))
    nyi = prof.shape[0]
    for j, yj in enumerate(y):
        if yj <= prof[0, 0]:
            out[j] = prof[0, 1:]
        elif yj >= prof[nyi - 1, 0]:
            out[j] = prof[nyi - 1, 1:]
        else:
            for i in range(nyi - 1):
                y1, y2 = prof[i, 0], prof[i + 1, 0]
                if y1 <= yj <= y2:
                    alpha = (yj - y1) / (y2 - y1)
                    out[j] = (1.0 - alpha) * prof[i, 1:] + alpha * prof[i + 1, 1:]
                    break
    return out


def _blq_derived(p: dict) -> dict:
    p = dict(p)
    if p.get("Lx") is None:
        p["Lx"] = 20.0 * p["blt"]
    return _bl_derived(p)


def _blq_init(p: dict, x, y, z=None) -> np.ndarray:
    """set_init (2D_solver/BL/set.f90:66-101); keeps the inflow column for the boundary."""
    prof = read_inflow_profile(p["inflow"])
    nyi = prof.shape[0]
    if nyi > y.size:
        raise ValueError(f"the inflow profile has {nyi} rows, more than the grid's {y.size} y nodes "
                         "(set_init averages p over the first nyi grid rows)")
    qp = interpolate_inflow(y, prof)
    ptbl = 0.0
    for j in range(nyi):  # the reference's sequential sum
        ptbl = ptbl + qp[j, 3]
    ptbl = ptbl / float(nyi)
    og1 = 1.0 / (p["gamma"] - 1.0)
    rho, u, v = qp[:, 0], qp[:, 1], qp[:, 2]
    Q = np.zeros((x.size, 4, y.size), order="F")
    Q[:, 0] = rho
    Q[:, 1] = rho * u
    Q[:, 2] = rho * v
    Q[:, 3] = ptbl * og1 + 0.5 * rho * (u * u + v * v)
    p["inflow_q"] = Q[0].copy()  # (4, ny): what set_bc leaves in the inflow column
    return Q


def _blq_boundary(p: dict, J: np.ndarray) -> dict:
    inflow = p["inflow_q"] * (1.0 / J[0, :])[None, :]
    return {"x_lo": ("fixed", inflow), "x_hi": "zero_gradient", "y_lo": "noslip_wall", "y_hi": "zero_gradient"}


# ---------------------------------------------------------------------------
# Temporally developing boundary layer on a wall: 2D_solver/SBLI (mod_globals.f90,
# set.f90, src/set_init_common.f90 set_init_tbl, src/set_compressible_bl.f90).  Its
# set_bc copies the x ghosts periodically (the x flux kernels are the boundary
# versions, which only change faces of ghost cells), a no-slip wall at y low and the
# free stream at y high.  The initial field is a compressible laminar layer of 99 %
# thickness blt.
# ---------------------------------------------------------------------------
def _sbli_derived(p: dict) -> dict:
    p = dict(p)
    p.setdefault("Lx", 100.0 * p["blt"])
    p.setdefault("Ly", 5.0 * p["blt"])
    p = _bl_derived(p)
    return p


def _sbli_grid(p: dict):
    """set_grid: the flat-plate grid, x shifted by -70 blt."""
    x, dx, y, dy = _bl_grid(p)
    return x - 70.0 * p["blt"], dx, y, dy


def _sbli_init(p: dict, x, y, z=None) -> np.ndarray:
    """set_init_tbl: the profile in every column, then the wall row of the no-slip rule."""
    from .blasius import compressible_profile
    gam, R = p["gamma"], p["R"]
    og1 = 1.0 / (gam - 1.0)
    mu0 = sutherland_mu(p["T0"])
    rho, u, v, T = compressible_profile(y, p["blt"], p["u0"], p["T0"], p["p0"], R, p["Cp"], p["rf"], p["Taw"], mu0)
    Q = np.zeros((x.size, 4, y.size), order="F")
    q1 = p["p0"] / (R * T)
    Q[:, 0] = q1
    Q[:, 1] = q1 * u
    Q[:, 2] = q1 * v
    Q[:, 3] = p["p0"] * og1 + 0.5 * (Q[:, 1] ** 2 + Q[:, 2] ** 2) / Q[:, 0]
    Q[:, 0, 0] = Q[:, 0, 1]
    Q[:, 1, 0] = 0.0
    Q[:, 2, 0] = 0.0
    p_wall = (gam - 1.0) * (Q[1, 3, 1] - 0.5 * (Q[1, 1, 1] ** 2 + Q[1, 2, 1] ** 2) / Q[1, 0, 1])
    Q[:, 3, 0] = p_wall * og1
    g = p["order"] // 2  # the x ghosts are periodic images (set_bc's x copies)
    N = x.size - 2 * g
    for i in list(range(g)) + list(range(x.size - g, x.size)):
        Q[i] = Q[g + (i - g) % N]
    return Q


def _sbli_boundary(p: dict, J: np.ndarray) -> dict:
    nx, ny = J.shape
    gam, rho, u0 = p["gamma"], p["rho_bc"], p["u0"]
    top = np.empty((4, nx))
    top[0] = rho
    top[1] = rho * u0
    top[2] = 0.0
    top[3] = p["p0"] * (1.0 / (gam - 1.0)) + 0.5 * rho * u0 ** 2
    top = top * (1.0 / J[:, ny - 1])[None, :]
    return {"y_lo": "noslip_wall", "y_hi": ("fixed", top)}


# ---------------------------------------------------------------------------
# Shock tube along z over two z slabs (COMMZ): 3D_solver/STZ (mod_globals.f90,
# set.f90).  Order-2 SLAU, slip walls in x and y (the mirrored ghost cells of its
# set_bc), zero gradient at the two z ends of the grid; the lower slab starts in the
# left state, the upper one in the right state.  `nz` is a slab's plane count (its
# interior + one ghost plane each end), as in the reference, whose four MPI ranks
# hold two z slabs.
# ---------------------------------------------------------------------------
def _stz_derived(p: dict) -> dict:
    p = dict(p)
    p["nz_grid"] = p["slabs"] * (p["nz"] - 2) + 2  # planes of the whole grid
    if p.get("dt") is None:
        p["dt"] = p["CFL"] * p["Lz"] / (float(p["nz"] - 1) * math.sqrt(p["p_L"] / p["rho_L"]))
    if p.get("nt") is None:
        p["nt"] = int(p["endT"] / (float(p["np"]) * p["dt"]))
    return p


def _stz_grid(p: dict):
    """set_grid: uniform cell centres, one ghost a side; z over all slabs."""
    def axis(n, L):
        d = L / (n - 2)
        return d * (np.arange(n) - 0.5), np.full(n - 1, d)  # first interior centre at d / 2
    nint = p["nz"] - 2
    x, dx = axis(p["nx"], p["Lx"])
    y, dy = axis(p["ny"], p["Ly"])
    z, dz = axis(p["slabs"] * nint + 2, p["Lz"])
    return x, dx, y, dy, z, dz


def _stz_init(p: dict, x, y, z) -> np.ndarray:
    """set_init: the left state in the first slab's planes (ghost included), the right
    state in the second's."""
    gam = p["gamma"]
    nx, ny, nz = x.size, y.size, z.size
    Q = np.zeros((nx, 5, ny, nz), order="F")
    left = np.arange(nz) < p["nz"] - 1
    Q[:, 0] = np.where(left, p["rho_L"], p["rho_R"])[None, None, :]
    Q[:, 4] = np.where(left, p["p_L"], p["p_R"])[None, None, :] / (gam - 1.0)
    return Q


def _stz_boundary(p: dict, J) -> dict:
    return {"x_lo": "slip_wall", "x_hi": "slip_wall", "y_lo": "slip_wall", "y_hi": "slip_wall",
            "z_lo": "zero_gradient", "z_hi": "zero_gradient"}


CASES: dict[str, CaseDef] = {
    "NSTGV": CaseDef(
        "NSTGV", 3,
        dict(VISC="NS", SCHEME="SLAU", ORDER=6, TVD="hybrid", SLAU_VARIANT="HRSLAU2", RK=3,
             BC_X=False, BC_Y=False, BC_Z=False, RESCALE=False, COMMZ=False, RESTART=False),
        dict(nx=513, ny=513, nz=513, L0=1.524e-3, Re=1600.0, M0=1.25, T=530.0 * 5.0 / 9.0,
             gamma=1.4, Pr=0.71, Prt=0.9, R=287.03, CFL=0.03, np=100, threshold=0.4, dt=None, nt=None,
             rho_mode="isothermal", cfl_mode="reference"),
        _tgv_init, _tgv_derived,
        "Viscous Taylor-Green vortex (3D_solver/NSTGV)"),
    "ETGV": CaseDef(
        "ETGV", 3,
        dict(VISC="Euler", SCHEME="KEEP", ORDER=6, TVD="hybrid", SLAU_VARIANT="HRSLAU2", RK=4,
             BC_X=False, BC_Y=False, BC_Z=False, RESCALE=False, COMMZ=False, RESTART=False),
        dict(nx=66, ny=66, nz=66, nt=200, np=100, dt=0.01, gamma=1.4, Pr=0.71, Prt=0.9, R=287.03,
             M0=0.4, RHO0=1.0, threshold=0.4),
        _etgv_init, _etgv_derived,
        "Inviscid Taylor-Green vortex (3D_solver/ETGV)"),
    "STZ": CaseDef(
        "STZ", 3,
        dict(VISC="Euler", SCHEME="SLAU", ORDER=2, TVD="tvd", SLAU_VARIANT="SLAU", RK=3,
             BC_X=False, BC_Y=False, BC_Z=True, RESCALE=False, COMMZ=True, RESTART=False),
        dict(nx=6, ny=6, nz=513, slabs=2, Lx=0.1, Ly=0.1, Lz=1.0, gamma=1.4, Pr=0.71, Prt=0.9, R=287.03,
             rho_L=1.0, p_L=1.0, rho_R=0.125, p_R=0.1, CFL=0.01, endT=0.1, np=50, dt=None, nt=None,
             threshold=0.4),
        _stz_init, _stz_derived,
        "Shock tube along z over two z slabs (3D_solver/STZ)",
        grid=_stz_grid, bc_x=True, bc_y=True, boundary=_stz_boundary, bc_z=True, slabs=2),
    "EVC": CaseDef(
        "EVC", 2,
        dict(VISC="Euler", SCHEME="KEEP", ORDER=6, TVD="none", SLAU_VARIANT="HRSLAU2", RK=4,
             BC_X=False, BC_Y=False, RESCALE=False, COMMZ=False, RESTART=False),
        dict(nx=258, ny=258, Lx=0.1, Ly=0.1, gamma=1.4, Pr=0.71, Prt=0.9, R=287.15, M0=0.05,
             beta=1.0 / 50.0, theta=0.0, Rc=0.005, p0=1.0e5, T0=300.0, u0=None, CFL=0.03, np=1,
             dt=None, nt=None, threshold=0.4),
        _evc_init, _evc_derived,
        "Euler vortex convection (2D_solver/EVC)"),
    "ST": CaseDef(
        "ST", 2,
        dict(VISC="NS", SCHEME="KEEP", ORDER=6, TVD="none", SLAU_VARIANT="HRSLAU2", RK=3,
             BC_X=True, BC_Y=False, RESCALE=False, COMMZ=False, RESTART=False),
        dict(nx=4097, ny=257, gamma=1.4, Pr=0.71, Prt=0.9, R=287.03, T0=300.0, C=1.461e-6, S=110.3,
             Re=25000.0, rho0=1.293, CFL=0.1, np=100, dt=None, nt=None, threshold=0.4),
        _st_init, _st_derived,
        "Inviscid shock tube, Sod problem (2D_solver/ST)",
        grid=_st_grid, bc_x=True),
    "KHI": CaseDef(
        "KHI", 3,
        dict(VISC="Euler", SCHEME="KEEP", ORDER=6, TVD="none", SLAU_VARIANT="HRSLAU2", RK=3,
             BC_X=False, BC_Y=False, BC_Z=False, RESCALE=False, COMMZ=False, RESTART=False),
        dict(nx=130, ny=130, nz=130, Lx=5.0e-3, Ly=5.0e-3, Lz=5.0e-3, gamma=1.4, Pr=0.71, Prt=0.9, R=287.15,
             p=2.72e3, T1=162.7908, T2=104.6303, amp=0.05, CFL=0.05, np=100, dt=None, nt=None,
             threshold=0.9),
        _khi_init, _khi_derived,
        "Kelvin-Helmholtz instability of a supersonic shear layer (3D_solver/KHI)"),
    "DSL": CaseDef(
        "DSL", 2,
        dict(VISC="Euler", SCHEME="KEEP", ORDER=6, TVD="none", SLAU_VARIANT="HRSLAU2", RK=4,
             BC_X=False, BC_Y=False, RESCALE=False, COMMZ=False, RESTART=False),
        dict(nx=513, ny=513, gamma=1.4, Pr=0.71, Prt=0.9, R=287.03, M0=0.1, rho0=1.0, u0=1.0, d1=None,
             d2=0.05, dt=0.25 * 0.25e-3, endT=8.0, np=10, nt=None, threshold=0.4),
        _dsl_init, _dsl_derived,
        "Double shear layer (2D_solver/DSL)"),
    "BL0": CaseDef(
        "BL0", 2,
        dict(VISC="NS", SCHEME="SLAU", ORDER=2, VISC_ORDER=2, TVD="none", SLAU_VARIANT="HRSLAU2", RK=3,
             BC_X=True, BC_Y=True, RESCALE=False, COMMZ=False, RESTART=False),
        dict(nx=1025, ny=129, blt=0.5e-3, endT=0.4e-3, np=40, dt=3.0e-9, nt=None, R=287.03, gamma=1.4, Pr=0.72,
             Prt=0.9, M0=2.0, p_tot=100.0e3, T_tot=295.0, rf=0.89, threshold=0.4),
        _bl_init, _bl_derived,
        "Laminar boundary layer on a flat plate at Mach 2 (2D_solver/BL0)",
        grid=_bl_grid, bc_x=True, bc_y=True, boundary=_bl_boundary, boundary_order="y_last"),
    "BL": CaseDef(
        "BL", 2,
        dict(VISC="NS", SCHEME="SLAU", ORDER=2, VISC_ORDER=4, TVD="none", SLAU_VARIANT="HRSLAU2", RK=3,
             BC_X=True, BC_Y=True, RESCALE=False, COMMZ=False, RESTART=False),
        dict(nx=257, ny=129, blt=1.0e-3, Lx=None, endT=0.3e-3, np=30, dt=3.0e-9, nt=None, R=287.03, gamma=1.4,
             Pr=0.72, Prt=0.9, M0=2.0, p_tot=100.0e3, T_tot=295.0, rf=0.89, threshold=0.4, inflow="Qin.dat"),
        _blq_init, _blq_derived,
        "Boundary layer from an inflow profile file at Mach 2 (2D_solver/BL)",
        grid=_bl_grid, bc_x=True, bc_y=True, boundary=_blq_boundary, boundary_order="y_last"),
    "SBLI": CaseDef(
        "SBLI", 2,
        dict(VISC="NS", SCHEME="SLAU", ORDER=6, TVD="hybrid", SLAU_VARIANT="HRSLAU2", RK=3,
             BC_X=True, BC_Y=True, RESCALE=False, COMMZ=False, RESTART=False),
        dict(nx=1025, ny=257, blt=0.8e-3, endT=0.1e-3, np=10, dt=3.0e-9, nt=None, R=287.03, gamma=1.4, Pr=0.72,
             Prt=0.9, M0=2.0, p_tot=100.0e3, T_tot=295.0, rf=0.89, threshold=0.4),
        _sbli_init, _sbli_derived,
        "Temporally developing laminar boundary layer on a wall (2D_solver/SBLI)",
        grid=_sbli_grid, bc_x=False, bc_y=True, boundary=_sbli_boundary, boundary_order="y_last",
        x_periodic_copy=True),
    "OS": CaseDef(
        "OS", 2,
        dict(VISC="Euler", SCHEME="SLAU", ORDER=6, TVD="hybrid", SLAU_VARIANT="HRSLAU2", RK=3,
             BC_X=True, BC_Y=True, RESCALE=False, COMMZ=False, RESTART=False),
        dict(nx=257, ny=129, blt=1.0e-3, endT=0.1e-3, np=10, dt=3.0e-9, nt=None, R=287.03, gamma=1.4,
             Pr=0.72, Prt=0.9, M0=2.0, p_tot=100.0e3, T_tot=295.0, beta=math.pi * 37.2 / 180.0,
             threshold=0.4),
        _os_init, _os_derived,
        "Reflection of an oblique shock from a slip wall (2D_solver/OS)",
        grid=_st_grid, bc_x=True, bc_y=True, boundary=_os_boundary),
}


def build_initial(case: CaseDef, params: dict):
    """Return (derived params, xc, yc, zc, dx, dy, dz, Q) for a case."""
    p = dict(params)
    order = p["order"]
    if case.derived:
        p = case.derived(p)
    if case.dim == 3:
        if case.grid is not None:
            xc, dx, yc, dy, zc, dz = case.grid(p)
        else:
            xc, dx = cyclic_axis(p["nx"], p["Lx"], order)
            yc, dy = cyclic_axis(p["ny"], p["Ly"], order)
            zc, dz = cyclic_axis(p["nz"], p["Lz"], order)
        Q = case.init(p, xc, yc, zc)
    else:
        if case.grid is not None:
            xc, dx, yc, dy = case.grid(p)
        else:
            xc, dx = cyclic_axis(p["nx"], p["Lx"], order)
            yc, dy = cyclic_axis(p["ny"], p["Ly"], order)
        zc, dz = np.zeros(1), None
        Q = case.init(p, xc, yc, None)
        if case.bc_x and not case.bc_y:
            from .grid import fill_periodic
            g = order // 2
            # boundary cells copy their neighbour; y ghost rows take the periodic images
            Q[0], Q[-1] = Q[1], Q[-2]
            ny = Q.shape[2]
            N = ny - 2 * g
            for j in list(range(g)) + list(range(ny - g, ny)):
                Q[:, :, j] = Q[:, :, g + (j - g) % N]
    return p, xc, yc, zc, dx, dy, dz, Q


# ---- batched 2D ensemble: independent isentropic-vortex convection solves -------
VORTEX_SIZES = (64, 96, 128, 192, 256, 384, 512)


@dataclass
class VortexMember:
    n: int          # interior cells per side
    beta: float     # vortex strength
    mach: float     # free-stream Mach number (= u_inf; c_inf = 1)
    L: float        # periodic box side
    dt: float


def vortex_member(m: VortexMember, order: int = 4, **cfg_kw):
    """SolverConfig and initial QJ of one 2D vortex (gamma 1.4, R 1, c_inf = 1)."""
    from .grid import jacobian, to_qj
    from .config import SolverConfig
    nx = m.n + order
    Q = isentropic_vortex(nx, nx, order, m.L, m.beta, m.mach)
    _, dx = cyclic_axis(nx, m.L, order)
    cfg = SolverConfig(dim=2, nx=nx, ny=nx, nz=1, order=order, dt=m.dt, gamma=1.4, R=1.0, Pr=0.71,
                       dx=dx, dy=dx.copy(), dz=None, **cfg_kw)
    return cfg, to_qj(Q, jacobian(dx, dx.copy(), None))


def vortex_exact(m: VortexMember, order: int, t: float) -> np.ndarray:
    """The exact solution at time t: the initial vortex translated by u_inf t (periodic)."""
    nx = m.n + order
    return isentropic_vortex(nx, nx, order, m.L, m.beta, m.mach, t=t)


def vortex_ensemble(count: int = 64, seed: int = 0, sizes=VORTEX_SIZES, L: float = 10.0, cfl: float = 0.4):
    """Seeded ensemble: side lengths uniform over `sizes`, beta ~ U[1, 5], Mach ~ U[0.1, 0.8];
    dt = cfl * h / (u_inf + 1) per member."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(rng.choice(sizes))
        beta = float(rng.uniform(1.0, 5.0))
        mach = float(rng.uniform(0.1, 0.8))
        out.append(VortexMember(n, beta, mach, L, cfl * (L / n) / (mach + 1.0)))
    return out
