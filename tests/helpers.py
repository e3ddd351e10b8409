"""Workload builders shared by the tests (initial fields, configurations)."""
from __future__ import annotations

import math

import numpy as np

from ouxsbli_b200.cases import CASES, build_initial, isentropic_vortex
from ouxsbli_b200.grid import cyclic_axis, jacobian, to_qj
from ouxsbli_b200.solver import SolverConfig


def tgv(n: int, order: int = 6, mach: float = 0.1, **kw):
    """Viscous TGV of the plain-method config: uniform rho, acoustic CFL 0.5."""
    case = CASES["NSTGV"]
    p = dict(case.params)
    p.update(nx=n + order, ny=n + order, nz=n + order, order=order, rho_mode="uniform",
             cfl_mode="acoustic", CFL=0.5, M0=mach, dt=None)
    p, xc, yc, zc, dx, dy, dz, Q = build_initial(case, p)
    cfg = SolverConfig(dim=3, nx=p["nx"], ny=p["ny"], nz=p["nz"], order=order, dt=p["dt"], gamma=p["gamma"],
                       R=p["R"], Pr=p["Pr"], Prt=p["Prt"], dx=dx, dy=dy, dz=dz, **kw)
    return cfg, to_qj(Q, jacobian(dx, dy, dz))


def random_turbulence(n: int, order: int = 6, seed: int = 0, mt: float = 0.3, **kw):
    """Seeded solenoidal random-phase velocity (E(k) ~ k^4 exp(-2 (k/k0)^2), k0 = 4) at uniform rho, p."""
    from ouxsbli_b200.turbulence import decaying_turbulence
    return decaying_turbulence(n, order=order, seed=seed, mt=mt, **kw)


def vortex2d(n: int, order: int = 4, beta: float = 5.0, mach: float = 0.5, L: float = 10.0, cfl: float = 0.4, **kw):
    Q = isentropic_vortex(n + order, n + order, order, L, beta, mach)
    _, dx = cyclic_axis(n + order, L, order)
    dy = dx.copy()
    dt = cfl * (L / n) / (mach + 1.0)
    cfg = SolverConfig(dim=2, nx=n + order, ny=n + order, nz=1, order=order, dt=dt, gamma=1.4, R=1.0,
                       Pr=0.71, dx=dx, dy=dy, dz=None, **kw)
    return cfg, to_qj(Q, jacobian(dx, dy, None))


def interior(a: np.ndarray, g: int, dim: int) -> np.ndarray:
    """Interior cells of a padded reference-layout array (nx, nv, ny[, nz])."""
    if dim == 3:
        return a[g:-g, :, g:-g, g:-g]
    return a[g:-g, :, g:-g]


def rhs_interior(r: np.ndarray, g: int, dim: int) -> np.ndarray:
    """Interior cells of an Rs(nx-2, nv, ny-2[, nz-2]) array."""
    s = slice(g - 1, -(g - 1) if g > 1 else None)
    if dim == 3:
        return r[s, :, s, s]
    return r[s, :, s]


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def diagnostics_numpy(cfg, qj):
    """FP64 KE, entropy and enstrophy means of a 3D state from the oracle's
    primitive fields (the definitions liboux's diagnostics use: vorticity by the
    6th-order central difference)."""
    from oracle import oracle
    f = oracle.fields(cfg, qj)
    g = cfg.g
    sl = (slice(g, -g),) * 3
    rho, u, v, w, p = (f[k][sl] for k in ("rho", "u", "v", "w", "p"))
    ke = np.mean(0.5 * rho * (u * u + v * v + w * w))
    ent = np.mean(rho * np.log(p * rho ** (-cfg.gamma)))
    inv = 1.0 / cfg.dx[0]

    def d6(a, axis):
        r = lambda m: np.roll(a, -m, axis=axis)
        return ((1.0 / 60.0) * (-r(-3) + r(3)) + 0.15 * (r(-2) - r(2)) + 0.75 * (-r(-1) + r(1))) * inv

    U, V, W = (f[k] for k in ("u", "v", "w"))
    om = [d6(W, 1) - d6(V, 2), d6(U, 2) - d6(W, 0), d6(V, 0) - d6(U, 1)]
    ens = np.mean(0.5 * f["rho"][sl] * sum(o[sl] ** 2 for o in om))
    return float(ke), float(ent), float(ens)


# ---- 3D viscous boxes with walls ----------------------------------------------------
H, R, GAMMA, T0, RHO0 = 1.0e-3, 287.03, 1.4, 300.0, 1.2


def _axis(n_int, L, order, nonper):
    """(n, coordinates, spacings) of an axis: one boundary cell a side or g ghost cells."""
    if nonper:
        n = n_int + 2
        d = np.full(n - 1, L / (n - 1))
        return n, np.concatenate([[0.0], np.cumsum(d)]), d
    n = n_int + 2 * (order // 2)
    x, d = cyclic_axis(n, L, order)
    return n, x, d


def wall_box(nx_int, ny, nz_int, order, rules, bc_x=0, bc_z=0, U=5.0, perturb=True, plate=False, visc="NS", **kw):
    """A 3D viscous (Sutherland, air) shear flow over a y range of 1 mm with walls at
    y = 0 (and y = H), periodic or non-periodic in x and z: u = U sin(pi y / H)
    (channel) or U sin(pi y / 2H) (plate: u = U at the top), plus a 3D perturbation."""
    g = order // 2
    Lx, Lz = 0.5e-3, 0.4e-3
    nx, x, dx = _axis(nx_int, Lx, order, bc_x)
    nz, z, dz = _axis(nz_int, Lz, order, bc_z)
    dy = np.full(ny - 1, H / (ny - 1))
    y = np.concatenate([[0.0], np.cumsum(dy)])
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    sy = np.sin(math.pi * Y / H)
    rho = np.full_like(X, RHO0)
    u = U * (np.sin(0.5 * math.pi * Y / H) if plate else sy)
    v = np.zeros_like(X)
    w = np.zeros_like(X)
    if perturb:
        rho = rho * (1.0 + 0.02 * np.sin(2 * math.pi * X / Lx) * np.cos(2 * math.pi * Z / Lz) * sy)
        v = 0.3 * U * np.sin(2 * math.pi * X / Lx) * sy ** 2
        w = 0.2 * U * np.sin(2 * math.pi * Z / Lz) * np.cos(2 * math.pi * X / Lx) * sy
    p = np.full_like(X, RHO0 * R * T0) * (1.0 + (0.01 * np.cos(2 * math.pi * Z / Lz) if perturb else 0.0))
    Q = np.zeros((nx, 5, ny, nz), order="F")
    Q[:, 0], Q[:, 1], Q[:, 2], Q[:, 3] = rho, rho * u, rho * v, rho * w
    Q[:, 4] = p / (GAMMA - 1.0) + 0.5 * rho * (u * u + v * v + w * w)
    # periodic directions: ghost cells are exact images of the interior
    if not bc_x:
        N = nx - 2 * g
        for i in list(range(g)) + list(range(nx - g, nx)):
            Q[i] = Q[g + (i - g) % N]
    if not bc_z:
        N = nz - 2 * g
        for k in list(range(g)) + list(range(nz - g, nz)):
            Q[:, :, :, k] = Q[:, :, :, g + (k - g) % N]
    qj = to_qj(Q, jacobian(dx, dy, dz))
    dt = 0.4 * min(dx.min(), dy.min(), dz.min()) / (U + math.sqrt(GAMMA * R * T0))
    cfg = SolverConfig(dim=3, nx=nx, ny=ny, nz=nz, order=order, visc=visc, bc_x=bc_x, bc_y=1, bc_z=bc_z, dt=dt,
                       gamma=GAMMA, R=R, Pr=0.72, dx=dx, dy=dy, dz=dz, boundary=rules, **kw)
    return cfg, qj, y
