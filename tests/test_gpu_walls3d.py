"""3D Navier-Stokes with non-periodic directions: the walled sweep variants (convective
order fallback next to a boundary, the 2nd-order viscous fallback of
3D_solver/src/calc_visc_high.f90.fypp outside its high-order guard) against the
oracle, the mixed form against FP64, and a shear-decay known answer."""
import math

import numpy as np
import pytest

from oracle import oracle
from ouxsbli_b200.grid import cyclic_axis, jacobian, to_qj
from ouxsbli_b200.solver import Solver, SolverConfig

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


def wall_box(nx_int, ny, nz_int, order, rules, bc_x=0, bc_z=0, U=5.0, perturb=True, **kw):
    """A viscous (Sutherland, air) shear flow between y walls 1 mm apart, periodic or
    non-periodic in x and z: u = U sin(pi y / H) plus a 3D perturbation."""
    g = order // 2
    Lx, Lz = 0.5e-3, 0.4e-3
    nx, x, dx = _axis(nx_int, Lx, order, bc_x)
    nz, z, dz = _axis(nz_int, Lz, order, bc_z)
    dy = np.full(ny - 1, H / (ny - 1))
    y = np.concatenate([[0.0], np.cumsum(dy)])
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    sy = np.sin(math.pi * Y / H)
    rho = np.full_like(X, RHO0)
    u = U * sy
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
    cfg = SolverConfig(dim=3, nx=nx, ny=ny, nz=nz, order=order, visc="NS", bc_x=bc_x, bc_y=1, bc_z=bc_z, dt=dt,
                       gamma=GAMMA, R=R, Pr=0.72, dx=dx, dy=dy, dz=dz, boundary=rules, **kw)
    return cfg, qj, y


CHANNEL = {"y_lo": "noslip_wall", "y_hi": "noslip_wall"}
# a flat-plate-like box: zero-gradient in / outflow, no-slip floor, zero-gradient top
PLATE = {"x_lo": "zero_gradient", "x_hi": "zero_gradient", "y_lo": "noslip_wall", "y_hi": "zero_gradient"}
# walls on every side
CLOSED = {"x_lo": "slip_wall", "x_hi": "slip_wall", "y_lo": "noslip_wall", "y_hi": "noslip_wall",
          "z_lo": "slip_wall", "z_hi": "noslip_wall"}
# periodic x, walls in y and z
DUCT = {f: r for f, r in CLOSED.items() if not f.startswith("x")}

CASES = [
    # (order, visc_order, stencil, scheme, rk, bc_x, bc_z, rules)
    (6, 6, "Central", "SLAU", 3, 1, 0, PLATE),      # the SBLI configuration (NS, SLAU-6, x / y walls)
    (6, 6, "ME4Base", "Hybrid", 3, 0, 0, CHANNEL),  # TBL-like: periodic x and z, y walls
    (6, 6, "Central", "KEEP", 4, 1, 1, CLOSED),
    (6, 4, "Central", "Hybrid", 3, 1, 0, PLATE),    # 4th-order viscous stencil at order 6
    (4, 4, "Central", "KEEP", 4, 1, 1, CLOSED),
    (4, 2, "Central", "SLAU", 3, 0, 1, DUCT),       # Gaitonde-Visbal viscous, order-4 convective
    (2, 2, "Central", "KEEP", 3, 1, 1, CLOSED),
]


@pytest.mark.gpu
@pytest.mark.parametrize("order,vo,stencil,scheme,rk,bc_x,bc_z,rules", CASES)
def test_3d_viscous_walls_bitexact_vs_oracle(order, vo, stencil, scheme, rk, bc_x, bc_z, rules, cuda_device):
    """3D Navier-Stokes with non-periodic x / y / z: the residual and the state after 4
    steps bit-identical to the oracle (the boundary faces' convective order fallback,
    the viscous faces' 2nd-order fallback next to every boundary, the boundary-cell
    rules)."""
    cfg, qj, _ = wall_box(14, 16, 10, order, rules, bc_x=bc_x, bc_z=bc_z, visc_order=vo, visc_stencil=stencil,
                          scheme=scheme, rk=rk, tvd="hybrid")
    s = Solver(cfg, cuda_device)
    s.set_state(qj)
    r = s.rhs()
    s.step(4)
    q = s.get_state()
    s.close()
    # residual of the updated cells: a periodic direction's ghost cells are refilled
    # from their images after each stage (the oracle, like the reference, updates them
    # first)
    per = lambda nonper: slice(cfg.g - 1, -(cfg.g - 1)) if not nonper and cfg.g > 1 else slice(None)
    upd = (per(bc_x), slice(None), slice(None), per(bc_z))
    np.testing.assert_array_equal(r[upd], oracle.rhs(cfg, qj)[upd])
    np.testing.assert_array_equal(q, oracle.step(cfg, qj, 4))


@pytest.mark.gpu
def test_3d_viscous_walls_mixed_close_to_fp64(cuda_device):
    """The mixed form on a walled 3D Navier-Stokes box (KEEP-6, Central-6, RK4): relative
    L2 against FP64 within the mixed form's bound for switch-free schemes (1e-5)."""
    out = {}
    for prec in ("fp64", "mixed"):
        cfg, qj, _ = wall_box(14, 16, 10, 6, CLOSED, bc_x=1, bc_z=1, scheme="KEEP", rk=4, precision=prec)
        s = Solver(cfg, cuda_device)
        s.set_state(qj)
        s.step(10)
        out[prec] = s.get_state()
        s.close()
    for l in range(5):
        a, b = out["mixed"][:, l], out["fp64"][:, l]
        assert np.linalg.norm(a - b) / np.linalg.norm(b) <= 1e-5, l


@pytest.mark.gpu
@pytest.mark.parametrize("order,vo,stencil", [(6, 6, "Central"), (6, 6, "ME4Base"), (4, 4, "Central")])
def test_3d_shear_decay_between_noslip_walls(order, vo, stencil, cuda_device):
    """u = U sin(pi y / H) between no-slip walls, uniform in x (non-periodic) and z
    (periodic), Mach 0.015: the mode decays as exp(-nu pi^2 t / H^2), nu = mu(T) / rho
    (Sutherland, 300 K, rho 1.2).  After 2 ms (amplitude ratio 0.74) the measured ratio
    is within 0.2 %."""
    cfg, qj, y = wall_box(6, 41, 4, order, {**CHANNEL, "x_lo": "zero_gradient", "x_hi": "zero_gradient"},
                          bc_x=1, bc_z=0, perturb=False, visc_order=vo, visc_stencil=stencil, scheme="KEEP", rk=3)
    mu = 1.716e-5 * 384.2 * 273.2 ** -1.5 / (T0 + 111.0) * T0 ** 1.5
    nu = mu / RHO0
    nsteps = int(round(2.0e-3 / cfg.dt))
    s = Solver(cfg, cuda_device)
    s.set_state(qj)
    s.step(nsteps)
    q = s.get_state()
    s.close()
    sin = np.sin(math.pi * y / H)
    g = cfg.g

    def amplitude(qq):
        u = (qq[:, 1] / qq[:, 0])[1:-1, :, g:-g].mean(axis=(0, 2))  # the flow is uniform in x and z
        return float(np.sum(u * sin) / np.sum(sin * sin))

    ratio = amplitude(q) / amplitude(qj)
    expect = math.exp(-nu * math.pi ** 2 * nsteps * cfg.dt / H ** 2)
    assert abs(ratio / expect - 1.0) < 2e-3, (ratio, expect)
