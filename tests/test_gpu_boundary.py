"""Non-periodic x and y (bc_x = 1, bc_y = 1, 2D Euler and Navier-Stokes) on the GPU.

* Parity: the boundary flux faces with the reference's order fallback
  (2D_solver/src/calc_{slau,keep,hybrid}_kernel.f90.fypp, calc_*_x / calc_*_y) and
  the boundary-cell rules (zero gradient, slip wall, no-slip wall, fixed values) and
  the viscous stencils next to them (calc_Ev2 / calc_Ev4 with their 2nd-order
  fallback, 2D_solver/src/calc_visc{2,4}.f90.fypp), against the
  oracle's restatement: bit-identical states and stage residuals (FP64, no FMA
  contraction on either side).
* Known answers: the inviscid shock tube (ouxsbli/tests/test_st.py:15-71) through
  the Case API with the reference test's settings (SLAU, TVD hybrid, 6th order,
  TVD-RK3, nx 513, ny 7, one output interval) against the exact Sod solution:
  relative L1 error of density and pressure < 1 %; the oblique shock reflected
  from a slip wall (ouxsbli/tests/test_os.py) with that test's settings against
  the shock relations: pre-shock and post-reflection means within 3 %; the viscous
  decay of a sine shear profile between no-slip walls against the incompressible
  solution u = U sin(pi y / H) exp(-nu pi^2 t / H^2).
"""
import math

import numpy as np
import pytest

from oracle import oracle
from ouxsbli_b200.grid import jacobian, to_qj
from ouxsbli_b200.solver import Solver, SolverConfig

pytestmark = pytest.mark.gpu


def tube(nx, ny, order, **kw):
    """A shock-tube field with a y perturbation, its ghost rows periodic in y."""
    g = order // 2
    L = 1.0
    dx = np.full(nx - 1, L / (nx - 1))
    dy = np.full(ny - 1, 0.3 * L / (ny - 1))
    x = np.concatenate([[0.0], np.cumsum(dx)])
    y = np.concatenate([[0.0], np.cumsum(dy)])
    X, Y = np.meshgrid(x, y, indexing="ij")
    rho = np.where(X < 0.5, 1.0, 0.125) * (1.0 + 0.05 * np.sin(2 * math.pi * Y / (0.3 * L)))
    p = np.where(X < 0.5, 1.0, 0.1)
    u = 0.1 * np.cos(2 * math.pi * Y / (0.3 * L))
    v = 0.05 * np.sin(2 * math.pi * X)
    gam = 1.4
    Q = np.zeros((nx, 4, ny), order="F")
    Q[:, 0], Q[:, 1], Q[:, 2] = rho, rho * u, rho * v
    Q[:, 3] = p / (gam - 1.0) + 0.5 * rho * (u * u + v * v)
    Q[0], Q[-1] = Q[1], Q[-2]
    N = ny - 2 * g
    for j in list(range(g)) + list(range(ny - g, ny)):
        Q[:, :, j] = Q[:, :, g + (j - g) % N]
    cmax = math.sqrt(gam * 1.0 / 0.125) + 0.2
    dt = 0.3 * dx[0] / cmax
    cfg = SolverConfig(dim=2, nx=nx, ny=ny, nz=1, order=order, visc="Euler", bc_x=1, dt=dt, gamma=gam, R=1.0,
                       dx=dx, dy=dy, dz=None, **kw)
    return cfg, to_qj(Q, jacobian(dx, dy, None))


CASES = [
    ("slau6_hybridtvd_rk3", dict(order=6, scheme="SLAU", tvd="hybrid", slau="HRSLAU2", rk=3)),
    ("slau6_tvd_slau1", dict(order=6, scheme="SLAU", tvd="tvd", slau="SLAU", rk=3)),
    ("hybrid6_rk3", dict(order=6, scheme="Hybrid", tvd="hybrid", rk=3)),
    ("keep4_rk4", dict(order=4, scheme="KEEP", rk=4)),
    ("slau4_none_rk4", dict(order=4, scheme="SLAU", tvd="none", rk=4)),
    ("slau2_rk3", dict(order=2, scheme="SLAU", rk=3)),
    ("keep6_rk3", dict(order=6, scheme="KEEP", rk=3)),
]


@pytest.mark.parametrize("name,kw", CASES, ids=[c[0] for c in CASES])
def test_boundary_faces_bitexact_vs_oracle(name, kw, cuda_device):
    cfg, qj = tube(45, 14, **kw)
    s = Solver(cfg, cuda_device)
    s.set_state(qj)
    r_gpu = s.rhs()
    s.step(6)
    q_gpu = s.get_state()
    s.close()
    # residual over every x cell 1..nx-2 and the interior y rows (the y ghost rows
    # are refilled from their periodic images after each stage)
    ys = slice(cfg.g - 1, -(cfg.g - 1) if cfg.g > 1 else None)
    np.testing.assert_array_equal(r_gpu[:, :, ys], oracle.rhs(cfg, qj)[:, :, ys])
    np.testing.assert_array_equal(q_gpu, oracle.step(cfg, qj, 6))


def test_shock_tube_vs_exact_sod(tmp_path, cuda_device):
    import sod_exact
    from ouxsbli_b200 import Case
    from ouxsbli_b200.output import read_vtr
    wd = tmp_path / "st"
    case = Case(source="2D_solver/ST", workdir=str(wd), visc="euler", tvd="hybrid", scheme="slau", accuracy=6,
                rk="tvd_rk3", nx=513, ny=7, np=1)
    case.build()
    case.run(nranks=2, device=cuda_device)
    x, y, z, f = read_vtr(sorted((wd / "data").glob("Q*.vtr"))[-1])
    p = case.globals_used
    rho_num = f["rho"].reshape(y.size, x.size)[3].astype(float)
    p_num = f["p"].reshape(y.size, x.size)[3].astype(float)
    t_end = p["nt"] * p["np"] * p["dt"]
    rho_ex, _, p_ex = sod_exact.solve(x.astype(float), t_end, p["rho0"], 0.0, p["p0"], p["rho1"], 0.0, p["p1"],
                                      gamma=1.4, x0=0.5 * p["Lx"])
    l1_rho = np.mean(np.abs(rho_num - rho_ex)) / np.mean(rho_ex)
    l1_p = np.mean(np.abs(p_num - p_ex)) / np.mean(p_ex)
    assert l1_rho < 0.01 and l1_p < 0.01, (l1_rho, l1_p)


def test_riemann_ic_sod_vs_exact(tmp_path, cuda_device):
    """RiemannIC (ouxsbli/ic.py) on the shock tube: Sod's states in units with
    rho_l = p_l = 1 on a unit tube (SLAU-6, TVD hybrid, RK3, 513 nodes) to t = 0.2,
    against the exact solution: relative L1 of density and pressure < 1 %."""
    import sod_exact
    from ouxsbli_b200 import Case
    from ouxsbli_b200.ic import RiemannIC
    from ouxsbli_b200.output import read_vtr
    wd = tmp_path / "rie"
    dt = 0.3 / 512 / 1.5
    nt = int(round(0.2 / dt))
    case = Case(source="2D_solver/ST", workdir=str(wd), ic=RiemannIC(), visc="euler", tvd="hybrid", scheme="slau",
                accuracy=6, rk="tvd_rk3", nx=513, ny=7, Lx=1.0, Ly=0.1, dt=dt, nt=nt, np=1)
    case.build()
    case.run(device=cuda_device)
    x, y, z, f = read_vtr(sorted((wd / "data").glob("Q*.vtr"))[-1])
    rho = f["rho"].reshape(y.size, x.size)[3].astype(float)
    p = f["p"].reshape(y.size, x.size)[3].astype(float)
    rho_ex, _, p_ex = sod_exact.solve(x.astype(float), nt * dt, 1.0, 0.0, 1.0, 0.125, 0.0, 0.1, gamma=1.4, x0=0.5)
    l1_rho = np.mean(np.abs(rho - rho_ex)) / np.mean(rho_ex)
    l1_p = np.mean(np.abs(p - p_ex)) / np.mean(p_ex)
    assert l1_rho < 0.01 and l1_p < 0.01, (l1_rho, l1_p)


def test_boundary_mixed_close_to_fp64(cuda_device):
    """The mixed form with a non-periodic x: smooth flow (KEEP-4, RK4), relative L2
    against FP64 within the mixed form's bound for switch-free schemes (1e-5)."""
    import dataclasses
    cfg, qj = tube(45, 14, order=4, scheme="KEEP", rk=4)
    out = {}
    for prec in ("fp64", "mixed"):
        s = Solver(dataclasses.replace(cfg, precision=prec), cuda_device)
        s.set_state(qj)
        s.step(20)
        out[prec] = s.get_state()
        s.close()
    for l in range(4):
        a, b = out["mixed"][:, l], out["fp64"][:, l]
        assert np.linalg.norm(a - b) / np.linalg.norm(b) <= 1e-5, l


def duct(nx, ny, order, rules, **kw):
    """A smooth supersonic field on a box non-periodic in x and y, with boundary rules."""
    L = 1.0
    dx = np.full(nx - 1, L / (nx - 1))
    dy = np.full(ny - 1, 0.6 * L / (ny - 1))
    x = np.concatenate([[0.0], np.cumsum(dx)])
    y = np.concatenate([[0.0], np.cumsum(dy)])
    X, Y = np.meshgrid(x, y, indexing="ij")
    gam = 1.4
    rho = 1.0 + 0.2 * np.sin(2 * math.pi * X) * np.cos(math.pi * Y)
    u = 1.8 + 0.1 * np.cos(2 * math.pi * Y)
    v = 0.1 * np.sin(2 * math.pi * X) * np.sin(math.pi * Y / 0.6)
    p = 1.0 / gam + 0.1 * np.cos(2 * math.pi * (X - Y))
    Q = np.zeros((nx, 4, ny), order="F")
    Q[:, 0], Q[:, 1], Q[:, 2] = rho, rho * u, rho * v
    Q[:, 3] = p / (gam - 1.0) + 0.5 * rho * (u * u + v * v)
    J = jacobian(dx, dy, None)
    qj = to_qj(Q, J)
    bnd = {}
    for face, kind in rules.items():
        if kind == "fixed":
            if face.startswith("x"):
                bnd[face] = ("fixed", np.ascontiguousarray(qj[0 if face == "x_lo" else -1, :, :]))
            else:
                bnd[face] = ("fixed", np.ascontiguousarray(qj[:, :, 0 if face == "y_lo" else -1].T))
        else:
            bnd[face] = kind
    dt = 0.3 * dx[0] / (2.0 + math.sqrt(gam * 1.2))
    cfg = SolverConfig(dim=2, nx=nx, ny=ny, nz=1, order=order, visc="Euler", bc_x=1, bc_y=1, dt=dt, gamma=gam,
                       R=1.0, dx=dx, dy=dy, dz=None, boundary=bnd, **kw)
    return cfg, qj


OS_RULES = {"x_lo": "fixed", "x_hi": "zero_gradient", "y_lo": "slip_wall", "y_hi": "fixed"}
WALLS = {"x_lo": "slip_wall", "x_hi": "slip_wall", "y_lo": "slip_wall", "y_hi": "zero_gradient"}
DUCT_CASES = [
    ("os_slau6_hybrid_rk3", OS_RULES, dict(order=6, scheme="SLAU", tvd="hybrid", slau="HRSLAU2", rk=3)),
    ("os_hybrid6_rk3", OS_RULES, dict(order=6, scheme="Hybrid", tvd="hybrid", rk=3)),
    ("walls_keep6_rk4", WALLS, dict(order=6, scheme="KEEP", rk=4)),
    ("walls_slau4_tvd_rk3", WALLS, dict(order=4, scheme="SLAU", tvd="tvd", slau="SLAU", rk=3)),
    ("os_keep4_rk4", OS_RULES, dict(order=4, scheme="KEEP", rk=4)),
    ("os_slau2_rk3", OS_RULES, dict(order=2, scheme="SLAU", rk=3)),
]


@pytest.mark.parametrize("name,rules,kw", DUCT_CASES, ids=[c[0] for c in DUCT_CASES])
def test_xy_boundaries_bitexact_vs_oracle(name, rules, kw, cuda_device):
    cfg, qj = duct(41, 23, rules=rules, **kw)
    s = Solver(cfg, cuda_device)
    s.set_state(qj)
    r_gpu = s.rhs()
    s.step(6)
    q_gpu = s.get_state()
    s.close()
    np.testing.assert_array_equal(r_gpu, oracle.rhs(cfg, qj))
    np.testing.assert_array_equal(q_gpu, oracle.step(cfg, qj, 6))


def test_xy_fill_matches_oracle(cuda_device):
    """oux_fill_ghosts with the OS rule set: every boundary cell, corners included."""
    cfg, qj = duct(33, 17, order=6, rules=OS_RULES, scheme="SLAU")
    rng = np.random.default_rng(5)
    q = np.asfortranarray(qj * (1.0 + 0.01 * rng.standard_normal(qj.shape)))
    s = Solver(cfg, cuda_device)
    s.set_state(q)
    s.fill_ghosts()
    out = s.get_state()
    s.close()
    np.testing.assert_array_equal(out, oracle.fill_ghosts(cfg, q))


def test_xy_mixed_close_to_fp64(cuda_device):
    """The mixed form with non-periodic x and y (KEEP-4, RK4, walls and fixed faces):
    relative L2 against FP64 within the mixed form's bound for switch-free schemes."""
    import dataclasses
    cfg, qj = duct(41, 23, order=4, rules=OS_RULES, scheme="KEEP", rk=4)
    out = {}
    for prec in ("fp64", "mixed"):
        s = Solver(dataclasses.replace(cfg, precision=prec), cuda_device)
        s.set_state(qj)
        s.step(20)
        out[prec] = s.get_state()
        s.close()
    for l in range(4):
        a, b = out["mixed"][:, l], out["fp64"][:, l]
        assert np.linalg.norm(a - b) / np.linalg.norm(b) <= 1e-5, l


def test_neumann_faces_2d_bitexact_vs_oracle(cuda_device):
    """OUX_BC_NEUMANN on 2D faces (the top and the outflow of a supersonic duct with a
    slip floor and fixed inflow; SLAU-4, RK3): the residual and the state after 6 steps
    bit-identical to the oracle."""
    rules = {"x_lo": "fixed", "x_hi": "neumann", "y_lo": "slip_wall", "y_hi": "neumann"}
    cfg, qj = duct(41, 23, order=4, rules=rules, scheme="SLAU", tvd="hybrid", rk=3)
    s = Solver(cfg, cuda_device)
    s.set_state(qj)
    r = s.rhs()
    s.step(6)
    q = s.get_state()
    s.close()
    np.testing.assert_array_equal(r, oracle.rhs(cfg, qj))
    np.testing.assert_array_equal(q, oracle.step(cfg, qj, 6))


def test_reflected_oblique_shock_vs_shock_relations(tmp_path, cuda_device):
    """ouxsbli/tests/test_os.py with its settings: M0 2, p_tot 100 kPa, T_tot 295 K,
    incident shock 37.2 deg, 257 x 129 nodes on 5 x 2 mm, dt 3 ns, 0.1 ms in one
    output interval.  Pre-shock region (left 10 %, upper half) against the free
    stream, post-reflection region (right 10 %, lower third) against the state
    behind the reflected shock; each mean within 3 %, and |v| / u3 < 3 %."""
    import oblique_shock as osk
    from ouxsbli_b200 import Case
    from ouxsbli_b200.output import read_vtr
    wd = tmp_path / "os"
    R, gamma, M0, p_tot, T_tot = 287.03, 1.4, 2.0, 100.0e3, 295.0
    beta, dt, endT = math.pi * 37.2 / 180.0, 3.0e-9, 0.1e-3
    case = Case(source="2D_solver/OS", workdir=str(wd), scheme="slau", accuracy=6, visc="euler", tvd="hybrid",
                nx=257, ny=129, Lx=5.0e-3, Ly=2.0e-3, gamma=gamma, Pr=0.72, R=R, M0=M0, p_tot=p_tot, T_tot=T_tot,
                beta=beta, dt=dt, np=1, nt=int(endT / dt))
    case.build()
    case.run(nranks=2, device=cuda_device)
    x, y, z, f = read_vtr(sorted((wd / "data").glob("Q*.vtr"))[-1])
    ni, nj = x.size, y.size
    rho = f["rho"].reshape(nj, ni).astype(float)
    p = f["p"].reshape(nj, ni).astype(float)
    vel = f["velocity"].reshape(nj, ni, 3).astype(float)
    u, v = vel[..., 0], vel[..., 1]
    rho1, u1, p1 = osk.free_stream(M0, p_tot, T_tot, gamma, R)
    rho3, ux3, _, p3, _ = osk.reflected_state(M0, p_tot, T_tot, beta, gamma, R)
    pre = (slice(nj // 2, None), slice(None, ni // 10))
    post = (slice(None, nj // 3), slice(9 * ni // 10, None))

    def close(a, b, label):
        assert abs(a - b) / abs(b) < 0.03, (label, a, b)

    close(rho[pre].mean(), rho1, "pre rho")
    close(u[pre].mean(), u1, "pre u")
    close(p[pre].mean(), p1, "pre p")
    close(rho[post].mean(), rho3, "post rho")
    close(u[post].mean(), ux3, "post u")
    close(p[post].mean(), p3, "post p")
    assert abs(v[post].mean()) / ux3 < 0.03, v[post].mean()


def wall_channel(nx_int, ny, order, visc_order, rules, bc_x=0, scheme="KEEP", U=5.0, perturb=True, **kw):
    """A viscous (Sutherland, air) shear flow between y walls 1 mm apart, periodic or
    non-periodic in x; u = U sin(pi y / H) (+ a perturbation), uniform rho and p."""
    from ouxsbli_b200.grid import cyclic_axis
    g = order // 2
    H, Lx, R, gam = 1.0e-3, 0.5e-3, 287.03, 1.4
    if bc_x:
        nx = nx_int + 2
        dx = np.full(nx - 1, Lx / (nx - 1))
        x = np.concatenate([[0.0], np.cumsum(dx)])
    else:
        nx = nx_int + 2 * g
        x, dx = cyclic_axis(nx, Lx, order)
    dy = np.full(ny - 1, H / (ny - 1))
    y = np.concatenate([[0.0], np.cumsum(dy)])
    X, Y = np.meshgrid(x, y, indexing="ij")
    rho = np.full_like(X, 1.2)
    u = U * np.sin(math.pi * Y / H)
    v = np.zeros_like(X)
    if perturb:
        rho = rho * (1.0 + 0.02 * np.sin(2 * math.pi * X / Lx) * np.sin(math.pi * Y / H))
        v = 0.3 * U * np.sin(2 * math.pi * X / Lx) * np.sin(math.pi * Y / H) ** 2
    p = np.full_like(X, 1.2 * R * 300.0)
    Q = np.zeros((nx, 4, ny), order="F")
    Q[:, 0], Q[:, 1], Q[:, 2] = rho, rho * u, rho * v
    Q[:, 3] = p / (gam - 1.0) + 0.5 * rho * (u * u + v * v)
    if not bc_x:
        N = nx - 2 * g
        for i in list(range(g)) + list(range(nx - g, nx)):
            Q[i] = Q[g + (i - g) % N]
    J = jacobian(dx, dy, None)
    qj = to_qj(Q, J)
    bnd = {}
    for face, kind in rules.items():
        if kind == "fixed":
            bnd[face] = ("fixed", np.ascontiguousarray(qj[0 if face == "x_lo" else -1, :, :]))
        else:
            bnd[face] = kind
    dt = 0.5 * min(dx.min(), dy.min()) / (U + math.sqrt(gam * R * 300.0))
    cfg = SolverConfig(dim=2, nx=nx, ny=ny, nz=1, order=order, visc="NS", visc_order=visc_order, bc_x=bc_x,
                       bc_y=1, dt=dt, gamma=gam, R=R, Pr=0.72, dx=dx, dy=dy, dz=None, scheme=scheme,
                       boundary=bnd, **kw)
    return cfg, qj, y


CHANNEL = {"y_lo": "noslip_wall", "y_hi": "noslip_wall"}
BL_RULES = {"x_lo": "fixed", "x_hi": "zero_gradient", "y_lo": "noslip_wall", "y_hi": "slip_wall"}
NS_CASES = [
    ("channel_keep4_v4_rk4", CHANNEL, 0, dict(order=4, visc_order=4, scheme="KEEP", rk=4)),
    ("channel_slau2_v2_rk3", CHANNEL, 0, dict(order=2, visc_order=2, scheme="SLAU", rk=3)),
    ("channel_hybrid6_v4_rk3", CHANNEL, 0, dict(order=6, visc_order=4, scheme="Hybrid", tvd="hybrid", rk=3)),
    ("bl_slau2_v4_rk3", BL_RULES, 1, dict(order=2, visc_order=4, scheme="SLAU", rk=3)),
    ("bl_slau6_v4_tvd_rk3", BL_RULES, 1, dict(order=6, visc_order=4, scheme="SLAU", tvd="hybrid", rk=3)),
    ("bl_keep4_v2_rk4", BL_RULES, 1, dict(order=4, visc_order=2, scheme="KEEP", rk=4)),
]


@pytest.mark.parametrize("name,rules,bc_x,kw", NS_CASES, ids=[c[0] for c in NS_CASES])
def test_viscous_walls_bitexact_vs_oracle(name, rules, bc_x, kw, cuda_device):
    cfg, qj, _ = wall_channel(24, 21, rules=rules, bc_x=bc_x, **kw)
    s = Solver(cfg, cuda_device)
    s.set_state(qj)
    r_gpu = s.rhs()
    s.step(6)
    q_gpu = s.get_state()
    s.close()
    # residual of the updated cells: with a periodic x the ghost columns are refilled
    # from their images after each stage (the oracle, like the reference, updates them
    # first)
    xs = slice(cfg.g - 1, -(cfg.g - 1)) if not bc_x and cfg.g > 1 else slice(None)
    np.testing.assert_array_equal(r_gpu[xs], oracle.rhs(cfg, qj)[xs])
    np.testing.assert_array_equal(q_gpu, oracle.step(cfg, qj, 6))


def test_viscous_walls_mixed_close_to_fp64(cuda_device):
    import dataclasses
    cfg, qj, _ = wall_channel(24, 21, rules=BL_RULES, bc_x=1, order=4, visc_order=4, scheme="KEEP", rk=4)
    out = {}
    for prec in ("fp64", "mixed"):
        s = Solver(dataclasses.replace(cfg, precision=prec), cuda_device)
        s.set_state(qj)
        s.step(20)
        out[prec] = s.get_state()
        s.close()
    for l in range(4):
        a, b = out["mixed"][:, l], out["fp64"][:, l]
        assert np.linalg.norm(a - b) / np.linalg.norm(b) <= 1e-5, l


@pytest.mark.parametrize("order,visc_order,scheme", [(4, 4, "KEEP"), (2, 2, "SLAU")])
def test_shear_decay_between_noslip_walls(order, visc_order, scheme, cuda_device):
    """u = U sin(pi y / H) between no-slip walls (periodic x, Mach 0.015): the mode
    decays as exp(-nu pi^2 t / H^2), nu = mu(T) / rho (Sutherland, 300 K, rho 1.2).
    After 2 ms (amplitude ratio 0.74) the measured ratio is within 0.2 %."""
    cfg, qj, y = wall_channel(8, 41, order, visc_order, CHANNEL, scheme=scheme, perturb=False, rk=3)
    H, T0 = 1.0e-3, 300.0
    mu = 1.716e-5 * 384.2 * 273.2 ** -1.5 / (T0 + 111.0) * T0 ** 1.5
    nu = mu / 1.2
    t_end = 2.0e-3
    nsteps = int(round(t_end / cfg.dt))
    s = Solver(cfg, cuda_device)
    s.set_state(qj)
    s.step(nsteps)
    q = s.get_state()
    s.close()
    J = jacobian(cfg.dx, cfg.dy, None)
    sin = np.sin(math.pi * y / H)

    def amplitude(qq):
        u = (qq[:, 1] / qq[:, 0])[cfg.g:-cfg.g].mean(axis=0)  # x-average (the flow is x-uniform)
        return float(np.sum(u * sin) / np.sum(sin * sin))

    ratio = amplitude(q) / amplitude(qj)
    expect = math.exp(-nu * math.pi ** 2 * nsteps * cfg.dt / H ** 2)
    assert abs(ratio / expect - 1.0) < 2e-3, (ratio, expect)


def test_walled_members_in_one_batch_bitexact(cuda_device):
    """Batched steps (one persistent kernel over all members) with non-periodic members
    beside a periodic one: every member bit-identical to its single-solve run."""
    from helpers import vortex2d
    from ouxsbli_b200.batch import Batch
    euler = [duct(33, 17, order=4, rules=OS_RULES, scheme="SLAU", tvd="hybrid", rk=3),
             duct(41, 23, order=4, rules=WALLS, scheme="KEEP", rk=3),
             vortex2d(36, order=4, beta=2.0, mach=0.4, scheme="KEEP", visc="Euler", rk=3)]
    viscous = [wall_channel(24, 21, order=4, visc_order=4, rules=CHANNEL, scheme="KEEP", rk=4)[:2],
               wall_channel(16, 25, order=4, visc_order=4, rules=BL_RULES, bc_x=1, scheme="SLAU", rk=4)[:2]]
    for cases in (euler, viscous):
        ref = []
        for cfg, qj in cases:
            s = Solver(cfg, cuda_device)
            s.set_state(qj)
            s.step(5)
            ref.append(s.get_state())
            s.close()
        solvers = []
        for cfg, qj in cases:
            s = Solver(cfg, cuda_device)
            s.set_state(qj)
            solvers.append(s)
        b = Batch(solvers)
        b.step(5)
        assert b.status() == 0
        for s, r in zip(solvers, ref):
            np.testing.assert_array_equal(s.get_state(), r)
        b.close()
        for s in solvers:
            s.close()


def test_bl0_case_matches_oracle(tmp_path, cuda_device):
    """The BL0 case (inflow, split bottom face with a no-slip plate, characteristic far
    field on top, y-last corners; NS SLAU-2 with the Gaitonde-Visbal stencil) through
    Case.run, 5 steps, against the oracle. The far-field rule evaluates pow (libm on
    the host, CUDA on the device), so the states agree to rounding, not bit for bit."""
    from ouxsbli_b200 import Case
    c = Case("2D_solver/BL0", tmp_path / "bl0", nx=65, ny=33, nt=5, np=1)
    c.build()
    c.run(device=cuda_device)
    p, xc, yc, zc, dx, dy, dz, Q = c._initial()
    cfg = c._solver_config(p, dx, dy, dz)
    want = oracle.step(cfg, to_qj(Q, jacobian(dx, dy, None)), 5)
    np.testing.assert_allclose(c.solver.get_state(), want, rtol=1e-12, atol=0)


def bl_profile_file(path, p, rows):
    """A compressible laminar layer (the BL0 constants, 99 % thickness 0.75 mm) written
    in the BL inflow profile format: rows of (y, rho, u, v, p)."""
    from ouxsbli_b200.blasius import compressible_profile
    from ouxsbli_b200.cases import sutherland_mu
    y = np.linspace(0.0, 3.0e-3, rows)
    cp = p["gamma"] * p["R"] / (p["gamma"] - 1.0)
    rho, u, v, T = compressible_profile(y, 0.75e-3, p["u0"], p["T0"], p["p0"], p["R"], cp, p["rf"], p["Taw"],
                                        sutherland_mu(p["T0"]))
    prof = np.stack([y, p["p0"] / (p["R"] * T), u, v, np.full_like(y, p["p0"])], axis=1)
    prof.astype("<f8").tofile(path)
    return path


def test_bl_case_matches_oracle(tmp_path, cuda_device):
    """The BL case (an inflow profile from a file, zero-gradient outlet and top, an
    adiabatic no-slip floor, y-last corners; NS SLAU-2 with the 4th-order viscous
    stencil on the 2nd-order grid) through Case.run, 5 steps, bit for bit against the
    oracle."""
    from ouxsbli_b200 import Case
    from ouxsbli_b200.cases import CASES, _bl_derived
    p = _bl_derived(dict(CASES["BL"].params, Lx=0.02))
    f = bl_profile_file(tmp_path / "Qin.dat", p, 30)
    c = Case("2D_solver/BL", tmp_path / "bl", nx=65, ny=33, nt=5, np=1, inflow=str(f))
    c.build()
    c.run(device=cuda_device)
    p, xc, yc, zc, dx, dy, dz, Q = c._initial()
    cfg = c._solver_config(p, dx, dy, dz)
    assert (cfg.order, cfg.visc_order) == (2, 4)
    want = oracle.step(cfg, to_qj(Q, jacobian(dx, dy, None)), 5)
    np.testing.assert_array_equal(c.solver.get_state(), want)


def test_bl0_flat_plate_skin_friction(tmp_path, cuda_device):
    """BL0 at its own settings (Mach 2, 1025 x 129 nodes, 0.4 ms = 5 flow-through
    times): the laminar boundary layer on the adiabatic plate. Skin friction from the
    discrete wall shear (face-averaged Sutherland mu times the wall-face velocity
    gradient) against the plate's similarity law: Cf sqrt(Re_x) constant downstream
    (spread < 3 %) and within 8 % of the Eckert reference-temperature value
    0.664 sqrt(C*), C* = rho* mu* / (rho_e mu_e) at T* = Te (1 + 0.032 M^2 +
    0.58 (Tw / Te - 1)), Tw = Te (1 + sqrt(Pr) (gamma - 1) / 2 M^2)."""
    from ouxsbli_b200 import Case
    c = Case("2D_solver/BL0", tmp_path / "bl0", np=1, nt=133333)
    c.build()
    c.run(device=cuda_device)
    p, xc, yc, zc, dx, dy, dz, Q = c._initial()
    q = c.solver.get_state()
    J = jacobian(dx, dy, None)
    g, R, M0 = p["gamma"], p["R"], p["M0"]
    rho = q[:, 0] * J
    u = q[:, 1] / q[:, 0]
    v = q[:, 2] / q[:, 0]
    pr = (g - 1.0) * (q[:, 3] * J - 0.5 * rho * (u * u + v * v))
    T = pr / (rho * R)

    def mu(t):
        return 1.716e-5 * 384.2 * 273.2 ** -1.5 / (t + 111.0) * t ** 1.5

    Te, rho_e, u_e = p["T0"], p["rho0"], p["u0"]
    x_le = xc[p["nx"] // 10 - 1]
    vals = []
    for frac in np.linspace(0.45, 0.95, 6):
        i = int(frac * (p["nx"] - 1))
        tau = 0.5 * (mu(T[i, 0]) + mu(T[i, 1])) * (u[i, 1] - u[i, 0]) / (yc[1] - yc[0])
        rex = rho_e * u_e * (xc[i] - x_le) / mu(Te)
        vals.append(tau / (0.5 * rho_e * u_e ** 2) * math.sqrt(rex))
    vals = np.array(vals)
    Tw = Te * (1.0 + math.sqrt(p["Pr"]) * 0.5 * (g - 1.0) * M0 ** 2)
    Ts = Te * (1.0 + 0.032 * M0 ** 2 + 0.58 * (Tw / Te - 1.0))
    eckert = 0.664 * math.sqrt(mu(Ts) / mu(Te) * Te / Ts)
    assert vals.max() / vals.min() - 1.0 < 0.03, vals
    assert abs(vals.mean() / eckert - 1.0) < 0.08, (vals, eckert)


def test_sbli_case_matches_oracle(tmp_path, cuda_device):
    """2D_solver/SBLI through Case.run (periodic x, no-slip wall and fixed free stream
    in y, NS SLAU-6 with the 2D 4th-order viscous stencil, the compressible laminar
    initial layer), 5 steps, against the oracle: bit-identical."""
    from ouxsbli_b200 import Case
    c = Case("2D_solver/SBLI", tmp_path / "sbli", nx=70, ny=41, nt=5, np=1)
    c.build()
    c.run(device=cuda_device)
    p, xc, yc, zc, dx, dy, dz, Q = c._initial()
    cfg = c._solver_config(p, dx, dy, dz)
    np.testing.assert_array_equal(c.solver.get_state(), oracle.step(cfg, to_qj(Q, jacobian(dx, dy, None)), 5))
