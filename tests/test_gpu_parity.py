"""GPU parity: liboux's FP64 path against the CPU oracle, through the C ABI.

The FP64 kernels are built without FMA contraction and evaluate the reference
formulas in the reference's operation order, so the expected agreement is
bit-for-bit (tolerance 0) for every configuration; the 100-step test also
states the north-star bound (relative L2 <= 1e-9 per conservative variable).
"""
import numpy as np
import pytest

from helpers import interior, random_turbulence, rel_l2, rhs_interior, tgv, vortex2d
from oracle import oracle

pytestmark = pytest.mark.gpu

CONFIGS = [
    ("ns_slau6_hrslau2_tvdhybrid", lambda: tgv(16, scheme="SLAU", visc="NS", slau="HRSLAU2", tvd="hybrid")),
    ("ns_slau6_slau1_tvd", lambda: tgv(16, scheme="SLAU", visc="NS", slau="SLAU", tvd="tvd")),
    ("ns_slau6_none", lambda: tgv(16, scheme="SLAU", visc="NS", tvd="none")),
    ("ns_hybrid6_c6", lambda: tgv(16, mach=1.25, scheme="Hybrid", visc="NS")),
    ("ns_hybrid6_me4", lambda: tgv(16, mach=1.25, scheme="Hybrid", visc="NS", visc_stencil="ME4Base")),
    ("ns_slau6_c4", lambda: tgv(16, scheme="SLAU", visc="NS", visc_order=4)),
    ("euler_keep6_rk4", lambda: tgv(16, scheme="KEEP", visc="Euler", rk=4)),
    ("euler_roe6_tvd", lambda: tgv(16, scheme="Roe", visc="Euler", tvd="tvd")),
    ("ns_roe4_c4", lambda: tgv(16, order=4, scheme="Roe", visc="NS")),
    ("les_slau6_c6", lambda: random_turbulence(16, seed=3, scheme="SLAU", visc="LES")),
    ("les_hybrid6_me4", lambda: random_turbulence(16, seed=4, scheme="Hybrid", visc="LES", visc_stencil="ME4Base")),
    ("les_keep4_c4", lambda: random_turbulence(16, order=4, seed=5, scheme="KEEP", visc="LES")),
    ("ns_keep4_gv2", lambda: tgv(16, order=4, scheme="KEEP", visc="NS", visc_order=2)),
    ("ns_keep2_gv2", lambda: tgv(16, order=2, scheme="KEEP", visc="NS")),
    ("les_hybrid2_gv2_rk4", lambda: random_turbulence(16, order=2, seed=6, scheme="Hybrid", visc="LES", rk=4)),
    ("euler_slau2_rk4", lambda: tgv(16, order=2, scheme="SLAU", visc="Euler", rk=4)),
    ("ragged_17x20x23", lambda: _ragged()),
    ("2d_keep4_rk4", lambda: vortex2d(32, order=4, scheme="KEEP", visc="Euler", rk=4)),
    ("2d_keep6_rk4", lambda: vortex2d(32, order=6, scheme="KEEP", visc="Euler", rk=4)),
    ("2d_keep2_rk3", lambda: vortex2d(32, order=2, scheme="KEEP", visc="Euler", rk=3)),
    ("2d_slau6", lambda: vortex2d(32, order=6, scheme="SLAU", visc="Euler")),
    ("2d_hybrid4_ns4", lambda: vortex2d(32, order=4, scheme="Hybrid", visc="NS", visc_order=4)),
    ("2d_slau4_gv2", lambda: vortex2d(32, order=4, scheme="SLAU", visc="NS", visc_order=2)),
    ("2d_hybrid2_gv2", lambda: vortex2d(32, order=2, scheme="Hybrid", visc="NS")),
]


def _ragged():
    """Non-cubic interior 17 x 20 x 23 (no dimension a multiple of the tiles)."""
    from ouxsbli_b200.grid import cyclic_axis, jacobian, to_qj
    from ouxsbli_b200.solver import SolverConfig
    from ouxsbli_b200.turbulence import solenoidal_field
    import math
    order = 6
    n = (17, 20, 23)
    axes = [cyclic_axis(m + order, 2.0 * math.pi, order) for m in n]
    rng = np.random.default_rng(11)
    Q = np.zeros((n[0] + 6, 5, n[1] + 6, n[2] + 6), order="F")
    Q[:, 0] = 1.0 + 0.05 * rng.standard_normal((n[0] + 6, n[1] + 6, n[2] + 6))
    for a in range(3):
        Q[:, 1 + a] = 0.2 * rng.standard_normal((n[0] + 6, n[1] + 6, n[2] + 6)) * Q[:, 0]
    Q[:, 4] = 2.5 + 0.5 * (Q[:, 1] ** 2 + Q[:, 2] ** 2 + Q[:, 3] ** 2) / Q[:, 0]
    from ouxsbli_b200.grid import fill_periodic
    fill_periodic(Q, 3)
    dx, dy, dz = axes[0][1], axes[1][1], axes[2][1]
    cfg = SolverConfig(dim=3, nx=n[0] + 6, ny=n[1] + 6, nz=n[2] + 6, order=6, scheme="Hybrid", visc="NS",
                       gamma=1.4, R=1.0, Pr=0.71, dt=1e-3, dx=dx, dy=dy, dz=dz)
    # Sutherland's law expects Kelvin temperatures: keep T = p / (R rho) ~ 2.5 / 1
    return cfg, to_qj(Q, jacobian(dx, dy, dz))


@pytest.mark.parametrize("name,make", CONFIGS, ids=[c[0] for c in CONFIGS])
def test_rhs_and_steps_bitexact(name, make, cuda_device):
    """Bit-exact for every configuration without transcendental functions.

    The LES configurations call pow/log/cosh in the SMS model (calc_les.f90:30-71);
    CUDA's libm and the host's glibc may round those 1 ulp apart, so LES is held
    to relative tolerances instead: max |dR| <= 1e-11 max |R| and, after 3 steps,
    relative L2 <= 1e-12 per conservative variable."""
    from ouxsbli_b200.solver import Solver
    cfg, qj = make()
    s = Solver(cfg, cuda_device)
    s.set_state(qj)
    g = cfg.g
    r_gpu = rhs_interior(s.rhs(), g, cfg.dim)
    r_orc = rhs_interior(oracle.rhs(cfg, qj), g, cfg.dim)
    assert np.isfinite(r_orc).all()
    les = cfg.visc == "LES"
    if les:
        assert np.abs(r_gpu - r_orc).max() <= 1e-11 * np.abs(r_orc).max()
    else:
        np.testing.assert_array_equal(r_gpu, r_orc)
    s.step(3)
    q_gpu = s.get_state()
    q_orc = oracle.step(cfg, qj, 3)
    if les:
        a, b = interior(q_gpu, g, cfg.dim), interior(q_orc, g, cfg.dim)
        for l in range(cfg.nv):
            assert rel_l2(a[:, l], b[:, l]) <= 1e-12
    else:
        np.testing.assert_array_equal(q_gpu, q_orc)
    s.close()


def test_plain_method_100_steps(cuda_device):
    """Plain-method config at reduced size: NS SLAU/HRSLAU2 6th, Central-6, RK3, 100 steps.

    Tolerance stated by the north star: relative L2 <= 1e-9 per conservative variable;
    the FP64 path is expected to be bit-identical (0)."""
    from ouxsbli_b200.solver import Solver
    cfg, qj = tgv(24, scheme="SLAU", visc="NS", slau="HRSLAU2", tvd="hybrid")
    s = Solver(cfg, cuda_device)
    s.set_state(qj)
    s.step(100)
    q_gpu = s.get_state()
    q_orc = oracle.step(cfg, qj, 100)
    a, b = interior(q_gpu, cfg.g, 3), interior(q_orc, cfg.g, 3)
    for l in range(5):
        assert rel_l2(a[:, l], b[:, l]) <= 1e-9
    assert np.array_equal(q_gpu, q_orc)
    s.close()


def test_ghost_fill_matches_periodic_images(cuda_device):
    from ouxsbli_b200.grid import fill_periodic
    from ouxsbli_b200.solver import Solver
    cfg, qj = tgv(12, scheme="KEEP", visc="Euler")
    noisy = qj.copy(order="F")
    rng = np.random.default_rng(1)
    noisy += 1e-3 * rng.standard_normal(noisy.shape) * np.abs(noisy).max()
    s = Solver(cfg, cuda_device)
    s.set_state(noisy)
    s.fill_ghosts()
    got = s.get_state()
    want = noisy.copy(order="F")
    fill_periodic(want, cfg.g)
    np.testing.assert_array_equal(got, want)


def test_diagnostics_fp64(cuda_device):
    """KE / entropy / enstrophy means against a numpy evaluation on the same state."""
    from ouxsbli_b200.grid import jacobian
    from ouxsbli_b200.solver import Solver
    cfg, qj = tgv(16, scheme="SLAU", visc="NS")
    s = Solver(cfg, cuda_device)
    s.set_state(qj)
    ke, ent, ens = s.diagnostics()
    f = oracle.fields(cfg, qj)
    g = cfg.g
    sl = (slice(g, -g),) * 3
    rho, u, v, w, p = (f[k][sl] for k in ("rho", "u", "v", "w", "p"))
    ke_ref = np.mean(0.5 * rho * (u * u + v * v + w * w))
    ent_ref = np.mean(rho * np.log(p * rho ** (-cfg.gamma)))
    inv = 1.0 / cfg.dx[0]

    def d6(a, axis):
        r = lambda m: np.roll(a, -m, axis=axis)
        return ((1.0 / 60.0) * (-r(-3) + r(3)) + 0.15 * (r(-2) - r(2)) + 0.75 * (-r(-1) + r(1))) * inv

    U, V, W = (f[k] for k in ("u", "v", "w"))
    om = [d6(W, 1) - d6(V, 2), d6(U, 2) - d6(W, 0), d6(V, 0) - d6(U, 1)]
    ens_ref = np.mean(0.5 * f["rho"][sl] * sum(o[sl] ** 2 for o in om))
    assert abs(ke - ke_ref) <= 1e-12 * abs(ke_ref)
    assert abs(ent - ent_ref) <= 1e-12 * abs(ent_ref)
    assert abs(ens - ens_ref) <= 1e-10 * abs(ens_ref)


def test_check_state_flags_bad_cells(cuda_device):
    """Host-planted NaN / negative density is reported by the device status word."""
    from ouxsbli_b200 import _lib
    from ouxsbli_b200.solver import Solver
    cfg, qj = tgv(12, scheme="KEEP", visc="Euler")
    s = Solver(cfg, cuda_device)
    s.set_state(qj)
    assert s.check_state() == 0
    bad = qj.copy(order="F")
    bad[5, 0, 5, 5] = -1.0
    s.set_state(bad)
    assert s.check_state() & _lib.FAULT_NONPOSITIVE
    bad[6, 4, 6, 6] = np.nan
    s.set_state(bad)
    assert s.check_state() & _lib.FAULT_NAN


@pytest.mark.parametrize("world,rk,precision", [(2, 3, "fp64"), (3, 4, "fp64"), (2, 3, "mixed")])
def test_z_slabs_match_the_undivided_solve(world, rk, precision, cuda_device):
    """COMMZ on one GPU: `world` z slabs of a 3D solve, each a bc_z = 2 handle, stepped
    stage by stage with halo exchange by device copies, against the undivided solve.
    FP64: bit-identical; mixed: each slab keeps its own p / T references, so FP32
    rounding differs from the undivided mixed run (relative L2 <= 1e-6)."""
    import dataclasses
    from ouxsbli_b200.slabs import LocalSlabs
    from ouxsbli_b200.solver import Solver, SolverConfig
    from ouxsbli_b200.cases import CASES, build_initial
    from ouxsbli_b200.grid import jacobian, to_qj
    p = dict(CASES["NSTGV"].params)
    n = 24 + 6
    p.update(nx=n, ny=n, nz=n, order=6, M0=1.25, rho_mode="uniform", cfl_mode="acoustic", CFL=0.5, dt=None)
    p, xc, yc, zc, dx, dy, dz, Q = build_initial(CASES["NSTGV"], p)
    cfg = SolverConfig(dim=3, nx=n, ny=n, nz=n, order=6, scheme="Hybrid", visc="NS", tvd="hybrid", rk=rk,
                       gamma=p["gamma"], R=p["R"], Pr=p["Pr"], dt=p["dt"], dx=dx, dy=dy, dz=dz,
                       precision=precision)
    qj = to_qj(Q, jacobian(dx, dy, dz))
    s = Solver(cfg, cuda_device)
    s.set_state(qj)
    s.step(4)
    whole = s.get_state()
    s.close()
    slabs = LocalSlabs(cfg, world, cuda_device)
    slabs.set_state(qj)
    slabs.step(4)
    got = slabs.get_state()
    slabs.close()
    g = cfg.g
    a, b = got[:, :, :, g:-g], whole[:, :, :, g:-g]
    if precision == "fp64":
        np.testing.assert_array_equal(a, b)
    else:
        for l in range(5):
            assert np.linalg.norm(a[:, l] - b[:, l]) / np.linalg.norm(b[:, l]) <= 1e-6, l


@pytest.mark.parametrize("slabs", [2, 4])
def test_stz_slabs_with_walls_match_the_oracle(slabs, tmp_path, cuda_device):
    """3D_solver/STZ through Case.run: the grid in z slabs (the first and last with
    the grid's zero-gradient ends, the inner ones exchanging halos) with slip walls in
    x and y, 6 steps, against the oracle on the undivided grid: bit-identical."""
    from ouxsbli_b200 import Case
    from ouxsbli_b200.grid import jacobian, to_qj
    c = Case("3D_solver/STZ", tmp_path / "stz", nz=33, nt=6, np=1, slabs=slabs)
    c.build()
    c.run(device=cuda_device)
    p, xc, yc, zc, dx, dy, dz, Q = c._initial()
    cfg = c._solver_config(p, dx, dy, dz)
    np.testing.assert_array_equal(c.solver.get_state(), oracle.step(cfg, to_qj(Q, jacobian(dx, dy, dz)), 6))


def test_stz_shock_tube_along_z_vs_exact_sod(tmp_path, cuda_device):
    """3D_solver/STZ at its own settings (two slabs of 511 interior planes, SLAU1 /
    TVD minmod order 2, 50 x 102 steps to t = 0.0996): the profile along z against
    the exact Sod solution, relative L1 of density and pressure < 1 %."""
    import sod_exact
    from ouxsbli_b200 import Case
    from ouxsbli_b200.grid import jacobian
    c = Case("3D_solver/STZ", tmp_path / "stz")
    c.build()
    c.run(device=cuda_device)
    p, xc, yc, zc, dx, dy, dz, Q = c._initial()
    q = c.solver.get_state()
    J = jacobian(dx, dy, dz)
    rho = q[2, 0, 2] * J[2, 2]
    w = q[2, 3, 2] / q[2, 0, 2]
    pr = 0.4 * (q[2, 4, 2] * J[2, 2] - 0.5 * rho * w * w)
    t = p["nt"] * p["np"] * p["dt"]
    z = zc[1:-1]
    re, _, pe = sod_exact.solve(z, t, p["rho_L"], 0.0, p["p_L"], p["rho_R"], 0.0, p["p_R"], gamma=1.4, x0=0.5)
    l1_rho = np.mean(np.abs(rho[1:-1] - re)) / np.mean(re)
    l1_p = np.mean(np.abs(pr[1:-1] - pe)) / np.mean(pe)
    assert l1_rho < 0.01 and l1_p < 0.01, (l1_rho, l1_p)


def _box3d(n, nz, order, rules, scheme, rk, tvd="hybrid", tube=False):
    """A 3D Euler field in a box non-periodic in x, y and z (one boundary cell a side)."""
    import math
    from ouxsbli_b200.grid import jacobian, to_qj
    from ouxsbli_b200.solver import SolverConfig
    L = 1.0
    dx = np.full(n - 1, 0.2 * L / (n - 1))
    dz = np.full(nz - 1, L / (nz - 2))
    x = np.concatenate([[0.0], np.cumsum(dx)])
    z = dz[0] * (np.arange(nz) - 0.5)
    X, Y, Z = np.meshgrid(x, x, z, indexing="ij")
    gam = 1.4
    if tube:
        rho = np.where(Z < 0.5, 1.0, 0.125)
        p = np.where(Z < 0.5, 1.0, 0.1)
        u = v = w = np.zeros_like(Z)
    else:
        rho = 1.0 + 0.2 * np.sin(2 * math.pi * Z) * np.cos(math.pi * X / 0.2)
        u = 0.1 * np.sin(math.pi * Y / 0.2)
        v = 0.05 * np.cos(2 * math.pi * Z)
        w = 0.3 + 0.1 * np.sin(math.pi * X / 0.2)
        p = 1.0 / gam + 0.05 * np.cos(2 * math.pi * (Z - X))
    Q = np.zeros((n, 5, n, nz), order="F")
    Q[:, 0], Q[:, 1], Q[:, 2], Q[:, 3] = rho, rho * u, rho * v, rho * w
    Q[:, 4] = p / (gam - 1.0) + 0.5 * rho * (u * u + v * v + w * w)
    dt = 0.3 * min(dx[0], dz[0]) / 1.6
    cfg = SolverConfig(dim=3, nx=n, ny=n, nz=nz, order=order, scheme=scheme, visc="Euler", tvd=tvd, rk=rk,
                       bc_x=1, bc_y=1, bc_z=1, dt=dt, gamma=gam, R=1.0, dx=dx, dy=dx.copy(), dz=dz, boundary=rules)
    return cfg, to_qj(Q, jacobian(dx, dx.copy(), dz)), z


BOX_RULES = {"x_lo": "slip_wall", "x_hi": "slip_wall", "y_lo": "noslip_wall", "y_hi": "zero_gradient",
             "z_lo": "zero_gradient", "z_hi": "slip_wall"}


@pytest.mark.parametrize("order,scheme,rk", [(6, "SLAU", 3), (4, "KEEP", 4), (6, "Hybrid", 3), (2, "SLAU", 3)])
def test_3d_walls_bitexact_vs_oracle(order, scheme, rk, cuda_device):
    """3D Euler with non-periodic x, y and z: the boundary faces with the reference's
    order fallback in all three sweeps and the x, y, z boundary-cell rules, against the
    oracle: bit-identical residual and state after 5 steps."""
    from ouxsbli_b200.solver import Solver
    cfg, qj, _ = _box3d(14, 26, order, BOX_RULES, scheme, rk)
    s = Solver(cfg, cuda_device)
    s.set_state(qj)
    r = s.rhs()
    s.step(5)
    q = s.get_state()
    s.close()
    np.testing.assert_array_equal(r, oracle.rhs(cfg, qj))
    np.testing.assert_array_equal(q, oracle.step(cfg, qj, 5))


def test_3d_sod_along_z_order6_vs_exact(cuda_device):
    """A Sod tube along z in a box with slip walls in x and y and zero-gradient ends,
    SLAU-6 with the TVD hybrid switch, RK3, 400 cells, t = 0.2: relative L1 of
    density and pressure < 1 % against the exact solution."""
    import sod_exact
    from ouxsbli_b200.grid import jacobian
    from ouxsbli_b200.solver import Solver
    rules = {"x_lo": "slip_wall", "x_hi": "slip_wall", "y_lo": "slip_wall", "y_hi": "slip_wall",
             "z_lo": "zero_gradient", "z_hi": "zero_gradient"}
    cfg, qj, z = _box3d(6, 402, 6, rules, "SLAU", 3, tube=True)
    nsteps = int(round(0.2 / cfg.dt))
    s = Solver(cfg, cuda_device)
    s.set_state(qj)
    s.step(nsteps)
    q = s.get_state()
    s.close()
    J = jacobian(cfg.dx, cfg.dy, cfg.dz)
    rho = q[2, 0, 2] * J[2, 2]
    w = q[2, 3, 2] / q[2, 0, 2]
    pr = 0.4 * (q[2, 4, 2] * J[2, 2] - 0.5 * rho * w * w)
    re, _, pe = sod_exact.solve(z[1:-1], nsteps * cfg.dt, 1.0, 0.0, 1.0, 0.125, 0.0, 0.1, gamma=1.4, x0=0.5)
    l1_rho = np.mean(np.abs(rho[1:-1] - re)) / np.mean(re)
    l1_p = np.mean(np.abs(pr[1:-1] - pe)) / np.mean(pe)
    assert l1_rho < 0.01 and l1_p < 0.01, (l1_rho, l1_p)
