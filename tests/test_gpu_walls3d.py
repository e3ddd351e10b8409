"""3D Navier-Stokes with non-periodic directions: the walled sweep variants (convective
order fallback next to a boundary, the 2nd-order viscous fallback of
3D_solver/src/calc_visc_high.f90.fypp outside its high-order guard) against the
oracle, the mixed form against FP64, and a shear-decay known answer."""
import math

import numpy as np
import pytest

from helpers import GAMMA, H, R, RHO0, T0, rel_l2, wall_box
from oracle import oracle
from ouxsbli_b200.solver import Solver

CHANNEL = {"y_lo": "noslip_wall", "y_hi": "noslip_wall"}
# a flat-plate-like box: zero-gradient in / outflow, no-slip floor, zero-gradient top
PLATE = {"x_lo": "zero_gradient", "x_hi": "zero_gradient", "y_lo": "noslip_wall", "y_hi": "zero_gradient"}
# walls on every side
CLOSED = {"x_lo": "slip_wall", "x_hi": "slip_wall", "y_lo": "noslip_wall", "y_hi": "noslip_wall",
          "z_lo": "slip_wall", "z_hi": "noslip_wall"}
# periodic x, walls in y and z
DUCT = {f: r for f, r in CLOSED.items() if not f.startswith("x")}

def assert_matches_oracle(cfg, r, q, r_want, q_want):
    """Navier-Stokes: bit-identical.  LES: its SGS model calls pow / log / cosh
    (3D_solver/src/calc_les.f90:30-71), which CUDA's libm and the host's may round 1 ulp
    apart, so max |dR| <= 1e-11 max |R| and relative L2 <= 1e-12 per conservative
    variable."""
    if cfg.visc != "LES":
        np.testing.assert_array_equal(r, r_want)
        np.testing.assert_array_equal(q, q_want)
        return
    assert np.abs(r - r_want).max() <= 1e-11 * np.abs(r_want).max()
    for l in range(q.shape[1]):
        assert rel_l2(q[:, l], q_want[:, l]) <= 1e-12, l


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


LES_CASES = [
    # (order, visc_order, stencil, scheme, rk, bc_x, bc_z, rules)
    (6, 6, "Central", "Hybrid", 3, 1, 0, PLATE),    # TBL's Hybrid-6 LES over a no-slip floor
    (6, 6, "ME4Base", "SLAU", 3, 0, 0, CHANNEL),
    (4, 4, "Central", "KEEP", 4, 1, 1, CLOSED),
    (4, 2, "Central", "SLAU", 3, 0, 1, DUCT),
    (2, 2, "Central", "KEEP", 3, 1, 1, CLOSED),
]


@pytest.mark.gpu
@pytest.mark.parametrize("order,vo,stencil,scheme,rk,bc_x,bc_z,rules", LES_CASES)
def test_3d_les_walls_vs_oracle(order, vo, stencil, scheme, rk, bc_x, bc_z, rules, cuda_device):
    """3D LES with non-periodic directions: the SGS viscosity's boundary values (0 on a
    no-slip wall, the neighbour's elsewhere) and the SGS terms of the viscous faces'
    2nd-order fallback; residual and state after 4 steps against the oracle within the
    LES tolerances (assert_matches_oracle)."""
    cfg, qj, _ = wall_box(14, 16, 10, order, rules, bc_x=bc_x, bc_z=bc_z, visc="LES", visc_order=vo,
                          visc_stencil=stencil, scheme=scheme, rk=rk, tvd="hybrid")
    s = Solver(cfg, cuda_device)
    s.set_state(qj)
    r = s.rhs()
    s.step(4)
    q = s.get_state()
    s.close()
    per = lambda nonper: slice(cfg.g - 1, -(cfg.g - 1)) if not nonper and cfg.g > 1 else slice(None)
    upd = (per(bc_x), slice(None), slice(None), per(bc_z))
    assert_matches_oracle(cfg, r[upd], q, oracle.rhs(cfg, qj)[upd], oracle.step(cfg, qj, 4))


@pytest.mark.gpu
@pytest.mark.parametrize("visc", ["NS", "LES"])
def test_3d_viscous_walls_mixed_close_to_fp64(visc, cuda_device):
    """The mixed form on a walled 3D Navier-Stokes / LES box (KEEP-6, Central-6, RK4):
    relative L2 against FP64 within the mixed form's bound for switch-free schemes
    (1e-5)."""
    out = {}
    for prec in ("fp64", "mixed"):
        cfg, qj, _ = wall_box(14, 16, 10, 6, CLOSED, bc_x=1, bc_z=1, scheme="KEEP", rk=4, precision=prec,
                              visc=visc)
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


@pytest.mark.gpu
@pytest.mark.parametrize("top", ["neumann", "farfield"])
def test_3d_tbl_top_rules_vs_oracle(top, cuda_device):
    """The TBL / SBLI top boundary (3D_solver/src/set_bc_tbl_sbli.f90) over a no-slip
    floor with zero-gradient x ends (NS SLAU-6 / Central-6, RK3, u = U at the top):
    with the Neumann top, residual and state after 4 steps bit-identical to the oracle;
    with the far-field top, whose rule calls pow (libm on the host, CUDA on the
    device), equal to rounding (1e-12 of each variable's largest value)."""
    c0 = math.sqrt(GAMMA * R * T0)
    rule = "neumann" if top == "neumann" else ("farfield", RHO0, 5.0, 0.0, c0)
    rules = {**PLATE, "y_hi": rule}
    cfg, qj, _ = wall_box(14, 16, 10, 6, rules, bc_x=1, bc_z=0, plate=True, scheme="SLAU", rk=3, tvd="hybrid")
    s = Solver(cfg, cuda_device)
    s.set_state(qj)
    r = s.rhs()
    s.step(4)
    q = s.get_state()
    s.close()
    zs = slice(cfg.g - 1, -(cfg.g - 1))  # updated cells of the periodic z
    r_want, q_want = oracle.rhs(cfg, qj), oracle.step(cfg, qj, 4)
    if top == "neumann":
        np.testing.assert_array_equal(r[..., zs], r_want[..., zs])
        np.testing.assert_array_equal(q, q_want)
    else:
        for l in range(5):
            np.testing.assert_allclose(r[:, l, :, zs], r_want[:, l, :, zs], rtol=0,
                                       atol=1e-12 * np.abs(r_want[:, l, :, zs]).max())
            np.testing.assert_allclose(q[:, l], q_want[:, l], rtol=0, atol=1e-12 * np.abs(q_want[:, l]).max())


@pytest.mark.gpu
@pytest.mark.parametrize("visc", ["NS", "LES"])
@pytest.mark.parametrize("sizes,bc_x,bc_z,rules", [
    ((2, 4, 2), 1, 1, CLOSED),   # the smallest walled grid: two interior cells per axis
    ((37, 19, 11), 1, 0, PLATE),  # ragged: no extent a multiple of the tile shapes
    ((33, 7, 3), 0, 1, DUCT),
])
def test_3d_viscous_walls_smallest_and_ragged_grids(visc, sizes, bc_x, bc_z, rules, cuda_device):
    """Walled 3D NS / LES (Central-6, SLAU-6, RK3) on the smallest grids the library
    accepts and on ragged extents: residual and state after 3 steps against the oracle
    (NS bit-identical, LES within its tolerances; every face of the smallest grid is on
    a fallback stencil)."""
    nx_int, ny, nz_int = sizes
    cfg, qj, _ = wall_box(nx_int, ny, nz_int, 6, rules, bc_x=bc_x, bc_z=bc_z, visc=visc, scheme="SLAU", rk=3,
                          tvd="hybrid")
    s = Solver(cfg, cuda_device)
    s.set_state(qj)
    r = s.rhs()
    s.step(3)
    q = s.get_state()
    s.close()
    per = lambda nonper: slice(cfg.g - 1, -(cfg.g - 1)) if not nonper and cfg.g > 1 else slice(None)
    upd = (per(bc_x), slice(None), slice(None), per(bc_z))
    assert_matches_oracle(cfg, r[upd], q, oracle.rhs(cfg, qj)[upd], oracle.step(cfg, qj, 3))


@pytest.mark.gpu
def test_3d_flat_plate_skin_friction(cuda_device):
    """The 2D_solver/BL0 flow in 3D: Mach 2 over an adiabatic no-slip plate along the
    whole floor (1025 x 129 nodes of BL0's grid, 4 periodic z cells; fixed free-stream
    inflow, zero-gradient outflow, characteristic far-field top; NS SLAU-2 / Gaitonde-
    Visbal, RK3, dt 3 ns, 0.4 ms).  The z-uniform flow stays identical in every z plane,
    and the skin friction from the discrete wall shear follows the similarity law: Cf
    sqrt(Re_x) constant downstream (spread < 3 %) and within 8 % of the Eckert
    reference-temperature value, as for BL0 in 2D."""
    from ouxsbli_b200.cases import CASES, _bl_derived, _bl_grid
    from ouxsbli_b200.grid import jacobian, to_qj
    from ouxsbli_b200.solver import SolverConfig
    p = _bl_derived(CASES["BL0"].params)
    x, dx, y, dy = _bl_grid(p)
    nx, ny, nz = x.size, y.size, 6
    dz = np.full(nz - 1, dx[0])
    g, Rg, M0 = p["gamma"], p["R"], p["M0"]
    rho0, u0, p0 = p["rho_bc"], p["u0"], p["p0"]
    free = np.array([rho0, rho0 * u0, 0.0, 0.0, p0 / (g - 1.0) + 0.5 * rho0 * u0 ** 2])
    Q = np.zeros((nx, 5, ny, nz), order="F")
    Q[:] = free[None, :, None, None]
    J = jacobian(dx, dy, dz)
    inflow = (free[:, None, None] * (1.0 / J[0, :])[None, :, None] * np.ones(nz)[None, None, :])
    rules = {"x_lo": ("fixed", inflow.reshape(5, ny * nz, order="F")), "x_hi": "zero_gradient",
             "y_lo": "noslip_wall", "y_hi": ("farfield", rho0, u0, 0.0, p["c_bc"])}
    cfg = SolverConfig(dim=3, nx=nx, ny=ny, nz=nz, order=2, scheme="SLAU", slau="HRSLAU2", tvd="none", visc="NS",
                       rk=3, bc_x=1, bc_y=1, bc_z=0, dt=p["dt"], gamma=g, R=Rg, Pr=p["Pr"],
                       threshold=p["threshold"], dx=dx, dy=dy, dz=dz, boundary=rules)
    s = Solver(cfg, cuda_device)
    s.set_state(to_qj(Q, J))
    s.step(int(round(p["endT"] / p["dt"])))
    q = s.get_state()
    s.close()
    for k in range(2, nz - 1):
        np.testing.assert_array_equal(q[..., k], q[..., 1])
    q = q[..., 1]
    rho = q[:, 0] * J
    u = q[:, 1] / q[:, 0]
    v = q[:, 2] / q[:, 0]
    pr = (g - 1.0) * (q[:, 4] * J - 0.5 * rho * (u * u + v * v))
    T = pr / (rho * Rg)

    def mu(t):
        return 1.716e-5 * 384.2 * 273.2 ** -1.5 / (t + 111.0) * t ** 1.5

    Te, rho_e, u_e = p["T0"], p["rho0"], p["u0"]
    vals = []
    for frac in np.linspace(0.45, 0.95, 6):
        i = int(frac * (nx - 1))
        tau = 0.5 * (mu(T[i, 0]) + mu(T[i, 1])) * (u[i, 1] - u[i, 0]) / (y[1] - y[0])
        rex = rho_e * u_e * (x[i] - x[0]) / mu(Te)
        vals.append(tau / (0.5 * rho_e * u_e ** 2) * math.sqrt(rex))
    vals = np.array(vals)
    Tw = Te * (1.0 + math.sqrt(p["Pr"]) * 0.5 * (g - 1.0) * M0 ** 2)
    Ts = Te * (1.0 + 0.032 * M0 ** 2 + 0.58 * (Tw / Te - 1.0))
    eckert = 0.664 * math.sqrt(mu(Ts) / mu(Te) * Te / Ts)
    print("Cf sqrt(Re_x):", vals, "Eckert:", eckert)
    assert vals.max() / vals.min() - 1.0 < 0.03, vals
    assert abs(vals.mean() / eckert - 1.0) < 0.08, (vals, eckert)


@pytest.mark.gpu
@pytest.mark.parametrize("order,bc_z,rules,world", [
    (6, 0, CHANNEL, 2),  # y walls, x periodic, z periodic split in 2 slabs (halo ends only)
    (4, 0, PLATE, 3),    # x / y walls, 3 slabs
    (2, 1, DUCT, 2),     # y / z walls: the first and last slab each own one z wall
])
def test_3d_viscous_walls_in_z_slabs_match_one_solve(order, bc_z, rules, world, cuda_device):
    """A walled 3D Navier-Stokes grid split into z slabs that exchange halos after
    every stage (the reference's COMMZ) against the undivided solve: interior planes
    bit-identical after 4 steps."""
    from ouxsbli_b200.slabs import LocalSlabs
    bc_x = 1 if "x_lo" in rules else 0
    cfg, qj, _ = wall_box(14, 16, 12, order, rules, bc_x=bc_x, bc_z=bc_z, scheme="SLAU", rk=3, tvd="hybrid")
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
    gz = 1 if bc_z else cfg.g
    np.testing.assert_array_equal(got[..., gz:-gz], whole[..., gz:-gz])


@pytest.mark.gpu
def test_3d_tbl_configuration_les_vs_oracle(cuda_device):
    """The numerics of 3D_solver/TBL (config.fypp: LES, Hybrid-6, RK3; set_bc: periodic
    x by its ghost copies, a no-slip floor, the Riemann far-field top of
    set_bc_tbl_sbli.f90, periodic z) on a plate-profile box: residual and state after 4
    steps against the oracle within the LES tolerances."""
    c0 = math.sqrt(GAMMA * R * T0)
    rules = {"y_lo": "noslip_wall", "y_hi": ("farfield", RHO0, 5.0, 0.0, c0)}
    cfg, qj, _ = wall_box(14, 16, 10, 6, rules, bc_x=0, bc_z=0, plate=True, visc="LES", scheme="Hybrid", rk=3,
                          tvd="hybrid")
    s = Solver(cfg, cuda_device)
    s.set_state(qj)
    r = s.rhs()
    s.step(4)
    q = s.get_state()
    s.close()
    g = cfg.g
    upd = (slice(g - 1, -(g - 1)), slice(None), slice(None), slice(g - 1, -(g - 1)))
    assert_matches_oracle(cfg, r[upd], q, oracle.rhs(cfg, qj)[upd], oracle.step(cfg, qj, 4))
