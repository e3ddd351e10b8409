"""Host-side logic that needs no GPU: patcher, Case configuration, writers, grids."""
import math
import re
import struct

import numpy as np
import pytest

from ouxsbli_b200 import patch
from ouxsbli_b200.case import _ALIAS, _RK_NORMALIZE, _VALUE_NORMALIZE, Case
from ouxsbli_b200.grid import cyclic_axis, fill_periodic, jacobian
from ouxsbli_b200.ic import PeriodicBC, RiemannIC, TaylorGreenIC, UniformIC, bc_to_params, ic_to_params
from ouxsbli_b200.output import fortran_e, make_1d_for_print, read_restart, read_vtr, ref_diagnostics, write_restart, write_vtr
from ouxsbli_b200.patcher import _to_fortran_double

GLOBALS = """module mod_globals
  implicit none
  integer, parameter :: nx = 513 ! points incl. ghosts
  integer, parameter :: ny = 513
  real(8), parameter :: Re   = 1600.d0
  real(8), parameter :: CFL  = 0.03d0
  integer, parameter :: np   = 100
  integer, parameter :: nt   = int(20.d0 / (dble(np) * dtn))
end module mod_globals
"""
CONFIG = "#:set VISC = 'NS'\n#:set SCHEME = 'SLAU'\n#:set ORDER = 6\n"


class TestPatcher:
    def test_fortran_double(self):
        assert _to_fortran_double(1600.0) == "1600.0d0"
        assert float(_to_fortran_double(0.03).replace("d0", "e0")) == pytest.approx(0.03)
        assert _to_fortran_double(1e-5) == "1d-05"

    def test_parameters_rewritten(self):
        out = patch(GLOBALS, {"Re": 800.0, "nx": 65, "nt": 500, "CFL": 0.1})
        lines = {ln.split("::")[1].split("=")[0].strip(): ln for ln in out.splitlines() if "::" in ln}
        assert "800.0d0" in lines["Re"]
        assert "= 65" in lines["nx"] and "513" not in lines["nx"]
        assert "! points incl. ghosts" in lines["nx"]
        assert "500" in lines["nt"] and "int(" not in lines["nt"]
        assert "0.1d0" in lines["CFL"]
        assert "= 513" in lines["ny"]
        assert "1600" in GLOBALS  # input untouched

    def test_macros_and_append(self):
        out = patch(CONFIG, {"SCHEME": "KEEP", "ORDER": 4, "RK": 4, "BC_X": False})
        assert "#:set SCHEME = 'KEEP'" in out
        assert "#:set ORDER = 4" in out
        # appended to a fypp file (as the reference's patcher writes them: "NAME =value")
        assert re.search(r"^#:set RK\s*=\s*4$", out, re.M)
        assert re.search(r"^#:set BC_X\s*=\s*False$", out, re.M)
        assert "RK" not in patch(GLOBALS, {"RK": 4})  # never appended to Fortran sources


class TestCaseConfig:
    def test_alias_tables(self):
        assert _ALIAS["scheme"] == "SCHEME" and _ALIAS["accuracy"] == "ORDER" and _ALIAS["recal"] == "RESTART"
        assert _VALUE_NORMALIZE["VISC"]["euler"] == "Euler"
        assert _VALUE_NORMALIZE["TVD"]["minmod"] == "tvd" and _VALUE_NORMALIZE["TVD"]["muscl4"] == "hybrid"
        assert _RK_NORMALIZE["classical_rk4"] == 4

    def test_routing_and_normalisation(self, tmp_path):
        c = Case("3D_solver/NSTGV", tmp_path / "w", scheme="keep", visc="euler", accuracy=4, rk="rk4",
                 nx=20, ny=20, nz=20, Re=800.0, tvd="minmod", visc_stencil="me4", np=1, nt=2)
        c._setup()
        assert c.config["SCHEME"] == "KEEP" and c.config["VISC"] == "Euler" and c.config["ORDER"] == 4
        assert c.config["RK"] == 4 and c.config["TVD"] == "tvd" and c.config["VISC_STENCIL"] == "ME4Base"
        assert c.globals["nx"] == 20 and c.globals["Re"] == 800.0

    def test_build_validates_without_gpu(self, tmp_path):
        c = Case("3D_solver/ETGV", tmp_path / "etgv", nx=14, ny=14, nz=14, np=1, nt=1)
        c.build()
        assert (tmp_path / "etgv" / "data").is_dir() and (tmp_path / "etgv" / "case.json").exists()
        with pytest.raises(RuntimeError):
            Case("3D_solver/ETGV", tmp_path / "x", nx=14, ny=14, nz=14, visc="ns", visc_order=2).build()

    def test_errors(self, tmp_path):
        with pytest.raises(FileNotFoundError):
            Case("3D_solver/NOPE", tmp_path / "n").build()
        with pytest.raises(RuntimeError):
            Case("3D_solver/ETGV", tmp_path / "r").run()
        with pytest.raises(RuntimeError):
            Case("3D_solver/ETGV", tmp_path / "b", bc_x=True).build()
        with pytest.raises(RuntimeError):
            Case("3D_solver/ETGV", tmp_path / "rie", ic=RiemannIC()).build()

    def test_riemann_ic_on_the_shock_tube(self, tmp_path):
        """RiemannIC on a case with a non-periodic x: the left state up to x0 * Lx."""
        c = Case("2D_solver/ST", tmp_path / "st", ic=RiemannIC(rho_l=2.0, p_l=3.0, x0=0.25), visc="euler",
                 nx=41, ny=7, Lx=1.0, Ly=0.1, dt=1e-3, nt=1, np=1)
        c._setup()
        p, xc, yc, zc, dx, dy, dz, Q = c._initial()
        assert p["Lx"] == 1.0
        left = xc < 0.25
        assert np.all(Q[left, 0] == 2.0) and np.all(Q[~left, 0] == 0.125)
        assert np.allclose(Q[left, 3], 3.0 / 0.4) and np.allclose(Q[~left, 3], 0.1 / 0.4)

    def test_ic_bc_specs(self):
        assert ic_to_params(TaylorGreenIC(Ma=0.2))["Ma"] == 0.2
        assert ic_to_params({"type": "uniform", "rho": 2.0})["rho0"] == 2.0
        assert bc_to_params("periodic") == {"BC_X": False, "BC_Y": False, "BC_Z": False}
        assert bc_to_params(PeriodicBC()) == bc_to_params({"type": "periodic"})
        with pytest.raises(ValueError):
            ic_to_params({"type": "nope"})
        with pytest.raises(ValueError):
            bc_to_params("wall")
        assert UniformIC().to_params()["ic_type"] == 1


class TestWriters:
    def test_fortran_e(self):
        assert fortran_e(1.0) == "  0.1000E+01"
        assert fortran_e(-3.3e-7) == " -0.3300E-06"
        assert fortran_e(0.0) == "  0.0000E+00"
        assert fortran_e(9.99995) == "  0.1000E+02"
        assert len(fortran_e(123456.7)) == 12

    def test_vtr_layout_and_roundtrip(self, tmp_path):
        x, y, z = np.arange(3, dtype=np.float32), np.arange(4, dtype=np.float32), np.zeros(2, np.float32)
        n = 3 * 4 * 2
        rho = np.linspace(1, 2, n, dtype=np.float32)
        p = rho * 3
        vel = np.arange(3 * n, dtype=np.float32)
        f = tmp_path / "Q00000.vtr"
        write_vtr(f, x, y, z, rho, p, vel)
        raw = f.read_bytes()
        head = raw[:raw.index(b"  _")].decode()
        assert 'WholeExtent="0    2 0    3 0    1"' in head
        # offsets advance by 4 + 4*N per block (the reference's header word)
        assert f'offset="{"{:>12}".format(4 + 12)}"' in head
        i0 = raw.index(b"  _") + 3
        assert struct.unpack("<i", raw[i0:i0 + 4])[0] == 4 + 4 * 3
        assert raw.endswith(b"  </AppendedData>\n</VTKFile>\n")
        xs, ys, zs, fields = read_vtr(f)
        np.testing.assert_array_equal(xs, x)
        np.testing.assert_array_equal(fields["rho"].ravel(), rho)
        np.testing.assert_array_equal(fields["velocity"].reshape(-1), vel)

    def test_restart_roundtrip(self, tmp_path):
        q = np.asfortranarray(np.random.default_rng(0).standard_normal((5, 5, 6, 7)))
        write_restart(tmp_path / "Q00001.dat", q)
        assert (tmp_path / "Q00001.dat").stat().st_size == q.size * 8
        np.testing.assert_array_equal(read_restart(tmp_path / "Q00001.dat", q.shape), q)

    def test_reference_diagnostics_match_oracle(self):
        """liboux's host KE/entropy helper and the oracle's restatement agree exactly."""
        from oracle import oracle
        rng = np.random.default_rng(2)
        nx = ny = nz = 12
        n = nx * ny * nz
        rho = (1.0 + 0.1 * rng.random(n)).astype(np.float32)
        p = (0.7 + 0.1 * rng.random(n)).astype(np.float32)
        vel = (0.3 * rng.standard_normal(3 * n)).astype(np.float32)
        a = ref_diagnostics(nx, ny, nz, 6, 1.4, rho, p, vel)
        b = oracle.diag_f32(nx, ny, nz, 6, 1.4, rho, p, vel)
        assert a == b


class TestGrid:
    @pytest.mark.parametrize("order", [2, 4, 6])
    def test_cyclic_axis(self, order):
        n = 16 + order
        xc, dx = cyclic_axis(n, 2.0 * math.pi, order)
        g = order // 2
        assert np.allclose(dx, 2.0 * math.pi / 16)
        assert xc[g] == pytest.approx(0.5 * dx[0])  # first interior cell centre at dx/2
        assert np.allclose(np.diff(xc), dx[0])

    def test_fill_periodic_and_jacobian(self):
        g = 3
        q = np.asfortranarray(np.random.default_rng(1).standard_normal((10, 5, 11, 12)))
        fill_periodic(q, g)
        # ghost cell c takes the interior image g + (c - g) mod N
        assert np.array_equal(q[0], q[g + (0 - g) % (10 - 2 * g)])
        assert np.array_equal(q[:, :, :, 11], q[:, :, :, g + (11 - g) % (12 - 2 * g)])
        assert np.array_equal(q[:, :, 1, :], q[:, :, g + (1 - g) % (11 - 2 * g), :])
        J = jacobian(np.full(9, 0.5), np.full(10, 0.25), np.full(11, 0.1))
        assert J.shape == (10, 11) and np.allclose(J, 1.0 / (0.5 * 0.25 * 0.1))


class TestSodExact:
    def test_star_state_matches_published_values(self):
        """Sod's problem (rho 1 / 0.125, p 1 / 0.1, gamma 1.4): p* = 0.30313, u* = 0.92745
        (Toro, Riemann Solvers and Numerical Methods for Fluid Dynamics, Table 4.3)."""
        from sod_exact import star_state
        ps, us = star_state(1.0, 0.0, 1.0, 0.125, 0.0, 0.1)
        assert abs(ps - 0.30313) < 5e-5 and abs(us - 0.92745) < 5e-5

    def test_profile_structure(self):
        from sod_exact import solve
        x = np.linspace(0.0, 1.0, 2001)
        rho, u, p = solve(x, 0.2, 1.0, 0.0, 1.0, 0.125, 0.0, 0.1, x0=0.5)
        assert rho[0] == 1.0 and rho[-1] == 0.125 and p[0] == 1.0 and p[-1] == 0.1
        assert np.all(np.diff(p) <= 1e-12)          # pressure falls monotonically
        assert abs(u.max() - 0.92745) < 5e-5       # the star velocity
        # mass conservation: integral of rho over [0, 1] equals the initial one
        assert abs(np.trapezoid(rho, x) - 0.5625) < 2e-3


class TestObliqueShock:
    def test_weak_angles_of_the_reflection_case(self):
        """M = 2, theta = 8 deg: weak incident angle 37.2 deg; the reflected shock at the
        downstream Mach number turns the flow back at 44.1 deg (the angles the
        reference's reflected-shock case and its test use)."""
        import math
        from oblique_shock import deflection, free_stream, shock, weak_beta
        b = weak_beta(2.0, math.radians(8.0))
        assert abs(math.degrees(b) - 37.21) < 0.01
        assert abs(math.degrees(deflection(2.0, b)) - 8.0) < 1e-9
        rho1, U1, p1 = free_stream(2.0, 100e3, 295.0, 1.4, 287.03)
        rho2, U2, p2, th = shock(rho1, U1, p1, math.radians(37.2), 1.4)
        M2 = U2 / math.sqrt(1.4 * p2 / rho2)
        assert abs(math.degrees(weak_beta(M2, th)) - 44.1) < 0.1

    def test_normal_shock_table_values(self):
        """Normal shock at Mn = 2 (NACA 1135 table): p2/p1 = 4.5, rho2/rho1 = 2.6667, Mn2 = 0.5774."""
        from oblique_shock import normal_jump
        pr, rr, mn2 = normal_jump(2.0)
        assert abs(pr - 4.5) < 1e-12 and abs(rr - 8.0 / 3.0) < 1e-12 and abs(mn2 - 0.57735) < 1e-5


class TestBoundaryRules:
    """The oracle's boundary-cell fill for non-periodic x and y (the OS rule set)."""

    def test_rules_and_corners(self):
        from oracle import oracle
        from ouxsbli_b200.solver import SolverConfig
        nx, ny = 9, 7
        rng = np.random.default_rng(3)
        q = np.asfortranarray(rng.uniform(1.0, 2.0, (nx, 4, ny)))
        top = rng.uniform(3.0, 4.0, (4, nx))
        inflow = rng.uniform(5.0, 6.0, (4, ny))
        cfg = SolverConfig(dim=2, nx=nx, ny=ny, nz=1, order=6, visc="Euler", bc_x=1, bc_y=1,
                           dx=np.ones(nx - 1), dy=np.ones(ny - 1), dz=None,
                           boundary={"x_lo": ("fixed", inflow), "x_hi": "zero_gradient",
                                     "y_lo": "slip_wall", "y_hi": ("fixed", top)})
        out = oracle.fill_ghosts(cfg, q)
        np.testing.assert_array_equal(out[1:-1, :, 1:-1], q[1:-1, :, 1:-1])   # interior untouched
        for i in range(1, nx - 1):
            np.testing.assert_array_equal(out[i, :, -1], top[:, i])
            np.testing.assert_array_equal(out[i, :, 0], q[i, :, 1] * np.array([1, 1, -1, 1]))
        for j in range(ny):
            np.testing.assert_array_equal(out[0, :, j], inflow[:, j])
        for j in range(1, ny - 1):
            np.testing.assert_array_equal(out[-1, :, j], q[-2, :, j])
        # corners at x high: the zero-gradient copy of the y-boundary cell beside them
        np.testing.assert_array_equal(out[-1, :, 0], q[-2, :, 1] * np.array([1, 1, -1, 1]))
        np.testing.assert_array_equal(out[-1, :, -1], top[:, -2])


class TestKnownAnswerHelpersAgainstReferenceUtils:
    """This project's exact-solution helpers (tests/sod_exact.py, tests/oblique_shock.py)
    against values produced by the reference's own test utilities
    (tests/golden/kat_analytic.json, made by tests/golden/make_kat_fixtures.py)."""

    @staticmethod
    def _fixtures():
        import json
        import pathlib
        return json.loads((pathlib.Path(__file__).parent / "golden" / "kat_analytic.json").read_text())

    def test_sod_profiles(self):
        from sod_exact import solve
        for c in self._fixtures()["sod"]:
            x = np.array(c["x"])
            rho, u, p = solve(x, c["t"], *c["states"], gamma=1.4, x0=0.5)
            np.testing.assert_allclose(rho, c["rho"], rtol=1e-9, atol=1e-12)
            np.testing.assert_allclose(u, c["u"], rtol=1e-9, atol=1e-12)
            np.testing.assert_allclose(p, c["p"], rtol=1e-9, atol=1e-12)

    def test_oblique_shock_states(self):
        import math
        from oblique_shock import free_stream, shock
        o = self._fixtures()["oblique"]
        g, R = o["gamma"], o["R"]
        rho1, u1, p1 = free_stream(o["M0"], o["p_tot"], o["T_tot"], g, R)
        u0_ref, p0_ref, T0_ref = o["free_stream"]
        assert math.isclose(u1, u0_ref, rel_tol=1e-13) and math.isclose(p1, p0_ref, rel_tol=1e-13)
        assert math.isclose(rho1, p0_ref / (R * T0_ref), rel_tol=1e-13)
        rho2, U2, p2, theta = shock(rho1, u1, p1, o["beta"], g)
        assert math.isclose(rho2, o["post_shock"][0], rel_tol=1e-12)
        assert math.isclose(p2, o["post_shock"][1], rel_tol=1e-12)
        assert abs(U2 / math.sqrt(g * p2 / rho2) - o["downstream_mach"]) < 2e-3  # theirs at theta = 8.0 deg
        # the reflected shock at the reference test's angle: density and pressure agree;
        # the reference utility resolves the velocity along the wall-referenced angle, so
        # its u3 differs from the wall-parallel state by about 2 % (inside the test's 3 %)
        rho3, U3, p3, _ = shock(rho2, U2, p2, o["beta_r"], g)
        assert math.isclose(rho3, o["reflected"][0], rel_tol=1e-12)
        assert math.isclose(p3, o["reflected"][3], rel_tol=1e-12)
        assert abs(U3 - o["reflected"][1]) / o["reflected"][1] < 0.03


def test_every_case_builds_its_initial_field(tmp_path):
    """Each case's defaults (scaled down) give a finite initial field of the right shape."""
    from ouxsbli_b200.cases import CASES
    small = {3: dict(nx=14, ny=14, nz=14), 2: dict(nx=22, ny=22)}
    # BL reads its inflow profile (rows of y, rho, u, v, p) from a file
    prof = np.array([[0.0, 0.2, 0.0, 0.0, 1.3e4], [1.0e-3, 0.25, 300.0, 0.5, 1.3e4], [3.0e-3, 0.28, 540.0, 1.4, 1.3e4]])
    prof.astype("<f8").tofile(tmp_path / "Qin.dat")
    extra = {"BL": dict(inflow=str(tmp_path / "Qin.dat"))}
    for name, case in CASES.items():
        src = f"{case.dim}D_solver/{name}"
        c = Case(src, tmp_path / name, nt=1, np=1, **small[case.dim], **extra.get(name, {}))
        c._setup()
        p, xc, yc, zc, dx, dy, dz, Q = c._initial()
        nv = case.dim + 2
        assert Q.shape[1] == nv and np.isfinite(Q).all() and (Q[:, 0] > 0).all(), name


def test_oracle_farfield_and_split_rules():
    """The oracle's far-field rule (Riemann invariants, the top row of
    2D_solver/BL0/set.f90) and a split face against numpy restatements."""
    from oracle import oracle
    from ouxsbli_b200.grid import jacobian
    from ouxsbli_b200.solver import SolverConfig
    nx, ny, g1 = 10, 8, 0.4
    rng = np.random.default_rng(11)
    dx, dy = rng.uniform(0.8, 1.2, nx - 1), rng.uniform(0.8, 1.2, ny - 1)
    J = jacobian(dx, dy, None)
    rho = rng.uniform(1.0, 1.2, (nx, ny))
    u, v = rng.uniform(1.5, 2.0, (nx, ny)), rng.uniform(-0.1, 0.1, (nx, ny))
    p = rng.uniform(0.7, 0.8, (nx, ny))
    q = np.zeros((nx, 4, ny), order="F")
    q[:, 0], q[:, 1], q[:, 2] = rho / J, rho * u / J, rho * v / J
    q[:, 3] = (p / g1 + 0.5 * rho * (u * u + v * v)) / J
    far = (1.1, 1.9, 0.0, 0.9)
    cfg = SolverConfig(dim=2, nx=nx, ny=ny, nz=1, order=2, visc="Euler", bc_x=1, bc_y=1, dx=dx, dy=dy, dz=None,
                       gamma=1.4, boundary={"y_hi": ("farfield",) + far,
                                            "y_lo": ("split", 4, "zero_gradient", "noslip_wall")},
                       boundary_order="y_last")
    out = oracle.fill_ghosts(cfg, q)
    for i in range(1, nx - 1):
        Jn, Jb = J[i, ny - 2], J[i, ny - 1]
        qn = q[i, :, ny - 2]
        pin = g1 * (qn[3] - 0.5 * (qn[1] ** 2 + qn[2] ** 2) / qn[0]) * Jn
        cin = np.sqrt(1.4 * pin / (qn[0] * Jn))
        Rp, Rm = qn[2] / qn[0] + 2 * cin / g1, far[2] - 2 * far[3] / g1
        vb, cb = 0.5 * (Rp + Rm), 0.25 * g1 * (Rp - Rm)
        rb = (cb / far[3]) ** (2 / g1) * far[0]
        pb = rb * cb * cb / 1.4
        want = np.array([rb, rb * far[1], rb * vb, pb / g1 + 0.5 * rb * (far[1] ** 2 + vb ** 2)]) / Jb
        np.testing.assert_allclose(out[i, :, ny - 1], want, rtol=1e-13)
        qw = q[i, :, 1]
        if i < 4:
            np.testing.assert_array_equal(out[i, :, 0], qw)
        else:
            pw = g1 * (qw[3] - 0.5 * (qw[1] ** 2 + qw[2] ** 2) / qw[0])
            np.testing.assert_allclose(out[i, :, 0], [qw[0], 0.0, 0.0, pw / g1], rtol=1e-15)


def test_blasius_solution_and_compressible_layer():
    """The Blasius solution (f''(0) = 0.332057, f'(4.91) = 0.99) and the compressible
    layer built on it: no-slip at the wall, the free stream at the edge, adiabatic
    wall temperature."""
    from ouxsbli_b200.blasius import blasius, compressible_profile
    eta, f, fp, fpp0 = blasius()
    assert abs(fpp0 - 0.332057) < 2e-6
    assert abs(np.interp(4.91, eta, fp) - 0.99) < 1e-4
    y = np.linspace(0.0, 3e-3, 61)
    T0, u0, p0, R, g, rf = 163.9, 513.25, 12780.0, 287.03, 1.4, 0.89
    Cp = g * R / (g - 1.0)
    Taw = T0 * (1.0 + rf * 0.2 * 4.0)
    rho, u, v, T = compressible_profile(y, 0.8e-3, u0, T0, p0, R, Cp, rf, Taw, 1.1e-5)
    assert u[0] == 0.0 and v[0] == 0.0 and abs(T[0] - Taw) < 1e-9
    assert abs(u[-1] - u0) < 1e-6 * u0 and abs(T[-1] - (Taw - rf * u0 ** 2 / (2 * Cp))) < 1e-6
    i99 = np.searchsorted(u, 0.99 * u0)
    assert abs(y[i99] - 0.8e-3) < 2 * (y[1] - y[0])


def test_3d_tbl_top_rules_of_the_oracle():
    """The oracle's TBL / SBLI top rules (3D_solver/src/set_bc_tbl_sbli.f90) on a 3D
    plate box: the Neumann top carries the neighbour's primitive state (rho, u, v, w,
    p) into the top cells; the far-field top keeps the neighbour's outgoing invariant
    v + 2c/(gamma-1), the far field's incoming one v - 2c/(gamma-1) and entropy
    p / rho^gamma, with u = u_inf and w = 0."""
    from helpers import GAMMA, R, RHO0, T0, wall_box
    from oracle import oracle
    from ouxsbli_b200.grid import jacobian
    c0, U = math.sqrt(GAMMA * R * T0), 5.0
    g1 = GAMMA - 1.0
    for top in ("neumann", ("farfield", RHO0, U, 0.0, c0)):
        rules = {"x_lo": "zero_gradient", "x_hi": "zero_gradient", "y_lo": "noslip_wall", "y_hi": top}
        cfg, qj, _ = wall_box(10, 12, 6, 6, rules, bc_x=1, plate=True, U=U)
        q = oracle.fill_ghosts(cfg, qj)
        J = jacobian(cfg.dx, cfg.dy, cfg.dz)
        g = cfg.g
        prim = []
        for j in (cfg.ny - 1, cfg.ny - 2):  # the top cells and their neighbours
            a = q[1:-1, :, j, g:-g]
            Jj = J[1:-1, j][:, None]
            rho = a[:, 0] * Jj
            u, v, w = a[:, 1] / a[:, 0], a[:, 2] / a[:, 0], a[:, 3] / a[:, 0]
            p = g1 * (a[:, 4] * Jj - 0.5 * rho * (u * u + v * v + w * w))
            prim.append((rho, u, v, w, p))
        (rb, ub, vb, wb, pb), (rn, un, vn, wn, pn) = prim
        if top == "neumann":
            for b, n in zip((rb, ub, vb, wb, pb), (rn, un, vn, wn, pn)):
                np.testing.assert_allclose(b, n, rtol=1e-13, atol=1e-13 * np.abs(n).max())
        else:
            cb, cn = np.sqrt(GAMMA * pb / rb), np.sqrt(GAMMA * pn / rn)
            np.testing.assert_allclose(vb + 2 * cb / g1, vn + 2 * cn / g1, rtol=1e-12)
            np.testing.assert_allclose(vb - 2 * cb / g1, -2 * c0 / g1, rtol=1e-12)
            np.testing.assert_allclose(pb / rb ** GAMMA, (RHO0 * c0 ** 2 / GAMMA) / RHO0 ** GAMMA, rtol=1e-12)
            np.testing.assert_allclose(ub, U, rtol=1e-13)
            assert np.all(wb == 0.0)


@pytest.mark.parametrize("order,visc,vo,stencil", [(6, "NS", 6, "Central"), (6, "LES", 6, "ME4Base"),
                                                   (4, "NS", 4, "Central"), (4, "NS", 2, "Central"),
                                                   (2, "LES", 2, "Central"), (6, "Euler", 0, "Central")])
def test_3d_walled_box_at_rest_stays_at_rest(order, visc, vo, stencil):
    """The oracle's walled 3D paths (convective order fallback, viscous 2nd-order
    fallback, SGS boundary values, slip and no-slip walls on every face) keep a uniform
    fluid at rest: the residual is at rounding level, below 1e-12 of the residual of
    the same box with its shear flow."""
    from helpers import wall_box
    from oracle import oracle
    rules = {"x_lo": "slip_wall", "x_hi": "noslip_wall", "y_lo": "noslip_wall", "y_hi": "slip_wall",
             "z_lo": "noslip_wall", "z_hi": "slip_wall"}
    kw = dict(bc_x=1, bc_z=1, visc=visc, scheme="SLAU", rk=3, tvd="hybrid")
    if visc != "Euler":
        kw.update(visc_order=vo, visc_stencil=stencil)
    cfg, moving, _ = wall_box(10, 12, 8, order, rules, **kw)
    _, rest, _ = wall_box(10, 12, 8, order, rules, U=0.0, perturb=False, **kw)
    r_rest = oracle.rhs(cfg, rest)
    r_moving = oracle.rhs(cfg, moving)
    assert np.abs(r_rest).max() <= 1e-12 * np.abs(r_moving).max(), np.abs(r_rest).max()


def test_2d_neumann_rule_of_the_oracle():
    """The oracle's Neumann rule in 2D carries the neighbour's primitive state (rho,
    u, v, p) into the boundary cells of both non-periodic faces it is set on."""
    from oracle import oracle
    from ouxsbli_b200.grid import jacobian, to_qj
    from ouxsbli_b200.solver import SolverConfig
    nx, ny, g1 = 20, 14, 0.4
    dx = np.full(nx - 1, 0.05)
    dy = 0.03 * (1.0 + 0.05 * np.arange(ny - 1))  # stretched
    x, y = np.concatenate([[0.0], np.cumsum(dx)]), np.concatenate([[0.0], np.cumsum(dy)])
    X, Y = np.meshgrid(x, y, indexing="ij")
    rho, u, v, p = 1.0 + 0.1 * np.sin(3 * X) * Y, 1.5 + 0.2 * Y, 0.1 * np.cos(4 * X), 1.0 + 0.1 * X * Y
    Q = np.zeros((nx, 4, ny), order="F")
    Q[:, 0], Q[:, 1], Q[:, 2], Q[:, 3] = rho, rho * u, rho * v, p / g1 + 0.5 * rho * (u * u + v * v)
    J = jacobian(dx, dy, None)
    rules = {"x_lo": "slip_wall", "x_hi": "neumann", "y_lo": "noslip_wall", "y_hi": "neumann"}
    cfg = SolverConfig(dim=2, nx=nx, ny=ny, nz=1, order=2, visc="Euler", bc_x=1, bc_y=1, dt=1e-3, gamma=1.4,
                       R=1.0, dx=dx, dy=dy, dz=None, boundary=rules)
    q = oracle.fill_ghosts(cfg, to_qj(Q, J))

    def prim(qq, Jv):
        r = qq[0] * Jv
        uu, vv = qq[1] / qq[0], qq[2] / qq[0]
        return np.array([r, uu, vv, g1 * (qq[3] * Jv - 0.5 * r * (uu * uu + vv * vv))])

    for i in range(1, nx - 1):  # top row (corners take the x rules in this order)
        np.testing.assert_allclose(prim(q[i, :, ny - 1], J[i, ny - 1]), prim(q[i, :, ny - 2], J[i, ny - 2]),
                                   rtol=1e-13, atol=1e-15)
    for j in range(1, ny - 1):  # x high column
        np.testing.assert_allclose(prim(q[nx - 1, :, j], J[nx - 1, j]), prim(q[nx - 2, :, j], J[nx - 2, j]),
                                   rtol=1e-13, atol=1e-15)


def test_bl_inflow_profile_as_set_init_reads_it(tmp_path):
    """2D_solver/BL/set.f90 set_init: the profile file's rows (y, rho, u, v, p) are
    interpolated linearly onto the grid's y nodes, held at the end rows outside their
    range, and one pressure, the mean of the interpolated p over the first nyi grid
    rows, fills every column (known answers for a 3-row profile on 4 nodes)."""
    from ouxsbli_b200.cases import _blq_init, read_inflow_profile
    prof = np.array([[0.0, 1.0, 0.0, 0.0, 100.0],
                     [1.0e-3, 2.0, 10.0, 1.0, 200.0],
                     [2.0e-3, 3.0, 20.0, 2.0, 300.0]])
    f = tmp_path / "Qin.dat"
    prof.astype("<f8").tofile(f)
    np.testing.assert_array_equal(read_inflow_profile(f), prof)
    y = np.array([0.0, 0.5e-3, 1.0e-3, 2.5e-3])
    x = np.zeros(3)
    p = {"inflow": str(f), "gamma": 1.4}
    Q = _blq_init(p, x, y)
    rho = np.array([1.0, 1.5, 2.0, 3.0])
    u = np.array([0.0, 5.0, 10.0, 20.0])
    v = np.array([0.0, 0.5, 1.0, 2.0])
    ptbl = (100.0 + 150.0 + 200.0) / 3.0  # the first nyi = 3 grid rows
    for i in range(3):
        np.testing.assert_allclose(Q[i, 0], rho, rtol=1e-15)
        np.testing.assert_allclose(Q[i, 1], rho * u, rtol=1e-15)
        np.testing.assert_allclose(Q[i, 2], rho * v, rtol=1e-15)
        np.testing.assert_allclose(Q[i, 3], ptbl / 0.4 + 0.5 * rho * (u * u + v * v), rtol=1e-15)
    np.testing.assert_array_equal(p["inflow_q"], Q[0])  # the inflow column the boundary keeps
    (tmp_path / "bad.dat").write_bytes(np.zeros(7).tobytes())
    with pytest.raises(ValueError, match="rows of 5"):
        read_inflow_profile(tmp_path / "bad.dat")
    with pytest.raises(ValueError, match="more than the grid"):
        _blq_init(dict(p), x, y[:2])
