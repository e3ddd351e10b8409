"""Case -- lifecycle of one simulation run, the drop-in for ``ouxsbli.Case``.

Usage (same keyword names as the reference, ouxsbli/case.py:68-256)::

    from ouxsbli_b200 import Case

    case = Case(source="3D_solver/NSTGV", workdir="/tmp/run_01",
                Re=800.0, nx=70, ny=70, nz=70, scheme="SLAU", visc="NS", accuracy=6,
                np=5, nt=20)
    case.build()
    case.run(nranks=2)

Differences from the reference, all on purpose:
  * build() compiles nothing: it validates the configuration against liboux (the
    sm_100a library is built once, in-tree) and prepares ``workdir``.
  * run() advances the solve in-process on one GPU; ``nranks`` is accepted and
    ignored (the reference pairs a GPU rank with an I/O rank).
  * ``visc_order``, ``visc_stencil`` and ``precision`` are first-class keys
    (the reference routes VISC_ORDER / VISC_STENCIL to mod_globals.f90, where
    they are silently dropped).
Outputs are byte-compatible with the reference writer: data/Q%05d.vtr,
data/kinetic_energy.d, data/entropy.d and recal/Q00001.dat; in addition
data/diagnostics_fp64.d holds t, ke, entropy, enstrophy computed on the GPU in FP64.
"""
from __future__ import annotations

import json
import math
import pathlib
from typing import Any

import numpy as np

from .cases import CASES, CaseDef, build_initial
from .grid import cyclic_axis, fill_periodic, from_qj, jacobian, to_qj
from .ic import bc_to_params, ic_to_params

_ALIAS = {
    "scheme": "SCHEME", "visc": "VISC", "accuracy": "ORDER", "visc_order": "VISC_ORDER",
    "visc_stencil": "VISC_STENCIL", "tvd": "TVD", "slau": "SLAU_VARIANT", "rescale": "RESCALE",
    "recal": "RESTART", "rk": "RK", "gpumpi": "GPUMPI", "bc_x": "BC_X", "bc_y": "BC_Y", "bc_z": "BC_Z",
    "commz": "COMMZ", "precision": "PRECISION",
}

_VALUE_NORMALIZE: dict[str, dict[str, str]] = {
    "SCHEME": {"keep": "KEEP", "slau": "SLAU", "roe": "Roe", "hybrid": "Hybrid"},
    "VISC": {"euler": "Euler", "ns": "NS", "les": "LES"},
    "TVD": {"none": "none", "tvd": "tvd", "hybrid": "hybrid", "minmod": "tvd", "muscl4": "hybrid"},
    "SLAU_VARIANT": {"slau": "SLAU", "hrslau2": "HRSLAU2"},
    "VISC_STENCIL": {"central": "Central", "me4base": "ME4Base", "me4": "ME4Base"},
    "PRECISION": {"fp64": "fp64", "mixed": "mixed"},
}

_RK_NORMALIZE: dict[str, int] = {"tvd_rk3": 3, "rk3": 3, "rk4": 4, "classical_rk4": 4}

_CONFIG_KEYS = {"SCHEME", "VISC", "ORDER", "VISC_ORDER", "VISC_STENCIL", "TVD", "SLAU_VARIANT", "RESCALE",
                "RESTART", "RK", "GPUMPI", "BC_X", "BC_Y", "BC_Z", "COMMZ", "PRECISION"}


class Case:
    """Manage one simulation run: configure -> build (validate) -> run on the GPU."""

    def __init__(self, source: str, workdir: str, **params: Any) -> None:
        self.source = str(source)
        self.workdir = pathlib.Path(workdir).resolve()
        raw = dict(params)
        ic_spec = raw.pop("ic", None)
        bc_spec = raw.pop("bc", None)
        if ic_spec is not None:
            raw.update(ic_to_params(ic_spec))
        if bc_spec is not None:
            raw.update(bc_to_params(bc_spec))
        self.params: dict[str, Any] = {_ALIAS.get(k.lower(), k): v for k, v in raw.items()}
        self._built = False
        self._case: CaseDef | None = None
        self.config: dict = {}
        self.globals: dict = {}
        self.solver = None
        self.history: list[tuple[float, float, float, float]] = []

    # ------------------------------------------------------------------ setup
    def _setup(self) -> None:
        name = pathlib.PurePath(self.source).name
        if name not in CASES:
            raise FileNotFoundError(f"config.fypp not found in {self.source} (known cases: {sorted(CASES)})")
        case = CASES[name]
        config = dict(case.config)
        glob = dict(case.params)
        for k, v in self.params.items():
            if k == "RK" and isinstance(v, str):
                v = _RK_NORMALIZE.get(v.lower(), v)
            if k in _CONFIG_KEYS or k.upper() in _CONFIG_KEYS:
                k = k.upper()
                if isinstance(v, str) and k in _VALUE_NORMALIZE:
                    v = _VALUE_NORMALIZE[k].get(v.lower(), v)
                config[k] = v
            else:
                glob[k] = v
        ic_type = glob.pop("ic_type", None)
        if ic_type == 3:
            if not case.bc_x or case.dim != 2:
                raise RuntimeError("RiemannIC needs a case with a non-periodic x (2D_solver/ST)")
            glob["riemann"] = {k: glob.pop(k) for k in ("rho_l", "u_l", "p_l", "rho_r", "u_r", "p_r", "x0_frac")
                               if k in glob}
        if ic_type == 2 and "Ma" in glob:
            glob["M0"] = glob.pop("Ma")
        if ic_type == 1:
            glob["uniform"] = {k: glob.pop(k) for k in ("rho0", "u0", "v0", "w0", "p0") if k in glob}
        for key in ("BC_X", "BC_Y", "BC_Z", "RESCALE", "COMMZ"):
            if (key == "BC_X" and (case.bc_x or case.x_periodic_copy)) or (key == "BC_Y" and case.bc_y) or \
                    (key == "BC_Z" and case.bc_z) or (key == "COMMZ" and case.slabs):
                continue  # built: the case's boundary-cell rules, its z slabs
            if config.get(key):
                raise RuntimeError(f"{key}=True needs wall/inflow or multi-rank code paths, which are not built "
                                   "(only fully periodic rectilinear cases)")
        self._case, self.config, self.globals = case, config, glob

    def _solver_config(self, p: dict, dx, dy, dz):
        from .config import SolverConfig
        c = self.config
        return SolverConfig(
            dim=self._case.dim, nx=p["nx"], ny=p["ny"],
            nz=p.get("nz_grid", p.get("nz", 1)) if self._case.dim == 3 else 1,
            order=int(c["ORDER"]), scheme=c["SCHEME"], visc=c["VISC"], visc_order=int(c.get("VISC_ORDER", 0) or 0),
            visc_stencil=c.get("VISC_STENCIL", "Central"), tvd=c["TVD"], slau=c["SLAU_VARIANT"], rk=int(c["RK"]),
            gamma=p["gamma"], R=p["R"], Pr=p.get("Pr", 0.71), Prt=p.get("Prt", 0.9),
            threshold=p.get("threshold", 0.4), dt=p["dt"], dx=dx, dy=dy, dz=dz,
            bc_x=1 if (c.get("BC_X") or self._case.bc_x) and not self._case.x_periodic_copy else 0,
            bc_y=1 if (c.get("BC_Y") or self._case.bc_y) else 0,
            bc_z=1 if self._case.dim == 3 and (c.get("BC_Z") or self._case.bc_z) else 0,
            boundary=self._case.boundary(p, jacobian(dx, dy, None)) if self._case.boundary else None,
            boundary_order=self._case.boundary_order)

    def _initial(self):
        p = dict(self.globals)
        p["order"] = int(self.config["ORDER"])
        p, xc, yc, zc, dx, dy, dz, Q = build_initial(self._case, p)
        if "riemann" in p:
            # RiemannIC (ouxsbli/ic.py): the left state at x < x0_frac * Lx, the right
            # state from there on, uniform in y
            r = p["riemann"]
            gam = p["gamma"]
            left = xc < r.get("x0_frac", 0.5) * (xc[-1] - xc[0]) + xc[0]
            for side, m in (("l", left), ("r", ~left)):
                rho, u, pr = r.get("rho_" + side, 1.0), r.get("u_" + side, 0.0), r.get("p_" + side, 1.0)
                Q[m, 0] = rho
                Q[m, 1] = rho * u
                Q[m, 2] = 0.0
                Q[m, 3] = pr / (gam - 1.0) + 0.5 * rho * u * u
        if "uniform" in p:
            u = p["uniform"]
            Q[:] = 0.0
            rho = u.get("rho0", 1.0)
            vel = [u.get("u0", 0.0), u.get("v0", 0.0)] + ([u.get("w0", 0.0)] if self._case.dim == 3 else [])
            Q[:, 0] = rho
            for a, va in enumerate(vel):
                Q[:, 1 + a] = rho * va
            Q[:, -1] = u.get("p0", 0.71429) / (p["gamma"] - 1.0) + 0.5 * rho * sum(va * va for va in vel)
        return p, xc, yc, zc, dx, dy, dz, Q

    # ------------------------------------------------------------------ build
    def build(self) -> None:
        """Validate the configuration against liboux and prepare the work directory."""
        import ctypes as C
        from . import _lib
        self._setup()
        p, xc, yc, zc, dx, dy, dz, Q = self._initial()
        cfg = self._solver_config(p, dx, dy, dz)
        c, keep = cfg.to_c()
        h = C.c_void_p()
        rc = _lib.LIB.oux_create(C.byref(c), C.byref(h))
        if rc != 0:
            raise RuntimeError(f"configuration rejected by liboux: {_lib.LIB.oux_last_error().decode()}")
        _lib.LIB.oux_destroy(h)
        self.workdir.mkdir(parents=True, exist_ok=True)
        (self.workdir / "data").mkdir(exist_ok=True)
        (self.workdir / "recal").mkdir(exist_ok=True)
        snap = {"source": self.source, "config": self.config,
                "globals": {k: v for k, v in p.items() if isinstance(v, (int, float, str, bool, type(None)))}}
        (self.workdir / "case.json").write_text(json.dumps(snap, indent=1, default=str))
        self._built = True

    # ------------------------------------------------------------------ run
    def run(self, nranks: int = 2, device: str = "cuda:0") -> None:
        """Advance np output intervals of nt steps on the GPU, writing the reference's files."""
        if not self._built:
            raise RuntimeError("Must call build() before run()")
        from .output import HistoryWriter, make_1d_for_print, read_restart, ref_diagnostics, write_restart, write_vtr
        from .solver import Solver
        p, xc, yc, zc, dx, dy, dz, Q = self._initial()
        self.globals_used = p  # the derived parameters of this run (dt, nt, ...)
        dim = self._case.dim
        J = jacobian(dx, dy, dz if dim == 3 else None)
        nv = dim + 2
        if self.config.get("RESTART"):
            shape = (p["nx"], nv, p["ny"], p.get("nz_grid", p["nz"])) if dim == 3 else (p["nx"], nv, p["ny"])
            Q = read_restart(self.workdir / "recal" / "Q00001.dat", shape)
        qj = to_qj(Q, J)
        cfg = self._solver_config(p, dx, dy, dz)
        data = self.workdir / "data"
        data.mkdir(exist_ok=True)
        (self.workdir / "recal").mkdir(exist_ok=True)
        for f in ("kinetic_energy.d", "entropy.d", "diagnostics_fp64.d"):
            (data / f).unlink(missing_ok=True)
        hist = HistoryWriter(data)
        order = cfg.order
        zc_out = zc if dim == 3 else np.zeros(1)
        step_offset = int(p.get("step_offset", 0))

        def output(step: int, qj_now: np.ndarray, s) -> None:
            rho, pr, vel = make_1d_for_print(qj_now, J, p["gamma"])
            t = p.get("nt", 0) * step * p["dt"]
            if dim == 3:
                ke, ent = ref_diagnostics(cfg.nx, cfg.ny, cfg.nz, order, p["gamma"], rho, pr, vel)
                hist.record(t, ke, ent, step)
            write_vtr(data / f"Q{step + step_offset:05d}.vtr", np.float32(xc), np.float32(yc), np.float32(zc_out),
                      rho, pr, vel, dimension=3)
            d = s.diagnostics()
            self.history.append((t, *d))
            with open(data / "diagnostics_fp64.d", "a") as fh:
                fh.write(f"{t:.16e} {d[0]:.16e} {d[1]:.16e} {d[2]:.16e}\n")

        if self.config.get("COMMZ") and self._case.slabs:
            # the reference's z slabs, in one process on one GPU (ouxsbli_b200.slabs)
            from .slabs import LocalSlabs
            s = LocalSlabs(cfg, int(p.get("slabs", self._case.slabs)), device)
        else:
            s = Solver(cfg, device)
        self.solver = s
        s.set_state(qj)
        output(0, qj, s)
        nt, npo = int(p["nt"]), int(p["np"])
        for t2 in range(1, npo + 1):
            s.step(nt)
            bits = s.check_state()
            if bits:
                raise RuntimeError(f"device fault after interval {t2} (status bits {bits:#x}: NaN or non-positive "
                                   "density/pressure)")
            qj = s.get_state()
            output(t2, qj, s)
        write_restart(self.workdir / "recal" / "Q00001.dat", from_qj(qj, J))

    def __repr__(self) -> str:
        return f"Case(source={self.source!r}, workdir={str(self.workdir)!r}, params={self.params})"
