#!/usr/bin/env python
"""Benchmark of the explicit time step on one B200 (or N replicas).

Default workload (tgv512): the large single solve -- supersonic Taylor-Green vortex,
512^3 interior cells (518^3 with the 6th-order ghost layers), Ma = 1.25, Re = 1600,
KEEP/SLAU hybrid with the Ducros sensor (HRSLAU2, MUSCL with the hybrid TVD switch),
6th-order central differences, ME4 viscous stencil, TVD-RK3, FP64.  A "step" is one
full time step (three RK stages) of that grid.  Metric: Mcell-steps/s = interior
cells x steps / s.  The mixed FP32/FP64 form runs beside it, with its error against
the FP64 run after --mixed-check-steps steps from the same initial field.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                    [--workload tgv512|tgv256|walls256]

N > 1 runs N independent replicas (one per GPU, torch.distributed for the
barrier and the max-over-ranks time); the solve itself has no cross-GPU step.
--impl reference times the CPU restatement of the reference's kernels on the
host cores instead (the reference is CUDA Fortran with no CPU build): each step is
one RK3 step of a block of z planes of the same grid.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mcell-steps/s"
ALG_BYTES_PER_CELL_STEP = 320.0  # FP64 RK3: 8 state accesses x 5 variables x 8 B

# name -> (interior cells per axis, viscous stencil, description of the stencil)
WORKLOADS = {
    "tgv512": (512, "ME4Base", "ME4 viscous"),
    "tgv256": (256, "Central", "Central-6 viscous"),
}
# z planes of the block the CPU legs time (per step: one RK3 step of that block)
CPU_SAMPLE_PLANES = 32


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="tgv512", choices=["tgv512", "tgv256", "walls256"],
                    help="tgv512: the 512^3 ME4 supersonic TGV (default); tgv256: the 256^3 Central-6 one; "
                         "walls256: a --n^3 Navier-Stokes shear layer, periodic and with no-slip walls")
    ap.add_argument("--n", type=int, default=None, help="interior cells per axis (default: the workload's)")
    ap.add_argument("--scheme", default="Hybrid")
    ap.add_argument("--visc", default="NS")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--mixed-check-steps", type=int, default=2000,
                    help="steps of the mixed-vs-FP64 accuracy check from the initial field")
    ap.add_argument("--history-every", type=int, default=100,
                    help="diagnostics (KE, entropy, enstrophy) every so many steps of the accuracy check")
    ap.add_argument("--commz", action="store_true",
                    help="split the one grid into z slabs over the ranks (halo exchange after every stage; "
                         "strong scaling) instead of running independent replicas")
    ap.add_argument("--walls-config", default="all", choices=["all", "periodic", "y", "xy", "xyz"],
                    help="walls256: which grid (all: the four in turn)")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the batched 2D ensemble section")
    ap.add_argument("--ensemble-steps", type=int, default=500)
    ap.add_argument("--no-serving", action="store_true", help="skip the serving-stream section")
    ap.add_argument("--serving-requests", type=int, default=16)
    ap.add_argument("--serving-rate", type=float, default=2.0)
    ap.add_argument("--serving-budget-gb", type=float, default=4.0)
    a = ap.parse_args()
    if a.n is None:
        a.n = WORKLOADS.get(a.workload, (256,))[0]
    return a


def tgv_params(n: int):
    """Derived parameters and cell-centre axes of the supersonic TGV on n^3 interior cells."""
    from ouxsbli_b200.cases import CASES
    from ouxsbli_b200.grid import cyclic_axis
    case = CASES["NSTGV"]
    p = dict(case.params)
    p.update(nx=n + 6, ny=n + 6, nz=n + 6, order=6, M0=1.25, Re=1600.0, rho_mode="uniform",
             cfl_mode="acoustic", CFL=0.5, dt=None)
    p = case.derived(p)
    xc, dx = cyclic_axis(p["nx"], p["Lx"], 6)
    yc, dy = cyclic_axis(p["ny"], p["Ly"], 6)
    zc, dz = cyclic_axis(p["nz"], p["Lz"], 6)
    return p, (xc, yc, zc), (dx, dy, dz)


def make_cfg(args, p, dx, dy, dz, nz=None, bc_z=0, **kw):
    """SolverConfig of the workload (ouxsbli_b200.config: building it loads no GPU library)."""
    from ouxsbli_b200.config import SolverConfig
    stencil = WORKLOADS.get(args.workload, (0, "Central"))[1]
    return SolverConfig(dim=3, nx=p["nx"], ny=p["ny"], nz=nz or p["nz"], order=6, scheme=args.scheme,
                        visc=args.visc, visc_stencil=stencil, tvd="hybrid", slau="HRSLAU2", rk=3,
                        gamma=p["gamma"], R=p["R"], Pr=p["Pr"], Prt=p["Prt"], threshold=0.4, dt=p["dt"],
                        dx=dx, dy=dy, dz=dz, bc_z=bc_z, **kw)


def workload(args, **kw):
    """SolverConfig + initial QJ (reference layout) of the supersonic TGV."""
    from ouxsbli_b200.cases import CASES
    from ouxsbli_b200.grid import jacobian, to_qj
    p, (xc, yc, zc), (dx, dy, dz) = tgv_params(args.n)
    Q = CASES["NSTGV"].init(p, xc, yc, zc)
    cfg = make_cfg(args, p, dx, dy, dz, **kw)
    return cfg, to_qj(Q, jacobian(dx, dy, dz))


def cpu_sample(args, planes: int = CPU_SAMPLE_PLANES):
    """The block of the workload the CPU legs time: its z planes 0 .. planes-1 (all x
    and y cells, the same spacings, scheme and physics) as a z slab whose ghost planes
    hold the neighbouring planes' initial values (bc_z = 2, left alone by the fill)."""
    from ouxsbli_b200.cases import tgv_planes
    from ouxsbli_b200.grid import jacobian, to_qj
    p, (xc, yc, zc), (dx, dy, dz) = tgv_params(args.n)
    planes = min(planes, args.n)
    Q = tgv_planes(p, xc, yc, zc, 0, planes + 6)
    cfg = make_cfg(args, p, dx, dy, dz[:planes + 5], nz=planes + 6, bc_z=2)
    return cfg, to_qj(Q, jacobian(dx, dy, dz))


def config_json(args, cfg, world: int = 1):
    stencil = WORKLOADS.get(args.workload, (0, "Central", "Central-6 viscous"))[2]
    return {"workload": f"supersonic Taylor-Green vortex {args.n}^3 (+6 ghost layers), Ma 1.25, Re 1600, "
                        f"{args.scheme}-6 (HRSLAU2, MUSCL TVD hybrid) / {args.visc} {stencil}, TVD-RK3",
            "grid": [cfg.nx, cfg.ny, cfg.nz], "interior_cells": cfg.interior_cells(), "order": 6,
            "scheme": args.scheme, "visc": args.visc, "visc_stencil": cfg.visc_stencil, "rk": 3,
            "precision": "fp64",
            "l2": "inputs larger than L2 (state %.2f GB + stage arrays %.2f GB)" % (
                5 * cfg.nx * cfg.ny * cfg.nz * 8 / 1e9, 10 * cfg.nx * cfg.ny * cfg.nz * 8 / 1e9),
            "parallelism": f"{world} independent replicas"}


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def time_cpu_steps(cfg, qj, steps: int, warmup: int = 0, budget_s: float | None = None):
    """Wall time of RK3 steps of the oracle (the C++/OpenMP restatement of the
    reference's kernels) on all host cores; returns (steps timed, seconds, threads)."""
    from oracle import oracle
    threads = os.cpu_count() or 1
    os.environ["OMP_NUM_THREADS"] = str(threads)
    oracle.build()
    st = oracle.Stepper(cfg, qj)

    def one():
        for k in range(st.stages):
            st.stage(k)

    for _ in range(warmup):
        one()
    t0 = time.perf_counter()
    n = 0
    while n < steps:
        one()
        n += 1
        if budget_s is not None and time.perf_counter() - t0 >= budget_s:
            break
    return n, time.perf_counter() - t0, threads


def sample_text(cfg, n: int, el: float, extra: str = "") -> str:
    return (f"{n} RK3 step(s) of z planes 0..{cfg.nz - 7} of the grid: {cfg.nx - 6} x {cfg.ny - 6} x "
            f"{cfg.nz - 6} interior cells with their ghost layers ({cfg.nx}x{cfg.ny}x{cfg.nz}), the same "
            f"spacings, scheme and physics; the z ghost planes hold the neighbouring planes' initial values "
            f"({el:.1f} s, OpenMP over z planes, FP64, no FMA{extra})")


def cpu_baseline(args, budget_s: float = 15.0):
    """The oracle on the host cores, on a bounded block of the same workload."""
    cfg, qj = cpu_sample(args)
    n, el, threads = time_cpu_steps(cfg, qj, steps=3, budget_s=budget_s)
    return {"value": cfg.interior_cells() * n / el / 1e6, "unit": METRIC, "cores": threads, "kind": "port",
            "sample": sample_text(cfg, n, el)}


def bench_ensemble(dev, steps: int, check_steps: int, single_steps: int, count: int = 64, seed: int = 0):
    """Batched 2D ensemble: `count` seeded isentropic-vortex solves (sides over
    {64..512}, beta ~ U[1,5], Mach ~ U[0.1,0.8]), KEEP-4, Euler, RK4.  Times the plain
    FP64 single-solve form (each solve alone through oux_step), and the batched form
    (one persistent launch per step, CUDA graph, autotuned) in FP64 and mixed."""
    import dataclasses
    import torch
    from ouxsbli_b200.batch import Autotuner, Batch, tuning_key
    from ouxsbli_b200.cases import vortex_ensemble, vortex_exact, vortex_member
    from ouxsbli_b200.grid import jacobian
    from ouxsbli_b200.solver import Solver
    members = vortex_ensemble(count, seed)
    cases = [vortex_member(m, order=4, scheme="KEEP", visc="Euler", rk=4) for m in members]
    cells = sum(c.interior_cells() for c, _ in cases)
    st = torch.cuda.current_stream(dev)

    def timed(fn, k):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        a.record(st)
        fn(k)
        b.record(st)
        b.synchronize()
        return a.elapsed_time(b)

    # plain FP64 single-solve form, one solve after another
    single_ms = 0.0
    single_launches = 0
    for cfg, qj in cases:
        s = Solver(cfg, dev)
        s.set_state(qj)
        s.step(3)
        single_ms += timed(s.step, single_steps)
        single_launches += s.launches()
        s.close()
    single = cells * single_steps / (single_ms / 1e3) / 1e6

    tuner = Autotuner()
    out, finals = {}, {}
    for prec in ("fp64", "mixed"):
        sol = []
        for cfg, qj in cases:
            s = Solver(dataclasses.replace(cfg, precision=prec), dev)
            s.set_state(qj)
            sol.append(s)
        tuning = tuner.tune(sol, steps=3)
        trials = tuner.cache[tuning_key(sol)]["trials"]
        best_by_mode = {}
        for ms_t, t in trials:
            best_by_mode[t["mode"]] = min(ms_t, best_by_mode.get(t["mode"], float("inf")))
        b = Batch(sol, tuning)
        b.step(3)
        ms = timed(b.step, steps)
        info = b.info()
        b.close()
        for s, (cfg, qj) in zip(sol, cases):  # accuracy run from the initial fields
            s.set_state(qj)
        b = Batch(sol, tuning)
        b.step(check_steps)
        if b.status() != 0:
            raise RuntimeError("batched step reported a dependency-wait timeout")
        finals[prec] = [s.get_state() for s in sol]
        b.close()
        for s in sol:
            s.close()
        out[prec] = {"value": cells * steps / (ms / 1e3) / 1e6, "unit": METRIC, "ms_per_step": ms / steps,
                     "tuning": dataclasses.asdict(tuning), "work_items_per_step": info["items"],
                     "phases_per_step": info["phases"], "persistent_grid": info["grid"],
                     "autotuner_best_ms_per_step_by_mode": best_by_mode,
                     "gpu_launches_per_step": 1 if tuning.mode == "persistent" else single_launches // single_steps}
    # after check_steps: mixed vs FP64 per field (worst member), FP64 vs the exact translated vortex
    worst = [0.0] * 4
    exact_l2 = []
    for m, (cfg, _), q64, q32 in zip(members, cases, finals["fp64"], finals["mixed"]):
        g = cfg.g
        a, b_ = q64[g:-g, :, g:-g], q32[g:-g, :, g:-g]
        for l in range(4):
            worst[l] = max(worst[l], float(np.linalg.norm(b_[:, l] - a[:, l]) / np.linalg.norm(a[:, l])))
        ex = vortex_exact(m, 4, check_steps * m.dt)
        J = jacobian(cfg.dx, cfg.dy, None)
        rho = (J[:, None, :] * q64)[g:-g, 0, g:-g]
        exact_l2.append(float(np.linalg.norm(rho - ex[g:-g, 0, g:-g]) / np.linalg.norm(ex[g:-g, 0, g:-g])))
    alg = 512.0  # B per cell-step: 2D FP64 RK4, 16 state accesses x 4 variables x 8 B
    return {"workload": f"{count} 2D isentropic vortices (seed {seed}), sides {sorted(set(m.n for m in members))}, "
                        "KEEP-4 Euler RK4", "interior_cells": cells,
            "single_fp64": {"value": single, "unit": METRIC, "steps_per_solve": single_steps,
                            "gpu_launches_per_step": single_launches // single_steps},
            "batched_fp64": out["fp64"], "batched_mixed": out["mixed"],
            "speedup_batched_mixed_vs_single_fp64": out["mixed"]["value"] / single,
            "speedup_batched_fp64_vs_single_fp64": out["fp64"]["value"] / single,
            "hbm_gbs_fp64_batched_at_512B_per_cell_step": alg * out["fp64"]["value"] * 1e6 / 1e9,
            "mixed_vs_fp64_rel_l2_worst_member": worst, "after_steps": check_steps,
            "fp64_rho_rel_l2_vs_exact_vortex": {"max": max(exact_l2), "median": float(np.median(exact_l2))}}


def bench_serving(dev, count: int, rate: float, budget_gb: float, seed: int = 0):
    """Serving stream of 3D decaying-turbulence LES requests (SLAU-6, SMS, RK3, mixed)."""
    import dataclasses
    from ouxsbli_b200.batch import Autotuner, Tuning, tuning_key
    from ouxsbli_b200.serving import GRID_SIZES, Server, SolveRequest, poisson_stream, summarize
    from ouxsbli_b200.solver import Solver
    srv = Server(device=dev, hbm_budget=int(budget_gb * (1 << 30)), quantum=100, tuner=Autotuner())
    # tune once on a representative mix (one request of every grid size); the server
    # then reuses the cached choice of the nearest size class
    rep = []
    for i, n in enumerate(GRID_SIZES):
        cfg, qj = SolveRequest(rid=i, n=n, steps=1, seed=1000 + i).build(srv.physics)
        s = Solver(cfg, dev)
        s.set_state(qj)
        rep.append(s)
    cands = (Tuning(), Tuning(pencil=8, chunk=2304), Tuning(mode="graph"))
    chosen = srv.tuner.tune(rep, steps=3, candidates=cands, force=True)
    key = tuning_key(rep)
    trials = srv.tuner.cache[key]["trials"]
    for s in rep:
        s.close()
    reqs = poisson_stream(count, rate, seed)
    # the same requests one after another, each alone (device time per step of each grid
    # size, measured after 3 warm-up steps): the rate without batching and host gaps
    import torch
    st = torch.cuda.current_stream(dev)
    ms_per_step = {}
    for n in sorted({r.n for r in reqs}):
        cfg, qj = SolveRequest(rid=0, n=n, steps=1, seed=1).build(srv.physics)
        s = Solver(cfg, dev)
        s.set_state(qj)
        s.step(3)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st)
        s.step(20)
        b.record(st)
        b.synchronize()
        ms_per_step[n] = a.elapsed_time(b) / 20
        s.close()
    solo_ms = sum(r.steps * ms_per_step[r.n] for r in reqs)
    solo_rate = sum(r.n ** 3 * r.steps for r in reqs) / (solo_ms / 1e3) / 1e6
    res = srv.run(reqs)
    return summarize(res) | {"unit_latency": "s", "arrival_rate_per_s": rate, "hbm_budget_gb": budget_gb,
                             "grids": sorted({r.n for r in reqs}), "steps_range": [200, 2000],
                             "physics": "SLAU-6 HRSLAU2, SMS LES, TVD-RK3, mixed FP32/FP64",
                             "tuning": dataclasses.asdict(chosen),
                             "tuning_trials_ms_per_step": {t[1]["mode"] + (f"-p{t[1]['pencil']}" if t[1]["mode"] == "persistent" else ""): t[0] for t in trials},
                             "server": srv.stats,
                             "solo_one_after_another": {"aggregate_mcell_steps_per_s": solo_rate,
                                                        "device_ms_per_step_by_grid": ms_per_step}}


def run_reference(args):
    """--impl reference: the reference's own path is CUDA Fortran with no CPU build, and
    it cannot be compiled here (no Fortran compiler, NVHPC, MPI or fypp), so its CPU
    stand-in is the oracle, the C++/OpenMP restatement of its kernels, on all host cores.
    Each step is one RK3 step of a block of z planes of the same workload (metric per
    cell-step).  Nothing here maps liboux.so: the configuration and the initial field
    come from ouxsbli_b200.config / cases / grid."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return 0
    cfg, qj = cpu_sample(args)
    n, el, threads = time_cpu_steps(cfg, qj, steps=args.steps, warmup=args.warmup)
    val = cfg.interior_cells() * n / el / 1e6
    p, _, (dx, dy, dz) = tgv_params(args.n)
    full = make_cfg(args, p, dx, dy, dz)
    line = {"metric": METRIC, "value": val, "unit": METRIC, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": el * 1e3 / n,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (analytic TGV initial field)", "impl": "reference",
            "config": config_json(args, full, world),
            "cpu_baseline": {"value": val, "unit": METRIC, "cores": threads, "kind": "port",
                             "sample": sample_text(cfg, n, el, f"; after {args.warmup} warm-up step(s)")},
            "e2e": {"value": val, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


WALL_GRIDS = {  # walls256: non-periodic x, z and the rules of the faces (y always has no-slip walls)
    "periodic": None,
    "y": (0, 0, {"y_lo": "noslip_wall", "y_hi": "noslip_wall"}),
    "xy": (1, 0, {"x_lo": "zero_gradient", "x_hi": "zero_gradient", "y_lo": "noslip_wall", "y_hi": "zero_gradient"}),
    "xyz": (1, 1, {"x_lo": "slip_wall", "x_hi": "slip_wall", "y_lo": "noslip_wall", "y_hi": "noslip_wall",
                   "z_lo": "slip_wall", "z_hi": "noslip_wall"}),
}


def walled_workload(n: int, which: str):
    """A viscous shear layer of air (Sutherland, 300 K) in a box of n^3 interior cells,
    KEEP-6 / Central-6 NS, RK3: u = 5 sin(pi y / H) m/s with a 3D perturbation, H = 1 mm.
    `which` picks the boundaries (WALL_GRIDS); "periodic" has all three axes periodic
    (y then with its own ghost layers)."""
    import math
    from ouxsbli_b200.grid import cyclic_axis, jacobian, to_qj
    from ouxsbli_b200.solver import SolverConfig
    order, g = 6, 3
    H, Rg, gam, T0, rho0, U = 1.0e-3, 287.03, 1.4, 300.0, 1.2, 5.0
    spec = WALL_GRIDS[which]
    bc_x, bc_z, rules = (0, 0, None) if spec is None else spec
    bc_y = 0 if spec is None else 1

    def axis(L, nonper):
        if nonper:
            m = n + 2
            d = np.full(m - 1, L / (m - 1))
            return m, np.concatenate([[0.0], np.cumsum(d)]), d
        x, d = cyclic_axis(n + 2 * g, L, order)
        return n + 2 * g, x, d

    nx, x, dx = axis(0.5e-3, bc_x)
    ny, y, dy = axis(H, bc_y)
    nz, z, dz = axis(0.4e-3, bc_z)
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    sy = np.sin(math.pi * Y / H)
    rho = rho0 * (1.0 + 0.02 * np.sin(2 * math.pi * X / 0.5e-3) * np.cos(2 * math.pi * Z / 0.4e-3) * sy)
    u = U * sy
    v = 0.3 * U * np.sin(2 * math.pi * X / 0.5e-3) * sy ** 2
    w = 0.2 * U * np.sin(2 * math.pi * Z / 0.4e-3) * np.cos(2 * math.pi * X / 0.5e-3) * sy
    Q = np.zeros((nx, 5, ny, nz), order="F")
    Q[:, 0], Q[:, 1], Q[:, 2], Q[:, 3] = rho, rho * u, rho * v, rho * w
    Q[:, 4] = rho0 * Rg * T0 / (gam - 1.0) + 0.5 * rho * (u * u + v * v + w * w)
    del X, Y, Z, sy, rho, u, v, w
    dt = 0.4 * min(dx.min(), dy.min(), dz.min()) / (U + math.sqrt(gam * Rg * T0))
    cfg = SolverConfig(dim=3, nx=nx, ny=ny, nz=nz, order=order, scheme="KEEP", visc="NS", rk=3, bc_x=bc_x,
                       bc_y=bc_y, bc_z=bc_z, dt=dt, gamma=gam, R=Rg, Pr=0.72, dx=dx, dy=dy, dz=dz, boundary=rules)
    return cfg, to_qj(Q, jacobian(dx, dy, dz))


def run_walls(args):
    """Step rate of --n^3 KEEP-6 / Central-6 NS grids with and without no-slip walls
    (the walled sweep variants beside the periodic ones), per-kernel times included."""
    import torch
    from ouxsbli_b200 import _lib
    from ouxsbli_b200.solver import Solver
    dev = torch.device("cuda", 0)
    kinds = KINDS
    out = {"workload": "walls256", "n": args.n, "steps": args.steps, "warmup": args.warmup,
           "config": "KEEP-6, Central-6 NS, RK3, FP64; u = 5 sin(pi y / H) m/s shear layer of air, H = 1 mm",
           "grids": {}}
    for which in (WALL_GRIDS if args.walls_config == "all" else [args.walls_config]):
        cfg, qj = walled_workload(args.n, which)
        s = Solver(cfg, dev)
        s.set_state(qj)
        del qj
        s.step(args.warmup)
        st = torch.cuda.current_stream(dev)
        _lib.check(_lib.LIB.oux_profile(s._h, 1))
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        a.record(st)
        s.step(args.steps)
        b.record(st)
        b.synchronize()
        kms, kcnt = (C.c_double * len(kinds))(), (C.c_int64 * len(kinds))()
        _lib.check(_lib.LIB.oux_profile_read(s._h, kms, kcnt, len(kinds)))
        _lib.check(_lib.LIB.oux_profile(s._h, 0))
        ms = a.elapsed_time(b) / max(args.steps, 1)
        out["grids"][which] = {
            "ms_per_step": ms, "value": cfg.interior_cells() / (ms / 1e3) / 1e6, "unit": METRIC,
            "status": s.check_state(),
            "per_kernel_avg_ms": {k: kms[i] / kcnt[i] for i, k in enumerate(kinds) if kcnt[i]}}
        s.close()
    print(json.dumps(out), flush=True)
    return 0


def run_commz(args):
    """The --n^3 workload split into z slabs over the torchrun ranks (one slab per GPU,
    halo exchange over NCCL after every stage, ouxsbli_b200.slabs): whole-grid
    cell-steps per second of the slowest rank, strong scaling."""
    import datetime
    import torch
    import torch.distributed as dist
    from ouxsbli_b200.replicas import max_over_ranks
    from ouxsbli_b200.slabs import SlabSolver
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    group = None
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    cfg, qj = workload(args)
    slab = SlabSolver(cfg, rank, world, dev, group)
    slab.set_global_state(qj)
    stream = torch.cuda.current_stream(dev)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    slab.step(args.warmup)
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    slab.step(args.steps)
    e1.record(stream)
    barrier()
    ms = max_over_ranks(e0.elapsed_time(e1), dev)
    cells = cfg.interior_cells()
    if rank == 0:
        print(json.dumps({"metric": METRIC, "value": cells * args.steps / (ms / 1e3) / 1e6, "unit": METRIC,
                          "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                          "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "strong",
                          "vs_baseline": None, "dtype": "f64", "data": "synthetic (analytic TGV initial field)",
                          "config": config_json(args, cfg, world) | {"parallelism": f"{world} z slabs (COMMZ)"},
                          "gpu_launches": None}))
    slab.close()
    if world > 1:
        dist.destroy_process_group()


# algorithmic HBM bytes per interior cell of each kernel launch (FP64, 3D, RK3 averaged
# over the three stages): fields read / state and accumulators read and written once
ALG_CELL = {"prim": 96.0, "sensor": 32.0, "prim_sensor": 104.0, "grad": 104.0,
            "sweep_x": 136.0, "sweep_y": 176.0, "sweep_z": (216.0 + 256.0 + 256.0) / 3.0}
# kernel kinds of oux_profile_read (enum KernelKind of oux_api.cu); prim_sensor: the 3D
# pass that writes the primitive fields and the Ducros sensor (the mixed form's sensor
# schemes); grad: the node velocity gradients (Central-4/6 and ME4 viscous stencils), and
# in FP64 the Ducros sensor too
KINDS = ["prim", "sensor", "sgs", "sgs_edges", "sweep_x", "sweep_y", "sweep_z", "ghost", "prim_sensor", "grad"]


def read_profile(h):
    """Per-kernel CUDA-event times recorded by oux_profile during the timed region."""
    from ouxsbli_b200 import _lib
    n = len(KINDS)
    kms, kcnt = (C.c_double * n)(), (C.c_int64 * n)()
    _lib.check(_lib.LIB.oux_profile_read(h, kms, kcnt, n))
    _lib.check(_lib.LIB.oux_profile(h, 0))
    tot = sum(kms[i] for i in range(n)) or 1.0
    return {nm: {"launches": int(kcnt[i]), "avg_ms": kms[i] / kcnt[i], "share": kms[i] / tot}
            for i, nm in enumerate(KINDS) if kcnt[i]}


def roofline_of(args, per_kernel, cells, ms_per_step, peaks):
    peak = float(peaks.get("hbm_gbs", 6650.0))
    dom = max(per_kernel, key=lambda k: per_kernel[k]["share"]) if per_kernel else None
    achieved = ALG_CELL.get(dom, 0.0) * cells / (per_kernel[dom]["avg_ms"] / 1e3) / 1e9 if dom else 0.0
    # ncu figures of the same kernels on a small case of the same physics (profiles/):
    # DRAM bytes per interior cell of one launch, scaled by the cells of one launch here,
    # and the FP64-pipe utilisation
    traffic, prof = None, {}
    try:
        prof = json.load(open(os.path.join(ROOT, "profiles", "sweep_traffic.json"))).get(args.workload, {})
        if dom in prof.get("dram_bytes_per_interior_cell", {}):
            traffic = prof["dram_bytes_per_interior_cell"][dom] * cells
    except Exception:
        pass
    step_achieved = ALG_BYTES_PER_CELL_STEP * cells / (ms_per_step / 1e3) / 1e9
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic, "kernel": dom,
            "alg_bytes_per_launch": f"{ALG_CELL.get(dom, 0.0):.1f} B x {cells} interior cells "
                                    "(per-kernel table in DESIGN.md; mean over the 3 RK3 stages)",
            "traffic_source": prof.get("source"), "fp64_pipe_pct_ncu": prof.get("fp64_pipe_pct"),
            "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
            "dominant_kernel": dom, "per_kernel": per_kernel,
            "step": {"achieved": step_achieved, "frac": step_achieved / peak,
                     "alg_bytes": "320 B per interior cell-step (8 state accesses x 5 vars x 8 B)"}}


def accuracy_run(cfg, qj, dev, steps: int, every: int):
    """Final state and (step, KE, entropy, enstrophy) history of `steps` steps from qj."""
    from ouxsbli_b200.solver import Solver
    s = Solver(cfg, dev)
    s.set_state(qj)
    hist = [(0,) + tuple(s.diagnostics())]
    n = 0
    while n < steps:
        k = min(every, steps - n)
        s.step(k)
        n += k
        hist.append((n,) + tuple(s.diagnostics()))
    status = s.check_state()
    q = s.get_state()
    s.close()
    return q, hist, status


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "walls256":
        return run_walls(args)
    if args.commz:
        return run_commz(args)
    import dataclasses
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    from ouxsbli_b200 import _lib
    from ouxsbli_b200.replicas import job_rate, max_over_ranks
    from ouxsbli_b200.solver import Solver
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass

    cfg, qj = workload(args)
    s = Solver(cfg, dev)
    s.set_state(qj)
    stream = torch.cuda.current_stream(dev)
    cells = cfg.interior_cells()

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    # warm-up
    s.step(args.warmup)
    barrier()
    # timed region: per-kernel CUDA events (live, on the launching stream)
    _lib.check(_lib.LIB.oux_profile(s._h, 1))
    clocks = ClockSampler(local)
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    ev0.record(stream)
    s.step(args.steps)
    ev1.record(stream)
    barrier()
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    launches_per_step = s.launches() / max(args.steps, 1)
    per_kernel = read_profile(s._h)
    value, ms_max = job_rate(cells * args.steps, ms, dev)
    value /= 1e6
    ms_per_step = ms_max / args.steps

    # end to end through the public API: every step is an independent job that copies
    # its input state in from pinned host memory, advances one step and copies the
    # result back to pinned host memory.  Jobs go round-robin over NPIPE handles, each
    # with its own stream, so one job's copies overlap another's compute (the copy
    # engines and the SMs work at the same time); the sequential figure is kept beside it.
    e2e = None
    if not args.no_e2e:
        n_el = qj.size
        lib = _lib.LIB
        h_in = torch.from_numpy(np.ascontiguousarray(qj.ravel(order="F"))).pin_memory()
        pin = C.cast(C.c_void_p(h_in.data_ptr()), C.POINTER(C.c_double))
        # three handles let one job's upload, another's step and a third's download run at
        # once (with two, each stream's own upload, step and download follow one another;
        # 512^3 on one B200: 826 with two, 962 with three, 961 with four Mcell-steps/s,
        # where the host link bounds it); two where the device cannot hold three solves
        per_handle = s.state.numel() * 8 + s.scratch.numel() * 8
        free_b, _ = torch.cuda.mem_get_info(dev)
        NPIPE = 3 if free_b > 2 * per_handle + (4 << 30) else 2
        pipes = [s] + [Solver(cfg, dev) for _ in range(NPIPE - 1)]
        streams = [torch.cuda.Stream(dev) for _ in range(NPIPE)]
        h_out = [torch.empty(n_el, dtype=torch.float64).pin_memory() for _ in range(NPIPE)]
        pouts = [C.cast(C.c_void_p(h.data_ptr()), C.POINTER(C.c_double)) for h in h_out]
        k_e2e = max(NPIPE, args.steps)  # the same step count as the device-timed value

        def pipelined(k):
            for n in range(k):
                q, st = n % NPIPE, streams[n % NPIPE]
                sv_ = C.c_void_p(st.cuda_stream)
                _lib.check(lib.oux_set_state(pipes[q]._h, pin, sv_))
                _lib.check(lib.oux_step(pipes[q]._h, 1, sv_))
                _lib.check(lib.oux_get_state_async(pipes[q]._h, pouts[q], sv_))

        def timed_multi(fn, k):
            barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for st in streams:
                st.wait_event(e0)
            fn(k)
            for st in streams:
                ev = torch.cuda.Event()
                ev.record(st)
                stream.wait_event(ev)
            e1.record(stream)
            barrier()
            return max_over_ranks(e0.elapsed_time(e1), dev)

        pipelined(NPIPE)  # warm-up
        ms_pipe = timed_multi(pipelined, k_e2e)

        def sequential(k):
            sv_ = C.c_void_p(streams[0].cuda_stream)
            for _ in range(k):
                _lib.check(lib.oux_set_state(s._h, pin, sv_))
                _lib.check(lib.oux_step(s._h, 1, sv_))
                _lib.check(lib.oux_get_state(s._h, pouts[0], sv_))  # synchronizes

        k_seq = max(1, min(args.steps, 3))
        ms_seq = timed_multi(sequential, k_seq)
        # every job advanced the same initial field by one step: all outputs agree
        for st in streams:
            st.synchronize()
        if not all(torch.equal(h_out[0], h) for h in h_out[1:]):
            raise RuntimeError("pipelined end-to-end jobs disagree")
        for q in pipes[1:]:
            q.close()
        del pipes, h_out, pouts, h_in
        e2e = {"value": cells * k_e2e * world / (ms_pipe / 1e3) / 1e6, "unit": METRIC,
               "h2d_bytes_per_step": int(n_el * 8), "d2h_bytes_per_step": int(n_el * 8),
               "steps": k_e2e,
               "path": f"per step: oux_set_state(pinned host QJ) -> oux_step(1) -> oux_get_state_async(pinned "
                       f"host QJ); steps round-robin over {NPIPE} handles / streams",
               "sequential": {"value": cells * k_seq * world / (ms_seq / 1e3) / 1e6, "steps": k_seq,
                              "path": "oux_set_state -> oux_step(1) -> oux_get_state (synchronous), one handle"}}
    s.close()
    del s
    torch.cuda.empty_cache()

    # mixed form on the same workload: throughput, and (one GPU) its error against the
    # FP64 run after --mixed-check-steps steps from the same initial field
    mixed = None
    if not args.no_mixed:
        cfg_m = dataclasses.replace(cfg, precision="mixed")
        sm = Solver(cfg_m, dev)
        sm.set_state(qj)
        sm.step(args.warmup)
        barrier()
        _lib.check(_lib.LIB.oux_profile(sm._h, 1))
        m0, m1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        m0.record(stream)
        sm.step(args.steps)
        m1.record(stream)
        barrier()
        mixed_kernels = read_profile(sm._h)
        sm.close()
        del sm
        tm = max_over_ranks(m0.elapsed_time(m1), dev)
        mval = cells * args.steps * world / (tm / 1e3) / 1e6
        mixed = {"value": mval, "unit": METRIC, "ms_per_step": tm / args.steps,
                 "speedup_vs_fp64": mval / value, "per_kernel": mixed_kernels,
                 "form": "FP32 stage increments, primitive fields (p, T as deviations from per-solve references) "
                         "and face fluxes; FP64 Q^n, flux differences, RK combinations, diagnostics"}
        if world == 1 and args.mixed_check_steps > 0:
            n_err, every = args.mixed_check_steps, max(1, args.history_every)
            q64, h64, st64 = accuracy_run(cfg, qj, dev, n_err, every)
            q32, h32, st32 = accuracy_run(cfg_m, qj, dev, n_err, every)
            g = cfg.g
            sl = (slice(g, -g), slice(None), slice(g, -g), slice(g, -g))
            a32, a64 = q32[sl], q64[sl]
            errs = [float(np.linalg.norm((a32[:, l] - a64[:, l]).ravel()) / np.linalg.norm(a64[:, l].ravel()))
                    for l in range(5)]
            mnorm = np.linalg.norm(a64[:, 1:4].ravel())
            errs_mom = [float(np.linalg.norm((a32[:, l] - a64[:, l]).ravel()) / mnorm) for l in (1, 2, 3)]
            del a32, a64, q32, q64
            ens64, ens32 = np.array([h[3] for h in h64]), np.array([h[3] for h in h32])
            ke64, ke32 = np.array([h[1] for h in h64]), np.array([h[1] for h in h32])
            ipk = int(np.argmax(ens64))
            mixed |= {"after_steps": n_err, "rel_l2_vs_fp64": errs, "rel_l2_momentum_vector_norm": errs_mom,
                      "fields": ["rho", "rho u", "rho v", "rho w", "E"],
                      "ke_rel_dev_final": float(abs(ke32[-1] - ke64[-1]) / abs(ke64[-1])),
                      "ke_rel_dev_max_over_history": float(np.max(np.abs(ke32 - ke64) / np.abs(ke64))),
                      "enstrophy_rel_dev_final": float(abs(ens32[-1] - ens64[-1]) / abs(ens64[-1])),
                      "enstrophy_rel_dev_max_over_history": float(np.max(np.abs(ens32 - ens64) / np.abs(ens64))),
                      "enstrophy_peak_fp64": {"step": int(h64[ipk][0]), "value": float(ens64[ipk])},
                      "enstrophy_peak_rel_dev": float(abs(np.max(ens32) - ens64[ipk]) / abs(ens64[ipk])),
                      "history_every": every, "status_bits": [st64, st32],
                      "history_fp64": [list(h) for h in h64], "history_mixed": [list(h) for h in h32]}

    roofline = roofline_of(args, per_kernel, cells, ms_per_step, peaks)
    line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (analytic TGV initial field)",
            "config": config_json(args, cfg, world),
            "roofline": roofline, "clocks": clk, "e2e": e2e, "mixed": mixed,
            "gpu_launches": int(round(launches_per_step * args.steps))}
    # the batched-ensemble and serving sections are single-GPU sub-lines (rank 0, N = 1)
    if rank == 0 and world == 1 and not args.no_ensemble:
        line["ensemble2d"] = bench_ensemble(dev, args.ensemble_steps, 1000, 50)
    if rank == 0 and world == 1 and not args.no_serving:
        line["serving"] = bench_serving(dev, args.serving_requests, args.serving_rate, args.serving_budget_gb)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
