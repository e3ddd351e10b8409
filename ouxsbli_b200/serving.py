"""Continuous-batching solve server.

Requests (case, grid, Reynolds / Mach numbers, step count) arrive over time.  The
server keeps every admitted solve's state resident in HBM, admits waiting requests
whenever the memory budget and the slot limit allow, and advances all admitted
solves together with one batched persistent-kernel launch per time step
(`ouxsbli_b200.batch.Batch`).  Time advances in quanta of at most `quantum` steps;
after each quantum finished solves are retired (their memory freed) and newly
arrived requests join, so a request that arrives while others are on the GPU runs
in the same launches as theirs from the next quantum on.  While the GPU runs a
quantum host threads build the initial fields of requests that have arrived, so
that work overlaps the device's and never holds up the loop that feeds it.

Each solve's arithmetic does not depend on which other solves share its batch: a
result is bit-for-bit the same alone and in a mix.
"""
from __future__ import annotations

import ctypes as C
import time
from concurrent.futures import Future, ThreadPoolExecutor
from dataclasses import dataclass, field
from typing import Callable, Sequence

import numpy as np
import torch

from ._lib import LIB, check
from .batch import Autotuner, Batch, Tuning, tuning_key
from .solver import Solver, SolverConfig

GRID_SIZES = (32, 48, 64, 96, 128)


@dataclass
class SolveRequest:
    """One decaying-turbulence LES request (the serving workload's case)."""
    rid: int
    n: int                 # interior cells per side
    steps: int
    seed: int
    arrival: float = 0.0   # seconds after the stream starts
    mt: float = 0.3        # turbulent Mach number
    re_lambda: float = 100.0

    def build(self, physics: dict):
        from .turbulence import decaying_turbulence
        return decaying_turbulence(self.n, order=physics.get("order", 6), seed=self.seed, mt=self.mt,
                                   re_lambda=self.re_lambda,
                                   **{k: v for k, v in physics.items() if k != "order"})


@dataclass
class SolveResult:
    rid: int
    n: int
    steps: int
    arrival: float
    admitted: float
    completed: float
    diagnostics: tuple
    state: np.ndarray | None = None

    @property
    def latency(self) -> float:
        return self.completed - self.arrival


def poisson_stream(count: int, rate: float, seed: int, sizes: Sequence[int] = GRID_SIZES,
                   steps: tuple[int, int] = (200, 2000)) -> list[SolveRequest]:
    """Seeded Poisson arrivals (exponential gaps of mean 1/rate seconds), grid sizes
    uniform over `sizes`, step counts uniform over [steps[0], steps[1]]."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(count):
        t += float(rng.exponential(1.0 / rate))
        out.append(SolveRequest(rid=i, n=int(rng.choice(sizes)), steps=int(rng.integers(steps[0], steps[1] + 1)),
                                seed=int(rng.integers(0, 2 ** 31 - 1)), arrival=t))
    return out


def request_bytes(cfg: SolverConfig) -> int:
    """Device bytes a solve holds while admitted (state + scratch)."""
    c, keep = cfg.to_c()
    sb, kb = C.c_size_t(), C.c_size_t()
    check(LIB.oux_state_bytes(C.byref(c), C.byref(sb)))
    check(LIB.oux_scratch_bytes(C.byref(c), C.byref(kb)))
    del keep
    return int(sb.value + kb.value)


def request_bytes_for(n: int, physics: dict) -> int:
    """Device bytes of a request of n^3 interior cells with the given physics, from its
    configuration alone (the initial field is not needed to size it)."""
    from .grid import cyclic_axis
    order = physics.get("order", 6)
    nx = n + order
    _, d = cyclic_axis(nx, 1.0, order)
    cfg = SolverConfig(dim=3, nx=nx, ny=nx, nz=nx, order=order, dx=d, dy=d.copy(), dz=d.copy(),
                       **{k: v for k, v in physics.items() if k != "order"})
    return request_bytes(cfg)


def summarize(results: Sequence[SolveResult]) -> dict:
    """p50 / p99 completion latency and aggregate Mcell-steps/s of a served stream."""
    lat = np.array([r.latency for r in results])
    cells = sum(r.n ** 3 * r.steps for r in results)
    t_first = min(r.arrival for r in results)
    t_last = max(r.completed for r in results)
    return {"requests": len(results), "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "cell_steps": int(cells),
            "aggregate_mcell_steps_per_s": cells / max(t_last - t_first, 1e-9) / 1e6,
            "span_s": t_last - t_first}


@dataclass
class _Active:
    req: SolveRequest
    solver: Solver
    bytes: int
    remaining: int
    admitted: float


@dataclass
class Server:
    device: torch.device | str = "cuda:0"
    hbm_budget: int = 8 << 30           # bytes of solve state + scratch admitted at once
    max_active: int = 64                # slot limit
    quantum: int = 100                  # steps between admission / retirement points
    physics: dict = field(default_factory=lambda: dict(order=6, scheme="SLAU", visc="LES", rk=3,
                                                       precision="mixed"))
    tuner: Autotuner | None = None      # cached tunings are used when present
    keep_states: bool = False           # return each final state (host copy)
    build_workers: int = 2              # host threads that build arriving requests' initial fields
    default_tuning: Tuning = field(default_factory=Tuning)  # when the tuner has nothing cached
    stats: dict = field(default_factory=dict)

    def _tuning(self, solvers) -> Tuning:
        if self.tuner is not None:
            t = self.tuner.lookup_nearest(tuning_key(solvers))
            if t is not None:
                return t
        return self.default_tuning

    def run(self, requests: Sequence[SolveRequest], clock: Callable[[], float] = time.perf_counter,
            sleep: Callable[[float], None] = time.sleep) -> list[SolveResult]:
        dev = torch.device(self.device)
        pending = sorted(requests, key=lambda r: (r.arrival, r.rid))
        # waiting requests in arrival order: (request, device bytes, future of (cfg, initial QJ))
        queue: list[tuple[SolveRequest, int, Future]] = []
        pool = ThreadPoolExecutor(max_workers=max(1, self.build_workers))
        sizes: dict[int, int] = {}
        active: list[_Active] = []
        results: list[SolveResult] = []
        used = 0
        batch: Batch | None = None
        dirty = True
        steps_run = quanta = 0
        peak_bytes = peak_active = 0
        # where the wall time goes (host seconds per part of the loop, device time of the quanta)
        split = {"arrivals_s": 0.0, "admit_s": 0.0, "batch_build_s": 0.0, "step_enqueue_s": 0.0,
                 "wait_device_s": 0.0, "retire_s": 0.0, "idle_s": 0.0}
        gpu_ms = 0.0
        stream = None  # the device's current stream, looked up when the first quantum runs

        class _Part:
            def __init__(self, key):
                self.key = key

            def __enter__(self):
                self.t = time.perf_counter()

            def __exit__(self, *exc):
                split[self.key] += time.perf_counter() - self.t

        t0 = clock()
        wall0 = time.perf_counter()

        def arrivals(now: float) -> None:
            # every request that has arrived joins the queue; its initial field is built
            # on a host thread, off the loop that feeds the device
            while pending and pending[0].arrival <= now:
                r = pending.pop(0)
                if r.n not in sizes:
                    sizes[r.n] = request_bytes_for(r.n, self.physics)
                need = sizes[r.n]
                if need > self.hbm_budget:
                    raise ValueError(f"request {r.rid} needs {need} bytes, more than the budget {self.hbm_budget}")
                queue.append((r, need, pool.submit(r.build, self.physics)))

        try:
            while pending or queue or active:
                with _Part("arrivals_s"):
                    arrivals(clock() - t0)
                # admission: FIFO while memory and slots allow
                with _Part("admit_s"):
                    # FIFO while memory and slots allow; a request whose initial field is still
                    # being built waits for it only when nothing else is on the device
                    while queue and len(active) < self.max_active and used + queue[0][1] <= self.hbm_budget:
                        if active and not queue[0][2].done():
                            break
                        r, need, fut = queue.pop(0)
                        cfg, qj = fut.result()
                        s = Solver(cfg, dev)
                        s.set_state(qj)
                        active.append(_Active(r, s, need, r.steps, clock() - t0))
                        used += need
                        dirty = True
                peak_bytes = max(peak_bytes, used)
                peak_active = max(peak_active, len(active))
                if not active:
                    if pending:
                        with _Part("idle_s"):
                            sleep(max(0.0, min(pending[0].arrival - (clock() - t0), 0.05)))
                    continue
                if dirty:
                    with _Part("batch_build_s"):
                        if batch is not None:
                            batch.close()
                        solvers = [a.solver for a in active]
                        batch = Batch(solvers, self._tuning(solvers))
                        dirty = False
                k = min(self.quantum, min(a.remaining for a in active))
                if stream is None:
                    stream = torch.cuda.current_stream(dev)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                with _Part("step_enqueue_s"):
                    e0.record(stream)
                    batch.step(k)                      # asynchronous on the device
                    e1.record(stream)
                steps_run += k
                quanta += 1
                with _Part("arrivals_s"):
                    arrivals(clock() - t0)             # overlaps the quantum
                with _Part("wait_device_s"):
                    stream.synchronize()
                gpu_ms += e0.elapsed_time(e1)
                done_t = clock() - t0
                keep = []
                with _Part("retire_s"):
                    for a in active:
                        a.remaining -= k
                        if a.remaining > 0:
                            keep.append(a)
                            continue
                        st = a.solver.get_state() if self.keep_states else None
                        results.append(SolveResult(a.req.rid, a.req.n, a.req.steps, a.req.arrival, a.admitted, done_t,
                                                   a.solver.diagnostics(), st))
                        a.solver.close()
                        used -= a.bytes
                        dirty = True
                    if dirty and batch is not None:
                        batch.close()
                        batch = None
                active = keep
        finally:
            pool.shutdown(wait=True, cancel_futures=True)
        if batch is not None:
            batch.close()
        wall = time.perf_counter() - wall0
        self.stats = {"batched_steps": steps_run, "quanta": quanta, "wall_s": clock() - t0,
                      "peak_bytes": peak_bytes, "peak_active": peak_active,
                      "split": {"host_wall_s": wall, "device_busy_s": gpu_ms / 1e3,
                                "device_busy_frac": gpu_ms / 1e3 / max(wall, 1e-9)} | split}
        return sorted(results, key=lambda r: r.rid)
