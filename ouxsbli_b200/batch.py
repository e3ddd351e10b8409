"""Batched solves: many independent periodic solves (uneven grids) advanced by one
persistent kernel launch per time step, replayed as one CUDA graph per step.

`Batch` wraps liboux's oux_batch_* entry points around a list of bound `Solver`s.
`Autotuner` picks the work-item shape (sweep tiles per item, cells per point-wise
item, resident blocks per SM) by timing candidates on the actual batch, and caches
the choice per (dimension, scheme, order, viscous model, precision, RK, size class)
in a JSON file, so a later batch of the same kind starts tuned.
"""
from __future__ import annotations

import ctypes as C
import json
import math
import os
import pathlib
from dataclasses import asdict, dataclass
from typing import Callable, Sequence

import torch

from ._lib import BATCH_MODES, LIB, OuxBatchTuning, check
from .solver import Solver

BATCH_THREADS = 288  # threads per block of the persistent kernel (csrc/oux_batch.cuh)


@dataclass(frozen=True)
class Tuning:
    pencil: int = 4                 # sweep tiles per work item (consecutive along the sweep)
    chunk: int = 4 * BATCH_THREADS  # cells per point-wise work item
    blocks_per_sm: int = 0          # persistent blocks per SM; 0 = as many as fit
    use_graph: bool = True          # replay one captured CUDA graph per step
    # "persistent": one persistent kernel per step over the tile work list;
    # "graph": one CUDA graph per step with every solve's own stage kernels on a
    # branch of their own (the work-list fields do not apply)
    mode: str = "persistent"

    def to_c(self) -> OuxBatchTuning:
        t = OuxBatchTuning()
        t.pencil, t.chunk, t.blocks_per_sm = self.pencil, self.chunk, self.blocks_per_sm
        t.use_graph = int(self.use_graph)
        t.mode = BATCH_MODES[self.mode]
        return t


class Batch:
    """One persistent-kernel time step for every member solve.

    Members must share dim, order, viscous stencil, LES, precision and RK; grids,
    schemes and physical constants may differ.  In FP64 each member ends every step
    with exactly the state its own `Solver.step` would give.  Set the members'
    states before creating the batch (the mixed form's references are taken then).
    """

    def __init__(self, solvers: Sequence[Solver], tuning: Tuning | None = None):
        if not solvers:
            raise ValueError("a batch needs at least one solve")
        dev = solvers[0].device
        if any(s.device != dev for s in solvers):
            raise ValueError("all solves of a batch must live on one device")
        self.solvers = list(solvers)
        self.device = dev
        self.tuning = tuning or Tuning()
        hs = (C.c_void_p * len(solvers))(*[s._h.value for s in solvers])
        t = self.tuning.to_c()
        b = C.c_void_p()
        check(LIB.oux_batch_create(hs, len(solvers), C.byref(t), C.byref(b)))
        self._b = b
        nb = C.c_size_t()
        check(LIB.oux_batch_workspace_bytes(self._b, C.byref(nb)))
        self.workspace = torch.empty(max(nb.value, 256), dtype=torch.uint8, device=dev)
        with torch.cuda.device(dev):
            check(LIB.oux_batch_bind(self._b, C.c_void_p(self.workspace.data_ptr()), C.c_size_t(nb.value),
                                     C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)))

    def step(self, nsteps: int = 1) -> None:
        with torch.cuda.device(self.device):
            st = torch.cuda.current_stream(self.device)
            check(LIB.oux_batch_step(self._b, int(nsteps), C.c_void_p(st.cuda_stream)))

    def status(self) -> int:
        v = C.c_int32()
        with torch.cuda.device(self.device):
            check(LIB.oux_batch_status(self._b, C.byref(v)))
        return v.value

    def set_spin_limit(self, polls: int) -> None:
        """Polls a dependency wait makes before it gives up with OUX_FAULT_TIMEOUT."""
        check(LIB.oux_batch_set_spin_limit(self._b, int(polls)))

    def dep_offset(self, member: int, phase: int) -> int:
        """Byte offset in `workspace` of the (phase waited for, count) int32 pair of
        (member, phase) -- for tests that make a wait run out."""
        off = C.c_size_t()
        check(LIB.oux_batch_dep_offset(self._b, int(member), int(phase), C.byref(off)))
        return off.value

    def info(self) -> dict:
        items, phases, grid = C.c_int64(), C.c_int32(), C.c_int32()
        check(LIB.oux_batch_info(self._b, C.byref(items), C.byref(phases), C.byref(grid)))
        return {"items": items.value, "phases": phases.value, "grid": grid.value}

    def interior_cells(self) -> int:
        return sum(s.cfg.interior_cells() for s in self.solvers)

    def close(self) -> None:
        if getattr(self, "_b", None) is not None and self._b.value:
            LIB.oux_batch_destroy(self._b)
            self._b = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------- autotuner --
CANDIDATES = tuple(Tuning(pencil=p, chunk=c * BATCH_THREADS, blocks_per_sm=b)
                   for p in (1, 2, 4, 8) for c in (2, 4, 8) for b in (0, 1)) + (Tuning(mode="graph"),)


def size_class(total_interior_cells: int) -> int:
    """log2 bucket of the batch's total interior cells."""
    return int(round(math.log2(max(total_interior_cells, 1))))


def tuning_key(solvers: Sequence) -> str:
    c = solvers[0].cfg
    schemes = sorted({s.cfg.scheme for s in solvers})
    scheme = schemes[0] if len(schemes) == 1 else "+".join(schemes)
    visc = c.visc if c.visc == "Euler" or c.dim == 2 else f"{c.visc}-{c.visc_stencil}-{c.visc_order or c.order}"
    cells = sum(s.cfg.interior_cells() for s in solvers)
    return f"{c.dim}d/{scheme}/o{c.order}/{visc}/{c.precision}/rk{c.rk}/2^{size_class(cells)}"


def default_cache_path() -> pathlib.Path:
    env = os.environ.get("OUX_TUNE_CACHE")
    if env:
        return pathlib.Path(env)
    return pathlib.Path.home() / ".cache" / "ouxsbli_b200" / "batch_tuning.json"


def _event_timer(batch: Batch, steps: int) -> float:
    """Device milliseconds per step of `steps` batched steps (CUDA events on the batch's stream)."""
    st = torch.cuda.current_stream(batch.device)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(st)
    batch.step(steps)
    b.record(st)
    b.synchronize()
    return a.elapsed_time(b) / steps


class Autotuner:
    """Times candidate tunings on a batch and caches the fastest per tuning key."""

    def __init__(self, path: str | os.PathLike | None = None):
        self.path = pathlib.Path(path) if path is not None else default_cache_path()
        self.cache: dict[str, dict] = {}
        if self.path.exists():
            try:
                self.cache = json.loads(self.path.read_text())
            except (OSError, ValueError):
                self.cache = {}

    def lookup(self, key: str) -> Tuning | None:
        e = self.cache.get(key)
        return Tuning(**e["tuning"]) if e else None

    def lookup_nearest(self, key: str) -> Tuning | None:
        """The cached tuning of `key`, else that of the nearest size class with the
        same dimension, scheme, order, viscous model, precision and RK."""
        hit = self.lookup(key)
        if hit is not None:
            return hit
        stem, _, cls = key.rpartition("/2^")
        best = None
        for k, e in self.cache.items():
            s2, _, c2 = k.rpartition("/2^")
            if s2 == stem:
                d = abs(int(c2) - int(cls))
                if best is None or d < best[0]:
                    best = (d, e)
        return Tuning(**best[1]["tuning"]) if best else None

    def save(self) -> None:
        self.path.parent.mkdir(parents=True, exist_ok=True)
        tmp = self.path.with_suffix(".tmp")
        tmp.write_text(json.dumps(self.cache, indent=1, sort_keys=True))
        tmp.replace(self.path)

    def tune(self, solvers: Sequence[Solver], steps: int = 3, candidates: Sequence[Tuning] = CANDIDATES,
             timer: Callable[[Batch, int], float] = _event_timer, force: bool = False) -> Tuning:
        """Best tuning for this batch (cached per key).  The members' states are
        restored after every trial, so tuning leaves the solves where they were."""
        key = tuning_key(solvers)
        if not force:
            hit = self.lookup(key)
            if hit is not None:
                return hit
        if not candidates:
            raise ValueError(f"no cached tuning for {key} and no candidates to time")
        saved = [s.state.clone() for s in solvers]
        results = []
        try:
            for cand in candidates:
                b = Batch(solvers, cand)
                try:
                    b.step(1)  # warm-up (graph capture)
                    ms = timer(b, steps)
                finally:
                    b.close()
                    for s, q in zip(solvers, saved):
                        s.state.copy_(q)
                results.append((ms, cand))
        finally:
            for s, q in zip(solvers, saved):
                s.state.copy_(q)
        ms, best = min(results, key=lambda r: r[0])
        self.cache[key] = {"tuning": asdict(best), "ms_per_step": ms,
                           "trials": [[m, asdict(c)] for m, c in results]}
        self.save()
        return best


def _main(argv=None) -> int:
    """Run the seeded 2D vortex ensemble as one batch (a driver for profiling):

        python -m ouxsbli_b200.batch [--count 64] [--seed 0] [--steps 5] [--precision fp64]
                                     [--pencil 8] [--chunk 2304] [--mode persistent|graph]
    """
    import argparse
    from .cases import vortex_ensemble, vortex_member
    ap = argparse.ArgumentParser(prog="python -m ouxsbli_b200.batch")
    ap.add_argument("--count", type=int, default=64)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--pencil", type=int, default=8)
    ap.add_argument("--chunk", type=int, default=8 * BATCH_THREADS)
    ap.add_argument("--mode", default="persistent", choices=["persistent", "graph"])
    a = ap.parse_args(argv)
    dev = torch.device("cuda:0")
    solvers = []
    for m in vortex_ensemble(a.count, a.seed):
        cfg, qj = vortex_member(m, order=4, scheme="KEEP", visc="Euler", rk=4, precision=a.precision)
        s = Solver(cfg, dev)
        s.set_state(qj)
        solvers.append(s)
    b = Batch(solvers, Tuning(pencil=a.pencil, chunk=a.chunk, mode=a.mode))
    ms = _event_timer(b, a.steps)
    st = b.status()
    print(json.dumps({"solves": a.count, "interior_cells": b.interior_cells(), "ms_per_step": ms,
                      "status": st, **b.info()}))
    b.close()
    return 0 if st == 0 else 1


if __name__ == "__main__":
    raise SystemExit(_main())
