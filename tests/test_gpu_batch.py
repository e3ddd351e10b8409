"""Batched solves (one persistent kernel per step over many uneven grids) against the
same solves run one at a time through oux_step.

Every member computes the same operations in the same order as its single-solve
run (FP64 units without FMA contraction), so FP64 members must agree bit for bit.
Mixed-form members evaluate the same FP32 expressions, but the compiler may
contract multiply-adds differently in the two kernels, and in the LES model those
rounding differences flip discrete switches: mixed LES members are held to the
mixed form's own LES bound against FP64, a relative L2 of 1e-2 per variable.
"""
import dataclasses

import numpy as np
import pytest

from helpers import random_turbulence, tgv, vortex2d
from ouxsbli_b200.batch import Autotuner, Batch, Tuning
from ouxsbli_b200.solver import Solver

pytestmark = pytest.mark.gpu


def singles(cases, nsteps, device):
    out = []
    for cfg, qj in cases:
        s = Solver(cfg, device)
        s.set_state(qj)
        s.step(nsteps)
        out.append(s.get_state())
        s.close()
    return out


def batched(cases, nsteps, device, tuning=None):
    solvers = []
    for cfg, qj in cases:
        s = Solver(cfg, device)
        s.set_state(qj)
        solvers.append(s)
    b = Batch(solvers, tuning)
    b.step(nsteps)
    assert b.status() == 0
    out = [s.get_state() for s in solvers]
    b.close()
    for s in solvers:
        s.close()
    return out


def vortex_ensemble():
    # uneven, non-multiple-of-tile sizes; per-member strength, Mach and dt
    spec = [(20, 1.0, 0.1), (36, 3.0, 0.5), (64, 5.0, 0.8), (45, 2.0, 0.3)]
    return [vortex2d(n, order=4, beta=b, mach=m, scheme="KEEP", visc="Euler", rk=4) for n, b, m in spec]


def test_batch_2d_keep4_rk4_bitexact(cuda_device):
    cases = vortex_ensemble()
    for x, y in zip(singles(cases, 7, cuda_device), batched(cases, 7, cuda_device)):
        np.testing.assert_array_equal(x, y)


def test_batch_3d_hybrid_ns_bitexact(cuda_device):
    cases = [tgv(12, mach=1.25, scheme="Hybrid", visc="NS"), tgv(17, mach=0.5, scheme="SLAU", visc="NS"),
             tgv(20, mach=0.8, scheme="KEEP", visc="NS")]
    for x, y in zip(singles(cases, 3, cuda_device), batched(cases, 3, cuda_device)):
        np.testing.assert_array_equal(x, y)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_3d_les_slau6(precision, cuda_device):
    cases = [random_turbulence(n, seed=s, scheme="SLAU", visc="LES", precision=precision)
             for n, s in ((12, 1), (16, 2))]
    for x, y in zip(singles(cases, 3, cuda_device), batched(cases, 3, cuda_device)):
        if precision == "fp64":
            # the SMS model's pow/log/cosh are the same device functions in both paths
            np.testing.assert_array_equal(x, y)
        else:
            # FP32 rounding differences flip the model's discrete switches (HRSLAU2
            # wiggle detector, TVD threshold, the SMS limiter): the same bound as the
            # mixed form against FP64 for LES
            for l in range(5):
                d = np.linalg.norm(x[:, l] - y[:, l]) / np.linalg.norm(y[:, l])
                assert d <= 1e-2, (l, d)


def test_batch_tunings_and_graph_agree(cuda_device):
    cases = vortex_ensemble()[:3]
    ref = batched(cases, 4, cuda_device, Tuning(pencil=1, chunk=288, blocks_per_sm=1, use_graph=False))
    for t in (Tuning(pencil=8, chunk=2304, blocks_per_sm=0, use_graph=True), Tuning(pencil=3, chunk=1000)):
        for x, y in zip(ref, batched(cases, 4, cuda_device, t)):
            np.testing.assert_array_equal(x, y)


def test_batch_mixed_2d_close_to_fp64(cuda_device):
    cases = vortex_ensemble()
    a = batched(cases, 50, cuda_device)
    b = batched([(dataclasses.replace(c, precision="mixed"), q) for c, q in cases], 50, cuda_device)
    for x, y, (cfg, _) in zip(a, b, cases):
        g = cfg.g
        xi, yi = x[g:-g, :, g:-g], y[g:-g, :, g:-g]
        err = np.linalg.norm(xi - yi) / np.linalg.norm(xi)
        assert err < 1e-5, err


def test_autotuner_caches_choice(tmp_path, cuda_device):
    cases = vortex_ensemble()[:2]
    solvers = []
    for cfg, qj in cases:
        s = Solver(cfg, cuda_device)
        s.set_state(qj)
        solvers.append(s)
    before = [s.get_state() for s in solvers]
    cands = (Tuning(pencil=1, chunk=576), Tuning(pencil=4, chunk=1152))
    tuner = Autotuner(tmp_path / "tune.json")
    best = tuner.tune(solvers, steps=2, candidates=cands)
    assert best in cands
    for s, q in zip(solvers, before):  # states untouched by the trials
        np.testing.assert_array_equal(s.get_state(), q)
    again = Autotuner(tmp_path / "tune.json")
    assert again.lookup(next(iter(again.cache))) == best
    assert again.tune(solvers, candidates=()) == best  # served from the cache
    for s in solvers:
        s.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_graph_mode_bitexact(precision, cuda_device):
    """Graph mode runs every member's own stage kernels on a graph branch: bit for bit
    the single-solve result, in the mixed form too."""
    cases = [random_turbulence(n, seed=s, scheme="SLAU", visc="LES", precision=precision)
             for n, s in ((12, 1), (16, 2), (14, 3))]
    ref = singles(cases, 4, cuda_device)
    got = batched(cases, 4, cuda_device, Tuning(mode="graph"))
    for x, y in zip(ref, got):
        np.testing.assert_array_equal(x, y)
    cases2 = vortex_ensemble()
    for x, y in zip(singles(cases2, 5, cuda_device), batched(cases2, 5, cuda_device, Tuning(mode="graph"))):
        np.testing.assert_array_equal(x, y)


def test_batch_dependency_wait_runs_out(cuda_device):
    """A dependency count that the work list can never reach, planted in the bound
    workspace from the host, makes every wait on it run out after the batch's spin
    limit: the kernel sets OUX_FAULT_TIMEOUT in the batch status word and its blocks
    return (no trap, no hang), and the device stays usable for the next batch."""
    import torch
    from ouxsbli_b200 import _lib
    cases = vortex_ensemble()[:2]
    solvers = []
    for cfg, qj in cases:
        s = Solver(cfg, cuda_device)
        s.set_state(qj)
        solvers.append(s)
    b = Batch(solvers, Tuning())
    b.set_spin_limit(64)
    # phase 1 of member 0 (its first x sweep) waits for all items of phase 0 (primitives)
    off = b.dep_offset(0, 1)
    dep = b.workspace[off:off + 8].view(torch.int32)
    assert int(dep[0]) == 0 and int(dep[1]) > 0
    dep[1] = 1 << 30
    b.step(1)
    torch.cuda.synchronize(cuda_device)
    assert b.status() & _lib.FAULT_TIMEOUT
    b.close()
    for s in solvers:
        s.close()
    # a fresh batch on the same device steps cleanly and matches the single solves
    want = singles(cases, 2, cuda_device)
    got = batched(cases, 2, cuda_device)
    for x, y in zip(want, got):
        np.testing.assert_array_equal(x, y)
