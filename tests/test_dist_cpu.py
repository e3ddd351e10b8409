"""The N > 1 replica path on CPU: two `gloo` ranks (one process each).

The solve does not shard across GPUs -- N processes run independent replicas -- so
the multi-process surface is the timing reduction: every rank contributes its device
time, the slowest one defines the whole-job rate, and the rate counts the units of
all ranks.  Each rank here also runs its own replica (the oracle, a 2D vortex
ensemble member) to show the replicas need no exchange: identical inputs give
identical states on every rank.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from ouxsbli_b200.replicas import job_rate, max_over_ranks, world as world_of
        assert world_of() == (rank, world)
        local_ms = [10.0, 25.0][rank]
        mx = max_over_ranks(local_ms)
        rate, ms = job_rate(1000.0, local_ms)
        # one replica per rank: a small 2D inviscid case through the oracle
        from oracle import oracle
        from ouxsbli_b200.cases import vortex_ensemble, vortex_member
        cfg, qj = vortex_member(vortex_ensemble(1, seed=7, sizes=(24,))[0], order=4, visc="Euler")
        q = oracle.step(cfg, qj, 2)
        digest = torch.tensor([float(np.sum(q * np.arange(q.size).reshape(q.shape) % 97))], dtype=torch.float64)
        gathered = [torch.zeros(1, dtype=torch.float64) for _ in range(world)]
        dist.all_gather(gathered, digest)
        out[rank] = (mx, rate, ms, [float(g.item()) for g in gathered])
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_max_over_ranks_and_independent_replicas():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_rank_main, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
        res = dict(out)
    assert set(res) == {0, 1}
    for r in (0, 1):
        mx, rate, ms, digests = res[r]
        assert mx == 25.0 and ms == 25.0
        # whole-job rate: 2 ranks x 1000 units in the slowest rank's 25 ms
        assert rate == pytest.approx(2 * 1000.0 / 0.025)
        assert digests[0] == digests[1]


def test_single_process_without_group():
    from ouxsbli_b200.replicas import job_rate, max_over_ranks, world
    assert world() == (0, 1)
    assert max_over_ranks(3.5) == 3.5
    assert job_rate(500.0, 2.0) == (pytest.approx(250000.0), 2.0)
