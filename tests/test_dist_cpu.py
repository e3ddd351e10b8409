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


# ---- z slabs (COMMZ) over two gloo ranks, each slab stepped by the oracle ----------
def _slab_cfg(rk, kind="tgv"):
    if kind == "walls":
        # Navier-Stokes over a no-slip floor, zero-gradient x ends and top, periodic z
        from helpers import wall_box
        rules = {"x_lo": "zero_gradient", "x_hi": "zero_gradient", "y_lo": "noslip_wall", "y_hi": "zero_gradient"}
        cfg, qj, _ = wall_box(10, 12, 12, 4, rules, bc_x=1, bc_z=0, scheme="Hybrid", rk=rk, tvd="hybrid")
        return cfg, qj
    from ouxsbli_b200.cases import CASES, build_initial
    from ouxsbli_b200.grid import jacobian, to_qj
    from ouxsbli_b200.solver import SolverConfig
    p = dict(CASES["NSTGV"].params)
    p.update(nx=16, ny=16, nz=16, order=4, M0=0.8, rho_mode="uniform", cfl_mode="acoustic", CFL=0.5, dt=None)
    p, xc, yc, zc, dx, dy, dz, Q = build_initial(CASES["NSTGV"], p)
    cfg = SolverConfig(dim=3, nx=16, ny=16, nz=16, order=4, scheme="Hybrid", visc="NS", visc_order=4, tvd="hybrid",
                       rk=rk, gamma=p["gamma"], R=p["R"], Pr=p["Pr"], dt=p["dt"], dx=dx, dy=dy, dz=dz)
    return cfg, to_qj(Q, jacobian(dx, dy, dz))


def _slab_rank(rank, world, port, rk, nsteps, out, kind="tgv"):
    import datetime
    import torch
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        from oracle import oracle
        from ouxsbli_b200.slabs import halo_exchange, slab_config, slab_state
        cfg, qj = _slab_cfg(rk, kind)
        lcfg, k0 = slab_config(cfg, rank, world)
        st = oracle.Stepper(lcfg, slab_state(qj, cfg, rank, world))
        g, n = cfg.g, lcfg.nz

        def flat(a):
            return torch.from_numpy(np.asfortranarray(a).ravel(order="F").copy())

        for _ in range(nsteps):
            for s in range(st.stages):
                st.stage(s)
                arr = st.written(s)
                send_lo, send_hi = flat(arr[:, :, :, g:2 * g]), flat(arr[:, :, :, n - 2 * g:n - g])
                recv_lo, recv_hi = torch.empty_like(send_lo), torch.empty_like(send_hi)
                halo_exchange(send_lo, send_hi, recv_lo, recv_hi, rank, world)
                shp = arr[:, :, :, :g].shape
                arr[:, :, :, :g] = recv_lo.numpy().reshape(shp, order="F")
                arr[:, :, :, n - g:] = recv_hi.numpy().reshape(shp, order="F")
        out[rank] = st.q
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("rk,kind", [(3, "tgv"), (4, "tgv"), (3, "walls")])
def test_two_gloo_ranks_z_slabs_match_the_global_oracle(rk, kind):
    """The halo exchange of the z-slab decomposition (which array after which stage,
    which planes go to which neighbour, the slab's z spacings): two ranks stepping
    their slabs stage by stage reproduce the undivided solve bit for bit, on a periodic
    grid and on a walled Navier-Stokes one."""
    from oracle import oracle
    cfg, qj = _slab_cfg(rk, kind)
    nsteps = 2
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_slab_rank, args=(2, _free_port(), rk, nsteps, out, kind), nprocs=2, join=True,
                           start_method="spawn")
        parts = [out[0], out[1]]
    g = cfg.g
    whole = oracle.step(cfg, qj, nsteps)
    glued = np.concatenate([parts[0][:, :, :, g:-g], parts[1][:, :, :, g:-g]], axis=3)
    np.testing.assert_array_equal(glued, whole[:, :, :, g:-g])


def test_slab_bounds_and_configs():
    from ouxsbli_b200.slabs import slab_bounds, slab_config
    cfg, _ = _slab_cfg(3)
    assert slab_bounds(16, 2, 0, 2) == (0, 10) and slab_bounds(16, 2, 1, 2) == (6, 10)
    with pytest.raises(ValueError):
        slab_bounds(16, 2, 0, 5)   # 12 planes over 5 ranks
    with pytest.raises(ValueError):
        slab_bounds(16, 2, 0, 12)  # 1-plane slabs, thinner than the halo
    lcfg, k0 = slab_config(cfg, 1, 2)
    assert lcfg.nz == 10 and lcfg.bc_z == 2 and k0 == 6 and lcfg.dz.size == 9
    np.testing.assert_array_equal(lcfg.dz, np.asarray(cfg.dz)[6:15])
