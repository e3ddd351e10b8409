"""The plain-method workload at full size against the oracle: viscous Taylor-Green
vortex on a periodic [0, 2 pi)^3 grid of 64^3 cells, FP64, SLAU (HRSLAU2, TVD
hybrid), 6th-order central differences, Central-6 viscous fluxes, TVD-RK3,
Re 1600, Ma 0.1, uniform rho, acoustic CFL 0.5, 100 steps.

Checked every 10 steps: the conservative fields (tolerance stated by the north
star: relative L2 <= 1e-9 per variable; the FP64 path is bit-identical) and the
kinetic-energy, entropy and enstrophy histories (device FP64 reductions against
numpy on the oracle's state: relative 1e-12, enstrophy 1e-10).
"""
import numpy as np
import pytest

from helpers import diagnostics_numpy, interior, rel_l2, tgv
from oracle import oracle

pytestmark = pytest.mark.gpu


def test_plain_method_64cubed_100_steps_with_histories(cuda_device):
    from ouxsbli_b200.solver import Solver
    cfg, qj = tgv(64, mach=0.1, scheme="SLAU", visc="NS", slau="HRSLAU2", tvd="hybrid")
    assert cfg.nx == 70 and cfg.rk == 3 and cfg.order == 6
    s = Solver(cfg, cuda_device)
    s.set_state(qj)
    q_orc = qj
    hist_gpu, hist_ref = [], []
    for _ in range(10):
        s.step(10)
        q_orc = oracle.step(cfg, q_orc, 10)
        q_gpu = s.get_state()
        a, b = interior(q_gpu, cfg.g, 3), interior(q_orc, cfg.g, 3)
        for l in range(5):
            assert rel_l2(a[:, l], b[:, l]) <= 1e-9
        assert np.array_equal(q_gpu, q_orc)
        hist_gpu.append(s.diagnostics())
        hist_ref.append(diagnostics_numpy(cfg, q_orc))
    s.close()
    for (ke, ent, ens), (ke0, ent0, ens0) in zip(hist_gpu, hist_ref):
        assert abs(ke - ke0) <= 1e-12 * abs(ke0)
        assert abs(ent - ent0) <= 1e-12 * abs(ent0)
        assert abs(ens - ens0) <= 1e-10 * abs(ens0)
    # the viscous TGV decays: kinetic energy falls monotonically over the 100 steps
    kes = [h[0] for h in hist_gpu]
    assert all(x > y for x, y in zip(kes, kes[1:]))
