"""Serving loop on the GPU: each result is bit-for-bit the same alone and in a mix
(tolerance 0: a solve's arithmetic does not depend on its batch companions), and
admission keeps the resident solves within the memory budget."""
import numpy as np
import pytest

from ouxsbli_b200.serving import Server, SolveRequest, poisson_stream, request_bytes, summarize

pytestmark = pytest.mark.gpu

PHYS = dict(order=6, scheme="SLAU", visc="LES", rk=3, precision="mixed")


class FakeClock:
    """Deterministic time: 10 ms per reading, plus whatever the server sleeps."""

    def __init__(self):
        self.t = 0.0

    def __call__(self):
        self.t += 0.01
        return self.t

    def sleep(self, d):
        self.t += max(d, 1e-3)


def serve(reqs, budget, quantum=10):
    clk = FakeClock()
    srv = Server(device="cuda:0", hbm_budget=budget, quantum=quantum, physics=PHYS, keep_states=True)
    res = srv.run(reqs, clock=clk, sleep=clk.sleep)
    return {r.rid: r for r in res}, srv.stats


def test_same_result_alone_and_in_mix(cuda_device):
    r = SolveRequest(rid=0, n=16, steps=37, seed=5)
    a = SolveRequest(rid=1, n=12, steps=15, seed=6)
    b = SolveRequest(rid=2, n=20, steps=25, seed=7)
    c = SolveRequest(rid=3, n=14, steps=30, seed=8, arrival=0.03)  # arrives while others run
    nbytes = {q.rid: request_bytes(q.build(PHYS)[0]) for q in (r, a, b, c)}
    # room for r + a but not b until a retires: b joins r mid-run; c joins b once r is done
    budget = nbytes[0] + nbytes[2] + 1
    mix, stats = serve([r, a, b, c], budget)
    assert stats["peak_bytes"] <= budget
    assert mix[2].admitted > mix[0].admitted  # b waited for memory
    for q in (r, a, b, c):
        alone, _ = serve([SolveRequest(q.rid, q.n, q.steps, q.seed)], budget=1 << 34)
        np.testing.assert_array_equal(alone[q.rid].state, mix[q.rid].state)
        assert np.isfinite(mix[q.rid].state).all()


def test_poisson_stream_summary(cuda_device):
    reqs = poisson_stream(6, rate=50.0, seed=3, sizes=(12, 16), steps=(10, 30))
    res, stats = serve(reqs, budget=1 << 33, quantum=8)
    s = summarize(list(res.values()))
    assert s["requests"] == 6 and s["p99_s"] >= s["p50_s"] >= 0.0
    assert stats["peak_active"] >= 2  # solves overlapped on the device
