"""Batch-layer and serving host logic that needs no GPU: member checks, tuning
validation, tuning keys, the autotuner's cache file, request streams and the
memory-budget check."""
import ctypes as C
import json
import types

import numpy as np
import pytest

from ouxsbli_b200 import _lib
from ouxsbli_b200.batch import Autotuner, Tuning, size_class, tuning_key
from ouxsbli_b200.solver import SolverConfig


def _handle(**kw):
    n = kw.pop("n", 16)
    d = np.full(n - 1, 0.1)
    base = dict(dim=3, nx=n, ny=n, nz=n, order=6, dx=d, dy=d, dz=d, dt=1e-4)
    base.update(kw)
    c, keep = SolverConfig(**base).to_c()
    h = C.c_void_p()
    assert _lib.LIB.oux_create(C.byref(c), C.byref(h)) == 0
    return h


def test_batch_rejects_unbound_members():
    h = _handle()
    arr = (C.c_void_p * 1)(h.value)
    out = C.c_void_p()
    rc = _lib.LIB.oux_batch_create(arr, 1, None, C.byref(out))
    assert rc == _lib.OUX_E_UNBOUND
    assert b"no device buffers" in _lib.LIB.oux_last_error()
    _lib.LIB.oux_destroy(h)


def test_batch_rejects_bad_tuning_and_empty():
    h = _handle()
    arr = (C.c_void_p * 1)(h.value)
    out = C.c_void_p()
    t = Tuning(pencil=0).to_c()
    assert _lib.LIB.oux_batch_create(arr, 1, C.byref(t), C.byref(out)) == _lib.OUX_E_INVALID
    assert _lib.LIB.oux_batch_create(arr, 0, None, C.byref(out)) == _lib.OUX_E_INVALID
    _lib.LIB.oux_destroy(h)


def _fake(dim=2, scheme="KEEP", order=4, n=64, precision="fp64", rk=4, visc="Euler"):
    cfg = SolverConfig(dim=dim, nx=n + order, ny=n + order, nz=1 if dim == 2 else n + order, order=order,
                       scheme=scheme, visc=visc, precision=precision, rk=rk)
    return types.SimpleNamespace(cfg=cfg)


def test_tuning_key_and_size_class():
    assert size_class(64 * 64) == 12 and size_class(1) == 0
    assert tuning_key([_fake(n=64), _fake(n=64)]) == "2d/KEEP/o4/Euler/fp64/rk4/2^13"
    assert "/KEEP+SLAU/" in tuning_key([_fake(scheme="KEEP"), _fake(scheme="SLAU")])
    k3 = tuning_key([_fake(dim=3, order=6, scheme="SLAU", visc="LES", precision="mixed", rk=3, n=32)])
    assert k3 == "3d/SLAU/o6/LES-Central-6/mixed/rk3/2^15"


def test_autotuner_cache_roundtrip(tmp_path):
    p = tmp_path / "sub" / "tune.json"
    t = Autotuner(p)
    assert t.lookup("x") is None
    t.cache["x"] = {"tuning": {"pencil": 2, "chunk": 576, "blocks_per_sm": 1, "use_graph": True},
                    "ms_per_step": 1.0, "trials": []}
    t.save()
    assert json.loads(p.read_text())["x"]["tuning"]["pencil"] == 2
    assert Autotuner(p).lookup("x") == Tuning(2, 576, 1, True)
    p.write_text("not json")
    assert Autotuner(p).cache == {}
    with pytest.raises(ValueError):
        Autotuner(p).tune([_fake()], candidates=())


def test_poisson_stream_is_seeded():
    from ouxsbli_b200.serving import poisson_stream
    a = poisson_stream(20, rate=2.0, seed=1)
    b = poisson_stream(20, rate=2.0, seed=1)
    assert [(r.n, r.steps, r.seed, r.arrival) for r in a] == [(r.n, r.steps, r.seed, r.arrival) for r in b]
    assert all(200 <= r.steps <= 2000 and r.n in (32, 48, 64, 96, 128) for r in a)
    assert all(x.arrival < y.arrival for x, y in zip(a, a[1:]))


def test_server_rejects_request_over_budget():
    from ouxsbli_b200.serving import Server, SolveRequest
    srv = Server(device="cuda:0", hbm_budget=1 << 20)
    with pytest.raises(ValueError, match="more than the budget"):
        srv.run([SolveRequest(rid=0, n=16, steps=5, seed=1)])


def test_vortex_ensemble_is_seeded():
    from ouxsbli_b200.cases import VORTEX_SIZES, vortex_ensemble
    a, b = vortex_ensemble(64, seed=0), vortex_ensemble(64, seed=0)
    assert a == b and len(a) == 64
    assert all(m.n in VORTEX_SIZES and 1.0 <= m.beta <= 5.0 and 0.1 <= m.mach <= 0.8 for m in a)


def test_autotuner_nearest_size_class(tmp_path):
    t = Autotuner(tmp_path / "t.json")
    t.cache["3d/SLAU/o6/LES-Central-6/mixed/rk3/2^20"] = {"tuning": {"mode": "graph"}}
    t.cache["3d/SLAU/o6/LES-Central-6/mixed/rk3/2^12"] = {"tuning": {"pencil": 1}}
    t.cache["2d/KEEP/o4/Euler/fp64/rk4/2^21"] = {"tuning": {"pencil": 8}}
    assert t.lookup_nearest("3d/SLAU/o6/LES-Central-6/mixed/rk3/2^19") == Tuning(mode="graph")
    assert t.lookup_nearest("3d/SLAU/o6/LES-Central-6/mixed/rk3/2^13") == Tuning(pencil=1)
    assert t.lookup_nearest("3d/KEEP/o6/NS-Central-6/fp64/rk3/2^20") is None
    assert Tuning(mode="graph").to_c().mode == 1
