"""oux_rhs_noalloc, the allocation-free stage residual, against oux_rhs through the C ABI.

Both entry points run the same FP64 kernels with the same arithmetic (the metric
tables are expanded on the device with the host's order of operations), so the
tolerance is the FP64 parity tests' one: bit-for-bit equality.  The fixed scratch
array keeps the previous call's contents, so the checks run several calls in a row,
on two different grids.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from helpers import tgv, vortex2d
from ouxsbli_b200 import _lib
from ouxsbli_b200.solver import Solver, SolverConfig


def _rhs_len(cfg):
    return cfg.nv * (cfg.nx - 2) * (cfg.ny - 2) * ((cfg.nz - 2) if cfg.dim == 3 else 1)


def rhs_handle(s: Solver) -> np.ndarray:
    """The existing entry point: oux_rhs on a bound handle."""
    out = torch.zeros(_rhs_len(s.cfg), dtype=torch.float64, device=s.device)
    with torch.cuda.device(s.device):
        st = torch.cuda.current_stream(s.device)
        _lib.check(_lib.LIB.oux_rhs(s._h, C.c_void_p(out.data_ptr()), C.c_void_p(st.cuda_stream)))
        st.synchronize()
    return out.cpu().numpy()


def rhs_noalloc(cfg, state: torch.Tensor, device) -> np.ndarray:
    """The allocation-free entry point on the same device state; the output starts as NaN
    so that the call's own clearing of the ghost entries is checked too."""
    c, keep = cfg.to_c()
    out = torch.full((_rhs_len(cfg),), float("nan"), dtype=torch.float64, device=device)
    with torch.cuda.device(device):
        st = torch.cuda.current_stream(device)
        _lib.check(_lib.LIB.oux_rhs_noalloc(C.byref(c), C.c_void_p(state.data_ptr()),
                                            C.c_void_p(out.data_ptr()), C.c_void_p(st.cuda_stream)))
        st.synchronize()
    del keep
    return out.cpu().numpy()


@pytest.mark.gpu
def test_noalloc_matches_rhs_on_calls_in_a_row(cuda_device):
    cases = [
        tgv(16, mach=1.25, scheme="Hybrid", visc="NS"),
        vortex2d(32, order=4, scheme="KEEP", visc="Euler", rk=4),
    ]
    for cfg, qj in cases:
        s = Solver(cfg, cuda_device)
        s.set_state(qj)
        ref = rhs_handle(s)
        assert np.isfinite(ref).all() and np.abs(ref).max() > 0
        for _ in range(2):
            got = rhs_noalloc(cfg, s.state, cuda_device)
            np.testing.assert_array_equal(got, ref)
        s.close()


@pytest.mark.gpu
def test_noalloc_matches_rhs_on_stretched_and_walled_grids(cuda_device):
    """Metric tables built on the device against the host's build_tables where the
    spacings vary along every axis, and a 2D Navier-Stokes grid with no-slip walls in
    y (boundary cells filled by the handle first; both calls read the same state)."""
    import dataclasses
    cfg, qj = tgv(16, mach=1.25, scheme="Hybrid", visc="NS", visc_stencil="ME4Base")
    def stretch(d, a):
        return d * (1.0 + a * np.sin(np.linspace(0.0, 2.0 * np.pi, d.size)))
    cfg = dataclasses.replace(cfg, dx=stretch(cfg.dx, 0.10), dy=stretch(cfg.dy, 0.07), dz=stretch(cfg.dz, 0.05))
    wcfg, wqj = vortex2d(24, order=4, scheme="SLAU", visc="NS", rk=3, mach=0.3)
    wcfg = dataclasses.replace(wcfg, ny=wcfg.ny - 2, dy=wcfg.dy[:-2], bc_y=1,
                               boundary={"y_lo": "noslip_wall", "y_hi": "slip_wall"})
    wqj = np.asfortranarray(wqj[:, :, 1:-1])
    for c, q in ((cfg, qj), (wcfg, wqj)):
        s = Solver(c, cuda_device)
        s.set_state(q)
        s.fill_ghosts()
        ref = rhs_handle(s)
        assert np.isfinite(ref).all() and np.abs(ref).max() > 0
        for _ in range(2):
            np.testing.assert_array_equal(rhs_noalloc(c, s.state, cuda_device), ref)
        s.close()


def _cfg(n, **kw):
    d = np.full(n - 1, 0.1)
    base = dict(dim=3, nx=n, ny=n, nz=n, order=6, dx=d, dy=d, dz=d, dt=1e-4)
    base.update(kw)
    return SolverConfig(**base)


def _call_without_device(cfg):
    # the size and precision checks return before any CUDA call, so a placeholder
    # (aligned, never dereferenced) pointer is enough on a machine without a GPU
    c, keep = cfg.to_c()
    rc = _lib.LIB.oux_rhs_noalloc(C.byref(c), C.c_void_p(1 << 20), C.c_void_p(1 << 20), None)
    del keep
    return rc, _lib.LIB.oux_last_error().decode()


def test_noalloc_rejects_grids_beyond_the_fixed_scratch():
    c, keep = _cfg(72).to_c()
    need = C.c_size_t()
    _lib.check(_lib.LIB.oux_scratch_bytes(C.byref(c), C.byref(need)))
    assert need.value > _lib.NOALLOC_SCRATCH_BYTES
    rc, msg = _call_without_device(_cfg(72))
    assert rc == _lib.OUX_E_TOO_SMALL
    assert str(need.value) in msg and str(_lib.NOALLOC_SCRATCH_BYTES) in msg


def test_noalloc_rejects_mixed_precision():
    rc, msg = _call_without_device(_cfg(16, precision="mixed"))
    assert rc == _lib.OUX_E_INVALID and "FP64" in msg


def test_noalloc_rejects_les_with_walls():
    # no handle means no boundary rules: the SGS viscosity of wall cells would differ
    rc, msg = _call_without_device(_cfg(16, visc="LES", bc_y=1))
    assert rc == _lib.OUX_E_INVALID and "LES" in msg
