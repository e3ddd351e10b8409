"""Mixed form (FP32 stage states and face fluxes, FP64 Q^n, flux differences and
RK combinations) against the FP64 path on the GPU.

Tolerances: the north star's bound for the mixed form is relative L2 <= 1e-5
against FP64 after 1000 steps; these shorter runs hold the same bound where the
scheme allows it (see CASES), and every field stays finite.  Density and energy are
normalised by their own L2 norms; the momentum components by the L2 norm of the
momentum vector field (the Taylor-Green w-momentum starts at zero, so its own norm
says nothing early in a run).
"""
import dataclasses

import numpy as np
import pytest

from helpers import interior, random_turbulence, rel_l2, tgv, vortex2d

pytestmark = pytest.mark.gpu


def mixed_errors(a, b, dim):
    """Per-variable relative L2; momenta normalised by the momentum-vector norm."""
    mom = slice(1, 1 + dim)
    mnorm = np.linalg.norm(b[:, mom].ravel())
    out = []
    for l in range(dim + 2):
        d = np.linalg.norm((a[:, l] - b[:, l]).ravel())
        out.append(d / (mnorm if 1 <= l <= dim else np.linalg.norm(b[:, l].ravel())))
    return out


def run(cfg, qj, nsteps, device):
    from ouxsbli_b200.solver import Solver
    s = Solver(cfg, device)
    s.set_state(qj)
    s.step(nsteps)
    q = s.get_state()
    d = s.diagnostics()
    s.close()
    return q, d


# (name, builder, steps, bound): KEEP and the hybrid scheme hold the north star's 1e-5
# over these runs (the hybrid's sensor is decoded from FP64 velocities, so its threshold
# decisions are the FP64 solve's for the same state); pure SLAU, Roe and LES, whose
# discrete switches (the HRSLAU2 wiggle detector, TVD limiters, the SMS model) act on
# FP32 values, are held to a looser, stated bound.
CASES = [
    ("keep6_ns_ma01", lambda: tgv(32, mach=0.1, scheme="KEEP", visc="NS"), 200, 1e-5),
    ("keep6_ns_me4_ma05", lambda: tgv(32, mach=0.5, scheme="KEEP", visc="NS", visc_stencil="ME4Base"), 200, 1e-5),
    ("keep4_2d_rk4_1000", lambda: vortex2d(64, order=4, scheme="KEEP", visc="Euler", rk=4), 1000, 1e-5),
    ("keep6_2d_rk4", lambda: vortex2d(64, order=6, scheme="KEEP", visc="Euler", rk=4), 500, 1e-5),
    ("hybrid6_ns_ma125", lambda: tgv(32, mach=1.25, scheme="Hybrid", visc="NS"), 200, 1e-5),
    ("slau6_ns_ma01", lambda: tgv(32, mach=0.1, scheme="SLAU", visc="NS"), 200, 1e-4),
    ("roe6_euler", lambda: tgv(24, mach=0.8, scheme="Roe", visc="Euler", tvd="tvd"), 100, 1e-4),
    ("les_slau6", lambda: random_turbulence(24, seed=9, scheme="SLAU", visc="LES"), 20, 1e-2),
]


@pytest.mark.parametrize("name,make,nsteps,bound", CASES, ids=[c[0] for c in CASES])
def test_mixed_close_to_fp64(name, make, nsteps, bound, cuda_device):
    cfg, qj = make()
    q64, d64 = run(cfg, qj, nsteps, cuda_device)
    cfgm = dataclasses.replace(cfg, precision="mixed")
    q32, d32 = run(cfgm, qj, nsteps, cuda_device)
    assert np.isfinite(q32).all()
    a, b = interior(q32, cfg.g, cfg.dim), interior(q64, cfg.g, cfg.dim)
    errs = mixed_errors(a, b, cfg.dim)
    assert max(errs) <= bound, errs
    # FP64 diagnostics of the mixed run track the FP64 run
    assert abs(d32[0] - d64[0]) <= bound * abs(d64[0])
    assert abs(d32[2] - d64[2]) <= 10 * bound * abs(d64[2])


def test_slau_low_mach_error_is_the_flows_sensitivity(cuda_device):
    """Why pure SLAU at Ma 0.1 is held to 1e-4: the flow amplifies perturbations at the
    rounding level (its HRSLAU2 wiggle detector switches on pressure differences), so the
    FP64 solve started from the initial field rounded once to FP32 departs from the FP64
    solve as far as the mixed form does.  No form that rounds through FP32 can hold
    1e-5 here; the mixed form stays within twice that one-time perturbation's effect."""
    cfg, qj = tgv(32, mach=0.1, scheme="SLAU", visc="NS")
    q64, _ = run(cfg, qj, 200, cuda_device)
    qr = np.asfortranarray(qj.astype(np.float32).astype(np.float64))
    q64r, _ = run(cfg, qr, 200, cuda_device)
    q32, _ = run(dataclasses.replace(cfg, precision="mixed"), qj, 200, cuda_device)
    ref = interior(q64, cfg.g, 3)
    e_round = max(mixed_errors(interior(q64r, cfg.g, 3), ref, 3))
    e_mixed = max(mixed_errors(interior(q32, cfg.g, 3), ref, 3))
    assert e_round > 1e-5, e_round
    assert e_mixed <= 2.0 * e_round, (e_mixed, e_round)
