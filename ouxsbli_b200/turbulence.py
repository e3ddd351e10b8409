"""Decaying isotropic turbulence initial fields (the serving workload's requests).

A seeded, solenoidal, random-phase velocity field with the model spectrum
E(k) ~ k^4 exp(-2 (k/k0)^2) on the periodic box [0, 2 pi L0)^3, at uniform
density and pressure.  The velocity is scaled to the requested turbulent Mach
number Mt = sqrt(<u.u>) / c, and the density to the requested Taylor-scale
Reynolds number Re_lambda = rho u' lambda / mu with u' = sqrt(<u.u>/3) and
lambda = sqrt(<u^2> / <(du/dx)^2>) measured on the generated field.

The reference's own DHIT initial condition (3D_solver/DHIT/set_init_dhit.f90,
a Pope spectrum built with cuFFT and the Fortran RNG) is a different
generator; this one is the project's own.
"""
from __future__ import annotations

import math

import numpy as np

from .cases import sutherland_mu
from .grid import cyclic_axis, fill_periodic, jacobian, to_qj


def solenoidal_field(n: int, seed: int, k0: float = 4.0) -> np.ndarray:
    """(3, n, n, n) divergence-free velocity with E(k) ~ k^4 exp(-2 (k/k0)^2), unit rms."""
    rng = np.random.default_rng(seed)
    w = rng.standard_normal((3, n, n, n))
    W = np.fft.fftn(w, axes=(1, 2, 3))
    k1 = np.fft.fftfreq(n, d=1.0 / n)
    KX, KY, KZ = np.meshgrid(k1, k1, k1, indexing="ij")
    K2 = KX ** 2 + KY ** 2 + KZ ** 2
    K2s = np.where(K2 == 0, 1.0, K2)
    div = (KX * W[0] + KY * W[1] + KZ * W[2]) / K2s
    W[0] -= KX * div
    W[1] -= KY * div
    W[2] -= KZ * div
    kk = np.sqrt(K2)
    E = kk ** 4 * np.exp(-2.0 * (kk / k0) ** 2)
    amp = np.sqrt(E / np.where(K2 == 0, 1.0, K2))
    amp[K2 == 0] = 0.0
    W *= amp[None]
    u = np.real(np.fft.ifftn(W, axes=(1, 2, 3)))
    u /= math.sqrt(np.mean(np.sum(u ** 2, axis=0)) / 3.0)
    return u


def decaying_turbulence(n: int, order: int = 6, seed: int = 0, mt: float = 0.3, re_lambda: float = 100.0,
                        k0: float = 4.0, T0: float = 300.0, R: float = 287.03, gamma: float = 1.4,
                        L0: float = 1.0e-3, cfl: float = 0.5, **cfg_kw):
    """SolverConfig and initial QJ of one decaying-turbulence request."""
    from .config import SolverConfig
    g = order // 2
    nx = n + 2 * g
    L = 2.0 * math.pi * L0
    xc, dx = cyclic_axis(nx, L, order)
    u = solenoidal_field(n, seed, k0)
    c = math.sqrt(gamma * R * T0)
    urms = mt * c / math.sqrt(3.0)  # per component
    u *= urms
    h = L / n
    dudx = (np.roll(u[0], -1, axis=0) - np.roll(u[0], 1, axis=0)) / (2.0 * h)
    lam = math.sqrt(np.mean(u[0] ** 2) / np.mean(dudx ** 2))
    mu0 = sutherland_mu(T0)
    rho0 = re_lambda * mu0 / (urms * lam)
    p0 = rho0 * R * T0
    Q = np.zeros((nx, 5, nx, nx), order="F")
    sl = slice(g, g + n)
    Q[sl, 0, sl, sl] = rho0
    for a in range(3):
        Q[sl, 1 + a, sl, sl] = rho0 * u[a]
    Q[sl, 4, sl, sl] = p0 / (gamma - 1.0) + 0.5 * rho0 * np.sum(u ** 2, axis=0)
    fill_periodic(Q, g)
    umax = float(np.abs(u).max())
    dt = cfl * h / (umax + c)
    cfg = SolverConfig(dim=3, nx=nx, ny=nx, nz=nx, order=order, gamma=gamma, R=R, dt=dt, dx=dx, dy=dx.copy(),
                       dz=dx.copy(), **cfg_kw)
    return cfg, to_qj(Q, jacobian(dx, dx, dx))
