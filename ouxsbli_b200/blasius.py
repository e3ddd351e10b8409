"""Laminar boundary-layer profiles for the wall-bounded cases' initial fields.

`blasius` solves the Blasius equation f''' + f f'' / 2 = 0, f(0) = f'(0) = 0,
f'(inf) = 1 (eta = y sqrt(U / (nu x))) by shooting on f''(0) with classical RK4
steps; `compressible_profile` maps it to a compressible, adiabatic-wall layer of a
given 99 % thickness as 2D_solver/src/set_init_common.f90 (set_init_tbl) and
src/set_compressible_bl.f90 (calc_HD_Blasius) do: u = U f'(eta), the
Crocco-Busemann temperature T = Taw - rf u^2 / (2 Cp), rho = p / (R T), the
Howarth-Dorodnitsyn stretching y = integral of T / T_inf d eta scaled so that the
stretched eta_99 = 4.91 sits at the given thickness, and the wall-normal velocity
v = nu_inf c (I f' - (T / T_inf) f) with I the stretched coordinate and c the scale.
"""
from __future__ import annotations

import functools

import numpy as np


def _rhs(y: np.ndarray) -> np.ndarray:
    f, fp, fpp = y
    return np.array([fp, fpp, -0.5 * f * fpp])


def _integrate(fpp0: float, eta_max: float, n: int) -> np.ndarray:
    h = eta_max / n
    y = np.array([0.0, 0.0, fpp0])
    out = np.empty((n + 1, 3))
    out[0] = y
    for k in range(n):
        k1 = _rhs(y)
        k2 = _rhs(y + 0.5 * h * k1)
        k3 = _rhs(y + 0.5 * h * k2)
        k4 = _rhs(y + h * k3)
        y = y + h / 6.0 * (k1 + 2.0 * k2 + 2.0 * k3 + k4)
        out[k + 1] = y
    return out


@functools.lru_cache(maxsize=4)
def blasius(eta_max: float = 10.0, n: int = 2000) -> tuple[np.ndarray, np.ndarray, np.ndarray, float]:
    """(eta, f, f', f''(0)) on a uniform grid of n + 1 points up to eta_max."""
    lo, hi = 0.3, 0.4
    for _ in range(45):  # bisection on f'(eta_max) - 1
        mid = 0.5 * (lo + hi)
        if _integrate(mid, eta_max, n)[-1, 1] < 1.0:
            lo = mid
        else:
            hi = mid
    fpp0 = 0.5 * (lo + hi)
    sol = _integrate(fpp0, eta_max, n)
    eta = np.linspace(0.0, eta_max, n + 1)
    return eta, sol[:, 0], sol[:, 1], fpp0


def compressible_profile(y: np.ndarray, delta99: float, u0: float, T0: float, p0: float, R: float, Cp: float,
                         rf: float, Taw: float, mu0: float) -> tuple[np.ndarray, np.ndarray, np.ndarray, np.ndarray]:
    """(rho, u, v, T) at wall distances y of an adiabatic-wall laminar layer whose
    stretched 99 % point sits at delta99."""
    eta, f, fp, _ = blasius()
    u = u0 * fp
    T = Taw - rf * u * u / (2.0 * Cp)
    Tr = T / T0
    rho = p0 / (R * T)
    integral = np.concatenate([[0.0], np.cumsum(0.5 * (Tr[1:] + Tr[:-1]) * np.diff(eta))])
    eta99 = 4.91
    i99 = np.searchsorted(eta, eta99, side="right")
    I99 = integral[i99 - 1]
    coeff = I99 / delta99
    nu0 = mu0 * R * T0 / p0
    yphys = integral / coeff
    v = nu0 * coeff * (integral * fp - Tr * f)
    interp = lambda a: np.interp(y, yphys, a)  # constant beyond the table ends
    return interp(rho), interp(u), interp(v), interp(T)
