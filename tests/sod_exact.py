"""Exact solution of the 1D Euler Riemann problem (ideal gas), for the shock-tube
known-answer test.

Method (the standard exact Riemann solver, e.g. E. F. Toro, "Riemann Solvers and
Numerical Methods for Fluid Dynamics", ch. 4): the star-region pressure p* solves
f_L(p) + f_R(p) + (u_R - u_L) = 0, where f_K is the shock (Rankine-Hugoniot) branch
for p > p_K and the isentropic rarefaction branch otherwise; p* by Newton iteration
from the two-rarefaction guess, u* from the same functions, and the solution at
(x, t) is sampled on the wave pattern that p* and u* fix.
"""
from __future__ import annotations

import math

import numpy as np


def _f(p, rho_k, p_k, c_k, g):
    """Velocity jump across the K wave for star pressure p, and its derivative."""
    if p > p_k:  # shock
        A = 2.0 / ((g + 1.0) * rho_k)
        B = (g - 1.0) / (g + 1.0) * p_k
        sq = math.sqrt(A / (p + B))
        return (p - p_k) * sq, sq * (1.0 - 0.5 * (p - p_k) / (B + p))
    pr = p / p_k  # rarefaction
    return (2.0 * c_k / (g - 1.0) * (pr ** ((g - 1.0) / (2.0 * g)) - 1.0),
            1.0 / (rho_k * c_k) * pr ** (-(g + 1.0) / (2.0 * g)))


def star_state(rho_l, u_l, p_l, rho_r, u_r, p_r, gamma=1.4, tol=1e-12, itmax=100):
    """(p*, u*) of the Riemann problem."""
    g = gamma
    c_l, c_r = math.sqrt(g * p_l / rho_l), math.sqrt(g * p_r / rho_r)
    z = (g - 1.0) / (2.0 * g)
    # two-rarefaction guess
    p = ((c_l + c_r - 0.5 * (g - 1.0) * (u_r - u_l)) / (c_l / p_l ** z + c_r / p_r ** z)) ** (1.0 / z)
    p = max(p, tol)
    for _ in range(itmax):
        fl, dl = _f(p, rho_l, p_l, c_l, g)
        fr, dr = _f(p, rho_r, p_r, c_r, g)
        pn = p - (fl + fr + (u_r - u_l)) / (dl + dr)
        pn = max(pn, tol)
        if abs(pn - p) <= tol * 0.5 * (pn + p):
            p = pn
            break
        p = pn
    fl, _ = _f(p, rho_l, p_l, c_l, g)
    fr, _ = _f(p, rho_r, p_r, c_r, g)
    return p, 0.5 * (u_l + u_r) + 0.5 * (fr - fl)


def solve(x, t, rho_l, u_l, p_l, rho_r, u_r, p_r, gamma=1.4, x0=0.0):
    """Density, velocity and pressure at positions x and time t > 0, the initial
    discontinuity at x0."""
    g = gamma
    ps, us = star_state(rho_l, u_l, p_l, rho_r, u_r, p_r, g)
    c_l, c_r = math.sqrt(g * p_l / rho_l), math.sqrt(g * p_r / rho_r)
    gm = (g - 1.0) / (g + 1.0)
    s = (np.asarray(x, dtype=float) - x0) / t
    rho, u, p = np.empty_like(s), np.empty_like(s), np.empty_like(s)
    for n, si in enumerate(s):
        if si <= us:  # left of the contact
            if ps > p_l:  # left shock
                sl = u_l - c_l * math.sqrt((g + 1.0) / (2.0 * g) * ps / p_l + (g - 1.0) / (2.0 * g))
                if si <= sl:
                    rho[n], u[n], p[n] = rho_l, u_l, p_l
                else:
                    rho[n] = rho_l * (ps / p_l + gm) / (gm * ps / p_l + 1.0)
                    u[n], p[n] = us, ps
            else:  # left rarefaction
                c_star = c_l * (ps / p_l) ** ((g - 1.0) / (2.0 * g))
                sh, st = u_l - c_l, us - c_star
                if si <= sh:
                    rho[n], u[n], p[n] = rho_l, u_l, p_l
                elif si >= st:
                    rho[n] = rho_l * (ps / p_l) ** (1.0 / g)
                    u[n], p[n] = us, ps
                else:
                    k = 2.0 / (g + 1.0) + gm / c_l * (u_l - si)
                    rho[n] = rho_l * k ** (2.0 / (g - 1.0))
                    u[n] = 2.0 / (g + 1.0) * (c_l + 0.5 * (g - 1.0) * u_l + si)
                    p[n] = p_l * k ** (2.0 * g / (g - 1.0))
        else:  # right of the contact
            if ps > p_r:  # right shock
                sr = u_r + c_r * math.sqrt((g + 1.0) / (2.0 * g) * ps / p_r + (g - 1.0) / (2.0 * g))
                if si >= sr:
                    rho[n], u[n], p[n] = rho_r, u_r, p_r
                else:
                    rho[n] = rho_r * (ps / p_r + gm) / (gm * ps / p_r + 1.0)
                    u[n], p[n] = us, ps
            else:  # right rarefaction
                c_star = c_r * (ps / p_r) ** ((g - 1.0) / (2.0 * g))
                sh, st = u_r + c_r, us + c_star
                if si >= sh:
                    rho[n], u[n], p[n] = rho_r, u_r, p_r
                elif si <= st:
                    rho[n] = rho_r * (ps / p_r) ** (1.0 / g)
                    u[n], p[n] = us, ps
                else:
                    k = 2.0 / (g + 1.0) - gm / c_r * (u_r - si)
                    rho[n] = rho_r * k ** (2.0 / (g - 1.0))
                    u[n] = 2.0 / (g + 1.0) * (-c_r + 0.5 * (g - 1.0) * u_r + si)
                    p[n] = p_r * k ** (2.0 * g / (g - 1.0))
    return rho, u, p
