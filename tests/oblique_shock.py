"""Oblique-shock relations of a calorically perfect gas, for the reflected-shock
known-answer test (2D_solver/OS, ouxsbli/tests/test_os.py).

Standard results (e.g. NACA Report 1135, "Equations, tables, and charts for
compressible flow", 1953):
  * theta-beta-M: tan(theta) = 2 cot(beta) (M^2 sin^2 beta - 1) / (M^2 (gamma + cos 2 beta) + 2);
  * across the shock the normal Mach number Mn = M sin(beta) obeys the normal-shock
    jumps (pressure, density), the tangential velocity is unchanged and the flow
    turns by theta;
  * a shock reflected from a wall turns the flow back by theta: its angle beta_r
    (measured from the flow ahead of it) is the weak solution for (M2, theta).
"""
from __future__ import annotations

import math


def deflection(M: float, beta: float, g: float = 1.4) -> float:
    """Flow deflection theta (radians) of a shock of angle beta (radians) at Mach M."""
    return math.atan(2.0 / math.tan(beta) * (M * M * math.sin(beta) ** 2 - 1.0) /
                     (M * M * (g + math.cos(2.0 * beta)) + 2.0))


def weak_beta(M: float, theta: float, g: float = 1.4, tol: float = 1e-14) -> float:
    """Weak-solution shock angle (radians) turning a Mach-M flow by theta (radians)."""
    lo, hi = math.asin(1.0 / M), 0.5 * math.pi
    # beta of the largest deflection: golden-section search of deflection on (lo, hi)
    a, b = lo, hi
    r = 0.5 * (math.sqrt(5.0) - 1.0)
    for _ in range(200):
        c, d = b - r * (b - a), a + r * (b - a)
        if deflection(M, c, g) > deflection(M, d, g):
            b = d
        else:
            a = c
    bmax = 0.5 * (a + b)
    if deflection(M, bmax, g) < theta:
        raise ValueError("detached shock: theta above the maximum deflection")
    a, b = lo, bmax  # deflection rises monotonically on (lo, bmax): bisection
    while b - a > tol:
        m = 0.5 * (a + b)
        if deflection(M, m, g) < theta:
            a = m
        else:
            b = m
    return 0.5 * (a + b)


def normal_jump(Mn: float, g: float = 1.4) -> tuple[float, float, float]:
    """(p2/p1, rho2/rho1, Mn2) across a normal shock of upstream normal Mach Mn."""
    m2 = Mn * Mn
    pr = 1.0 + 2.0 * g / (g + 1.0) * (m2 - 1.0)
    rr = (g + 1.0) * m2 / ((g - 1.0) * m2 + 2.0)
    mn2 = math.sqrt((1.0 + 0.5 * (g - 1.0) * m2) / (g * m2 - 0.5 * (g - 1.0)))
    return pr, rr, mn2


def free_stream(M0: float, p_tot: float, T_tot: float, g: float, R: float) -> tuple[float, float, float]:
    """(rho, u, p) of the free stream from the stagnation state (isentropic relations)."""
    f = 1.0 + 0.5 * (g - 1.0) * M0 * M0
    p0, T0 = p_tot / f ** (g / (g - 1.0)), T_tot / f
    return p0 / (R * T0), M0 * math.sqrt(g * R * T0), p0


def shock(rho: float, U: float, p: float, beta: float, g: float) -> tuple[float, float, float, float]:
    """(rho, |u|, p, theta) behind a shock of angle beta (from the flow) on a flow of speed U."""
    a = math.sqrt(g * p / rho)
    M = U / a
    pr, rr, _ = normal_jump(M * math.sin(beta), g)
    ut, un = U * math.cos(beta), U * math.sin(beta) / rr
    return rho * rr, math.hypot(ut, un), p * pr, deflection(M, beta, g)


def reflected_state(M0: float, p_tot: float, T_tot: float, beta: float, g: float = 1.4, R: float = 287.03):
    """(rho3, ux3, uy3, p3, beta_r) behind the shock that an incident shock of angle beta
    makes on reflecting from a wall parallel to the free stream."""
    rho1, U1, p1 = free_stream(M0, p_tot, T_tot, g, R)
    rho2, U2, p2, theta = shock(rho1, U1, p1, beta, g)
    M2 = U2 / math.sqrt(g * p2 / rho2)
    beta_r = weak_beta(M2, theta, g)
    rho3, U3, p3, _ = shock(rho2, U2, p2, beta_r, g)
    return rho3, U3, 0.0, p3, beta_r
