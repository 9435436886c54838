"""Exact solution of the 1D Riemann problem for an ideal gas (test helper).

The textbook method: the star-region pressure p* solves
f_L(p*) + f_R(p*) + (u_R - u_L) = 0, where f_K is the shock branch
(Rankine-Hugoniot) for p > p_K and the rarefaction branch (isentropic) for
p <= p_K; p* is found by Newton's method from the two-rarefaction estimate,
and the solution at x/t is sampled from the wave pattern (left wave, contact,
right wave).  Pressure p = rho T with a unit gas constant, so the sound speed
is sqrt(gamma p / rho).
"""
from __future__ import annotations

import numpy as np


def _pressure_function(p, rho_k, p_k, a_k, gamma):
    """f_K and its derivative for one side."""
    if p > p_k:  # shock
        A = 2.0 / ((gamma + 1.0) * rho_k)
        B = (gamma - 1.0) / (gamma + 1.0) * p_k
        sq = np.sqrt(A / (p + B))
        return (p - p_k) * sq, sq * (1.0 - 0.5 * (p - p_k) / (p + B))
    # rarefaction
    e = (gamma - 1.0) / (2.0 * gamma)
    return (2.0 * a_k / (gamma - 1.0) * ((p / p_k) ** e - 1.0),
            (p / p_k) ** (-(gamma + 1.0) / (2.0 * gamma)) / (rho_k * a_k))


def star_state(left, right, gamma, tol=1e-14, max_iter=200):
    """(p*, u*) of the states left/right = (rho, u, p)."""
    rl, ul, pl = left
    rr, ur, pr = right
    al, ar = np.sqrt(gamma * pl / rl), np.sqrt(gamma * pr / rr)
    if 2.0 * (al + ar) / (gamma - 1.0) <= ur - ul:
        raise ValueError("the states generate a vacuum")
    e = (gamma - 1.0) / (2.0 * gamma)
    p = ((al + ar - 0.5 * (gamma - 1.0) * (ur - ul)) / (al / pl ** e + ar / pr ** e)) ** (1.0 / e)
    for _ in range(max_iter):
        fl, dl = _pressure_function(p, rl, pl, al, gamma)
        fr, dr = _pressure_function(p, rr, pr, ar, gamma)
        dp = (fl + fr + ur - ul) / (dl + dr)
        p_new = max(p - dp, 1e-3 * tol)
        if abs(p_new - p) <= tol * 0.5 * (p_new + p):
            p = p_new
            break
        p = p_new
    fl, _ = _pressure_function(p, rl, pl, al, gamma)
    fr, _ = _pressure_function(p, rr, pr, ar, gamma)
    return p, 0.5 * (ul + ur) + 0.5 * (fr - fl)


def sample(left, right, gamma, xi):
    """(rho, u, p) at the similarity coordinates xi = (x - x0) / t."""
    rl, ul, pl = left
    rr, ur, pr = right
    al, ar = np.sqrt(gamma * pl / rl), np.sqrt(gamma * pr / rr)
    ps, us = star_state(left, right, gamma)
    g1 = (gamma - 1.0) / (gamma + 1.0)
    xi = np.asarray(xi, dtype=np.float64)
    rho = np.empty_like(xi); u = np.empty_like(xi); p = np.empty_like(xi)
    for n, s in enumerate(xi):
        if s <= us:  # left of the contact
            if ps > pl:  # left shock
                sl = ul - al * np.sqrt((gamma + 1.0) / (2.0 * gamma) * ps / pl + (gamma - 1.0) / (2.0 * gamma))
                if s <= sl:
                    rho[n], u[n], p[n] = rl, ul, pl
                else:
                    rho[n] = rl * (ps / pl + g1) / (g1 * ps / pl + 1.0)
                    u[n], p[n] = us, ps
            else:  # left rarefaction
                als = al * (ps / pl) ** ((gamma - 1.0) / (2.0 * gamma))
                if s <= ul - al:
                    rho[n], u[n], p[n] = rl, ul, pl
                elif s >= us - als:
                    rho[n] = rl * (ps / pl) ** (1.0 / gamma)
                    u[n], p[n] = us, ps
                else:  # inside the fan
                    c = 2.0 / (gamma + 1.0) + g1 / al * (ul - s)
                    rho[n] = rl * c ** (2.0 / (gamma - 1.0))
                    u[n] = 2.0 / (gamma + 1.0) * (al + 0.5 * (gamma - 1.0) * ul + s)
                    p[n] = pl * c ** (2.0 * gamma / (gamma - 1.0))
        else:  # right of the contact
            if ps > pr:  # right shock
                sr = ur + ar * np.sqrt((gamma + 1.0) / (2.0 * gamma) * ps / pr + (gamma - 1.0) / (2.0 * gamma))
                if s >= sr:
                    rho[n], u[n], p[n] = rr, ur, pr
                else:
                    rho[n] = rr * (ps / pr + g1) / (g1 * ps / pr + 1.0)
                    u[n], p[n] = us, ps
            else:  # right rarefaction
                ars = ar * (ps / pr) ** ((gamma - 1.0) / (2.0 * gamma))
                if s >= ur + ar:
                    rho[n], u[n], p[n] = rr, ur, pr
                elif s <= us + ars:
                    rho[n] = rr * (ps / pr) ** (1.0 / gamma)
                    u[n], p[n] = us, ps
                else:
                    c = 2.0 / (gamma + 1.0) - g1 / ar * (ur - s)
                    rho[n] = rr * c ** (2.0 / (gamma - 1.0))
                    u[n] = 2.0 / (gamma + 1.0) * (-ar + 0.5 * (gamma - 1.0) * ur + s)
                    p[n] = pr * c ** (2.0 * gamma / (gamma - 1.0))
    return rho, u, p
