"""Derived fields of the reference's viewer (lbm_draw, lbm.cu:30-73), headless.

lbm_draw fills the GL image with one of 15 per-node quantities (nFunc):
rho; u_x / dt; u_x / sqrt(T) (the x Mach number without the heat-capacity
factor); T / dt^2; the fourth moment M4 = sum_i f_i v_ix^4 with
v_i = (sqrt(T/TLat) xi_i + u) / dt; the node's iteration count; and the first
nine populations.  The iteration count is the one LBMpull stores per node
(cinf.niter, steps.cu:508).  Inactive nodes of a 1D mesh show 0.  Here the same
quantities come back as arrays (and Solver.drop writes them as .arr files).

One deliberate difference: the reference's D3Q27 build never uploads the ef
table lbm_draw reads (lbm.cu:202-205 skip it for D3Q27), so its M4 there is
sum_i f_i u_x^4; here M4 uses the lattice velocities on every lattice.
"""
from __future__ import annotations

import numpy as np

# lbm_draw's nFunc order (lbm.cu:55-70)
FIELD_NAMES = ("rho", "ux", "mach", "T", "M4", "niter") + tuple(f"f{i}" for i in range(9))


def draw_fields(f, rho, g, xi_x, tlat, dt=1.0, niter=None, mask=None, names=None) -> dict:
    """The viewer's fields of a state in the host layout (f[Q, N], rho[N],
    g[4, N]); xi_x[Q] is the x velocity of each population at T = TLat.
    `niter` (int[N]) is needed only for "niter", which the default list holds
    only when `niter` is given; `mask` zeroes inactive nodes."""
    if names is None:
        names = tuple(n for n in FIELD_NAMES if n != "niter" or niter is not None)
    names = tuple(names)
    unknown = [n for n in names if n not in FIELD_NAMES]
    if unknown:
        raise ValueError(f"unknown fields {unknown}; known: {FIELD_NAMES}")
    f = np.asarray(f, dtype=np.float64)
    rho = np.asarray(rho, dtype=np.float64)
    g = np.asarray(g, dtype=np.float64)
    ux = g[0] / dt           # uT /= dt (lbm.cu:45)
    T = g[3] / dt / dt       # uT.w /= dt once more (lbm.cu:45)
    out = {}
    for name in names:
        if name == "rho":
            v = rho.copy()
        elif name == "ux":
            v = ux.copy()
        elif name == "mach":
            with np.errstate(divide="ignore", invalid="ignore"):
                v = ux / np.sqrt(T)
        elif name == "T":
            v = T.copy()
        elif name == "M4":  # lbm.cu:47-51
            vx = np.sqrt(T / tlat)[None, :] * np.asarray(xi_x, dtype=np.float64)[:, None] + ux[None, :]
            v = (f * vx ** 4).sum(axis=0)
        elif name == "niter":
            if niter is None:
                raise ValueError("the niter field needs the per-node iteration counts (Solver.keep_niter)")
            v = np.asarray(niter, dtype=np.float64).copy()
        else:
            i = int(name[1:])
            v = f[i].copy() if i < f.shape[0] else np.zeros_like(rho)
        if mask is not None:  # lbm.cu:53
            v = np.where(np.asarray(mask) != 0, v, 0.0)
        out[name] = v
    return out
