"""Presets of the five benchmark configurations of the PonD step.

The reference fixes its problem at compile time (lattice and precision in
consts.h / params.h, the initial condition as overwritten assignments in
init.cu:2-108).  Here each configuration is a preset: the Solver arguments,
the initial condition, the number of steps of the full run, and a one-line
description.

    from lbmpond_b200 import configs
    s = configs.build("sphere_d3q27")          # a Solver holding the initial state
    s.step(configs.PRESETS["sphere_d3q27"].steps)

Sizes can be overridden (``build("tgv_d3q27", size=64)``), as can any Solver
argument (``build("sod_d1q5", precision="fp32")``).  The batched 1D
configuration has no single grid: ``batch_problems()`` gives its lengths and
states for lbmpond_b200.batch.Batch.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Callable

import numpy as np

SPHERE_LAMBDA = 0.25  # dt/dx of the spherical Riemann problem: T_lattice = lambda^2 p / rho
SOD_LAMBDA2 = 0.01    # (dt/dx)^2 of the Sod tube: T_lattice = 0.01 p / rho


def sphere_params(lam: float = SPHERE_LAMBDA):
    """Spherical Riemann problem on the unit box (pond_init POND_IC_SPHERE):
    cx, cy, cz, radius, rho_in, T_in, rho_out, T_out; inside r < 0.2 rho = 1,
    p = 1, outside rho = 0.125, p = 0.1, u = 0."""
    return (0.5, 0.5, 0.5, 0.2, 1.0, lam ** 2 * 1.0, 0.125, lam ** 2 * 0.1 / 0.125)


def sphere_state(n: int, lam: float = SPHERE_LAMBDA):
    """The spherical Riemann problem's rho[N] and gauge g[4, N] on the host
    (cell-centred, x fastest), as pond_init builds it on the device."""
    c = (np.arange(n) + 0.5) / n - 0.5
    z, y, x = np.meshgrid(c, c, c, indexing="ij")
    inside = (x * x + y * y + z * z < 0.2 ** 2).reshape(-1)
    p = sphere_params(lam)
    rho = np.where(inside, p[4], p[6])
    T = np.where(inside, p[5], p[7])
    zero = np.zeros(n ** 3)
    return rho, np.stack([zero, zero, zero, T])


SHOCK_T1 = 0.05  # pre-shock lattice temperature: every |v| stays below 1.1 nodes per step (TLat = 1)


def shock_vortex_state(n, mach=1.5, T1=SHOCK_T1, eps=0.3, radius=0.05, gamma=5.0 / 3.0):
    """Stationary normal shock at x = 0.5 (pre-shock rho = 1, T = T1, flow
    along +x at `mach`; post-shock state from the Rankine-Hugoniot
    relations) and an isentropic vortex of strength `eps` (velocity scale
    eps * c1) and radius `radius` at (0.25, 0.5) in x, y on the unit box, in
    lattice units of the D3Q125 gauge (TLat = 1).  gamma = 5/3 is the
    monatomic 3D gas the one-population step models; other values need the
    energy populations (Solver(..., ddf_dof=...))."""
    x = (np.arange(n) + 0.5) / n
    X, Y, _ = np.meshgrid(x, x, x, indexing="ij")  # [x, y, z]
    c1 = np.sqrt(gamma * T1)
    u1 = mach * c1
    r21 = (gamma + 1) * mach ** 2 / ((gamma - 1) * mach ** 2 + 2)
    p21 = 1 + 2 * gamma / (gamma + 1) * (mach ** 2 - 1)
    pre = X < 0.5
    dx, dy = X - 0.25, Y - 0.5
    e = np.exp(0.5 * (1 - (dx * dx + dy * dy) / radius ** 2)) * pre
    ux = np.where(pre, u1, u1 / r21) - eps * c1 * dy / radius * e
    uy = eps * c1 * dx / radius * e
    T = np.where(pre, T1, T1 * p21 / r21) * (1 - (gamma - 1) / 2 * eps ** 2 * e * e)
    rho = np.where(pre, (1 - (gamma - 1) / 2 * eps ** 2 * e * e) ** (1 / (gamma - 1)), r21)
    flat = lambda a: np.ascontiguousarray(a.transpose(2, 1, 0)).ravel()  # noqa: E731  (x fastest)
    return flat(rho), np.stack([flat(ux), flat(uy), np.zeros(n ** 3), flat(T)])


def shock_vortex_inflow(mach=1.5, T1=SHOCK_T1, gamma=5.0 / 3.0):
    """The pre-shock state (rho, u_x, u_y, u_z, T) the inflow boundary holds
    below x = 0: the upstream side of shock_vortex_state."""
    return (1.0, mach * np.sqrt(gamma * T1), 0.0, 0.0, T1)


def tgv_params(gamma: float = 5.0 / 3.0, mach: float = 0.5):
    """Compressible Taylor-Green vortex (pond_init POND_IC_TGV): U0, T0, rho0,
    gamma with T0 = TLat/4 of D3Q27 and U0 = mach * sqrt(gamma T0)."""
    T0 = (1.0 / 3.0) / 4
    return (mach * np.sqrt(gamma * T0), T0, 1.0, gamma)


@dataclass
class Preset:
    description: str
    size: int
    solver: Callable[[int], dict]           # size -> Solver keyword arguments
    init: Callable[[object, int], None]     # (solver, size) -> initial state
    steps: int
    extra: dict = field(default_factory=dict)


def _sod_init(s, n):
    s.init("sod", 0.5, 1.0, 0.0, SOD_LAMBDA2 * 1.0, 0.125, 0.0, SOD_LAMBDA2 * 0.1 / 0.125)


def _shock_vortex_init(gamma):
    def init(s, n):
        rho, g = shock_vortex_state(n, gamma=gamma)
        s.set_state(rho, g)
        s.set_inflow(*shock_vortex_inflow(gamma=gamma))
    return init


PRESETS = {
    "sod_d1q5": Preset(
        "D1Q5 Sod tube on [0,1], interface at 0.5, (rho, p) = (1, 1) | (0.125, 0.1), TVD, tau 0.55, "
        "zero-gradient ends, float64, gamma 3 (one population)",
        1000, lambda n: dict(lattice="D1Q5", shape=(n, 1, 1), interp=7, precision="fp64", tau=0.55,
                             bc=("clamp", "clamp", "clamp")), _sod_init, 500),
    "sod_d1q5_gamma14": Preset(
        "the Sod tube as a gamma = 1.4 gas (energy populations, 4 extra degrees of freedom)",
        1000, lambda n: dict(lattice="D1Q5", shape=(n, 1, 1), interp=7, precision="fp64", tau=0.55,
                             bc=("clamp", "clamp", "clamp"), ddf_dof=4), _sod_init, 500),
    "tgv_d3q27": Preset(
        "D3Q27 compressible Taylor-Green vortex on [0, 2 pi)^3, Mach 0.5, quadratic Lagrange, tau 0.51, float32",
        128, lambda n: dict(lattice="D3Q27", shape=(n, n, n), interp=3, precision="fp32", tau=0.51),
        lambda s, n: s.init("tgv", *tgv_params()), 2000),
    "tgv_d3q27_gamma14": Preset(
        "the Taylor-Green vortex as a gamma = 1.4 gas (energy populations, 2 extra degrees of freedom)",
        128, lambda n: dict(lattice="D3Q27", shape=(n, n, n), interp=3, precision="fp32", tau=0.51, ddf_dof=2),
        lambda s, n: s.init("tgv", *tgv_params(1.4)), 2000),
    "sphere_d3q27": Preset(
        "D3Q27 spherical Riemann problem on the unit box, r < 0.2: (rho, p) = (1, 1), outside (0.125, 0.1), "
        "dt/dx 0.25, cubic Lagrange, tau 0.52, float32 with tolerance 1e-7 + 1e-6 |v|; at 256^3 the state goes "
        "non-finite between steps 250 and 275, where the inward rarefaction focuses at the centre (the float64 "
        "path fails there too), so runs of the full 1500 steps stop early",
        256, lambda n: dict(lattice="D3Q27", shape=(n, n, n), interp=4, precision="fp32", tau=0.52,
                            tol_abs=1e-7, tol_rel=1e-6),
        lambda s, n: s.init("sphere", *sphere_params()), 1500),
    "shock_vortex_d3q125": Preset(
        "D3Q125 Mach 1.5 normal shock at x = 0.5 + isentropic vortex (strength 0.3, radius 0.05) at (0.25, 0.5), "
        "centred WENO5 (POND_WENO5_ROW), tau 0.9, inflow of the pre-shock state below x = 0 "
        "and zero-gradient outflow above x = 1, periodic y and z, float32",
        192, lambda n: dict(lattice="D3Q125", shape=(n, n, n), precision="fp32", tau=0.9, interp=11,
                            bc=("inflow", "periodic", "periodic")), _shock_vortex_init(5.0 / 3.0), 1000),
    "shock_vortex_d3q125_fixed3": Preset(
        "the shock and vortex with the reference's D3Q125 scheme (fixed-origin quadratic, steps.cu:151-250)",
        192, lambda n: dict(lattice="D3Q125", shape=(n, n, n), precision="fp32", tau=0.9,
                            bc=("inflow", "periodic", "periodic")), _shock_vortex_init(5.0 / 3.0), 1000),
    "shock_vortex_d3q125_gamma14": Preset(
        "the shock and vortex as a gamma = 1.4 gas (energy populations, 2 extra degrees of freedom; "
        "fixed-origin quadratic)",
        192, lambda n: dict(lattice="D3Q125", shape=(n, n, n), precision="fp32", tau=0.9,
                            bc=("inflow", "periodic", "periodic"), ddf_dof=2), _shock_vortex_init(1.4), 1000),
}


def solver_kwargs(name: str, size: int | None = None, **overrides) -> dict:
    p = PRESETS[name]
    kw = p.solver(size or p.size)
    kw.update(overrides)
    return kw


def build(name: str, size: int | None = None, **overrides):
    """A Solver set up with the preset's parameters and initial state."""
    from . import Solver
    p = PRESETS[name]
    n = size or p.size
    s = Solver(**solver_kwargs(name, n, **overrides))
    try:
        p.init(s, n)
    except Exception:
        s.close()
        raise
    return s


def batch_problems(nproblems: int = 4096, seed: int = 0):
    """The batched D1Q5 configuration: lengths, rho, u, T of `nproblems`
    independent Riemann tubes (lengths U[256, 4096], rho and p log-uniform in
    [0.1, 10], u uniform in [-1, 1], jump at the midpoint) and the Batch
    arguments (WENO5, tau 0.9, float32, 1000 steps)."""
    from .batch import riemann_problems
    lengths, rho, u, T = riemann_problems(nproblems, seed=seed)
    return (lengths, rho, u, T), dict(interp=8, tau=0.9), 1000
