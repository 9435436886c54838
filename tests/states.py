"""Seeded synthetic states shared by the CPU and GPU tests (host layout:
rho[N], g[4, N] = (u_x, u_y, u_z, T), x fastest)."""
from __future__ import annotations

import numpy as np


def smooth_state(shape, dim, seed=0, rho0=1.0, T0=0.1, du=0.05, dT=0.02, drho=0.05, modes=2):
    """A smooth periodic random field: a few low Fourier modes per quantity."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = shape
    x = np.arange(nx)[None, None, :] / nx
    y = np.arange(ny)[None, :, None] / ny
    z = np.arange(nz)[:, None, None] / nz

    def field(amp):
        out = np.zeros((nz, ny, nx))
        for _ in range(modes):
            kx = rng.integers(1, 3)
            ky = rng.integers(0, 3) if ny > 1 else 0
            kz = rng.integers(0, 3) if nz > 1 else 0
            ph = rng.uniform(0, 2 * np.pi)
            out += amp * rng.uniform(0.5, 1.0) * np.sin(2 * np.pi * (kx * x + ky * y + kz * z) + ph)
        return out.reshape(-1)

    rho = rho0 * (1 + field(drho))
    T = T0 * (1 + field(dT / T0 * 0.5))
    ux = field(du)
    uy = field(du) if dim == 3 else np.zeros_like(ux)
    uz = field(du) if dim == 3 else np.zeros_like(ux)
    return rho, np.stack([ux, uy, uz, T])


def sod_state(nx, left=(1.0, 0.0, 0.01), right=(0.125, 0.0, 0.008), x0=0.5):
    """Planar Riemann problem along x: (rho, u, T) on each side."""
    x = np.arange(nx)
    lft = x < x0 * nx
    rho = np.where(lft, left[0], right[0]).astype(np.float64)
    ux = np.where(lft, left[1], right[1]).astype(np.float64)
    T = np.where(lft, left[2], right[2]).astype(np.float64)
    z = np.zeros(nx)
    return rho, np.stack([ux, z, z, T])


def perturbed_populations(orc_mod, lattice, rho, g, seed=0, eps=0.02):
    """f = w*rho*(1 + eps*noise): a non-equilibrium population set."""
    t = orc_mod.tables(lattice)
    rng = np.random.default_rng(seed)
    f = t.w[:, None] * rho[None, :] * (1 + eps * rng.standard_normal((t.Q, rho.size)))
    return f
