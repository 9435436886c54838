"""ctypes front end of the FP64 CPU oracle (TEST INFRASTRUCTURE ONLY).

The oracle restates the reference PonD pull step (engrab6/lbmPonD steps.cu
``LBMpull`` / ``PonDstepD3Q125``) in plain C++.  Only the tests, the smoke
check and the CPU-baseline leg of bench.py use it, and only as the checker or
the timed CPU baseline; the product library never imports it.

State arrays are numpy float64 in the library's host layout:
``f[Q, N]``, ``rho[N]``, ``g[4, N]`` (u_x, u_y, u_z, T), N = nx*ny*nz with x
fastest, populations in the reference's order.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liborc.so")

D1Q5, D3Q27, D3Q125 = 0, 1, 2
LAGR2, LAGR3, LAGR4, LAGR5, FIXED3, TVD, WENO5 = 2, 3, 4, 5, 6, 7, 8
BC_PERIODIC, BC_CLAMP, BC_MIRROR = 0, 1, 2

# reference defaults: steps.cu:451 propagate<4> for D1Q5/D3Q27, and the
# fixed-origin quadratic D3Q125 kernel (steps.cu:151, launched update.cu:98)
DEFAULT_INTERP = {D1Q5: LAGR4, D3Q27: LAGR4, D3Q125: FIXED3}


class _Params(ctypes.Structure):
    _fields_ = [
        ("lattice", ctypes.c_int),
        ("interp", ctypes.c_int),
        ("nx", ctypes.c_int64),
        ("ny", ctypes.c_int64),
        ("nz", ctypes.c_int64),
        ("bc", ctypes.c_int * 3),
        ("tau", ctypes.c_double),
        ("tol_abs", ctypes.c_double),
        ("tol_rel", ctypes.c_double),
        ("max_iter", ctypes.c_int),
        ("nthreads", ctypes.c_int),
        ("dof", ctypes.c_double),
    ]


_lib = None


def build(force: bool = False) -> str:
    """Compile liborc.so with the Makefile beside this file."""
    if force or not os.path.exists(LIB_PATH) or (
        os.path.getmtime(LIB_PATH) < os.path.getmtime(os.path.join(HERE, "pond_oracle.cpp"))
    ):
        subprocess.run(["make", "-s", "-C", HERE, "-B" if force else "liborc.so"], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        L.orc_q.argtypes = [ctypes.c_int]
        L.orc_tables.argtypes = [ctypes.c_int, dp, ip, dp, dp]
        L.orc_reverse.argtypes = [ctypes.c_int, ip, ip, ip]
        L.orc_set_base.argtypes = [ctypes.c_int, ctypes.c_double, dp, dp]
        L.orc_transfer_gauge.argtypes = [ctypes.c_int, dp, dp, dp, ctypes.c_int]
        L.orc_transfer_gauge.restype = ctypes.c_double
        L.orc_calc_moments.argtypes = [ctypes.c_int, dp, dp, dp, dp]
        L.orc_lagr_pol.argtypes = [ctypes.c_int] * 4 + [ctypes.c_double] * 3
        L.orc_lagr_pol.restype = ctypes.c_double
        L.orc_step.argtypes = [ctypes.POINTER(_Params), dp, dp, dp, dp, dp, dp, dp, ip]
        L.orc_step.restype = ctypes.c_int64
        L.orc_set_energy.argtypes = [ctypes.c_int, ctypes.c_double, dp, ctypes.c_double, dp]
        L.orc_step_ddf.argtypes = [ctypes.POINTER(_Params), dp, dp, dp, dp, dp, dp, dp, dp, dp, ip]
        L.orc_step_ddf.restype = ctypes.c_int64
        L.orc_max_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


@dataclass
class Tables:
    Q: int
    xi: np.ndarray  # [Q,3] real directions
    e: np.ndarray   # [Q,3] integer directions
    w: np.ndarray   # [Q]
    tlat: float
    dim: float


def tables(lattice: int) -> Tables:
    L = lib()
    Q = L.orc_q(lattice)
    xi = np.zeros((Q, 3)); e = np.zeros((Q, 3), dtype=np.int32); w = np.zeros(Q); td = np.zeros(2)
    L.orc_tables(lattice, _dp(xi), _ip(e), _dp(w), _dp(td))
    return Tables(Q, xi, e, w, float(td[0]), float(td[1]))


def reverse_maps(lattice: int):
    L = lib()
    Q = L.orc_q(lattice)
    r = np.zeros((3, Q), dtype=np.int32)
    L.orc_reverse(lattice, _ip(r[0]), _ip(r[1]), _ip(r[2]))
    return r


def set_base(lattice: int, rho: float, uT) -> np.ndarray:
    L = lib()
    Q = L.orc_q(lattice)
    f = np.zeros(Q)
    u = np.ascontiguousarray(uT, dtype=np.float64)
    L.orc_set_base(lattice, float(rho), _dp(u), _dp(f))
    return f


def transfer_gauge(lattice: int, f, uT_src, uT_dst, inew: int) -> float:
    f = np.ascontiguousarray(f, dtype=np.float64)
    a = np.ascontiguousarray(uT_src, dtype=np.float64)
    b = np.ascontiguousarray(uT_dst, dtype=np.float64)
    return lib().orc_transfer_gauge(lattice, _dp(f), _dp(a), _dp(b), int(inew))


def calc_moments(lattice: int, f, vi):
    f = np.ascontiguousarray(f, dtype=np.float64)
    v = np.ascontiguousarray(vi, dtype=np.float64)
    rho = np.zeros(1); uT = np.zeros(4)
    lib().orc_calc_moments(lattice, _dp(f), _dp(v), _dp(rho), _dp(uT))
    return float(rho[0]), uT


def lagr_pol(n, ix, iy, iz, sx, sy, sz) -> float:
    return lib().orc_lagr_pol(n, ix, iy, iz, sx, sy, sz)


def set_energy(lattice: int, rho: float, uT, dof: float) -> np.ndarray:
    """Equilibrium energy populations of one node (double-distribution
    extension): h_i = rho w_i (|v_i|^2 + dof T)."""
    L = lib()
    h = np.zeros(L.orc_q(lattice))
    u = np.ascontiguousarray(uT, dtype=np.float64)
    L.orc_set_energy(lattice, float(rho), _dp(u), float(dof), _dp(h))
    return h


@dataclass
class State:
    f: np.ndarray    # [Q, N]
    rho: np.ndarray  # [N]
    g: np.ndarray    # [4, N]
    h: np.ndarray | None = None  # [Q, N] energy populations (double-distribution extension)

    def copy(self):
        return State(self.f.copy(), self.rho.copy(), self.g.copy(), None if self.h is None else self.h.copy())


def with_energy(state: State, lattice: int, dof: float) -> State:
    """The state plus equilibrium energy populations in every node's gauge."""
    t = tables(lattice)
    rho, g = state.rho, state.g
    s = np.sqrt(np.abs(g[3]) / t.tlat)
    v2 = sum((s[None, :] * t.xi[:, a:a + 1] + g[a][None, :]) ** 2 for a in range(3))
    h = t.w[:, None] * rho[None, :] * (v2 + dof * g[3][None, :])
    return State(state.f.copy(), rho.copy(), g.copy(), np.ascontiguousarray(h))


def base_state(lattice: int, rho, ux, uy, uz, T) -> State:
    """Cell::set_base on every node (lbpack.cu:15-21): f_i = w_i * rho."""
    t = tables(lattice)
    rho = np.ascontiguousarray(rho, dtype=np.float64).ravel()
    g = np.stack([np.broadcast_to(np.asarray(a, dtype=np.float64).ravel(), rho.shape)
                  for a in (ux, uy, uz, T)]).copy()
    f = t.w[:, None] * rho[None, :]
    return State(np.ascontiguousarray(f), rho.copy(), g)


def step(state: State, lattice: int, shape, interp=None, tau=0.9, tol_abs=1e-12, tol_rel=1e-10,
         max_iter=100, bc=(BC_PERIODIC,) * 3, guess=None, nthreads=0, dof=None):
    """One pull step; returns (new_state, niter[N], nonconverged_count).  A
    state with energy populations (``state.h``) steps with the
    double-distribution extension and needs ``dof``."""
    L = lib()
    nx, ny, nz = shape
    N = nx * ny * nz
    Q = L.orc_q(lattice)
    if interp is None:
        interp = DEFAULT_INTERP[lattice]
    ddf = state.h is not None
    if ddf and dof is None:
        raise ValueError("a state with energy populations needs dof")
    p = _Params(lattice, interp, nx, ny, nz, (ctypes.c_int * 3)(*bc), tau, tol_abs, tol_rel,
                max_iter, nthreads, float(dof) if ddf else 0.0)
    f_in = np.ascontiguousarray(state.f, dtype=np.float64)
    r_in = np.ascontiguousarray(state.rho, dtype=np.float64)
    g_in = np.ascontiguousarray(state.g, dtype=np.float64)
    assert f_in.shape == (Q, N) and r_in.shape == (N,) and g_in.shape == (4, N)
    out = State(np.empty((Q, N)), np.empty(N), np.empty((4, N)))
    niter = np.zeros(N, dtype=np.int32)
    gp = None
    if guess is not None:
        guess = np.ascontiguousarray(guess, dtype=np.float64)
        assert guess.shape == (4, N)
        gp = _dp(guess)
    if ddf:
        h_in = np.ascontiguousarray(state.h, dtype=np.float64)
        assert h_in.shape == (Q, N)
        out.h = np.empty((Q, N))
        nc = L.orc_step_ddf(ctypes.byref(p), _dp(f_in), _dp(h_in), _dp(r_in), _dp(g_in), gp,
                            _dp(out.f), _dp(out.h), _dp(out.rho), _dp(out.g), _ip(niter))
    else:
        nc = L.orc_step(ctypes.byref(p), _dp(f_in), _dp(r_in), _dp(g_in), gp,
                        _dp(out.f), _dp(out.rho), _dp(out.g), _ip(niter))
    if nc < 0:
        raise ValueError("oracle step rejected its parameters")
    return out, niter, int(nc)


def diagnostics(state: State, lattice: int, shape):
    """Conservation sums of update.cu:52-69 and the TGV kinetic energy of diagn.cu:3-22."""
    dim = tables(lattice).dim
    rho = state.rho
    ux, uy, uz, T = state.g
    nx, ny, nz = shape
    u2 = ux * ux + uy * uy + uz * uz
    d8pi3 = 1.0 / (8 * np.pi ** 3)
    dxyz = (2 * np.pi / nx) * (2 * np.pi / ny) * (2 * np.pi / nz)
    return {
        "mass": float(np.sum(rho)),
        "moment": float(np.sum(rho * ux)),
        "enrg": float(np.sum(rho * (u2 + dim * T))),
        "k": float(np.sum(0.5 * d8pi3 * u2 * dxyz)),
    }


def max_threads() -> int:
    return lib().orc_max_threads()
