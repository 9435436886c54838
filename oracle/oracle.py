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
LAGR2, LAGR3, LAGR4, LAGR5, FIXED3, TVD, WENO5, GAP2, NONUNIFORM3, WENO5_ROW = 2, 3, 4, 5, 6, 7, 8, 9, 10, 11
BC_PERIODIC, BC_CLAMP, BC_MIRROR, BC_INFLOW = 0, 1, 2, 3

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
        ("inflow", ctypes.c_double * 5),
        ("tolg", ctypes.c_double * 2),
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
        u8p = ctypes.POINTER(ctypes.c_uint8)
        L.orc_step_mesh.argtypes = [ctypes.POINTER(_Params), dp, dp, dp, u8p, dp, dp, dp, dp, ip]
        L.orc_step_mesh.restype = ctypes.c_int64
        L.orc_amr_refine.argtypes = [ctypes.POINTER(_Params), dp, dp, dp, u8p, ctypes.c_double,
                                     ctypes.POINTER(ctypes.c_int64)]
        L.orc_amr_refine.restype = ctypes.c_int64
        L.orc_amr_coarsen.argtypes = [ctypes.POINTER(_Params), dp, dp, u8p, ctypes.c_double]
        L.orc_amr_coarsen.restype = ctypes.c_int64
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
         max_iter=100, bc=(BC_PERIODIC,) * 3, guess=None, nthreads=0, dof=None, inflow=None, tolg=None):
    """One pull step; returns (new_state, niter[N], nonconverged_count).  A
    state with energy populations (``state.h``) steps with the
    double-distribution extension and needs ``dof``.  ``inflow`` = (rho,
    u_x, u_y, u_z, T) of the ghost node of BC_INFLOW axes; ``tolg`` = (abs,
    rel) tolerance of the gauge's convergence test (default: tol_abs, tol_rel)."""
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
                max_iter, nthreads, float(dof) if ddf else 0.0,
                (ctypes.c_double * 5)(*(inflow if inflow is not None else (1.0, 0.0, 0.0, 0.0, 1.0))),
                (ctypes.c_double * 2)(*(tolg if tolg is not None else (-1.0, -1.0))))
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


def _u8p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))


def _mesh_params(nx, interp=LAGR2, tau=0.9, tol_abs=1e-12, tol_rel=1e-10, max_iter=100, nthreads=0):
    return _Params(D1Q5, interp, nx, 1, 1, (ctypes.c_int * 3)(BC_PERIODIC, BC_PERIODIC, BC_PERIODIC), tau,
                   tol_abs, tol_rel, max_iter, nthreads, 0.0, (ctypes.c_double * 5)(1.0, 0.0, 0.0, 0.0, 1.0),
                   (ctypes.c_double * 2)(-1.0, -1.0))


def step_mesh(state: State, nx: int, interp=GAP2, mask=None, pos=None, tau=0.9, tol_abs=1e-12, tol_rel=1e-10,
              max_iter=100, nthreads=0):
    """One D1Q5 pull step on a periodic 1D mesh with a node mask (Cinfo::set;
    None = all active) and node positions (Cell::p.x; None = p_x = x).
    Inactive nodes are carried over unchanged.  Returns (state, niter, nonconverged)."""
    L = lib()
    N = nx
    p = _mesh_params(nx, interp, tau, tol_abs, tol_rel, max_iter, nthreads)
    f_in = np.ascontiguousarray(state.f, dtype=np.float64)
    r_in = np.ascontiguousarray(state.rho, dtype=np.float64)
    g_in = np.ascontiguousarray(state.g, dtype=np.float64)
    assert f_in.shape == (5, N) and r_in.shape == (N,) and g_in.shape == (4, N)
    mp = pp = None
    if mask is not None:
        mask = np.ascontiguousarray(mask, dtype=np.uint8)
        assert mask.shape == (N,)
        mp = _u8p(mask)
    if pos is not None:
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        assert pos.shape == (N,)
        pp = _dp(pos)
    out = State(np.empty((5, N)), np.empty(N), np.empty((4, N)))
    niter = np.zeros(N, dtype=np.int32)
    nc = L.orc_step_mesh(ctypes.byref(p), _dp(f_in), _dp(r_in), _dp(g_in), mp, pp,
                         _dp(out.f), _dp(out.rho), _dp(out.g), _ip(niter))
    if nc < 0:
        raise ValueError("oracle mesh step rejected its parameters")
    return out, niter, int(nc)


def amr_refine(state: State, mask, tol=0.01):
    """AMR_add (amr.cu:1-27) on a D1Q5 1D state; returns (state, mask, added, limit_hits)."""
    st = state.copy()
    m = np.array(mask, dtype=np.uint8, copy=True)
    nx = m.size
    p = _mesh_params(nx)
    lim = ctypes.c_int64(0)
    st.f = np.ascontiguousarray(st.f); st.rho = np.ascontiguousarray(st.rho); st.g = np.ascontiguousarray(st.g)
    added = lib().orc_amr_refine(ctypes.byref(p), _dp(st.f), _dp(st.rho), _dp(st.g), _u8p(m), float(tol),
                                 ctypes.byref(lim))
    if added < 0:
        raise ValueError("oracle refine rejected its parameters")
    return st, m, int(added), int(lim.value)


def amr_coarsen(state: State, mask, tol=0.01):
    """AMR_remove (amr.cu:28-55); returns (mask, removed)."""
    m = np.array(mask, dtype=np.uint8, copy=True)
    p = _mesh_params(m.size)
    rho = np.ascontiguousarray(state.rho, dtype=np.float64)
    g = np.ascontiguousarray(state.g, dtype=np.float64)
    removed = lib().orc_amr_coarsen(ctypes.byref(p), _dp(rho), _dp(g), _u8p(m), float(tol))
    if removed < 0:
        raise ValueError("oracle coarsen rejected its parameters")
    return m, int(removed)


def mesh_sums(state: State, mask=None, pos=None):
    """calcTotMoments (update.cu:52-69) on a D1Q5 1D mesh: active nodes only,
    each weighted by half the distance between its neighbours' positions
    (lifted by Nx across the periodic seam) under NRMESH, else by 1."""
    rho = state.rho
    ux, uy, uz, T = state.g
    nx = rho.size
    act = np.ones(nx, dtype=bool) if mask is None else np.asarray(mask) != 0
    if pos is None:
        d = np.ones(nx)
    else:
        pm, pp = np.roll(pos, 1), np.roll(pos, -1)
        pp = np.where(pp < pm, pp + nx, pp)
        d = 0.5 * (pp - pm)
    w = np.where(act, d, 0.0)
    return {"mass": float(np.sum(rho * w)), "moment": float(np.sum(rho * ux * w)),
            "enrg": float(np.sum(rho * (ux * ux + uy * uy + uz * uz + 1.0 * T) * w))}


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
