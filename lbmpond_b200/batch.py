"""Batched 1D PonD (host-side front end of the pond_batch_* C ABI).

`Batch` advances many independent D1Q5 problems of uneven length (1..4096
nodes, zero-gradient ends) with persistent, graph-replayed kernel launches;
all arithmetic runs in libpond_b200.so.  `riemann_problems` makes the seeded
Riemann-problem set the batch benchmark runs: lengths uniform in
[lmin, lmax], left/right rho and p log-uniform in [0.1, 10], u uniform in
[-1, 1], the discontinuity at the midpoint, T = p / rho.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import LAGR4, WENO5

NPAIR_IN, NPAIR_OUT = 21, 2
# autotuner candidates: (threads per CTA, lane_cap)
TILES = tuple((t, c) for t in (256, 512, 768, 1024) for c in (2, 4, 8, 16)) + ((768, 100),)


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if a is not None else None


def riemann_problems(nproblems=4096, seed=0, lmin=256, lmax=4096):
    """lengths (int32 [P]) and concatenated float64 rho, u, T."""
    rng = np.random.default_rng(seed)
    lengths = rng.integers(lmin, lmax + 1, nproblems).astype(np.int32)
    lo, hi = np.log(0.1), np.log(10.0)
    rho_lr = np.exp(rng.uniform(lo, hi, (nproblems, 2)))
    p_lr = np.exp(rng.uniform(lo, hi, (nproblems, 2)))
    u_lr = rng.uniform(-1.0, 1.0, (nproblems, 2))
    side = np.concatenate([(np.arange(n) >= n // 2).astype(np.int64) for n in lengths])
    prob = np.repeat(np.arange(nproblems), lengths)
    rho = rho_lr[prob, side]
    u = u_lr[prob, side]
    T = p_lr[prob, side] / rho
    return lengths, rho, u, T


def riemann_problems_moderate(nproblems=4096, seed=0, lmin=256, lmax=4096, lam=0.3, rho_ratio=4.0, T_ratio=1.5,
                              u_scale=0.2):
    """A well-posed companion of riemann_problems: per side rho log-uniform
    with a ratio of at most `rho_ratio` across the jump, temperature
    log-uniform with a ratio of at most `T_ratio`, in lattice units
    T = lam^2 * T_phys with T_phys around 1, and u uniform in
    lam * u_scale * [-1, 1].  The specified set (ratios up to 100 in rho and
    in p, independently) drives the reference iteration non-finite on most
    problems within a few steps; with density ratios up to 10 and
    temperature ratios up to 2 the float64 oracle still loses some problems
    (density ratio ~9: non-finite by step 21-23), while on this set it keeps
    every sampled problem finite."""
    rng = np.random.default_rng(seed)
    lengths = rng.integers(lmin, lmax + 1, nproblems).astype(np.int32)
    rho_lr = np.exp(rng.uniform(-0.5 * np.log(rho_ratio), 0.5 * np.log(rho_ratio), (nproblems, 2)))
    T_lr = lam ** 2 * np.exp(rng.uniform(-0.5 * np.log(T_ratio), 0.5 * np.log(T_ratio), (nproblems, 2)))
    u_lr = lam * u_scale * rng.uniform(-1.0, 1.0, (nproblems, 2))
    side = np.concatenate([(np.arange(n) >= n // 2).astype(np.int64) for n in lengths])
    prob = np.repeat(np.arange(nproblems), lengths)
    return lengths, rho_lr[prob, side], u_lr[prob, side], T_lr[prob, side]


class Batch:
    """A set of independent D1Q5 problems stepped together on one GPU."""

    def __init__(self, lengths, interp=WENO5, tau=0.9, tol_abs=1e-7, tol_rel=1e-6, max_iter=100, device=0):
        if isinstance(interp, str):
            interp = {"WENO5": WENO5, "LAGR4": LAGR4}[interp.upper()]
        L = _lib.load()
        self.lengths = np.ascontiguousarray(lengths, np.int32)
        h = ctypes.c_void_p()
        _lib.check(L.pond_batch_create(int(self.lengths.size),
                                       self.lengths.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), int(interp),
                                       float(tau), float(tol_abs), float(tol_rel), int(max_iter), int(device),
                                       ctypes.byref(h)))
        self._L, self._h = L, h
        self.nodes = int(L.pond_batch_nodes(h))
        self.bins = int(L.pond_batch_bins(h))
        self.offsets = np.concatenate([[0], np.cumsum(self.lengths, dtype=np.int64)])

    @property
    def handle(self):
        return self._h

    def close(self):
        if getattr(self, "_h", None):
            self._L.pond_batch_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_state(self, rho, u, T):
        rho, u, T = (np.ascontiguousarray(a, np.float64).ravel() for a in (rho, u, T))
        if not (rho.size == u.size == T.size == self.nodes):
            raise ValueError(f"state arrays must hold {self.nodes} nodes")
        _lib.check(self._L.pond_batch_set_state(self._h, _dp(rho), _dp(u), _dp(T)))

    def get_state(self):
        """(f [5, nodes], rho, u, T), float64, problems concatenated."""
        f = np.empty((5, self.nodes))
        rho, u, T = np.empty(self.nodes), np.empty(self.nodes), np.empty(self.nodes)
        _lib.check(self._L.pond_batch_get_state(self._h, _dp(f), _dp(rho), _dp(u), _dp(T)))
        return f, rho, u, T

    def problem(self, arr, p):
        """View of problem p's nodes in a concatenated array (last axis)."""
        return arr[..., self.offsets[p]:self.offsets[p + 1]]

    def run(self, nsteps, steps_per_launch=None):
        """Advance every problem; returns the device time in ms."""
        ms = ctypes.c_float()
        k = int(steps_per_launch or max(nsteps, 1))
        _lib.check(self._L.pond_batch_run(self._h, int(nsteps), k, ctypes.byref(ms)))
        return float(ms.value)

    def stats(self):
        s, n = ctypes.c_int64(), ctypes.c_int64()
        m = ctypes.c_int32()
        _lib.check(self._L.pond_batch_stats(self._h, ctypes.byref(s), ctypes.byref(n), ctypes.byref(m)))
        return {"niter_sum": int(s.value), "nonconverged": int(n.value), "niter_max": int(m.value)}

    def set_pairs(self, X=None, Y=None, every=0, stride=1):
        """Sample training pairs into torch float32 CUDA buffers X [cap, 21],
        Y [cap, 2] during the following runs (every = 0 switches off)."""
        if every and (X is None or Y is None or X.shape[0] != Y.shape[0]):
            raise ValueError("X and Y must be given with the same row count")
        cap = X.shape[0] if X is not None else 0
        for t in (X, Y):  # torch's queued work on the buffers ends before the library writes them
            if t is not None and t.is_cuda:
                import torch
                torch.cuda.current_stream(t.device).synchronize()
        _lib.check(self._L.pond_batch_set_pairs(self._h, X.data_ptr() if X is not None else None,
                                                Y.data_ptr() if Y is not None else None, int(cap), int(every),
                                                int(stride)))

    def pairs_written(self):
        n = ctypes.c_int64()
        _lib.check(self._L.pond_batch_pairs_written(self._h, ctypes.byref(n)))
        return int(n.value)

    @property
    def tile(self):
        """(threads per CTA, lane_cap)"""
        t, c = ctypes.c_int(), ctypes.c_int()
        _lib.check(self._L.pond_batch_get_tile(self._h, ctypes.byref(t), ctypes.byref(c)))
        return int(t.value), int(c.value)

    @tile.setter
    def tile(self, tc):
        _lib.check(self._L.pond_batch_set_tile(self._h, int(tc[0]), int(tc[1])))

    def autotune(self, probe_steps=10, tiles=TILES):
        """Pick the fastest tile; returns (tile, {tile: ms})."""
        cand = np.ascontiguousarray(np.asarray(tiles, np.int32).reshape(-1, 2))
        ms = (ctypes.c_float * len(cand))()
        best = ctypes.c_int()
        _lib.check(self._L.pond_batch_autotune(self._h, int(probe_steps),
                                               cand.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), len(cand), ms,
                                               ctypes.byref(best)))
        return tuple(int(v) for v in cand[best.value]), {tuple(int(v) for v in t): float(m) for t, m in zip(cand, ms)}
