"""Learned starting gauge for the PonD iteration (host-side front end).

`Predictor` wraps a pond_mlp (39 -> H -> H -> 4, BF16 tensor-core kernels,
float32 master weights, Adam; all arithmetic in libpond_b200.so).  Training
pairs come from plain steps (`collect_pairs`); device buffers for them are
torch tensors (plumbing only).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib

NIN, NOUT = 39, 4


def _torch_idle(*tensors):
    """Wait for torch's queued work on the tensors' devices.  The library runs
    on its own streams: a tensor torch has just written (or a block its
    caching allocator has just handed back while a kernel still reads it)
    must be settled before the library reads or writes that memory.  Every
    library call synchronises its own stream before returning, so the other
    direction needs nothing."""
    import torch
    for t in tensors:
        if t is not None and t.is_cuda:
            torch.cuda.current_stream(t.device).synchronize()


class Predictor:
    def __init__(self, hidden=64, seed=0, device=0):
        L = _lib.load()
        h = ctypes.c_void_p()
        _lib.check(L.pond_mlp_create(int(hidden), int(seed), int(device), ctypes.byref(h)))
        self._L, self._h = L, h
        self.hidden = hidden
        self.device = device
        self.nparams = L.pond_mlp_num_params(h)

    @property
    def handle(self):
        return self._h

    def close(self):
        if getattr(self, "_h", None):
            self._L.pond_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- parameters
    def get_params(self):
        p = np.empty(self.nparams, np.float32)
        st = np.empty(2 * NIN + 2 * NOUT, np.float32)
        _lib.check(self._L.pond_mlp_get_params(self._h, p.ctypes.data, st.ctypes.data))
        return p, st

    def set_params(self, params=None, stats=None):
        p = None if params is None else np.ascontiguousarray(params, np.float32)
        s = None if stats is None else np.ascontiguousarray(stats, np.float32)
        _lib.check(self._L.pond_mlp_set_params(self._h, p.ctypes.data if p is not None else None,
                                               s.ctypes.data if s is not None else None))

    def save(self, path):
        p, st = self.get_params()
        np.savez(path, params=p, stats=st, hidden=self.hidden)

    @classmethod
    def load(cls, path, device=0):
        z = np.load(path)
        pr = cls(int(z["hidden"]), device=device)
        pr.set_params(z["params"], z["stats"])
        return pr

    # -- training (X, Y: torch float32 CUDA tensors [n, 35], [n, 4])
    def fit_stats(self, X, Y):
        _torch_idle(X, Y)
        _lib.check(self._L.pond_mlp_fit_stats(self._h, X.data_ptr(), Y.data_ptr(), X.shape[0]))

    def train(self, X, Y, steps=1000, batch=4096, lr=2e-3):
        loss = np.empty(steps, np.float32)
        _torch_idle(X, Y)
        _lib.check(self._L.pond_mlp_train(self._h, X.data_ptr(), Y.data_ptr(), X.shape[0], int(batch), int(steps),
                                          float(lr), loss.ctypes.data))
        return loss

    def gradients(self, X, Y):
        g = np.empty(self.nparams, np.float32)
        loss = np.empty(1, np.float32)
        _torch_idle(X, Y)
        _lib.check(self._L.pond_mlp_gradients(self._h, X.data_ptr(), Y.data_ptr(), X.shape[0], g.ctypes.data,
                                              loss.ctypes.data))
        return float(loss[0]), g

    def forward(self, X, out=None):
        import torch
        if out is None:
            out = torch.empty((X.shape[0], NOUT), dtype=torch.float32, device=X.device)
        _torch_idle(X, out)
        _lib.check(self._L.pond_mlp_forward(self._h, X.data_ptr(), out.data_ptr(), X.shape[0]))
        return out


def collect_pairs(solver, X, Y, offset_rows=0, stride=7, seed=0, nodes=None):
    """Append the pairs of the solver's last step to rows [offset_rows, ...)
    of the torch buffers X [cap, 39] and Y [cap, 4] (and their node indices
    to the int64 buffer `nodes`, if given); returns rows written."""
    import torch
    L = _lib.load()
    cap = X.shape[0] - offset_rows
    if cap <= 0:
        return 0
    if nodes is None:  # the node of every row, to put the rows in a repeatable order
        nodes_all = torch.empty(cap, dtype=torch.int64, device=X.device)
        base = 0
    else:
        nodes_all, base = nodes, offset_rows
    n = ctypes.c_int64()
    xp = X.data_ptr() + offset_rows * NIN * 4
    yp = Y.data_ptr() + offset_rows * NOUT * 4
    np_ = nodes_all.data_ptr() + base * 8
    _torch_idle(X, Y, nodes_all)
    _lib.check(L.pond_collect_pairs(solver.handle, xp, yp, np_, int(cap), int(stride), int(seed), ctypes.byref(n)))
    n = int(n.value)
    if n > 1:  # the kernel appends rows in arrival order: sort them by node, then shuffle with the seed
        rows = slice(offset_rows, offset_rows + n)
        gen = torch.Generator(device=X.device)
        gen.manual_seed(int(seed))
        order = torch.argsort(nodes_all[base:base + n])
        order = order[torch.randperm(n, generator=gen, device=X.device)]
        X[rows] = X[rows][order]
        Y[rows] = Y[rows][order]
        nodes_all[base:base + n] = nodes_all[base:base + n][order]
    return n


def calibrate_gate(net, X, Y, tol=1e-6, candidates=(0.0, 1e-6, 3e-6, 1e-5, 3e-5, 1e-4, 3e-4, 1e-3, 3e-3, 1e-2,
                                                  float("inf"))):
    """Choose the activity gate: the last-increment threshold above which the
    network's increment replaces the previous gauge as the start.  The score
    of a candidate is the mean of log10(max |start error| + tol) over the
    pairs -- the starting error enters the iteration count through its
    logarithm; below the gate the start error is the increment itself."""
    import torch
    pred = net.forward(X)
    act = X[:, 35:39].abs().max(dim=1).values
    base = torch.log10(Y.abs().max(dim=1).values + tol)
    corr = torch.log10((Y - pred).abs().max(dim=1).values + tol)
    best, best_score = None, None
    for gt in candidates:
        use = act >= gt
        score = float(torch.where(use, corr, base).mean())
        if best_score is None or score < best_score:
            best, best_score = gt, score
    return best, best_score


def keep_history(solver, on=True):
    """Keep one more gauge level so that collect_pairs can run after a step."""
    _lib.check(_lib.load().pond_keep_history(solver.handle, 1 if on else 0))


def attach(solver, predictor, gate=0.0):
    """Start every following step of `solver` from the predicted gauge
    (None detaches)."""
    L = _lib.load()
    _lib.check(L.pond_set_predictor(solver.handle, predictor.handle if predictor else None, float(gate)))
    solver.params.learned = 1 if predictor else 0
