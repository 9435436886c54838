"""B200-native Particles-on-Demand (PonD) lattice-Boltzmann step.

Host-side mirror of the reference's step interface (engrab6/lbmPonD):

    reference                          here
    ---------------------------------  -----------------------------------
    init()           init.cu:109       Solver.init(ic, ...)
    calcStep()       update.cu:86      Solver.step(n) / Solver.calcStep()
    diagnostics()    diagn.cu:24       Solver.diagnostics()
    drop(&dir)       drop.cu:2         Solver.drop(dir)  (.arr files)

All arithmetic runs in the CUDA library libpond_b200.so (sm_100a) behind the
C ABI of include/pond.h; this module only marshals arguments.  There is no
CPU fallback: constructing a Solver without the built library or a CUDA
device raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _lib
from ._lib import (BC_CLAMP, BC_INFLOW, BC_MIRROR, BC_PERIODIC, D1Q5, D3Q27, D3Q125, FIXED3, FP32, FP64, GAP2,
                   IC_ACOUSTIC, IC_SOD_X, IC_SPHERE, IC_TGV, IC_UNIFORM, LAGR2, LAGR3, LAGR4, LAGR5, NONUNIFORM3, TVD,
                   WENO5, WENO5_ROW, PondError)

__all__ = ["Solver", "PondError", "lattice_q", "lattice_tables", "D1Q5", "D3Q27", "D3Q125", "LAGR2", "LAGR3", "LAGR4", "LAGR5",
           "FIXED3", "TVD", "WENO5", "WENO5_ROW", "GAP2", "NONUNIFORM3", "BC_PERIODIC", "BC_CLAMP", "BC_MIRROR",
           "BC_INFLOW", "FP32", "FP64",
           "IC_ACOUSTIC", "IC_SOD_X", "IC_SPHERE", "IC_TGV", "IC_UNIFORM", "write_arr", "read_arr"]

_LATTICES = {"D1Q5": D1Q5, "D3Q27": D3Q27, "D3Q125": D3Q125}
_BCS = {"periodic": BC_PERIODIC, "clamp": BC_CLAMP, "zero_gradient": BC_CLAMP, "mirror": BC_MIRROR,
        "inflow": BC_INFLOW}
_ICS = {"acoustic": IC_ACOUSTIC, "sod": IC_SOD_X, "sphere": IC_SPHERE, "tgv": IC_TGV, "uniform": IC_UNIFORM}


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if a is not None else None


def lattice_q(lattice) -> int:
    lat = _LATTICES.get(lattice, lattice)
    return _lib.load().pond_q(int(lat))


def lattice_tables(lattice):
    """(xi[Q, 3], w[Q], TLat, Dim) in the reference's population order (consts.h)."""
    lat = int(_LATTICES.get(lattice, lattice))
    L = _lib.load()
    Q = L.pond_q(lat)
    if Q <= 0:
        raise ValueError(f"unknown lattice {lattice}")
    xi, w, td = np.zeros(3 * Q), np.zeros(Q), np.zeros(2)
    _lib.check(L.pond_lattice_tables(lat, _dp(xi), _dp(w), _dp(td)))
    return xi.reshape(Q, 3), w, float(td[0]), float(td[1])


class Solver:
    """One PonD simulation context on one GPU (wraps pond_ctx)."""

    def __init__(self, lattice="D3Q27", shape=(32, 32, 32), interp=None, precision="fp32", tau=0.9,
                 tol_abs=None, tol_rel=None, max_iter=100, bc=("periodic",) * 3, device=0, dt=1.0,
                 learned=False, ddf_dof=None):
        """``ddf_dof``: carry energy populations with that many extra degrees
        of freedom (D1Q5 1D grids; gamma = (Dim + dof + 2) / (Dim + dof))."""
        L = _lib.load()
        lat = _LATTICES.get(lattice, lattice)
        p = _lib.PondParams()
        _lib.check(L.pond_params_default(int(lat), ctypes.byref(p)))
        p.Nx, p.Ny, p.Nz = (int(v) for v in shape)
        if interp is not None:
            p.interp = int(interp)
        p.precision = {"fp32": FP32, "fp64": FP64}.get(precision, precision)
        if p.precision == FP64:  # the reference's USE_DOUBLE tolerances (steps.cu:62-63)
            p.tol_abs, p.tol_rel = 1e-12, 1e-10
        if tol_abs is not None:
            p.tol_abs = tol_abs
        if tol_rel is not None:
            p.tol_rel = tol_rel
        p.tau = tau
        p.dt = dt
        p.max_iter = max_iter
        p.device = device
        p.learned = 1 if learned else 0
        if ddf_dof is not None:
            p.ddf, p.ddf_dof = 1, int(ddf_dof)
        for a in range(3):
            p.bc[a] = _BCS.get(bc[a], bc[a])
        ctx = ctypes.c_void_p()
        _lib.check(L.pond_create(ctypes.byref(p), ctypes.byref(ctx)))
        self._L = L
        self._ctx = ctx
        self.params = p
        self.lattice = int(lat)
        self.shape = (int(p.Nx), int(p.Ny), int(p.Nz))
        self.N = self.shape[0] * self.shape[1] * self.shape[2]
        self.Q = L.pond_q(self.lattice)

    # -- lifetime
    def close(self):
        if getattr(self, "_ctx", None):
            self._L.pond_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._ctx

    # -- reference entry points
    def init(self, ic="acoustic", *params):
        """Built-in initial condition + set_base on both buffers (init.cu:109-128)."""
        code = _ICS.get(ic, ic)
        arr = np.ascontiguousarray(params, dtype=np.float64) if params else None
        _lib.check(self._L.pond_init(self._ctx, int(code), _dp(arr), len(params)))

    def set_state(self, rho, g, f=None):
        rho = np.ascontiguousarray(rho, dtype=np.float64).reshape(self.N)
        g = np.ascontiguousarray(g, dtype=np.float64).reshape(4, self.N)
        if f is not None:
            f = np.ascontiguousarray(f, dtype=np.float64).reshape(self.Q, self.N)
        _lib.check(self._L.pond_set_state(self._ctx, _dp(f), _dp(rho), _dp(g)))

    def get_state(self):
        f = np.empty((self.Q, self.N)); rho = np.empty(self.N); g = np.empty((4, self.N))
        _lib.check(self._L.pond_get_state(self._ctx, _dp(f), _dp(rho), _dp(g)))
        return f, rho, g

    def set_energy(self, h):
        """Energy populations h[Q, N] of a context made with ``ddf_dof``."""
        h = np.ascontiguousarray(h, dtype=np.float64).reshape(self.Q, self.N)
        _lib.check(self._L.pond_set_energy(self._ctx, _dp(h)))

    def get_energy(self):
        h = np.empty((self.Q, self.N))
        _lib.check(self._L.pond_get_energy(self._ctx, _dp(h)))
        return h

    def fields(self):
        out = [np.empty(self.N) for _ in range(5)]
        _lib.check(self._L.pond_get_fields(self._ctx, *[_dp(a) for a in out]))
        return dict(zip(("rho", "ux", "uy", "uz", "T"), out))

    def set_inflow(self, rho, ux, uy, uz, T):
        """State of the ghost node of ``"inflow"`` axes (equilibrium populations)."""
        _lib.check(self._L.pond_set_inflow(self._ctx, float(rho), float(ux), float(uy), float(uz), float(T)))

    def set_gauge_tolerance(self, tol_abs, tol_rel=0.0):
        """A separate convergence tolerance on u and T (the populations keep
        the Solver's); negative values restore the Solver's pair."""
        _lib.check(self._L.pond_set_gauge_tolerance(self._ctx, float(tol_abs), float(tol_rel)))

    def step(self, n=1):
        _lib.check(self._L.pond_step(self._ctx, int(n)))

    calcStep = step

    def diagnostics(self) -> dict:
        d = _lib.PondDiag()
        _lib.check(self._L.pond_diagnostics(self._ctx, ctypes.byref(d)))
        return {"mass": d.mass, "moment": tuple(d.moment), "enrg": d.enrg, "k": d.k, "niter_max": d.niter_max,
                "niter_mean": d.niter_mean, "niter_sum": d.niter_sum, "nonconverged": d.nonconverged,
                "istep": d.istep, "curtime": d.curtime}

    # -- one-dimensional mesh (GAP2 / NONUNIFORM3): node mask, AMR, node positions
    def set_mask(self, mask):
        """Node mask (Cinfo::set): nonzero = active; inactive nodes are skipped by the step."""
        m = np.ascontiguousarray(mask, dtype=np.uint8).reshape(self.N)
        _lib.check(self._L.pond_set_mask(self._ctx, m.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))))

    def get_mask(self):
        m = np.empty(self.N, dtype=np.uint8)
        _lib.check(self._L.pond_get_mask(self._ctx, m.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))))
        return m

    def set_positions(self, x):
        """Node positions (Cell::p.x) of a NONUNIFORM3 context: increasing, spanning less than Nx."""
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(self.N)
        _lib.check(self._L.pond_set_positions(self._ctx, _dp(x)))

    def get_positions(self):
        x = np.empty(self.N)
        _lib.check(self._L.pond_get_positions(self._ctx, _dp(x)))
        return x

    def amr_refine(self, tol=0.01):
        """AMR_add (amr.cu:1-27) on the current state; returns (added, limit_hits)."""
        a, h = ctypes.c_int64(), ctypes.c_int64()
        _lib.check(self._L.pond_amr_refine(self._ctx, float(tol), ctypes.byref(a), ctypes.byref(h)))
        return int(a.value), int(h.value)

    def amr_coarsen(self, tol=0.01):
        """AMR_remove (amr.cu:28-55) on the current state; returns the nodes removed."""
        r = ctypes.c_int64()
        _lib.check(self._L.pond_amr_coarsen(self._ctx, float(tol), ctypes.byref(r)))
        return int(r.value)

    # -- time-step rescaling (TimeCorr)
    def rescale_time(self, s):
        """u *= s, T *= s*s in the current state and dt *= s (update.cu:15-28)."""
        _lib.check(self._L.pond_rescale_time(self._ctx, float(s)))

    def set_dt_adapt(self, on=True, niter_hi=1000, niter_lo=4):
        """After every step: dt halves when NiterMax >= niter_hi, doubles when <= niter_lo (update.cu:121-123)."""
        _lib.check(self._L.pond_set_dt_adapt(self._ctx, 1 if on else 0, int(niter_hi), int(niter_lo)))

    @property
    def dt(self) -> float:
        return float(self.get_params().dt)

    def get_params(self):
        """The context's current pond_params (dt follows rescalings)."""
        p = _lib.PondParams()
        _lib.check(self._L.pond_get_params(self._ctx, ctypes.byref(p)))
        return p

    def set_strict(self, on=True):
        """Make step() raise PondError (status -6) after a step that left nodes at max_iter."""
        _lib.check(self._L.pond_set_strict(self._ctx, 1 if on else 0))

    def set_clock(self, istep, curtime, dt=0.0):
        """Step counter, simulated time and (if > 0) dt of a resumed run."""
        _lib.check(self._L.pond_set_clock(self._ctx, int(istep), float(curtime), float(dt)))

    # -- checkpoint / resume (no counterpart in the reference)
    def checkpoint(self, path):
        """Write everything the next step reads to one .npz (lbmpond_b200.checkpoint)."""
        from . import checkpoint
        checkpoint.save(self, path)

    @classmethod
    def resume(cls, path, device=0) -> "Solver":
        """A new Solver continuing a checkpointed run."""
        from . import checkpoint
        return checkpoint.load(path, device)

    def keep_niter(self, on=True):
        _lib.check(self._L.pond_keep_niter(self._ctx, 1 if on else 0))

    def niter(self):
        out = np.empty(self.N, dtype=np.int32)
        _lib.check(self._L.pond_get_niter(self._ctx, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))))
        return out

    def last_step_ms(self) -> float:
        ms = ctypes.c_float()
        _lib.check(self._L.pond_last_step_ms(self._ctx, ctypes.byref(ms)))
        return float(ms.value)

    def last_step_work(self) -> int:
        w = ctypes.c_int64()
        _lib.check(self._L.pond_last_step_work(self._ctx, ctypes.byref(w)))
        return int(w.value)

    def upload_native(self, f, rho, g):
        """Host arrays already in the context's precision (C-contiguous, ideally pinned)."""
        _lib.check(self._L.pond_upload_state(self._ctx, ctypes.c_void_p(f), ctypes.c_void_p(rho),
                                             ctypes.c_void_p(g)))

    def download_native(self, f=None, rho=None, g=None):
        """Copy the state to host arrays in the context's precision (any may be None)."""
        vp = lambda a: ctypes.c_void_p(a) if a else None  # noqa: E731
        _lib.check(self._L.pond_download_state(self._ctx, vp(f), vp(rho), vp(g)))

    def step_host(self, f, rho, g, rho_out=None, g_out=None):
        """Queue one plain step from host buffers in the context's precision
        (addresses of pinned arrays, as upload_native) and the read-back of the
        result's rho and g; returns at once.  Copies overlap neighbouring calls'
        steps.  The buffers must stay untouched until sync()."""
        vp = lambda a: ctypes.c_void_p(a) if a else None  # noqa: E731
        _lib.check(self._L.pond_step_host(self._ctx, vp(f), vp(rho), vp(g), vp(rho_out), vp(g_out)))

    def sync(self):
        """Wait for every queued step_host call."""
        _lib.check(self._L.pond_sync(self._ctx))

    def copy_state_from(self, other: "Solver"):
        """Device-side copy of another context's current state (precision converted)."""
        _lib.check(self._L.pond_copy_state(self._ctx, other._ctx))

    def stream(self) -> int:
        return int(self._L.pond_stream(self._ctx) or 0)

    def device_state(self):
        f, r, g = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        _lib.check(self._L.pond_device_state(self._ctx, ctypes.byref(f), ctypes.byref(r), ctypes.byref(g)))
        return f.value, r.value, g.value

    def draw_fields(self, names=None) -> dict:
        """The viewer's per-node fields (lbm_draw, lbm.cu:30-73; see
        lbmpond_b200.fields): rho, ux, mach, T, M4, f0..f8 by default, and
        "niter" when named (it needs keep_niter(True) before the last step)."""
        from .fields import FIELD_NAMES, draw_fields
        names = tuple(n for n in FIELD_NAMES if n != "niter") if names is None else tuple(names)
        f, rho, g = self.get_state()
        xi, _, tlat, _ = lattice_tables(self.lattice)
        niter = self.niter() if "niter" in names else None
        mask = self.get_mask() if self.params.interp in (GAP2, NONUNIFORM3) else None
        return draw_fields(f, rho, g, xi[:, 0], tlat, dt=self.dt, niter=niter, mask=mask, names=names)

    def drop(self, directory: str, fields=()):
        """Write Rho/Vx/Vy/Vz/T_%07d.arr for the current step (drop.cu:2-34),
        and one <Name>_%07d.arr per extra viewer field in `fields` (names of
        draw_fields, e.g. ("mach", "M4"))."""
        fl = self.fields()
        istep = self.diagnostics()["istep"]
        os.makedirs(directory, exist_ok=True)
        names = {"Rho": "rho", "Vx": "ux", "Vy": "uy", "Vz": "uz", "T": "T"}
        paths = []
        for prefix, key in names.items():
            path = os.path.join(directory, f"{prefix}_{istep:07d}.arr")
            write_arr(path, fl[key], self.shape)
            paths.append(path)
        if fields:
            for key, data in self.draw_fields(fields).items():
                path = os.path.join(directory, f"{key[0].upper() + key[1:]}_{istep:07d}.arr")
                write_arr(path, data, self.shape)
                paths.append(path)
        return paths


def write_arr(path: str, data, shape):
    """The reference's .arr layout (drop.cu:12-30): int32 comment length (0),
    int32 dim (3), int32 sizeof(value) (8), int32 Nx, Ny, Nz, then float64
    values with x fastest."""
    nx, ny, nz = shape
    with open(path, "wb") as fp:
        np.array([0, 3, 8, nx, ny, nz], dtype=np.int32).tofile(fp)
        np.ascontiguousarray(data, dtype=np.float64).reshape(nx * ny * nz).tofile(fp)


def read_arr(path: str):
    with open(path, "rb") as fp:
        clen = int(np.fromfile(fp, dtype=np.int32, count=1)[0])
        if clen:
            fp.read(clen)
        dim, size, nx, ny, nz = (int(v) for v in np.fromfile(fp, dtype=np.int32, count=5))
        dt = {8: np.float64, 4: np.float32}[size]
        data = np.fromfile(fp, dtype=dt, count=nx * ny * nz)
    return data, (nx, ny, nz)
