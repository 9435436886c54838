"""Checkpoint / resume (lbmpond_b200.checkpoint) on the CPU: the file format,
the Solver arguments it recreates, and the order in which a resume loads the
state.  A stand-in object plays the CUDA context; the GPU round trip (a
resumed context stepping bit for bit like the original) is in
tests/test_zy_api_gpu.py."""
import ctypes

import numpy as np
import pytest

from lbmpond_b200 import _lib, checkpoint


class FakeSolver:
    def __init__(self, lattice=0, shape=(16, 1, 1), interp=4, ddf=0, seed=0):
        rng = np.random.default_rng(seed)
        self.p = _lib.PondParams()
        ctypes.memset(ctypes.byref(self.p), 0, ctypes.sizeof(self.p))
        self.p.lattice, self.p.interp, self.p.precision = lattice, interp, 1
        self.p.tau, self.p.dt, self.p.tol_abs, self.p.tol_rel, self.p.max_iter = 0.7, 0.125, 1e-12, 1e-10, 100
        self.p.bc[0], self.p.bc[1], self.p.bc[2] = 0, 1, 2
        self.p.ddf, self.p.ddf_dof = ddf, 4 if ddf else 0
        self.shape = shape
        N = int(np.prod(shape))
        Q = {0: 5, 1: 27, 2: 125}[lattice]
        self.f, self.rho, self.g = rng.random((Q, N)), rng.random(N), rng.random((4, N))
        self.h = rng.random((Q, N)) if ddf else None
        self.mask = (rng.random(N) < 0.6).astype(np.uint8)
        self.pos = np.arange(N) + 0.1 * rng.random(N)
        self.calls = []

    def get_params(self):
        return self.p

    def diagnostics(self):
        return {"istep": 42, "curtime": 5.25}

    def get_state(self):
        return self.f.copy(), self.rho.copy(), self.g.copy()

    def get_energy(self):
        return self.h.copy()

    def get_mask(self):
        return self.mask.copy()

    def get_positions(self):
        return self.pos.copy()

    def set_state(self, rho, g, f=None):
        self.calls.append(("state", f, rho, g))

    def set_energy(self, h):
        self.calls.append(("energy", h))

    def set_mask(self, m):
        self.calls.append(("mask", m))

    def set_positions(self, x):
        self.calls.append(("positions", x))

    def set_clock(self, istep, curtime, dt):
        self.calls.append(("clock", istep, curtime, dt))


@pytest.mark.parametrize("interp,ddf", [(4, 0), (4, 1), (9, 0), (10, 0)])
def test_roundtrip_and_restore_order(tmp_path, interp, ddf):
    src = FakeSolver(interp=interp, ddf=ddf, seed=interp + ddf)
    path = str(tmp_path / "run.ckpt.npz")
    checkpoint.save(src, path)
    d = checkpoint.read(path)
    assert int(d["istep"]) == 42 and float(d["curtime"]) == 5.25 and float(d["dt"]) == 0.125
    assert np.array_equal(d["f"], src.f) and np.array_equal(d["g"], src.g) and np.array_equal(d["rho"], src.rho)
    assert ("h" in d) == bool(ddf)
    assert ("mask" in d) == (interp in (9, 10)) and ("positions" in d) == (interp == 10)
    kw = checkpoint.solver_kwargs(d, device=3)
    assert kw["shape"] == (16, 1, 1) and kw["bc"] == (0, 1, 2) and kw["device"] == 3
    assert kw["interp"] == interp and kw["precision"] == 1 and kw["tol_abs"] == 1e-12 and kw["dt"] == 0.125
    assert kw.get("ddf_dof") == (4 if ddf else None)
    dst = FakeSolver(interp=interp, ddf=ddf, seed=99)
    checkpoint.restore(dst, d)
    kinds = [c[0] for c in dst.calls]
    assert kinds[0] == "state" and kinds[-1] == "clock"  # the state first: it resets the energy populations
    assert np.array_equal(dst.calls[0][1], src.f)
    assert dst.calls[-1][1:] == (42, 5.25, 0.125)
    if ddf:
        assert np.array_equal(dict((c[0], c) for c in dst.calls)["energy"][1], src.h)
    if interp == 10:
        assert np.array_equal(dict((c[0], c) for c in dst.calls)["positions"][1], src.pos)


def test_read_rejects_other_files(tmp_path):
    path = str(tmp_path / "x.npz")
    np.savez(path, f=np.zeros(3))
    with pytest.raises(ValueError):
        checkpoint.read(path)


def test_set_clock_validates_before_device(pond):
    L = _lib.load()
    assert L.pond_set_clock(None, 1, 0.0, 1.0) == -1
    assert L.pond_set_strict(None, 1) == -1
    assert L.pond_status_string(-6).decode() == "iteration did not converge"

