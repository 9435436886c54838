"""API round trips on the GPU, through the C ABI: a context resumed from a
checkpoint continues the run bit for bit, the viewer's derived fields and
.arr files of a stepped context equal the host formulas applied to its state,
and the strict mode turns an iteration-cap hit into an error status.
These exercise the host-side API around the step; the step's own parity with
the oracle is in the test_gpu_* files."""
import numpy as np
import pytest

from lbmpond_b200.fields import FIELD_NAMES, draw_fields


@pytest.mark.gpu
@pytest.mark.parametrize("interp,precision", [(4, "fp32"), (4, "fp64"), (9, "fp32"), (10, "fp64")])
def test_resumed_context_continues_the_run(tmp_path, pond, interp, precision):
    """Checkpoint after 3 steps, 2 more steps on the original and on a context
    resumed from the file: the same state bit for bit, the same clock."""
    nx = 64
    with pond.Solver(lattice="D1Q5", shape=(nx, 1, 1), interp=interp, precision=precision, tau=0.7, dt=0.5) as s:
        s.init("sod")
        if interp == 9:
            s.set_mask(np.arange(nx) % 3 != 1)
        if interp == 10:
            s.set_positions(np.arange(nx) + 0.2 * np.sin(2 * np.pi * np.arange(nx) / nx))
        s.step(3)
        path = str(tmp_path / "run.npz")
        s.checkpoint(path)
        s.step(2)
        a, da = s.get_state(), s.diagnostics()
    with pond.Solver.resume(path) as r:
        assert r.diagnostics()["istep"] == 3 and r.dt == 0.5
        r.step(2)
        b, db = r.get_state(), r.diagnostics()
        if interp in (9, 10):
            assert r.get_mask().sum() == (nx - nx // 3 if interp == 9 else nx)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    assert db["istep"] == da["istep"] == 5 and db["curtime"] == da["curtime"] == 2.5
    assert np.isclose(db["mass"], da["mass"], rtol=1e-14)


@pytest.mark.gpu
def test_solver_draw_fields_and_drop(tmp_path, pond):
    nx = 64
    with pond.Solver(lattice="D1Q5", shape=(nx, 1, 1), interp=pond.GAP2, precision="fp64", tau=0.7, dt=0.5) as s:
        s.init("sod")
        s.set_mask(np.arange(nx) % 4 != 2)
        s.keep_niter(True)
        s.step(2)
        out = s.draw_fields(FIELD_NAMES)
        f, rho, g = s.get_state()
        mask, niter = s.get_mask(), s.niter()
        xi, _, tlat, _ = pond.lattice_tables("D1Q5")
        expect = draw_fields(f, rho, g, xi[:, 0], tlat, dt=0.5, niter=niter, mask=mask)
        for name in FIELD_NAMES:
            assert np.array_equal(out[name], expect[name]), name
        assert out["niter"][mask == 1].min() >= 1
        paths = s.drop(str(tmp_path), fields=("mach", "M4"))
    names = sorted(p.rsplit("/", 1)[1] for p in paths)
    assert names == ["M4_0000002.arr", "Mach_0000002.arr", "Rho_0000002.arr", "T_0000002.arr",
                     "Vx_0000002.arr", "Vy_0000002.arr", "Vz_0000002.arr"]
    data, shape = pond.read_arr(str(tmp_path / "Mach_0000002.arr"))
    assert shape == (nx, 1, 1) and np.allclose(data, expect["mach"], equal_nan=True)


@pytest.mark.gpu
def test_strict_mode_reports_nonconvergence(pond):
    """With pond_set_strict a step that leaves nodes at max_iter returns
    POND_ERR_NOT_CONVERGED (the step itself is complete and counted); without
    it the same step succeeds and the count is in the diagnostics."""
    nx = 32
    kw = dict(lattice="D1Q5", shape=(nx, 1, 1), precision="fp64", tau=0.8, max_iter=1)
    with pond.Solver(**kw) as s:
        s.init("sod")
        s.step(1)
        assert s.diagnostics()["nonconverged"] > 0
    with pond.Solver(**kw) as s:
        s.init("sod")
        s.set_strict(True)
        with pytest.raises(pond.PondError) as e:
            s.step(3)
        assert e.value.status == -6
        d = s.diagnostics()
        assert d["istep"] == 1 and d["nonconverged"] > 0
        s.set_strict(False)
        s.step(1)
        assert s.diagnostics()["istep"] == 2
