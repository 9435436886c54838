"""The viewer's derived fields (lbmpond_b200.fields, lbm_draw lbm.cu:30-73) and
the library's lattice tables, on the CPU; one GPU test reads them off a
stepped context."""
import ctypes

import numpy as np
import pytest

from lbmpond_b200 import _lib
from lbmpond_b200.fields import FIELD_NAMES, draw_fields


@pytest.mark.parametrize("lat", [0, 1, 2])
def test_lattice_tables_match_the_oracle(orc, pond, lat):
    xi, w, tlat, dim = pond.lattice_tables(lat)
    t = orc.tables(lat)
    assert np.array_equal(xi, t.xi) and np.array_equal(w, t.w)
    assert tlat == t.tlat and dim == t.dim
    L = _lib.load()
    assert L.pond_lattice_tables(lat, None, None, None) == 0
    assert L.pond_lattice_tables(9, None, None, None) == -1


@pytest.mark.parametrize("lat", [0, 1, 2])
@pytest.mark.parametrize("dt", [1.0, 0.25])
def test_equilibrium_fourth_moment(pond, lat, dt):
    """f_i = w_i rho in the node's gauge: the Gauss-Hermite lattices reproduce
    the Maxwellian's fourth moment, M4 = rho (3 T^2 + 6 T u^2 + u^4) in the
    viewer's units (u / dt, T / dt^2)."""
    xi, w, tlat, _ = pond.lattice_tables(lat)
    rng = np.random.default_rng(lat)
    N = 50
    rho = rng.uniform(0.5, 2.0, N)
    g = np.stack([rng.uniform(-0.1, 0.1, N), rng.uniform(-0.1, 0.1, N), np.zeros(N), rng.uniform(0.05, 0.4, N)])
    f = w[:, None] * rho[None, :]
    out = draw_fields(f, rho, g, xi[:, 0], tlat, dt=dt)
    assert "niter" not in out
    u, T = g[0] / dt, g[3] / dt / dt
    assert np.allclose(out["M4"], rho * (3 * T * T + 6 * T * u * u + u ** 4), rtol=1e-12)
    assert np.allclose(out["mach"], g[0] / np.sqrt(g[3]), rtol=1e-14)
    assert np.array_equal(out["rho"], rho) and np.allclose(out["ux"], u) and np.allclose(out["T"], T)
    for i in range(9):
        expect = f[i] if i < f.shape[0] else np.zeros(N)
        assert np.array_equal(out[f"f{i}"], expect)


def test_mask_and_niter():
    xi = np.array([0.0, 1.0, -1.0, 2.0, -2.0])
    N = 6
    f = np.ones((5, N)); rho = np.ones(N); g = np.zeros((4, N)); g[3] = 0.5
    mask = np.array([1, 0, 1, 1, 0, 1], np.uint8)
    out = draw_fields(f, rho, g, xi, 1.0, niter=np.arange(N), mask=mask)
    for name in FIELD_NAMES:
        assert not out[name][mask == 0].any()
    assert np.array_equal(out["niter"], np.where(mask == 1, np.arange(N), 0))
    with pytest.raises(ValueError):
        draw_fields(f, rho, g, xi, 1.0, names=("niter",))
    with pytest.raises(ValueError):
        draw_fields(f, rho, g, xi, 1.0, names=("vorticity",))


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
