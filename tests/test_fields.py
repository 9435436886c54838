"""The viewer's derived fields (lbmpond_b200.fields, lbm_draw lbm.cu:30-73) and
the library's lattice tables, on the CPU (the GPU test that reads them off a
stepped context is in tests/test_zy_api_gpu.py)."""

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

