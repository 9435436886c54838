"""CPU tests of the FP64 oracle: lattice tables, the gauge transform's moment
invariants (the property the reference's fgauge*.py scripts check by eye,
e.g. fgauge_D1Q5.py:69-72), interpolation weights, and step-level
invariants.  The oracle is pinned to the reference's own kernels by
tests/test_golden.py."""
import numpy as np
import pytest

from tests.states import perturbed_populations, smooth_state

LATS = [0, 1, 2]  # D1Q5, D3Q27, D3Q125


@pytest.mark.parametrize("lat", LATS)
def test_tables(orc, lat):
    t = orc.tables(lat)
    assert t.Q == {0: 5, 1: 27, 2: 125}[lat]
    assert abs(t.w.sum() - 1) < 1e-14
    # second moment per axis equals TLat; odd moments vanish
    for a in range(int(t.dim)):
        assert abs(np.sum(t.w * t.xi[:, a] ** 2) - t.tlat) < 1e-14
        assert abs(np.sum(t.w * t.xi[:, a])) < 1e-14
        assert abs(np.sum(t.w * t.xi[:, a] ** 3)) < 1e-14
    if lat != 1:  # the 5-speed sets also carry the fourth moment 3 TLat^2
        assert abs(np.sum(t.w * t.xi[:, 0] ** 4) - 3 * t.tlat ** 2) < 1e-13


def test_d3q27_tables_match_reference_listing(orc):
    # consts.h:20-30 directions and :38-47 weights (W by number of nonzero components)
    t = orc.tables(1)
    e = t.e
    assert e[1].tolist() == [1, 0, 0] and e[7].tolist() == [1, 1, 1] and e[26].tolist() == [-1, -1, -1]
    TL = 1.0 / 3.0
    W = [(1 - TL) ** 3, (1 - TL) ** 2 * TL / 2, (1 - TL) * TL * TL / 4, TL ** 3 / 8]
    for i in range(27):
        assert abs(t.w[i] - W[int(np.count_nonzero(e[i]))]) < 1e-16
    # consts.h:62-65 reverse maps
    rx = [0, 8, 2, 3, 9, 10, 6, 11, 1, 4, 5, 7, 12, 13, 20, 21, 16, 22, 18, 23, 14, 15, 17, 19, 24, 26, 25]
    ry = [0, 1, 12, 3, 14, 5, 13, 15, 8, 20, 10, 21, 2, 6, 4, 7, 16, 17, 24, 25, 9, 11, 22, 26, 18, 19, 23]
    rz = [0, 1, 2, 16, 4, 17, 18, 19, 8, 9, 22, 23, 12, 24, 14, 25, 3, 5, 6, 7, 20, 26, 10, 11, 13, 15, 21]
    r = orc.reverse_maps(1)
    assert r[0].tolist() == rx and r[1].tolist() == ry and r[2].tolist() == rz


def _moments(t, f, uT, maxdeg):
    v = np.sqrt(uT[3] / t.tlat) * t.xi + np.asarray(uT[:3])
    out = []
    rng_y = range(maxdeg + 1) if t.dim == 3 else [0]
    for a in range(maxdeg + 1):
        for b in rng_y:
            for c in rng_y:
                out.append(np.sum(f * v[:, 0] ** a * v[:, 1] ** b * v[:, 2] ** c))
    return np.array(out)


@pytest.mark.parametrize("lat", LATS)
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_transfer_gauge_preserves_moments(orc, lat, seed):
    t = orc.tables(lat)
    rng = np.random.default_rng(seed)
    f = t.w * (1 + 0.2 * rng.standard_normal(t.Q))
    d3 = t.dim == 3
    src = np.array([rng.uniform(-.1, .1), rng.uniform(-.1, .1) * d3, rng.uniform(-.1, .1) * d3, rng.uniform(.05, .2)])
    dst = np.array([rng.uniform(-.1, .1), rng.uniform(-.1, .1) * d3, rng.uniform(-.1, .1) * d3, rng.uniform(.05, .2)])
    g = np.array([orc.transfer_gauge(lat, f, src, dst, i) for i in range(t.Q)])
    maxdeg = 2 if lat == 1 else 4
    ms, md = _moments(t, f, src, maxdeg), _moments(t, g, dst, maxdeg)
    assert np.allclose(ms, md, rtol=1e-11, atol=1e-12)
    # round trip back to the source gauge
    back = np.array([orc.transfer_gauge(lat, g, dst, src, i) for i in range(t.Q)])
    assert np.allclose(back, f, rtol=1e-10, atol=1e-13)
    # identity transfer
    same = np.array([orc.transfer_gauge(lat, f, src, src, i) for i in range(t.Q)])
    assert np.allclose(same, f, rtol=1e-12, atol=1e-15)


@pytest.mark.parametrize("lat", LATS)
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_transfer_through_reference_gauge(orc, lat, seed):
    """The tile kernels transfer every staged node once per step into a
    reference gauge R and, per iteration, apply the transfer R -> target.
    That equals the direct transfer source -> target because the Lagrange
    basis of the transfer reproduces the polynomials it is built from;
    checked here on the reference's own transfer (transfer_gauge)."""
    t = orc.tables(lat)
    rng = np.random.default_rng(10 + seed)
    f = t.w * (1 + 0.2 * rng.standard_normal(t.Q))
    d3 = t.dim == 3

    def gauge():
        return np.array([rng.uniform(-.1, .1), rng.uniform(-.1, .1) * d3, rng.uniform(-.1, .1) * d3,
                         rng.uniform(.05, .2)])
    src, ref, dst = gauge(), gauge(), gauge()
    direct = np.array([orc.transfer_gauge(lat, f, src, dst, i) for i in range(t.Q)])
    f_ref = np.array([orc.transfer_gauge(lat, f, src, ref, i) for i in range(t.Q)])
    via = np.array([orc.transfer_gauge(lat, f_ref, ref, dst, i) for i in range(t.Q)])
    assert np.allclose(via, direct, rtol=1e-10, atol=1e-13 * np.abs(f).max())


@pytest.mark.parametrize("lat", LATS)
def test_set_base_and_moments(orc, lat):
    t = orc.tables(lat)
    uT = [0.03, -0.02 if t.dim == 3 else 0, 0.01 if t.dim == 3 else 0, 0.12]
    f = orc.set_base(lat, 1.7, uT)
    assert np.allclose(f, 1.7 * t.w)
    vi = np.sqrt(uT[3] / t.tlat) * t.xi + np.array(uT[:3])
    rho, m = orc.calc_moments(lat, f, vi)
    assert abs(rho - 1.7) < 1e-14
    assert np.allclose(m, uT, atol=1e-14)


@pytest.mark.parametrize("n", [2, 3, 4, 5])
def test_lagrange_weights(orc, n):
    rng = np.random.default_rng(n)
    for _ in range(5):
        s = rng.uniform(0, n - 1, 3)
        w = np.array([[[orc.lagr_pol(n, i, j, k, *s) for k in range(n)] for j in range(n)] for i in range(n)])
        assert abs(w.sum() - 1) < 1e-12
        # reproduces linear functions exactly
        gx = np.arange(n)[:, None, None] * np.ones((n, n, n))
        assert abs(np.sum(w * gx) - s[0]) < 1e-12


@pytest.mark.parametrize("lat,shape,interp", [(0, (64, 1, 1), 4), (0, (64, 1, 1), 3), (0, (64, 1, 1), 7),
                                              (0, (64, 1, 1), 8), (1, (6, 5, 4), 4), (1, (6, 5, 4), 3),
                                              (2, (4, 4, 3), 6)])
def test_uniform_state_is_fixed_point(orc, lat, shape, interp):
    t = orc.tables(lat)
    N = int(np.prod(shape))
    uT = [0.02, 0.01 if t.dim == 3 else 0, -0.01 if t.dim == 3 else 0, 0.1]
    st = orc.base_state(lat, np.full(N, 1.3), *uT)
    out, niter, nc = orc.step(st, lat, shape, interp=interp)
    assert nc == 0
    assert np.allclose(out.rho, 1.3, atol=1e-12)
    for k in range(4):
        assert np.allclose(out.g[k], uT[k], atol=1e-12)
    assert np.allclose(out.f, st.f, atol=1e-12)


@pytest.mark.parametrize("lat,shape,tol", [(0, (96, 1, 1), 1e-5), (1, (12, 10, 8), 2e-3)])
def test_mass_and_energy_drift_small(orc, lat, shape, tol):
    t = orc.tables(lat)
    rho, g = smooth_state(shape, int(t.dim), seed=3, modes=1)
    st = orc.base_state(lat, rho, *g)
    d0 = orc.diagnostics(st, lat, shape)
    for _ in range(3):
        st, niter, nc = orc.step(st, lat, shape)
        assert nc == 0
    d1 = orc.diagnostics(st, lat, shape)
    # semi-Lagrangian PonD is not conservative by construction; the drift is
    # interpolation error and falls at third order with resolution
    assert abs(d1["mass"] - d0["mass"]) / d0["mass"] < tol
    assert abs(d1["enrg"] - d0["enrg"]) / d0["enrg"] < 10 * tol


def test_step_rejects_bad_params(orc):
    st = orc.base_state(0, np.ones(8), 0, 0, 0, 0.1)
    with pytest.raises(ValueError):
        orc.step(st, 0, (8, 1, 1), max_iter=0)


def test_guess_changes_only_start(orc):
    # a perfect starting guess reaches the same fixed point
    shape = (48, 1, 1)
    rho, g = smooth_state(shape, 1, seed=4)
    st = orc.base_state(0, rho, *g)
    st.f = perturbed_populations(orc, 0, rho, g, seed=4)
    out, n0, _ = orc.step(st, 0, shape)
    out2, n1, _ = orc.step(st, 0, shape, guess=out.g)
    assert np.allclose(out2.g, out.g, rtol=1e-9, atol=1e-11)
    assert np.allclose(out2.f, out.f, rtol=1e-9, atol=1e-11)
    assert n1.mean() <= n0.mean()


def test_weno5_row_equals_weno5_on_1d_grids(orc):
    """On a 1D grid the reference's smoothness row (y = z = floor(crd.x+0.5),
    wrapped) and the row through the departure point are both row 0."""
    from tests.states import perturbed_populations, smooth_state
    shape = (64, 1, 1)
    rho, g = smooth_state(shape, 1, seed=5, modes=2)
    st = orc.State(perturbed_populations(orc, 0, rho, g, seed=5), rho, g)
    a, na, _ = orc.step(st, 0, shape, interp=orc.WENO5, tau=0.7)
    b, nb, _ = orc.step(st, 0, shape, interp=orc.WENO5_ROW, tau=0.7)
    assert np.array_equal(a.f, b.f) and np.array_equal(a.g, b.g) and np.array_equal(na, nb)


@pytest.mark.parametrize("lat,interp", [(2, 6), (2, 11), (1, 8)])
def test_inflow_ghost_equals_clamp_on_an_equilibrium_face(orc, lat, interp):
    """The inflow ghost holds set_base(rho, u, T) of the inflow state; when the
    x = 0 face is uniform, at equilibrium and in that state, one step with
    inflow/outflow in x equals one step with zero gradient at both x ends."""
    from tests.states import smooth_state
    shape = (7, 4, 3)
    rho, g = smooth_state(shape, 3, seed=8, modes=1, du=0.01)
    face = np.arange(rho.size) % shape[0] == 0
    state0 = (1.05, 0.1, -0.02, 0.01, 0.11)
    rho[face] = state0[0]
    for k in range(4):
        g[k][face] = state0[1 + k]
    t = orc.tables(lat)
    f = t.w[:, None] * rho[None, :]
    st = orc.State(f, rho, g)
    a, na, nca = orc.step(st, lat, shape, interp=interp, tau=0.8, bc=(3, 0, 0), inflow=state0)
    b, nb, ncb = orc.step(st, lat, shape, interp=interp, tau=0.8, bc=(1, 0, 0))
    assert nca == 0 and ncb == 0
    assert np.array_equal(a.f, b.f) and np.array_equal(a.g, b.g)


@pytest.mark.parametrize("lat,interp,T0", [(2, 6, 0.1), (2, 11, 0.1), (1, 11, 0.25)])
def test_uniform_inflow_flow_is_a_fixed_point(orc, lat, interp, T0):
    shape = (8, 3, 3)
    N = int(np.prod(shape))
    state0 = (1.0, 0.3, 0.0, 0.0, T0)
    g = np.zeros((4, N)); g[0] = state0[1]; g[3] = T0
    rho = np.full(N, 1.0)
    t = orc.tables(lat)
    st = orc.State(t.w[:, None] * rho[None, :], rho, g)
    for _ in range(2):
        st, niter, nc = orc.step(st, lat, shape, interp=interp, tau=0.9, bc=(3, 0, 0), inflow=state0)
        assert nc == 0
    assert np.abs(st.rho - 1).max() < 1e-13 and np.abs(st.g[0] - 0.3).max() < 1e-13
    assert np.abs(st.g[3] - T0).max() < 1e-13
