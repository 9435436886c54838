"""The oracle's one-dimensional mesh paths (CPU only): the node mask with the
gap-bridging linear interpolation (steps.cu:1122-1149 propagate_nonequal_1D<2>),
node positions with the non-uniform quadratic (steps.cu:882-908
propagateNR_1D), AMR refinement and coarsening (amr.cu:1-55) and the
calcTotMoments sums (update.cu:52-69).

The reference ships these disabled and has no fixtures for them, so they
are pinned here to exact answers: the equivalences with the uniform schemes,
polynomial reproduction across gaps and on stretched meshes, the coarsening
pattern of a uniform field worked out by hand from amr.cu:29-54, and the
C restatement against a literal Python transcription of the same loops.
"""
import numpy as np
import pytest

from tests.states import smooth_state, sod_state


def _base(orc, rho, g):
    t = orc.tables(0)
    return orc.State(t.w[:, None] * rho[None, :], rho.copy(), g.copy())


def test_gap2_full_mask_is_linear_lagrange(orc):
    nx = 64
    rho, g = smooth_state((nx, 1, 1), 1, seed=1, modes=1, du=0.02)
    st = _base(orc, rho, g)
    a, _, _ = orc.step(st, 0, (nx, 1, 1), interp=orc.LAGR2, tau=0.8)
    for mask in (None, np.ones(nx, np.uint8)):
        b, _, nc = orc.step_mesh(st, nx, interp=orc.GAP2, mask=mask, tau=0.8)
        assert nc == 0
        for x, y in ((a.f, b.f), (a.rho, b.rho), (a.g, b.g)):
            assert np.allclose(x, y, rtol=0, atol=1e-15)


def test_nonuniform_on_uniform_positions_is_fixed_quadratic(orc):
    nx = 48
    rho, g = smooth_state((nx, 1, 1), 1, seed=2, modes=2, du=0.03)
    st = _base(orc, rho, g)
    a, _, _ = orc.step(st, 0, (nx, 1, 1), interp=orc.FIXED3, tau=0.7)
    for pos in (None, np.arange(nx, dtype=float)):
        b, _, nc = orc.step_mesh(st, nx, interp=orc.NONUNIFORM3, pos=pos, tau=0.7)
        assert nc == 0
        for x, y in ((a.f, b.f), (a.rho, b.rho), (a.g, b.g)):
            assert np.allclose(x, y, rtol=0, atol=1e-14)


def _one_iteration_expectation(orc, fstar, tau):
    """The first iterate f* of LBMpull followed by the BGK of steps.cu:557-564
    (max_iter = 1 stops after one iteration)."""
    t = orc.tables(0)
    rho = fstar.sum(axis=0)
    return fstar + (1 / tau) * (t.w[:, None] * rho[None, :] - fstar), rho


def test_gap2_reproduces_a_linear_profile_across_gaps(orc):
    """Uniform gauge, density linear in x: the transfer is the identity and
    the linear interpolation between the nearest active nodes is exact, so
    the first iterate is f_i = w_i rho(x - v_i) at every interior active node."""
    nx, u0, T0, tau = 64, 0.05, 0.1, 0.7
    rng = np.random.default_rng(5)
    mask = np.ones(nx, np.uint8)
    x = 1
    while x < nx - 1:  # gaps of at most two inactive nodes
        k = int(rng.integers(0, 3))
        mask[x:x + k] = 0
        x += k + 1
    rho = 1 + 0.01 * np.arange(nx)
    st = orc.base_state(0, rho, u0, 0, 0, T0)
    out, _, _ = orc.step_mesh(st, nx, interp=orc.GAP2, mask=mask, tau=tau, max_iter=1)
    t = orc.tables(0)
    v = np.sqrt(T0 / t.tlat) * t.xi[:, 0] + u0
    xs = np.arange(nx)
    fstar = t.w[:, None] * (1 + 0.01 * (xs[None, :] - v[:, None]))
    fexp, rexp = _one_iteration_expectation(orc, fstar, tau)
    sel = (mask == 1) & (xs >= 8) & (xs < nx - 8)
    assert np.allclose(out.f[:, sel], fexp[:, sel], rtol=0, atol=1e-14)
    assert np.allclose(out.rho[sel], rexp[sel], rtol=0, atol=1e-14)
    # inactive nodes are carried over
    assert np.array_equal(out.f[:, mask == 0], st.f[:, mask == 0])
    assert np.array_equal(out.g[:, mask == 0], st.g[:, mask == 0])


def test_nonuniform_reproduces_a_quadratic_profile(orc):
    """Stretched positions, density quadratic in position, uniform gauge: the
    three-point Lagrange basis on the node positions is exact for quadratics."""
    nx, u0, T0, tau = 64, -0.04, 0.08, 0.8
    xs = np.arange(nx)
    pos = xs + 0.3 * np.sin(2 * np.pi * xs / nx)
    prof = lambda p: 1 + 0.01 * p + 0.0005 * p * p  # noqa: E731
    st = orc.base_state(0, prof(pos), u0, 0, 0, T0)
    out, _, _ = orc.step_mesh(st, nx, interp=orc.NONUNIFORM3, pos=pos, tau=tau, max_iter=1)
    t = orc.tables(0)
    v = np.sqrt(T0 / t.tlat) * t.xi[:, 0] + u0
    fstar = t.w[:, None] * prof(pos[None, :] - v[:, None])
    fexp, rexp = _one_iteration_expectation(orc, fstar, tau)
    sel = (xs >= 2) & (xs < nx - 2)
    assert np.allclose(out.f[:, sel], fexp[:, sel], rtol=0, atol=1e-13)
    assert np.allclose(out.rho[sel], rexp[sel], rtol=0, atol=1e-13)


def test_nonuniform_periodic_seam(orc):
    """The abscissae lifted by Nx across the seam: on positions that are a
    uniform shift of the nodes (p = x + 0.25), a uniform state stays a fixed
    point everywhere, seam nodes included."""
    nx = 20
    st = orc.base_state(0, np.full(nx, 0.9), 0.03, 0, 0, 0.2)
    out, _, nc = orc.step_mesh(st, nx, interp=orc.NONUNIFORM3, pos=np.arange(nx) + 0.25, tau=0.6)
    assert nc == 0
    assert np.allclose(out.f, st.f, rtol=1e-12, atol=1e-15)
    assert np.allclose(out.g, st.g, rtol=1e-11, atol=1e-14)


def test_mesh_sums(orc):
    nx = 40
    rho, g = smooth_state((nx, 1, 1), 1, seed=4, modes=1, du=0.02)
    st = _base(orc, rho, g)
    d = orc.diagnostics(st, 0, (nx, 1, 1))
    s = orc.mesh_sums(st)
    assert np.isclose(s["mass"], d["mass"], rtol=1e-14) and np.isclose(s["enrg"], d["enrg"], rtol=1e-14)
    mask = (np.arange(nx) % 3 != 0).astype(np.uint8)
    s = orc.mesh_sums(st, mask=mask)
    assert np.isclose(s["mass"], rho[mask == 1].sum(), rtol=1e-14)
    # cell widths of a stretched periodic mesh add up to its length Nx
    pos = np.arange(nx) + 0.4 * np.sin(2 * np.pi * np.arange(nx) / nx)
    one = orc.State(st.f, np.ones(nx), st.g)
    assert np.isclose(orc.mesh_sums(one, pos=pos)["mass"], nx, rtol=1e-14)


def test_amr_refine_known_answer(orc):
    """Every other node active, a density jump between nodes 14 and 16 and
    across the seam (30 -> 0): exactly nodes 15 and 31 are activated, each
    holding the average of its two neighbours' records."""
    nx = 32
    mask = (np.arange(nx) % 2 == 0).astype(np.uint8)
    rho = np.where(np.arange(nx) < 16, 1.0, 0.125)
    g = np.zeros((4, nx)); g[3] = np.where(np.arange(nx) < 16, 1.0, 0.8)
    st = _base(orc, rho, g)
    out, m, added, hits = orc.amr_refine(st, mask)
    assert added == 2 and hits == 0
    assert np.flatnonzero(m != mask).tolist() == [15, 31]
    for mid, a, b in ((15, 14, 16), (31, 30, 0)):
        assert out.rho[mid] == 0.5 * (rho[a] + rho[b])
        assert np.array_equal(out.g[:, mid], 0.5 * (g[:, a] + g[:, b]))
        assert np.array_equal(out.f[:, mid], 0.5 * (st.f[:, a] + st.f[:, b]))
    untouched = np.ones(nx, bool); untouched[[15, 31]] = False
    assert np.array_equal(out.f[:, untouched], st.f[:, untouched])
    # adjacent active nodes over the threshold are counted (pairs 15-16 and
    # 31-0); the gap 16..20 joins two equal records and is left alone
    mask2 = np.ones(nx, np.uint8); mask2[17:20] = 0
    _, m2, added2, hits2 = orc.amr_refine(st, mask2)
    assert hits2 == 2 and added2 == 0 and np.array_equal(m2, mask2)
    # an odd distance between unequal records is not split either
    mask3 = np.ones(nx, np.uint8); mask3[13:16] = 0  # node 12 -> 16: distance 4, split at 14
    mask3[[0, 1]] = 0  # node 31 -> 2: distance 3, not split
    _, m3, added3, _ = orc.amr_refine(st, mask3)
    assert added3 == 1 and np.flatnonzero(m3 != mask3).tolist() == [14]


def _coarsen_literal(rho, g, mask, tol):
    """amr.cu:29-54, transcribed loop for loop."""
    m = mask.copy()
    nx = m.size
    for ix in range(nx):
        if m[ix] == 0:
            continue
        xm, xp, dM, dP = ix, ix, 0, 0
        while True:
            xm = (xm - 1 + nx) % nx; dM += 1
            if m[xm] != 0:
                break
        while True:
            xp = (xp + 1) % nx; dP += 1
            if m[xp] != 0:
                break
        vm, vp = g[0, xm] - g[0, ix], g[0, xp] - g[0, ix]
        T0 = g[3, ix]
        if (vm * vm / T0 < tol and vp * vp / T0 < tol and abs(rho[xp] / rho[ix] - 1) < tol
                and abs(rho[xm] / rho[ix] - 1) < tol and dM < 4 and dP < 4):
            m[ix] = 0
    return m


@pytest.mark.parametrize("seed", range(6))
def test_amr_coarsen_matches_the_literal_pass(orc, seed):
    rng = np.random.default_rng(seed)
    nx = int(rng.integers(3, 90))
    mask = (rng.random(nx) < rng.uniform(0.3, 1.0)).astype(np.uint8)
    rho = 1 + rng.choice([0.0, 0.002, 0.05], size=nx) * rng.standard_normal(nx)
    g = np.zeros((4, nx))
    g[0] = rng.choice([0.0, 0.002, 0.1], size=nx) * rng.standard_normal(nx)
    g[3] = rng.uniform(0.3, 0.6, size=nx)
    st = orc.State(np.zeros((5, nx)), rho, g)
    m, removed = orc.amr_coarsen(st, mask)
    lit = _coarsen_literal(rho, g, mask, 0.01)
    assert np.array_equal(m, lit)
    assert removed == int(mask.sum() - lit.sum())


def test_amr_coarsen_uniform_field_keeps_every_fourth_node(orc):
    """All nodes active and equal: node 0 goes (neighbours at distance 1),
    then 1 and 2 (left neighbour at distance 2 and 3), node 3 stays (its left
    neighbour is 4 away), and so on: nodes 3, 7, 11, ... remain."""
    nx = 32
    st = orc.base_state(0, np.ones(nx), 0.01, 0, 0, 0.5)
    m, removed = orc.amr_coarsen(st, np.ones(nx, np.uint8))
    assert np.flatnonzero(m).tolist() == list(range(3, nx, 4))
    assert removed == nx - nx // 4


def test_mesh_step_rejects_walls(orc):
    """The mesh schemes are periodic (steps.cu:1128-1130, :891-893)."""
    import ctypes
    rho, g = sod_state(16)
    st = _base(orc, rho, g)
    p = orc._mesh_params(16, orc.GAP2)
    p.bc[0] = orc.BC_CLAMP
    out = [st.f.copy(), st.rho.copy(), st.g.copy()]
    nc = orc.lib().orc_step_mesh(ctypes.byref(p), orc._dp(st.f), orc._dp(st.rho), orc._dp(st.g), None, None,
                                 *[orc._dp(a) for a in out], None)
    assert nc < 0


def test_amr_sod_characterisation(orc):
    """The reference's AMR on a periodic Sod tube (400 nodes, gamma 3, tau
    0.55, 120 steps, GAP2), started on every other node with refinement and
    coarsening after every step: it keeps well under half the nodes active
    and stays within a few percent (L1 in rho, central half, away from the
    seam's second jump) of the exact solution, coarser than the full grid."""
    from tests.riemann import sample
    nx, steps, lam2 = 400, 120, 0.01
    x = np.arange(nx)
    left, right = (1.0, 0.0, lam2), (0.125, 0.0, lam2 * 0.1 / 0.125)
    rho = np.where(x < nx // 2, left[0], right[0])
    g = np.stack([np.zeros(nx), np.zeros(nx), np.zeros(nx), np.where(x < nx // 2, left[2], right[2])])
    t = orc.tables(0)
    st0 = orc.State(t.w[:, None] * rho[None, :], rho.copy(), g)
    er = sample((left[0], 0.0, left[0] * left[2]), (right[0], 0.0, right[0] * right[2]), 3.0,
                (x - (nx / 2 - 0.5)) / steps)[0]
    mid = (x > nx * 0.25) & (x < nx * 0.75)

    def l1(st, mask):
        m = mid & (mask == 1)
        return float(np.abs(st.rho[m] - er[m]).mean() / er[m].mean())

    st = st0.copy()
    for _ in range(steps):
        st, _, nc = orc.step_mesh(st, nx, interp=orc.GAP2, tau=0.55)
        assert nc == 0
    full = l1(st, np.ones(nx, np.uint8))
    st, mask, active = st0.copy(), (x % 2 == 0).astype(np.uint8), []
    for _ in range(steps):
        st, _, nc = orc.step_mesh(st, nx, interp=orc.GAP2, mask=mask, tau=0.55)
        assert nc == 0
        st, mask, _, _ = orc.amr_refine(st, mask, 0.01)
        mask, _ = orc.amr_coarsen(st, mask, 0.01)
        active.append(int(mask.sum()))
    amr = l1(st, mask)
    assert full < 0.02 and full < amr < 0.05, (full, amr)
    assert 90 < min(active) and max(active) < 200, (min(active), max(active))


def test_nonuniform_sod_on_a_stretched_mesh(orc):
    """NONUNIFORM3 on a Sod tube (400 nodes, gamma 3, tau 0.55, 120 steps)
    with the positions stretched by +-0.1 node: every node converges and the
    density's L1 distance to the exact solution (central half) stays within
    10 % of the uniform mesh's."""
    from tests.riemann import sample
    nx, steps, lam2 = 400, 120, 0.01
    x = np.arange(nx)
    left, right = (1.0, 0.0, lam2), (0.125, 0.0, lam2 * 0.1 / 0.125)
    t = orc.tables(0)

    def l1(pos):
        p = x.astype(float) if pos is None else pos
        rho = np.where(p < nx / 2, left[0], right[0])
        g = np.stack([np.zeros(nx), np.zeros(nx), np.zeros(nx), np.where(p < nx / 2, left[2], right[2])])
        st = orc.State(t.w[:, None] * rho[None, :], rho.copy(), g)
        for _ in range(steps):
            st, _, nc = orc.step_mesh(st, nx, interp=orc.NONUNIFORM3, pos=pos, tau=0.55)
            assert nc == 0
        er = sample((left[0], 0.0, left[0] * left[2]), (right[0], 0.0, right[0] * right[2]), 3.0,
                    (p - (nx / 2 - 0.5)) / steps)[0]
        mid = (p > nx * 0.25) & (p < nx * 0.75)
        return float(np.abs(st.rho[mid] - er[mid]).mean() / er[mid].mean())

    uniform = l1(None)
    stretched = l1(x + 0.1 * np.sin(2 * np.pi * x / nx))
    assert uniform < 0.02 and abs(stretched / uniform - 1) < 0.1, (uniform, stretched)
