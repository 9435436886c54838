"""GPU parity of the one-dimensional mesh path (through the C ABI) with the
FP64 oracle: the gap-bridging and non-uniform steps, the mask-aware
diagnostics, AMR refinement and coarsening, and time-step rescaling.

Tolerances: steps as in test_gpu_parity (FP64 1e-9, FP32 3e-5 relative to
the field's scale); AMR masks bit-exact in both precisions (the oracle is
fed the state the GPU holds, so both decide on the same numbers); refined
records bit-exact in float64 and equal to the float32 rounding of the
oracle's float64 averages in float32.
"""
import numpy as np
import pytest

from tests.states import perturbed_populations, smooth_state, sod_state
from tests.test_gpu_parity import TOL, _compare

pytestmark = pytest.mark.gpu


def _mesh_state(orc, nx, kind, seed):
    if kind == "sod":
        rho, g = sod_state(nx)
    else:
        rho, g = smooth_state((nx, 1, 1), 1, seed=seed, modes=2, du=0.03)
    f = perturbed_populations(orc, 0, rho, g, seed=seed, eps=0.01)
    return orc.State(f, rho, g)


def _random_mask(nx, seed, density=0.7):
    rng = np.random.default_rng(seed)
    m = (rng.random(nx) < density).astype(np.uint8)
    m[::5] = 1  # gaps of at most four nodes
    return m


def _stretched(nx, amp=0.3):
    x = np.arange(nx, dtype=np.float64)
    return x + amp * np.sin(2 * np.pi * x / nx)


def _solver(pond, nx, interp, precision, tau=0.8):
    return pond.Solver(lattice="D1Q5", shape=(nx, 1, 1), interp=interp, precision=precision, tau=tau)


def _float_state(st, precision):
    """The state a float32 context holds: every value rounded to float32."""
    if precision == "fp64":
        return st
    r = lambda a: a.astype(np.float32).astype(np.float64)  # noqa: E731
    return type(st)(r(st.f), r(st.rho), r(st.g))


CASES = [
    ("GAP2", "smooth", 128), ("GAP2", "sod", 200), ("GAP2", "smooth", 97),
    ("NONUNIFORM3", "smooth", 128), ("NONUNIFORM3", "sod", 200), ("NONUNIFORM3", "smooth", 3),
]


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("scheme,kind,nx", CASES)
def test_mesh_step_parity(orc, pond, scheme, kind, nx, precision):
    interp = getattr(pond, scheme)
    st = _float_state(_mesh_state(orc, nx, kind, seed=nx), precision)
    mask = _random_mask(nx, seed=nx)
    pos = _stretched(nx) if scheme == "NONUNIFORM3" else None
    with _solver(pond, nx, interp, precision) as s:
        s.set_state(st.rho, st.g, f=st.f)
        s.set_mask(mask)
        if pos is not None:
            s.set_positions(pos)
        ref = st
        for _ in range(3):
            s.step(1)
            ref, _, nc = orc.step_mesh(ref, nx, interp=interp, mask=mask, pos=pos, tau=0.8)
        out = s.get_state()
        d = s.diagnostics()
        assert np.array_equal(s.get_mask(), mask)
    _compare(out, ref, TOL[precision], f"{scheme} {kind} {nx} {precision}")
    f, rho, g = out
    # inactive nodes are carried over unchanged through every step
    assert np.array_equal(f[:, mask == 0], _float_state(st, precision).f[:, mask == 0])
    # the step's conservation sums: active nodes, cell-width weighted on the stretched mesh
    sums = orc.mesh_sums(orc.State(f, rho, g), mask=mask, pos=pos)
    tol = 1e-12 if precision == "fp64" else 1e-6
    assert np.isclose(d["mass"], sums["mass"], rtol=tol)
    assert np.isclose(d["enrg"], sums["enrg"], rtol=tol)
    if precision == "fp64":  # same tolerances as the oracle
        assert d["nonconverged"] == nc


def test_mesh_diagnostics_before_a_step(orc, pond):
    nx = 64
    st = _mesh_state(orc, nx, "smooth", 3)
    mask, pos = _random_mask(nx, 3), _stretched(nx, 0.2)
    with _solver(pond, nx, pond.NONUNIFORM3, "fp64") as s:
        s.set_state(st.rho, st.g, f=st.f)
        s.set_mask(mask)
        s.set_positions(pos)
        d = s.diagnostics()
        assert np.allclose(s.get_positions(), pos, rtol=0, atol=0)
    sums = orc.mesh_sums(st, mask=mask, pos=pos)
    assert np.isclose(d["mass"], sums["mass"], rtol=1e-13)
    assert np.isclose(d["moment"][0], sums["moment"], rtol=1e-12, atol=1e-14)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("nx,stride", [(32, 2), (256, 2), (1001, 3), (4096, 4)])
def test_amr_refine_parity(orc, pond, nx, stride, precision):
    rho, g = sod_state(nx)
    g[0] = 0.05 * np.sin(2 * np.pi * np.arange(nx) / nx)
    st0 = _float_state(orc.State(perturbed_populations(orc, 0, rho, g, seed=1, eps=0.01), rho, g), precision)
    mask = (np.arange(nx) % stride == 0).astype(np.uint8)
    with _solver(pond, nx, pond.GAP2, precision) as s:
        s.set_state(st0.rho, st0.g, f=st0.f)
        s.set_mask(mask)
        added, hits = s.amr_refine(0.01)
        m = s.get_mask()
        out = s.get_state()
    ref, mref, aref, href = orc.amr_refine(st0, mask, 0.01)
    assert np.array_equal(m, mref) and added == aref and hits == href
    assert added > 0
    if precision == "fp32":
        ref = _float_state(ref, "fp32")
    for a, b in ((out[0], ref.f), (out[1], ref.rho), (out[2], ref.g)):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("nx", [3, 5, 7, 8, 9, 64, 67, 1000, 4099, 70001])
def test_amr_coarsen_parity(orc, pond, nx, precision):
    """Parallel prefix over the pass's automaton against the serial pass:
    small grids (serial path), one and many chunks, ragged chunk ends."""
    for seed in range(3):
        rng = np.random.default_rng(seed * 1000 + nx)
        mask = (rng.random(nx) < rng.uniform(0.4, 1.0)).astype(np.uint8)
        rho = 1 + rng.choice([0.0, 0.002, 0.05], size=nx) * rng.standard_normal(nx)
        g = np.zeros((4, nx))
        g[0] = rng.choice([0.0, 0.002, 0.1], size=nx) * rng.standard_normal(nx)
        g[3] = rng.uniform(0.3, 0.6, size=nx)
        t = orc.tables(0)
        st = _float_state(orc.State(t.w[:, None] * rho[None, :], rho, g), precision)
        with _solver(pond, nx, pond.GAP2, precision) as s:
            s.set_state(st.rho, st.g, f=st.f)
            s.set_mask(mask)
            removed = s.amr_coarsen(0.01)
            m = s.get_mask()
        mref, rref = orc.amr_coarsen(st, mask, 0.01)
        assert np.array_equal(m, mref), (nx, seed, np.flatnonzero(m != mref)[:10])
        assert removed == rref


def test_amr_coarsen_uniform_field(pond):
    nx = 1 << 16
    with _solver(pond, nx, pond.GAP2, "fp32") as s:
        s.init("uniform", 1.0, 0.01, 0.0, 0.0, 0.5)
        assert s.amr_coarsen(0.01) == nx - nx // 4
        assert np.flatnonzero(s.get_mask()).tolist() == list(range(3, nx, 4))
        s.step(1)
        assert s.diagnostics()["niter_mean"] > 0


def test_amr_cycle_lockstep(orc, pond):
    """Sod tube on a coarse mask, float64: step, refine, coarsen, twenty
    times.  Each operation is checked against the oracle applied to the
    state the GPU held before it."""
    nx = 400
    rho, g = sod_state(nx)
    t = orc.tables(0)
    st = orc.State(t.w[:, None] * rho[None, :], rho, g)
    mask = (np.arange(nx) % 2 == 0).astype(np.uint8)
    with _solver(pond, nx, pond.GAP2, "fp64", tau=0.6) as s:
        s.set_state(st.rho, st.g, f=st.f)
        s.set_mask(mask)
        totals = [0, 0]
        for _ in range(20):
            f, r, gg = s.get_state()
            cur = orc.State(f, r, gg)
            s.step(1)
            ref, _, _ = orc.step_mesh(cur, nx, interp=orc.GAP2, mask=mask, tau=0.6)
            _compare(s.get_state(), ref, TOL["fp64"], "cycle step")
            f, r, gg = s.get_state()
            cur = orc.State(f, r, gg)
            added, _ = s.amr_refine(0.01)
            ref, mask, aref, _ = orc.amr_refine(cur, mask, 0.01)
            assert added == aref and np.array_equal(s.get_mask(), mask)
            f, r, gg = s.get_state()
            assert np.array_equal(f, ref.f) and np.array_equal(gg, ref.g)
            removed = s.amr_coarsen(0.01)
            mask, rref = orc.amr_coarsen(ref, mask, 0.01)
            assert removed == rref and np.array_equal(s.get_mask(), mask)
            totals[0] += added
            totals[1] += removed
        assert totals[0] > 0 and totals[1] > 0


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_rescale_time(orc, pond, precision):
    nx = 64
    st = _mesh_state(orc, nx, "smooth", 7)
    with pond.Solver(lattice="D1Q5", shape=(nx, 1, 1), interp=pond.LAGR4, precision=precision, tau=0.8, dt=0.25) as s:
        s.set_state(st.rho, st.g, f=st.f)
        s.step(1)
        f0, r0, g0 = s.get_state()
        d0 = s.diagnostics()
        s.rescale_time(0.5)
        f1, r1, g1 = s.get_state()
        d1 = s.diagnostics()
        assert s.dt == 0.125
        assert np.array_equal(f1, f0) and np.array_equal(r1, r0)
        assert np.array_equal(g1[:3], 0.5 * g0[:3]) and np.array_equal(g1[3], 0.25 * g0[3])
        assert d1["mass"] == d0["mass"] and d1["moment"][0] == 0.5 * d0["moment"][0]
        assert d1["enrg"] == 0.25 * d0["enrg"]
        with pytest.raises(pond.PondError):
            s.rescale_time(0.0)


def test_dt_adapt_policy(orc, pond):
    """A uniform state converges in very few iterations, so NiterMax <= 4
    doubles dt after every step (update.cu:121-122), curtime advancing by the
    dt in force during the step."""
    nx = 32
    with pond.Solver(lattice="D1Q5", shape=(nx, 1, 1), interp=pond.LAGR4, precision="fp64", dt=0.01) as s:
        s.init("uniform", 1.0, 0.002, 0.0, 0.0, 0.1)
        s.set_dt_adapt(True, 1000, 4)
        s.step(3)
        d = s.diagnostics()
        assert d["niter_max"] <= 4
        assert np.isclose(s.dt, 0.08) and np.isclose(d["curtime"], 0.01 + 0.02 + 0.04)
        fl = s.fields()
        assert np.allclose(fl["ux"], 0.002 * 8) and np.allclose(fl["T"], 0.1 * 64)
        s.set_dt_adapt(False)
        s.step(1)
        assert np.isclose(s.dt, 0.08)


def test_mesh_argument_errors(pond):
    with pytest.raises(pond.PondError):  # mesh schemes are one-dimensional
        pond.Solver(lattice="D1Q5", shape=(16, 2, 1), interp=pond.GAP2)
    with pytest.raises(pond.PondError):  # and periodic
        pond.Solver(lattice="D1Q5", shape=(16, 1, 1), interp=pond.GAP2, bc=("clamp", "periodic", "periodic"))
    with pond.Solver(lattice="D1Q5", shape=(16, 1, 1), interp=pond.LAGR4) as s:
        with pytest.raises(pond.PondError):
            s.set_mask(np.ones(16))
    with _solver(pond, 16, pond.NONUNIFORM3, "fp32") as s:
        s.init("uniform")
        with pytest.raises(pond.PondError):
            s.set_positions(np.arange(16)[::-1])
        with pytest.raises(pond.PondError):
            s.set_positions(np.arange(16) * 1.5)  # spans Nx or more
        with pytest.raises(pond.PondError):
            s.amr_coarsen(0.0)
        with pytest.raises(pond.PondError):
            s.set_dt_adapt(True, 4, 4)


def test_init_reactivates_the_mesh(pond):
    """pond_init's fill sets every node active and p_x = x (init.cu:100-106)."""
    nx = 64
    with _solver(pond, nx, pond.NONUNIFORM3, "fp32") as s:
        s.init("sod")
        s.set_mask(np.arange(nx) % 3 == 0)
        s.set_positions(_stretched(nx))
        s.init("uniform")
        assert np.array_equal(s.get_mask(), np.ones(nx, np.uint8))
        assert np.array_equal(s.get_positions(), np.arange(nx, dtype=np.float64))
        s.step(1)
        assert s.diagnostics()["nonconverged"] == 0
