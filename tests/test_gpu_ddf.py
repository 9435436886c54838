"""GPU parity of the double-distribution extension (energy populations) with
the float64 oracle, through the C ABI.

A D1Q5, D3Q27 or D3Q125 context made with ``ddf_dof`` carries energy
populations h beside f;
its temperature comes from them and gamma = (Dim + dof + 2) / (Dim + dof).
The oracle restates the same extension (``orc.step(..., dof=...)``); both are
pinned to physics by ``tests/test_ddf_oracle.py`` (exact Riemann solutions).

Tolerances as in ``test_gpu_parity.py``: float64 1e-9, float32 3e-5 of each
quantity's scale (u against sqrt(T)).
"""
import numpy as np
import pytest

from tests.riemann import sample
from tests.states import perturbed_populations, smooth_state, sod_state

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-9, "fp32": 3e-5}


def _state(orc, nx, kind, seed, dof):
    if kind == "sod":
        rho, g = sod_state(nx)
    else:
        rho, g = smooth_state((nx, 1, 1), 1, seed=seed, modes=1, du=0.03)
    f = perturbed_populations(orc, 0, rho, g, seed=seed, eps=0.01)
    st = orc.with_energy(orc.State(f, rho, g), 0, dof)
    rng = np.random.default_rng(100 + seed)
    st.h = st.h * (1 + 0.01 * rng.standard_normal(st.h.shape))  # off equilibrium, like f
    return st


def _errors(s, ref):
    f, rho, g = s.get_state()
    h = s.get_energy()
    cs = np.sqrt(np.abs(ref.g[3]).max())
    return {"f": np.abs(f - ref.f).max() / np.abs(ref.f).max(),
            "h": np.abs(h - ref.h).max() / np.abs(ref.h).max(),
            "rho": np.abs(rho - ref.rho).max() / np.abs(ref.rho).max(),
            "u": np.abs(g[:3] - ref.g[:3]).max() / cs,
            "T": np.abs(g[3] - ref.g[3]).max() / np.abs(ref.g[3]).max()}


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("interp,kind", [(2, "smooth"), (3, "smooth"), (4, "smooth"), (5, "smooth"),
                                         (4, "sod"), (7, "sod"), (8, "sod")])
def test_energy_step_matches_oracle(orc, pond, interp, kind, precision):
    nx, dof, tau, bc = 97, 4, 0.6, ("clamp",) * 3
    st = _state(orc, nx, kind, seed=interp, dof=dof)
    with pond.Solver(lattice="D1Q5", shape=(nx, 1, 1), interp=interp, precision=precision, tau=tau, bc=bc,
                     ddf_dof=dof) as s:
        s.set_state(st.rho, st.g, f=st.f)
        s.set_energy(st.h)
        ref = st
        for _ in range(3):
            s.step(1)
            ref, niter, nc = orc.step(ref, 0, (nx, 1, 1), interp=interp, tau=tau, bc=(1, 1, 1), dof=dof,
                                      tol_abs=s.params.tol_abs, tol_rel=s.params.tol_rel)
        err = _errors(s, ref)
        d = s.diagnostics()
    assert all(v <= TOL[precision] for v in err.values()), err
    assert d["nonconverged"] == 0
    f, rho, g = ref.f, ref.rho, ref.g
    total = np.sum(rho * (np.sum(g[:3] ** 2, axis=0) + (1 + dof) * g[3]))
    assert abs(d["enrg"] - total) <= 1e-6 * abs(total)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("interp,shape,bc", [(2, (8, 6, 4), (0, 0, 0)), (3, (9, 6, 5), (1, 0, 2)),
                                             (4, (9, 7, 5), (0, 0, 0)), (4, (8, 8, 6), (2, 1, 0))])
def test_d3q27_energy_step_matches_oracle(orc, pond, interp, shape, bc, precision):
    dof, tau = 2, 0.7
    N = int(np.prod(shape))
    rho, g = smooth_state(shape, 3, seed=interp, modes=1, du=0.03)
    f = perturbed_populations(orc, 1, rho, g, seed=interp, eps=0.01)
    st = orc.with_energy(orc.State(f, rho, g), 1, dof)
    st.h = st.h * (1 + 0.01 * np.random.default_rng(7).standard_normal(st.h.shape))
    names = {0: "periodic", 1: "clamp", 2: "mirror"}
    with pond.Solver(lattice="D3Q27", shape=shape, interp=interp, precision=precision, tau=tau,
                     bc=tuple(names[b] for b in bc), ddf_dof=dof) as s:
        s.set_state(st.rho, st.g, f=st.f)
        s.set_energy(st.h)
        ref = st
        for _ in range(2):
            s.step(1)
            ref, niter, nc = orc.step(ref, 1, shape, interp=interp, tau=tau, bc=bc, dof=dof,
                                      tol_abs=s.params.tol_abs, tol_rel=s.params.tol_rel)
        err = _errors(s, ref)
        d = s.diagnostics()
    assert all(v <= TOL[precision] for v in err.values()), err
    assert d["nonconverged"] == 0 and N > 0
    total = np.sum(ref.rho * (np.sum(ref.g[:3] ** 2, axis=0) + (3 + dof) * ref.g[3]))
    assert abs(d["enrg"] - total) <= 1e-6 * abs(total)


@pytest.mark.parametrize("interp,bc", [(2, (0, 2, 1)), (3, (2, 0, 0)), (4, (0, 0, 0)), (4, (1, 2, 2))])
def test_d3q27_energy_tile_spans_several_ctas(orc, pond, interp, bc):
    """The float32 energy tile kernel (8 x 4 x 4 nodes per CTA, f and h on
    paired warps) on a box of 3 x 3 x 3 ragged tiles."""
    dof, tau, shape = 2, 0.7, (20, 9, 10)
    rho, g = smooth_state(shape, 3, seed=20 + interp, modes=2, du=0.04, T0=0.2)
    f = perturbed_populations(orc, 1, rho, g, seed=20 + interp, eps=0.01)
    st = orc.with_energy(orc.State(f, rho, g), 1, dof)
    st.h = st.h * (1 + 0.01 * np.random.default_rng(11).standard_normal(st.h.shape))
    names = {0: "periodic", 1: "clamp", 2: "mirror"}
    with pond.Solver(lattice="D3Q27", shape=shape, interp=interp, precision="fp32", tau=tau,
                     bc=tuple(names[b] for b in bc), ddf_dof=dof) as s:
        s.set_state(st.rho, st.g, f=st.f)
        s.set_energy(st.h)
        ref = st
        for _ in range(3):
            s.step(1)
            ref, niter, nc = orc.step(ref, 1, shape, interp=interp, tau=tau, bc=bc, dof=dof,
                                      tol_abs=s.params.tol_abs, tol_rel=s.params.tol_rel)
        err = _errors(s, ref)
        d = s.diagnostics()
    assert all(v <= TOL["fp32"] for v in err.values()), err
    assert d["nonconverged"] == 0 and d["niter_max"] >= 2


@pytest.mark.parametrize("interp", [2, 3, 4])
def test_d3q27_energy_departures_beyond_staged_halo(orc, pond, interp):
    """A fast, hot flow sends departure points past the energy tile's +-2
    halo; those lanes read f and h from global memory."""
    dof, tau, shape = 2, 0.8, (40, 6, 4)
    rho, g = smooth_state(shape, 3, seed=9, modes=1, du=0.05)
    g[0] += 0.75
    g[3] = 0.12 * (1 + 0.1 * np.sin(np.arange(rho.size)))
    f = perturbed_populations(orc, 1, rho, g, seed=9, eps=0.01)
    st = orc.with_energy(orc.State(f, rho, g), 1, dof)
    with pond.Solver(lattice="D3Q27", shape=shape, interp=interp, precision="fp32", tau=tau, ddf_dof=dof) as s:
        s.set_state(st.rho, st.g, f=st.f)
        s.set_energy(st.h)
        ref = st
        for _ in range(2):
            s.step(1)
            ref, niter, nc = orc.step(ref, 1, shape, interp=interp, tau=tau, dof=dof,
                                      tol_abs=s.params.tol_abs, tol_rel=s.params.tol_rel)
        err = _errors(s, ref)
    assert all(v <= TOL["fp32"] for v in err.values()), err


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
@pytest.mark.parametrize("shape,bc", [((5, 4, 4), (0, 0, 0)), ((9, 6, 5), (1, 0, 2))])
def test_d3q125_energy_step_matches_oracle(orc, pond, shape, bc, precision):
    """The staged D3Q125 tile kernel with energy populations (float32: 4^3
    tiles; float64: 2^3 tiles)."""
    dof, tau = 2, 0.9
    rho, g = smooth_state(shape, 3, seed=5, modes=1, du=0.03)
    f = perturbed_populations(orc, 2, rho, g, seed=5, eps=0.01)
    st = orc.with_energy(orc.State(f, rho, g), 2, dof)
    st.h = st.h * (1 + 0.01 * np.random.default_rng(9).standard_normal(st.h.shape))
    names = {0: "periodic", 1: "clamp", 2: "mirror"}
    with pond.Solver(lattice="D3Q125", shape=shape, precision=precision, tau=tau,
                     bc=tuple(names[b] for b in bc), ddf_dof=dof) as s:
        s.set_state(st.rho, st.g, f=st.f)
        s.set_energy(st.h)
        ref = st
        for _ in range(2):
            s.step(1)
            ref, niter, nc = orc.step(ref, 2, shape, interp=6, tau=tau, bc=bc, dof=dof,
                                      tol_abs=s.params.tol_abs, tol_rel=s.params.tol_rel)
        err = _errors(s, ref)
        d = s.diagnostics()
    assert all(v <= TOL[precision] for v in err.values()), err
    assert d["nonconverged"] == 0
    total = np.sum(ref.rho * (np.sum(ref.g[:3] ** 2, axis=0) + (3 + dof) * ref.g[3]))
    assert abs(d["enrg"] - total) <= 1e-6 * abs(total)


def test_sod_gamma_14_on_the_gpu(orc, pond):
    """200 float64 steps of the 400-node Sod tube with dof = 4: the same
    state as the oracle, and the exact gamma = 1.4 solution to 1.5 % (L1)."""
    nx, steps, dof = 400, 200, 4
    rho, g = sod_state(nx)
    with pond.Solver(lattice="D1Q5", shape=(nx, 1, 1), interp=7, precision="fp64", tau=0.55,
                     bc=("clamp",) * 3, ddf_dof=dof) as s:
        s.set_state(rho, g)
        s.step(steps)
        _, r_gpu, g_gpu = s.get_state()
    t = orc.tables(0)
    st = orc.with_energy(orc.State(t.w[:, None] * rho[None, :], rho.copy(), g.copy()), 0, dof)
    for _ in range(steps):
        st, _, _ = orc.step(st, 0, (nx, 1, 1), interp=7, tau=0.55, bc=(1, 1, 1), dof=dof)
    assert np.abs(r_gpu - st.rho).max() <= 1e-7 and np.abs(g_gpu[3] - st.g[3]).max() <= 1e-8
    x = (np.arange(nx) - (nx / 2 - 0.5)) / steps
    er, _, ep = sample((1.0, 0.0, 0.01), (0.125, 0.0, 0.001), 1.4, x)
    assert np.abs(r_gpu - er).mean() / er.mean() < 0.015
    assert np.abs(r_gpu * g_gpu[3] - ep).mean() / ep.mean() < 0.02


def test_energy_api(orc, pond):
    nx = 32
    rho, g = sod_state(nx)
    with pond.Solver(lattice="D1Q5", shape=(nx, 1, 1), interp=4, precision="fp64", ddf_dof=2) as s:
        s.set_state(rho, g)
        h_eq = orc.with_energy(orc.State(np.zeros((5, nx)), rho, g), 0, 2).h
        assert np.allclose(s.get_energy(), h_eq, rtol=1e-14, atol=0)  # set_state puts h at equilibrium
        h = h_eq * 1.01
        s.set_energy(h)
        assert np.array_equal(s.get_energy(), h)
        s.init("sod")  # built-in initial conditions fill h as well
        assert np.all(s.get_energy()[0] > 0)
        with pytest.raises(pond._lib.PondError):  # the host-buffer pipeline carries no h
            f = np.zeros((5, nx))
            s.step_host(f.ctypes.data, rho.ctypes.data, g.ctypes.data)
    with pond.Solver(lattice="D1Q5", shape=(nx, 1, 1), interp=4) as s:
        s.set_state(rho, g)
        with pytest.raises(pond._lib.PondError):
            s.get_energy()
    with pytest.raises(pond._lib.PondError):  # no energy populations on the D3Q27 WENO5 schemes
        pond.Solver(lattice="D3Q27", shape=(8, 4, 4), interp=pond.WENO5, ddf_dof=2)
