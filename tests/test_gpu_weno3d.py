"""GPU parity of the 3D WENO5 step (propagateWENO<3,5>, steps.cu:774-825, on
D3Q27 and D3Q125) and of the inflow/outflow boundary, through the C ABI,
against the FP64 oracle.

Tolerances as in tests/test_gpu_parity.py: float64 1e-9 and float32 3e-5
relative to the largest value (u relative to sqrt(T)).  The states are
smooth with small velocities: with the reference's smoothness row
(y = z = floor(crd.x+0.5), steps.cu:783) larger perturbations leave a few
float64 nodes cycling at the iteration cap in the oracle itself."""
import numpy as np
import pytest

from tests.states import perturbed_populations, smooth_state
from tests.test_gpu_parity import TOL, _compare

pytestmark = pytest.mark.gpu

WENO5, WENO5_ROW, FIXED3 = 8, 11, 6


def _pair(orc, pond, lat, shape, interp, precision, tau=0.8, nsteps=2, seed=4, du=0.01, bc=(0, 0, 0), inflow=None,
          ux_shift=0.0):
    # D3Q27 (TLat = 1/3) at T = 0.2: at lower temperatures some float64 nodes of
    # the oracle cycle at the iteration cap on these random non-equilibrium states
    T0 = 0.2 if lat == 1 else 0.1
    rho, g = smooth_state(shape, 3, seed=seed, modes=1, du=du, T0=T0)
    if inflow is not None:  # a flow along x into the box
        g[0] += inflow[1]
    g[0] += ux_shift
    st = orc.State(perturbed_populations(orc, lat, rho, g, seed=seed, eps=0.01), rho, g)
    names = {0: "periodic", 1: "clamp", 2: "mirror", 3: "inflow"}
    with pond.Solver(lattice=lat, shape=shape, interp=interp, precision=precision, tau=tau,
                     bc=tuple(names[b] for b in bc)) as s:
        s.set_state(st.rho, st.g, f=st.f)
        if inflow is not None:
            s.set_inflow(*inflow)
        ref = st
        for _ in range(nsteps):
            s.step(1)
            ref, niter, nc = orc.step(ref, lat, shape, interp=interp, tau=tau, bc=bc, inflow=inflow)
            assert nc == 0
        out = s.get_state()
        d = s.diagnostics()
    return out, ref, niter, d


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("lat,shape,interp,seed", [
    (1, (9, 6, 5), WENO5, 4), (1, (9, 6, 5), WENO5_ROW, 4), (1, (12, 8, 8), WENO5, 4),
    (2, (7, 5, 4), WENO5, 3), (2, (7, 5, 4), WENO5_ROW, 3), (2, (10, 6, 6), WENO5_ROW, 4),
])
def test_weno3d_matches_oracle(orc, pond, lat, shape, interp, seed, precision):
    out, ref, niter, d = _pair(orc, pond, lat, shape, interp, precision, seed=seed)
    _compare(out, ref, TOL[precision], f"lat {lat} {shape} interp {interp} {precision}")
    if precision == "fp64":
        assert d["niter_max"] == int(niter.max()) and d["nonconverged"] == 0


@pytest.mark.parametrize("shift", [0.7, -0.75])
def test_weno_tile_fast_flow_matches_oracle(orc, pond, shift):
    """D3Q125 WENO5 (row through the departure point) in float32 runs the
    staged tile; with |u_x| + 2.86 sqrt(T) > 1.5 some x windows leave the
    tile's halo and those iterations read global memory instead."""
    out, ref, niter, d = _pair(orc, pond, 2, (9, 5, 4), WENO5_ROW, "fp32", seed=5, ux_shift=shift)
    _compare(out, ref, TOL["fp32"], f"fast flow {shift}")


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("lat,shape,interp", [(2, (9, 5, 4), FIXED3), (2, (9, 5, 4), WENO5_ROW),
                                              (1, (10, 6, 5), WENO5_ROW)])
def test_inflow_outflow_matches_oracle(orc, pond, lat, shape, interp, precision):
    """Inflow ghost below x = 0 (equilibrium of the inflow state), zero
    gradient above x = Nx-1, periodic y and z."""
    T = 0.1 if lat == 2 else 0.2
    inflow = (1.02, 0.2, 0.01, -0.01, T * 1.05)
    out, ref, niter, d = _pair(orc, pond, lat, shape, interp, precision, bc=(3, 0, 0), inflow=inflow)
    _compare(out, ref, TOL[precision], f"inflow lat {lat} interp {interp} {precision}")


@pytest.mark.parametrize("lat,interp", [(2, FIXED3), (2, WENO5_ROW), (1, WENO5)])
def test_uniform_inflow_is_a_fixed_point(pond, lat, interp):
    """A box filled with the inflow state stays in it: the ghost, the
    zero-gradient outflow and every interior node agree."""
    shape = (12, 4, 4)
    N = int(np.prod(shape))
    rho0, u0, T0 = 1.0, 0.3, 0.1 if lat == 2 else 0.25
    with pond.Solver(lattice=lat, shape=shape, interp=interp, precision="fp64", tau=0.9,
                     bc=("inflow", "periodic", "periodic")) as s:
        g = np.zeros((4, N)); g[0] = u0; g[3] = T0
        s.set_state(np.full(N, rho0), g)
        s.set_inflow(rho0, u0, 0.0, 0.0, T0)
        s.step(3)
        f, rho, gg = s.get_state()
    assert np.abs(rho - rho0).max() < 1e-12
    assert np.abs(gg[0] - u0).max() < 1e-12 and np.abs(gg[1:3]).max() < 1e-12
    assert np.abs(gg[3] - T0).max() < 1e-12


def test_inflow_needs_its_state(pond):
    with pond.Solver(lattice=2, shape=(8, 4, 4), interp=WENO5_ROW, precision="fp32",
                     bc=("inflow", "periodic", "periodic")) as s:
        s.init("uniform", 1.0, 0.1, 0.0, 0.0, 0.1)
        with pytest.raises(pond.PondError):
            s.step(1)
        with pytest.raises(pond.PondError):
            s.set_inflow(-1.0, 0.0, 0.0, 0.0, 0.1)
        s.set_inflow(1.0, 0.1, 0.0, 0.0, 0.1)
        s.step(1)
