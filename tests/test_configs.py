"""The configuration presets (lbmpond_b200.configs) on the CPU: their Solver
parameters pass the library's own validation, and the host-built initial
states have the physics they claim."""
import numpy as np
import pytest

from lbmpond_b200 import configs


@pytest.mark.parametrize("name", sorted(configs.PRESETS))
def test_presets_pass_parameter_validation(pond, name):
    """pond_create checks every parameter before it touches a device: here
    (no GPU) a valid preset gets as far as the device query."""
    try:
        s = pond.Solver(**configs.solver_kwargs(name, size=8))
    except pond.PondError as e:
        assert e.status == -2, str(e)  # POND_ERR_CUDA: validation passed
    else:
        s.close()


@pytest.mark.parametrize("gamma", [5.0 / 3.0, 1.4])
def test_shock_vortex_rankine_hugoniot(gamma):
    """Away from the vortex the two states satisfy the jump conditions of a
    stationary shock: mass, momentum and energy fluxes are continuous
    (p = rho T, enthalpy gamma/(gamma-1) p/rho)."""
    n = 32
    rho, g = configs.shock_vortex_state(n, gamma=gamma)
    x = (np.arange(n) + 0.5) / n
    X, Y, _ = np.meshgrid(x, x, x, indexing="ij")
    flat = lambda a: np.ascontiguousarray(a.transpose(2, 1, 0)).ravel()  # noqa: E731
    far = flat(np.abs(Y - 0.5) > 0.3)
    pre, post = far & flat(X < 0.5), far & flat(X > 0.5)
    ux, T = g[0], g[3]
    p = rho * T

    def fluxes(sel):
        r, u, pp = rho[sel].mean(), ux[sel].mean(), p[sel].mean()
        return np.array([r * u, r * u * u + pp, u * (0.5 * r * u * u + gamma / (gamma - 1) * pp)])

    f1, f2 = fluxes(pre), fluxes(post)
    assert np.allclose(f1, f2, rtol=1e-12)
    c1 = np.sqrt(gamma * T[pre].mean())
    assert np.isclose(ux[pre].mean() / c1, 1.5)  # Mach 1.5 upstream


def test_sphere_state_volume():
    n = 48
    rho, g = configs.sphere_state(n)
    inside = rho == 1.0
    assert abs(inside.mean() / (4 / 3 * np.pi * 0.2 ** 3) - 1) < 0.03
    p = rho * g[3] / configs.SPHERE_LAMBDA ** 2
    assert np.allclose(p[inside], 1.0) and np.allclose(p[~inside], 0.1)
    assert not g[:3].any()


@pytest.mark.parametrize("gamma", [5.0 / 3.0, 1.4])
def test_tgv_mach(gamma):
    U0, T0, rho0, gm = configs.tgv_params(gamma)
    assert gm == gamma and rho0 == 1.0 and np.isclose(T0, 1.0 / 12.0)
    assert np.isclose(U0 / np.sqrt(gamma * T0), 0.5)


def test_batch_problems():
    (lengths, rho, u, T), kw, steps = configs.batch_problems(64, seed=0)
    assert lengths.size == 64 and rho.size == int(lengths.sum()) and kw["interp"] == 8 and steps == 1000


def test_preset_overrides():
    kw = configs.solver_kwargs("sod_d1q5", size=200, precision="fp32")
    assert kw["shape"] == (200, 1, 1) and kw["precision"] == "fp32" and kw["interp"] == 7
    assert configs.solver_kwargs("sphere_d3q27")["shape"] == (256, 256, 256)
