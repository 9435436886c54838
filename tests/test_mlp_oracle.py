"""CPU checks of the float64 predictor oracle (oracle/mlp.py): its analytic
gradient against central finite differences, and its features on simple
states."""
import numpy as np
import pytest

from oracle import mlp as M


@pytest.mark.parametrize("H", [64, 128])
def test_gradient_matches_finite_differences(H):
    rng = np.random.default_rng(H)
    n = 96
    npar = H * M.NIN + H + H * H + H + M.NOUT * H + M.NOUT
    p = rng.standard_normal(npar) * 0.2
    Xs = rng.standard_normal((n, M.NIN))
    Ys = rng.standard_normal((n, M.NOUT))
    loss, g = M.loss_and_grad(p, H, Xs, Ys)
    idx = rng.choice(npar, 40, replace=False)
    eps = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += eps
        pm[i] -= eps
        fd = (M.loss_and_grad(pp, H, Xs, Ys)[0] - M.loss_and_grad(pm, H, Xs, Ys)[0]) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd))


def test_features_of_uniform_state_are_zero_differences():
    shape = (6, 5, 4)
    N = 120
    rho = np.full(N, 1.3)
    g = np.stack([np.full(N, 0.01), np.full(N, -0.02), np.zeros(N), np.full(N, 0.09)])
    F, nonuni = M.features(rho, g, shape)
    assert not nonuni.any()
    assert np.allclose(F[:, 5:], 0)
    c = np.sqrt(0.09 * 3)
    assert np.allclose(F[:, 0], c) and np.allclose(F[:, 1], 0.01 / c) and np.allclose(F[:, 4], 0.27)


def test_features_see_a_single_perturbed_node():
    shape = (6, 6, 6)
    N = 216
    rho = np.ones(N)
    g = np.stack([np.zeros(N), np.zeros(N), np.zeros(N), np.full(N, 0.1)])
    rho[0] = 1.5  # node (0,0,0)
    F, nonuni = M.features(rho, g, shape)
    # itself and its six periodic face neighbours see it
    assert nonuni.sum() == 7
    assert abs(F[1, 5] - 0.5) < 1e-15          # node (1,0,0): its -x neighbour is node 0
    assert abs(F[5, 10] - 0.5) < 1e-15         # node (5,0,0): +x neighbour wraps to node 0
