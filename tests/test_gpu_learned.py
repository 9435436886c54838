"""GPU tests of the learned starting gauge: the BF16 tensor-core network
against the float64 oracle (oracle/mlp.py), the training pairs against the
oracle's features, and the learned step against the plain step (same fixed
point, fewer iterations).

Tolerances (BF16 operands, float32 accumulation):
  forward outputs      |d| <= 3e-2 * std(output)
  gradients            ||d||_2 <= 6e-2 * ||g||_2 per parameter tensor
"""
import numpy as np
import pytest

from oracle import mlp as M

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    return torch


def _random_data(n, seed, scale=1.0):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((n, M.NIN)) * rng.uniform(0.01, 2.0, M.NIN) + rng.uniform(-1, 1, M.NIN)
    A = rng.standard_normal((M.NIN, M.NOUT)) / np.sqrt(M.NIN)
    Y = np.tanh(((X - X.mean(0)) / X.std(0)) @ A) * scale + rng.uniform(-0.1, 0.1, M.NOUT)
    return X.astype(np.float32), Y.astype(np.float32)


def _tensors_of(params, H):
    W1, b1, W2, b2, W3, b3 = M.unpack(params, H)
    return {"W1": W1, "b1": b1, "W2": W2, "b2": b2, "W3": W3, "b3": b3}


@pytest.mark.parametrize("H", [64, 128])
def test_forward_matches_oracle(H):
    torch = _torch()
    from lbmpond_b200.learned import Predictor
    X, Y = _random_data(1000, H)
    net = Predictor(H, seed=3)
    Xd, Yd = torch.from_numpy(X).cuda(), torch.from_numpy(Y).cuda()
    net.fit_stats(Xd, Yd)
    out = net.forward(Xd).cpu().numpy()
    p, st = net.get_params()
    Xs, _ = M.standardise(X, Y, st)
    ys = M.forward(p, H, Xs)[2]
    ref = ys * st[2 * M.NIN + M.NOUT:] + st[2 * M.NIN:2 * M.NIN + M.NOUT]
    assert np.abs(out - ref).max() <= 3e-2 * ref.std(0).max()
    net.close()


@pytest.mark.parametrize("H", [64, 128])
def test_gradients_match_oracle(H):
    torch = _torch()
    from lbmpond_b200.learned import Predictor
    n = 1024
    X, Y = _random_data(n, 10 + H)
    net = Predictor(H, seed=5)
    Xd, Yd = torch.from_numpy(X).cuda(), torch.from_numpy(Y).cuda()
    net.fit_stats(Xd, Yd)
    loss, g = net.gradients(Xd, Yd)
    p, st = net.get_params()
    Xs, Ys = M.standardise(X, Y, st)
    loss_ref, g_ref = M.loss_and_grad(p, H, Xs, Ys)
    assert abs(loss - loss_ref) <= 2e-2 * loss_ref
    gt, rt = _tensors_of(g, H), _tensors_of(g_ref, H)
    for k in gt:
        err = np.linalg.norm(gt[k] - rt[k]) / max(np.linalg.norm(rt[k]), 1e-30)
        assert err <= 6e-2, (k, err)
    net.close()


def test_training_reduces_loss():
    torch = _torch()
    from lbmpond_b200.learned import Predictor
    X, Y = _random_data(20000, 7)
    net = Predictor(64, seed=1)
    Xd, Yd = torch.from_numpy(X).cuda(), torch.from_numpy(Y).cuda()
    net.fit_stats(Xd, Yd)
    loss = net.train(Xd, Yd, steps=600, batch=2048, lr=3e-3)
    assert np.all(np.isfinite(loss))
    assert loss[-20:].mean() < 0.1 * loss[:5].mean()
    net.close()


def test_pairs_match_oracle_features(orc, pond):
    torch = _torch()
    from lbmpond_b200.learned import collect_pairs, keep_history
    from tests.states import perturbed_populations, smooth_state
    shape = (16, 12, 10)
    N = int(np.prod(shape))
    rho, g = smooth_state(shape, 3, seed=31, modes=1, du=0.03)
    f = perturbed_populations(orc, 1, rho, g, seed=31, eps=0.01)
    with pond.Solver(lattice="D3Q27", shape=shape, precision="fp64", tau=0.8) as s:
        s.set_state(rho, g, f=f)
        keep_history(s)
        s.step(1)
        _, _, g_next = s.get_state()
        X = torch.zeros((N, M.NIN), dtype=torch.float32, device="cuda")
        Y = torch.zeros((N, M.NOUT), dtype=torch.float32, device="cuda")
        nodes = torch.zeros(N, dtype=torch.int64, device="cuda")
        n = collect_pairs(s, X, Y, stride=1, seed=0, nodes=nodes)
    F, nonuni = M.features(rho, g, shape, g_old=g)
    T = M.targets(g, g_next)
    assert n == int(nonuni.sum())
    idx = nodes[:n].cpu().numpy()
    assert np.array_equal(np.sort(idx), np.flatnonzero(nonuni))
    got = np.concatenate([X[:n].cpu().numpy(), Y[:n].cpu().numpy()], axis=1)
    ref = np.concatenate([F[idx], T[idx]], axis=1)
    scale = np.maximum(np.abs(ref).max(0), 1e-12)
    assert np.all(np.abs(got - ref).max(0) <= 2e-5 * scale + 1e-12)


def test_learned_step_keeps_fixed_point_and_cuts_iterations(pond):
    """Train on pairs from a plain run, then take one held-out step both ways
    from the same state: the converged states agree to the iteration
    tolerance, and the predicted start needs fewer iterations."""
    torch = _torch()
    from lbmpond_b200.learned import Predictor, attach, collect_pairs, keep_history
    n = 32
    lam = 0.25
    sphere = (0.5, 0.5, 0.5, 0.2, 1.0, lam * lam, 0.125, lam * lam * 0.8)
    cap = 600000
    X = torch.zeros((cap, M.NIN), dtype=torch.float32, device="cuda")
    Y = torch.zeros((cap, M.NOUT), dtype=torch.float32, device="cuda")
    rows = 0
    src = pond.Solver(lattice="D3Q27", shape=(n, n, n), precision="fp64", tau=0.52)
    src.init("sphere", *sphere)
    keep_history(src)
    for k in range(24):
        src.step(1)
        rows += collect_pairs(src, X, Y, offset_rows=rows, stride=1, seed=k)
    assert rows > 10000
    net = Predictor(64, seed=0)
    net.fit_stats(X[:rows], Y[:rows])
    loss = net.train(X[:rows], Y[:rows], steps=1500, batch=4096, lr=2e-3)
    assert loss[-50:].mean() < 0.5 * loss[:10].mean()
    res = {}
    for learned in (False, True):
        with pond.Solver(lattice="D3Q27", shape=(n, n, n), precision="fp64", tau=0.52) as s:
            s.copy_state_from(src)  # both time levels
            if learned:
                attach(s, net, gate=0.0)
            s.step(1)
            d = s.diagnostics()
            res[learned] = (s.get_state(), d["niter_mean"], d["nonconverged"])
    src.close()
    (fa, ra, ga), ia, nca = res[False]
    (fb, rb, gb), ib, ncb = res[True]
    assert nca == 0 and ncb == 0
    assert np.abs(fa - fb).max() <= 1e-8 * np.abs(fa).max()
    assert np.abs(ga[3] - gb[3]).max() <= 1e-8 * np.abs(ga[3]).max()
    assert ib < ia, (ia, ib)
    net.close()


def test_learned_start_on_d3q125(pond):
    """The predictor is lattice-generic: on a D3Q125 blast (float64, the
    width-128 network of the D3Q125 workload) the learned start reaches the
    plain step's fixed point."""
    torch = _torch()
    from lbmpond_b200.learned import Predictor, attach, collect_pairs, keep_history
    n = 12
    sphere = (0.5, 0.5, 0.5, 0.25, 1.0, 0.1, 0.3, 0.06)
    cap = 200000
    X = torch.zeros((cap, M.NIN), dtype=torch.float32, device="cuda")
    Y = torch.zeros((cap, M.NOUT), dtype=torch.float32, device="cuda")
    rows = 0
    src = pond.Solver(lattice="D3Q125", shape=(n, n, n), precision="fp64", tau=0.6)
    src.init("sphere", *sphere)
    keep_history(src)
    for k in range(12):
        src.step(1)
        rows += collect_pairs(src, X, Y, offset_rows=rows, stride=1, seed=k)
    assert rows > 2000
    net = Predictor(128, seed=0)
    net.fit_stats(X[:rows], Y[:rows])
    loss = net.train(X[:rows], Y[:rows], steps=800, batch=2048, lr=2e-3)
    assert loss[-50:].mean() < loss[:10].mean()
    res = {}
    for learned in (False, True):
        with pond.Solver(lattice="D3Q125", shape=(n, n, n), precision="fp64", tau=0.6) as s:
            s.copy_state_from(src)
            if learned:
                attach(s, net, gate=0.0)
            s.step(1)
            d = s.diagnostics()
            res[learned] = (s.get_state(), d["niter_mean"], d["nonconverged"])
    src.close()
    (fa, ra, ga), ia, nca = res[False]
    (fb, rb, gb), ib, ncb = res[True]
    assert nca == 0 and ncb == 0
    assert np.abs(fa - fb).max() <= 1e-8 * np.abs(fa).max()
    assert np.abs(ga[3] - gb[3]).max() <= 1e-8 * np.abs(ga[3]).max()
    net.close()
