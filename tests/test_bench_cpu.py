"""CPU checks of bench.py's host-side legs: the oracle sample on blocks of a
stored state (the CPU baseline and the reference arm) and the batch problem
generators.  No GPU."""
import numpy as np

import bench


def test_oracle_blocks_on_a_stored_sample(orc, tmp_path, monkeypatch):
    from tests.states import perturbed_populations, smooth_state
    e, nb = 5, 2
    fs, rs, gs = [], [], []
    for b in range(nb):
        rho, g = smooth_state((e, e, e), 3, seed=40 + b, modes=1, du=0.02)
        fs.append(perturbed_populations(orc, 1, rho, g, seed=40 + b, eps=0.01))
        rs.append(rho)
        gs.append(g)
    path = tmp_path / "blocks.npz"
    np.savez(path, f=np.stack(fs, 1).astype(np.float32), rho=np.stack(rs).astype(np.float32),
             g=np.stack(gs, 1).astype(np.float32), niter_gpu=np.full((nb, e ** 3), 3, np.int8),
             corners=np.zeros((nb, 3), int), edge=e, size=64, spinup=10, tau=bench.TAU,
             tol=(bench.TOL_ABS, bench.TOL_REL), niter_mean_domain=2.5)
    monkeypatch.setattr(bench, "SAMPLE", str(path))
    v, dt, it, it_gpu, cores, desc = bench._oracle_blocks(0, 2)
    assert v > 0 and dt > 0 and cores >= 1
    assert 1 <= it < 100 and it_gpu == 3.0
    assert "2 blocks of 5^3" in desc
    # the same blocks stepped directly by the oracle iterate as often
    its = []
    for b in range(nb):
        st = orc.State(fs[b].astype(np.float32).astype(np.float64), rs[b].astype(np.float32).astype(np.float64),
                       gs[b].astype(np.float32).astype(np.float64))
        _, niter, _ = orc.step(st, 1, (e, e, e), tau=bench.TAU, tol_abs=bench.TOL_ABS, tol_rel=bench.TOL_REL,
                               bc=(orc.BC_CLAMP,) * 3)
        its.append(niter.mean())
    assert abs(np.mean(its) - it) < 1e-12


def test_moderate_batch_set_bounds():
    from lbmpond_b200.batch import riemann_problems, riemann_problems_moderate
    lengths, rho, u, T = riemann_problems_moderate(64, seed=3)
    assert lengths.min() >= 256 and lengths.max() <= 4096 and rho.size == lengths.sum()
    off = np.concatenate([[0], np.cumsum(lengths)])
    for p in range(64):
        r, t, uu = rho[off[p]:off[p + 1]], T[off[p]:off[p + 1]], u[off[p]:off[p + 1]]
        assert r.max() / r.min() <= 4 + 1e-9 and t.max() / t.min() <= 1.5 + 1e-9
        assert np.abs(uu).max() <= 0.06 + 1e-12 and 0.09 / 1.5 ** 0.5 * 0.999 <= t.min()
    # the specified set reaches ratios of up to 100 in rho and p
    lengths, rho, u, T = riemann_problems(64, seed=3)
    assert rho.max() / rho.min() > 10
