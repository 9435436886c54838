"""GPU test of the pipelined host-buffer step (pond_step_host / pond_sync):
each call must give exactly what pond_step gives from the same input state,
also when two different inputs alternate between the calls (so the two input
slots and the two output buffers are both in use), and the context must be
usable by the ordinary calls afterwards."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pinned(torch, shape):
    return torch.empty(shape, dtype=torch.float32, pin_memory=True)


def test_step_host_matches_step(pond):
    import torch
    shape = (20, 12, 9)
    N = int(np.prod(shape))
    states = []
    with pond.Solver(lattice="D3Q27", shape=shape, precision="fp32", tau=0.6) as s:
        for ic in (("sphere", 0.5, 0.5, 0.5, 0.25, 1.0, 0.06, 0.3, 0.04), ("tgv", 0.05, 0.08, 1.0, 5 / 3)):
            s.init(*ic)
            s.step(2)  # a non-trivial state
            f, r, g = _pinned(torch, (27, N)), _pinned(torch, N), _pinned(torch, (4, N))
            s.download_native(f.data_ptr(), r.data_ptr(), g.data_ptr())
            states.append((f, r, g))
        # the reference results: one pond_step from each state
        ref = []
        for f, r, g in states:
            s.upload_native(f.data_ptr(), r.data_ptr(), g.data_ptr())
            s.step(1)
            ro, go = _pinned(torch, N), _pinned(torch, (4, N))
            s.download_native(None, ro.data_ptr(), go.data_ptr())
            ref.append((ro.clone(), go.clone()))
        # five pipelined calls alternating the two inputs, each with its own outputs
        outs = []
        for k in range(5):
            f, r, g = states[k % 2]
            ro, go = _pinned(torch, N), _pinned(torch, (4, N))
            s.step_host(f.data_ptr(), r.data_ptr(), g.data_ptr(), ro.data_ptr(), go.data_ptr())
            outs.append((k % 2, ro, go))
        s.sync()
        for which, ro, go in outs:
            assert torch.equal(ro, ref[which][0]) and torch.equal(go, ref[which][1])
        # the last result is the current state; ordinary calls work afterwards
        f_last = np.empty((27, N))
        _, rho_now, g_now = s.get_state()
        assert np.array_equal(rho_now, ref[0][0].numpy().astype(np.float64))
        s.step(1)
        d = s.diagnostics()
        assert d["nonconverged"] == 0 and np.isfinite(d["mass"])
        del f_last


def test_step_host_rejects_a_bound_predictor(pond):
    from lbmpond_b200 import _lib
    from lbmpond_b200.learned import Predictor, attach
    with pond.Solver(lattice="D3Q27", shape=(8, 8, 8), precision="fp32") as s:
        s.init("sphere", 0.5, 0.5, 0.5, 0.25, 1.0, 0.06, 0.3, 0.04)
        net = Predictor(64, seed=0)
        attach(s, net, gate=0.0)
        with pytest.raises(_lib.PondError):
            s.step_host(1, 1, 1)
        attach(s, None)
        net.close()
