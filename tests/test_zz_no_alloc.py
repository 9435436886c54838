"""pond_step_noalloc: the step for callers that cannot let the library
allocate device memory (their own memory pool, a fixed budget, or no
allocation stalls allowed inside the time loop).  The caller owns every
buffer; the entry point keeps its scratch in a fixed array inside the library.

Checked through the C ABI against the context entry points (pond_create /
pond_step) on two calls in a row, within the float32 tolerance of the parity
tests.  This file is collected last so that a failure here leaves every other
test already run."""
import ctypes

import numpy as np
import pytest

from tests.states import perturbed_populations, smooth_state

pytestmark = pytest.mark.gpu

TOL = 3e-5  # the float32 tolerance of tests/test_gpu_parity.py


def _bind(L):
    from lbmpond_b200 import _lib
    fn = L.pond_step_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.POINTER(_lib.PondParams)] + [ctypes.c_void_p] * 8
    return fn


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


@pytest.mark.parametrize("shape,interp", [((40, 12, 6), 4), ((64, 8, 8), 3)])
def test_noalloc_step_matches_context_step(orc, pond, shape, interp):
    import torch
    from lbmpond_b200 import _lib
    L = _lib.load()
    step_noalloc = _bind(L)
    N = int(np.prod(shape))
    rho, g = smooth_state(shape, 3, seed=21, modes=1, du=0.03)
    f = perturbed_populations(orc, 1, rho, g, seed=21, eps=0.01)

    # the existing entry points: a context that owns its buffers
    ref = []
    with pond.Solver(lattice="D3Q27", shape=shape, interp=interp, precision="fp32", tau=0.8) as s:
        s.set_state(rho, g, f=f)
        for _ in range(2):
            s.step(1)
            fo = np.empty((27, N), np.float32); ro = np.empty(N, np.float32); go = np.empty((4, N), np.float32)
            s.download_native(fo.ctypes.data, ro.ctypes.data, go.ctypes.data)
            ref.append((fo, ro, go, s.diagnostics()))

    # the allocation-free entry point on buffers the caller allocated
    p = _lib.PondParams()
    assert L.pond_params_default(1, ctypes.byref(p)) == 0
    p.Nx, p.Ny, p.Nz = shape
    p.interp = interp
    p.tau = 0.8
    dev = torch.device("cuda", 0)
    bufs = [(torch.from_numpy(f.astype(np.float32)).to(dev), torch.from_numpy(rho.astype(np.float32)).to(dev),
             torch.from_numpy(g.astype(np.float32)).to(dev))]
    bufs.append(tuple(torch.empty_like(t) for t in bufs[0]))
    diag = torch.zeros(ctypes.sizeof(_lib.PondDiag), dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    for call in range(2):  # two calls in a row, ping-ponging the caller's buffers
        src, dst = bufs[call % 2], bufs[(call + 1) % 2]
        st = step_noalloc(ctypes.byref(p), *(t.data_ptr() for t in src), *(t.data_ptr() for t in dst),
                          diag.data_ptr(), stream)
        assert st == 0, L.pond_last_error_string().decode()
        torch.cuda.synchronize(dev)
        fo, ro, go, dref = ref[call]
        assert _rel(dst[0].cpu().numpy(), fo) <= TOL
        assert _rel(dst[1].cpu().numpy(), ro) <= TOL
        assert _rel(dst[2].cpu().numpy()[3], go[3]) <= TOL
        assert np.abs(dst[2].cpu().numpy()[:3] - go[:3]).max() <= TOL * np.sqrt(np.abs(go[3]).max())
        d = _lib.PondDiag.from_buffer_copy(bytes(diag.cpu().numpy()))
        assert abs(d.mass - dref["mass"]) <= 1e-12 * abs(dref["mass"])
        assert abs(d.enrg - dref["enrg"]) <= 1e-12 * abs(dref["enrg"])
        assert d.niter_max == dref["niter_max"] and d.nonconverged == dref["nonconverged"]
        assert d.niter_sum == dref["niter_sum"]


def test_noalloc_rejects_grids_beyond_its_scratch(pond):
    from lbmpond_b200 import _lib
    L = _lib.load()
    step_noalloc = _bind(L)
    p = _lib.PondParams()
    L.pond_params_default(1, ctypes.byref(p))
    p.Nx, p.Ny, p.Nz = 256, 256, 264  # one z-layer of tiles too many
    one = ctypes.c_void_p(16)  # never dereferenced: the size check comes first
    st = step_noalloc(ctypes.byref(p), one, one, one, one, one, one, one, None)
    assert st == -1
    assert "scratch" in L.pond_last_error_string().decode()


def test_noalloc_step_leaves_guard_bands_untouched(orc, pond):
    """Guard-band canaries around every caller-owned array: each plane set
    sits inside a larger allocation whose first and last 1024 elements (4 KB,
    keeping every interior pointer 16-byte aligned) hold a sentinel pattern;
    after two steps the bands are bit for bit unchanged and every output value
    is finite."""
    import torch
    from lbmpond_b200 import _lib
    L = _lib.load()
    step_noalloc = _bind(L)
    shape = (40, 12, 6)
    N = int(np.prod(shape))
    rho, g = smooth_state(shape, 3, seed=22, modes=1, du=0.03)
    f = perturbed_populations(orc, 1, rho, g, seed=22, eps=0.01)
    p = _lib.PondParams()
    assert L.pond_params_default(1, ctypes.byref(p)) == 0
    p.Nx, p.Ny, p.Nz = shape
    p.tau = 0.8
    dev = torch.device("cuda", 0)
    G = 1024
    sentinel = torch.tensor([-1.234567e30], dtype=torch.float32).view(torch.int32).item()

    def guarded(host):
        n = host.size
        t = torch.full((n + 2 * G,), sentinel, dtype=torch.int32, device=dev).view(torch.float32)
        t[G:G + n] = torch.from_numpy(host.astype(np.float32).ravel()).to(dev)
        return t, n

    sets = [[guarded(a) for a in (f, rho, g)] for _ in range(2)]
    diag = torch.zeros(ctypes.sizeof(_lib.PondDiag), dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    for call in range(2):
        src, dst = sets[call % 2], sets[(call + 1) % 2]
        ptrs = [t.data_ptr() + 4 * G for t, _ in src] + [t.data_ptr() + 4 * G for t, _ in dst]
        st = step_noalloc(ctypes.byref(p), *ptrs, diag.data_ptr(), stream)
        assert st == 0, L.pond_last_error_string().decode()
    torch.cuda.synchronize(dev)
    for group in sets:
        for t, n in group:
            bits = t.view(torch.int32)
            assert bool((bits[:G] == sentinel).all()) and bool((bits[G + n:] == sentinel).all())
            assert bool(torch.isfinite(t[G:G + n]).all())
    assert N == sets[0][1][1]
