"""CPU tests of the C ABI: the library loads, exports every symbol that
include/pond.h declares, and validates its arguments before touching a GPU.
No compute call runs here."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    names = []
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not h.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"^\s*[\w\s\*]+?\b(pond_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol(pond):
    from lbmpond_b200 import _lib
    L = ctypes.CDLL(_lib.LIB_PATH)
    names = header_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_binding_covers_header(pond):
    from lbmpond_b200 import _lib
    declared = set(header_functions())
    bound = set(_lib.SIGNATURES)
    assert declared <= bound, sorted(declared - bound)


def test_params_default_and_strings(pond):
    from lbmpond_b200 import _lib
    L = _lib.load()
    assert L.pond_abi_version() == 1
    for lat, q in ((0, 5), (1, 27), (2, 125)):
        p = _lib.PondParams()
        assert L.pond_params_default(lat, ctypes.byref(p)) == 0
        assert L.pond_q(lat) == q
        assert p.max_iter == 100 and abs(p.tau - 0.9) < 1e-15
        assert p.interp == (6 if lat == 2 else 4)
    assert L.pond_params_default(7, ctypes.byref(_lib.PondParams())) == -1
    assert L.pond_status_string(-5).decode().startswith("unsupported")


@pytest.mark.parametrize("field,value,status", [
    ("interp", 6, -5),       # FIXED3 is the D3Q125 kernel only
    ("interp", 7, -5),       # TVD is 1D only
    ("tau", 0.4, -1),        # BGK needs tau > 0.5
    ("max_iter", 0, -1),
    ("Nx", 0, -1),
    ("precision", 3, -1),
])
def test_create_validates_before_device(pond, field, value, status):
    from lbmpond_b200 import _lib
    L = _lib.load()
    p = _lib.PondParams()
    L.pond_params_default(1, ctypes.byref(p))
    setattr(p, field, value)
    ctx = ctypes.c_void_p()
    assert L.pond_create(ctypes.byref(p), ctypes.byref(ctx)) == status
    assert not ctx.value
    assert L.pond_last_error_string().decode()


def test_null_arguments(pond):
    from lbmpond_b200 import _lib
    L = _lib.load()
    assert L.pond_create(None, None) == -1
    assert L.pond_step(None, 1) == -1
    assert L.pond_destroy(None) == 0
    assert L.pond_diagnostics(None, None) == -1


def test_arr_roundtrip(tmp_path, pond):
    import numpy as np
    data = np.arange(24, dtype=np.float64)
    p = str(tmp_path / "Rho_0000001.arr")
    pond.write_arr(p, data, (4, 3, 2))
    back, shape = pond.read_arr(p)
    assert shape == (4, 3, 2) and np.array_equal(back, data)
    raw = np.fromfile(p, dtype=np.int32, count=6)
    assert raw.tolist() == [0, 3, 8, 4, 3, 2]  # drop.cu:12-20 header


@pytest.mark.parametrize("lengths,interp,tau,status", [
    ([10, 0, 5], 8, 0.9, -1),      # empty problem
    ([10, 4097], 8, 0.9, -1),      # longer than a bin
    ([], 8, 0.9, -1),              # no problems
    ([10, 20], 7, 0.9, -5),        # TVD is not built for the batch
    ([10, 20], 8, 0.5, -1),        # BGK needs tau > 0.5
])
def test_batch_create_validates_before_device(pond, lengths, interp, tau, status):
    from lbmpond_b200 import _lib
    L = _lib.load()
    arr = (ctypes.c_int32 * max(len(lengths), 1))(*lengths)
    h = ctypes.c_void_p()
    assert L.pond_batch_create(len(lengths), arr, interp, tau, 1e-7, 1e-6, 100, 0, ctypes.byref(h)) == status
    assert not h.value
    assert L.pond_last_error_string().decode()
    assert L.pond_batch_destroy(None) == 0
    assert L.pond_batch_run(None, 1, 1, None) == -1
    assert L.pond_batch_nodes(None) == 0


def test_riemann_problem_set():
    import numpy as np
    from lbmpond_b200.batch import riemann_problems
    lengths, rho, u, T = riemann_problems(4096, seed=0)
    assert lengths.size == 4096 and lengths.min() >= 256 and lengths.max() <= 4096
    assert rho.size == u.size == T.size == int(lengths.sum())
    assert 1500 < lengths.mean() < 2900
    p = rho * T
    assert rho.min() >= 0.1 - 1e-12 and rho.max() <= 10 + 1e-9
    assert p.min() >= 0.1 - 1e-12 and p.max() <= 10 + 1e-9
    assert np.abs(u).max() <= 1
    # two constant states per problem, the jump at the midpoint
    off = np.concatenate([[0], np.cumsum(lengths)])
    for q in (0, 17, 4095):
        r = rho[off[q]:off[q + 1]]
        n = lengths[q]
        assert np.all(r[:n // 2] == r[0]) and np.all(r[n // 2:] == r[-1])
    again = riemann_problems(4096, seed=0)
    assert np.array_equal(again[0], lengths) and np.array_equal(again[3], T)


def test_step_host_validates_before_device(pond):
    from lbmpond_b200 import _lib
    L = _lib.load()
    assert L.pond_step_host(None, None, None, None, None, None) == -1
    assert L.pond_sync(None) == -1


@pytest.mark.parametrize("change,status", [
    ({"Ny": 2}, -5),                           # the mesh schemes are one-dimensional
    ({"Nx": 2}, -5),                           # and need three nodes for the quadratic stencil
    ({"bc0": 1}, -5),                          # and periodic (steps.cu:1128-1130, :891-893)
    ({"ddf": 1, "ddf_dof": 4}, -5),            # no energy populations on the mesh
    ({"learned": 1}, -5),                      # nor the learned start
    ({"lattice_q27": True}, -5),               # D1Q5 only
])
@pytest.mark.parametrize("scheme", [9, 10])  # POND_GAP2, POND_NONUNIFORM3
def test_mesh_schemes_validate_before_device(pond, scheme, change, status):
    from lbmpond_b200 import _lib
    L = _lib.load()
    p = _lib.PondParams()
    L.pond_params_default(1 if change.get("lattice_q27") else 0, ctypes.byref(p))
    p.interp = scheme
    for k, v in change.items():
        if k == "bc0":
            p.bc[0] = v
        elif k != "lattice_q27":
            setattr(p, k, v)
    ctx = ctypes.c_void_p()
    assert L.pond_create(ctypes.byref(p), ctypes.byref(ctx)) == status
    assert not ctx.value
    assert L.pond_last_error_string().decode()


def test_mesh_calls_reject_null_context(pond):
    from lbmpond_b200 import _lib
    L = _lib.load()
    buf = (ctypes.c_uint8 * 4)()
    pos = (ctypes.c_double * 4)()
    n = ctypes.c_int64()
    assert L.pond_set_mask(None, buf) == -1
    assert L.pond_get_mask(None, buf) == -1
    assert L.pond_set_positions(None, pos) == -1
    assert L.pond_get_positions(None, pos) == -1
    assert L.pond_amr_refine(None, 0.01, ctypes.byref(n), ctypes.byref(n)) == -1
    assert L.pond_amr_coarsen(None, 0.01, ctypes.byref(n)) == -1
    assert L.pond_rescale_time(None, 2.0) == -1
    assert L.pond_set_dt_adapt(None, 1, 1000, 4) == -1


def _noalloc(L):
    from lbmpond_b200 import _lib
    fn = L.pond_step_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.POINTER(_lib.PondParams)] + [ctypes.c_void_p] * 8
    return fn


@pytest.mark.parametrize("field,value,status,word", [
    ("max_iter", 100001, -1, "max_iter"),   # bounds one launch on a shared GPU
    ("tau", float("inf"), -1, "tau"),       # dtau would be 0
    ("tol_abs", float("nan"), -1, "toleran"),
    ("tol_rel", float("inf"), -1, "toleran"),
    ("learned", 1, -5, "learned"),          # no predictor on this path
    ("ddf", 1, -5, "energy"),
])
def test_noalloc_validates_before_device(pond, field, value, status, word):
    """pond_step_noalloc applies pond_create's parameter checks and refuses
    what it does not run, before any CUDA call (the pointers are never
    dereferenced)."""
    from lbmpond_b200 import _lib
    L = _lib.load()
    fn = _noalloc(L)
    p = _lib.PondParams()
    L.pond_params_default(1, ctypes.byref(p))
    p.Nx, p.Ny, p.Nz = 32, 8, 4
    setattr(p, field, value)
    N = 32 * 8 * 4
    bufs = [4096 + k * 4 * 32 * N for k in range(6)]  # disjoint fake addresses
    assert fn(ctypes.byref(p), *bufs, 16, None) == status
    assert word in L.pond_last_error_string().decode()


@pytest.mark.parametrize("alias", ["f_out=f_in", "rho_out=g_in", "g_out inside f_in", "rho_out=g_out"])
def test_noalloc_rejects_overlapping_buffers(pond, alias):
    from lbmpond_b200 import _lib
    L = _lib.load()
    fn = _noalloc(L)
    p = _lib.PondParams()
    L.pond_params_default(1, ctypes.byref(p))
    p.Nx, p.Ny, p.Nz = 32, 8, 4
    N = 32 * 8 * 4
    b = {k: 4096 + i * 4 * 32 * N for i, k in enumerate(("fi", "ri", "gi", "fo", "ro", "go"))}
    if alias == "f_out=f_in":
        b["fo"] = b["fi"]
    elif alias == "rho_out=g_in":
        b["ro"] = b["gi"] + 4 * N
    elif alias == "g_out inside f_in":
        b["go"] = b["fi"] + 4 * 26 * N
    else:
        b["ro"] = b["go"] + 4
    st = fn(ctypes.byref(p), b["fi"], b["ri"], b["gi"], b["fo"], b["ro"], b["go"], 16, None)
    assert st == -1
    assert "overlaps" in L.pond_last_error_string().decode()
