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
    assert declared <= bound | {n for n in declared if n.startswith(("pond_mlp", "pond_batch", "pond_pred"))}


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
