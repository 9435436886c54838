"""ctypes binding of the C ABI in include/pond.h (libpond_b200.so)."""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpond_b200.so")

POND_OK = 0
STATUS = {
    0: "ok", -1: "invalid argument", -2: "CUDA runtime error", -3: "out of device memory",
    -4: "call out of order", -5: "unsupported lattice/scheme/precision", -6: "iteration did not converge",
}

D1Q5, D3Q27, D3Q125 = 0, 1, 2
LAGR2, LAGR3, LAGR4, LAGR5, FIXED3, TVD, WENO5, GAP2, NONUNIFORM3, WENO5_ROW = 2, 3, 4, 5, 6, 7, 8, 9, 10, 11
BC_PERIODIC, BC_CLAMP, BC_MIRROR, BC_INFLOW = 0, 1, 2, 3
FP32, FP64 = 0, 1
IC_ACOUSTIC, IC_SOD_X, IC_SPHERE, IC_TGV, IC_UNIFORM = 0, 1, 2, 3, 4


class PondParams(ctypes.Structure):
    _fields_ = [
        ("Nx", ctypes.c_int64), ("Ny", ctypes.c_int64), ("Nz", ctypes.c_int64),
        ("lattice", ctypes.c_int), ("interp", ctypes.c_int), ("precision", ctypes.c_int),
        ("bc", ctypes.c_int * 3),
        ("tau", ctypes.c_double), ("dt", ctypes.c_double),
        ("tol_abs", ctypes.c_double), ("tol_rel", ctypes.c_double),
        ("max_iter", ctypes.c_int), ("device", ctypes.c_int), ("learned", ctypes.c_int),
        ("ddf", ctypes.c_int), ("ddf_dof", ctypes.c_int),
        ("reserved", ctypes.c_int * 3),
    ]


class PondDiag(ctypes.Structure):
    _fields_ = [
        ("mass", ctypes.c_double), ("moment", ctypes.c_double * 3), ("enrg", ctypes.c_double),
        ("k", ctypes.c_double), ("niter_max", ctypes.c_int32), ("pad", ctypes.c_int32),
        ("niter_mean", ctypes.c_double), ("niter_sum", ctypes.c_int64),
        ("nonconverged", ctypes.c_int64), ("istep", ctypes.c_int64), ("curtime", ctypes.c_double),
    ]


# every symbol the header declares: name -> (restype, argtypes)
_vp = ctypes.c_void_p
_dp = ctypes.POINTER(ctypes.c_double)
_i32p = ctypes.POINTER(ctypes.c_int32)
_i64p = ctypes.POINTER(ctypes.c_int64)
_u8p = ctypes.POINTER(ctypes.c_uint8)
SIGNATURES = {
    "pond_abi_version": (ctypes.c_int, []),
    "pond_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "pond_last_error_string": (ctypes.c_char_p, []),
    "pond_params_default": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(PondParams)]),
    "pond_create": (ctypes.c_int, [ctypes.POINTER(PondParams), ctypes.POINTER(_vp)]),
    "pond_destroy": (ctypes.c_int, [_vp]),
    "pond_get_params": (ctypes.c_int, [_vp, ctypes.POINTER(PondParams)]),
    "pond_q": (ctypes.c_int, [ctypes.c_int]),
    "pond_lattice_tables": (ctypes.c_int, [ctypes.c_int, _dp, _dp, _dp]),
    "pond_init": (ctypes.c_int, [_vp, ctypes.c_int, _dp, ctypes.c_int]),
    "pond_set_state": (ctypes.c_int, [_vp, _dp, _dp, _dp]),
    "pond_get_state": (ctypes.c_int, [_vp, _dp, _dp, _dp]),
    "pond_set_energy": (ctypes.c_int, [_vp, _dp]),
    "pond_get_energy": (ctypes.c_int, [_vp, _dp]),
    "pond_get_fields": (ctypes.c_int, [_vp, _dp, _dp, _dp, _dp, _dp]),
    "pond_step": (ctypes.c_int, [_vp, ctypes.c_int]),
    "pond_set_inflow": (ctypes.c_int, [_vp] + [ctypes.c_double] * 5),
    "pond_set_gauge_tolerance": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_double]),
    "pond_diagnostics": (ctypes.c_int, [_vp, ctypes.POINTER(PondDiag)]),
    "pond_set_clock": (ctypes.c_int, [_vp, ctypes.c_int64, ctypes.c_double, ctypes.c_double]),
    "pond_set_strict": (ctypes.c_int, [_vp, ctypes.c_int]),
    "pond_keep_niter": (ctypes.c_int, [_vp, ctypes.c_int]),
    "pond_get_niter": (ctypes.c_int, [_vp, _i32p]),
    "pond_keep_history": (ctypes.c_int, [_vp, ctypes.c_int]),
    "pond_stream": (_vp, [_vp]),
    "pond_device_state": (ctypes.c_int, [_vp, ctypes.POINTER(_vp), ctypes.POINTER(_vp), ctypes.POINTER(_vp)]),
    "pond_last_step_ms": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_float)]),
    "pond_upload_state": (ctypes.c_int, [_vp, _vp, _vp, _vp]),
    "pond_download_state": (ctypes.c_int, [_vp, _vp, _vp, _vp]),
    "pond_last_step_work": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int64)]),
    "pond_copy_state": (ctypes.c_int, [_vp, _vp]),
    "pond_step_noalloc": (ctypes.c_int, [ctypes.POINTER(PondParams)] + [_vp] * 8),
    "pond_set_mask": (ctypes.c_int, [_vp, _u8p]),
    "pond_get_mask": (ctypes.c_int, [_vp, _u8p]),
    "pond_set_positions": (ctypes.c_int, [_vp, _dp]),
    "pond_get_positions": (ctypes.c_int, [_vp, _dp]),
    "pond_amr_refine": (ctypes.c_int, [_vp, ctypes.c_double, _i64p, _i64p]),
    "pond_amr_coarsen": (ctypes.c_int, [_vp, ctypes.c_double, _i64p]),
    "pond_rescale_time": (ctypes.c_int, [_vp, ctypes.c_double]),
    "pond_set_dt_adapt": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "pond_mlp_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_uint64, ctypes.c_int, ctypes.POINTER(_vp)]),
    "pond_mlp_destroy": (ctypes.c_int, [_vp]),
    "pond_mlp_num_params": (ctypes.c_int, [_vp]),
    "pond_mlp_get_params": (ctypes.c_int, [_vp, _vp, _vp]),
    "pond_mlp_set_params": (ctypes.c_int, [_vp, _vp, _vp]),
    "pond_mlp_fit_stats": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int64]),
    "pond_mlp_train": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.c_float, _vp]),
    "pond_mlp_gradients": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int64, _vp, _vp]),
    "pond_mlp_forward": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int64]),
    "pond_collect_pairs": (ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_int64, ctypes.c_int64, ctypes.c_uint64,
                                          ctypes.POINTER(ctypes.c_int64)]),
    "pond_set_predictor": (ctypes.c_int, [_vp, _vp, ctypes.c_float]),
    "pond_predict": (ctypes.c_int, [_vp, _vp]),
    "pond_set_extrapolation": (ctypes.c_int, [_vp, ctypes.c_int]),
    "pond_step_host": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "pond_sync": (ctypes.c_int, [_vp]),
    "pond_batch_create": (ctypes.c_int, [ctypes.c_int, _i32p, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.POINTER(_vp)]),
    "pond_batch_destroy": (ctypes.c_int, [_vp]),
    "pond_batch_nodes": (ctypes.c_int64, [_vp]),
    "pond_batch_bins": (ctypes.c_int32, [_vp]),
    "pond_batch_set_state": (ctypes.c_int, [_vp, _dp, _dp, _dp]),
    "pond_batch_get_state": (ctypes.c_int, [_vp, _dp, _dp, _dp, _dp]),
    "pond_batch_set_pairs": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int64, ctypes.c_int, ctypes.c_int]),
    "pond_batch_pairs_written": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int64)]),
    "pond_batch_run": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_float)]),
    "pond_batch_stats": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64),
                                        _i32p]),
    "pond_batch_set_tile": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int]),
    "pond_batch_get_tile": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    "pond_batch_autotune": (ctypes.c_int, [_vp, ctypes.c_int, _i32p, ctypes.c_int, ctypes.POINTER(ctypes.c_float),
                                           ctypes.POINTER(ctypes.c_int)]),
}

_lib = None


class PondError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


def load(path: str | None = None):
    """Load the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or LIB_PATH
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: run `python -m lbmpond_b200.build`")
    L = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def check(status: int):
    if status != POND_OK:
        msg = _lib.pond_last_error_string().decode() if _lib else ""
        raise PondError(status, msg)
    return status
