"""ctypes binding of libibpm_b200.so (the C ABI in include/ibpm_b200.h).

The library is built in-tree (``build.py``) into ``lib/libibpm_b200.so``.  There
is no CPU fallback: if the library is missing, loading raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

LIB_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib")
LIB_PATH = os.path.join(LIB_DIR, "libibpm_b200.so")

IBPM_OK = 0
IBPM_WARN_CG_MAXITER = 1
IBPM_ERR_INVALID = -1
IBPM_ERR_CUDA = -2
IBPM_ERR_REGION = -3
IBPM_ERR_NOMEM = -4
IBPM_ERR_NONFINITE = -5
IBPM_FP64 = 0
IBPM_FP32 = 1
IBPM_MIXED_L1 = 2

_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int32)


class ibpm_problem(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nlevel", C.c_int32),
                ("h", C.c_double), ("x0", C.c_double), ("y0", C.c_double),
                ("Re", C.c_double), ("dt", C.c_double),
                ("npanel", C.c_int32), ("nbody", C.c_int32),
                ("body_kind", _ip), ("body_start", _ip), ("body_xb", _dp), ("body_ds", _dp),
                ("grid_moving", C.c_int32)]


class ibpm_options(C.Structure):
    _fields_ = [("precision", C.c_int32), ("device", C.c_int32), ("cg_maxiter", C.c_int32),
                ("cg_reltol", C.c_double), ("cg_abstol", C.c_double)]


class ibpm_step_params(C.Structure):
    _fields_ = [("freestream", C.c_double * 2), ("grid_motion", C.c_double * 6), ("body_motion", _dp)]


class ibpm_state_view(C.Structure):
    _fields_ = [("index", C.c_int64), ("t0", C.c_double),
                ("q", _dp), ("q0", _dp), ("gamma", _dp), ("psi", _dp), ("nonlin1", _dp), ("nonlin2", _dp),
                ("xb", _dp), ("ds", _dp), ("ub", _dp), ("fbt", _dp),
                ("freestream", C.c_double * 2)]


class ibpm_info(C.Structure):
    _fields_ = [("nq", C.c_int64), ("ng", C.c_int64), ("nbc", C.c_int64), ("static_bodies", C.c_int32),
                ("last_cg_iters", C.c_int32), ("last_cg_residual", C.c_double), ("device_bytes", C.c_int64),
                ("first_cg_residual", C.c_double), ("warm_start_coef", C.c_double * 2)]


EXPORTS = {
    "ibpm_default_options": (None, [C.POINTER(ibpm_options)]),
    "ibpm_create": (C.c_int, [C.POINTER(ibpm_problem), C.POINTER(ibpm_options), C.POINTER(C.c_void_p)]),
    "ibpm_destroy": (None, [C.c_void_p]),
    "ibpm_set_state": (C.c_int, [C.c_void_p, C.POINTER(ibpm_state_view)]),
    "ibpm_get_state": (C.c_int, [C.c_void_p, C.POINTER(ibpm_state_view)]),
    "ibpm_advance": (C.c_int, [C.c_void_p, C.c_int64, C.POINTER(ibpm_step_params)]),
    "ibpm_get_forces": (C.c_int, [C.c_void_p, _dp, _dp]),
    "ibpm_get_field": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, _dp]),
    "ibpm_get_time": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64), _dp]),
    "ibpm_get_info": (C.c_int, [C.c_void_p, C.POINTER(ibpm_info)]),
    "ibpm_last_error": (C.c_char_p, [C.c_void_p]),
    "ibpm_stream": (C.c_void_p, [C.c_void_p]),
    "ibpm_kernel_launches": (C.c_int64, [C.c_void_p]),
    "ibpm_profile": (C.c_int, [C.c_void_p, C.c_int]),
    "ibpm_profile_read": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int64), _dp, _dp]),
    "ibpm_diag_solve": (C.c_int, [C.c_void_p, C.c_int, C.c_int, _dp, _dp]),
    "ibpm_diag_apply_B": (C.c_int, [C.c_void_p, _dp, _dp]),
    "ibpm_diag_binv": (C.c_int, [C.c_void_p, _dp]),
    "ibpm_diag_vort2flux": (C.c_int, [C.c_void_p, _dp, _dp, _dp]),
    "ibpm_diag_reg": (C.c_int, [C.c_void_p, _dp, _dp, _dp, _dp]),
    "ibpm_ensemble_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_int32, C.POINTER(C.c_void_p)]),
    "ibpm_ensemble_advance": (C.c_int, [C.c_void_p, C.c_int64, C.POINTER(ibpm_step_params)]),
    "ibpm_ensemble_destroy": (None, [C.c_void_p]),
    "ibpm_ensemble_last_error": (C.c_char_p, [C.c_void_p]),
    "ibpm_ensemble_groups": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "ibpm_tune_table": (C.c_int, [C.c_char_p, C.c_int32]),
    "ibpm_net_create": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_uint64, C.c_int32,
                                  C.POINTER(C.c_void_p)]),
    "ibpm_net_destroy": (None, [C.c_void_p]),
    "ibpm_net_num_params": (C.c_int64, [C.c_void_p]),
    "ibpm_net_get_params": (C.c_int, [C.c_void_p, _fp]),
    "ibpm_net_set_params": (C.c_int, [C.c_void_p, _fp]),
    "ibpm_net_set_normalisation": (C.c_int, [C.c_void_p, _fp, _fp, _fp, _fp]),
    "ibpm_net_get_normalisation": (C.c_int, [C.c_void_p, _fp, _fp, _fp, _fp]),
    "ibpm_net_forward": (C.c_int, [C.c_void_p, _fp, C.c_int64, C.c_int32, _fp]),
    "ibpm_net_loss_grad": (C.c_int, [C.c_void_p, _fp, _fp, C.c_int64, C.c_int32, _fp, _fp]),
    "ibpm_net_train": (C.c_int, [C.c_void_p, _fp, _fp, C.c_int64, C.c_int32, C.c_int32, C.c_int32, C.c_float,
                                 C.c_uint64, _fp]),
    "ibpm_net_last_error": (C.c_char_p, [C.c_void_p]),
    "ibpm_set_warm_start": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32]),
    "ibpm_set_rebuild_transform": (C.c_int, [C.c_void_p, C.c_int32]),
    "ibpm_warm_start_sample": (C.c_int, [C.c_void_p, _fp, _fp, _fp]),
    "ibpm_lap_inv_noalloc": (C.c_int, [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
    "ibpm_noalloc_last_error": (C.c_char_p, []),
}
(IBPM_WS_PREVIOUS, IBPM_WS_LEARNED, IBPM_WS_EXTRAPOLATED, IBPM_WS_PROJECTED, IBPM_WS_DIRECT,
 IBPM_WS_PRECONDITIONED, IBPM_WS_PRECOND_EXTRAP) = 0, 1, 2, 3, 4, 5, 6
KCLASS = {"xpass": 0, "ypass": 1, "nonlinear": 2, "curl": 3, "xtrial": 4, "ytrial": 5, "tcdst": 6, "tclines": 7}

_lib = None


def load(path: str = LIB_PATH):
    """Load the CUDA library; raises OSError when it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise OSError(f"{path} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'`")
    lib = C.CDLL(path)
    for name, (res, args) in EXPORTS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def dptr(a):
    """Pointer to a contiguous float64 numpy array (None -> NULL)."""
    if a is None:
        return None
    if a.dtype != np.float64 or not (a.flags.f_contiguous or a.flags.c_contiguous):
        raise ValueError("expected a contiguous float64 array")
    return a.ctypes.data_as(_dp)


class IbpmError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(msg)
        self.code = code


def check(lib, h, rc: int):
    if rc < 0:
        msg = lib.ibpm_last_error(h)
        raise IbpmError(rc, msg.decode() if msg else f"ibpm error {rc}")
    return rc


def fptr(a):
    """Pointer to a contiguous float32 numpy array (None -> NULL)."""
    if a is None:
        return None
    if a.dtype != np.float32 or not a.flags.c_contiguous:
        raise ValueError("expected a C-contiguous float32 array")
    return a.ctypes.data_as(_fp)


def tune_table() -> dict:
    """The pass-shape autotuner's choices so far: {key: line pairs per block}."""
    lib = load()
    n = lib.ibpm_tune_table(None, 0)
    buf = C.create_string_buffer(max(n, 1))
    lib.ibpm_tune_table(buf, n)
    out = {}
    for line in buf.value.decode().splitlines():
        k, _, v = line.rpartition(" ")
        if k:
            out[k] = int(v)
    return out
