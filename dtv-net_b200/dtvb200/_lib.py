"""ctypes binding of the C ABI in include/dtv_b200.h (libdtvb200.so, in-tree).

Importing this module never falls back to anything: if the library is missing
or cannot be loaded, every call raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdtvb200.so")

DTV_OK, DTV_ERR_INVALID, DTV_ERR_CUDA, DTV_ERR_ALLOC, DTV_ERR_UNSUPPORTED = 0, 1, 2, 3, 4
DTV_F32, DTV_F16, DTV_BF16 = 0, 1, 2
DTV_PHASE_STANDARD, DTV_PHASE_VECTOR, DTV_PHASE_BOX = 0, 1, 2
DTV_PLAN_SOFT, DTV_PLAN_TEX, DTV_PLAN_STAGE_F16, DTV_PLAN_TEX_PAIRS = 0x0, 0x1, 0x2, 0x4
DTV_PLAN_ADJOINT = 0x8
DTV_PLAN_TMA = 0x10
DTV_PLAN_PAIRS_EXACT = 0x20
DTV_TUNE_FP_RAY_TILE = 1
DTV_TUNE_FP_TEX_SHARE = 2
DTV_TUNE_ADJOINT = 3
DTV_TUNE_FP_BAND = 4
DTV_TUNE_BP_WARP = 5
DTV_EPI_STORE, DTV_EPI_RESIDUAL, DTV_EPI_PDHG = 0, 1, 2


class DtvError(RuntimeError):
    """A C-ABI call returned an error status."""

    def __init__(self, fn: str, code: int, msg: str):
        super().__init__(f"{fn}: {msg} (code {code})")
        self.code = code


class dtv_geometry(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
        ("nu", ctypes.c_int32), ("nv", ctypes.c_int32), ("n_views", ctypes.c_int32),
        ("voxel", ctypes.c_double * 3), ("vol_offset", ctypes.c_double * 3),
        ("det_offset", ctypes.c_double * 2),
        ("fp_step", ctypes.c_double), ("fp_scale", ctypes.c_double),
        ("fp_phase", ctypes.c_int32), ("bp_weight_power", ctypes.c_int32),
        ("bp_scale", ctypes.c_double),
        ("bp_extent_check", ctypes.c_int32), ("reserved", ctypes.c_int32),
        ("views", ctypes.POINTER(ctypes.c_double)),
    ]


class dtv_pdhg_params(ctypes.Structure):
    _fields_ = [
        ("sigma", ctypes.c_float), ("tau", ctypes.c_float), ("mu", ctypes.c_float),
        ("v", ctypes.c_float * 3), ("quirk", ctypes.c_int32), ("f_dtype", ctypes.c_int32),
    ]


_P = ctypes.c_void_p
_I = ctypes.c_int32
_L = ctypes.c_int64
_F = ctypes.c_float
_D = ctypes.c_double
_IP = ctypes.POINTER(ctypes.c_int32)
_FP = ctypes.POINTER(ctypes.c_float)
_DP = ctypes.POINTER(ctypes.c_double)
_GP = ctypes.POINTER(dtv_geometry)

# name -> argtypes (all return int status unless listed in _RESTYPES)
SIGNATURES = {
    "dtv_version": [],
    "dtv_error_string": [ctypes.c_int],
    "dtv_last_error_message": [],
    "dtv_launch_count": [],
    "dtv_geometry_standard": [_GP, _DP, _FP, _I, _IP, _IP, _F, _F],
    "dtv_geometry_vector": [_GP, _DP, _FP, _I, _IP, _IP],
    "dtv_geometry_circular": [_GP, _DP, _DP, _I, _IP, _DP, _IP, _DP, _D, _D],
    "dtv_plan_create": [_GP, _I, _I, _I, ctypes.POINTER(_P)],
    "dtv_plan_destroy": [_P],
    "dtv_plan_set_tuning": [_P, _I, _I],
    "dtv_plan_get_tuning": [_P, _I, _IP],
    "dtv_plan_device_status": [_P, _IP, _I],
    "dtv_fbp_filter": [_P, _P, ctypes.c_int64, _I, _I, _F, _F, _F, _I, _P],
    "dtv_forward_many": [_P, _P, _I, _P, _I, _I, _P, _F, _P],
    "dtv_fista_update_many": [_P, _P, _P, _P, _I, _F, _F, _F, _P],
    "dtv_backward_many": [_P, _P, _P, _I, _I, _P],
    "dtv_plan_fp_samples": [_P, _DP],
    "dtv_forward": [_P, _P, _I, _I, _P, _I, _P, _F, _P, _P],
    "dtv_backward": [_P, _P, _I, _P, _I, _P],
    "dtv_backward_adjoint": [_P, _P, _I, _P, _P],
    "dtv_backward_onto": [_P, _P, _I, _P, _P, _P],
    "dtv_pdhg_forward_refresh": [_P, _P, _P, _I, _I, _P, _F, _P, _P, _P, _P],
    "dtv_backward_refresh": [_P, _P, _P, _I, _P, _P, _P],
    "dtv_standard_forward": [_P, _I, _FP, _I, _IP, _IP, _F, _F, _I, _P, _P],
    "dtv_standard_backward": [_P, _I, _FP, _I, _IP, _IP, _F, _F, _I, _P, _P],
    "dtv_vector_forward": [_P, _I, _IP, _IP, _FP, _I, _I, _P, _P],
    "dtv_vector_backward": [_P, _I, _IP, _IP, _FP, _I, _I, _P, _P],
    "dtv_diff": [_P, _P, _IP, _I, _I, _I, _I, _P],
    "dtv_diff_abs_sums": [_P, _I, _IP, _I, _I, _P, _P],
    "dtv_l1ball_workspace_bytes": [],
    "dtv_l1ball": [_P, _P, _L, _P, _P, _P, _P],
    "dtv_l1ball_noalloc": [_P, _P, _L, _P, _P, _P],
    "dtv_pdhg_workspace_bytes": [],
    "dtv_pdhg_dual": [_P, _P, _P, _P, _P, _IP, _I, ctypes.POINTER(dtv_pdhg_params), _P, _P, _P],
    "dtv_pdhg_primal": [_P, _P, _P, _P, _P, _P, _P, _IP, _I, ctypes.POINTER(dtv_pdhg_params),
                        _P, _P],
    "dtv_pdhg_dual_defer": [_P, _P, _P, _P, _P, _IP, _I, ctypes.POINTER(dtv_pdhg_params), _P, _P,
                            _P, _P],
    "dtv_pdhg_primal_defer": [_P, _P, _P, _P, _P, _P, _P, _IP, _I,
                              ctypes.POINTER(dtv_pdhg_params), _P, _P, _P],
    "dtv_fista_update": [_P, _P, _P, _L, _F, _F, _F, _P],
    "dtv_relu_step": [_P, _P, _P, _L, _F, _P],
    "dtv_dtvfista_maxes": [_P, _IP, _I, _FP, _P, _P],
    "dtv_dtvfista_update": [_P, _P, _IP, _I, _FP, _FP, _F, _I, _P, _P],
    "dtv_axpy_l1": [_P, _P, _F, _P, _L, _P],
    "dtv_tv_descent": [_P, _P, _IP, _I, _I, _P, _P],
    "dtv_scale_scalar": [_P, _D, _P, _P],
    "dtv_l1_distance": [_P, _P, _L, _P, _P],
    "dtv_lincomb": [_P, _F, _P, _F, _P, _L, _P],
    "dtv_pdhg_sino_dual": [_P, _P, _P, _F, _L, _P, _P],
    "dtv_asd_adapt": [_P, _P, _F, _F, _P, _P],
    "dtv_measure_texture_fetch_rate": [_I, _DP],
    "dtv_measure_texture_gather_rate": [_I, _DP],
    "dtv_measure_atomic_v4_rate": [_L, _I, _DP],
}
_RESTYPES = {
    "dtv_error_string": ctypes.c_char_p,
    "dtv_last_error_message": ctypes.c_char_p,
    "dtv_l1ball_workspace_bytes": ctypes.c_int64,
    "dtv_launch_count": ctypes.c_int64,
    "dtv_pdhg_workspace_bytes": ctypes.c_int64,
}

_lib = None


def load() -> ctypes.CDLL:
    """Load libdtvb200.so (raises if it is absent: there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing; build it with `python dtv-net_b200/build.py` "
            "(the CUDA kernels are the only implementation)")
    L = ctypes.CDLL(LIB_PATH)
    for name, args in SIGNATURES.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = _RESTYPES.get(name, ctypes.c_int)
    _lib = L
    return L


def call(name: str, *args) -> int:
    L = load()
    rc = getattr(L, name)(*args)
    if rc != DTV_OK:
        msg = L.dtv_last_error_message().decode(errors="replace")
        raise DtvError(name, rc, msg)
    return rc


def measure_texture_fetch_rate(texel_bits: int = 32) -> float:
    """Bilinear texture fetches per second of the current device (benchmarks)."""
    out = ctypes.c_double()
    call("dtv_measure_texture_fetch_rate", texel_bits, ctypes.byref(out))
    return out.value


def measure_texture_gather_rate(gather: int = 1) -> float:
    """Gathers (or bilinear fetches) per second from a tiled 2-D texture (benchmarks)."""
    out = ctypes.c_double()
    call("dtv_measure_texture_gather_rate", gather, ctypes.byref(out))
    return out.value


def measure_atomic_v4_rate(records: int = 72 << 16, pattern: int = 0) -> float:
    """16-byte vector reductions per second into L2-resident records (benchmarks)."""
    out = ctypes.c_double()
    call("dtv_measure_atomic_v4_rate", records, pattern, ctypes.byref(out))
    return out.value


def ivec(vals) -> ctypes.Array:
    vals = [int(v) for v in vals]
    return (ctypes.c_int32 * len(vals))(*vals)


def fvec(vals) -> ctypes.Array:
    vals = [float(v) for v in vals]
    return (ctypes.c_float * len(vals))(*vals)


def dvec(vals) -> ctypes.Array:
    vals = [float(v) for v in vals]
    return (ctypes.c_double * len(vals))(*vals)
