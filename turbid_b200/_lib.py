"""ctypes binding of libturbid_gpu.so (declarations mirror include/turbid_gpu.h).

The library is loaded from this package directory only; a missing or stale
library is an error, never a silent fallback.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libturbid_gpu.so")

TG_OK = 0
TG_ERR_CUDA = 1
TG_ERR_SHAPE = 2
TG_ERR_ARG = 3
TG_ERR_NAN = 4
TG_ERR_SETUP = 5
TG_ERR_NOMEM = 6
TG_ERR_STATE = 7
TG_ERR_TIMEOUT = 8
TG_PREC_FP64 = 0
TG_PREC_MIXED = 1
TG_NFEATURE = 50
TG_PROF_NCAT = 10
PROF_NAMES = ["zgemm", "fft_fwd_x", "fft_fwd_y", "fft_bwd_y", "fft_bwd_x", "elementwise", "filter",
              "features", "advection_x", "islice"]

_c_d = ctypes.c_double
_c_i = ctypes.c_int
_pd = ctypes.POINTER(ctypes.c_double)
_pf = ctypes.POINTER(ctypes.c_float)
_pi = ctypes.POINTER(ctypes.c_int)
_vp = ctypes.c_void_p


class TgCase(ctypes.Structure):
    """struct tg_case (include/turbid_gpu.h)."""

    _fields_ = [
        ("nx", _c_i), ("ny", _c_i), ("nz", _c_i),
        ("lx", _c_d), ("ly", _c_d),
        ("nphase", _c_i),
        ("mapping", _c_i),
        ("mapping_coef", _c_d),
        ("slope", _c_d), ("slope_direction", _c_i),
        ("dt", _c_d),
        ("output_based_on_step", _c_i),
        ("reynolds", _c_d), ("froude", _c_d), ("averaged_concentration", _c_d), ("specific_gravity", _c_d),
        ("affected_by_scalar", _c_i),
        ("bc_u", _c_d * 5), ("bc_v", _c_d * 5), ("bc_w", _c_d * 5), ("bc_p", _c_d * 5),
        ("force_type", _c_i),
        ("force_direction", _c_i * 2),
        ("force_amplitude", _c_d * 4),
        ("schmidt", _c_d), ("settling", _c_d), ("erosion_rate", _c_d), ("critical_shear", _c_d),
        ("scalar_bc", _c_i),
        ("precision", _c_i),
    ]


class TgError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[tg status {code}] {msg}")
        self.code = code


# (name, restype, argtypes)
_SIGS = [
    ("tg_last_error", ctypes.c_char_p, []),
    ("tg_version", _c_i, []),
    ("tg_launch_count", ctypes.c_longlong, []),
    ("tg_create", _c_i, [ctypes.POINTER(TgCase), ctypes.POINTER(_vp)]),
    ("tg_destroy", _c_i, [_vp]),
    ("tg_get_dims", _c_i, [_vp, _pi]),
    ("tg_set_stream", _c_i, [_vp, _vp]),
    ("tg_synchronize", _c_i, [_vp]),
    ("tg_set_decomposition", _c_i, [_vp, _c_i, _pd, _pd, _pd, _pd, _pd, _pd, _pd]),
    ("tg_get_decomposition", _c_i, [_vp, _c_i, _pd, _pd, _pd, _pd, _pd, _pd, _pd]),
    ("tg_operators_host", _c_i, [_c_i, _c_i, _c_d, _pd, _pd]),
    ("tg_decomposition_host", _c_i, [_c_i, _c_i, _c_d, _pd, _pd, _pd, _pd, _pd, _pd, _pd, _pd]),
    ("tg_get_operators", _c_i, [_vp, _pd, _pd]),
    ("tg_upload_state", _c_i, [_vp, _pd, _pd, _pd, _c_i]),
    ("tg_download_state", _c_i, [_vp, _pd, _pd, _pd]),
    ("tg_set_time", _c_i, [_vp, _c_i, _c_d, _c_d, _c_i]),
    ("tg_get_time", _c_i, [_vp, _pi, _pd, _pd, _pi, _pi, _pd]),
    ("tg_carrier_predict", _c_i, [_vp, _c_i]),
    ("tg_carrier_correct", _c_i, [_vp, _c_i]),
    ("tg_scalar_predict", _c_i, [_vp, _c_i]),
    ("tg_scalar_correct", _c_i, [_vp, _c_i]),
    ("tg_run_steps", _c_i, [_vp, _c_i, _c_i, _c_d, _pd, _pi]),
    ("tg_set_graphs", _c_i, [_vp, _c_i]),
    ("tg_autotune", _c_i, [_vp, ctypes.c_char_p, _pi]),
    ("tg_swirling_strength", _c_i, [_vp, _pd]),
    ("tg_run_ensemble", _c_i, [ctypes.POINTER(ctypes.c_void_p), _c_i, _c_i, _c_i, _c_d, _pi]),
    ("tg_features", _c_i, [_vp, _pd]),
    ("tg_profile_begin", _c_i, [_vp]),
    ("tg_profile_end", _c_i, [_vp, _c_i, _pd, _pd, _pd, _pi]),
    ("tg_profile_executed", _c_i, [_vp, _c_i, _pd]),
    ("tg_dft_forward_f64", _c_i, [_vp, _vp, _vp, _c_i]),
    ("tg_dft_forward_f32", _c_i, [_vp, _vp, _vp, _c_i]),
    ("tg_dft_forward_f64_noalloc", _c_i, [_c_i, _c_i, _c_i, _vp, _vp, _c_i, _vp]),
    ("tg_dft_forward_planes", _c_i, [_vp, _vp, _vp, _c_i, _c_i]),
    ("tg_dft_backward_planes", _c_i, [_vp, _vp, _vp, _c_i, _c_i]),
    ("tg_dft_backward_f64", _c_i, [_vp, _vp, _vp, _c_i]),
    ("tg_dft_backward_f32", _c_i, [_vp, _vp, _vp, _c_i]),
    ("tg_multiply", _c_i, [_vp, _pd, _vp, _vp, _c_i]),
    ("tg_multiply_islice", _c_i, [_vp, _pd, _vp, _vp, _c_i]),
    ("tg_set_zsolver", _c_i, [_vp, _c_i]),
    ("tg_zsolver_error", _c_i, [_vp, _pi]),
    ("tg_islice_selftest", _c_i, [_vp]),
    ("tg_helmholtz", _c_i, [_vp, _c_i, _c_i, _vp, _vp]),
]

_lib = None


def load() -> ctypes.CDLL:
    """Load the in-tree library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: run `python -m turbid_b200.build` (no CPU fallback exists)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, res, args in _SIGS:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(status: int):
    if status != TG_OK:
        msg = load().tg_last_error()
        raise TgError(status, msg.decode() if msg else "")


def exported_names():
    return [s[0] for s in _SIGS]
