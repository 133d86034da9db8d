"""turbid_b200: B200 (sm_100a) implementation of TURBID's flat-bottom
Fourier-Chebyshev RK3 substep behind the reference's plugin interface.

The compute path is libturbid_gpu.so (hand-written CUDA, C ABI in
include/turbid_gpu.h); this package only loads it and mirrors the reference's
host-side interface for Python callers.
"""
from ._lib import TgCase, TgError, load, TG_PREC_FP64, TG_PREC_MIXED  # noqa: F401
from .config import Ini, make_case, params_from_ini, expression  # noqa: F401
from .solver import ChannelCase, decomposition_host, operators_host, run_ensemble, to_slab, from_slab  # noqa: F401
