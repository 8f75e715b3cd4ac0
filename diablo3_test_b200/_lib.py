"""ctypes binding of libdiablo_gpu (the C ABI in include/diablo_gpu.h).

The shared library is built in-tree (``diablo3_test_b200/libdiablo_gpu.so``,
see ``diablo3_test_b200/build.py``).  Loading fails loudly when it is missing:
there is no CPU fallback for the channel step.
"""
from __future__ import annotations

import ctypes
import os

from .config import CParams

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libdiablo_gpu.so")

# status codes (enum diablo_status)
OK = 0
ENSEMBLE_BRANCHES, ENSEMBLE_PERSISTENT = 0, 1
ERR_ARG = -1
ERR_SIZE = -2
ERR_CUDA = -3
ERR_NONFINITE = -4
ERR_TIMEOUT = -5
ERR_UNSUPPORTED = -6
ERR_STATE = -7
ERR_NOMEM = -8

# field ids and layouts
U1, U2, U3, P, TH = 0, 1, 2, 3, 4
LAYOUT_FOURIER, LAYOUT_PHYSICAL = 0, 1

# diablo_stats output: profile names in the order of the DIABLO_STAT_* enums
STAT_PROFILES = ("ume", "vme", "wme", "mke", "urms", "vrms", "wrms", "uv", "uw", "wv",
                 "uu_dudx", "vv_dvdy", "wu_dwdx", "vu_dvdx", "uv_dudy", "wv_dwdy",
                 "dudy", "dwdy", "cp", "shear", "omega_x", "omega_y", "omega_z",
                 "epsilon", "epsilon_m", "nu_sgs", "eps_sgs2")
STAT_TH_PROFILES = ("thme", "dthdy", "thrms", "thv", "thv_m", "pe_diss", "kappa_sgs")
STAT_SCALARS = ("time", "dt", "ubulk", "urms_b", "vrms_b", "wrms_b", "u1y_left_b", "bpe")
STAT_ZSTAR = ("shear2", "thw", "chi", "epsilon", "TKE", "KE")

# every symbol include/diablo_gpu.h declares: name -> (restype, argtypes)
_vp = ctypes.c_void_p
_i = ctypes.c_int
_d = ctypes.c_double
SIGNATURES = {
    "diablo_create": (_vp, [ctypes.POINTER(CParams), _vp, ctypes.POINTER(_i)]),
    "diablo_destroy": (_i, [_vp]),
    "diablo_upload_state": (_i, [_vp, _i, _vp, _i]),
    "diablo_download_state": (_i, [_vp, _i, _vp, _i]),
    "diablo_download_nu_t": (_i, [_vp, _vp]),
    "diablo_adjoint_record": (_i, [_vp, _i, _i]),
    "diablo_adjoint_run": (_i, [_vp, _vp]),
    "diablo_autotune": (_i, [_vp, _vp]),
    "diablo_tiles": (_i, [_vp, _vp]),
    "diablo_ensemble_create": (_vp, [_vp, _i, _vp]),
    "diablo_ensemble_step": (_i, [_vp, _i]),
    "diablo_ensemble_synchronize": (_i, [_vp]),
    "diablo_ensemble_stream": (_vp, [_vp]),
    "diablo_ensemble_autotune": (_i, [_vp, _i]),
    "diablo_ensemble_set_mode": (_i, [_vp, _i]),
    "diablo_step_host": (_i, [_vp, _vp, _i]),
    "diablo_ensemble_mode": (_i, [_vp]),
    "diablo_ensemble_destroy": (_i, [_vp]),
    "diablo_fft_xz_to_fourier": (_i, [_vp, _vp, _vp]),
    "diablo_fft_xz_to_physical": (_i, [_vp, _vp, _vp]),
    "diablo_rk_substep": (_i, [_vp, _i]),
    "diablo_step": (_i, [_vp, _i]),
    "diablo_pre_first_step": (_i, [_vp, _i]),
    "diablo_apply_bc_post": (_i, [_vp]),
    "diablo_filter_chan": (_i, [_vp, _i]),
    "diablo_stats_size": (_i, [_vp]),
    "diablo_stats": (_i, [_vp, _i, ctypes.POINTER(_d), _i]),
    "diablo_les_eps_sgs1": (_i, [_vp, ctypes.POINTER(_d), _i]),
    "diablo_set_precision": (_i, [_vp, _i]),
    "diablo_get_time": (_i, [_vp, ctypes.POINTER(_d), ctypes.POINTER(_i), ctypes.POINTER(_d)]),
    "diablo_set_time": (_i, [_vp, _d, _i, _d]),
    "diablo_set_stream": (_i, [_vp, _vp]),
    "diablo_synchronize": (_i, [_vp]),
    "diablo_check_finite": (_i, [_vp]),
    "diablo_set_wait_bound": (_i, [_vp, ctypes.c_longlong, _i]),
    "diablo_kernel_launches": (ctypes.c_longlong, [_vp]),
    "diablo_set_profiling": (_i, [_vp, _i]),
    "diablo_kernel_times": (_i, [_vp, _i, ctypes.POINTER(_d), ctypes.POINTER(ctypes.c_longlong)]),
    "diablo_kernel_slots": (_i, []),
    "diablo_kernel_name": (ctypes.c_char_p, [_i]),
    "diablo_status_string": (ctypes.c_char_p, [_i]),
    "diablo_fft_xz_to_fourier_noalloc": (_i, [_i, _i, _i, _vp, _vp, _vp]),
    "diablo_abi_version": (_i, []),
}

_lib = None


class DiabloError(RuntimeError):
    def __init__(self, status: int, what: str):
        self.status = status
        msg = load().diablo_status_string(status).decode() if _lib is not None else str(status)
        super().__init__(f"{what} failed: {msg} ({status})")


def load() -> ctypes.CDLL:
    """Load libdiablo_gpu.so once and declare its signatures."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is missing; build it with `python -c 'import __graft_entry__ as g; g.build()'` "
            "(there is no CPU fallback for the channel step)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(status: int, what: str) -> None:
    if status != OK:
        raise DiabloError(status, what)
