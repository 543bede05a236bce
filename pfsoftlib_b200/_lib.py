"""ctypes binding of the engine's C ABI (include/pfsoft_b200.h).

Loading fails loudly: there is no CPU implementation behind these names, so a missing or
unbuildable ``libpfsoft_b200.so`` raises instead of degrading.
"""
from __future__ import annotations

import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpfsoft_b200.so")

PFSOFT_OK, PFSOFT_EINVAL, PFSOFT_ENOMEM, PFSOFT_ETIMEOUT, PFSOFT_ECUDA, PFSOFT_EBUSY, PFSOFT_ECANCELED = range(7)

_c_int, _c_size, _c_double, _vp = ctypes.c_int, ctypes.c_size_t, ctypes.c_double, ctypes.c_void_p

# name -> (restype, argtypes); every symbol declared in include/pfsoft_b200.h
SIGNATURES = {
    "pfsoft_status_string": (ctypes.c_char_p, [_c_int]),
    "pfsoft_last_error": (ctypes.c_char_p, []),
    "pfsoft_version": (_c_int, []),
    "pfsoft_coef_count": (_c_size, [_c_int]),
    "pfsoft_grid_bytes": (_c_size, [_c_int]),
    "pfsoft_workspace_bytes": (_c_size, [_c_int]),
    "pfsoft_cuda_dsoft": (_c_int, [_vp, _c_int, _vp, _vp, _c_size, _vp]),
    "pfsoft_cuda_idsoft": (_c_int, [_vp, _c_int, _vp, _vp, _c_size, _vp]),
    "pfsoft_cuda_dsoft_noalloc": (_c_int, [_vp, _c_int, _vp, _vp]),
    "pfsoft_batch_create": (_c_int, [_vp, _c_int, _c_int, _c_int, _vp]),
    "pfsoft_batch_destroy": (_c_int, [_vp]),
    "pfsoft_batch_workspace_bytes": (_c_size, [_vp]),
    "pfsoft_batch_transforms_per_cta": (_c_int, [_vp]),
    "pfsoft_batch_dsoft": (_c_int, [_vp, _vp, _vp, _vp]),
    "pfsoft_batch_idsoft": (_c_int, [_vp, _vp, _vp, _vp]),
    "pfsoft_split_supported": (_c_int, [_c_int]),
    "pfsoft_batch_status": (_c_int, [_vp]),
    "pfsoft_dsoft_host": (_c_int, [_vp, _c_int, _vp]),
    "pfsoft_idsoft_host": (_c_int, [_vp, _c_int, _vp]),
    "pfsoft_cuda_layer_wise_dft2": (_c_int, [_c_int, _c_int, _c_int, _vp, _c_double, _vp]),
    "pfsoft_cuda_layer_wise_idft2": (_c_int, [_c_int, _c_int, _c_int, _vp, _c_double, _vp]),
    "pfsoft_layer_wise_dft2_host": (_c_int, [_c_int, _c_int, _c_int, _vp, _c_double]),
    "pfsoft_layer_wise_idft2_host": (_c_int, [_c_int, _c_int, _c_int, _vp, _c_double]),
    "pfsoft_cuda_quadrature_weights": (_c_int, [_c_int, _vp, _vp]),
    "pfsoft_cuda_wigner_d_matrix": (_c_int, [_c_int, _c_int, _c_int, _c_int, _vp, _vp]),
    "pfsoft_cuda_random_coeffs": (_c_int, [_vp, _c_int, ctypes.c_ulonglong, _c_int, _c_double, _vp]),
    "pfsoft_launch_count": (ctypes.c_longlong, []),
    "pfsoft_tune_dwt_case_split": (_c_int, [_c_int, _c_int]),
    "pfsoft_tune_fft_fused": (_c_int, [_c_int, _c_int]),
    "pfsoft_tune_split_bandwidth": (_c_int, [_c_int, _c_int]),
    "pfsoft_test_split_wait_ns": (_c_int, [ctypes.c_ulonglong]),
    "pfsoft_server_create": (_c_int, [_c_size, _c_int, _c_int, _vp]),
    "pfsoft_server_create_ex": (_c_int, [_c_size, _c_int, _c_int, _c_int, _vp]),
    "pfsoft_server_destroy": (_c_int, [_vp]),
    "pfsoft_server_submit": (_c_int, [_vp, _c_int, _c_int, _vp, _vp, _vp, _vp]),
    "pfsoft_server_poll": (_c_int, [_vp, ctypes.c_longlong]),
    "pfsoft_server_wait": (_c_int, [_vp, ctypes.c_longlong, _c_double]),
    "pfsoft_server_cancel": (_c_int, [_vp, ctypes.c_longlong]),
    "pfsoft_server_pause": (_c_int, [_vp, _c_int]),
    "pfsoft_server_drain": (_c_int, [_vp, _c_double]),
    "pfsoft_server_get_stats": (_c_int, [_vp, _vp]),
    "pfsoft_server_reset_stats": (_c_int, [_vp]),
    "pfsoft_shard_create": (_c_int, [_c_int, _c_int, _c_int, _vp]),
    "pfsoft_shard_destroy": (None, [_vp]),
    "pfsoft_shard_layers": (_c_int, [_vp, _c_int, _vp, _vp]),
    "pfsoft_shard_classes": (_c_int, [_vp, _c_int, _vp, _c_int]),
    "pfsoft_shard_bins": (ctypes.c_longlong, [_vp, _c_int, _vp, ctypes.c_longlong]),
    "pfsoft_shard_counts": (_c_int, [_vp, _c_int, _vp, _vp]),
    "pfsoft_shard_runs": (ctypes.c_longlong, [_vp, _c_int, _c_int, _vp, _vp, _vp, _vp, ctypes.c_longlong]),
    "pfsoft_shard_fft_forward": (_c_int, [_vp, _vp, _vp, _vp]),
    "pfsoft_shard_dwt_forward": (_c_int, [_vp, _vp, _vp, _vp]),
    "pfsoft_shard_dwt_inverse": (_c_int, [_vp, _vp, _vp, _vp]),
    "pfsoft_shard_fft_inverse": (_c_int, [_vp, _vp, _vp, _vp]),
    "pfsoft_shard_scatter": (_c_int, [_vp, _c_int, _vp, _vp, _vp]),
    "pfsoft_shard_pack": (_c_int, [_vp, _c_int, _vp, _vp, _vp]),
    "pfsoft_shard_unpack": (_c_int, [_vp, _c_int, _vp, _vp, _vp]),
    "pfsoft_profile_enable": (_c_int, [_c_int]),
    "pfsoft_profile_read": (_c_int, [_vp, _vp, _c_int]),
    "pfsoft_profile_stage_name": (ctypes.c_char_p, [_c_int]),
}


class PfsoftError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{msg} (status {status})")
        self.status = status


_lock = threading.Lock()
_lib = None


def load(build_if_missing: bool = True):
    """The loaded library. Builds it with nvcc if the .so is absent or stale."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        from . import build as _build
        if build_if_missing and not _build.up_to_date():
            _build.build()
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing; build it with `python -m pfsoftlib_b200.build`")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _lib = lib
        return lib


def check(rc: int) -> None:
    if rc != PFSOFT_OK:
        lib = load()
        detail = lib.pfsoft_last_error().decode() or lib.pfsoft_status_string(rc).decode()
        raise PfsoftError(rc, detail)
