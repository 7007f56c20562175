"""ctypes binding of ``libnngp_b200.so`` (the C ABI declared in ``include/nngp_b200.h``).

The library is built in-tree by ``nngpr_b200.build``.  There is no fallback: if the
shared library is missing or does not load, every GPU entry point raises.
"""

from __future__ import annotations

import ctypes
import os
import threading

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, 'libnngp_b200.so')

NNGP_OK = 0
NNGP_FLAG_BAD_INDEX = 1
NNGP_FLAG_NOT_PD = 2
NNGP_FLAG_TIMEOUT = 4
NNGP_FLAG_FP64_FALLBACK = 8

# every symbol include/nngp_b200.h declares
EXPORTED = (
    'nngp_abi_version', 'nngp_last_error', 'nngp_status_string', 'nngp_check_device', 'nngp_set_wait_limit_ns',
    'nngp_knn_workspace_size_f32', 'nngp_knn_f32', 'nngp_knn_workspace_size_f64', 'nngp_knn_f64',
    'nngp_loglik_workspace_size', 'nngp_loglik_f32', 'nngp_loglik_f64', 'nngp_loglik_fp64_count',
    'nngp_loglik_rows_f32', 'nngp_loglik_rows_f64', 'nngp_loglik_f64_noalloc',
    'nngp_predict_f32', 'nngp_predict_f64', 'nngp_fma_probe', 'nngp_fma_probe_f64', 'nngp_tc_layout_selftest',
    'nngp_tc_layout_selftest_bf16',
    'nngp_plain_knn_f32', 'nngp_knn_reuse_prepare_f32', 'nngp_knn_reuse_rank_f32',
    'nngp_predict_full_workspace_size', 'nngp_predict_full_f64', 'nngp_sample_full_f64',
    'nngp_predict_cov_full_f64', 'nngp_theta_params', 'nngp_knn_f32_ls_device', 'nngp_knn_f64_ls_device',
)


class NngpKernel(ctypes.Structure):
    """``struct nngp_kernel`` of ``include/nngp_b200.h``."""
    _fields_ = [
        ('rbf_level', ctypes.c_double),
        ('const_value', ctypes.c_double),
        ('noise_level', ctypes.c_double),
        ('alpha', ctypes.c_double),
        ('length_scale', ctypes.POINTER(ctypes.c_double)),
        ('n_ls', ctypes.c_int32),
        ('idx_rbf_level', ctypes.c_int32),
        ('idx_const', ctypes.c_int32),
        ('idx_noise', ctypes.c_int32),
        ('idx_ls', ctypes.c_int32),
        ('n_theta', ctypes.c_int32),
        ('family', ctypes.c_int32),
        ('dev_params', ctypes.c_void_p),  # device block of nngp_theta_params, or None
    ]


class NngpError(RuntimeError):
    """A failed libnngp_b200 call (status name and the library's message)."""


_lib = None
_lock = threading.Lock()

_vp, _i32, _i64, _f64, _sz = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_double, ctypes.c_size_t
_kp = ctypes.POINTER(NngpKernel)
_dp = ctypes.POINTER(ctypes.c_double)

_SIGS = {
    'nngp_abi_version': ([], _i32),
    'nngp_last_error': ([], ctypes.c_char_p),
    'nngp_status_string': ([ctypes.c_int], ctypes.c_char_p),
    'nngp_check_device': ([], ctypes.c_int),
    'nngp_knn_workspace_size_f32': ([_i64, _i64, _i32, _i32], _sz),
    'nngp_knn_workspace_size_f64': ([_i64, _i64, _i32, _i32], _sz),
    'nngp_knn_f32': ([_vp, _i64, _vp, _i64, _i32, _dp, _i32, _i32, _i32, _i64, _vp, _vp, _vp, _sz, _vp], ctypes.c_int),
    'nngp_knn_f64': ([_vp, _i64, _vp, _i64, _i32, _dp, _i32, _i32, _i32, _i64, _vp, _vp, _vp, _sz, _vp], ctypes.c_int),
    'nngp_knn_f32_ls_device': ([_vp, _i64, _vp, _i64, _i32, _vp, _i32, _i32, _i32, _i64, _vp, _vp, _vp, _sz, _vp],
                               ctypes.c_int),
    'nngp_knn_f64_ls_device': ([_vp, _i64, _vp, _i64, _i32, _vp, _i32, _i32, _i32, _i64, _vp, _vp, _vp, _sz, _vp],
                               ctypes.c_int),
    'nngp_theta_params': ([_kp, _vp, _i32, _f64, _vp, _vp], ctypes.c_int),
    'nngp_loglik_workspace_size': ([_i64, _i32, _i32, _i32, _i32], _sz),
    'nngp_loglik_fp64_count': ([_vp], _vp),
    'nngp_set_wait_limit_ns': ([ctypes.c_uint64], ctypes.c_uint64),
    'nngp_loglik_f32': ([_vp, _vp, _i64, _i32, _i32, _vp, _i32, _kp, _i32, _f64, _vp, _vp, _vp, _sz, _vp], ctypes.c_int),
    'nngp_loglik_f64': ([_vp, _vp, _i64, _i32, _i32, _vp, _i32, _kp, _i32, _f64, _vp, _vp, _vp, _sz, _vp], ctypes.c_int),
    'nngp_loglik_rows_f32': ([_vp, _vp, _i64, _i32, _i32, _i64, _i64, _vp, _i32, _kp, _i32, _f64, _vp, _vp, _vp, _sz, _vp],
                             ctypes.c_int),
    'nngp_loglik_rows_f64': ([_vp, _vp, _i64, _i32, _i32, _i64, _i64, _vp, _i32, _kp, _i32, _f64, _vp, _vp, _vp, _sz, _vp],
                             ctypes.c_int),
    'nngp_loglik_f64_noalloc': ([_vp, _vp, _i64, _i32, _i32, _vp, _i32, _kp, _i32, _vp, _vp, _vp], ctypes.c_int),
    'nngp_predict_f32': ([_vp, _vp, _i64, _vp, _i64, _i32, _i32, _vp, _i32, _kp, _f64, _vp, _vp, _vp, _vp], ctypes.c_int),
    'nngp_predict_f64': ([_vp, _vp, _i64, _vp, _i64, _i32, _i32, _vp, _i32, _kp, _f64, _vp, _vp, _vp, _vp], ctypes.c_int),
    'nngp_fma_probe': ([_vp, _i64, _i32, _vp], ctypes.c_int),
    'nngp_fma_probe_f64': ([_vp, _i64, _i32, _vp], ctypes.c_int),
    'nngp_tc_layout_selftest': ([_vp, _vp, _i32, _vp, _vp, _vp], ctypes.c_int),
    'nngp_tc_layout_selftest_bf16': ([_vp, _vp, _i32, _vp, _vp, _vp], ctypes.c_int),
    'nngp_plain_knn_f32': ([_vp, _i64, _vp, _i64, _i32, _i32, _i32, _i64, _vp, _vp], ctypes.c_int),
    'nngp_predict_full_workspace_size': ([_i64, _i32], ctypes.c_size_t),
    'nngp_predict_full_f64': ([_vp, _vp, _i64, _i64, _i32, _i32, _vp, _i32, ctypes.POINTER(NngpKernel), _i32, _vp,
                               _vp, _vp, _vp, ctypes.c_size_t, _vp], ctypes.c_int),
    'nngp_predict_cov_full_f64': ([_vp, _vp, _i64, _i64, _i32, _i32, _vp, _i32, ctypes.POINTER(NngpKernel), _vp,
                                   _vp, _vp, _vp, ctypes.c_size_t, _vp], ctypes.c_int),
    'nngp_sample_full_f64': ([_vp, _vp, _i64, _i64, _i32, _i32, _vp, _i32, ctypes.POINTER(NngpKernel), _i32, _vp,
                              _vp, _vp, _vp, ctypes.c_size_t, _vp], ctypes.c_int),
    'nngp_knn_reuse_prepare_f32': ([_vp, _i64, _i32, ctypes.c_double, _vp, _i32, ctypes.c_double, _vp, _vp],
                                   ctypes.c_int),
    'nngp_knn_reuse_rank_f32': ([_vp, _i64, _i32, ctypes.c_double, _vp, _i32, _vp, _i32, _vp, _vp, _vp],
                                ctypes.c_int),
}


def lib() -> ctypes.CDLL:
    """The loaded library (loaded once); raises ``ImportError`` if it is not built."""
    global _lib
    if _lib is None:
        with _lock:
            if _lib is None:
                if not os.path.exists(LIB_PATH):
                    raise ImportError(f'{LIB_PATH} is missing: build it with `python -m nngpr_b200.build`')
                handle = ctypes.CDLL(LIB_PATH)
                for name, (args, res) in _SIGS.items():
                    fn = getattr(handle, name)
                    fn.argtypes = args
                    fn.restype = res
                _lib = handle
    return _lib


def check(status: int, what: str) -> None:
    """Raise ``NngpError`` for a non-OK status, with the library's message."""
    if status != NNGP_OK:
        L = lib()
        name = L.nngp_status_string(status).decode()
        msg = L.nngp_last_error().decode()
        if status == 2:  # NNGP_ERR_UNSUPPORTED
            raise NotImplementedError(f'{what}: {name}: {msg}')
        raise NngpError(f'{what}: {name}: {msg}')
