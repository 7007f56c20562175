"""Torch-facing wrappers of the C ABI (one call = one stream-ordered library call).

Tensors must be CUDA, contiguous, float32 or float64 (``nbr``: int32).  Workspaces come
from torch's caching allocator, the stream is torch's current stream.  Each wrapper
returns device tensors plus a device int32 status word (``NNGP_FLAG_*`` bits) that the
caller reads when it synchronises anyway; ``raise_on_flags`` turns it into exceptions.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .kernel_params import RbfParams

# FP32 local systems with a Cholesky pivot (sigma^2 included) below this fraction of the kernel
# diagonal are re-solved in FP64.  Measured on 20,000 points of the n=434,874, d=3, l=0.2,
# noise 1e-3 workload against the FP64 oracle: 1e-3 -> 2.4e-5 relative lml error (FP32 keeps
# the sigma^2 ~ 1e-3 systems), 3e-3 -> 6e-8, 1e-2 -> 6e-9.
DEFAULT_PIVOT_TOL = 1e-2


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _check_tensor(t, name, dtypes=(torch.float32, torch.float64)):
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError(f'{name} must be a CUDA tensor')
    if t.dtype not in dtypes:
        raise TypeError(f'{name} must have dtype in {dtypes}, got {t.dtype}')
    if not t.is_contiguous():
        raise ValueError(f'{name} must be contiguous')


def _ls_array(length_scale, d):
    """Host double array of the length scales (``None``: no scaling)."""
    if length_scale is None:
        return None, 0
    ls = np.ascontiguousarray(np.asarray(length_scale, dtype=np.float64).reshape(-1))
    if ls.size not in (1, d):
        raise ValueError(f'length_scale has {ls.size} entries for {d} features')
    return ls, ls.size


def new_flags(device) -> torch.Tensor:
    return torch.zeros(1, dtype=torch.int32, device=device)


def predict_full(x_train: torch.Tensor, y_train: torch.Tensor, x_query: torch.Tensor, nbr: torch.Tensor,
                 p: RbfParams, alpha: float, want_var: bool = True, flags: torch.Tensor | None = None):
    """Predict with ``conditioning_method='full'`` (FP64): mean ``(nq, ydim)`` and variance ``(nq,)``
    (``None`` without ``want_var``).  ``nbr`` indexes ``[x_train; x_query]``: the search of that
    array for ``x_query`` with ``ref_cut_index = n_train``."""
    for t, nm in ((x_train, 'x_train'), (y_train, 'y_train'), (x_query, 'x_query')):
        _check_tensor(t, nm, (torch.float64,))
    _check_tensor(nbr, 'nbr', (torch.int32,))
    nt, d = x_train.shape
    nq = x_query.shape[0]
    y2 = y_train if y_train.dim() == 2 else y_train.reshape(nt, 1)
    ydim = y2.shape[1]
    m = nbr.shape[1] if nbr.dim() == 2 else 0
    x_full = torch.cat([x_train, x_query]).contiguous()
    mean = torch.empty((nq, ydim), dtype=torch.float64, device=x_query.device)
    var = torch.empty((nq,), dtype=torch.float64, device=x_query.device) if want_var else None
    if nq == 0:
        return mean, var
    keep = []
    k = _kernel_struct(p, alpha, d, keep)
    L = _lib.lib()
    ws_bytes = int(L.nngp_predict_full_workspace_size(nq, m))
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=x_query.device)
    st = L.nngp_predict_full_f64(_ptr(x_full), _ptr(y2), nt, nq, d, ydim, _ptr(nbr), m, ctypes.byref(k),
                                 1 if want_var else 0, _ptr(mean), _ptr(var), _ptr(flags), _ptr(ws), ws_bytes,
                                 _stream())
    _lib.check(st, 'nngp_predict_full_f64')
    return mean, var


def predict_cov_full(x_train: torch.Tensor, y_train: torch.Tensor, x_query: torch.Tensor, nbr: torch.Tensor,
                     p: RbfParams, alpha: float, flags: torch.Tensor | None = None):
    """Predict with ``conditioning_method='full'`` and the dense predictive covariance (FP64):
    mean ``(nq, ydim)`` and covariance ``(nq, nq)`` (normalised y units)."""
    for t, nm in ((x_train, 'x_train'), (y_train, 'y_train'), (x_query, 'x_query')):
        _check_tensor(t, nm, (torch.float64,))
    _check_tensor(nbr, 'nbr', (torch.int32,))
    nt, d = x_train.shape
    nq = x_query.shape[0]
    y2 = y_train if y_train.dim() == 2 else y_train.reshape(nt, 1)
    ydim = y2.shape[1]
    m = nbr.shape[1] if nbr.dim() == 2 else 0
    x_full = torch.cat([x_train, x_query]).contiguous()
    mean = torch.empty((nq, ydim), dtype=torch.float64, device=x_query.device)
    cov = torch.empty((nq, nq), dtype=torch.float64, device=x_query.device)
    if nq == 0:
        return mean, cov
    keep = []
    k = _kernel_struct(p, alpha, d, keep)
    L = _lib.lib()
    ws_bytes = int(L.nngp_predict_full_workspace_size(nq, m))
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=x_query.device)
    st = L.nngp_predict_cov_full_f64(_ptr(x_full), _ptr(y2), nt, nq, d, ydim, _ptr(nbr), m, ctypes.byref(k),
                                     _ptr(mean), _ptr(cov), _ptr(flags), _ptr(ws), ws_bytes, _stream())
    _lib.check(st, 'nngp_predict_cov_full_f64')
    return mean, cov


def sample_full(x_train: torch.Tensor, y_train: torch.Tensor, x_query: torch.Tensor, nbr: torch.Tensor,
                p: RbfParams, alpha: float, z: torch.Tensor, flags: torch.Tensor | None = None) -> torch.Tensor:
    """Samples with ``conditioning_method='full'`` (FP64) from the standard normals ``z``
    ``(nq, ydim, n_samples)``: query ``i`` conditions on the training y and on the samples of the
    queries before it.  ``nbr`` as for :func:`predict_full`."""
    for t, nm in ((x_train, 'x_train'), (y_train, 'y_train'), (x_query, 'x_query'), (z, 'z')):
        _check_tensor(t, nm, (torch.float64,))
    _check_tensor(nbr, 'nbr', (torch.int32,))
    nt, d = x_train.shape
    nq = x_query.shape[0]
    y2 = y_train if y_train.dim() == 2 else y_train.reshape(nt, 1)
    ydim = y2.shape[1]
    if z.dim() != 3 or z.shape[0] != nq or z.shape[1] != ydim:
        raise ValueError('z must be (n_query, ydim, n_samples)')
    ns = z.shape[2]
    m = nbr.shape[1] if nbr.dim() == 2 else 0
    x_full = torch.cat([x_train, x_query]).contiguous()
    out = torch.empty_like(z)
    if nq == 0 or ns == 0:
        return out
    keep = []
    k = _kernel_struct(p, alpha, d, keep)
    L = _lib.lib()
    ws_bytes = int(L.nngp_predict_full_workspace_size(nq, m))
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=x_query.device)
    st = L.nngp_sample_full_f64(_ptr(x_full), _ptr(y2), nt, nq, d, ydim, _ptr(nbr), m, ctypes.byref(k), ns,
                                _ptr(z.contiguous()), _ptr(out), _ptr(flags), _ptr(ws), ws_bytes, _stream())
    _lib.check(st, 'nngp_sample_full_f64')
    return out


def knn_reuse_prepare(x: torch.Tensor, cand: torch.Tensor, length_scale, max_norm: float) -> torch.Tensor:
    """Per-point thresholds (float64 ``(n,)``) that let :func:`knn_reuse_rank` prove a reused
    list exact: ``cand`` is the FP32 prefix search of ``x`` (float32 ``(n, d)``) at the scalar
    ``length_scale`` (``None``: input space) with more slots than the lists will need;
    ``max_norm`` bounds every row's 2-norm."""
    _check_tensor(x, 'x', (torch.float32,))
    _check_tensor(cand, 'cand', (torch.int32,))
    n, d = x.shape
    thr = torch.empty(n, dtype=torch.float64, device=x.device)
    ls = 1.0 if length_scale is None else float(np.asarray(length_scale).reshape(-1)[0])
    st = _lib.lib().nngp_knn_reuse_prepare_f32(_ptr(x), n, d, ls, _ptr(cand), cand.shape[1], float(max_norm),
                                              _ptr(thr), _stream())
    _lib.check(st, 'nngp_knn_reuse_prepare_f32')
    return thr


def knn_reuse_rank(x: torch.Tensor, cand: torch.Tensor, thr: torch.Tensor, length_scale, num_nn: int):
    """Top-``num_nn`` of the candidates at a new scalar length scale, and a device int32 count
    of the points whose list is not proven equal to :func:`knn`'s (0: every list is exact)."""
    _check_tensor(x, 'x', (torch.float32,))
    _check_tensor(cand, 'cand', (torch.int32,))
    n, d = x.shape
    out = torch.empty((n, num_nn), dtype=torch.int32, device=x.device)
    failed = torch.zeros(1, dtype=torch.int32, device=x.device)
    ls = 1.0 if length_scale is None else float(np.asarray(length_scale).reshape(-1)[0])
    st = _lib.lib().nngp_knn_reuse_rank_f32(_ptr(x), n, d, ls, _ptr(cand), cand.shape[1], _ptr(thr), num_nn,
                                           _ptr(out), _ptr(failed), _stream())
    _lib.check(st, 'nngp_knn_reuse_rank_f32')
    return out, failed


def raise_on_flags(flags: int, what: str) -> None:
    """Turn a status word into an exception (bad index / timeout) or a LinAlgError."""
    if flags & _lib.NNGP_FLAG_TIMEOUT:
        raise _lib.NngpError(f'{what}: a bounded wait inside the kernel gave up (results invalid)')
    if flags & _lib.NNGP_FLAG_BAD_INDEX:
        raise IndexError(f'{what}: a neighbour index was outside the training set')
    if flags & _lib.NNGP_FLAG_NOT_PD:
        raise np.linalg.LinAlgError(f'{what}: a local covariance matrix is not positive definite')


def knn(ref: torch.Tensor, query: torch.Tensor, num_nn: int, ref_cut_index=None, length_scale=None,
        flags: torch.Tensor | None = None) -> torch.Tensor:
    """Nearest neighbours of each query among ``ref`` (int32 ``(n_query, num_nn)``, -1 padded).

    Same contract as ``NngprWorker.find_nearest_neighbors`` (``base_nngpr.py:1613-1686``):
    kernel-space search divides by ``length_scale`` (``None`` = input space), ``ref_cut_index``
    restricts query ``j`` to refs ``[0, j + ref_cut_index)``.  Computes in the dtype of the
    inputs (both must match).  ``length_scale`` may be a float64 CUDA tensor (1 or d values): it
    is then read on the device (``nngp_knn_f32_ls_device`` / ``_f64_ls_device``).
    """
    _check_tensor(ref, 'ref')
    _check_tensor(query, 'query')
    if ref.dtype != query.dtype:
        raise TypeError('ref and query must have the same dtype')
    if ref.dim() != 2 or query.dim() != 2 or ref.shape[1] != query.shape[1]:
        raise ValueError('ref and query must be 2-D with the same number of features')
    n_ref, d = ref.shape
    n_q = query.shape[0]
    out = torch.empty((n_q, num_nn), dtype=torch.int32, device=query.device)
    if n_q == 0 or num_nn == 0:
        return out
    L = _lib.lib()
    f64 = ref.dtype == torch.float64
    size_fn = L.nngp_knn_workspace_size_f64 if f64 else L.nngp_knn_workspace_size_f32
    ws_bytes = int(size_fn(n_ref, n_q, d, num_nn))
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=query.device)
    if isinstance(length_scale, torch.Tensor) and length_scale.is_cuda:
        _check_tensor(length_scale, 'length_scale', (torch.float64,))
        n_ls = length_scale.numel()
        if n_ls not in (1, d):
            raise ValueError('length_scale must hold 1 or d values')
        has_cut = ref_cut_index is not None
        fn = L.nngp_knn_f64_ls_device if f64 else L.nngp_knn_f32_ls_device
        st = fn(_ptr(ref), n_ref, _ptr(query), n_q, d, _ptr(length_scale), n_ls, num_nn, int(has_cut),
                int(ref_cut_index) if has_cut else 0, _ptr(out), _ptr(flags), _ptr(ws), ws_bytes, _stream())
        _lib.check(st, 'nngp_knn')
        return out
    ls, n_ls = _ls_array(length_scale, d)
    fn = L.nngp_knn_f64 if f64 else L.nngp_knn_f32
    ls_p = ls.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if ls is not None else None
    has_cut = ref_cut_index is not None
    st = fn(_ptr(ref), n_ref, _ptr(query), n_q, d, ls_p, n_ls, num_nn, int(has_cut),
            int(ref_cut_index) if has_cut else 0, _ptr(out), _ptr(flags), _ptr(ws), ws_bytes, _stream())
    _lib.check(st, 'nngp_knn')
    return out


def _kernel_struct(p: RbfParams, alpha: float, d: int, keep: list) -> _lib.NngpKernel:
    k = _lib.NngpKernel()
    k.rbf_level = float(p.rbf_level)
    k.const_value = float(p.const_value)
    k.noise_level = float(p.noise_level)
    k.alpha = float(alpha)
    if p.length_scale is None:
        k.length_scale = None
        k.n_ls = 0
    else:
        ls = np.ascontiguousarray(np.asarray(p.length_scale, dtype=np.float64).reshape(-1))
        keep.append(ls)
        k.length_scale = ls.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        k.n_ls = ls.size
    k.idx_rbf_level = p.idx_rbf_level
    k.idx_const = p.idx_const
    k.idx_noise = p.idx_noise
    k.idx_ls = p.idx_ls
    k.n_theta = p.n_theta
    k.family = int(p.family)
    k.dev_params = None
    return k


def theta_params(p: RbfParams, theta: torch.Tensor, alpha: float, d: int,
                 pivot_tol: float | None = DEFAULT_PIVOT_TOL) -> torch.Tensor:
    """The hyperparameter values at a DEVICE ``theta`` (float64 CUDA tensor, the layout of
    ``kernel.theta``), computed on the device (``nngp_theta_params``): a float64 tensor
    ``[rbf, const, noise, pivot_abs, 1/l_0..1/l_{d-1}, l_0..l_{d-1}]`` for ``loglik(...,
    params_dev=...)`` and, from index ``4 + d``, the device length scale of :func:`knn`.  ``p``
    gives the structure (which hyperparameters are free, the fixed values)."""
    _check_tensor(theta, 'theta', (torch.float64,))
    if theta.numel() != p.n_theta:
        raise ValueError(f'theta has {theta.numel()} entries, the kernel {p.n_theta}')
    keep = []
    k = _kernel_struct(p, alpha, d, keep)
    out = torch.empty(4 + 2 * d, dtype=torch.float64, device=theta.device)
    th = theta.contiguous()
    st = _lib.lib().nngp_theta_params(ctypes.byref(k), _ptr(th), d,
                                      float(DEFAULT_PIVOT_TOL if pivot_tol is None else pivot_tol), _ptr(out),
                                      _stream())
    _lib.check(st, 'nngp_theta_params')
    return out


def loglik(x: torch.Tensor, y: torch.Tensor, nbr: torch.Tensor, p: RbfParams, alpha: float,
           eval_gradient: bool, pivot_tol: float | None = DEFAULT_PIVOT_TOL,
           flags: torch.Tensor | None = None, out: torch.Tensor | None = None,
           row_begin: int = 0, stats: dict | None = None,
           params_dev: torch.Tensor | None = None) -> torch.Tensor:
    """Fit-step log-likelihood (and gradient) on the device: float64 tensor ``[lml, grad...]``.

    ``x (n, d)``, ``y (n, ydim)`` of one dtype (float32: FP32 systems with FP64 fallback;
    float64: FP64), ``nbr (rows, m)`` int32 without the self column, for the points
    ``[row_begin, row_begin + rows)`` (default: all points).  ``params_dev`` (from
    :func:`theta_params`) makes the kernels read the hyperparameter values from the device
    instead of ``p``'s (``p`` still gives the structure).  With a ``stats`` dict,
    ``stats['fp64_systems']`` receives a device int64 0-d tensor: the systems this call re-solved
    in FP64 (``nngp_loglik_fp64_count``).
    """
    _check_tensor(x, 'x')
    _check_tensor(y, 'y')
    _check_tensor(nbr, 'nbr', (torch.int32,))
    if y.dtype != x.dtype:
        raise TypeError('x and y must have the same dtype')
    n, d = x.shape
    y2 = y if y.dim() == 2 else y.reshape(n, 1)
    ydim = y2.shape[1]
    m = nbr.shape[1] if nbr.dim() == 2 else 0
    rows = nbr.shape[0]
    if row_begin < 0 or row_begin + rows > n:
        raise ValueError('nbr rows fall outside the points')
    nt = 1 + (p.n_theta if eval_gradient else 0)
    if out is None:
        out = torch.empty(nt, dtype=torch.float64, device=x.device)
    keep = []
    k = _kernel_struct(p, alpha, d, keep)
    if params_dev is not None:  # the values of a device theta (theta_params), read by the kernels
        _check_tensor(params_dev, 'params_dev', (torch.float64,))
        if params_dev.numel() < 4 + 2 * d:
            raise ValueError('params_dev is shorter than theta_params writes')
        k.dev_params = params_dev.data_ptr()
    L = _lib.lib()
    ws_bytes = int(L.nngp_loglik_workspace_size(max(rows, 1), d, ydim, m, p.n_theta))
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=x.device)
    fn = L.nngp_loglik_rows_f64 if x.dtype == torch.float64 else L.nngp_loglik_rows_f32
    st = fn(_ptr(x), _ptr(y2), n, d, ydim, int(row_begin), rows, _ptr(nbr), m, ctypes.byref(k),
            int(bool(eval_gradient)), float(DEFAULT_PIVOT_TOL if pivot_tol is None else pivot_tol), _ptr(out),
            _ptr(flags), _ptr(ws), ws_bytes, _stream())
    _lib.check(st, 'nngp_loglik')
    if stats is not None:
        off = int(L.nngp_loglik_fp64_count(_ptr(ws))) - ws.data_ptr()
        stats['fp64_systems'] = ws[off:off + 8].view(torch.int64)[0]
    return out


def predict(x_train: torch.Tensor, y_train: torch.Tensor, x_query: torch.Tensor, nbr: torch.Tensor,
            p: RbfParams, alpha: float, pivot_tol: float | None = DEFAULT_PIVOT_TOL,
            flags: torch.Tensor | None = None):
    """Predictive mean ``(nq, ydim)`` and variance ``(nq,)`` conditioned on the training set."""
    for t, nm in ((x_train, 'x_train'), (y_train, 'y_train'), (x_query, 'x_query')):
        _check_tensor(t, nm)
    _check_tensor(nbr, 'nbr', (torch.int32,))
    if not (x_train.dtype == y_train.dtype == x_query.dtype):
        raise TypeError('x_train, y_train and x_query must have the same dtype')
    nt, d = x_train.shape
    nq = x_query.shape[0]
    y2 = y_train if y_train.dim() == 2 else y_train.reshape(nt, 1)
    ydim = y2.shape[1]
    m = nbr.shape[1] if nbr.dim() == 2 else 0
    mean = torch.empty((nq, ydim), dtype=x_query.dtype, device=x_query.device)
    var = torch.empty((nq,), dtype=x_query.dtype, device=x_query.device)
    if nq == 0:
        return mean, var
    keep = []
    k = _kernel_struct(p, alpha, d, keep)
    L = _lib.lib()
    fn = L.nngp_predict_f64 if x_query.dtype == torch.float64 else L.nngp_predict_f32
    st = fn(_ptr(x_train), _ptr(y2), nt, _ptr(x_query), nq, d, ydim, _ptr(nbr), m, ctypes.byref(k),
            float(DEFAULT_PIVOT_TOL if pivot_tol is None else pivot_tol), _ptr(mean), _ptr(var), _ptr(flags),
            _stream())
    _lib.check(st, 'nngp_predict')
    return mean, var
