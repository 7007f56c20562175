"""The plain FP32 GPU form of the fit step and of predict: the comparator the optimised path is
measured against (``bench.py`` reports it beside the headline number).

It is what the reference's GPU backends do for one call, in FP32 and one launch per stage:

* neighbour search: ``nngp_plain_knn_f32`` -- one thread per query scanning its eligible refs
  and keeping a sorted list, the structure of the reference's ``calc_nn``
  (``nngpr/cuda_kernel_accelerators.py:663-743``); inputs divided by the length scale first
  (``:237-240``);
* local systems: the reference's worker arithmetic (``nngpr/base_nngpr.py:453-614`` for the
  log-likelihood and its gradient, ``:1032-1135`` for predict) on batched torch tensors --
  ``K`` and the materialised ``dK`` of every point, batched Cholesky, ``cholesky_solve`` per
  right-hand side, the same formulas -- in FP32, batch by batch.

Nothing here is used by the estimator; the optimised kernels are in ``csrc/``.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import _lib
from .kernel_params import RbfParams

LOG_2PI = math.log(2.0 * math.pi)


def _torch():
    import torch
    return torch


def plain_knn(ref, query, num_nn: int, ref_cut_index, length_scale, ref_root: str | None = None) -> 'torch.Tensor':
    """Neighbour lists ``(n_query, num_nn)`` int32 by the plain FP32 search (same lists as
    :func:`nngpr_b200.ops.knn`).  With ``ref_root`` (the installed reference), the reference's own
    ``calc_nn`` compiled from its source (:mod:`nngpr_b200.plain_ref`)."""
    torch = _torch()
    if ref_root is not None:
        from . import plain_ref
        return plain_ref.calc_nn(ref_root, ref, query, num_nn, ref_cut_index, length_scale)
    ref = ref.to(torch.float32)
    query = query.to(torch.float32)
    if length_scale is not None:
        ls = torch.as_tensor(np.broadcast_to(np.asarray(length_scale, dtype=np.float32), (ref.shape[1],)).copy(),
                             device=ref.device)
        ref = ref / ls
        query = query / ls
    ref = ref.contiguous()
    query = query.contiguous()
    out = torch.empty((query.shape[0], num_nn), dtype=torch.int32, device=ref.device)
    stream = torch.cuda.current_stream(ref.device).cuda_stream
    has_cut = ref_cut_index is not None
    st = _lib.lib().nngp_plain_knn_f32(ctypes.c_void_p(ref.data_ptr()), ref.shape[0],
                                       ctypes.c_void_p(query.data_ptr()), query.shape[0], ref.shape[1], num_nn,
                                       1 if has_cut else 0, int(ref_cut_index or 0), ctypes.c_void_p(out.data_ptr()),
                                       ctypes.c_void_p(stream))
    _lib.check(st, 'nngp_plain_knn_f32')
    return out


def _stationary(family: int, sq):
    """Stationary part and its length-scale gradient factor (RBF, ``batched_kernels.py:884-898``;
    Matern nu = 1/2, 3/2, 5/2, ``:1070-1120``)."""
    torch = _torch()
    if family == 0:
        S = torch.exp(-0.5 * sq)
        return S, S
    r = torch.sqrt(sq)
    if family == 1:
        S = torch.exp(-r)
        return S, torch.where(r > 0, S / torch.where(r > 0, r, 1.0), 0.0)
    if family == 2:
        a = math.sqrt(3.0) * r
        return (1.0 + a) * torch.exp(-a), 3.0 * torch.exp(-a)
    a = math.sqrt(5.0) * r
    return (1.0 + a + a * a / 3.0) * torch.exp(-a), 5.0 / 3.0 * (1.0 + a) * torch.exp(-a)


def _fill(xn, valid, p: RbfParams, ls, eval_gradient: bool):
    """``K (b, k, k)`` and, with ``eval_gradient``, ``dK (b, k, k, n_theta)`` of gathered points
    ``xn (b, k, d)`` -- the reference's fill (``cuda_kernel_accelerators.py:748-863``)."""
    torch = _torch()
    k = xn.shape[1]
    diff = (xn[:, :, None, :] - xn[:, None, :, :]) / ls
    sq = diff * diff
    S, Sg = _stationary(p.family, sq.sum(-1))
    E = p.rbf_level * S
    Eg = p.rbf_level * Sg  # d E / d log l_f = Eg * sq_f
    eye = torch.eye(k, dtype=torch.bool, device=xn.device)[None]
    pair = valid[:, :, None] & valid[:, None, :]
    K = torch.where(pair, E + p.const_value + torch.where(eye, p.noise_level, 0.0), 0.0)
    K = torch.where(~pair & eye, 1.0, K)
    if not eval_gradient:
        return K, None
    G = torch.zeros(K.shape + (p.n_theta,), dtype=K.dtype, device=K.device)
    if p.idx_noise >= 0:
        G[..., p.idx_noise] = torch.where(pair & eye, p.noise_level, 0.0)
    if p.idx_const >= 0:
        G[..., p.idx_const] = torch.where(pair, p.const_value, 0.0)
    if p.idx_rbf_level >= 0:
        G[..., p.idx_rbf_level] = torch.where(pair, E, 0.0)
    if p.idx_ls >= 0:
        if p.ard:
            for f in range(xn.shape[2]):
                G[..., p.idx_ls + f] = torch.where(pair, Eg * sq[..., f], 0.0)
        else:
            G[..., p.idx_ls] = torch.where(pair, Eg * sq.sum(-1), 0.0)
    return K, G


def plain_loglik(x, y, nbr, p: RbfParams, alpha: float, eval_gradient: bool = True, batch: int = 65536,
                 ref_root: str | None = None):
    """Log-likelihood (and gradient w.r.t. log theta) of all points in FP32 (per-point terms
    summed in FP64), ``x (n, d)``, ``y (n,)`` or ``(n, ydim)``, ``nbr (n, m)`` on the GPU.  With
    ``ref_root`` the fill is the reference's own ``fill_nn_kernel`` (:mod:`nngpr_b200.plain_ref`)."""
    torch = _torch()
    x = x.to(torch.float32)
    y = y.to(torch.float32)
    if y.dim() == 1:
        y = y[:, None]
    n, d = x.shape
    ls = torch.as_tensor(p.ls_vector(d), dtype=torch.float32, device=x.device)
    nbr = nbr.to(torch.int64)
    total = torch.zeros((), dtype=torch.float64, device=x.device)
    grad = torch.zeros(p.n_theta, dtype=torch.float64, device=x.device)
    for r0 in range(0, n, batch):
        rows = torch.arange(r0, min(n, r0 + batch), device=x.device)
        idx = torch.cat([rows[:, None], nbr[rows]], dim=1)
        valid = idx >= 0
        cl = idx.clamp(min=0)
        if ref_root is not None:
            from . import plain_ref
            K, G = plain_ref.fill_nn_kernel(ref_root, x, idx, p, eval_gradient)
        else:
            K, G = _fill(x[cl], valid, p, ls, eval_gradient)
        ii = torch.arange(idx.shape[1], device=x.device)
        K[:, ii, ii] += torch.where(valid, alpha, 0.0)
        L = torch.linalg.cholesky(K[:, 1:, 1:])
        y_nn = y[cl] * valid[..., None]
        yt = y[rows]
        K_xn = K[:, :1, 1:]
        a = torch.cholesky_solve(y_nn[:, 1:], L)
        b = torch.cholesky_solve(K_xn.transpose(1, 2), L)
        mu = (K_xn @ a)[:, 0, :]
        sigma = torch.sqrt(K[:, 0, 0][:, None] - (K_xn @ b)[:, 0, :])
        r = yt - mu
        ll = -0.5 * r ** 2 / sigma ** 2 - 0.5 * LOG_2PI - torch.log(sigma)
        total += ll.sum(-1).to(torch.float64).sum()
        if eval_gradient:
            for t in range(p.n_theta):
                Gt = G[..., t]
                dKnn = Gt[:, 1:, 1:]
                dkx = Gt[:, :1, 1:]
                dinv_y = -torch.cholesky_solve(dKnn @ a, L)
                dinv_k = -torch.cholesky_solve(dKnn @ b, L)
                dmu = (dkx @ a)[:, 0, :] + (K_xn @ dinv_y)[:, 0, :]
                dsig = 0.5 / sigma * (Gt[:, 0, 0][:, None] - 2 * (dkx @ b)[:, 0, :] - (K_xn @ dinv_k)[:, 0, :])
                g = (-1 / sigma + r ** 2 / sigma ** 3) * dsig + r / sigma ** 2 * dmu
                grad[t] += g.sum(-1).to(torch.float64).sum()
    return (total, grad) if eval_gradient else total


def plain_predict(x_train, y_train, x_query, nbr, p: RbfParams, alpha: float, batch: int = 65536,
                  ref_root: str | None = None):
    """Predictive mean ``(nq, ydim)`` and standard deviation ``(nq,)`` in FP32, conditioning on the
    training set only (the reference's ``only-train`` worker); with ``ref_root`` the fill is the
    reference's own ``fill_nn_kernel``."""
    torch = _torch()
    x_train = x_train.to(torch.float32)
    x_query = x_query.to(torch.float32)
    y_train = y_train.to(torch.float32)
    if y_train.dim() == 1:
        y_train = y_train[:, None]
    nt, nq = x_train.shape[0], x_query.shape[0]
    d = x_train.shape[1]
    ls = torch.as_tensor(p.ls_vector(d), dtype=torch.float32, device=x_train.device)
    x_full = torch.cat([x_train, x_query])
    nbr = nbr.to(torch.int64)
    means, stds = [], []
    for q0 in range(0, nq, batch):
        rows = torch.arange(q0, min(nq, q0 + batch), device=x_train.device)
        idx = torch.cat([(nt + rows)[:, None], nbr[rows]], dim=1)
        valid = idx >= 0
        if ref_root is not None:
            from . import plain_ref
            K, _ = plain_ref.fill_nn_kernel(ref_root, x_full, idx, p, False)
        else:
            K, _ = _fill(x_full[idx.clamp(min=0)], valid, p, ls, False)
        train = valid & (idx < nt)
        ii = torch.arange(idx.shape[1], device=x_train.device)
        K[:, ii, ii] += torch.where(train, alpha, 0.0)
        L = torch.linalg.cholesky(K[:, 1:, 1:])
        nb = idx[:, 1:]
        y_nn = y_train[nb.clamp(min=0)] * (nb >= 0)[..., None]
        K_xn = K[:, :1, 1:]
        means.append((K_xn @ torch.cholesky_solve(y_nn, L))[:, 0, :])
        stds.append(torch.sqrt(K[:, 0, 0] - (K_xn @ torch.cholesky_solve(K_xn.transpose(1, 2), L))[:, 0, 0]))
    return torch.cat(means), torch.cat(stds)
