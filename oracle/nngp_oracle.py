"""CPU oracle for the NNGP fit/predict hot path.

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` leg of ``bench.py`` may import this module, and only as the
checker.  The product path (``nngpr_b200``) never calls it and has no CPU
fallback.

This is a numpy restatement of the reference nngpr (stavoltafunzia/nngpr 0.1.1)
algorithm for the accelerated ``WhiteKernel + ConstantKernel * RBF`` path.
Every function names the reference lines it restates.  The restatement is
pinned by the golden vectors in ``tests/golden/`` that ``tests/golden/make_golden.py``
produced by running the reference ``NumpyNngpr`` itself (FP64, sequential), and
by the reference's own known-answer test (NNGP with ``num_nn = n`` equals the exact
GP of scikit-learn, ``nngpr/test/nngpr_base_tester.py:174-192``).

Kernel parameters are passed explicitly (``KernelParams``); turning a kernel
object into them is product code (``nngpr_b200.kernel_params``) and is tested
against the reference separately.
"""

from __future__ import annotations

import dataclasses
import math

import numpy as np

LOG_2PI = math.log(2.0 * math.pi)


@dataclasses.dataclass
class KernelParams:
    """Parameters of ``White(noise) + const + rbf_level * RBF(length_scale)``.

    Mirrors the dictionary returned by ``RbfAccelerator.get_kernel_params``
    (``nngpr/cuda_kernel_accelerators.py:520-581``) and the theta index map of
    ``get_kernel_theta_mapping`` (``:583-649``).  ``idx_*`` are positions in
    ``kernel.theta`` (``-1`` when the hyperparameter is fixed or absent);
    ``idx_ls`` is the first of ``len(length_scale)`` consecutive positions.
    """

    rbf_level: float = 1.0
    const_value: float = 0.0
    noise_level: float = 0.0
    length_scale: object = 1.0  # float (isotropic) or 1-D array (ARD)
    idx_rbf_level: int = -1
    idx_const: int = -1
    idx_noise: int = -1
    idx_ls: int = -1
    n_theta: int = 0
    family: int = 0  # stationary part: 0 RBF, 1/2/3 Matern nu = 1/2, 3/2, 5/2

    @property
    def ard(self) -> bool:
        return np.ndim(self.length_scale) > 0

    def ls_vector(self, d: int) -> np.ndarray:
        ls = np.asarray(self.length_scale, dtype=np.float64).reshape(-1)
        if ls.size == 1:
            return np.full(d, ls[0])
        assert ls.size == d
        return ls


# ----------------------------------------------------------------------------------------------
# Nearest neighbours
# ----------------------------------------------------------------------------------------------

def scale_for_search(x: np.ndarray, length_scale, dtype=np.float32) -> np.ndarray:
    """Inputs divided by the length scale in the search dtype.

    Restates ``cuda_kernel_accelerators.py:235-239``: the search arrays are cast
    to the search dtype first (``base_nngpr.py:1170-1173`` downcasts to float32
    unless ``allow_downcast_f32 == 'no'``), then ``x / ls`` is evaluated in that
    dtype (numpy promotion rules: a Python float length scale is cast to the
    array dtype; an ARD vector is cast with ``cp.array(ls, dtype=data_type)``).
    ``length_scale=None`` means input-space search (plain Euclidean, no scaling).
    """
    xs = np.asarray(x).astype(dtype, copy=False)
    if length_scale is None:
        return np.array(xs, dtype=dtype, copy=True)
    ls = np.asarray(length_scale, dtype=np.float64).reshape(-1).astype(dtype)
    return (xs / ls).astype(dtype, copy=False)


def pairwise_sqdist(query: np.ndarray, ref: np.ndarray) -> np.ndarray:
    """Squared distances ``sum_f (ref_f - query_f)^2`` accumulated feature by feature.

    Same operation order as the ``calc_nn`` kernel (``cuda_kernel_accelerators.py:718-723``):
    ``tmp = ref_f - query_f; distance += tmp * tmp`` for ``f = 0 .. d-1``.  numpy
    evaluates each step with one IEEE rounding (no fused multiply-add), which is the
    arithmetic the GPU kernels use for their exact distances, so the results agree
    bit for bit in float32 and float64.
    """
    dt = query.dtype
    out = np.zeros((query.shape[0], ref.shape[0]), dtype=dt)
    for f in range(query.shape[1]):
        t = ref[None, :, f] - query[:, None, f]
        out += t * t
    return out


def knn(ref: np.ndarray, query: np.ndarray, num_nn: int, ref_cut_index=None, length_scale=1.0,
        dtype=np.float32, chunk: int = 512, query_index=None) -> np.ndarray:
    """Exact top-``num_nn`` search, ascending distance, ties broken by the lower index.

    Semantics of ``NngprWorker.find_nearest_neighbors`` (``base_nngpr.py:1613-1686``) with
    the accelerated ``calc_nn`` ranking (``cuda_kernel_accelerators.py:663-743``):

    * kernel space = squared Euclidean distance of the length-scale-scaled inputs
      (``length_scale=None``: input space, unscaled);
    * with ``ref_cut_index = c`` query ``j`` may only use refs ``[0, j + c)``
      (``base_nngpr.py:1660-1671``, ``cuda_kernel_accelerators.py:357-362``);
      ``None`` means every ref;
    * equal distances keep the lower index first (the ``<=`` break of the insertion
      sort, ``cuda_kernel_accelerators.py:728``);
    * missing slots are ``-1`` (``base_nngpr.py:1648``, ``:1675-1681``).

    ``query_index`` (optional) gives each query row's position in the full query set, so
    that a sample of rows can be checked with the cut of its original position.

    Returns int32 of shape ``(n_query, num_nn)``.
    """
    refs = scale_for_search(ref, length_scale, dtype)
    qs = scale_for_search(query, length_scale, dtype)
    nr, nq = refs.shape[0], qs.shape[0]
    out = np.full((nq, num_nn), -1, dtype=np.int32)
    if nr == 0 or num_nn == 0:
        return out
    ar = np.arange(nr, dtype=np.int64)
    qidx = np.arange(nq, dtype=np.int64) if query_index is None else np.asarray(query_index, dtype=np.int64)
    for q0 in range(0, nq, chunk):
        q1 = min(nq, q0 + chunk)
        d2 = pairwise_sqdist(qs[q0:q1], refs)
        # (distance, index) packed into one int64: the bit pattern of a non-negative
        # IEEE float is monotone, so integer order == lexicographic (distance, index).
        if dtype == np.float32:
            bits = d2.view(np.int32).astype(np.int64)
            key = (bits << 32) | ar[None, :]
            big = np.int64(np.iinfo(np.int64).max)
        else:
            # float64 distances: sort with a stable argsort (ties -> lower index).
            key = None
        if ref_cut_index is not None:
            allowed = (qidx[q0:q1, None] + ref_cut_index) > ar[None, :]
        else:
            allowed = np.ones((q1 - q0, nr), dtype=bool)
        k = min(num_nn, nr)
        if key is not None:
            key = np.where(allowed, key, big)
            part = np.argpartition(key, k - 1, axis=1)[:, :k] if k < nr else np.tile(ar, (q1 - q0, 1))
            pk = np.take_along_axis(key, part, axis=1)
            order = np.argsort(pk, axis=1, kind='stable')
            sel = np.take_along_axis(part, order, axis=1)
        else:
            d2 = np.where(allowed, d2, np.inf)
            sel = np.argsort(d2, axis=1, kind='stable')[:, :k]
        ok = np.take_along_axis(allowed, sel, axis=1)
        sel = np.where(ok, sel, -1).astype(np.int32)
        out[q0:q1, :k] = sel
    return out


def fit_neighbours(x: np.ndarray, num_nn: int, length_scale=1.0, dtype=np.float32) -> np.ndarray:
    """Neighbour lists of the fit step: point ``i`` uses the ``num_nn`` nearest of the points
    ``[0, i)`` in input order (``base_nngpr.py:530-535`` with ``ref_cut_index = i0`` over the
    whole training set).  Returns ``(n, num_nn)`` without the self column."""
    return knn(x, x, num_nn, ref_cut_index=0, length_scale=length_scale, dtype=dtype)


# ----------------------------------------------------------------------------------------------
# Local covariance fill
# ----------------------------------------------------------------------------------------------

def stationary(family: int, sq: np.ndarray):
    """Unit-amplitude stationary kernel ``S`` at squared scaled distance ``sq`` and the factor
    ``Sg`` of its length-scale gradient, ``d S / d log l_f = Sg * sq_f``: RBF
    (``batched_kernels.py:884-898``) or Matern nu = 1/2, 3/2, 5/2 (``:1070-1120``; at distance 0
    the nu = 1/2 factor is taken as 0, its numerator vanishing there, as the reference does with
    its unit denominator)."""
    if family == 0:
        S = np.exp(-0.5 * sq)
        return S, S
    r = np.sqrt(sq)
    if family == 1:
        S = np.exp(-r)
        return S, np.where(r > 0, S / np.where(r > 0, r, 1.0), 0.0)
    if family == 2:
        a = np.sqrt(3.0) * r
        return (1.0 + a) * np.exp(-a), 3.0 * np.exp(-a)
    if family == 3:
        a = np.sqrt(5.0) * r
        return (1.0 + a + a * a / 3.0) * np.exp(-a), 5.0 / 3.0 * (1.0 + a) * np.exp(-a)
    raise ValueError(f'unknown kernel family {family}')


def fill_nn_kernel(x_full: np.ndarray, nn_indices: np.ndarray, p: KernelParams, eval_gradient: bool):
    """Local covariance ``K (b, k, k)`` and gradient ``dK (b, k, k, n_theta)`` of a neighbour list.

    Restates the ``fill_nn_kernel`` CUDA kernel (``cuda_kernel_accelerators.py:748-863``) and
    the generic fill (``base_nngpr.py:1781-1805``): for valid pairs
    ``K = rbf_level * exp(-sum_f d_f^2 / (2 l_f^2)) + const (+ noise on the index diagonal)``;
    a ``-1`` slot gives an identity row/column and a zero gradient.  Gradients are with
    respect to the log hyperparameters: noise -> ``noise`` on the diagonal, const -> ``const``,
    rbf_level -> the RBF part, isotropic l -> ``RBF * sum_f d_f^2 / l^2``, ARD l_f ->
    ``RBF * d_f^2 / l_f^2``.
    """
    x_full = np.asarray(x_full, dtype=np.float64)
    idx = np.asarray(nn_indices)
    b, k = idx.shape
    d = x_full.shape[1]
    valid = idx >= 0
    xn = x_full[np.where(valid, idx, 0)]  # (b, k, d)
    ls = p.ls_vector(d)
    diff = (xn[:, :, None, :] - xn[:, None, :, :]) / ls  # (b, k, k, d)
    sq = diff * diff
    S, Sg = stationary(p.family, sq.sum(-1))
    E = p.rbf_level * S
    Eg = p.rbf_level * Sg  # d E / d log l_f = Eg * sq_f
    eye = np.eye(k, dtype=bool)[None]
    pair = valid[:, :, None] & valid[:, None, :]
    K = np.where(pair, E + p.const_value + np.where(eye, p.noise_level, 0.0), 0.0)
    K = np.where(~pair & eye, 1.0, K)
    if not eval_gradient:
        return K, None
    G = np.zeros((b, k, k, p.n_theta))
    if p.idx_noise >= 0:
        G[..., p.idx_noise] = np.where(pair & eye, p.noise_level, 0.0)
    if p.idx_const >= 0:
        G[..., p.idx_const] = np.where(pair, p.const_value, 0.0)
    if p.idx_rbf_level >= 0:
        G[..., p.idx_rbf_level] = np.where(pair, E, 0.0)
    if p.idx_ls >= 0:
        if p.ard:
            for f in range(d):
                G[..., p.idx_ls + f] = np.where(pair, Eg * sq[..., f], 0.0)
        else:
            G[..., p.idx_ls] = np.where(pair, Eg * sq.sum(-1), 0.0)
    return K, G


# ----------------------------------------------------------------------------------------------
# Log-likelihood and gradient
# ----------------------------------------------------------------------------------------------

def _gather_y(y: np.ndarray, idx: np.ndarray) -> np.ndarray:
    """``_build_ytrain_given_nn_indices`` (``base_nngpr.py:1336-1368``): y of each neighbour,
    zero for ``-1`` slots."""
    valid = idx >= 0
    out = y[np.where(valid, idx, 0)]
    out[~valid] = 0.0
    return out


def _chol_solve(L: np.ndarray, rhs: np.ndarray) -> np.ndarray:
    """``K^-1 rhs`` from the lower Cholesky factor, batched (``numpy_nngpr.py:140-170`` does the
    same with LAPACK ``cho_solve`` one matrix at a time)."""
    z = np.linalg.solve(L, rhs)
    return np.linalg.solve(np.swapaxes(L, -1, -2), z)


def loglik_terms(x: np.ndarray, y: np.ndarray, nbr: np.ndarray, p: KernelParams, alpha: float,
                 eval_gradient: bool, rows=None):
    """Per-point log-likelihood (summed over outputs) and its per-point gradient.

    Restates ``Nngpr._log_likelihood_worker`` (``base_nngpr.py:453-614``) in FP64 for the
    points ``rows`` (default: all).  ``nbr`` is ``(n, m)`` without the self column; the
    self column is prepended as in ``base_nngpr.py:533-535``.
    """
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    if y.ndim == 1:
        y = y[:, None]
    rows = np.arange(x.shape[0]) if rows is None else np.asarray(rows)
    idx = np.concatenate([rows[:, None], np.asarray(nbr)[rows]], axis=1)
    K, dK = fill_nn_kernel(x, idx, p, eval_gradient)
    valid = idx >= 0
    # K[ind[0], ind[1], ind[1]] += alpha on every valid slot (base_nngpr.py:555-556)
    ii = np.arange(idx.shape[1])
    K[:, ii, ii] += np.where(valid, alpha, 0.0)
    n = K.shape[0]
    L = np.linalg.cholesky(K[:, 1:, 1:])  # base_nngpr.py:564
    y_nn = _gather_y(y, idx)  # (n, k, ydim)
    yt = y[rows]
    K_xn = K[:, 0, 1:][:, None, :]  # (n, 1, m)
    a = _chol_solve(L, y_nn[:, 1:])  # K_nn^-1 y_nn
    b = _chol_solve(L, np.swapaxes(K_xn, 1, 2))  # K_nn^-1 K_xn^T
    mu = (K_xn @ a)[:, 0, :]  # base_nngpr.py:578
    sigma = np.sqrt(K[:, 0, 0][:, None] - (K_xn @ b)[:, 0, :])  # :579-580
    ll = -0.5 * (yt - mu) ** 2 / sigma ** 2 - 0.5 * LOG_2PI - np.log(sigma)  # :581
    ll = ll.sum(-1)
    if not eval_gradient:
        return ll, None
    dK = np.moveaxis(dK, -1, 0)  # (t, n, k, k)
    dKnn = dK[:, :, 1:, 1:]
    dkx = dK[:, :, 0, 1:][:, :, None, :]  # (t, n, 1, m)
    # dK_nn^-1 r = -K_nn^-1 dK_nn K_nn^-1 r (base_nngpr.py:591-592)
    dinv_y = -_chol_solve(L[None], dKnn @ a[None])
    dinv_k = -_chol_solve(L[None], dKnn @ b[None])
    dmu = (dkx @ a[None])[:, :, 0, :] + (K_xn[None] @ dinv_y)[:, :, 0, :]  # :596-598
    dsig = 0.5 / sigma[None] * (dK[:, :, 0, 0][..., None] - 2 * (dkx @ b[None])[:, :, 0, :]
                                - (K_xn[None] @ dinv_k)[:, :, 0, :])  # :602-606
    r = (yt - mu)[None]
    g = (-1 / sigma[None] + r ** 2 / sigma[None] ** 3) * dsig + r / sigma[None] ** 2 * dmu  # :609-610
    return ll, g.sum(-1).T  # (n, t)


def log_marginal_likelihood(x, y, nbr, p: KernelParams, alpha: float, eval_gradient: bool = False,
                            chunk: int = 4096):
    """``Nngpr.log_marginal_likelihood`` (``base_nngpr.py:385-451``): sum of the per-point terms
    over all points and outputs (FP64)."""
    n = np.asarray(x).shape[0]
    total = 0.0
    grad = np.zeros(p.n_theta)
    for i0 in range(0, n, chunk):
        rows = np.arange(i0, min(n, i0 + chunk))
        ll, g = loglik_terms(x, y, nbr, p, alpha, eval_gradient, rows)
        total += float(ll.sum())
        if eval_gradient:
            grad += g.sum(0)
    return (total, grad) if eval_gradient else total


# ----------------------------------------------------------------------------------------------
# Predict (conditioning on the training set only)
# ----------------------------------------------------------------------------------------------

def predict(x_train, y_train, x_query, nbr, p: KernelParams, alpha: float):
    """Predictive mean ``(nq, ydim)`` and standard deviation ``(nq,)``.

    Restates ``Nngpr._predict_worker`` (``base_nngpr.py:1032-1135``) for
    ``conditioning_method='only-train'``: the query is column 0 of the local system
    (index ``nt + i`` in ``x_full = [x_train; x_query]``, ``base_nngpr.py:1461-1462``);
    alpha is added only to training slots (``:1106-1107``), so ``K_00`` carries the
    white noise but no alpha; ``mean = K_xn K_nn^-1 y_nn``, ``std = sqrt(K_00 - K_xn K_nn^-1 K_xn^T)``.
    ``nbr`` is ``(nq, m)`` of training indices (``-1`` padded).
    """
    x_train = np.asarray(x_train, dtype=np.float64)
    x_query = np.asarray(x_query, dtype=np.float64)
    y_train = np.asarray(y_train, dtype=np.float64)
    if y_train.ndim == 1:
        y_train = y_train[:, None]
    nt, nq = x_train.shape[0], x_query.shape[0]
    x_full = np.concatenate([x_train, x_query])
    idx = np.concatenate([np.arange(nt, nt + nq)[:, None], np.asarray(nbr)], axis=1)
    K, _ = fill_nn_kernel(x_full, idx, p, False)
    train = (idx >= 0) & (idx < nt)
    ii = np.arange(idx.shape[1])
    K[:, ii, ii] += np.where(train, alpha, 0.0)
    L = np.linalg.cholesky(K[:, 1:, 1:])
    y_nn = _gather_y(y_train, np.asarray(nbr))
    K_xn = K[:, :1, 1:]
    mean = (K_xn @ _chol_solve(L, y_nn))[:, 0, :]
    var = K[:, 0, 0] - (K_xn @ _chol_solve(L, np.swapaxes(K_xn, 1, 2)))[:, 0, 0]
    return mean, np.sqrt(var)


# ----------------------------------------------------------------------------------------------
# Neighbour-list reuse across length scales (restates nngpr_b200/csrc/knn_reuse.cu)
# ----------------------------------------------------------------------------------------------

UNIT_ROUNDOFF_F32 = 2.0 ** -24


def _scale_of(length_scale) -> np.float32:
    return np.float32(1.0) if length_scale is None else np.float32(np.asarray(length_scale).reshape(-1)[0])


def _cand_sqdist(xs: np.ndarray, rows: np.ndarray, cols: np.ndarray) -> np.ndarray:
    """Squared distances of the pairs (rows[k], cols[k]) in the search arithmetic (float32,
    ``ref - query`` per feature, accumulated feature by feature)."""
    out = np.zeros(rows.shape, dtype=xs.dtype)
    for f in range(xs.shape[1]):
        t = xs[cols, f] - xs[rows, f]
        out += t * t
    return out


def reuse_thresholds(x: np.ndarray, cand: np.ndarray, length_scale, max_norm: float) -> np.ndarray:
    """Per point: ``l0^2 D_l0(i, last candidate) - 2 * 2 (d + 6) u (|x_i| + max_norm)^2``, +inf
    when the candidate list holds every earlier point (its last slot is -1).  ``cand`` is the
    exact prefix search at ``length_scale`` (float32) with more slots than the lists need."""
    x32 = np.asarray(x, dtype=np.float32)
    n, d = x32.shape
    xs = scale_for_search(x32, length_scale)
    ls2 = float(_scale_of(length_scale)) ** 2
    thr = np.full(n, np.inf)
    last = np.asarray(cand)[:, -1]
    rows = np.nonzero(last >= 0)[0]
    tau = ls2 * _cand_sqdist(xs, rows, last[rows]).astype(np.float64)
    r = np.sqrt((x32[rows].astype(np.float64) ** 2).sum(1)) * (1 + 1e-12) + max_norm
    thr[rows] = tau - 2.0 * (2.0 * (d + 6) * UNIT_ROUNDOFF_F32) * r * r
    return thr


def reuse_rank(x: np.ndarray, cand: np.ndarray, thr: np.ndarray, length_scale, num_nn: int):
    """Exact top-``num_nn`` of each point's candidates at ``length_scale`` (ascending distance,
    lower index first) and the number of points whose ``num_nn``-th distance does not clear the
    threshold (for those the lists are not proven exact)."""
    x32 = np.asarray(x, dtype=np.float32)
    n = x32.shape[0]
    xs = scale_for_search(x32, length_scale)
    ls2 = float(_scale_of(length_scale)) ** 2
    cand = np.asarray(cand)
    out = np.full((n, num_nn), -1, dtype=np.int32)
    failed = 0
    rr, cc = np.nonzero(cand >= 0)
    dist = np.full(cand.shape, np.inf, dtype=np.float32)
    dist[rr, cc] = _cand_sqdist(xs, rr, cand[rr, cc])
    for i in range(n):
        ok = cand[i] >= 0
        js, ds = cand[i][ok], dist[i][ok]
        order = np.lexsort((js, ds))[:num_nn]
        out[i, :order.size] = js[order]
        if np.isinf(thr[i]):
            continue
        if order.size < num_nn or not (ls2 * float(ds[order[-1]]) * (1 + 1e-12) < thr[i]):
            failed += 1
    return out, failed


def double_nn_lists(x_train, x_query, num_nn: int, length_scale=1.0, dtype=np.float32) -> np.ndarray:
    """Neighbour lists of ``conditioning_method='full-double-nn'``
    (``base_nngpr.py:1418-1449``): ``min(num_nn, nt)`` nearest training points and
    ``min(num_nn, nq - 1)`` nearest earlier queries (indices offset by ``nt``), packed per row as
    the valid training entries, then the valid query entries, then ``-1``."""
    x_train = np.asarray(x_train)
    x_query = np.asarray(x_query)
    nt, nq = x_train.shape[0], x_query.shape[0]
    mq = max(0, min(num_nn, nq - 1))
    q = knn(x_query, x_query, mq, 0, length_scale, dtype) if mq > 0 else np.empty((nq, 0), np.int32)
    q = np.where(q >= 0, q + nt, -1).astype(np.int32)
    if nt == 0:
        return q
    t = knn(x_train, x_query, min(num_nn, nt), None, length_scale, dtype)
    both = np.concatenate([t, q], axis=1)
    out = np.full_like(both, -1)
    for i in range(nq):
        v = both[i][both[i] >= 0]
        out[i, :v.size] = v
    return out


def predict_full(x_train, y_train, x_query, nbr, p: KernelParams, alpha: float, return_std: bool = True):
    """Predict with ``conditioning_method='full'``: restates the sequential algorithm of
    ``Nngpr.predict`` (``base_nngpr.py:896-1030``) for ``return_cov=False``.  ``nbr`` is
    ``(nq, m)`` of indices into ``x_full = [x_train; x_query]`` (query ``i`` may use indices below
    ``nt + i``; ``-1`` padded).  Query neighbours contribute their predicted means; the variance
    adds ``w^T C w`` with ``C`` the covariance of the query neighbours, known only between a query
    and its own query neighbours (the reference's sparse partial covariance, ``:923-930``)."""
    x_train = np.asarray(x_train, dtype=np.float64)
    x_query = np.asarray(x_query, dtype=np.float64)
    y_train = np.asarray(y_train, dtype=np.float64)
    if y_train.ndim == 1:
        y_train = y_train[:, None]
    nt, nq = x_train.shape[0], x_query.shape[0]
    x_full = np.concatenate([x_train, x_query])
    nbr = np.asarray(nbr)
    m = nbr.shape[1]
    idx = np.concatenate([np.arange(nt, nt + nq)[:, None], nbr], axis=1)
    K, _ = fill_nn_kernel(x_full, idx, p, False)
    train = (idx >= 0) & (idx < nt)
    ii = np.arange(idx.shape[1])
    K[:, ii, ii] += np.where(train, alpha, 0.0)  # :952-954
    mean = np.full((nt + nq, y_train.shape[1]), np.nan)
    mean[:nt] = y_train
    var = np.full(nq, np.nan)
    pcov = {}  # (i, j) with j a query neighbour of query i (both query positions) -> covariance
    for i in range(nq):
        Kn = K[i, 1:, 1:]
        kx = K[i, 0, 1:]
        w = np.linalg.solve(Kn, kx)  # K_nn^-1 k (Kn symmetric)
        js = nbr[i]
        vals = np.where(js[:, None] >= 0, mean[np.where(js >= 0, js, 0)], 0.0)
        mean[nt + i] = w @ vals
        if not return_std:
            continue
        q = js >= nt
        C = np.zeros((m, m))
        for s in np.nonzero(q)[0]:
            a = js[s] - nt
            C[s, s] = var[a]
            for t in np.nonzero(q)[0]:
                b = js[t] - nt
                if a > b:
                    C[s, t] = C[t, s] = pcov.get((a, b), 0.0)
        raw = max(0.0, K[i, 0, 0] - kx @ w)
        var[i] = max(0.0, raw + w @ C @ w)
        cw = C @ w
        for s in np.nonzero(q)[0]:
            pcov[(i, js[s] - nt)] = cw[s]
    return mean[nt:], (np.sqrt(var) if return_std else None)


def sample_full(x_train, y_train, x_query, nbr, p: KernelParams, alpha: float, z: np.ndarray) -> np.ndarray:
    """Samples with ``conditioning_method='full'``: restates ``Nngpr.sample_y``'s sequential
    algorithm (``base_nngpr.py:691-750``) with the standard normals ``z (nq, ydim, n_samples)``
    given: query ``i``'s samples are ``w . v + max(0, sqrt(K_00 - k^T w)) z_i`` where ``v`` holds
    the training y and the samples of earlier query neighbours (normalised y units)."""
    x_train = np.asarray(x_train, dtype=np.float64)
    x_query = np.asarray(x_query, dtype=np.float64)
    y_train = np.asarray(y_train, dtype=np.float64)
    if y_train.ndim == 1:
        y_train = y_train[:, None]
    nt, nq = x_train.shape[0], x_query.shape[0]
    x_full = np.concatenate([x_train, x_query])
    nbr = np.asarray(nbr)
    idx = np.concatenate([np.arange(nt, nt + nq)[:, None], nbr], axis=1)
    K, _ = fill_nn_kernel(x_full, idx, p, False)
    train = (idx >= 0) & (idx < nt)
    ii = np.arange(idx.shape[1])
    K[:, ii, ii] += np.where(train, alpha, 0.0)
    out = np.full(z.shape, np.nan)
    for i in range(nq):
        w = np.linalg.solve(K[i, 1:, 1:], K[i, 0, 1:])
        v = np.zeros((nbr.shape[1],) + z.shape[1:])
        for s, j in enumerate(nbr[i]):
            if j < 0:
                continue
            v[s] = y_train[j][:, None] if j < nt else out[j - nt]
        s2 = K[i, 0, 0] - K[i, 0, 1:] @ w
        sig = np.sqrt(s2) if s2 > 0 else 0.0
        out[i] = np.einsum('i,ijk->jk', w, v) + sig * z[i]
    return out


def predict_cov_full(x_train, y_train, x_query, nbr, p: KernelParams, alpha: float):
    """Predict with ``conditioning_method='full'`` and ``return_cov=True``: restates the dense
    branch of the sequential algorithm (``base_nngpr.py:896-1030``): the covariance of every pair
    of queries is kept, ``cov[i, :i] = w_q^T cov[q-neighbours, :i]``, ``cov[i, i]`` the variance
    (normalised y units)."""
    x_train = np.asarray(x_train, dtype=np.float64)
    x_query = np.asarray(x_query, dtype=np.float64)
    y_train = np.asarray(y_train, dtype=np.float64)
    if y_train.ndim == 1:
        y_train = y_train[:, None]
    nt, nq = x_train.shape[0], x_query.shape[0]
    x_full = np.concatenate([x_train, x_query])
    nbr = np.asarray(nbr)
    idx = np.concatenate([np.arange(nt, nt + nq)[:, None], nbr], axis=1)
    K, _ = fill_nn_kernel(x_full, idx, p, False)
    train = (idx >= 0) & (idx < nt)
    ii = np.arange(idx.shape[1])
    K[:, ii, ii] += np.where(train, alpha, 0.0)
    mean = np.full((nt + nq, y_train.shape[1]), np.nan)
    mean[:nt] = y_train
    cov = np.zeros((nq, nq))
    for i in range(nq):
        w = np.linalg.solve(K[i, 1:, 1:], K[i, 0, 1:])
        js = nbr[i]
        vals = np.where(js[:, None] >= 0, mean[np.where(js >= 0, js, 0)], 0.0)
        mean[nt + i] = w @ vals
        q = np.nonzero(js >= nt)[0]
        a = js[q] - nt
        C = cov[np.ix_(a, a)]
        raw = max(0.0, K[i, 0, 0] - K[i, 0, 1:] @ w)
        var = max(0.0, raw + w[q] @ C @ w[q])
        if i > 0 and q.size:
            row = w[q] @ cov[a, :i]
            cov[i, :i] = row
            cov[:i, i] = row
        cov[i, i] = var
    return mean[nt:], cov
