"""``B200Nngpr``: the scikit-learn NNGP regressor with its hot path on one B200.

Drop-in beside the reference's ``NumpyNngpr`` / ``TorchNngpr`` (``nngpr/base_nngpr.py:26``):
same constructor keywords, the same ``fit`` / ``log_marginal_likelihood`` / ``predict``
contract, the same kernels (``WhiteKernel + ConstantKernel * RBF`` trees built from
scikit-learn or ``nngpr.batched_kernels`` classes).  What changes is below the API:

* the reference's multi-process worker pool (``distribute``, ``base_nngpr.py:193-269``) is
  replaced by a single-device scheduler: one stream-ordered sequence of library calls per
  fit step, with the training set kept resident in HBM between calls;
* the per-batch worker arithmetic (``_log_likelihood_worker`` :453-614, ``_predict_worker``
  :1032-1135) runs in the fused CUDA kernels of ``libnngp_b200.so``.

Precision follows the reference's ``allow_downcast_f32`` (``base_nngpr.py:66-72``):
``'only-nn'`` (default) searches neighbours in FP32 and solves the local systems in FP64;
``'yes'`` solves them in FP32 (FP64 re-solve below ``pivot_tol``); ``'no'`` is FP64 throughout.

``predict`` and ``sample_y`` support ``conditioning_method='only-train'``, ``'full'`` and
``'full-double-nn'`` (the reference's sequential algorithms, on the device), ``return_std`` and
``return_cov``; the sequential ones take up to 64 neighbour slots (``num_nn <= 64`` for
``'full'``, ``<= 32`` for ``'full-double-nn'``) and raise ``NotImplementedError`` above.
Kernels outside the accelerated family raise
``NotImplementedError("Cannot accelerate this kernel ...")`` as the reference's CUDA path does.
"""

from __future__ import annotations

import multiprocessing
from numbers import Integral, Real

import numpy as np
import torch
from sklearn import base as sk_base
from sklearn.gaussian_process import GaussianProcessRegressor
from sklearn.gaussian_process import kernels as skk
from sklearn.preprocessing._data import _handle_zeros_in_scale
from sklearn.utils import check_random_state
from sklearn.utils._param_validation import Interval, StrOptions
from sklearn.utils.validation import validate_data

from . import _lib, ops
from .kernel_params import RbfParams, extract


class B200Nngpr(GaussianProcessRegressor):
    """Nearest Neighbour Gaussian Process regressor (Datta 2016) on one B200 GPU.

    Parameters are those of the reference ``Nngpr`` (``base_nngpr.py:40-123``) plus:

    device : str or torch.device, default 'cuda'
        The CUDA device holding the training set and running the kernels.
    pivot_tol : float, default 1e-2
        With ``allow_downcast_f32='yes'``, an FP32 local system whose Cholesky pivot falls
        below ``pivot_tol`` times the kernel diagonal is re-solved in FP64 (1e-2 keeps the
        log-likelihood within 1e-5 of FP64 for nuggets down to 1e-3; ``ops.DEFAULT_PIVOT_TOL``).
    keep_resident : bool, default True
        Keep the training set in HBM between calls.  ``False`` uploads it on every call, the
        reference's behaviour.
    reuse_neighbours : bool, default False
        Reuse the fit step's neighbour lists across calls whose length scale changes
        (isotropic or no length scale, FP32 search): one wider search keeps 16 candidates more
        per point, later calls rank the candidates at the new length scale and keep the result
        only where a rounding bound proves it equal to a fresh search (``ops.knn_reuse_rank``);
        otherwise the search runs again.  Results are identical either way.
    optimizer : 'fmin_l_bfgs_b', 'device-lbfgs', callable or None
        As scikit-learn's, plus ``'device-lbfgs'``: ``torch.optim.LBFGS`` on the device through
        the differentiable log-likelihood (``nngpr_b200.autograd``).

    ``distribute_method``, ``mp_start_method``, ``random_gen_batch_byte_size`` and
    ``distribute_environ`` are accepted for signature compatibility; with one device and
    no worker pool they have no effect.  ``batch_size`` is accepted and ignored: the
    kernels stream over all points in one launch.
    """

    _parameter_constraints: dict = {
        **GaussianProcessRegressor._parameter_constraints,
        "num_nn": [Interval(Integral, 1, None, closed="left"), None],
        "nn_type": [StrOptions({"kernel-space", "input-space"}), None],
        "batch_size": [Interval(Integral, 1, None, closed="left"), None],
        "allow_downcast_f32": [StrOptions({"yes", "no", "only-nn"}), None],
        "distribute_method": [StrOptions({"joblib", "multiprocessing", "multiprocessing-heterogenous",
                                          "sequential"}), None],
        "mp_start_method": [StrOptions(set(multiprocessing.get_all_start_methods())), None],
        "random_gen_batch_byte_size": [Interval(Integral, 1, None, closed="left"), None],
        "distribute_environ": [dict, None],
        "device": [str, torch.device, None],
        "pivot_tol": [Interval(Real, 0, None, closed="left")],
        "keep_resident": ["boolean"],
        "reuse_neighbours": ["boolean"],
        "optimizer": [StrOptions({"fmin_l_bfgs_b", "device-lbfgs"}), callable, None],
    }

    def __init__(self, kernel=None, *, alpha=1e-10, optimizer="fmin_l_bfgs_b", n_restarts_optimizer=0,
                 normalize_y=False, copy_X_train=True, n_targets=None, random_state=None, num_nn=None,
                 nn_type=None, batch_size=None, allow_downcast_f32=None, distribute_method=None,
                 mp_start_method=None, random_gen_batch_byte_size=None, distribute_environ=None,
                 device=None, pivot_tol=1e-2, keep_resident=True, reuse_neighbours=False):
        super().__init__(kernel=kernel, alpha=alpha, optimizer=optimizer,
                         n_restarts_optimizer=n_restarts_optimizer, normalize_y=normalize_y,
                         copy_X_train=copy_X_train, n_targets=n_targets, random_state=random_state)
        self.num_nn = num_nn
        self.nn_type = nn_type
        self.batch_size = batch_size
        self.allow_downcast_f32 = allow_downcast_f32
        self.distribute_method = distribute_method
        self.mp_start_method = mp_start_method
        self.random_gen_batch_byte_size = random_gen_batch_byte_size
        self.distribute_environ = distribute_environ
        self.device = device
        self.pivot_tol = pivot_tol
        self.keep_resident = keep_resident
        self.reuse_neighbours = reuse_neighbours

    # ---- resolved settings ----------------------------------------------------------------
    @property
    def _num_nn(self) -> int:
        return 32 if self.num_nn is None else int(self.num_nn)

    @property
    def _nn_type(self) -> str:
        return 'kernel-space' if self.nn_type is None else self.nn_type

    @property
    def _downcast(self) -> str:
        return 'only-nn' if self.allow_downcast_f32 is None else self.allow_downcast_f32

    @property
    def _device(self) -> torch.device:
        dev = torch.device('cuda' if self.device is None else self.device)
        if dev.type != 'cuda':
            raise ValueError('B200Nngpr runs on a CUDA device only (no CPU fallback)')
        return dev

    def get_default_kernel(self):
        """Default kernel of the reference (``base_nngpr.py:1137-1150``)."""
        return skk.ConstantKernel(1.0, constant_value_bounds="fixed") * skk.RBF(1.0, length_scale_bounds="fixed")

    def _params(self, kernel) -> RbfParams:
        return extract(kernel)

    def _search_ls(self, p: RbfParams):
        """Length scales of the neighbour search (``None``: input-space / no RBF term),
        ``cuda_kernel_accelerators.py:235-239``."""
        if self._nn_type == 'kernel-space' and p.length_scale is not None:
            return p.length_scale
        return None

    # ---- device residency -----------------------------------------------------------------
    def _pinned(self, dtype):
        """Pinned host copies of the training arrays in ``dtype`` (made once per fit)."""
        cache = self.__dict__.setdefault('_pinned_cache', {})
        if dtype not in cache:
            x = np.ascontiguousarray(self.X_train_, dtype=np.float64)
            y = np.asarray(self.y_train_, dtype=np.float64)
            y = np.ascontiguousarray(y[:, None] if y.ndim == 1 else y)
            xt = torch.from_numpy(x).to(dtype)
            yt = torch.from_numpy(y).to(dtype)
            if torch.cuda.is_available():
                xt, yt = xt.pin_memory(), yt.pin_memory()
            cache[dtype] = (xt, yt)
        return cache[dtype]

    def _train_tensors(self, dtype):
        """Device copies of (X, y) in ``dtype``.  With ``keep_resident`` they are uploaded once
        per fit and stay in HBM; otherwise every call uploads them again from pinned host
        memory, as the reference does on every worker call (``base_nngpr.py:498``)."""
        dev = self._device
        if self.keep_resident:
            cache = self.__dict__.setdefault('_device_cache', {})
            if dtype not in cache:
                xh, yh = self._pinned(dtype)
                cache[dtype] = (xh.to(dev, non_blocking=True), yh.to(dev, non_blocking=True))
            return cache[dtype]
        xh, yh = self._pinned(dtype)
        return xh.to(dev, non_blocking=True), yh.to(dev, non_blocking=True)

    def _drop_device_copies(self):
        self.__dict__.pop('_nn_cache', None)
        self.__dict__.pop('_device_cache', None)
        self.__dict__.pop('_pinned_cache', None)

    # ---- fit ------------------------------------------------------------------------------
    @sk_base._fit_context(prefer_skip_nested_validation=True)
    def fit(self, X, y):
        """Fit the regressor (``base_nngpr.py:272-383``): validate, normalise y, then maximise
        the log-likelihood with scikit-learn's L-BFGS-B driver over device fit steps."""
        _lib.lib()  # fail loudly before any work if the extension is missing
        if self.kernel is None:
            self.kernel_ = self.get_default_kernel()
        else:
            self.kernel_ = sk_base.clone(self.kernel)
        self._rng = check_random_state(self.random_state)
        if self.kernel_.requires_vector_input:
            dtype, ensure_2d = "numeric", True
        else:
            dtype, ensure_2d = None, False
        X, y = validate_data(self, X, y, multi_output=True, y_numeric=True, ensure_2d=ensure_2d, dtype=dtype)
        n_targets_seen = y.shape[1] if y.ndim > 1 else 1
        if self.n_targets is not None and n_targets_seen != self.n_targets:
            raise ValueError("The number of targets seen in `y` is different from the parameter "
                             f"`n_targets`. Got {n_targets_seen} != {self.n_targets}.")
        if self.normalize_y:
            self._y_train_mean = np.mean(y, axis=0)
            self._y_train_std = _handle_zeros_in_scale(np.std(y, axis=0), copy=False)
            y = (y - self._y_train_mean) / self._y_train_std
        else:
            shape_y_stats = (y.shape[1],) if y.ndim == 2 else 1
            self._y_train_mean = np.zeros(shape=shape_y_stats)
            self._y_train_std = np.ones(shape=shape_y_stats)
        if np.iterable(self.alpha):
            if self.alpha.shape[0] == 1:
                self.alpha = self.alpha[0]
            else:
                raise ValueError("alpha must be a scalar or an array with only one element")
        self.X_train_ = np.copy(X) if self.copy_X_train else X
        self.y_train_ = np.copy(y) if self.copy_X_train else y
        self._drop_device_copies()
        self._params(self.kernel_)  # unsupported kernels fail here

        if self.optimizer is not None and self.kernel_.n_dims > 0:
            def obj_func(theta, eval_gradient=True):
                if eval_gradient:
                    lml, grad = self.log_marginal_likelihood(theta, eval_gradient=True, clone_kernel=False)
                    return -lml, -grad
                return -self.log_marginal_likelihood(theta, clone_kernel=False)

            optima = [self._constrained_optimization(obj_func, self.kernel_.theta, self.kernel_.bounds)]
            if self.n_restarts_optimizer > 0:
                if not np.isfinite(self.kernel_.bounds).all():
                    raise ValueError("Multiple optimizer restarts (n_restarts_optimizer>0) "
                                     "requires that all bounds are finite.")
                bounds = self.kernel_.bounds
                for _ in range(self.n_restarts_optimizer):
                    theta_initial = self._rng.uniform(bounds[:, 0], bounds[:, 1])
                    optima.append(self._constrained_optimization(obj_func, theta_initial, bounds))
            lml_values = [o[1] for o in optima]
            self.kernel_.theta = optima[int(np.argmin(lml_values))][0]
            self.kernel_._check_bounds_params()
            self.log_marginal_likelihood_value_ = -np.min(lml_values)
        else:
            self.log_marginal_likelihood_value_ = self.log_marginal_likelihood(self.kernel_.theta, clone_kernel=False)
        return self

    def _constrained_optimization(self, obj_func, initial_theta, bounds):
        """``optimizer='device-lbfgs'``: ``torch.optim.LBFGS`` on the device through the
        differentiable log-likelihood (:mod:`nngpr_b200.autograd`), at most 50 iterations;
        every other optimizer as scikit-learn runs it."""
        if self.optimizer == 'device-lbfgs':
            from .autograd import LogLikProblem, fit_lbfgs
            theta, lml, _ = fit_lbfgs(LogLikProblem.from_estimator(self), initial_theta, bounds)
            return theta, -lml
        return super()._constrained_optimization(obj_func, initial_theta, bounds)

    # ---- fit step -------------------------------------------------------------------------
    def _dtypes(self):
        """(search dtype, local-system dtype) of the ``allow_downcast_f32`` setting."""
        mode = self._downcast
        search = torch.float64 if mode == 'no' else torch.float32
        local = torch.float32 if mode == 'yes' else torch.float64
        return search, local

    def fit_neighbours(self, kernel=None, x_search=None, flags=None):
        """Neighbour lists of the fit step on the device, ``(n, min(num_nn, n-1))`` int32:
        point ``i``'s nearest among points ``[0, i)`` (``base_nngpr.py:530-535``)."""
        kernel = self.kernel_ if kernel is None else kernel
        p = self._params(kernel)
        if x_search is None:
            x_search = self._train_tensors(self._dtypes()[0])[0]
        n = x_search.shape[0]
        m = min(self._num_nn, max(n - 1, 0))
        ls = self._search_ls(p)
        if (self.reuse_neighbours and x_search.dtype == torch.float32 and 0 < m <= 32
                and (ls is None or np.ndim(ls) == 0 or np.size(ls) == 1)):
            return self._reused_neighbours(x_search, m, ls, flags)
        return ops.knn(x_search, x_search, m, ref_cut_index=0, length_scale=ls, flags=flags)

    def _reused_neighbours(self, xs, m, ls, flags):
        """Fit-step lists through the reuse cache (see ``reuse_neighbours``)."""
        n = xs.shape[0]
        cache = self.__dict__.get('_nn_cache')
        if cache is not None and cache['m'] == m and cache['n'] == n:
            if ls is None:  # input space: the lists do not depend on theta
                return cache['cand'][:, :m].contiguous()
            nbr, failed = ops.knn_reuse_rank(xs, cache['cand'], cache['thr'], ls, m)
            if int(failed.item()) == 0:
                return nbr
        # (re)build at this length scale: a wider search, the first m columns are its lists
        c = min(m + 16, 64, n - 1)
        cand = ops.knn(xs, xs, c, ref_cut_index=0, length_scale=ls, flags=flags)
        max_norm = float(torch.linalg.vector_norm(xs.double(), dim=1).max()) if n else 0.0
        thr = ops.knn_reuse_prepare(xs, cand, ls, max_norm)
        self.__dict__['_nn_cache'] = {'m': m, 'n': n, 'cand': cand, 'thr': thr}
        return cand[:, :m].contiguous()

    def log_marginal_likelihood(self, theta=None, eval_gradient=False, clone_kernel=True):
        """Log-likelihood of ``theta`` (and its gradient), ``base_nngpr.py:385-451``."""
        if theta is None:
            if eval_gradient:
                raise ValueError("Gradient can only be evaluated for theta!=None")
            return self.log_marginal_likelihood_value_
        if clone_kernel:
            kernel = self.kernel_.clone_with_theta(theta)
        else:
            kernel = self.kernel_
            kernel.theta = theta
        p = self._params(kernel)
        search_dt, local_dt = self._dtypes()
        x, y = self._train_tensors(local_dt)
        if search_dt == local_dt:
            xs = x
        elif self.keep_resident:
            xs = self._train_tensors(search_dt)[0]
        else:
            xs = x.to(search_dt)  # one upload per call; the search copy is cast on the device
        flags = ops.new_flags(x.device)
        nbr = self.fit_neighbours(kernel, xs, flags)
        out = ops.loglik(x, y, nbr, p, float(self.alpha), eval_gradient, self.pivot_tol, flags=flags)
        res = torch.cat([out, flags.to(torch.float64)]).cpu().numpy()  # one device -> host read
        ops.raise_on_flags(int(res[-1]), 'log_marginal_likelihood')
        if eval_gradient:
            return float(res[0]), res[1:-1].copy()
        return float(res[0])

    # ---- predict --------------------------------------------------------------------------
    def predict(self, X, return_std=False, return_cov=False, conditioning_method=None):
        """Predictive mean (and std or covariance), ``base_nngpr.py:763-1030``: conditioned on the
        training set (``'only-train'``, the default) or, query by query, on the training set and
        the earlier queries (``'full'``, ``'full-double-nn'``)."""
        conditioning_method = 'only-train' if conditioning_method is None else conditioning_method
        if conditioning_method not in {'only-train', 'full', 'full-double-nn'}:
            raise ValueError(f"unknown conditioning_method {conditioning_method!r}")
        if return_std:
            return_cov = False  # the reference returns the standard deviation when both are asked for
        if self.kernel is None or self.kernel.requires_vector_input:
            dtype, ensure_2d = "numeric", True
        else:
            dtype, ensure_2d = None, False
        X = validate_data(self, X, ensure_2d=ensure_2d, dtype=dtype, reset=False)
        _lib.lib()
        if not hasattr(self, "X_train_"):  # unfitted: the GP prior (base_nngpr.py:817-833)
            kernel = self.kernel if self.kernel is not None else self.get_default_kernel()
            p = self._params(kernel)
            mean = np.zeros(X.shape[0])
            if return_cov:
                if conditioning_method != 'only-train':
                    raise NotImplementedError(f"predict(return_cov=True, conditioning_method={conditioning_method!r}) "
                                              "needs a fitted model")
                return mean, np.diag(np.full(X.shape[0], p.rbf_level + p.const_value + p.noise_level))
            if return_std:
                return mean, np.full(X.shape[0], np.sqrt(p.rbf_level + p.const_value + p.noise_level))
            return mean
        kernel = self.kernel_
        p = self._params(kernel)
        dev = self._device
        search_dtype, local_dtype = self._dtypes()
        if conditioning_method != 'only-train':
            return self._predict_full(X, p, search_dtype, return_std, return_cov,
                                      conditioning_method == 'full-double-nn')
        xt, yt = self._train_tensors(local_dtype)
        xs_train = xt if search_dtype == local_dtype else self._train_tensors(search_dtype)[0]
        xq_host = np.ascontiguousarray(X, dtype=np.float64)
        xq = torch.from_numpy(xq_host).to(dev)
        xq_search = xq.to(search_dtype)
        xq_local = xq.to(local_dtype)
        nt = xt.shape[0]
        m = min(self._num_nn, nt)
        flags = ops.new_flags(dev)
        nbr = ops.knn(xs_train, xq_search, m, None, self._search_ls(p), flags=flags)
        mean, var = ops.predict(xt, yt, xq_local, nbr, p, float(self.alpha), self.pivot_tol, flags=flags)
        mean = mean.double().cpu().numpy()
        var = var.double().cpu().numpy()
        ops.raise_on_flags(int(flags.item()) & ~_lib.NNGP_FLAG_NOT_PD, 'predict')
        # undo the y normalisation and squeeze like format_mean / format_sigma (:843-858)
        y_std = np.asarray(self._y_train_std, dtype=np.float64).reshape(1, -1)
        y_mean = np.asarray(self._y_train_mean, dtype=np.float64).reshape(1, -1)
        mean = y_std * mean + y_mean
        if mean.shape[1] == 1:
            mean = mean[:, 0]
        if return_cov:  # queries conditioned on the training set only are independent
            return mean, self._format_cov(np.diag(np.maximum(var, 0.0)))
        if not return_std:
            return mean
        std = np.sqrt(var).reshape(-1, 1) * y_std
        if std.shape[1] == 1:
            std = std[:, 0]
        return mean, std

    def _full_lists(self, xt, xq, p, search_dtype, double_nn, flags):
        """Neighbour lists of the sequential algorithm, ``(nq, m)`` int32 indices into
        ``[x_train; x_query]`` (``base_nngpr.py:1370-1464``).  ``'full'``: the prefix search of the
        queries over the training set and the earlier queries (``ref_cut_index = n_train``).
        ``'full-double-nn'``: ``num_nn`` training neighbours plus ``num_nn`` earlier-query
        neighbours, each row packed as valid training entries, valid query entries, then ``-1``
        (``:1418-1449``).  At most 64 slots (the device recursions' limit)."""
        nt, nq = xt.shape[0], xq.shape[0]
        ls = self._search_ls(p)
        k = self._num_nn
        if not double_nn:
            m = min(k, nt + nq)
            if m > 64:
                raise NotImplementedError("conditioning_method='full' supports num_nn <= 64")
            x_full_s = torch.cat([xt, xq]).to(search_dtype)
            return ops.knn(x_full_s, x_full_s[nt:], m, ref_cut_index=nt, length_scale=ls, flags=flags)
        mt, mq = (min(k, nt) if nt > 0 else 0), max(0, min(k, nq - 1))
        if mt + mq > 64:
            raise NotImplementedError("conditioning_method='full-double-nn' supports num_nn <= 32")
        xq_s = xq.to(search_dtype)
        q = ops.knn(xq_s, xq_s, mq, ref_cut_index=0, length_scale=ls, flags=flags)
        q = torch.where(q >= 0, q + nt, q)
        if mt == 0:
            return q
        t = ops.knn(xt.to(search_dtype), xq_s, mt, None, length_scale=ls, flags=flags)
        both = torch.cat([t, q], dim=1)
        # stable sort on "missing": valid entries keep their order (training first), -1 last
        order = torch.sort((both < 0).to(torch.int8), dim=1, stable=True).indices
        return torch.gather(both, 1, order).contiguous()

    def _predict_full(self, X, p, search_dtype, return_std, return_cov=False, double_nn=False):
        """``conditioning_method='full'`` or ``'full-double-nn'`` (``base_nngpr.py:896-1030``):
        every query conditions on the training set and on the queries before it; FP64 local
        systems."""
        dev = self._device
        xt, yt = self._train_tensors(torch.float64)
        xq = torch.from_numpy(np.ascontiguousarray(X, dtype=np.float64)).to(dev)
        flags = ops.new_flags(dev)
        nbr = self._full_lists(xt, xq, p, search_dtype, double_nn, flags)
        if return_cov:
            mean, cov = ops.predict_cov_full(xt, yt, xq, nbr, p, float(self.alpha), flags=flags)
        else:
            mean, var = ops.predict_full(xt, yt, xq, nbr, p, float(self.alpha), return_std, flags=flags)
        mean = mean.cpu().numpy()
        ops.raise_on_flags(int(flags.item()) & ~_lib.NNGP_FLAG_NOT_PD, 'predict')
        y_std = np.asarray(self._y_train_std, dtype=np.float64).reshape(1, -1)
        y_mean = np.asarray(self._y_train_mean, dtype=np.float64).reshape(1, -1)
        mean = y_std * mean + y_mean
        if mean.shape[1] == 1:
            mean = mean[:, 0]
        if return_cov:
            return mean, self._format_cov(cov)
        if not return_std:
            return mean
        std = np.sqrt(var.cpu().numpy()).reshape(-1, 1) * y_std
        if std.shape[1] == 1:
            std = std[:, 0]
        return mean, std

    def _format_cov(self, cov):
        """Covariance in y units, ``(nq, nq)`` or ``(nq, nq, n_targets)`` (``base_nngpr.py:1017-1022``)."""
        ys = np.asarray(self._y_train_std, dtype=np.float64).reshape(1, 1, -1)
        c = (cov.cpu().numpy() if torch.is_tensor(cov) else np.asarray(cov))[:, :, None] * ys ** 2
        return c[:, :, 0] if c.shape[2] == 1 else c

    def sample_y(self, X, n_samples=1, random_state=0, conditioning_method=None):
        """Samples of the predictive marginals at ``X``, ``base_nngpr.py:616-689`` with
        ``conditioning_method='only-train'``: every query point is conditioned on the training
        set only, so its samples are independent draws ``mean + std * N(0, 1)`` (the reference's
        own fast path, ``:672-689``).  The normal draws come from a device generator seeded by
        ``random_state`` (an int, a ``RandomState`` or ``None``), so they differ from the
        reference's worker streams, not in distribution.  With ``'full'`` or ``'full-double-nn'``
        the samples follow the sequential algorithm (``:691-750``, :meth:`_sample_full`) and an
        int ``random_state`` reproduces the reference's.  Shape ``(n_samples_X, n_samples)`` or
        ``(n_samples_X, n_targets, n_samples)``."""
        conditioning_method = 'only-train' if conditioning_method is None else conditioning_method
        if conditioning_method not in {'only-train', 'full', 'full-double-nn'}:
            raise ValueError(f"unknown conditioning_method {conditioning_method!r}")
        if conditioning_method != 'only-train':
            return self._sample_full(X, n_samples, random_state, conditioning_method == 'full-double-nn')
        mean, std = self.predict(X, return_std=True)
        mu = np.asarray(mean, dtype=np.float64)
        sd = np.asarray(std, dtype=np.float64)
        single = mu.ndim == 1
        if single:
            mu, sd = mu[:, None], sd[:, None]
        rs = check_random_state(random_state)
        seed = int(rs.randint(0, 2 ** 31))
        dev = self._device
        gen = torch.Generator(device=dev)
        gen.manual_seed(seed)
        z = torch.randn((mu.shape[0], mu.shape[1], int(n_samples)), generator=gen, device=dev, dtype=torch.float64)
        out = torch.from_numpy(mu).to(dev)[..., None] + torch.from_numpy(sd).to(dev)[..., None] * z
        out = out.cpu().numpy()
        return out[:, 0, :] if single else out

    def _sample_full(self, X, n_samples, random_state, double_nn=False):
        """``sample_y`` with ``conditioning_method='full'`` or ``'full-double-nn'``
        (``base_nngpr.py:691-750``): each query's samples condition on the training y and on the
        samples of the queries before it.  The standard
        normals are drawn on the host exactly as the reference draws them (scikit-learn's
        ``check_random_state``, query by query, ``(n_targets, n_samples)`` each), so an int
        ``random_state`` reproduces the reference's samples; the recursion runs on the device."""
        if not hasattr(self, 'X_train_'):
            raise NotImplementedError("sample_y with conditioning on the queries needs a fitted model")
        if self.kernel is None or self.kernel.requires_vector_input:
            dtype, ensure_2d = "numeric", True
        else:
            dtype, ensure_2d = None, False
        X = validate_data(self, X, ensure_2d=ensure_2d, dtype=dtype, reset=False)
        p = self._params(self.kernel_)
        dev = self._device
        search_dtype, _ = self._dtypes()
        xt, yt = self._train_tensors(torch.float64)
        xq = torch.from_numpy(np.ascontiguousarray(X, dtype=np.float64)).to(dev)
        nq = xq.shape[0]
        ydim = yt.shape[1]
        z = check_random_state(random_state).standard_normal((nq, ydim, int(n_samples)))
        flags = ops.new_flags(dev)
        nbr = self._full_lists(xt, xq, p, search_dtype, double_nn, flags)
        out = ops.sample_full(xt, yt, xq, nbr, p, float(self.alpha), torch.from_numpy(z).to(dev), flags=flags)
        out = out.cpu().numpy()
        ops.raise_on_flags(int(flags.item()) & ~_lib.NNGP_FLAG_NOT_PD, 'sample_y')
        y_std = np.asarray(self._y_train_std, dtype=np.float64).reshape(1, -1, 1)
        y_mean = np.asarray(self._y_train_mean, dtype=np.float64).reshape(1, -1, 1)
        out = out * y_std + y_mean
        return out[:, 0, :] if ydim == 1 else out

    # ---- persistence ------------------------------------------------------------------------
    def __getstate__(self):
        """Pickle without the device and pinned copies of the training set: they are rebuilt
        from ``X_train_``/``y_train_`` on first use after loading."""
        state = super().__getstate__() if hasattr(super(), '__getstate__') else self.__dict__.copy()
        state = dict(state)
        state.pop('_device_cache', None)
        state.pop('_pinned_cache', None)
        state.pop('_nn_cache', None)
        return state
