"""The binding a maintainer of the reference adds to run the reference's own estimator on this
library.

``b200_backed(base)`` takes one of the reference's estimator classes (a subclass of
``nngpr.base_nngpr.Nngpr``: ``NumpyNngpr``, ``TorchNngpr``, ...) and returns a subclass whose two
hot calls run on the B200 through the C ABI:

* ``log_marginal_likelihood(theta, eval_gradient)`` (``base_nngpr.py:385-451``): the fit-step
  neighbour search (``nngp_knn_f32`` / ``_f64``) and the fused local systems with the adjoint
  gradient (``nngp_loglik_f64`` / ``_f32``), in the precision ``allow_downcast_f32`` asks for
  (``'no'``: FP64 search and systems; ``'only-nn'``, the default: FP32 search, FP64 systems;
  ``'yes'``: FP32 search and systems with the FP64 re-solve of small pivots);
* ``predict(X, return_std)`` with ``conditioning_method='only-train'`` and no ``return_cov``
  (``base_nngpr.py:861-894``, ``:1032-1135``): the search of the queries against the training set
  and ``nngp_predict_f64`` / ``_f32``.

Everything else -- parameter validation, ``fit`` with scikit-learn's optimizer loop, ``normalize_y``,
the prior, ``return_cov``, ``'full'`` / ``'full-double-nn'`` conditioning, ``sample_y`` -- stays
the reference's own code.  Kernels outside the accelerated family (``White + Constant +
Constant * RBF`` or ``* Matern(nu = 1/2, 3/2, 5/2)``) raise ``NotImplementedError`` as the
reference's CUDA accelerator does (``cuda_kernel_accelerators.py:114-115``).  The reference's own
accelerator helpers (``RbfAccelerator.get_kernel_params`` / ``get_kernel_theta_mapping``,
``cuda_kernel_accelerators.py:520-649``) need cupy at import time, so the kernel parameters and
the theta map come from :func:`nngpr_b200.kernel_params.extract`, which applies the same rules.
"""

from __future__ import annotations

import numpy as np
import torch

from . import ops
from .kernel_params import extract


def b200_backed(base):
    """Subclass of the reference estimator class ``base`` with the B200 fit step and predict."""

    class B200Backed(base):
        _b200_device = 'cuda'

        def _b200_dtypes(self):
            mode = getattr(self, 'allow_downcast_f32', 'only-nn') or 'only-nn'
            search = torch.float64 if mode == 'no' else torch.float32
            local = torch.float32 if mode == 'yes' else torch.float64
            return search, local

        def _b200_search_ls(self, p):
            if getattr(self, 'nn_type', 'kernel-space') == 'kernel-space' and p.length_scale is not None:
                return p.length_scale
            return None

        def log_marginal_likelihood(self, theta=None, eval_gradient=False, clone_kernel=True):
            if theta is None:
                if eval_gradient:
                    raise ValueError("Gradient can only be evaluated for theta!=None")
                return self.log_marginal_likelihood_value_
            if clone_kernel:
                kernel = self.kernel_.clone_with_theta(theta)
            else:
                kernel = self.kernel_
                kernel.theta = theta
            p = extract(kernel)
            search_dt, local_dt = self._b200_dtypes()
            y = np.asarray(self.y_train_, dtype=np.float64)
            y = y[:, None] if y.ndim == 1 else y
            x = torch.from_numpy(np.ascontiguousarray(self.X_train_, dtype=np.float64)).to(self._b200_device)
            xl = x.to(local_dt).contiguous()
            yl = torch.from_numpy(np.ascontiguousarray(y)).to(self._b200_device, local_dt)
            xs = x.to(search_dt).contiguous()
            n = x.shape[0]
            m = min(self.num_nn, max(n - 1, 0))
            flags = ops.new_flags(x.device)
            nbr = ops.knn(xs, xs, m, ref_cut_index=0, length_scale=self._b200_search_ls(p), flags=flags)
            out = ops.loglik(xl, yl, nbr, p, float(self.alpha), eval_gradient, flags=flags)
            res = torch.cat([out, flags.to(torch.float64)]).cpu().numpy()
            ops.raise_on_flags(int(res[-1]), 'log_marginal_likelihood')
            if eval_gradient:
                return float(res[0]), res[1:-1].copy()
            return float(res[0])

        def predict(self, X, return_std=False, return_cov=False, conditioning_method=None):
            method = 'only-train' if conditioning_method is None else conditioning_method
            if return_cov or method != 'only-train' or not hasattr(self, 'X_train_'):
                return super().predict(X, return_std=return_std, return_cov=return_cov,
                                       conditioning_method=conditioning_method)
            xq_h = np.ascontiguousarray(np.asarray(X, dtype=np.float64))
            if xq_h.ndim != 2 or xq_h.shape[1] != self.X_train_.shape[1]:
                return super().predict(X, return_std=return_std, return_cov=return_cov,
                                       conditioning_method=conditioning_method)
            p = extract(self.kernel_)
            search_dt, local_dt = self._b200_dtypes()
            y = np.asarray(self.y_train_, dtype=np.float64)
            y = y[:, None] if y.ndim == 1 else y
            dev = self._b200_device
            xt = torch.from_numpy(np.ascontiguousarray(self.X_train_, dtype=np.float64)).to(dev)
            xq = torch.from_numpy(xq_h).to(dev)
            yt = torch.from_numpy(np.ascontiguousarray(y)).to(dev, local_dt)
            m = min(self.num_nn, xt.shape[0])
            flags = ops.new_flags(xt.device)
            nbr = ops.knn(xt.to(search_dt).contiguous(), xq.to(search_dt).contiguous(), m, None,
                          self._b200_search_ls(p), flags=flags)
            mean, var = ops.predict(xt.to(local_dt).contiguous(), yt, xq.to(local_dt).contiguous(), nbr, p,
                                    float(self.alpha), flags=flags)
            ops.raise_on_flags(int(flags.item()), 'predict')
            mean = mean.double().cpu().numpy()
            std = np.sqrt(np.maximum(var.double().cpu().numpy(), 0.0))
            if hasattr(self, '_y_train_std'):  # undo normalize_y (base_nngpr.py:843-858)
                ys = np.asarray(self._y_train_std, dtype=np.float64).reshape(1, -1)
                mean = ys * mean + np.asarray(self._y_train_mean, dtype=np.float64).reshape(1, -1)
                std = std.reshape(-1, 1) * ys
            else:
                std = std.reshape(-1, 1)
            if mean.shape[1] == 1:
                mean = mean[:, 0]
            if std.shape[1] == 1:
                std = std[:, 0]
            return (mean, std) if return_std else mean

    B200Backed.__name__ = 'B200Backed' + base.__name__
    B200Backed.__qualname__ = B200Backed.__name__
    return B200Backed
