"""The fit-step log-likelihood as a ``torch.autograd.Function`` and an L-BFGS fit driven by it.

``NngpLogLik.apply(theta, problem)`` returns the log marginal likelihood of ``problem``'s
training set at log-hyperparameters ``theta`` (a float64 tensor of the kernel's ``theta``
layout, on any device) as a 0-d tensor on ``theta``'s device.  The same fused kernel pass
computes the gradient (the adjoint identity, no ``dK`` tensor), so ``backward`` only scales the
saved gradient.  What the reference does in ``Nngpr.log_marginal_likelihood``
(``nngpr/base_nngpr.py:385-451``), one neighbour search and one local-systems pass per call.

A CUDA ``theta`` never leaves the device: ``nngp_theta_params`` turns it into the
hyperparameter values on the device, the search reads its length scale there and the
local-systems kernels read their values there, so an evaluation makes no host round trip
(``torch.cuda.set_sync_debug_mode('error')`` passes over forward and backward).  A host
``theta`` takes the by-value path.  Everything of size n stays on the device.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib, ops
from .kernel_params import RbfParams, params_from_theta


class LogLikProblem:
    """A training set on the device and the settings of its fit step.

    ``x_search`` is the search copy of X (float32 by default), ``x``/``y`` the local-system
    copies (float64, or float32 for FP32 systems with FP64 re-solves), ``template`` the kernel
    structure (:func:`nngpr_b200.kernel_params.extract`).  ``nn_type='kernel-space'`` divides
    the search by the length scale as the reference does (``base_nngpr.py:1664-1665``).
    """

    def __init__(self, x_search: torch.Tensor, x: torch.Tensor, y: torch.Tensor, template: RbfParams,
                 num_nn: int, alpha: float, nn_type: str = 'kernel-space', pivot_tol: float | None = None):
        self.x_search, self.x = x_search, x
        self.y = y if y.dim() == 2 else y.reshape(-1, 1)
        self.template = template
        self.num_nn = int(num_nn)
        self.alpha = float(alpha)
        self.nn_type = nn_type
        self.pivot_tol = ops.DEFAULT_PIVOT_TOL if pivot_tol is None else float(pivot_tol)
        self.flags = ops.new_flags(x.device)
        self.evaluations = 0

    @classmethod
    def from_estimator(cls, gpr) -> 'LogLikProblem':
        """The problem of a fitted :class:`nngpr_b200.B200Nngpr` (its precision settings)."""
        from .kernel_params import extract
        search_dt, local_dt = gpr._dtypes()
        x, y = gpr._train_tensors(local_dt)
        xs = x if search_dt == local_dt else x.to(search_dt)
        return cls(xs, x, y, extract(gpr.kernel_), gpr._num_nn, gpr.alpha, gpr._nn_type, gpr.pivot_tol)

    def params(self, theta) -> RbfParams:
        return params_from_theta(self.template, theta)

    def evaluate(self, theta) -> torch.Tensor:
        """``[lml, d lml / d theta...]`` (float64, on the device) at ``theta`` (host array)."""
        p = self.params(theta)
        n = self.x.shape[0]
        m = min(self.num_nn, max(n - 1, 0))
        ls = p.length_scale if (self.nn_type == 'kernel-space' and p.length_scale is not None) else None
        self.flags.zero_()
        nbr = ops.knn(self.x_search, self.x_search, m, 0, ls, flags=self.flags)
        out = ops.loglik(self.x, self.y, nbr, p, self.alpha, True, pivot_tol=self.pivot_tol, flags=self.flags)
        self.evaluations += 1
        return out

    def evaluate_device(self, theta: torch.Tensor) -> torch.Tensor:
        """``[lml, d lml / d theta...]`` at a float64 CUDA ``theta`` without copying it to the
        host: the values come from ``ops.theta_params`` on the device."""
        p = self.template
        n, d = self.x.shape
        m = min(self.num_nn, max(n - 1, 0))
        params = ops.theta_params(p, theta.to(self.x.device, torch.float64), self.alpha, d, self.pivot_tol)
        ls = None
        if self.nn_type == 'kernel-space' and p.length_scale is not None:
            n_ls = d if p.n_ls == d else 1
            ls = params[4 + d:4 + d + n_ls]
        self.flags.zero_()
        nbr = ops.knn(self.x_search, self.x_search, m, 0, ls, flags=self.flags)
        out = ops.loglik(self.x, self.y, nbr, p, self.alpha, True, pivot_tol=self.pivot_tol, flags=self.flags,
                         params_dev=params)
        self.evaluations += 1
        return out

    def check(self) -> None:
        """Raise on a status raised by the kernels of the last evaluation (reads one int)."""
        ops.raise_on_flags(int(self.flags.item()) & ~_lib.NNGP_FLAG_FP64_FALLBACK, 'log-likelihood')


class NngpLogLik(torch.autograd.Function):
    """``lml = NngpLogLik.apply(theta, problem)``; ``lml.backward()`` gives ``theta.grad``."""

    @staticmethod
    def forward(ctx, theta: torch.Tensor, problem: LogLikProblem):
        if theta.is_cuda:
            out = problem.evaluate_device(theta.detach())
        else:
            out = problem.evaluate(theta.detach().to(torch.float64).numpy())
        ctx.save_for_backward(out[1:].to(theta.device, theta.dtype))
        return out[0].to(theta.device, theta.dtype)

    @staticmethod
    def backward(ctx, grad_out):
        (grad,) = ctx.saved_tensors
        return grad_out * grad, None


def log_marginal_likelihood(theta: torch.Tensor, problem: LogLikProblem) -> torch.Tensor:
    """Differentiable log marginal likelihood (see :class:`NngpLogLik`)."""
    return NngpLogLik.apply(theta, problem)


def fit_lbfgs(problem: LogLikProblem, theta0, bounds=None, max_iter: int = 50, history_size: int = 10,
              device=None):
    """Maximise the log-likelihood over theta with ``torch.optim.LBFGS`` (strong-Wolfe line
    search) on ``device``; ``bounds (n_theta, 2)`` in log space are enforced by evaluating at
    the clamped point.  Returns ``(theta_opt (numpy), lml_opt, evaluations)``."""
    device = problem.x.device if device is None else device
    theta = torch.tensor(np.asarray(theta0, dtype=np.float64), device=device, requires_grad=True)
    lo = hi = None
    if bounds is not None:
        b = torch.as_tensor(np.asarray(bounds, dtype=np.float64), device=device)
        lo, hi = b[:, 0], b[:, 1]
    opt = torch.optim.LBFGS([theta], lr=1.0, max_iter=max_iter, history_size=history_size,
                            line_search_fn='strong_wolfe', tolerance_grad=1e-7, tolerance_change=1e-12)
    start = problem.evaluations

    def closure():
        opt.zero_grad()
        th = theta if lo is None else torch.maximum(torch.minimum(theta, hi), lo)
        loss = -log_marginal_likelihood(th, problem)
        loss.backward()
        return loss

    opt.step(closure)
    problem.check()
    with torch.no_grad():
        th = theta if lo is None else torch.maximum(torch.minimum(theta, hi), lo)
    th_np = th.detach().cpu().numpy()
    lml = float(problem.evaluate(th_np)[0].item())
    return th_np, lml, problem.evaluations - start
