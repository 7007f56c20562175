"""The differentiable log-likelihood (torch.autograd.Function): its gradient against the
reference's, against central finite differences (h = 1e-3) on an ARD d = 8 problem, and the
device L-BFGS fit against scikit-learn's L-BFGS-B driving the same likelihood."""
import numpy as np
import pytest
import torch
from sklearn.gaussian_process import kernels as skk

from nngpr_b200 import B200Nngpr
from nngpr_b200.autograd import LogLikProblem, NngpLogLik, fit_lbfgs
from nngpr_b200.kernel_params import extract

from _common import KERNELS, load, rel

pytestmark = pytest.mark.gpu


def _problem(name, mode='no'):
    g = load(name)
    gpr = B200Nngpr(kernel=KERNELS[name](), num_nn=int(g['num_nn']), alpha=float(g['alpha']),
                    normalize_y=bool(g['normalize_y']), optimizer=None, allow_downcast_f32=mode).fit(g['x'], g['y'])
    return g, gpr, LogLikProblem.from_estimator(gpr)


@pytest.mark.parametrize('name', ['cpu_n2000_d3_m16', 'ard_n400_d5_m12_y2', 'const_n300_d2_m10'])
def test_backward_gives_reference_gradient(name):
    g, gpr, prob = _problem(name)
    theta = torch.tensor(g['theta'], dtype=torch.float64, device='cuda', requires_grad=True)
    lml = NngpLogLik.apply(theta, prob)
    lml.backward()
    assert abs(float(lml.detach()) / float(g['lml']) - 1) < 1e-10
    assert rel(theta.grad.cpu().numpy(), g['grad']) < 1e-9
    # a scaled upstream gradient scales the result
    theta.grad = None
    (3.0 * NngpLogLik.apply(theta, prob)).backward()
    assert rel(theta.grad.cpu().numpy(), 3.0 * g['grad']) < 1e-9


@pytest.mark.parametrize('mode', ['no', 'yes'])
@pytest.mark.parametrize('name', ['cpu_n2000_d3_m16', 'ard_n400_d5_m12_y2', 'const_n300_d2_m10'])
def test_device_theta_equals_host_theta(name, mode):
    """A CUDA theta stays on the device (nngp_theta_params, the search's device length scale,
    the kernels' device parameter block); the result equals the by-value path up to the last
    bits of exp (FP64 systems 1e-12, FP32 systems 1e-6), and both search paths give the same
    lists."""
    from nngpr_b200 import ops
    g, gpr, prob = _problem(name, mode)
    th = np.asarray(g['theta'], dtype=np.float64)
    host = prob.evaluate(th).cpu().numpy()
    dev = prob.evaluate_device(torch.tensor(th, device='cuda')).cpu().numpy()
    tol = 1e-12 if mode == 'no' else 1e-6
    assert abs(dev[0] / host[0] - 1) < tol
    assert rel(dev[1:], host[1:]) < 10 * tol
    p = prob.params(th)
    if p.length_scale is not None:
        d = prob.x.shape[1]
        params = ops.theta_params(prob.template, torch.tensor(th, device='cuda'), prob.alpha, d, prob.pivot_tol)
        n_ls = d if p.n_ls == d else 1
        m = min(prob.num_nn, prob.x.shape[0] - 1)
        a = ops.knn(prob.x_search, prob.x_search, m, 0, p.length_scale).cpu().numpy()
        b = ops.knn(prob.x_search, prob.x_search, m, 0, params[4 + d:4 + d + n_ls]).cpu().numpy()
        np.testing.assert_array_equal(a, b)
        np.testing.assert_allclose(params[4 + d:4 + 2 * d].cpu().numpy(), p.ls_vector(d), rtol=1e-15)


def test_device_theta_evaluation_makes_no_host_sync():
    """Forward and backward at a CUDA theta make no synchronising CUDA call (torch's sync debug
    mode raises on one): theta is never read on the host."""
    g, gpr, prob = _problem('ard_n400_d5_m12_y2', 'yes')
    theta = torch.tensor(g['theta'], dtype=torch.float64, device='cuda', requires_grad=True)
    torch.cuda.synchronize()
    torch.cuda.set_sync_debug_mode('error')
    try:
        lml = NngpLogLik.apply(theta, prob)
        lml.backward()
    finally:
        torch.cuda.set_sync_debug_mode('default')
    # FP32 systems against the FP64 golden values: a sanity bound, the point here is the sync
    assert abs(float(lml.detach()) / float(g['lml']) - 1) < 1e-4
    assert rel(theta.grad.cpu().numpy(), g['grad']) < 1e-3


def _rff_problem(n=20000, d=8, seed=4):
    """The differentiation workload's shape on a 20,000-point subset: x ~ U[0, 1]^8, y a
    512-feature random Fourier draw with log-uniform ARD length scales in [0.1, 1]."""
    rng = np.random.default_rng(seed)
    x = rng.uniform(0, 1, (n, d))
    ls = np.exp(rng.uniform(np.log(0.1), np.log(1.0), d))
    omega = rng.normal(size=(512, d)) / ls
    y = np.cos(x @ omega.T + rng.uniform(0, 2 * np.pi, 512)) @ (rng.normal(size=512) * np.sqrt(2 / 512))
    y += rng.normal(0, 0.02, n)
    kernel = skk.ConstantKernel(1.0) * skk.RBF(np.full(d, 0.4)) + skk.WhiteKernel(1e-3)
    return x, y, kernel


def test_gradient_matches_central_differences_ard_d8():
    """The adjoint gradient is the derivative of the log-likelihood with the neighbour lists held
    fixed (as the reference's gradient is); central differences with h = 1e-3 on those lists."""
    from nngpr_b200 import ops
    from nngpr_b200.kernel_params import params_from_theta
    x, y, kernel = _rff_problem()
    dev = torch.device('cuda')
    x64 = torch.from_numpy(x).to(dev)
    y64 = torch.from_numpy(y).to(dev)[:, None]
    prob = LogLikProblem(x64.to(torch.float32), x64, y64, extract(kernel), 32, 1e-10)
    theta0 = kernel.theta.copy()
    grad = prob.evaluate(theta0)[1:].cpu().numpy()
    prob.check()
    p0 = prob.params(theta0)
    nbr = ops.knn(prob.x_search, prob.x_search, 32, 0, p0.length_scale)

    def f(th):
        return float(ops.loglik(x64, y64, nbr, params_from_theta(prob.template, th), 1e-10, False)[0])

    h = 1e-3
    fd = np.empty_like(grad)
    for t in range(theta0.size):
        tp, tm = theta0.copy(), theta0.copy()
        tp[t] += h
        tm[t] -= h
        fd[t] = (f(tp) - f(tm)) / (2 * h)
    assert np.max(np.abs(fd - grad)) / np.max(np.abs(grad)) < 1e-4


def test_device_lbfgs_matches_scipy_lbfgsb():
    g = load('cpu_n2000_d3_m16')
    kw = dict(kernel=KERNELS['cpu_n2000_d3_m16'](), num_nn=16, allow_downcast_f32='no')
    a = B200Nngpr(optimizer='device-lbfgs', **kw).fit(g['x'], g['y'])
    b = B200Nngpr(**kw).fit(g['x'], g['y'])
    assert abs(a.log_marginal_likelihood_value_ - b.log_marginal_likelihood_value_) < 1e-6 * abs(
        b.log_marginal_likelihood_value_)
    assert np.max(np.abs(a.kernel_.theta - b.kernel_.theta)) < 1e-3


def test_fit_lbfgs_respects_bounds():
    g, gpr, prob = _problem('cpu_n2000_d3_m16')
    bounds = np.array([[-0.5, 0.5], [-1.5, -1.0], [-4.0, -3.0]])
    theta, lml, evals = fit_lbfgs(prob, np.array([0.0, -1.2, -3.5]), bounds, max_iter=20)
    assert np.all(theta >= bounds[:, 0] - 1e-12) and np.all(theta <= bounds[:, 1] + 1e-12)
    assert 1 <= evals <= 60
    assert np.isfinite(lml)


def test_fp32_gradient_on_the_differentiation_subset():
    """The FP32 path (FP32 search, FP32 local systems with the FP64 re-solve of small pivots) on
    20,000 points of the d = 8 ARD workload: lml within 1e-5 of |lml| and the gradient w.r.t. the
    10 log hyperparameters within 1e-5 (max-norm relative) of the FP64 oracle's (the reference's
    formulas, base_nngpr.py:586-614) on the same lists, and within 1e-4 of central differences
    (h = 1e-3) of the FP64 log-likelihood on those lists."""
    from nngpr_b200 import ops
    from nngpr_b200.kernel_params import params_from_theta
    from oracle import nngp_oracle as O

    from _common import oracle_params
    x, y, kernel = _rff_problem()
    p = extract(kernel)
    dev = torch.device('cuda')
    x64 = torch.from_numpy(x).to(dev)
    y64 = torch.from_numpy(y).to(dev)[:, None]
    x32, y32 = x64.to(torch.float32), y64.to(torch.float32)
    nbr = ops.knn(x32, x32, 32, 0, p.length_scale)
    flags = ops.new_flags(dev)
    got = ops.loglik(x32, y32, nbr, p, 1e-10, True, flags=flags).cpu().numpy()
    assert int(flags.item()) & ~8 == 0  # only the informational FP64-re-solve bit may be set
    want_l, want_g = O.log_marginal_likelihood(x, y[:, None], nbr.cpu().numpy(), oracle_params(p), 1e-10, True)
    assert abs(got[0] / want_l - 1) < 1e-5, (got[0], want_l)
    assert rel(got[1:], want_g) < 1e-5, (got[1:], want_g)

    theta0 = kernel.theta.copy()
    prob_template = extract(kernel)

    def f(th):
        return float(ops.loglik(x64, y64, nbr, params_from_theta(prob_template, th), 1e-10, False)[0])

    h = 1e-3
    fd = np.empty(theta0.size)
    for t in range(theta0.size):
        tp, tm = theta0.copy(), theta0.copy()
        tp[t] += h
        tm[t] -= h
        fd[t] = (f(tp) - f(tm)) / (2 * h)
    assert np.max(np.abs(fd - got[1:])) / np.max(np.abs(fd)) < 1e-4
