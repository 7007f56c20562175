"""Neighbour-list reuse on the GPU: the C-ABI pair against the oracle's restatement (bit for
bit), reused lists against a fresh search, and the estimator with and without reuse."""
import numpy as np
import pytest
import torch
from sklearn.gaussian_process import kernels as skk

from nngpr_b200 import B200Nngpr, ops
from oracle import nngp_oracle as O

pytestmark = pytest.mark.gpu


def _data(n=3000, d=3, offset=0.0, seed=0):
    rng = np.random.default_rng(seed)
    return (rng.uniform(-1, 1, (n, d)) * np.linspace(1.0, 0.4, d) + offset).astype(np.float32)


@pytest.mark.parametrize('d,offset', [(3, 0.0), (3, 2.0), (8, 0.0), (16, 0.0)])
def test_prepare_and_rank_match_oracle(d, offset):
    x = _data(2000, d, offset, seed=d)
    xt = torch.from_numpy(x).cuda()
    ls0, m, c = 0.3, 16, 28
    cand = ops.knn(xt, xt, c, 0, ls0)
    max_norm = float(np.sqrt((x.astype(np.float64) ** 2).sum(1)).max())
    thr = ops.knn_reuse_prepare(xt, cand, ls0, max_norm).cpu().numpy()
    want_thr = O.reuse_thresholds(x, cand.cpu().numpy(), ls0, max_norm)
    fin = np.isfinite(want_thr)
    assert np.array_equal(np.isfinite(thr), fin)
    np.testing.assert_allclose(thr[fin], want_thr[fin], rtol=1e-12, atol=1e-15)
    for ls in (0.15, 0.3, 0.55, 2.0):
        nbr, failed = ops.knn_reuse_rank(xt, cand, torch.from_numpy(want_thr).cuda(), ls, m)
        want, want_failed = O.reuse_rank(x, cand.cpu().numpy(), want_thr, ls, m)
        assert np.array_equal(nbr.cpu().numpy(), want)
        assert int(failed.item()) == want_failed
        if want_failed == 0:
            assert np.array_equal(nbr.cpu().numpy(), ops.knn(xt, xt, m, 0, ls).cpu().numpy())


def test_estimator_with_reuse_gives_identical_results():
    rng = np.random.default_rng(5)
    x = _data(4000, 3, 0.0, seed=5).astype(np.float64)
    y = np.sin(3 * x).sum(1) + rng.normal(0, 0.05, len(x))
    kw = dict(kernel=skk.ConstantKernel(1.0) * skk.RBF(0.2) + skk.WhiteKernel(1e-3), num_nn=32, optimizer=None)
    a = B200Nngpr(reuse_neighbours=True, **kw).fit(x, y)
    b = B200Nngpr(**kw).fit(x, y)
    for ls in (0.2, 0.17, 0.26, 0.4, 0.11):
        theta = np.log([1.3, ls, 2e-3])
        la, ga = a.log_marginal_likelihood(theta, eval_gradient=True)
        lb, gb = b.log_marginal_likelihood(theta, eval_gradient=True)
        assert la == lb and np.array_equal(ga, gb)
    assert '_nn_cache' in a.__dict__
    # an L-BFGS fit takes the same path with and without reuse
    kw['optimizer'] = 'fmin_l_bfgs_b'
    fa = B200Nngpr(reuse_neighbours=True, **kw).fit(x, y)
    fb = B200Nngpr(**kw).fit(x, y)
    assert np.array_equal(fa.kernel_.theta, fb.kernel_.theta)
    assert fa.log_marginal_likelihood_value_ == fb.log_marginal_likelihood_value_


def test_estimator_falls_back_when_the_bound_refuses():
    """Points far from the origin: the rounding bound exceeds the margins, every reused list is
    refused and the estimator searches again (same results)."""
    rng = np.random.default_rng(6)
    x = _data(1500, 2, 0.0, seed=6).astype(np.float64) + 3000.0
    y = np.cos(x[:, 0]) + rng.normal(0, 0.05, len(x))
    kw = dict(kernel=skk.ConstantKernel(1.0) * skk.RBF(0.05) + skk.WhiteKernel(1e-2), num_nn=8, optimizer=None)
    a = B200Nngpr(reuse_neighbours=True, **kw).fit(x, y)
    b = B200Nngpr(**kw).fit(x, y)
    for ls in (0.05, 0.07):
        theta = np.log([1.0, ls, 1e-2])
        assert a.log_marginal_likelihood(theta) == b.log_marginal_likelihood(theta)
