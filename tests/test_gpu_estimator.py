"""B200Nngpr end to end (the scikit-learn API a user calls) vs the reference's golden values
and the reference's own known-answer tests (nngpr/test/nngpr_base_tester.py)."""
import numpy as np
import pytest
from sklearn import gaussian_process as skgp
from sklearn.gaussian_process import kernels as skk

from nngpr_b200 import B200Nngpr

from _common import CASES, KERNELS, lml_scale, load, rel

pytestmark = pytest.mark.gpu


def make(name, g, **kw):
    kw.setdefault('allow_downcast_f32', 'no')
    return B200Nngpr(kernel=KERNELS[name](), num_nn=int(g['num_nn']), alpha=float(g['alpha']),
                     normalize_y=bool(g['normalize_y']), optimizer=None, **kw)


@pytest.mark.parametrize('name', CASES)
@pytest.mark.parametrize('mode,tl,tg', [('no', 1e-10, 1e-9), ('only-nn', 1e-10, 1e-9), ('yes', 1e-5, 1e-5)])
def test_lml_and_grad_match_reference(name, mode, tl, tg):
    g = load(name)
    gpr = make(name, g, allow_downcast_f32=mode).fit(g['x'], g['y'])
    lml, grad = gpr.log_marginal_likelihood(g['theta'], eval_gradient=True)
    # FP32 systems ('yes'): error relative to the summed magnitude of the per-point terms
    scale = abs(float(g['lml'])) if mode != 'yes' else lml_scale(name)
    assert abs(lml - g['lml']) < tl * scale
    assert rel(grad, g['grad']) < tg
    assert abs(gpr.log_marginal_likelihood(g['theta']) - g['lml']) < tl * scale


@pytest.mark.parametrize('name', CASES)
@pytest.mark.parametrize('mode', ['no', 'only-nn', 'yes'])
def test_predict_matches_reference(name, mode):
    g = load(name)
    gpr = make(name, g, allow_downcast_f32=mode).fit(g['x'], g['y'])
    mean, std = gpr.predict(g['xq'], return_std=True)
    assert mean.shape == g['pred_mean'].shape and std.shape == g['pred_std'].shape
    if mode == 'yes':
        assert rel(mean, g['pred_mean']) < 1e-5 and rel(std, g['pred_std']) < 1e-5
    else:
        assert np.max(np.abs(mean - g['pred_mean'])) < 1e-10
        assert np.max(np.abs(std - g['pred_std'])) < 1e-10
    assert np.array_equal(gpr.predict(g['xq']), mean)


def _fixture():
    r = np.random.RandomState(234058)
    x = r.rand(150, 4)
    xe = r.rand(50, 4)
    beta = r.rand(4, 3)
    beta[:, -1] += 1
    y = x @ beta + r.rand(150, 3)
    y[:, 0] *= 10
    return x, xe, y


@pytest.mark.parametrize('y_dim', [1, 3])
def test_same_fit_results_as_exact_gp(y_dim):
    """test_same_fit_results (nngpr_base_tester.py:194-205): num_nn = n gives sklearn's fit."""
    x, _, y = _fixture()
    yy = y[:, :y_dim] if y_dim > 1 else y[:, 0]
    kern = lambda: skk.ConstantKernel(1) * skk.RBF(length_scale=1) + skk.WhiteKernel(1)
    ref = skgp.GaussianProcessRegressor(kernel=kern(), normalize_y=True).fit(x, yy)
    gpr = B200Nngpr(kernel=kern(), normalize_y=True, num_nn=150, allow_downcast_f32='no').fit(x, yy)
    assert np.max(np.abs(ref.kernel_.theta / gpr.kernel_.theta - 1)) < 1e-6
    assert abs(gpr.log_marginal_likelihood_value_ / ref.log_marginal_likelihood_value_ - 1) < 1e-9


def test_prior_predict():
    x, _, _ = _fixture()
    gpr = B200Nngpr(kernel=skk.ConstantKernel(2.0) * skk.RBF(1.0) + skk.WhiteKernel(0.5))
    mean, std = gpr.predict(x, return_std=True)
    assert np.all(mean == 0) and np.allclose(std, np.sqrt(2.5))


def test_out_of_scope_calls_raise():
    x, xe, y = _fixture()
    with pytest.raises(NotImplementedError):
        B200Nngpr(kernel=skk.RBF(1.0), num_nn=40, optimizer=None).fit(x, y[:, 0]).predict(
            xe, conditioning_method='full-double-nn')  # 80 slots: more than the recursions' 64
    with pytest.raises(NotImplementedError, match='Cannot accelerate'):
        B200Nngpr(kernel=skk.Matern(1.0, nu=2.0), optimizer=None).fit(x, y[:, 0])


def test_fit_with_optimizer_default_settings():
    """Default settings (num_nn=32, FP32 search, FP64 local systems) converge like the FP64 run."""
    g = load('cpu_n2000_d3_m16')
    kw = dict(kernel=KERNELS['cpu_n2000_d3_m16'](), num_nn=16)
    a = B200Nngpr(**kw).fit(g['x'], g['y'])
    b = B200Nngpr(allow_downcast_f32='no', **kw).fit(g['x'], g['y'])
    assert np.max(np.abs(a.kernel_.theta - b.kernel_.theta)) < 1e-6


def test_sample_y_only_train_shapes_seed_and_moments():
    """sample_y (base_nngpr.py:616-689, only-train): independent draws mean + std * N(0, 1)."""
    g = load('ard_n400_d5_m12_y2')
    gpr = make('ard_n400_d5_m12_y2', g).fit(g['x'], g['y'])
    xq = g['xq'][:40]
    mean, std = gpr.predict(xq, return_std=True)
    s = gpr.sample_y(xq, n_samples=6000, random_state=3)
    assert s.shape == (40, 2, 6000)
    np.testing.assert_array_equal(s, gpr.sample_y(xq, n_samples=6000, random_state=3))
    assert not np.array_equal(s[..., :10], gpr.sample_y(xq, n_samples=10, random_state=4))
    se = std / np.sqrt(6000)
    assert np.all(np.abs(s.mean(-1) - mean) < 6 * se)
    assert np.all(np.abs(s.std(-1) / std - 1) < 0.06)
    g1 = load('cpu_n2000_d3_m16')
    gpr1 = make('cpu_n2000_d3_m16', g1).fit(g1['x'], g1['y'])
    assert gpr1.sample_y(g1['xq'][:7], n_samples=3).shape == (7, 3)
    assert gpr1.sample_y(g1['xq'][:7], n_samples=3, conditioning_method='full-double-nn').shape == (7, 3)


def test_pickle_round_trip():
    import pickle
    g = load('cpu_n2000_d3_m16')
    gpr = make('cpu_n2000_d3_m16', g).fit(g['x'], g['y'])
    mean, std = gpr.predict(g['xq'], return_std=True)
    blob = pickle.dumps(gpr)
    assert len(blob) < 2 * (g['x'].nbytes + g['y'].nbytes) + 200_000  # no device or pinned copies inside
    back = pickle.loads(blob)
    m2, s2 = back.predict(g['xq'], return_std=True)
    np.testing.assert_array_equal(mean, m2)
    np.testing.assert_array_equal(std, s2)
    assert back.log_marginal_likelihood(back.kernel_.theta) == gpr.log_marginal_likelihood(gpr.kernel_.theta)


@pytest.mark.parametrize('mode', ['only-nn', 'yes', 'no'])
def test_keep_resident_false_uploads_each_call_with_identical_results(mode):
    """keep_resident=False uploads X and y on every call (the reference's behaviour): the
    results equal the resident path's bit for bit, call after call."""
    g = load('cpu_n2000_d3_m16')
    kw = dict(kernel=KERNELS['cpu_n2000_d3_m16'](), num_nn=16, optimizer=None, allow_downcast_f32=mode)
    a = B200Nngpr(**kw).fit(g['x'], g['y'])
    b = B200Nngpr(keep_resident=False, **kw).fit(g['x'], g['y'])
    for theta in (g['theta'], g['theta'] + 0.1, g['theta']):
        la, ga = a.log_marginal_likelihood(theta, eval_gradient=True)
        lb, gb = b.log_marginal_likelihood(theta, eval_gradient=True)
        assert la == lb and np.array_equal(ga, gb)
