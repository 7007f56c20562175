"""The CPU oracle pinned against the reference's golden vectors (CPU only)."""
import numpy as np
import pytest

from nngpr_b200 import kernel_params as KP
from oracle import nngp_oracle as O

from _common import CASES, KERNELS, format_std, load, normalized_y, oracle_params, rel


@pytest.mark.parametrize('name', CASES)
def test_oracle_loglik_matches_reference(name):
    """lml and gradient of the restatement == the reference NumpyNngpr (FP64) to 1e-10."""
    g = load(name)
    p = oracle_params(KP.extract(KERNELS[name]().clone_with_theta(g['theta'])))
    y, _, _ = normalized_y(g)
    m = int(g['num_nn'])
    nbr = O.fit_neighbours(g['x'], min(m, g['x'].shape[0] - 1), p.length_scale, np.float64)
    lml, grad = O.log_marginal_likelihood(g['x'], y, nbr, p, float(g['alpha']), True)
    assert abs(lml / g['lml'] - 1) < 1e-10
    assert rel(grad, g['grad']) < 1e-10


@pytest.mark.parametrize('name', CASES)
def test_oracle_neighbours_match_reference(name):
    """Exact search == the reference's own lists (FP64 and its default FP32 kernel-space search)."""
    g = load(name)
    kern = KERNELS[name]().clone_with_theta(g['theta'])
    ls = KP.extract(kern).length_scale
    m = int(g['num_nn'])
    mm = min(m, g['x'].shape[0] - 1)
    assert np.array_equal(O.fit_neighbours(g['x'], mm, ls, np.float64), g['nbr_fit_f64'])
    assert np.array_equal(O.fit_neighbours(g['x'], mm, ls, np.float32), g['nbr_fit_f32'])
    assert np.array_equal(O.knn(g['x'], g['xq'], min(m, g['x'].shape[0]), None, ls, np.float64), g['nbr_pred_f64'])


@pytest.mark.parametrize('name', CASES)
def test_oracle_predict_matches_reference(name):
    g = load(name)
    p = oracle_params(KP.extract(KERNELS[name]().clone_with_theta(g['theta_pred'])))
    y, ym, ys = normalized_y(g)
    m = min(int(g['num_nn']), g['x'].shape[0])
    nbr = O.knn(g['x'], g['xq'], m, None, p.length_scale, np.float64)
    mean, std = O.predict(g['x'], y, g['xq'], nbr, p, float(g['alpha']))
    mean = (mean * np.reshape(ys, (1, -1)) + np.reshape(ym, (1, -1))).reshape(g['pred_mean'].shape)
    assert np.max(np.abs(mean - g['pred_mean'])) < 1e-10
    assert np.max(np.abs(format_std(std, ys, g['pred_std'].shape) - g['pred_std'])) < 1e-10


@pytest.mark.parametrize('ydim', [1, 3])
def test_oracle_equals_exact_gp(ydim):
    """The reference's known-answer test: NNGP with num_nn = n is the exact GP of scikit-learn
    (nngpr/test/nngpr_base_tester.py:174-192, 228-257)."""
    g = load(f'reftest_n150_y{ydim}')
    sk = load('reftest_sklearn')
    y, ym, ys = normalized_y(g)
    p = oracle_params(KP.extract(KERNELS['reftest_n150_y1']().clone_with_theta(np.full(3, 0.5))))
    nbr = O.fit_neighbours(g['x'], 149, p.length_scale, np.float64)
    lml, grad = O.log_marginal_likelihood(g['x'], y, nbr, p, float(g['alpha']), True)
    assert abs(lml / sk[f'lml_y{ydim}'] - 1) < 1e-10
    assert rel(grad, sk[f'grad_y{ydim}']) < 1e-9
    pp = oracle_params(KP.extract(KERNELS['reftest_n150_y1']()))
    nq = O.knn(g['x'], g['xq'], 150, None, pp.length_scale, np.float64)
    mean, std = O.predict(g['x'], y, g['xq'], nq, pp, float(g['alpha']))
    mean = mean * np.reshape(ys, (1, -1)) + np.reshape(ym, (1, -1))
    assert np.max(np.abs(mean.reshape(sk[f'mean_y{ydim}'].shape) - sk[f'mean_y{ydim}'])) < 1e-9
    assert np.max(np.abs(format_std(std, ys, sk[f'std_y{ydim}'].shape) - sk[f'std_y{ydim}'])) < 1e-9


def test_knn_ties_keep_lower_index():
    """Duplicated points: equal distances are ordered by index (calc_nn's `<=` break)."""
    x = np.repeat(np.array([[0.0, 0.0], [1.0, 0.0], [0.0, 2.0]]), 4, axis=0)
    q = np.array([[0.1, 0.0], [0.5, 0.0]])
    out = O.knn(x, q, 6, None, None)
    assert out[0].tolist() == [0, 1, 2, 3, 4, 5]
    assert out[1].tolist() == [0, 1, 2, 3, 4, 5]


@pytest.mark.parametrize('cut', [None, 0, 2, -1])
def test_knn_ref_cut(cut):
    """ref_cut_index semantics of base_nngpr.py:1660-1681 (query j sees refs [0, j + cut))."""
    rng = np.random.default_rng(3)
    ref = rng.normal(size=(10, 3))
    q = rng.normal(size=(6, 3))
    out = O.knn(ref, q, 4, cut, None, np.float64)
    d2 = ((q[:, None, :] - ref[None]) ** 2).sum(-1)
    for j in range(6):
        lim = 10 if cut is None else max(0, min(10, j + cut))
        order = np.argsort(d2[j, :lim], kind='stable')[:4]
        expect = list(order) + [-1] * (4 - len(order))
        assert out[j].tolist() == expect


def test_knn_more_neighbours_than_refs():
    out = O.knn(np.zeros((2, 1)), np.ones((3, 1)), 5, None, None)
    assert out.shape == (3, 5)
    assert (out[:, 2:] == -1).all() and (out[:, :2] == [0, 1]).all()
