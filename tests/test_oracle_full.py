"""The oracle's restatement of predict(conditioning_method='full') (the reference's sequential
algorithm, base_nngpr.py:896-1030) against the reference's own outputs on three golden cases."""
import numpy as np
import pytest

from nngpr_b200 import kernel_params as KP
from oracle import nngp_oracle as O

from _common import FULL_CASES, KERNELS, format_std, load, load_full, normalized_y, oracle_params


@pytest.mark.parametrize('name', FULL_CASES)
def test_oracle_full_predict_matches_reference(name):
    g, f = load(name), load_full(name)
    y, ym, ys = normalized_y(g)
    p = oracle_params(KP.extract(KERNELS[name]().clone_with_theta(g['theta_pred'])))
    mean, std = O.predict_full(g['x'], y, g['xq'], f['nbr'], p, float(g['alpha']), True)
    mean = mean * np.asarray(ys).reshape(1, -1) + np.asarray(ym).reshape(1, -1)
    want = np.asarray(f['mean']).reshape(mean.shape)
    assert np.max(np.abs(mean - want)) < 1e-10
    assert np.max(np.abs(format_std(std, ys, f['std'].shape) - f['std'])) < 1e-10
    np.testing.assert_array_equal(np.asarray(f['mean_only']), np.asarray(f['mean']))


@pytest.mark.parametrize('name', FULL_CASES)
def test_full_neighbour_lists_are_the_prefix_search(name):
    """The reference's lists for 'full' are the search of [x_train; x_query] where query i may
    use the training set and the queries before it (ref_cut_index = n_train)."""
    g, f = load(name), load_full(name)
    x_full = np.concatenate([g['x'], g['xq']])
    ls = KP.extract(KERNELS[name]().clone_with_theta(g['theta_pred'])).length_scale
    got = O.knn(x_full, g['xq'], f['nbr'].shape[1], g['x'].shape[0], ls, np.float64)
    assert np.array_equal(got, f['nbr'])


@pytest.mark.parametrize('name', FULL_CASES)
def test_oracle_full_samples_reproduce_the_reference_stream(name):
    """sample_y(conditioning_method='full', random_state=11): the reference draws its normals
    query by query from sklearn's check_random_state(11), a numpy RandomState; with the same
    normals the restatement gives the reference's samples."""
    g, f = load(name), load_full(name)
    y, ym, ys = normalized_y(g)
    y2 = y if y.ndim == 2 else y[:, None]
    p = oracle_params(KP.extract(KERNELS[name]().clone_with_theta(g['theta_pred'])))
    z = np.random.RandomState(11).standard_normal((60, y2.shape[1], 4))
    out = O.sample_full(g['x'], y2, g['xq'][:60], f['nbr60'], p, float(g['alpha']), z)
    out = out * np.asarray(ys).reshape(1, -1, 1) + np.asarray(ym).reshape(1, -1, 1)
    want = np.asarray(f['samples60']).reshape(out.shape)
    assert np.max(np.abs(out - want)) < 1e-9


@pytest.mark.parametrize('name', FULL_CASES)
def test_oracle_dense_covariance_matches_reference(name):
    """predict(return_cov=True, conditioning_method='full') on the first 80 queries."""
    g, f = load(name), load_full(name)
    y, ym, ys = normalized_y(g)
    p = oracle_params(KP.extract(KERNELS[name]().clone_with_theta(g['theta_pred'])))
    _, cov = O.predict_cov_full(g['x'], y, g['xq'][:80], f['nbr80'], p, float(g['alpha']))
    c = cov[:, :, None] * np.asarray(ys).reshape(1, 1, -1) ** 2
    want = np.asarray(f['cov80_full']).reshape(c.shape)
    assert np.max(np.abs(c - want)) < 1e-10
    assert np.abs(want[~np.eye(80, dtype=bool)]).max() > 0  # the covariance is dense


@pytest.mark.parametrize('name', FULL_CASES)
def test_double_nn_lists_match_reference(name):
    """'full-double-nn' lists: the training search and the prefix search of the queries,
    packed valid-first (base_nngpr.py:1418-1449)."""
    g, f = load(name), load_full(name)
    ls = KP.extract(KERNELS[name]().clone_with_theta(g['theta_pred'])).length_scale
    got = O.double_nn_lists(g['x'], g['xq'], int(g['num_nn']), ls, np.float64)
    assert got.shape == f['dn_nbr'].shape == (g['xq'].shape[0], 2 * int(g['num_nn']))
    assert np.array_equal(got, f['dn_nbr'])


@pytest.mark.parametrize('name', FULL_CASES)
def test_oracle_double_nn_predict_sample_cov_match_reference(name):
    """The sequential algorithm on the double lists gives the reference's 'full-double-nn' mean,
    std, samples (random_state=12) and dense covariance."""
    g, f = load(name), load_full(name)
    y, ym, ys = normalized_y(g)
    y2 = y if y.ndim == 2 else y[:, None]
    p = oracle_params(KP.extract(KERNELS[name]().clone_with_theta(g['theta_pred'])))
    nb = f['dn_nbr']
    mean, std = O.predict_full(g['x'], y, g['xq'], nb, p, float(g['alpha']), True)
    mean = mean * np.asarray(ys).reshape(1, -1) + np.asarray(ym).reshape(1, -1)
    assert np.max(np.abs(mean - np.asarray(f['dn_mean']).reshape(mean.shape))) < 1e-10
    assert np.max(np.abs(format_std(std, ys, f['dn_std'].shape) - f['dn_std'])) < 1e-10
    z = np.random.RandomState(12).standard_normal((60, y2.shape[1], 4))
    out = O.sample_full(g['x'], y2, g['xq'][:60], nb[:60], p, float(g['alpha']), z)
    out = out * np.asarray(ys).reshape(1, -1, 1) + np.asarray(ym).reshape(1, -1, 1)
    assert np.max(np.abs(out - np.asarray(f['dn_samples60']).reshape(out.shape))) < 1e-9
    _, cov = O.predict_cov_full(g['x'], y, g['xq'][:80], nb[:80], p, float(g['alpha']))
    c = cov[:, :, None] * np.asarray(ys).reshape(1, 1, -1) ** 2
    assert np.max(np.abs(c - np.asarray(f['dn_cov80']).reshape(c.shape))) < 1e-10


def test_oracle_full_48_neighbours_matches_reference():
    """'full' with num_nn = 48 (more slots than one warp has lanes) on the first 150 queries."""
    name = 'cpu_n2000_d3_m16'
    g, f = load(name), load_full(name)
    y, ym, ys = normalized_y(g)
    kp = KP.extract(KERNELS[name]().clone_with_theta(g['theta_pred']))
    x_full = np.concatenate([g['x'], g['xq'][:150]])
    nb = O.knn(x_full, g['xq'][:150], 48, g['x'].shape[0], kp.length_scale, np.float64)
    assert np.array_equal(nb, f['f48_nbr'])
    mean, std = O.predict_full(g['x'], y, g['xq'][:150], nb, oracle_params(kp), float(g['alpha']), True)
    mean = mean * np.asarray(ys).reshape(1, -1) + np.asarray(ym).reshape(1, -1)
    assert np.max(np.abs(mean - np.asarray(f['f48_mean']).reshape(mean.shape))) < 1e-10
    assert np.max(np.abs(format_std(std, ys, f['f48_std'].shape) - f['f48_std'])) < 1e-10
