"""Predict with conditioning_method='full' through the C ABI and the estimator against the
reference's own outputs (its sequential algorithm, base_nngpr.py:896-1030), FP64: 1e-10."""
import numpy as np
import pytest
import torch

from nngpr_b200 import B200Nngpr, _lib, ops
from nngpr_b200 import kernel_params as KP

from _common import FULL_CASES, KERNELS, format_std, load, load_full, normalized_y

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('name', FULL_CASES)
def test_predict_full_abi_matches_reference(name):
    g, f = load(name), load_full(name)
    y, ym, ys = normalized_y(g)
    p = KP.extract(KERNELS[name]().clone_with_theta(g['theta_pred']))
    dev = torch.device('cuda')
    xt = torch.from_numpy(g['x']).to(dev)
    yt = torch.from_numpy(np.ascontiguousarray(y.reshape(len(y), -1))).to(dev)
    xq = torch.from_numpy(g['xq']).to(dev)
    nbr = torch.from_numpy(np.ascontiguousarray(f['nbr'], dtype=np.int32)).to(dev)
    flags = ops.new_flags(dev)
    mean, var = ops.predict_full(xt, yt, xq, nbr, p, float(g['alpha']), True, flags=flags)
    assert int(flags.item()) & ~_lib.NNGP_FLAG_NOT_PD == 0
    mean = mean.cpu().numpy() * np.asarray(ys).reshape(1, -1) + np.asarray(ym).reshape(1, -1)
    assert np.max(np.abs(mean - np.asarray(f['mean']).reshape(mean.shape))) < 1e-10
    std = np.sqrt(var.cpu().numpy())
    assert np.max(np.abs(format_std(std, ys, f['std'].shape) - f['std'])) < 1e-10
    mean2, var2 = ops.predict_full(xt, yt, xq, nbr, p, float(g['alpha']), False)
    assert var2 is None
    np.testing.assert_array_equal(mean2.cpu().numpy() * np.asarray(ys).reshape(1, -1) + np.asarray(ym).reshape(1, -1),
                                  mean)


@pytest.mark.parametrize('name', FULL_CASES)
def test_estimator_full_conditioning(name):
    g, f = load(name), load_full(name)
    gpr = B200Nngpr(kernel=KERNELS[name](), num_nn=int(g['num_nn']), alpha=float(g['alpha']),
                    normalize_y=bool(g['normalize_y']), optimizer=None, allow_downcast_f32='no').fit(g['x'], g['y'])
    gpr.kernel_ = gpr.kernel_.clone_with_theta(g['theta_pred'])
    mean, std = gpr.predict(g['xq'], return_std=True, conditioning_method='full')
    assert mean.shape == f['mean'].shape and std.shape == f['std'].shape
    assert np.max(np.abs(mean - f['mean'])) < 1e-10
    assert np.max(np.abs(std - f['std'])) < 1e-10
    np.testing.assert_array_equal(gpr.predict(g['xq'], conditioning_method='full'), mean)


def test_predict_full_flags_a_later_query_as_neighbour():
    g, f = load('cpu_n2000_d3_m16'), load_full('cpu_n2000_d3_m16')
    p = KP.extract(KERNELS['cpu_n2000_d3_m16']().clone_with_theta(g['theta_pred']))
    dev = torch.device('cuda')
    nbr = np.ascontiguousarray(f['nbr'], dtype=np.int32)
    nt = g['x'].shape[0]
    nbr[3, 0] = nt + 10  # query 3 cannot condition on query 10
    flags = ops.new_flags(dev)
    ops.predict_full(torch.from_numpy(g['x']).to(dev), torch.from_numpy(g['y'][:, None]).to(dev),
                     torch.from_numpy(g['xq']).to(dev), torch.from_numpy(nbr).to(dev), p, 1e-10, True, flags=flags)
    assert int(flags.item()) & _lib.NNGP_FLAG_BAD_INDEX


@pytest.mark.parametrize('name', FULL_CASES)
def test_sample_y_full_reproduces_the_reference(name):
    """sample_y(conditioning_method='full', random_state=11) returns the reference's own samples
    (same normals, drawn as the reference draws them; recursion on the device)."""
    g, f = load(name), load_full(name)
    gpr = B200Nngpr(kernel=KERNELS[name](), num_nn=int(g['num_nn']), alpha=float(g['alpha']),
                    normalize_y=bool(g['normalize_y']), optimizer=None, allow_downcast_f32='no').fit(g['x'], g['y'])
    s = gpr.sample_y(g['xq'][:60], n_samples=4, random_state=11, conditioning_method='full')
    assert s.shape == f['samples60'].shape
    assert np.max(np.abs(s - f['samples60'])) < 1e-9


@pytest.mark.parametrize('name', FULL_CASES)
@pytest.mark.parametrize('method', ['full', 'only-train'])
def test_return_cov_matches_reference(name, method):
    """predict(return_cov=True): the dense predictive covariance of the sequential algorithm
    ('full'), diagonal for 'only-train' (its queries are independent); the reference's outputs
    on the first 80 queries, FP64: 1e-10."""
    g, f = load(name), load_full(name)
    gpr = B200Nngpr(kernel=KERNELS[name](), num_nn=int(g['num_nn']), alpha=float(g['alpha']),
                    normalize_y=bool(g['normalize_y']), optimizer=None, allow_downcast_f32='no').fit(g['x'], g['y'])
    mean, cov = gpr.predict(g['xq'][:80], return_cov=True, conditioning_method=method)
    want = f['cov80_full'] if method == 'full' else f['cov80_train']
    assert cov.shape == want.shape
    assert np.max(np.abs(cov - want)) < 1e-10
    want_mean = gpr.predict(g['xq'][:80], conditioning_method=method)
    np.testing.assert_array_equal(mean, want_mean)
    _, std = gpr.predict(g['xq'][:80], return_std=True, return_cov=True, conditioning_method=method)
    assert std.shape == want_mean.shape  # both asked for: the standard deviation, as the reference


def _fitted(name, g, **kw):
    return B200Nngpr(kernel=KERNELS[name](), num_nn=int(g['num_nn']), alpha=float(g['alpha']),
                     normalize_y=bool(g['normalize_y']), optimizer=None, allow_downcast_f32='no',
                     **kw).fit(g['x'], g['y'])


@pytest.mark.parametrize('name', FULL_CASES)
def test_double_nn_matches_reference(name):
    """conditioning_method='full-double-nn' (base_nngpr.py:1418-1449): the device lists are the
    reference's (training search + prefix search of the queries, packed valid-first), and predict
    (mean, std, dense covariance of the first 80) and sample_y (random_state=12, first 60) give
    the reference's outputs, FP64: 1e-10 (samples 1e-9)."""
    g, f = load(name), load_full(name)
    gpr = _fitted(name, g)
    dev = torch.device('cuda')
    p = gpr._params(gpr.kernel_)
    xt, _ = gpr._train_tensors(torch.float64)
    nbr = gpr._full_lists(xt, torch.from_numpy(g['xq']).to(dev), p, torch.float64, True, ops.new_flags(dev))
    np.testing.assert_array_equal(nbr.cpu().numpy(), f['dn_nbr'])
    mean, std = gpr.predict(g['xq'], return_std=True, conditioning_method='full-double-nn')
    assert mean.shape == f['dn_mean'].shape and std.shape == f['dn_std'].shape
    assert np.max(np.abs(mean - f['dn_mean'])) < 1e-10
    assert np.max(np.abs(std - f['dn_std'])) < 1e-10
    _, cov = gpr.predict(g['xq'][:80], return_cov=True, conditioning_method='full-double-nn')
    assert cov.shape == f['dn_cov80'].shape
    assert np.max(np.abs(cov - f['dn_cov80'])) < 1e-10
    s = gpr.sample_y(g['xq'][:60], n_samples=4, random_state=12, conditioning_method='full-double-nn')
    assert s.shape == f['dn_samples60'].shape
    assert np.max(np.abs(s - f['dn_samples60'])) < 1e-9


def test_full_with_48_neighbours_matches_reference():
    """'full' with num_nn = 48: the local systems take the one-CTA-per-system kernel and the
    recursions two slots per lane; the reference's mean and std on the first 150 queries
    (1e-10), and the dense covariance and the samples against the oracle on the same lists."""
    name = 'cpu_n2000_d3_m16'
    g, f = load(name), load_full(name)
    gpr = B200Nngpr(kernel=KERNELS[name](), num_nn=48, alpha=float(g['alpha']), normalize_y=bool(g['normalize_y']),
                    optimizer=None, allow_downcast_f32='no').fit(g['x'], g['y'])
    xq = g['xq'][:150]
    mean, std = gpr.predict(xq, return_std=True, conditioning_method='full')
    assert np.max(np.abs(mean - f['f48_mean'])) < 1e-10
    assert np.max(np.abs(std - f['f48_std'])) < 1e-10
    from oracle import nngp_oracle as O
    from _common import oracle_params
    y, ym, ys = normalized_y(g)
    po = oracle_params(KP.extract(gpr.kernel_))
    _, cov_o = O.predict_cov_full(g['x'], y, xq, f['f48_nbr'], po, float(g['alpha']))
    _, cov = gpr.predict(xq, return_cov=True, conditioning_method='full')
    assert np.max(np.abs(cov - cov_o * float(np.asarray(ys).reshape(-1)[0]) ** 2)) < 1e-10
    z = np.random.RandomState(5).standard_normal((150, 1, 3))
    s_o = O.sample_full(g['x'], y[:, None], xq, f['f48_nbr'], po, float(g['alpha']), z)
    s = gpr.sample_y(xq, n_samples=3, random_state=5, conditioning_method='full')
    assert np.max(np.abs(s - (s_o[:, 0, :] * float(np.asarray(ys).reshape(-1)[0]) + float(np.asarray(ym).reshape(-1)[0])))) < 1e-9


def test_sequential_conditioning_slot_limit():
    g = load('cpu_n2000_d3_m16')
    x, y, xq = g['x'][:300], g['y'][:300], g['xq'][:20]
    k = KERNELS['cpu_n2000_d3_m16']
    with pytest.raises(NotImplementedError):
        B200Nngpr(kernel=k(), num_nn=70, optimizer=None).fit(x, y).predict(xq, conditioning_method='full')
    gpr40 = B200Nngpr(kernel=k(), num_nn=40, optimizer=None).fit(x, y)
    with pytest.raises(NotImplementedError):  # 40 training + 29 query slots
        gpr40.sample_y(g['xq'][:30], conditioning_method='full-double-nn')
    assert gpr40.predict(xq, conditioning_method='full-double-nn').shape == (20,)  # 40 + 19 slots
    # one query: no earlier query to condition on, the double lists are the training lists, so
    # both give the same prediction; equal to rounding, not bit for bit: 'only-train' forms
    # mu = l . z (l = L^-1 k, z = L^-1 y) and the recursion mu = w . y with w = L^-T l
    gpr = B200Nngpr(kernel=k(), num_nn=8, optimizer=None, allow_downcast_f32='no').fit(x, y)
    np.testing.assert_allclose(gpr.predict(xq[:1], conditioning_method='full-double-nn'),
                               gpr.predict(xq[:1], conditioning_method='only-train'), rtol=1e-13, atol=0)
