"""Predict (conditioning on the training set) through the C ABI vs the golden vectors.

Tolerances: FP64 1e-10 absolute on the un-normalised mean/std (the reference's own test
bound, nngpr/test/nngpr_base_tester.py:228-257); FP32 1e-5 relative to max |value|.
"""
import numpy as np
import pytest
import torch

from nngpr_b200 import ops
from nngpr_b200.kernel_params import extract
from oracle import nngp_oracle as O
from sklearn.gaussian_process import kernels as skk

from _common import CASES, KERNELS, format_std, load, normalized_y, oracle_params, rel

pytestmark = pytest.mark.gpu


def gpu_predict(xt, yt, xq, nbr, p, alpha, dtype):
    tdt = torch.float32 if dtype == np.float32 else torch.float64
    a = torch.from_numpy(np.ascontiguousarray(xt)).to('cuda', tdt)
    b = torch.from_numpy(np.ascontiguousarray(yt if yt.ndim == 2 else yt[:, None])).to("cuda", tdt)
    c = torch.from_numpy(np.ascontiguousarray(xq)).to('cuda', tdt)
    nb = torch.from_numpy(np.ascontiguousarray(nbr, dtype=np.int32)).cuda()
    flags = ops.new_flags(a.device)
    mean, var = ops.predict(a, b, c, nb, p, alpha, flags=flags)
    return mean.double().cpu().numpy(), var.double().cpu().numpy(), int(flags.item())


@pytest.mark.parametrize('name', CASES)
@pytest.mark.parametrize('dtype', [np.float64, np.float32])
def test_predict_golden(name, dtype):
    g = load(name)
    p = extract(KERNELS[name]().clone_with_theta(g['theta_pred']))
    y, ym, ys = normalized_y(g)
    nbr = g['nbr_pred_f64']
    mean, var, flags = gpu_predict(g['x'], y, g['xq'], nbr, p, float(g['alpha']), dtype)
    assert flags & 7 == 0
    mean = (mean * np.reshape(ys, (1, -1)) + np.reshape(ym, (1, -1))).reshape(g['pred_mean'].shape)
    std = format_std(np.sqrt(var), ys, g['pred_std'].shape)
    if dtype == np.float64:
        assert np.max(np.abs(mean - g['pred_mean'])) < 1e-10
        assert np.max(np.abs(std - g['pred_std'])) < 1e-10
    else:
        assert rel(mean, g['pred_mean']) < 1e-5
        assert rel(std, g['pred_std']) < 1e-5


def test_predict_large_subset_fp32():
    rng = np.random.default_rng(1)
    nt, nq = 20000, 5000
    x = rng.uniform(-1, 1, (nt, 3)) * np.array([1.0, 0.7, 0.4])
    y = np.sin(3 * x).sum(1) + rng.normal(0, 0.05, nt)
    xq = rng.uniform(-1, 1, (nq, 3)) * np.array([1.0, 0.7, 0.4])
    p = extract(skk.ConstantKernel(1.0) * skk.RBF(0.2) + skk.WhiteKernel(1e-3))
    nbr = O.knn(x, xq, 32, None, 0.2)
    want_m, want_s = O.predict(x, y, xq, nbr, oracle_params(p), 1e-10)
    mean, var, flags = gpu_predict(x, y, xq, nbr, p, 1e-10, np.float32)
    assert flags & 7 == 0
    assert rel(mean[:, 0], want_m[:, 0]) < 1e-5
    assert rel(np.sqrt(var), want_s) < 1e-5


def test_predict_without_training_points_is_the_prior():
    p = extract(skk.ConstantKernel(2.0) * skk.RBF(0.5) + skk.WhiteKernel(0.1))
    xq = np.random.default_rng(0).normal(size=(10, 2))
    mean, var, _ = gpu_predict(np.zeros((0, 2)), np.zeros((0, 1)), xq, np.zeros((10, 0), np.int32), p, 1e-10,
                               np.float64)
    assert np.all(mean == 0)
    np.testing.assert_allclose(var, 2.1, rtol=1e-15)
