"""The plain FP32 form (the benchmark's comparator) against the reference's golden values.

Its local-system part is pure torch, so it runs here on the CPU; its search needs the GPU
(tests/test_gpu_plain.py).  Tolerances are FP32-level: the comparator computes in FP32 and is
only required to be the same computation, not an accurate one.
"""
import numpy as np
import pytest
import torch

from nngpr_b200.kernel_params import extract
from nngpr_b200.plain import plain_loglik, plain_predict

from _common import CASES, KERNELS, load, normalized_y, rel


@pytest.mark.parametrize('name', CASES)
def test_plain_loglik_matches_reference(name):
    g = load(name)
    p = extract(KERNELS[name]().clone_with_theta(g['theta']))
    y, _, _ = normalized_y(g)
    nbr = g['nbr_fit_f64'] if 'nbr_fit_f64' in g else None
    if nbr is None:
        pytest.skip('case has no stored neighbour lists')
    lml, grad = plain_loglik(torch.from_numpy(g['x']), torch.from_numpy(np.asarray(y)), torch.from_numpy(nbr), p,
                             float(g['alpha']), batch=700)
    assert abs(float(lml) / float(g['lml']) - 1) < 2e-4
    assert rel(grad.numpy(), g['grad']) < 2e-3


@pytest.mark.parametrize('name', CASES)
def test_plain_predict_matches_reference(name):
    g = load(name)
    if 'nbr_pred_f64' not in g:
        pytest.skip('case has no stored neighbour lists')
    p = extract(KERNELS[name]().clone_with_theta(g['theta_pred']))
    y, y_mean, y_std = normalized_y(g)
    mean, std = plain_predict(torch.from_numpy(g['x']), torch.from_numpy(np.asarray(y)), torch.from_numpy(g['xq']),
                              torch.from_numpy(g['nbr_pred_f64']), p, float(g['alpha']), batch=300)
    mean = mean.numpy().astype(np.float64) * np.asarray(y_std).reshape(1, -1) + np.asarray(y_mean).reshape(1, -1)
    want = np.asarray(g['pred_mean']).reshape(mean.shape)
    assert rel(mean, want) < 1e-4
    s = std.numpy().astype(np.float64)[:, None] * np.asarray(y_std).reshape(1, -1)
    assert rel(s.reshape(-1)[:g['pred_std'].size], np.asarray(g['pred_std']).reshape(-1)) < 1e-4
