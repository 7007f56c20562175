"""Kernel-tree reduction and theta map (CPU only).

Checked against hand-derived values and, when the reference source is importable in this
environment (``baseline/_ref``), against the reference's batched kernel classes.
"""
import os
import sys

import numpy as np
import pytest
from sklearn.gaussian_process import kernels as skk

from nngpr_b200.kernel_params import extract, theta_map

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_white_plus_c_rbf():
    p = extract(skk.ConstantKernel(2.0) * skk.RBF(0.3) + skk.WhiteKernel(0.01))
    assert p.rbf_level == pytest.approx(2.0) and p.noise_level == pytest.approx(0.01)
    assert p.length_scale == pytest.approx(0.3) and p.const_value == 0.0
    assert (p.idx_rbf_level, p.idx_ls, p.idx_noise, p.idx_const, p.n_theta) == (0, 1, 2, -1, 3)


def test_ard_and_constant():
    k = skk.ConstantKernel(0.5) + skk.ConstantKernel(1.3) * skk.RBF(np.array([0.1, 0.2, 0.3])) + skk.WhiteKernel(0.02)
    p = extract(k)
    assert p.ard and p.n_ls == 3
    np.testing.assert_allclose(p.length_scale, [0.1, 0.2, 0.3])
    assert p.const_value == pytest.approx(0.5) and p.rbf_level == pytest.approx(1.3)
    assert (p.idx_const, p.idx_rbf_level, p.idx_ls, p.idx_noise, p.n_theta) == (0, 1, 2, 5, 6)


def test_fixed_hyperparameters_have_no_theta():
    k = skk.ConstantKernel(1.0, constant_value_bounds='fixed') * skk.RBF(0.4) + skk.WhiteKernel(
        0.1, noise_level_bounds='fixed')
    p = extract(k)
    assert (p.idx_rbf_level, p.idx_ls, p.idx_noise, p.n_theta) == (-1, 0, -1, 1)


def test_rbf_alone_and_white_alone():
    p = extract(skk.RBF(2.0))
    assert p.rbf_level == 1.0 and p.idx_ls == 0
    q = extract(skk.WhiteKernel(0.3) + skk.ConstantKernel(0.2))
    assert q.length_scale is None and q.rbf_level == 0.0 and q.n_theta == 2


@pytest.mark.parametrize('kernel', [
    skk.RBF(1.0) + skk.RBF(2.0),
    skk.RBF(1.0) * skk.RBF(2.0),
    skk.Matern(1.0, nu=2.0),
    skk.ConstantKernel(1.0) * skk.ConstantKernel(2.0) * skk.RBF(1.0),
])
def test_unsupported_kernels_raise(kernel):
    with pytest.raises(NotImplementedError, match='Cannot accelerate'):
        extract(kernel)


def _reference_kernels():
    for path in (os.path.join(ROOT, 'baseline', '_ref'), os.environ.get('NNGPR_REFERENCE', '')):
        if path and os.path.isdir(os.path.join(path, 'nngpr')):
            sys.path.insert(0, path)
            try:
                from nngpr import batched_kernels
                return batched_kernels
            except Exception:  # pragma: no cover
                return None
            finally:
                sys.path.remove(path)
    return None


def test_reference_batched_kernels_are_accepted():
    bk = _reference_kernels()
    if bk is None:
        pytest.skip('reference source not available here')
    k = bk.ConstantKernel(0.7) * bk.RBF(np.array([0.3, 0.5])) + bk.WhiteKernel(0.05)
    p = extract(k)
    assert p.rbf_level == pytest.approx(0.7) and p.noise_level == pytest.approx(0.05)
    assert theta_map(k) == {'rbf_level': 0, 'length_scale': [1, 2], 'noise_level': 3}


@pytest.mark.parametrize('kernel', [
    skk.ConstantKernel(2.0) * skk.RBF(0.3) + skk.WhiteKernel(0.01),
    skk.ConstantKernel(0.5) + skk.ConstantKernel(1.3) * skk.RBF(np.array([0.1, 0.2, 0.3])) + skk.WhiteKernel(0.02),
    skk.ConstantKernel(1.0, constant_value_bounds='fixed') * skk.RBF(0.4) + skk.WhiteKernel(0.1),
    skk.RBF(np.array([0.5, 2.0])) + skk.WhiteKernel(0.3, noise_level_bounds='fixed'),
])
def test_params_from_theta_equals_clone_with_theta(kernel):
    from nngpr_b200.kernel_params import params_from_theta
    rng = np.random.default_rng(3)
    theta = kernel.theta + rng.normal(0, 0.3, kernel.theta.shape)
    want = extract(kernel.clone_with_theta(theta))
    got = params_from_theta(extract(kernel), theta)
    for f in ('rbf_level', 'const_value', 'noise_level'):
        assert getattr(got, f) == pytest.approx(getattr(want, f), rel=1e-14)
    if want.length_scale is None:
        assert got.length_scale is None
    else:
        np.testing.assert_allclose(np.asarray(got.length_scale), np.asarray(want.length_scale), rtol=1e-14)
    assert (got.idx_rbf_level, got.idx_const, got.idx_noise, got.idx_ls, got.n_theta) == (
        want.idx_rbf_level, want.idx_const, want.idx_noise, want.idx_ls, want.n_theta)


@pytest.mark.parametrize('nu,family', [(0.5, 1), (1.5, 2), (2.5, 3), (np.inf, 0)])
def test_matern_families(nu, family):
    k = skk.ConstantKernel(0.7) * skk.Matern(np.array([0.3, 0.9]), nu=nu) + skk.WhiteKernel(0.05)
    p = extract(k)
    assert p.family == family and p.ard and p.rbf_level == pytest.approx(0.7)
    assert (p.idx_rbf_level, p.idx_ls, p.idx_noise, p.n_theta) == (0, 1, 3, 4)
    assert extract(skk.RBF(1.0)).family == 0
