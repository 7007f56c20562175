"""Helpers shared by the tests: golden fixtures, the matching kernels, oracle parameters."""
import os

import numpy as np
from sklearn.gaussian_process import kernels as skk

from oracle import nngp_oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')

# kernels of the golden cases (tests/golden/make_golden.py), as scikit-learn kernels
KERNELS = {
    'cpu_n2000_d3_m16': lambda: skk.ConstantKernel(1.0) * skk.RBF(0.3) + skk.WhiteKernel(0.01),
    'reftest_n150_y1': lambda: skk.ConstantKernel(1) * skk.RBF(length_scale=1) + skk.WhiteKernel(1),
    'reftest_n150_y3': lambda: skk.ConstantKernel(1) * skk.RBF(length_scale=1) + skk.WhiteKernel(1),
    'ard_n400_d5_m12_y2': lambda: skk.ConstantKernel(0.7) * skk.RBF(np.array([0.3, 0.5, 0.8, 1.2, 2.0]))
    + skk.WhiteKernel(0.05),
    'const_n300_d2_m10': lambda: skk.ConstantKernel(0.5) + skk.ConstantKernel(1.3) * skk.RBF(0.4)
    + skk.WhiteKernel(0.02),
    'matern12_n500_d3_m16': lambda: skk.ConstantKernel(0.9) * skk.Matern(0.4, nu=0.5) + skk.WhiteKernel(0.01),
    'matern32_n450_d4_m12': lambda: skk.ConstantKernel(1.2) * skk.Matern(0.7, nu=1.5) + skk.WhiteKernel(0.02),
    'matern52_n400_d2_m10': lambda: skk.ConstantKernel(1.0) * skk.Matern(0.6, nu=2.5) + skk.WhiteKernel(0.005),
    'wide_n300_d3_m16_y100': lambda: skk.ConstantKernel(1.0) * skk.RBF(0.4) + skk.WhiteKernel(0.02),
}
CASES = sorted(KERNELS)


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name + '.npz')))


def oracle_params(p):
    """nngpr_b200.kernel_params.RbfParams -> oracle KernelParams."""
    return O.KernelParams(rbf_level=p.rbf_level, const_value=p.const_value, noise_level=p.noise_level,
                          length_scale=1.0 if p.length_scale is None else p.length_scale,
                          idx_rbf_level=p.idx_rbf_level, idx_const=p.idx_const, idx_noise=p.idx_noise,
                          idx_ls=p.idx_ls, n_theta=p.n_theta, family=p.family)


def normalized_y(g):
    """y as the fitted reference model holds it (normalize_y applied, base_nngpr.py:310-320)."""
    y = g['y']
    if g['normalize_y']:
        return (y - y.mean(0)) / y.std(0), y.mean(0), y.std(0)
    return y, np.zeros(y.shape[1:] or (1,)), np.ones(y.shape[1:] or (1,))


def format_std(std, y_std, shape):
    """format_sigma of the reference (base_nngpr.py:851-858)."""
    s = std.reshape(-1, 1) * np.asarray(y_std).reshape(1, -1)
    return s.reshape(shape) if s.size == np.prod(shape) else s[:, 0]


def rel(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


_SCALE = {}


def lml_scale(name):
    """Sum over points of |per-point log-likelihood| of a golden case (oracle, FP64): the scale
    the FP32 paths' error is measured against (the total lml can be a heavily cancelled sum)."""
    if name not in _SCALE:
        from nngpr_b200.kernel_params import extract
        g = load(name)
        p = extract(KERNELS[name]().clone_with_theta(g['theta']))
        y, _, _ = normalized_y(g)
        y2 = y if y.ndim == 2 else y[:, None]
        ll, _ = O.loglik_terms(g['x'], y2, g['nbr_fit_f64'], oracle_params(p), float(g['alpha']), False)
        _SCALE[name] = max(float(np.abs(ll).sum()), abs(float(g['lml'])))
    return _SCALE[name]


FULL_CASES = ['cpu_n2000_d3_m16', 'ard_n400_d5_m12_y2', 'matern52_n400_d2_m10']


def load_full(name):
    """The reference's predict(conditioning_method='full') on a golden case (make_golden.py)."""
    return dict(np.load(os.path.join(GOLDEN, 'full_' + name + '.npz')))
