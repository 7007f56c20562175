"""The plain FP32 form's search (the benchmark's comparator) returns the optimised search's lists,
and its FP32 log-likelihood agrees with the optimised path within FP32 accuracy."""
import numpy as np
import pytest
import torch

from nngpr_b200 import ops
from nngpr_b200.kernel_params import extract
from nngpr_b200.plain import plain_knn, plain_loglik
from oracle import nngp_oracle as O

from _common import KERNELS, load, normalized_y, rel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('d,m,cut', [(3, 32, 0), (3, 16, None), (8, 32, 0), (16, 32, 0), (5, 7, 2)])
def test_plain_knn_equals_optimised(d, m, cut):
    rng = np.random.default_rng(d * 100 + m)
    x = torch.from_numpy(rng.uniform(-1, 1, (3000, d)).astype(np.float32)).cuda()
    q = x if cut is not None else torch.from_numpy(rng.uniform(-1, 1, (700, d)).astype(np.float32)).cuda()
    ls = 0.3 if d != 5 else [0.3, 0.5, 0.7, 1.1, 2.0]
    a = plain_knn(x, q, m, cut, ls).cpu().numpy()
    b = ops.knn(x, q, m, cut, ls).cpu().numpy()
    assert np.array_equal(a, b)
    rows = np.arange(0, q.shape[0], 37)
    want = O.knn(x.cpu().numpy(), q.cpu().numpy()[rows], m, cut, ls, query_index=rows if cut is not None else None)
    assert np.array_equal(a[rows], want)


def test_plain_loglik_on_gpu():
    g = load('cpu_n2000_d3_m16')
    p = extract(KERNELS['cpu_n2000_d3_m16']().clone_with_theta(g['theta']))
    y, _, _ = normalized_y(g)
    x = torch.from_numpy(g['x']).cuda()
    nbr = plain_knn(x, x, 16, 0, p.length_scale)
    lml, grad = plain_loglik(x, torch.from_numpy(np.asarray(y)).cuda(), nbr, p, float(g['alpha']))
    assert abs(float(lml) / float(g['lml']) - 1) < 2e-4
    assert rel(grad.cpu().numpy(), g['grad']) < 2e-3


def _ref_root():
    import os
    root = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), 'baseline', '_ref')
    from nngpr_b200 import plain_ref
    if not plain_ref.available(root):
        pytest.skip('the reference is not installed under baseline/_ref')
    return root


@pytest.mark.parametrize('d,m,cut', [(3, 32, 0), (16, 32, 0), (5, 16, None)])
def test_reference_calc_nn_compiled_from_its_source(d, m, cut):
    """The reference's own calc_nn (compiled with NVRTC from the installed reference, as cupy
    would) against this library's search: NVRTC contracts its distance sum into FMAs, so a row may
    order a near tie differently; at least 99 % of the rows are identical here."""
    root = _ref_root()
    rng = np.random.default_rng(d + m)
    x = torch.from_numpy(rng.uniform(-1, 1, (3000, d)).astype(np.float32)).cuda()
    q = x if cut is not None else torch.from_numpy(rng.uniform(-1, 1, (700, d)).astype(np.float32)).cuda()
    ls = 0.3 if d != 5 else [0.3, 0.5, 0.7, 1.1, 2.0]
    a = plain_knn(x, q, m, cut, ls, ref_root=root).cpu().numpy()
    b = ops.knn(x, q, m, cut, ls).cpu().numpy()
    same_rows = np.all(a == b, axis=1).mean()
    assert same_rows >= 0.99, same_rows
    # where the lists differ it is a near tie at the edge or a swap: at most two refs differ per row
    differ = np.array([len(set(r.tolist()) ^ set(s.tolist())) for r, s in zip(a, b)])
    assert differ.max() <= 4


def test_reference_fill_kernel_compiled_from_its_source():
    """The reference's own fill_nn_kernel inside the plain log-likelihood: golden value at FP32
    accuracy."""
    root = _ref_root()
    g = load('cpu_n2000_d3_m16')
    p = extract(KERNELS['cpu_n2000_d3_m16']().clone_with_theta(g['theta']))
    y, _, _ = normalized_y(g)
    x = torch.from_numpy(g['x']).cuda()
    nbr = torch.from_numpy(np.ascontiguousarray(g['nbr_fit_f32'], dtype=np.int32)).cuda()
    lml, grad = plain_loglik(x, torch.from_numpy(np.asarray(y)).cuda(), nbr, p, float(g['alpha']), ref_root=root)
    assert abs(float(lml) / float(g['lml']) - 1) < 2e-4
    assert rel(grad.cpu().numpy(), g['grad']) < 2e-3
