"""GPU kNN through the C ABI vs the exact oracle search: bit-exact index lists."""
import numpy as np
import pytest
import torch

from nngpr_b200 import _lib, ops
from oracle import nngp_oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(params=['tc', 'simt', 'generic'], autouse=True)
def knn_kernel(request, monkeypatch):
    """Every test runs on each search kernel: the tensor-core screen ('tc', where the shape has
    one), the SIMT screen and the generic kernel."""
    monkeypatch.setenv('NNGP_KNN_KERNEL', request.param)
    return request.param


def run_knn(ref, q, m, cut, ls, dtype=np.float32):
    tdt = torch.float32 if dtype == np.float32 else torch.float64
    r = torch.from_numpy(np.ascontiguousarray(ref, dtype=dtype)).cuda()
    qq = r if q is ref else torch.from_numpy(np.ascontiguousarray(q, dtype=dtype)).cuda()
    assert r.dtype == tdt
    flags = ops.new_flags(r.device)
    out = ops.knn(r, qq, m, cut, ls, flags=flags)
    assert int(flags.item()) == 0
    return out.cpu().numpy()


@pytest.mark.parametrize('d', [1, 2, 3, 5, 8, 12, 16, 18, 22, 33])
@pytest.mark.parametrize('m', [1, 7, 16, 32, 48, 70])
def test_knn_prefix_matches_oracle(d, m):
    """The fit-step search (ref = query, cut 0) across the register and generic kernels."""
    rng = np.random.default_rng(100 * d + m)
    n = 700
    x = rng.uniform(-1, 1, (n, d))
    ls = rng.uniform(0.3, 2.0, d) if d % 2 else 0.4
    got = run_knn(x, x, m, 0, ls)
    want = O.knn(x, x, m, 0, ls)
    assert np.array_equal(got, want)


@pytest.mark.parametrize('cut', [None, 0, 2, -1, 5000])
def test_knn_ref_cut_variants(cut):
    rng = np.random.default_rng(7)
    ref = rng.normal(size=(900, 4))
    q = rng.normal(size=(1000, 4))
    got = run_knn(ref, q, 16, cut, [0.5, 1.0, 2.0, 0.7])
    want = O.knn(ref, q, 16, cut, [0.5, 1.0, 2.0, 0.7])
    assert np.array_equal(got, want)


def test_knn_ties_and_duplicates_lower_index_first():
    """Integer grid with duplicated points: many exact ties, resolved by lower index."""
    rng = np.random.default_rng(11)
    x = rng.integers(0, 4, (3000, 3)).astype(np.float64)
    got = run_knn(x, x, 32, 0, None)
    want = O.knn(x, x, 32, 0, None)
    assert np.array_equal(got, want)
    q = rng.integers(0, 4, (500, 3)).astype(np.float64)
    assert np.array_equal(run_knn(x, q, 20, None, None), O.knn(x, q, 20, None, None))


def test_knn_more_neighbours_than_refs_and_empty():
    x = np.random.default_rng(1).normal(size=(5, 3))
    q = np.random.default_rng(2).normal(size=(40, 3))
    assert np.array_equal(run_knn(x, q, 8, None, 1.0), O.knn(x, q, 8, None, 1.0))
    r = torch.zeros((0, 3), device='cuda')
    out = ops.knn(r, torch.zeros((4, 3), device='cuda'), 3, None, None)
    assert (out.cpu().numpy() == -1).all()
    out = ops.knn(torch.zeros((4, 3), device='cuda'), torch.zeros((0, 3), device='cuda'), 3, None, None)
    assert out.shape == (0, 3)


@pytest.mark.parametrize('m', [4, 32, 80])
def test_knn_float64(m):
    rng = np.random.default_rng(5)
    x = rng.uniform(0, 1, (600, 3))
    got = run_knn(x, x, m, 0, 0.3, np.float64)
    want = O.knn(x, x, m, 0, 0.3, np.float64)
    assert np.array_equal(got, want)


def test_knn_large_prefix_sampled_rows():
    """n = 60,000, d = 3, m = 32 fit-step search; 400 sampled rows checked exactly."""
    rng = np.random.default_rng(0)
    n = 60000
    x = rng.uniform(-1, 1, (n, 3)) * np.array([1.0, 0.7, 0.4])
    got = run_knn(x, x, 32, 0, 0.2)
    rows = np.sort(rng.choice(n, 400, replace=False))
    want = O.knn(x, x[rows], 32, 0, 0.2, query_index=rows)
    assert np.array_equal(got[rows], want)


def test_knn_reports_no_flags_and_workspace_errors():
    x = torch.zeros((10, 3), device='cuda')
    out = torch.empty((10, 4), dtype=torch.int32, device='cuda')
    L = _lib.lib()
    import ctypes
    st = L.nngp_knn_f32(ctypes.c_void_p(x.data_ptr()), 10, ctypes.c_void_p(x.data_ptr()), 10, 3, None, 0, 4, 1, 0,
                        ctypes.c_void_p(out.data_ptr()), None, None, 0, None)
    assert st == 3  # NNGP_ERR_WORKSPACE
