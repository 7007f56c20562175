"""The allocation-free log-likelihood entry point, nngp_loglik_f64_noalloc.

It exists for callers that cannot allocate device memory (a serving process whose device
memory is fixed at start-up, a cgo/JNI/ctypes binding that cannot own CUDA allocations) and so
cannot pass the workspace that nngp_loglik_f64 needs.  Its scratch is a fixed device array
inside the library, shared by all calls, so this test calls it twice in a row and checks both
results against nngp_loglik_f64 (bit for bit on a 148-SM B200, else with the FP64 tolerances of the
other log-likelihood tests): with and without the gradient, through the one-warp-per-point kernel
(up to 32 neighbours) and the one-CTA-per-point kernel (more).
This file is collected last so that a run stopping at the first failure has already run every
other test; it also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest
import torch

from nngpr_b200 import _lib, ops
from nngpr_b200.kernel_params import extract

from _common import KERNELS, load, rel

pytestmark = pytest.mark.gpu

F64_LML, F64_GRAD = 1e-10, 1e-9


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)


def _both(x, y, nbr, p, alpha, grad):
    """nngp_loglik_f64 with a workspace once, then nngp_loglik_f64_noalloc twice in a row (the
    second call finds the first call's partial sums in the shared array)."""
    n, d = x.shape
    ydim, m = y.shape[1], nbr.shape[1]
    keep = []
    k = ops._kernel_struct(p, alpha, d, keep)
    L = _lib.lib()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    nt = 1 + (p.n_theta if grad else 0)
    ws_bytes = int(L.nngp_loglik_workspace_size(n, d, ydim, m, p.n_theta))
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device='cuda')
    ref = torch.empty(nt, dtype=torch.float64, device='cuda')
    _lib.check(L.nngp_loglik_f64(_p(x), _p(y), n, d, ydim, _p(nbr), m, ctypes.byref(k), int(grad), 1e-2, _p(ref),
                                 None, _p(ws), ws_bytes, stream), 'nngp_loglik_f64')
    got = []
    for _ in range(2):
        out = torch.full((nt,), float('nan'), dtype=torch.float64, device='cuda')
        flags = ops.new_flags('cuda')
        _lib.check(L.nngp_loglik_f64_noalloc(_p(x), _p(y), n, d, ydim, _p(nbr), m, ctypes.byref(k), int(grad),
                                             _p(out), _p(flags), stream), 'nngp_loglik_f64_noalloc')
        assert int(flags.item()) == 0
        got.append(out.cpu().numpy())
    return ref.cpu().numpy(), got


def _check(want, got):
    # same kernels, grid and summation order as the workspace entry point on a 148-SM B200:
    # bit for bit there; elsewhere within the FP64 tolerances
    exact = torch.cuda.get_device_properties(0).multi_processor_count == 148
    for g in got:
        if exact:
            np.testing.assert_array_equal(g, want)
        assert abs(g[0] / want[0] - 1) < F64_LML
        if len(want) > 1:
            assert rel(g[1:], want[1:]) < F64_GRAD


def _golden(name):
    g = load(name)
    p = extract(KERNELS[name]().clone_with_theta(g['theta']))
    x = torch.from_numpy(np.ascontiguousarray(g['x'], dtype=np.float64)).cuda()
    y2 = g['y'] if g['y'].ndim == 2 else g['y'][:, None]
    y = torch.from_numpy(np.ascontiguousarray(y2, dtype=np.float64)).cuda()
    nbr = torch.from_numpy(np.ascontiguousarray(g['nbr_fit_f32'], dtype=np.int32)).cuda()
    return g, p, x, y, nbr


@pytest.mark.parametrize('name', ['cpu_n2000_d3_m16', 'ard_n400_d5_m12_y2'])
@pytest.mark.parametrize('grad', [True, False])
def test_noalloc_matches_workspace_entry_point_twice(name, grad):
    g, p, x, y, nbr = _golden(name)
    want, got = _both(x, y, nbr, p, float(g['alpha']), grad)
    _check(want, got)
    assert abs(got[1][0] / g['lml'] - 1) < F64_LML


@pytest.mark.parametrize('grad', [True, False])
def test_noalloc_block_kernel_twice(grad):
    """40 neighbours: the one-CTA-per-point kernel, whose grid (2 CTAs per SM) also fits the array."""
    from oracle import nngp_oracle as O
    from sklearn.gaussian_process import kernels as skk
    rng = np.random.default_rng(40)
    n, d = 600, 3
    xh = rng.uniform(0, 1, (n, d))
    yh = np.sin(4 * xh[:, :1]) + rng.normal(0, 0.05, (n, 1))
    p = extract(skk.ConstantKernel(0.8) * skk.RBF(0.3) + skk.WhiteKernel(0.02))
    nbr = O.fit_neighbours(xh, 40, p.length_scale, np.float32)
    want, got = _both(torch.from_numpy(xh).cuda(), torch.from_numpy(yh).cuda(), torch.from_numpy(nbr).cuda(), p,
                      1e-10, grad)
    _check(want, got)


def test_noalloc_rejects_too_many_hyperparameters():
    L = _lib.lib()
    k = _lib.NngpKernel()
    ls = np.full(40, 0.5)
    k.rbf_level, k.noise_level, k.n_ls = 1.0, 0.1, 40
    k.length_scale = ls.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    k.idx_rbf_level, k.idx_ls, k.idx_noise, k.idx_const, k.n_theta = 0, 1, 41, -1, 42
    out = torch.zeros(43, dtype=torch.float64, device='cuda')
    st = L.nngp_loglik_f64_noalloc(None, None, 10, 40, 1, None, 4, ctypes.byref(k), 1, _p(out), None, None)
    assert st == 2  # NNGP_ERR_UNSUPPORTED
    assert b'at most 35' in L.nngp_last_error()
