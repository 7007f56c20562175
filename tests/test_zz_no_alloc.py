"""The allocation-free log-likelihood entry point, nngp_loglik_f64_noalloc.

It exists for callers that cannot allocate device memory (a serving process whose device
memory is fixed at start-up, a cgo/JNI/ctypes binding that cannot own CUDA allocations) and so
cannot pass the workspace that nngp_loglik_f64 needs.  Its scratch is a fixed device array
inside the library, shared by all calls, so this test calls it twice in a row and checks both
results against nngp_loglik_f64 with the FP64 tolerances of the other log-likelihood tests.
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


@pytest.mark.parametrize('name', ['cpu_n2000_d3_m16', 'ard_n400_d5_m12_y2'])
def test_noalloc_matches_workspace_entry_point_twice(name):
    g = load(name)
    p = extract(KERNELS[name]().clone_with_theta(g['theta']))
    x = torch.from_numpy(np.ascontiguousarray(g['x'], dtype=np.float64)).cuda()
    y2 = g['y'] if g['y'].ndim == 2 else g['y'][:, None]
    y = torch.from_numpy(np.ascontiguousarray(y2, dtype=np.float64)).cuda()
    nbr = torch.from_numpy(np.ascontiguousarray(g['nbr_fit_f32'], dtype=np.int32)).cuda()
    n, d = x.shape
    ydim, m = y.shape[1], nbr.shape[1]
    keep = []
    k = ops._kernel_struct(p, float(g['alpha']), d, keep)
    L = _lib.lib()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    ws_bytes = int(L.nngp_loglik_workspace_size(n, d, ydim, m, p.n_theta))
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device='cuda')
    ref = torch.empty(1 + p.n_theta, dtype=torch.float64, device='cuda')
    _lib.check(L.nngp_loglik_f64(_p(x), _p(y), n, d, ydim, _p(nbr), m, ctypes.byref(k), 1, 1e-2, _p(ref), None,
                                 _p(ws), ws_bytes, stream), 'nngp_loglik_f64')
    want = ref.cpu().numpy()
    for _ in range(2):
        out = torch.full((1 + p.n_theta,), float('nan'), dtype=torch.float64, device='cuda')
        flags = ops.new_flags('cuda')
        _lib.check(L.nngp_loglik_f64_noalloc(_p(x), _p(y), n, d, ydim, _p(nbr), m, ctypes.byref(k), 1, _p(out),
                                             _p(flags), stream), 'nngp_loglik_f64_noalloc')
        got = out.cpu().numpy()
        assert int(flags.item()) == 0
        assert abs(got[0] / want[0] - 1) < F64_LML
        assert rel(got[1:], want[1:]) < F64_GRAD
        assert abs(got[0] / g['lml'] - 1) < F64_LML


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
