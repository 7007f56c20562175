"""Tensor-core operand layout self-test: the UMMA path of the search kernel multiplies two
128 x K matrices exactly like A @ B^T (TF32 inputs, and BF16 inputs for the d >= 12 search, that
are exactly representable, so the comparison is exact up to FP32 accumulation order)."""
import ctypes

import numpy as np
import pytest
import torch

from nngpr_b200 import _lib, ops

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('kp', [8, 16, 32])
def test_tc_layout_matches_matmul(kp):
    rng = np.random.default_rng(kp)
    # small integers scaled by powers of two: exact in TF32, exact products, exact FP32 sums
    a = (rng.integers(-8, 9, (128, kp)) * 2.0 ** rng.integers(-4, 4, (128, kp))).astype(np.float32)
    b = (rng.integers(-8, 9, (128, kp)) * 2.0 ** rng.integers(-4, 4, (128, kp))).astype(np.float32)
    ta, tb = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
    d = torch.full((128, 128), float('nan'), device='cuda')
    flags = ops.new_flags('cuda')
    L = _lib.lib()
    st = L.nngp_tc_layout_selftest(ctypes.c_void_p(ta.data_ptr()), ctypes.c_void_p(tb.data_ptr()), kp,
                                   ctypes.c_void_p(d.data_ptr()), ctypes.c_void_p(flags.data_ptr()),
                                   ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    _lib.check(st, 'nngp_tc_layout_selftest')
    got = d.cpu().numpy()
    assert int(flags.item()) == 0
    want = a.astype(np.float64) @ b.astype(np.float64).T
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-6 * np.abs(want).max())


@pytest.mark.parametrize('kp', [16, 32, 64])
def test_tc_layout_bf16_matches_matmul(kp):
    rng = np.random.default_rng(100 + kp)
    # small integers scaled by powers of two: exact in BF16 (8 significant bits), exact products
    a = (rng.integers(-8, 9, (128, kp)) * 2.0 ** rng.integers(-4, 4, (128, kp))).astype(np.float32)
    b = (rng.integers(-8, 9, (128, kp)) * 2.0 ** rng.integers(-4, 4, (128, kp))).astype(np.float32)
    ta, tb = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
    d = torch.full((128, 128), float('nan'), device='cuda')
    flags = ops.new_flags('cuda')
    L = _lib.lib()
    st = L.nngp_tc_layout_selftest_bf16(ctypes.c_void_p(ta.data_ptr()), ctypes.c_void_p(tb.data_ptr()), kp,
                                        ctypes.c_void_p(d.data_ptr()), ctypes.c_void_p(flags.data_ptr()),
                                        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    _lib.check(st, 'nngp_tc_layout_selftest_bf16')
    got = d.cpu().numpy()
    assert int(flags.item()) == 0
    want = a.astype(np.float64) @ b.astype(np.float64).T
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-6 * np.abs(want).max())
