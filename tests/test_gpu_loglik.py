"""Fit-step log-likelihood and gradient through the C ABI vs the oracle / golden vectors.

Tolerances: FP64 entry point 1e-10 relative (lml) and 1e-9 (gradient, max-norm relative);
FP32 entry point 1e-5 relative to |lml| and 1e-5 for the gradient (max-norm relative).
"""
import numpy as np
import pytest
import torch

from nngpr_b200 import _lib, ops
from nngpr_b200.kernel_params import extract
from oracle import nngp_oracle as O
from sklearn.gaussian_process import kernels as skk

from _common import CASES, KERNELS, lml_scale, load, normalized_y, oracle_params, rel

pytestmark = pytest.mark.gpu

F64_LML, F64_GRAD = 1e-10, 1e-9
F32_LML, F32_GRAD = 1e-5, 1e-5


def gpu_loglik(x, y, nbr, p, alpha, grad, dtype, pivot_tol=ops.DEFAULT_PIVOT_TOL):
    tdt = torch.float32 if dtype == np.float32 else torch.float64
    xt = torch.from_numpy(np.ascontiguousarray(x)).to('cuda', tdt)
    yt = torch.from_numpy(np.ascontiguousarray(y.reshape(len(y), -1))).to('cuda', tdt)
    nt = torch.from_numpy(np.ascontiguousarray(nbr, dtype=np.int32)).cuda()
    flags = ops.new_flags(xt.device)
    out = ops.loglik(xt, yt, nt, p, alpha, grad, pivot_tol, flags=flags).cpu().numpy()
    return out, int(flags.item())


@pytest.mark.parametrize('name', CASES)
@pytest.mark.parametrize('dtype', [np.float64, np.float32])
def test_loglik_golden(name, dtype):
    g = load(name)
    p = extract(KERNELS[name]().clone_with_theta(g['theta']))
    y, _, _ = normalized_y(g)
    nbr = g['nbr_fit_f32']
    out, flags = gpu_loglik(g['x'], y, nbr, p, float(g['alpha']), True, dtype)
    assert flags & ~_lib.NNGP_FLAG_FP64_FALLBACK == 0
    if dtype == np.float64:
        tol_g = F64_GRAD
        assert abs(out[0] / g['lml'] - 1) < F64_LML, (out[0], g['lml'])
    else:
        tol_g = F32_GRAD
        assert abs(out[0] - g['lml']) < F32_LML * abs(g['lml']), (out[0], g['lml'], lml_scale(name))
    assert rel(out[1:], g['grad']) < tol_g, (out[1:], g['grad'])


@pytest.mark.parametrize('dtype', [np.float64, np.float32])
def test_loglik_without_gradient(dtype):
    g = load('cpu_n2000_d3_m16')
    p = extract(KERNELS['cpu_n2000_d3_m16']().clone_with_theta(g['theta']))
    out, _ = gpu_loglik(g['x'], g['y'], g['nbr_fit_f32'], p, float(g['alpha']), False, dtype)
    assert out.shape == (1,)
    assert abs(out[0] / g['lml'] - 1) < (F64_LML if dtype == np.float64 else F32_LML)


@pytest.mark.parametrize('m', [40, 64])
def test_loglik_block_kernel_matches_oracle(m):
    """m > 32 runs the one-CTA-per-point FP64 kernel."""
    rng = np.random.default_rng(m)
    n, d = 500, 4
    x = rng.uniform(0, 1, (n, d))
    y = np.stack([np.sin(4 * x[:, 0]) + x[:, 1], np.cos(3 * x[:, 2])], 1) + rng.normal(0, 0.05, (n, 2))
    k = skk.ConstantKernel(0.8) * skk.RBF(np.array([0.3, 0.4, 0.5, 0.6])) + skk.WhiteKernel(0.02) + skk.ConstantKernel(0.1)
    p = extract(k)
    nbr = O.fit_neighbours(x, m, p.length_scale, np.float32)
    want_l, want_g = O.log_marginal_likelihood(x, y, nbr, oracle_params(p), 1e-8, True)
    for dtype, tl, tg in ((np.float64, F64_LML, F64_GRAD), (np.float32, F32_LML, F32_GRAD)):
        out, flags = gpu_loglik(x, y, nbr, p, 1e-8, True, dtype)
        assert flags == 0
        assert abs(out[0] / want_l - 1) < tl
        assert rel(out[1:], want_g) < tg


def test_loglik_subset_of_config2_vs_fp64_oracle():
    """20,000 points of the n=434,874, d=3, m=32 workload (noise 1e-3): the FP64 local
    systems match the FP64 oracle to 1e-10; FP32 systems meet 1e-5 with the default FP64
    re-solve threshold (1e-2 of the kernel diagonal, which covers the small-nugget pivots);
    a 1e-6 threshold leaves FP32 systems with sigma^2 ~ 1e-3 and an error of ~2.4e-5,
    recorded here as a bound."""
    rng = np.random.default_rng(0)
    n = 20000
    x = rng.uniform(-1, 1, (n, 3)) * np.array([1.0, 0.7, 0.4])
    y = np.sin(3 * x).sum(1) + rng.normal(0, 0.05, n)
    k = skk.ConstantKernel(1.0) * skk.RBF(0.2) + skk.WhiteKernel(1e-3)
    p = extract(k)
    nbr = O.fit_neighbours(x, 32, 0.2, np.float32)
    want_l, want_g = O.log_marginal_likelihood(x, y, nbr, oracle_params(p), 1e-10, True)
    out64, _ = gpu_loglik(x, y, nbr, p, 1e-10, True, np.float64)
    assert abs(out64[0] / want_l - 1) < F64_LML
    assert rel(out64[1:], want_g) < F64_GRAD
    out, flags = gpu_loglik(x, y, nbr, p, 1e-10, True, np.float32)
    assert flags & ~_lib.NNGP_FLAG_FP64_FALLBACK == 0
    assert abs(out[0] / want_l - 1) < F32_LML
    assert rel(out[1:], want_g) < F32_GRAD
    out, _ = gpu_loglik(x, y, nbr, p, 1e-10, True, np.float32, pivot_tol=1e-6)
    assert abs(out[0] / want_l - 1) < 1e-4


def test_fp64_fallback_on_near_singular_systems():
    """Duplicated points and a 1e-6 nugget: every local system is near singular; with the
    default FP64 re-solve threshold they are re-solved in FP64, the result stays at the FP64
    oracle's value and the status word says so."""
    rng = np.random.default_rng(4)
    base = rng.uniform(0, 1, (300, 2))
    x = np.concatenate([base, base + 1e-7])
    y = np.sin(5 * x[:, 0]) + rng.normal(0, 0.01, len(x))
    p = extract(skk.ConstantKernel(1.0) * skk.RBF(0.5) + skk.WhiteKernel(1e-6))
    nbr = O.fit_neighbours(x, 16, 0.5, np.float32)
    want_l, want_g = O.log_marginal_likelihood(x, y, nbr, oracle_params(p), 1e-10, True)
    out, flags = gpu_loglik(x, y, nbr, p, 1e-10, True, np.float32, pivot_tol=ops.DEFAULT_PIVOT_TOL)
    assert flags & _lib.NNGP_FLAG_FP64_FALLBACK
    assert abs(out[0] / want_l - 1) < F32_LML
    assert rel(out[1:], want_g) < F32_GRAD


@pytest.mark.parametrize('row_begin', [0, 3000])
@pytest.mark.parametrize('kind', ['rbf', 'matern'])
def test_every_fp32_system_resolved_in_fp64(row_begin, kind):
    """pivot_tol = 1e30 marks every FP32 system for the FP64 re-solve kernel (the fit step's FP32
    kernel carries no FP64 path; a bitmask over the launch's points hands them over).  The result
    equals the FP64 kernel on the same FP32-rounded inputs up to the order of the partial sums
    (1e-12), whole set and a row range, and the re-solve count is every system."""
    rng = np.random.default_rng(11)
    n = 8000
    x = (rng.uniform(-1, 1, (n, 3)) * np.array([1.0, 0.7, 0.4])).astype(np.float32)
    y = (np.sin(3 * x).sum(1) + rng.normal(0, 0.05, n)).astype(np.float32)
    stat = skk.RBF(0.2) if kind == 'rbf' else skk.Matern(0.3, nu=1.5)
    p = extract(skk.ConstantKernel(1.0) * stat + skk.WhiteKernel(1e-3))
    nbr_all = O.fit_neighbours(x.astype(np.float64), 32, 0.2, np.float32)
    rows = n - row_begin
    nbr = torch.from_numpy(np.ascontiguousarray(nbr_all[row_begin:], dtype=np.int32)).cuda()
    outs = {}
    for dt in (torch.float32, torch.float64):
        xt = torch.from_numpy(x).to('cuda', dt)
        yt = torch.from_numpy(y.reshape(n, 1)).to('cuda', dt)
        flags = ops.new_flags(xt.device)
        st = {}
        outs[dt] = ops.loglik(xt, yt, nbr, p, 1e-10, True, 1e30, flags=flags, row_begin=row_begin,
                              stats=st).cpu().numpy()
        f = int(flags.item())
        if dt == torch.float32:
            assert f & _lib.NNGP_FLAG_FP64_FALLBACK
            assert int(st['fp64_systems'].item()) == rows
        assert f & ~_lib.NNGP_FLAG_FP64_FALLBACK == 0
    a, b = outs[torch.float32], outs[torch.float64]
    assert abs(a[0] / b[0] - 1) < 1e-12
    assert rel(a[1:], b[1:]) < 1e-12


def test_bad_neighbour_index_is_flagged_not_read():
    g = load('const_n300_d2_m10')
    p = extract(KERNELS['const_n300_d2_m10']().clone_with_theta(g['theta']))
    nbr = g['nbr_fit_f32'].copy()
    nbr[50, 3] = 10 ** 6
    _, flags = gpu_loglik(g['x'], g['y'], nbr, p, 1e-6, True, np.float32)
    assert flags & _lib.NNGP_FLAG_BAD_INDEX
    with pytest.raises(IndexError):
        ops.raise_on_flags(flags, 'loglik')


@pytest.mark.parametrize('nu', [0.5, 1.5, 2.5])
@pytest.mark.parametrize('m', [16, 40])
def test_matern_ard_loglik_matches_oracle(nu, m):
    """ARD Matern (the reference's batched Matern cannot take ARD length scales on its batched
    input, so this is pinned by the oracle): warp kernel (m <= 32) and block kernel (m > 32)."""
    rng = np.random.default_rng(int(nu * 10) + m)
    n, d = 600, 3
    x = rng.uniform(-1, 1, (n, d))
    y = np.sin(2 * x[:, 0]) * x[:, 1] + rng.normal(0, 0.05, n)
    kernel = skk.ConstantKernel(0.8) * skk.Matern(np.array([0.4, 0.9, 1.7]), nu=nu) + skk.WhiteKernel(0.02)
    p = extract(kernel)
    nbr = O.knn(x, x, m, 0, p.length_scale)
    want_l, want_g = O.log_marginal_likelihood(x, y[:, None], nbr, oracle_params(p), 1e-10, True)
    out, flags = gpu_loglik(x, y, nbr, p, 1e-10, True, np.float64)
    assert flags == 0
    assert abs(out[0] / want_l - 1) < F64_LML
    assert rel(out[1:], want_g) < F64_GRAD
    out32, flags32 = gpu_loglik(x, y, nbr, p, 1e-10, True, np.float32)
    assert flags32 & ~_lib.NNGP_FLAG_FP64_FALLBACK == 0
    assert abs(out32[0] / want_l - 1) < F32_LML
    assert rel(out32[1:], want_g) < F32_GRAD


def test_row_shards_sum_to_the_whole_step():
    """The multi-GPU fit step's per-rank call: ops.loglik(..., row_begin=r0) on each row range of
    a partition (nngp_loglik_rows_*, one task of the reference's row-batched worker loop,
    base_nngpr.py:503-538) sums to the single launch and to the FP64 oracle, FP64 and FP32."""
    rng = np.random.default_rng(11)
    n = 20000
    x = rng.uniform(-1, 1, (n, 3)) * np.array([1.0, 0.7, 0.4])
    y = np.sin(3 * x).sum(1) + rng.normal(0, 0.05, n)
    p = extract(skk.ConstantKernel(1.0) * skk.RBF(0.2) + skk.WhiteKernel(1e-3))
    nbr = O.fit_neighbours(x, 32, 0.2, np.float32)
    want_l, want_g = O.log_marginal_likelihood(x, y, nbr, oracle_params(p), 1e-10, True)
    bounds = [0, 1, 4999, 12000, 19999, n]  # a one-row shard and the last row alone included
    for dtype, tdt, tl, tg in ((np.float64, torch.float64, F64_LML, F64_GRAD),
                               (np.float32, torch.float32, F32_LML, F32_GRAD)):
        xt = torch.from_numpy(x).to('cuda', tdt)
        yt = torch.from_numpy(y[:, None]).to('cuda', tdt)
        nt = torch.from_numpy(nbr).cuda()
        whole = ops.loglik(xt, yt, nt, p, 1e-10, True).cpu().numpy()
        parts = np.zeros_like(whole)
        for r0, r1 in zip(bounds[:-1], bounds[1:]):
            flags = ops.new_flags(xt.device)
            part = ops.loglik(xt, yt, nt[r0:r1].contiguous(), p, 1e-10, True, flags=flags, row_begin=r0)
            assert int(flags.item()) & ~_lib.NNGP_FLAG_FP64_FALLBACK == 0
            parts += part.cpu().numpy()
        assert abs(parts[0] / whole[0] - 1) < 1e-12
        assert rel(parts[1:], whole[1:]) < 1e-11
        assert abs(parts[0] / want_l - 1) < tl
        assert rel(parts[1:], want_g) < tg


def test_fit_step_rows_shards_equal_the_whole_step():
    """sharding.fit_step_rows, what one rank of the multi-GPU step runs (its rows' seeded and
    pruned search against the prefix, then their local systems), over three shards run one after
    the other on this GPU: the partial sums add up to the single-GPU fit step."""
    from nngpr_b200.sharding import fit_step_rows, row_partition
    rng = np.random.default_rng(12)
    n = 100_000
    x = rng.uniform(-1, 1, (n, 3)) * np.array([1.0, 0.7, 0.4])
    y = np.sin(3 * x).sum(1) + rng.normal(0, 0.05, n)
    p = extract(skk.ConstantKernel(1.0) * skk.RBF(0.2) + skk.WhiteKernel(1e-3))
    x64 = torch.from_numpy(x).cuda()
    y64 = torch.from_numpy(y[:, None]).cuda()
    x32 = x64.to(torch.float32)
    nbr = ops.knn(x32, x32, 32, 0, 0.2)
    whole = ops.loglik(x64, y64, nbr, p, 1e-10, True).cpu().numpy()
    for equal_rows in (True, False):
        b = row_partition(n, 3, equal_rows=equal_rows)
        parts = np.zeros_like(whole)
        for r0, r1 in zip(b[:-1], b[1:]):
            flags = ops.new_flags(x64.device)
            parts += fit_step_rows(x32, x64, y64, p, 1e-10, 32, r0, r1, 0.2, flags=flags).cpu().numpy()
            assert int(flags.item()) == 0
        assert abs(parts[0] / whole[0] - 1) < 1e-12
        assert rel(parts[1:], whole[1:]) < 1e-11
