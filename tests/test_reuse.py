"""Neighbour-list reuse across length scales (CPU): the rounding bound behind it and the
argument itself, on the oracle's arithmetic.

The bound: for the search's FP32 arithmetic, |l^2 D_l(i, j) - |x_i - x_j|^2| <= 2 (d + 6) u
(|x_i| + |x_j|)^2 at every length scale l.  The argument: when no row fails the threshold test,
ranking the candidates found at l0 gives exactly the search's lists at l.
"""
import numpy as np
import pytest

from oracle import nngp_oracle as O


@pytest.mark.parametrize('d,offset', [(1, 0.0), (3, 0.0), (3, 7.5), (8, 0.0), (16, 2.0)])
def test_rounding_bound_holds(d, offset):
    rng = np.random.default_rng(d)
    x = (rng.normal(size=(3000, d)) * rng.uniform(0.01, 3.0) + offset).astype(np.float32)
    i = rng.integers(0, 3000, 20000)
    j = rng.integers(0, 3000, 20000)
    exact = ((x[i].astype(np.float64) - x[j].astype(np.float64)) ** 2).sum(1)
    nrm = np.sqrt((x.astype(np.float64) ** 2).sum(1))
    bound = 2 * (d + 6) * O.UNIT_ROUNDOFF_F32 * (nrm[i] + nrm[j]) ** 2
    for ls in (0.013, 0.2, 0.77, 3.1, 40.0):
        xs = O.scale_for_search(x, ls)
        D = O._cand_sqdist(xs, i, j).astype(np.float64)
        l2 = float(np.float32(ls)) ** 2
        assert np.all(np.abs(l2 * D - exact) <= bound), (ls, np.max(np.abs(l2 * D - exact) / bound))


@pytest.mark.parametrize('offset', [0.0, 0.5])
def test_reused_lists_equal_the_search_when_no_row_fails(offset):
    rng = np.random.default_rng(3)
    n, m, c = 1500, 12, 20
    x = (rng.uniform(-1, 1, (n, 3)) * np.array([1.0, 0.7, 0.4]) + offset).astype(np.float32)
    ls0 = 0.2
    cand = O.knn(x, x, c, 0, ls0)
    thr = O.reuse_thresholds(x, cand, ls0, float(np.sqrt((x.astype(np.float64) ** 2).sum(1)).max()))
    for ls in (0.1, 0.19, 0.2, 0.35, 1.7):
        got, failed = O.reuse_rank(x, cand, thr, ls, m)
        assert failed == 0
        assert np.array_equal(got, O.knn(x, x, m, 0, ls))


def test_far_from_the_origin_the_test_refuses():
    """Large coordinates make the rounding bound exceed the candidate margin: the rows are
    reported, never silently accepted."""
    rng = np.random.default_rng(4)
    x = (rng.uniform(-1, 1, (800, 2)) + 3000.0).astype(np.float32)
    cand = O.knn(x, x, 12, 0, 0.05)
    thr = O.reuse_thresholds(x, cand, 0.05, float(np.sqrt((x.astype(np.float64) ** 2).sum(1)).max()))
    _, failed = O.reuse_rank(x, cand, thr, 0.07, 8)
    assert failed > 700
