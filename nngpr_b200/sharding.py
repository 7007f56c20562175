"""Row sharding of one fit step across ranks (one process per GPU).

The fit-step log-likelihood is a sum over points, and point i's term depends only on X, y
and its neighbours among points [0, i) (``base_nngpr.py:453-614``).  A rank therefore owns a
contiguous row range: it searches its rows against the prefix (``ref_cut_index = row_begin``,
the reference's own batching rule, ``base_nngpr.py:530-535``), solves their local systems
(``nngp_loglik_rows_*``) and contributes a (1 + n_theta) partial sum; one all-reduce per step
gives every rank the full value and gradient.  X and y are replicated.

Rows are split so that the prefix-search pair counts (row i scans i refs) are equal:
rank r owns ``[n sqrt(r / R), n sqrt((r + 1) / R))`` (``row_partition``), the right split when
the search cost grows with the prefix.  When the library prunes the search (FP32, d <= 24,
65,536 <= n <= 2,000,000, see ``search_is_pruned``) a row costs about the same wherever it is
(its tile list covers its neighbourhood, not its prefix), and so do the local systems: equal row
counts balance the ranks (``row_partition(..., equal_rows=True)``).
"""

from __future__ import annotations

import math


def search_is_pruned(n: int, d: int, float32: bool = True) -> bool:
    """Whether the library's fit-step search of n points in d dimensions is pruned."""
    return float32 and d <= 24 and 65536 <= n <= 2_000_000


def row_partition(n: int, world: int, equal_rows: bool = False) -> list[int]:
    """Boundaries ``b[0] = 0 <= b[1] <= ... <= b[world] = n`` with equal pair counts (or, with
    ``equal_rows``, equal row counts)."""
    if world < 1:
        raise ValueError('world must be >= 1')
    if equal_rows:
        return [n * r // world for r in range(world + 1)]
    b = [int(round(n * math.sqrt(r / world))) for r in range(world + 1)]
    b[0], b[-1] = 0, n
    for r in range(1, world + 1):
        b[r] = max(b[r], b[r - 1])
    return b


def rebalance(bounds: list[int], seconds: list[float]) -> list[int]:
    """A partition of the same rows with equal predicted time per rank, from the time each rank
    took on its current range (``seconds[r]`` for ``[bounds[r], bounds[r + 1])``, e.g. the device
    time of one fit step, gathered from every rank).

    The cost of a row is taken as uniform inside each current range (that range's time over its
    rows), so the cumulative cost is piecewise linear in the row index; the new boundaries cut it
    into equal parts.  This balances what the static rules cannot see: a shard whose tile lists
    fell back to index order on the device, or one whose rows are costlier for the data at hand.
    """
    world = len(bounds) - 1
    if world < 1 or len(seconds) != world:
        raise ValueError('one time per range')
    n = bounds[-1]
    t = [max(float(s), 0.0) for s in seconds]
    total = sum(t)
    if total <= 0.0 or n == 0:
        return list(bounds)
    cum = [0.0]
    for v in t:
        cum.append(cum[-1] + v)
    out = [0]
    r = 0
    for k in range(1, world):
        target = total * k / world
        while r < world - 1 and cum[r + 1] < target:
            r += 1
        lo, hi = bounds[r], bounds[r + 1]
        frac = (target - cum[r]) / t[r] if t[r] > 0 else 0.0
        out.append(max(out[-1], min(n, int(round(lo + frac * (hi - lo))))))
    out.append(n)
    return out


def prefix_pairs(r0: int, r1: int) -> int:
    """Prefix-search pairs of rows [r0, r1): sum of i for i in [r0, r1)."""
    return (r1 * (r1 - 1) - r0 * (r0 - 1)) // 2


def fit_step_rows(x_search, x, y, p, alpha, num_nn, row_begin, row_end, length_scale, eval_gradient=True,
                  pivot_tol=None, flags=None, out=None):
    """This rank's partial [lml, grad...] of one fit step on the device (torch tensors).

    ``x_search`` is the search copy of X (float32 for the default precision), ``x``/``y`` the
    local-system copies; rows ``[row_begin, row_end)``.  The caller all-reduces the result.
    """
    from . import ops
    q = x_search[row_begin:row_end]
    m = min(num_nn, max(x_search.shape[0] - 1, 0))
    nbr = ops.knn(x_search, q, m, row_begin, length_scale, flags=flags)
    kw = {} if pivot_tol is None else {'pivot_tol': pivot_tol}
    return ops.loglik(x, y, nbr, p, alpha, eval_gradient, flags=flags, out=out, row_begin=row_begin, **kw)
