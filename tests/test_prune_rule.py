"""The exactness margin of the pruned search's tile rule, checked in IEEE float32 on the CPU.

A ref tile is dropped for a group of rows only if

    lb * (1 - gamma) - 1e-37 > seed,   lb = sum_f gap_f^2 (double, from the float32 box bounds),
    gamma = (d + 3) * 2^-23,

so the rule is exact if every pair (query q in the group's box, ref r in the tile's box) has an
FP32 squared distance, computed the way the search rescores candidates (t_f = fl(r_f - q_f),
acc = fl(acc + fl(t_f * t_f)) feature by feature), of at least lb * (1 - gamma) - 1e-37.  The
closest pairs (points on the facing box faces) are the tight case; magnitudes from subnormal to
1e18 and separations from 1e-30 to 1e6 cover the rounding regimes.
"""
import numpy as np


def fp32_sqdist(q, r):
    """The search's exact rescoring arithmetic, in float32 (numpy rounds every operation)."""
    q = q.astype(np.float32)
    r = r.astype(np.float32)
    acc = np.zeros(q.shape[:-1], dtype=np.float32)
    for f in range(q.shape[-1]):
        t = (r[..., f] - q[..., f]).astype(np.float32)
        acc = (acc + (t * t).astype(np.float32)).astype(np.float32)
    return acc


def box_bound(glo, ghi, tlo, thi):
    """lb of the rule: squared box distance in double from the float32 bounds (NaN gaps -> 0)."""
    gap = np.fmax(0.0, np.fmax(tlo.astype(np.float64) - ghi.astype(np.float64),
                               glo.astype(np.float64) - thi.astype(np.float64)))
    return (gap * gap).sum(-1)


def test_tile_rule_never_exceeds_the_fp32_distance():
    rng = np.random.default_rng(11)
    worst = np.inf
    for d in (1, 2, 3, 4):
        gamma = (d + 3) * 2.0 ** -23
        for center_scale in (0.0, 1e-20, 1.0, 1e3, 1e12, 1e18):
            for sep in (1e-30, 1e-20, 1e-6, 1e-2, 1.0, 1e3, 1e6):
                n = 4000
                c = rng.normal(size=(n, d)) * center_scale
                # group box [c, c + w1] and tile box [c + w1 + sep * u, ... + w2], per feature
                w1 = np.abs(rng.normal(size=(n, d))) * sep * rng.uniform(0, 3)
                u = rng.uniform(0.0, 1.5, size=(n, d))
                side = rng.choice([-1.0, 1.0], size=(n, d))
                glo = c.astype(np.float32)
                ghi = (c + w1).astype(np.float32)
                gap = sep * u
                tlo = np.where(side > 0, ghi.astype(np.float64) + gap, glo.astype(np.float64) - gap - w1)
                thi = np.where(side > 0, tlo + w1, glo.astype(np.float64) - gap)
                tlo, thi = tlo.astype(np.float32), thi.astype(np.float32)
                tlo, thi = np.minimum(tlo, thi), np.maximum(tlo, thi)
                lb = box_bound(glo, ghi, tlo, thi)
                # the closest pair on the facing faces, and random pairs inside the boxes
                q_face = np.where(side > 0, ghi, glo)
                r_face = np.where(side > 0, tlo, thi)
                qs = [q_face, (glo + (ghi - glo) * rng.uniform(size=(n, d))).astype(np.float32)]
                rs = [r_face, (tlo + (thi - tlo) * rng.uniform(size=(n, d))).astype(np.float32)]
                for q, r in zip(qs, rs):
                    q = np.clip(q, glo, ghi)
                    r = np.clip(r, tlo, thi)
                    d2 = fp32_sqdist(q, r).astype(np.float64)
                    slack = d2 - (lb * (1.0 - gamma) - 1e-37)
                    finite = np.isfinite(d2) & np.isfinite(lb)
                    assert np.all(slack[finite] >= 0.0), (d, center_scale, sep, slack[finite].min())
                    big = finite & (lb > 1e-30)  # below, underflow is what the 1e-37 term covers
                    if big.any():
                        worst = min(worst, float((d2[big] / lb[big]).min()))
    assert worst > 0.999  # in the normal range the FP32 distance stays within rounding of the bound


def test_dropped_tiles_hold_no_neighbour_of_any_row():
    """End to end on a small set: groups and tiles along a sort order, seeds = the m-th smallest
    FP32 distance over a window of earlier points; every tile the rule drops holds no ref of any
    row's true top-m (nor a ref tied with its m-th distance)."""
    rng = np.random.default_rng(3)
    n, d, m, G, T = 6000, 3, 16, 128, 128
    x = (rng.uniform(-1, 1, (n, d)) / 0.2).astype(np.float32)
    order = np.lexsort(x.T[::-1])  # any spatial order works for the argument
    tiles = [order[k:k + T] for k in range(0, n, T)]
    gamma = (d + 3) * 2.0 ** -23
    dropped = kept = 0
    pos = np.empty(n, dtype=np.int64)
    pos[order] = np.arange(n)
    rows = np.arange(n // 2, n)
    rows = rows[np.argsort(pos[rows], kind='stable')]  # groups of rows along the same order
    for g0 in range(0, rows.size, G):
        grp = rows[g0:g0 + G]
        seeds = []
        for i in grp:
            win = np.arange(max(0, i - 600), i)
            d2 = fp32_sqdist(np.broadcast_to(x[i], (win.size, d)), x[win])
            seeds.append(np.partition(d2, m - 1)[m - 1])
        tau = float(max(seeds))
        glo, ghi = x[grp].min(0), x[grp].max(0)
        lim = grp.max()
        true_refs = set()
        for i in grp:
            d2 = fp32_sqdist(np.broadcast_to(x[i], (i, d)), x[:i])
            kth = np.partition(d2, m - 1)[m - 1]
            true_refs.update(np.nonzero(d2 <= kth)[0].tolist())
        for t in tiles:
            lb = box_bound(glo, ghi, x[t].min(0), x[t].max(0))
            drop = t.min() >= lim or lb * (1.0 - gamma) - 1e-37 > tau
            if drop:
                dropped += 1
                assert not true_refs.intersection(t.tolist())
            else:
                kept += 1
    assert dropped > 0.25 * (dropped + kept)  # the rule does prune (slab tiles of a sort order here)


def _rd(x):
    """x (float64 array, the exact result of one FP32 operation) rounded to FP32 toward -inf."""
    f = x.astype(np.float32)
    lower = f.astype(np.float64) > x
    f[lower] = np.nextafter(f[lower], np.float32(-np.inf))
    return f


def test_round_down_box_bound_never_exceeds_the_exact_bound():
    """The search planning evaluates the rule's left side in FP32 rounded toward -inf (every
    operation: gap, square, sum, shrink, minus 1e-37).  Emulated here operation by operation
    (each FP32 operation's exact value is a float64 sum / product of floats, rounded down), the
    result never exceeds the exact left side, so whatever the FP32 form drops the exact rule
    drops too."""
    rng = np.random.default_rng(5)
    for d in (1, 3, 8, 16, 24):
        shrink = np.float32(1.0 - (d + 3) * 2.0 ** -23)
        for scale in (1e-20, 1.0, 1e6, 1e18):
            n = 5000
            glo = (rng.normal(size=(n, d)) * scale).astype(np.float32)
            ghi = (glo + np.abs(rng.normal(size=(n, d))) * scale).astype(np.float32)
            tlo = (rng.normal(size=(n, d)) * scale * 3).astype(np.float32)
            thi = (tlo + np.abs(rng.normal(size=(n, d))) * scale).astype(np.float32)
            lb = np.zeros(n, dtype=np.float32)
            for f in range(d):
                a = _rd(tlo[:, f].astype(np.float64) - ghi[:, f].astype(np.float64))
                b = _rd(glo[:, f].astype(np.float64) - thi[:, f].astype(np.float64))
                gap = np.maximum(np.float32(0), np.maximum(a, b))
                sq = _rd(gap.astype(np.float64) * gap.astype(np.float64))
                lb = _rd(lb.astype(np.float64) + sq.astype(np.float64))
            lhs = _rd(_rd(lb.astype(np.float64) * np.float64(shrink)).astype(np.float64) - 1e-37)
            exact = box_bound(glo, ghi, tlo, thi) * (1.0 - (d + 3) * 2.0 ** -23) - 1e-37
            ok = np.isfinite(exact)
            assert np.all(lhs.astype(np.float64)[ok] <= exact[ok]), (d, scale)

