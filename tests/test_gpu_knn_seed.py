"""Seeded prefix search: the fit step's search (ref = query, cut 0) starts every row from a
proven upper bound of its m-th distance, taken from the row's neighbours along two Morton
orders.  The lists must be bit-identical to the unseeded search (NNGP_KNN_SEED_W=0) and to the
oracle; only the amount of candidate work changes."""
import numpy as np
import pytest
import torch

from nngpr_b200 import ops
from oracle import nngp_oracle as O

pytestmark = pytest.mark.gpu


def search(monkeypatch, x, m, ls, window):
    monkeypatch.setenv('NNGP_KNN_SEED_W', str(window))
    t = torch.from_numpy(np.ascontiguousarray(x, dtype=np.float32)).cuda()
    flags = ops.new_flags(t.device)
    out = ops.knn(t, t, m, 0, ls, flags=flags)
    assert int(flags.item()) == 0
    return out.cpu().numpy()


def check_rows(x, got, m, ls, rng, k=200):
    rows = np.sort(rng.choice(x.shape[0], k, replace=False))
    rows = np.union1d(rows, np.arange(x.shape[0] - 50, x.shape[0]))  # the longest rows too
    want = O.knn(x, x[rows], m, 0, ls, query_index=rows)
    assert np.array_equal(got[rows], want)


@pytest.mark.parametrize('d', [1, 2, 3, 5, 8, 12, 16, 20, 24])
@pytest.mark.parametrize('m', [1, 16, 32])
def test_seeded_lists_equal_unseeded_and_oracle(monkeypatch, d, m):
    rng = np.random.default_rng(1000 * d + m)
    n = 20000
    x = rng.uniform(-1, 1, (n, d))
    ls = rng.uniform(0.3, 2.0, d) if d % 2 else 0.4
    plain = search(monkeypatch, x, m, ls, 0)
    for w in (128, 256):
        assert np.array_equal(search(monkeypatch, x, m, ls, w), plain)
    check_rows(x, plain, m, ls, rng)


def test_seeded_ties_duplicates_outlier_and_clusters(monkeypatch):
    """Integer lattice with many duplicates (exact ties, lower index first); one far outlier
    that squeezes every other point into a few Morton cells; a 16-d Gaussian mixture."""
    rng = np.random.default_rng(3)
    x = rng.integers(0, 6, (30000, 3)).astype(np.float64)
    a = search(monkeypatch, x, 32, None, 256)
    assert np.array_equal(a, search(monkeypatch, x, 32, None, 0))
    check_rows(x, a, 32, None, rng)
    y = rng.normal(size=(25000, 3))
    y[12345] = 1e6
    b = search(monkeypatch, y, 16, 0.5, 256)
    assert np.array_equal(b, search(monkeypatch, y, 16, 0.5, 0))
    check_rows(y, b, 16, 0.5, rng)
    means = rng.uniform(-3, 3, (64, 16))
    z = means[rng.integers(0, 64, 30000)] + 0.5 * rng.normal(size=(30000, 16))
    c = search(monkeypatch, z, 32, 0.8, 256)
    assert np.array_equal(c, search(monkeypatch, z, 32, 0.8, 0))
    check_rows(z, c, 32, 0.8, rng, k=100)


def test_seeding_engages_only_on_the_prefix_self_search(monkeypatch, capfd):
    monkeypatch.setenv('NNGP_KNN_DEBUG', '1')
    rng = np.random.default_rng(4)
    x = rng.uniform(0, 1, (20000, 3))
    search(monkeypatch, x, 32, 0.3, 256)
    assert 'seeded=1' in capfd.readouterr().err
    search(monkeypatch, x, 32, 0.3, 0)
    assert 'seeded=0' in capfd.readouterr().err
    monkeypatch.setenv('NNGP_KNN_SEED_W', '256')
    t = torch.from_numpy(x.astype(np.float32)).cuda()
    ops.knn(t, t[:5000].clone(), 32, None, 0.3)  # predict-style search: no seeds
    assert 'seeded=0' in capfd.readouterr().err
    small = torch.from_numpy(x[:5000].astype(np.float32)).cuda()
    ops.knn(small, small, 32, 0, 0.3)  # below the size where seeding pays
    assert 'seeded=0' in capfd.readouterr().err


def search_mode(monkeypatch, x, m, ls, prune):
    monkeypatch.setenv('NNGP_KNN_PRUNE', '1' if prune else '0')
    return search(monkeypatch, x, m, ls, 128)


@pytest.mark.parametrize('d', [1, 2, 3, 5, 8, 16, 24])
@pytest.mark.parametrize('m', [1, 32])
def test_pruned_lists_equal_unpruned_and_oracle(monkeypatch, d, m):
    """n >= 65,536: groups of rows visit only the ref tiles their seeds allow (bounding boxes
    along the curve order); the lists stay bit-identical."""
    rng = np.random.default_rng(50 * d + m)
    n = 70000
    x = rng.uniform(-1, 1, (n, d)) * rng.uniform(0.3, 1.0, d)
    ls = rng.uniform(0.3, 2.0, d) if d % 2 else 0.4
    a = search_mode(monkeypatch, x, m, ls, True)
    assert np.array_equal(a, search_mode(monkeypatch, x, m, ls, False))
    check_rows(x, a, m, ls, rng, k=150)


def test_pruned_ties_outlier_and_clusters(monkeypatch, capfd):
    rng = np.random.default_rng(9)
    lattice = rng.integers(0, 8, (80000, 3)).astype(np.float64)  # duplicates: exact ties
    monkeypatch.setenv('NNGP_KNN_DEBUG', '1')
    a = search_mode(monkeypatch, lattice, 32, None, True)
    assert 'pruned=1' in capfd.readouterr().err
    assert np.array_equal(a, search_mode(monkeypatch, lattice, 32, None, False))
    check_rows(lattice, a, 32, None, rng, k=100)
    y = rng.normal(size=(70000, 3))
    y[33333] = [1e7, -1e7, 5e6]  # squeezes the other points into a few curve cells
    b = search_mode(monkeypatch, y, 16, 0.5, True)
    assert np.array_equal(b, search_mode(monkeypatch, y, 16, 0.5, False))
    check_rows(y, b, 16, 0.5, rng, k=100)
    means = rng.uniform(-3, 3, (64, 16))
    z = means[rng.integers(0, 64, 70000)] + 0.5 * rng.normal(size=(70000, 16))
    c = search_mode(monkeypatch, z, 32, 0.8, True)
    assert np.array_equal(c, search_mode(monkeypatch, z, 32, 0.8, False))
    check_rows(z, c, 32, 0.8, rng, k=80)


def test_split_work_items_merge_to_the_same_lists(monkeypatch, capfd):
    """An outlier squeezes the other points into one Morton cell: seeds come from random windows
    and groups need most tiles, so long tile ranges are split into several work items whose
    partial lists are merged (in whichever launch takes the rows); the result equals the
    unpruned search and the oracle."""
    import re
    rng = np.random.default_rng(21)
    y = rng.normal(size=(90000, 3))
    y[777] = [3e7, 3e7, -3e7]
    monkeypatch.setenv('NNGP_KNN_DEBUG', '1')
    a = search_mode(monkeypatch, y, 32, 0.5, True)
    err = capfd.readouterr().err
    mt = re.search(r'pruned rows=(\d+) groups=(\d+) items=(\d+) .* index-order rows=(\d+) items=(\d+)', err)
    assert mt
    _, pg, pi, ir, ii = map(int, mt.groups())
    # some groups were split: in the pruned launch, or in the index-order launch (128-row groups)
    # when the lists fall back to index order
    assert pi > pg or ii > -(-ir // 128)
    assert np.array_equal(a, search_mode(monkeypatch, y, 32, 0.5, False))
    check_rows(y, a, 32, 0.5, rng, k=100)


def query_search(monkeypatch, ref, q, m, ls, window, prune=True):
    monkeypatch.setenv('NNGP_KNN_SEED_W', str(window))
    monkeypatch.setenv('NNGP_KNN_PRUNE', '1' if prune else '0')
    r = torch.from_numpy(np.ascontiguousarray(ref, dtype=np.float32)).cuda()
    qq = torch.from_numpy(np.ascontiguousarray(q, dtype=np.float32)).cuda()
    flags = ops.new_flags(r.device)
    out = ops.knn(r, qq, m, None, ls, flags=flags)
    assert int(flags.item()) == 0
    return out.cpu().numpy()


@pytest.mark.parametrize('d,n_ref,n_query', [(2, 70000, 20000), (3, 70000, 100000), (4, 30000, 40000),
                                             (5, 30000, 20000), (16, 20000, 30000), (8, 70000, 30000),
                                             (16, 70000, 20000)])
def test_query_search_seeded_and_pruned_equal_plain_and_oracle(monkeypatch, d, n_ref, n_query):
    """Queries against a set (the predict search): seeds from the refs' curve windows around each
    query and curve-ordered query groups with tile lists; the same lists."""
    rng = np.random.default_rng(7 * d + n_query)
    ref = rng.uniform(-1, 1, (n_ref, d))
    q = rng.uniform(-1.2, 1.2, (n_query, d))  # some queries outside the refs' box
    ls = rng.uniform(0.3, 2.0, d) if d % 2 else 0.35
    plain = query_search(monkeypatch, ref, q, 32, ls, 0)
    assert np.array_equal(query_search(monkeypatch, ref, q, 32, ls, 128), plain)
    assert np.array_equal(query_search(monkeypatch, ref, q, 32, ls, 128, prune=False), plain)
    rows = np.sort(rng.choice(n_query, 150, replace=False))
    assert np.array_equal(plain[rows], O.knn(ref, q[rows], 32, None, ls))


def test_query_search_engages_and_handles_duplicates_and_outliers(monkeypatch, capfd):
    rng = np.random.default_rng(5)
    ref = rng.integers(0, 10, (70000, 3)).astype(np.float64)  # many exact ties
    ref[123] = [5e6, 5e6, 5e6]
    q = rng.integers(0, 10, (30000, 3)).astype(np.float64)
    q[77] = [-4e6, 0, 0]
    monkeypatch.setenv('NNGP_KNN_DEBUG', '1')
    a = query_search(monkeypatch, ref, q, 16, None, 128)
    err = capfd.readouterr().err
    assert 'seeded=1 pruned=1' in err
    b = query_search(monkeypatch, ref, q, 16, None, 0)
    assert np.array_equal(a, b)
    rows = np.sort(np.r_[77, rng.choice(30000, 100, replace=False)])
    assert np.array_equal(a[rows], O.knn(ref, q[rows], 16, None, None))


@pytest.mark.parametrize('d', [3, 8])
def test_row_shards_of_the_prefix_search(monkeypatch, capfd, d):
    """The multi-GPU fit step searches row shards: query = rows [r0, r1) of the set as a view,
    ref_cut_index = r0.  Shards are seeded and pruned over their own rows and
    equal the corresponding rows of the whole search."""
    rng = np.random.default_rng(40 + d)
    n = 100000
    x = rng.uniform(-1, 1, (n, d))
    ls = 0.3
    monkeypatch.setenv('NNGP_KNN_SEED_W', '128')
    monkeypatch.setenv('NNGP_KNN_PRUNE', '1')
    t = torch.from_numpy(x.astype(np.float32)).cuda()
    full = ops.knn(t, t, 32, 0, ls).cpu().numpy()
    monkeypatch.setenv('NNGP_KNN_DEBUG', '1')
    for r0, r1 in [(0, 30000), (30000, 71000), (71000, n)]:
        got = ops.knn(t, t[r0:r1], 32, r0, ls).cpu().numpy()
        err = capfd.readouterr().err
        assert 'seeded=1' in err and 'pruned=1' in err
        assert np.array_equal(got, full[r0:r1])
    monkeypatch.setenv('NNGP_KNN_SEED_W', '0')
    np.testing.assert_array_equal(ops.knn(t, t[50000:60000], 32, 50000, ls).cpu().numpy(), full[50000:60000])


def test_index_order_fallback_when_boxes_do_not_prune(monkeypatch, capfd):
    """Uniform points in 24 dimensions: every group's box meets nearly every tile's, so the tile
    lists would stream more tiles than index order; the search puts every row back in index order
    (the pruned launch is empty).  Whole set and row shards equal the unpruned search; 3-d points
    keep their pruned rows."""
    rng = np.random.default_rng(77)
    n = 100000
    x = rng.uniform(-1, 1, (n, 24))
    monkeypatch.setenv('NNGP_KNN_DEBUG', '1')
    a = search_mode(monkeypatch, x, 32, 0.5, True)
    assert 'pruned rows=0 ' in capfd.readouterr().err
    assert np.array_equal(a, search_mode(monkeypatch, x, 32, 0.5, False))
    check_rows(x, a, 32, 0.5, rng, k=60)
    monkeypatch.setenv('NNGP_KNN_PRUNE', '1')
    t = torch.from_numpy(x.astype(np.float32)).cuda()
    for r0, r1 in [(0, 40000), (40000, n)]:
        got = ops.knn(t, t[r0:r1], 32, r0, 0.5).cpu().numpy()
        assert 'pruned rows=0 ' in capfd.readouterr().err
        assert np.array_equal(got, a[r0:r1])
    y = rng.uniform(-1, 1, (n, 3))
    search_mode(monkeypatch, y, 32, 0.3, True)
    err = capfd.readouterr().err
    assert 'pruned rows=' in err and 'pruned rows=0 ' not in err
