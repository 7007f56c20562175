"""Continuous-batching predict server: each request's result equals the estimator's predict on
the same points, alone or batched with others (bit for bit: every query row is computed
independently), with and without CUDA graphs, including requests split across batches."""
import threading

import numpy as np
import pytest
from sklearn.gaussian_process import kernels as skk

from nngpr_b200 import B200Nngpr
from nngpr_b200.serving import PredictServer

pytestmark = pytest.mark.gpu


def _model(n=3000, d=18, seed=0):
    rng = np.random.default_rng(seed)
    x = rng.normal(size=(n, d))
    ls = np.exp(rng.uniform(np.log(0.5), np.log(5.0), d))
    y = np.sin(x @ (rng.normal(size=d) / ls)) + 0.1 * rng.normal(size=n)
    kernel = skk.ConstantKernel(1.0) * skk.RBF(ls) + skk.WhiteKernel(1e-2)
    return B200Nngpr(kernel=kernel, num_nn=32, optimizer=None, normalize_y=True).fit(x, y), rng


def test_server_equals_estimator_predict():
    gpr, rng = _model()
    xq = rng.normal(size=(777, 18))
    want_mean, want_std = gpr.predict(xq, return_std=True)
    with PredictServer(gpr, buckets=(64, 256, 1024), slots=2) as srv:
        mean, std = srv.predict(xq)
    np.testing.assert_array_equal(mean, want_mean)
    np.testing.assert_array_equal(std, want_std)


@pytest.mark.parametrize('use_graphs', [True, False])
def test_alone_equals_in_the_mix(use_graphs):
    gpr, rng = _model(seed=1)
    sizes = [1, 5, 64, 65, 300, 1024, 1500, 3000, 7, 2]  # 1500 and 3000 span several batches
    reqs = [rng.normal(size=(s, 18)) for s in sizes]
    with PredictServer(gpr, buckets=(64, 256, 1024), slots=3, use_graphs=use_graphs) as srv:
        alone = [srv.predict(r) for r in reqs]
        futures = [None] * len(reqs)

        def client(k):
            futures[k] = srv.submit(reqs[k])

        threads = [threading.Thread(target=client, args=(k,)) for k in range(len(reqs))]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        mixed = [f.result(timeout=60) for f in futures]
    for (ma, sa), (mm, sm) in zip(alone, mixed):
        np.testing.assert_array_equal(ma, mm)
        np.testing.assert_array_equal(sa, sm)
    want_mean, want_std = gpr.predict(reqs[7], return_std=True)
    np.testing.assert_array_equal(mixed[7][0], want_mean)
    np.testing.assert_array_equal(mixed[7][1], want_std)


def test_empty_request_and_latency_record():
    gpr, rng = _model(n=500, seed=2)
    with PredictServer(gpr, buckets=(128,), slots=1) as srv:
        mean, std = srv.predict(np.zeros((0, 18)))
        assert mean.shape == (0,) and std.shape == (0,)
        srv.predict(rng.normal(size=(10, 18)))
        assert len(srv.completed) == 2 and all(t >= 0 for t in srv.completed)


def test_mixed_stream_equals_the_oracle():
    """Requests submitted concurrently from several client threads (batched together, split
    across batches): every result equals the CPU oracle's predict (the reference's _predict_worker
    restated, base_nngpr.py:1032-1135) on the oracle's own exact neighbour lists, FP64 systems, to
    1e-9 relative."""
    from nngpr_b200.kernel_params import extract
    from oracle import nngp_oracle as O

    from _common import oracle_params
    gpr, rng = _model(seed=3)
    x = np.asarray(gpr.X_train_)
    y = np.asarray(gpr.y_train_).reshape(len(x), -1)  # normalised, as the fitted model holds it
    p = extract(gpr.kernel_)
    sizes = [3, 700, 64, 2500, 1, 130]
    reqs = [rng.normal(size=(s, 18)) for s in sizes]
    futures = [None] * len(reqs)
    with PredictServer(gpr, buckets=(64, 256, 1024), slots=3) as srv:
        threads = [threading.Thread(target=lambda k=k: futures.__setitem__(k, srv.submit(reqs[k])))
                   for k in range(len(reqs))]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        got = [f.result(timeout=60) for f in futures]
    for xq, (mean, std) in zip(reqs, got):
        nbr = O.knn(x, xq, 32, None, p.length_scale)
        wm, ws = O.predict(x, y, xq, nbr, oracle_params(p), float(gpr.alpha))
        wm = wm[:, 0] * gpr._y_train_std + gpr._y_train_mean
        ws = ws * gpr._y_train_std
        assert np.max(np.abs(mean - wm)) <= 1e-9 * np.max(np.abs(wm))
        assert np.max(np.abs(std - ws)) <= 1e-9 * np.max(np.abs(ws))


def test_slots_are_added_when_memory_allows_and_refused_when_it_does_not():
    """Free-memory admission: starting from one slot, a burst of concurrent requests makes the
    server add slots (up to max) while the free device memory holds them; with a budget of one
    slot it never adds one.  Every result still equals the estimator's predict."""
    gpr, rng = _model(seed=4)
    reqs = [rng.normal(size=(int(s), 18)) for s in rng.integers(200, 3000, 24)]
    want = [gpr.predict(r, return_std=True) for r in reqs]
    for budget, grows in ((None, True), ('one', False)):
        kw = dict(buckets=(256, 1024), slots=3, min_slots=1)
        with PredictServer(gpr, **kw) as probe:
            one = probe.slot_bytes
        if budget == 'one':
            kw['memory_budget'] = one
        with PredictServer(gpr, **kw) as srv:
            assert srv.n_slots == 1
            futs = [srv.submit(r) for r in reqs]
            got = [f.result(timeout=120) for f in futs]
            if grows:
                assert srv.n_slots > 1 and srv.slots_added == srv.n_slots - 1
            else:
                assert srv.n_slots == 1 and srv.slots_added == 0 and srv.slots_refused > 0
        for (m, s), (wm, ws) in zip(got, want):
            np.testing.assert_array_equal(m, wm)
            np.testing.assert_array_equal(s, ws)
