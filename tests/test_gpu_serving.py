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
