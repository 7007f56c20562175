"""Failure detection on the GPU without a fault: every wait inside the tensor-core search is
bounded, and a wait that runs out makes the kernel raise NNGP_FLAG_TIMEOUT, drain the copies and
MMAs it issued, free its tensor memory and return.  Here nothing is broken: the wait limit of the
search's main loop is set to 1 ns (nngp_set_wait_limit_ns), so the first wait that has to wait
at all gives up.  The test checks that the call returns with the flag set, that the host turns
the flag into an exception, and that the next call, with the default limit, runs on the same
context and returns the exact lists."""
import numpy as np
import pytest
import torch

from nngpr_b200 import _lib, ops
from oracle import nngp_oracle as O

pytestmark = pytest.mark.gpu


def _gmm(n=20000, d=16, seed=3):
    rng = np.random.default_rng(seed)
    means = rng.uniform(-3, 3, (8, d))
    return means[rng.integers(0, 8, n)] + 0.5 * rng.normal(size=(n, d))


@pytest.mark.parametrize('d', [16, 3])
def test_search_wait_runs_out_cleanly(d):
    L = _lib.lib()
    x = _gmm(d=d)
    xt = torch.from_numpy(x).to('cuda', torch.float32)
    flags = ops.new_flags(xt.device)
    prev = L.nngp_set_wait_limit_ns(1)
    try:
        ops.knn(xt, xt, 32, 0, 0.8, flags=flags)
        torch.cuda.synchronize()
    finally:
        L.nngp_set_wait_limit_ns(0)
    assert prev == 2_000_000_000
    f = int(flags.item())
    assert f & _lib.NNGP_FLAG_TIMEOUT
    with pytest.raises(_lib.NngpError):
        ops.raise_on_flags(f, 'knn')

    # the same context, the default limit: a clean call with the oracle's lists
    flags2 = ops.new_flags(xt.device)
    out = ops.knn(xt, xt, 32, 0, 0.8, flags=flags2).cpu().numpy()
    assert int(flags2.item()) == 0
    rows = np.random.default_rng(0).choice(np.arange(1, len(x)), 200, replace=False)
    want = O.knn(x, x[rows], 32, 0, 0.8, query_index=rows)
    np.testing.assert_array_equal(out[rows], want)
