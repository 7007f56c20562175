"""Row sharding of the fit step (CPU, gloo, world size 2).

Each rank computes the partial log-likelihood and gradient of its row range with the CPU oracle
standing in for the device kernels (the same search cut and row range that
``nngpr_b200.sharding.fit_step_rows`` passes to the C ABI), all-reduces it over gloo, and the sum
must equal the single-process value.
"""
import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from nngpr_b200.sharding import prefix_pairs, row_partition


def test_row_partition_equal_rows_for_the_pruned_search():
    from nngpr_b200.sharding import search_is_pruned
    assert search_is_pruned(434874, 3) and search_is_pruned(434874, 8) and not search_is_pruned(434874, 33)
    assert not search_is_pruned(30000, 3)
    for n, world in [(434874, 8), (10, 3), (1, 4)]:
        b = row_partition(n, world, equal_rows=True)
        assert b[0] == 0 and b[-1] == n and all(b[i] <= b[i + 1] for i in range(world))
        assert max(b[i + 1] - b[i] for i in range(world)) - min(b[i + 1] - b[i] for i in range(world)) <= 1


def test_row_partition_balances_prefix_pairs():
    for n, world in [(434874, 2), (434874, 8), (1000, 3), (7, 4), (1, 2)]:
        b = row_partition(n, world)
        assert b[0] == 0 and b[-1] == n and all(b[i] <= b[i + 1] for i in range(world))
        pairs = [prefix_pairs(b[r], b[r + 1]) for r in range(world)]
        assert sum(pairs) == n * (n - 1) // 2
        if n > 1000:
            assert max(pairs) / min(pairs) < 1.01


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, result_file):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, 'tests'))
    from oracle import nngp_oracle as O
    from nngpr_b200.sharding import row_partition as part
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    from datetime import timedelta
    dist.init_process_group('gloo', rank=rank, world_size=world, timeout=timedelta(seconds=60))
    g = np.load(os.path.join(root, 'tests', 'golden', 'cpu_n2000_d3_m16.npz'))
    x, y = g['x'], g['y']
    p = O.KernelParams(rbf_level=1.0, const_value=0.0, noise_level=0.01, length_scale=0.3, idx_rbf_level=0,
                       idx_const=-1, idx_noise=2, idx_ls=1, n_theta=3)
    b = part(len(x), world)
    r0, r1 = b[rank], b[rank + 1]
    rows = np.arange(r0, r1)
    nbr = np.full((len(x), 16), -1, np.int32)
    nbr[rows] = O.knn(x, x[rows], 16, r0, 0.3, query_index=np.arange(r1 - r0))  # cut = row_begin, local index
    ll, gr = O.loglik_terms(x, y, nbr, p, 1e-10, True, rows)
    part_sum = torch.tensor(np.concatenate([[ll.sum()], gr.sum(0)]), dtype=torch.float64)
    dist.all_reduce(part_sum)
    if rank == 0:
        np.save(result_file, part_sum.numpy())
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_fit_step_equals_single_process(tmp_path):
    from oracle import nngp_oracle as O
    world = 2
    out = str(tmp_path / 'res.npy')
    mp.start_processes(_rank_main, args=(world, _free_port(), out), nprocs=world, start_method='spawn', join=True)
    got = np.load(out)
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden', 'cpu_n2000_d3_m16.npz'))
    assert abs(got[0] / g['lml'] - 1) < 1e-10
    assert np.max(np.abs(got[1:] - g['grad'])) / np.max(np.abs(g['grad'])) < 1e-9


def test_rebalance_equalises_measured_times():
    from nngpr_b200.sharding import rebalance, row_partition
    # rows whose cost density is 1 on [0, 600) and 4 on [600, 1000): a rank's time is its cost
    dens = np.where(np.arange(1000) < 600, 1.0, 4.0)

    def times(b):
        return [float(dens[b[r]:b[r + 1]].sum()) for r in range(len(b) - 1)]

    b = row_partition(1000, 4, equal_rows=True)
    t = times(b)
    assert max(t) / min(t) == 4.0
    for _ in range(3):  # each round narrows the spread, also where a range straddles the change
        b = rebalance(b, times(b))
        assert b[0] == 0 and b[-1] == 1000 and all(b[i] <= b[i + 1] for i in range(4))
        t2 = times(b)
        assert max(t2) / min(t2) <= max(t) / min(t)
        t = t2
    assert max(t) / min(t) < 1.06
    # equal times leave the partition as it is; zero times too
    assert rebalance([0, 5, 10], [1.0, 1.0]) == [0, 5, 10]
    assert rebalance([0, 5, 10], [0.0, 0.0]) == [0, 5, 10]
