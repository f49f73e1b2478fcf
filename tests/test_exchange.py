"""The multi-GPU partition exchange on CPU: the partition ranges, and the
exchange itself over gloo with 2 and 3 ranks, checked against the oracle
(each rank's range counted from what it received equals the single-process
oracle's table of that range)."""
import numpy as np
import pytest
import torch.multiprocessing as mp

import dist_workers
from rapidgkc_b200.exchange import partition_ranges


@pytest.mark.parametrize("world", [1, 2, 3, 8])
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_partition_ranges_balance(world, seed):
    r = np.random.default_rng(seed)
    P = 512
    loads = r.integers(0, 1000, P) * (r.random(P) < 0.9) + (r.random(P) < 0.01) * 20_000
    b = partition_ranges(loads, world)
    assert b[0] == 0 and b[-1] == P and len(b) == world + 1 and np.all(np.diff(b) >= 0)
    sums = np.array([loads[b[i]:b[i + 1]].sum() for i in range(world)])
    assert sums.sum() == loads.sum()
    # every cut is within one partition of its target: no range exceeds an
    # equal share by more than twice the largest partition
    assert sums.max() <= loads.sum() / world + 2 * loads.max()


def test_partition_ranges_edge_cases():
    assert list(partition_ranges(np.zeros(8), 4)) == [0, 2, 4, 6, 8]
    assert list(partition_ranges([5], 3)) in ([0, 0, 1, 1], [0, 1, 1, 1], [0, 0, 0, 1])
    b = partition_ranges([0, 0, 100, 0, 0, 100, 0], 2)
    assert b[0] == 0 and b[-1] == 7 and 3 <= b[1] <= 5
    with pytest.raises(ValueError):
        partition_ranges([1, 2], 0)


@pytest.mark.parametrize("world,k", [(2, 25), (3, 25), (2, 45)])
def test_exchange_over_gloo_matches_oracle(world, k):
    mp.spawn(dist_workers.oracle_exchange, args=(world, dist_workers.free_port(), 31, k), nprocs=world, join=True)
