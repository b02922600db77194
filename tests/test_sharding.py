"""Batched solves sharded over ranks (mpd_b200.sharding): the assignment on
its own, then the collectives with two gloo ranks on the CPU (a stand-in for
the per-rank batch, no GPU)."""
import os
import pickle
import socket
import tempfile

import numpy as np
import pytest
import torch.multiprocessing as mp


def test_shard_covers_every_solve_once_and_balances(pkg):
    rng = np.random.default_rng(3)
    for world in (1, 2, 3, 8):
        costs = rng.choice([4.0e3, 1.6e4, 6.4e4, 2.56e5], size=37) * rng.uniform(0.9, 1.1, 37)
        shares = pkg.sharding.shard(costs, world)
        assert len(shares) == world
        flat = sorted(i for s in shares for i in s)
        assert flat == list(range(len(costs)))
        assert all(s == sorted(s) for s in shares)
        loads = [costs[s].sum() if s else 0.0 for s in shares]
        # the LPT bound: no share exceeds the mean by more than one solve's cost
        assert max(loads) <= costs.sum() / world + costs.max() + 1e-9
    assert pkg.sharding.shard([], 2) == [[], []]
    with pytest.raises(ValueError):
        pkg.sharding.shard([1.0], 0)


def test_shard_is_deterministic_and_cost_ordered(pkg):
    costs = [5.0, 1.0, 5.0, 3.0]
    assert pkg.sharding.shard(costs, 2) == pkg.sharding.shard(list(costs), 2)
    # the two largest solves land on different ranks
    a, b = pkg.sharding.shard(costs, 2)
    assert (0 in a) != (2 in a)


def test_solve_cost_follows_cells_and_steps(pkg):
    small = pkg.workloads.channel_config(L=100, M=40)
    big = pkg.workloads.channel_config(L=200, M=80)
    assert pkg.sharding.solve_cost(big, 10**9) > 15 * pkg.sharding.solve_cost(small, 10**9)
    assert pkg.sharding.solve_cost(big, 1000) == 200 * 81 * 1000


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import sys
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    if root not in sys.path:
        sys.path.insert(0, root)
    import __graft_entry__
    pkg = __graft_entry__.load_package()
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    costs = [float(c) for c in (9, 1, 4, 4, 7, 2, 3)]

    def run_share(idx):
        # stand-in for this rank's batch: a result that names its solve
        runs = [("solve", i, rank) for i in idx]
        return runs, np.array([10.0 * i for i in idx]), 1.0 + rank

    res = pkg.sharding.run_sharded(costs, run_share)
    with open(os.path.join(out_dir, f"rank{rank}.pkl"), "wb") as f:
        pickle.dump(res, f)
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_gather_results_in_sweep_order():
    world = 2
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_rank_main, args=(world, _free_port(), d), nprocs=world,
                           join=True, start_method="spawn")
        with open(os.path.join(d, "rank0.pkl"), "rb") as f:
            r0 = pickle.load(f)
        with open(os.path.join(d, "rank1.pkl"), "rb") as f:
            r1 = pickle.load(f)
    assert r1 is None
    assert [r[1] for r in r0.runs] == list(range(7))
    # each solve ran on the rank its share names, and only there
    for rank, share in enumerate(r0.shares):
        assert all(r0.runs[i][2] == rank for i in share)
    np.testing.assert_array_equal(r0.solve_ms, 10.0 * np.arange(7))
    assert r0.device_ms == 2.0   # the slower rank's batch
