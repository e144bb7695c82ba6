"""Sharding a batch across ranks (cushg_b200/shard.py): the partition on its own, and the
N>1 path as world-size-2 gloo process groups on CPU (no GPU: each rank stands in a
deterministic function of the instance for its solve)."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from cushg_b200 import params as P
from cushg_b200 import shard as S


def test_partition_covers_every_instance_once_and_balances():
    ps = P.config_sweep(256, seed=0)
    costs = [S.instance_cost(p) for p in ps]
    for world in (1, 2, 3, 8):
        parts = S.partition(costs, world)
        flat = sorted(i for part in parts for i in part)
        assert flat == list(range(len(ps)))
        loads = [sum(costs[i] for i in part) for part in parts]
        # greedy longest-first: no rank exceeds the mean by more than the largest instance
        assert max(loads) - sum(loads) / world <= max(costs) + 1e-6
    assert S.partition(costs, 4) == S.partition(costs, 4)  # deterministic


def test_partition_rejects_bad_world():
    with pytest.raises(ValueError):
        S.partition([1.0, 2.0], 0)


def fake_power(p):
    return 1e-9 * S.instance_cost(p) + p.power


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ps = P.config_sweep(64, seed=0)
        idx, mine = S.shard(ps, rank, world)
        powers = S.gather_powers(idx, [fake_power(p) for p in mine], len(ps))
        np.save(os.path.join(out_dir, f"rank{rank}.npy"), powers)
        np.save(os.path.join(out_dir, f"idx{rank}.npy"), np.array(idx))
    finally:
        dist.destroy_process_group()


def test_two_ranks_shard_and_gather(tmp_path):
    world = 2
    mp.start_processes(_rank, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn")
    ps = P.config_sweep(64, seed=0)
    expect = np.array([fake_power(p) for p in ps])
    for r in range(world):
        assert np.array_equal(np.load(tmp_path / f"rank{r}.npy"), expect)
    i0, i1 = np.load(tmp_path / "idx0.npy"), np.load(tmp_path / "idx1.npy")
    assert not set(i0) & set(i1) and len(i0) + len(i1) == len(ps)
