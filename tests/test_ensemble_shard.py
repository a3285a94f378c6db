"""Scene sharding of a V&V ensemble across ranks (CPU: the partition and a gloo world of 2)."""
import os
import socket

import numpy as np
import pytest

from mpm_b200.ensemble import LEDGER_FIELDS, gather_ledgers, imbalance, shard_scenes


def costs_like_ensemble(count=256, seed=3):
    # particle counts log-uniform in [5e3, 2e5], as the ensemble's scenes
    rng = np.random.default_rng(seed)
    return list(np.exp(rng.uniform(np.log(5e3), np.log(2e5), count)))


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_every_scene_owned_once_and_balanced(world):
    costs = costs_like_ensemble()
    shards = shard_scenes(costs, world)
    assert len(shards) == world
    owned = sorted(k for s in shards for k in s)
    assert owned == list(range(len(costs)))
    assert imbalance(costs, shards) < 1.05


def test_sharding_is_deterministic_and_handles_few_scenes():
    costs = [5.0, 5.0, 5.0]
    assert shard_scenes(costs, 2) == shard_scenes(costs, 2)
    shards = shard_scenes(costs, 4)
    assert sorted(len(s) for s in shards) == [0, 1, 1, 1]
    with pytest.raises(ValueError):
        shard_scenes(costs, 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, costs, out):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        shards = shard_scenes(costs, world)
        mine = shards[rank]
        # a stand-in ledger row per owned scene: (k, 2k, ...) so the gather can be checked
        rows = np.array([[k * (f + 1) for f in range(len(LEDGER_FIELDS))] for k in mine], dtype=np.float64)
        full = gather_ledgers(rows.reshape(len(mine), len(LEDGER_FIELDS)), mine, len(costs), dist)
        out[rank] = full.tolist()
    finally:
        dist.destroy_process_group()


def test_gloo_world_of_two_gathers_every_scene_ledger():
    import torch.multiprocessing as mp
    costs = costs_like_ensemble(37, seed=9)
    manager = mp.Manager()
    out = manager.dict()
    mp.spawn(_rank_main, args=(2, _free_port(), costs, out), nprocs=2, join=True)
    expect = np.array([[k * (f + 1) for f in range(len(LEDGER_FIELDS))] for k in range(len(costs))], dtype=np.float64)
    for r in range(2):
        np.testing.assert_array_equal(np.array(out[r]), expect)
