"""Sharding a V&V ensemble of independent scenes across ranks (one process per GPU).

Scenes never exchange data, so the multi-GPU form of an ensemble is a partition: every rank owns
whole scenes and steps them on its own batch handle; nothing crosses NVLink while stepping. The
only collective is the gather of each scene's small FP64 ledger (and timing) at the end, on the
host side of torch.distributed.

The reference steps its cases one after another in one worker (src/simulation/vv-mpm.js:30-60);
the partition replaces that loop across GPUs.
"""
import heapq

import numpy as np


def scene_cost(scene, substeps=1):
    """Work of one scene: particles x substeps (the G2P2G pass dominates, linear in particles)."""
    return float(scene.n) * substeps


def shard_scenes(costs, world):
    """Greedy longest-processing-time partition: scenes sorted by cost, each given to the rank
    with the least work so far. Returns, per rank, the sorted list of scene indices it owns.
    Deterministic for equal costs (ties broken by scene index, then rank)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda k: (-costs[k], k))
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    owned = [[] for _ in range(world)]
    for k in order:
        load, r = heapq.heappop(heap)
        owned[r].append(k)
        heapq.heappush(heap, (load + costs[k], r))
    return [sorted(o) for o in owned]


def imbalance(costs, shards):
    """max rank load / mean rank load (1.0 = perfect balance)."""
    loads = [sum(costs[k] for k in s) for s in shards]
    mean = sum(loads) / len(loads)
    return max(loads) / mean if mean > 0 else 1.0


LEDGER_FIELDS = ("mass", "kinetic", "affine", "potential", "elastic", "min_j", "max_j", "max_plastic",
                 "max_von_mises", "count")


def ledger_rows(batch, indices):
    """(len(indices), len(LEDGER_FIELDS)) float64 rows of the per-scene ledgers of a batch whose
    scene k is global scene indices[k]."""
    rows = np.zeros((len(indices), len(LEDGER_FIELDS)))
    for k in range(len(indices)):
        L = batch.scene_ledger(k)
        rows[k] = [getattr(L, f) for f in LEDGER_FIELDS]
    return rows


def gather_ledgers(rows, indices, nscenes, dist=None):
    """All ranks' per-scene ledger rows in global scene order (sum-reduce of disjoint rows; every
    rank takes the same collective step). Without a process group the rows are placed locally."""
    import torch
    full = torch.zeros((nscenes, len(LEDGER_FIELDS)), dtype=torch.float64)
    if len(indices):
        full[torch.as_tensor(indices, dtype=torch.long)] = torch.as_tensor(rows, dtype=torch.float64)
    if dist is not None and dist.is_initialized() and dist.get_world_size() > 1:
        dev = torch.device("cuda") if dist.get_backend() == "nccl" else torch.device("cpu")
        t = full.to(dev)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        full = t.cpu()
    return full.numpy()
