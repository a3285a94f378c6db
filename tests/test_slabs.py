"""One scene split into slabs along z (mpm_b200.slabs): grid alignment, the particle partition and
the overlap-exchange protocol between ranks, on the CPU (gloo, world size 2 and 3, over numpy
stand-ins for the device planes). GPU tests of the device paths: tests/test_gpu_slabs.py."""
import os

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from mpm_b200 import scenes
from mpm_b200.slabs import halo_exchange, partition, slab_domains


def test_slab_grids_align_and_share_the_planes():
    sc = scenes.j2_drop(shape=(16, 16, 16), grid=48)
    for nslabs in (2, 3):
        slabs = slab_domains(sc.domain, nslabs, 6)
        d = sc.domain
        assert slabs[0].nodes[0] == 0 and slabs[-1].nodes[1] == d.dims[2]
        for k, s in enumerate(slabs):
            assert s.domain.dims[:2] == d.dims[:2] and s.domain.origin[:2] == d.origin[:2]
            assert abs(s.domain.origin[2] - (d.origin[2] + s.nodes[0] * d.H)) < 1e-12
            assert s.domain.dims[2] == s.nodes[1] - s.nodes[0]
            if k > 0:
                assert slabs[k - 1].nodes[1] - s.nodes[0] == 6  # the shared planes
                assert s.own[0] - s.nodes[0] == 3 and slabs[k - 1].nodes[1] - slabs[k - 1].own[1] == 3
        parts = partition(sc, slabs)
        idx = np.sort(np.concatenate([i for _, i in parts]))
        assert np.array_equal(idx, np.arange(sc.n))  # every particle in exactly one slab
        for k, ((p, _), s) in enumerate(zip(parts, slabs)):
            zq = (p.x[:, 2] - s.domain.origin[2]) / d.H
            # own range: 3 planes (half the shared ones) inside the slab's grid at each seam
            lo = 3 if k > 0 else 0
            hi = s.domain.dims[2] - (3 if k < nslabs - 1 else 0)
            assert p.n == 0 or (zq.min() >= lo and zq.max() < hi)


def test_bad_slab_requests_are_rejected():
    sc = scenes.elastic_cube()
    with pytest.raises(ValueError):
        slab_domains(sc.domain, 2, 5)  # odd
    with pytest.raises(ValueError):
        slab_domains(sc.domain, 20, 6)  # too thin


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch
    dist.init_process_group("gloo", rank=rank, world_size=world)
    rng = np.random.default_rng(rank)
    planes = {0: rng.normal(size=8), 1: rng.normal(size=8)}  # this rank's own seam contributions
    send, recv, held = {}, {}, {0: planes[0].copy(), 1: planes[1].copy()}

    def export(s):
        send[s] = torch.from_numpy(held[s].copy())

    def swap(s, peer):
        recv[s] = torch.empty(8, dtype=torch.float64)
        ops = [dist.P2POp(dist.isend, send[s], peer), dist.P2POp(dist.irecv, recv[s], peer)]
        for r in dist.batch_isend_irecv(ops):
            r.wait()

    def add(s):
        held[s] = held[s] + recv[s].numpy()

    sides = halo_exchange(rank, world, export, add, swap)
    out[rank] = (sides, {s: held[s].tolist() for s in sides}, {s: planes[s].tolist() for s in (0, 1)})
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_rank_exchange_sums_both_sides_of_every_seam(world):
    port = 29600 + world
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    for r in range(world):
        sides, held, own = res[r]
        assert sides == [s for s, p in ((0, r - 1), (1, r + 1)) if 0 <= p < world]
        for s in sides:
            peer = r - 1 if s == 0 else r + 1
            other = res[peer][2][1 - s]  # the neighbour's contribution on the same seam
            np.testing.assert_allclose(held[s], np.add(own[s], other), rtol=0, atol=0)
    # both copies of a seam hold the same sum (addition is commutative in floating point)
    for r in range(world - 1):
        np.testing.assert_array_equal(res[r][1][1], res[r + 1][1][0])


class _FakeSolver:
    """Stands in for a slab's single-scene handle: a stable dt of its own, a log of fixed substeps."""

    def __init__(self, dt):
        self.dt, self.taken = dt, []

    def stable_dt(self):
        return self.dt

    def step_fixed(self, dt, n):
        self.taken += [dt] * n


def _advance_worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch
    from mpm_b200.slabs import SlabRank
    dist.init_process_group("gloo", rank=rank, world_size=world)

    def reduce_min(x):
        t = torch.tensor([x], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MIN)
        return float(t.item())

    sr = SlabRank.__new__(SlabRank)
    sr.rank, sr.world, sr.reduce_min = rank, world, reduce_min
    sr.solver = _FakeSolver(dt=3e-4 * (1 + rank))  # rank 0 is the slowest to stay stable
    exchanges = []
    sr.exchange = lambda: exchanges.append(len(sr.solver.taken))
    n = sr.advance(1e-3)
    out[rank] = (n, sr.solver.taken, exchanges)
    dist.destroy_process_group()


def test_ranks_advance_with_the_same_substeps():
    world = 2
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_advance_worker, args=(world, 29610, out), nprocs=world, join=True)
        res = dict(out)
    n0, taken0, ex0 = res[0]
    assert n0 == 4 and ex0 == [1, 2, 3, 4]  # 3 x 3e-4 and the 1e-4 left; one exchange after each
    np.testing.assert_allclose(taken0, [3e-4, 3e-4, 3e-4, 1e-4], rtol=1e-12)
    assert res[1] == res[0]
