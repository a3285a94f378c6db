"""One scene split into slabs along z against the same scene on one handle (GPU tests).

A plastic J2 impact block spans the seams. On one handle (a batch of slab scenes with the
on-device overlap sum) and as two ranks in one process (single-scene handles with the seams open,
exchanging their overlap planes through device buffers, which a multi-GPU run moves with NCCL),
the particles must follow the undivided scene: positions within 1e-6 m, velocities and F within
1e-5 relative after 20 substeps (the overlap nodes sum the two slabs' contributions in another
order than one grid does, so FP32 rounding differs), with the same dt every substep.
"""
import numpy as np
import pytest
import torch

from mpm_b200 import scenes
from mpm_b200.slabs import SlabRank, partition, slab_batch, slab_domains
from mpm_b200.solver import Solver

pytestmark = pytest.mark.gpu
PLANES = 6


def rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    s = float(np.max(np.abs(b)))
    return float(np.max(np.abs(a - b)) / (s if s > 0 else 1.0))


def block():
    return scenes.j2_drop(shape=(24, 12, 24), grid=48, plastic=True)


def whole(sc, dt, n):
    s = Solver(sc.domain, sc.n)
    s.upload(sc)
    dts = []
    for _ in range(n):
        dts.append(s.stable_dt())
        s.step_fixed(dt if dt else dts[-1], 1)
    out = s.download(("x", "v", "F", "ep"))
    s.close()
    return out, dts


def compare(parts_out, index, ref, n):
    got = {f: np.empty_like(ref[f]) for f in ref}
    for o, idx in zip(parts_out, index):
        for f in ref:
            got[f][idx] = o[f]
    assert np.max(np.abs(got["x"] - ref["x"])) <= 1e-6
    assert rel(got["v"], ref["v"]) <= 1e-5
    assert np.max(np.abs(got["F"] - ref["F"])) <= 1e-5
    assert np.max(np.abs(got["ep"] - ref["ep"])) <= 1e-6 + 1e-4 * np.max(ref["ep"])


@pytest.mark.parametrize("nslabs", [2, 3])
def test_slab_batch_matches_the_undivided_scene(nslabs):
    sc = block()
    dt = 2e-6
    ref, _ = whole(sc, dt, 20)
    assert np.max(ref["ep"]) > 0  # the impact yields near the floor, across the seams
    b, index = slab_batch(sc, nslabs, PLANES)
    b.step_fixed(dt, 20)
    out = b.split(b.download(("x", "v", "F", "ep")))
    compare(out, index, ref, sc.n)
    assert b.status() == 0
    b.close()


def test_slab_batch_takes_one_cfl_dt_for_all_slabs():
    sc = block()
    b, index = slab_batch(sc, 2, PLANES)
    s = Solver(sc.domain, sc.n)
    s.upload(sc)
    for _ in range(3):
        sub_b, adv_b = b.step(1e-5)
        sub_s, adv_s = s.step(1e-5)
        assert sub_b == sub_s and abs(adv_b - adv_s) <= 1e-12
    _, dts = b.times()
    assert np.ptp(dts) == 0  # every slab took the same substep
    compare(b.split(b.download(("x", "v", "F", "ep"))), index, s.download(("x", "v", "F", "ep")), sc.n)
    s.close()
    b.close()


class _Buf:
    def __init__(self, nbytes):
        self.t = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
        self.ptr = self.t.data_ptr()


def test_two_ranks_exchanging_overlap_planes_match_the_undivided_scene():
    sc = block()
    slabs = slab_domains(sc.domain, 2, PLANES)
    parts = partition(sc, slabs)
    ranks = [SlabRank(p, s, r, 2, PLANES, None, None, _Buf, start=False) for r, ((p, _), s) in
             enumerate(zip(parts, slabs))]

    def exchange():  # both ranks in one process: export, swap the buffers, add
        ranks[0].export(1)
        ranks[1].export(0)
        ranks[1].recv[0].t.copy_(ranks[0].send[1].t)
        ranks[0].recv[1].t.copy_(ranks[1].send[0].t)
        torch.cuda.synchronize()
        ranks[0].add(1)
        ranks[1].add(0)

    exchange()
    ref, dts = whole(sc, None, 20)
    for k in range(20):
        dt = min(r.solver.stable_dt() for r in ranks)
        assert abs(dt - dts[k]) <= 1e-6 * dts[k]  # the min over slabs is the undivided scene's dt
        for r in ranks:
            r.solver.step_fixed(dts[k], 1)
        exchange()
    compare([r.solver.download(("x", "v", "F", "ep")) for r in ranks], [i for _, i in parts], ref, sc.n)
    for r in ranks:
        r.close()
