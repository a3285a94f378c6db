"""Batched ensembles (mpm_batch_*) and per-particle edits (mpm_reset_particle / mpm_remove_particle).

A batch handle must give every scene exactly the physics a single-scene handle gives it: the
same CFL dt, the same state after the same number of substeps (within FP32 rounding of the
order-dependent grid atomics, 1e-6 relative), the same grid, and its own FP64 ledger. A graph
replay must match eager launches, and the autotuner must leave the state as it found it.
"""
import ctypes

import numpy as np
import pytest

from mpm_b200 import _lib
from mpm_b200.params import Domain, Material, MODEL_FIXED_COROTATED, MODEL_J2
from mpm_b200.scenes import _scene, block_particles

TOL = 1e-6


def small_scenes():
    """Three scenes of different grids, block sizes, materials and velocities."""
    out = []
    specs = [(16, (5, 4, 5), (10, 9, 10), Material.from_young(MODEL_J2, 2e6, .3, density=1000., yield_stress=2e3),
              (0, -2, 0)),
             (24, (8, 3, 7), (14, 8, 13), Material.from_young(MODEL_FIXED_COROTATED, 1e5, .25, density=1000.),
              (1, -1, 0)),
             (20, (6, 5, 6), (12, 10, 11), Material.from_young(MODEL_J2, 7e10, .33, density=2700., yield_stress=2.5e8),
              (0, -20, 0))]
    for k, (g, lo, hi, mat, v0) in enumerate(specs):
        d = Domain(lower=(0, 0, 0), upper=(1, 1, 1), H=1 / g, gravity=(0, -9.8, 0), sticky_floor=True)
        x = block_particles(d, lo, hi, 77 + k)
        out.append(_scene(f"small_{k}", d, [mat], x, v0))
    return out


def rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    s = float(np.max(np.abs(b)))
    return float(np.max(np.abs(a - b)) / (s if s > 0 else 1.0))


def test_batch_structs_match_header():
    assert ctypes.sizeof(_lib.MpmSceneDesc) == ctypes.sizeof(_lib.MpmDomain) + 16
    assert ctypes.sizeof(_lib.MpmTuning) == 6 * 4 + 2 * 8


def test_batch_create_rejects_bad_tables_without_a_device():
    L = _lib.lib()
    h = ctypes.c_void_p()
    assert L.mpm_batch_create(None, 1, ctypes.byref(h)) == -1
    descs = (_lib.MpmSceneDesc * 1)()
    assert L.mpm_batch_create(descs, 0, ctypes.byref(h)) == -1
    descs[0].count = -1
    assert L.mpm_batch_create(descs, 1, ctypes.byref(h)) == -1
    descs[0].count = 10
    descs[0].material = 256
    assert L.mpm_batch_create(descs, 1, ctypes.byref(h)) == -1


@pytest.mark.gpu
def test_batch_matches_single_scene_handles():
    from mpm_b200.solver import Batch, Solver
    scenes = small_scenes()
    b = Batch(scenes)
    b.upload()
    b.run(7, graph=False)
    parts = b.split(b.download())
    t_batch, _ = b.times()
    for k, sc in enumerate(scenes):
        s = Solver(sc.domain, sc.n)
        s.upload(sc)
        t = s.step_cfl(7)
        o = s.download()
        assert abs(t_batch[k] - t) <= 1e-6 * t, (k, t_batch[k], t)
        for f in ("x", "v", "F"):
            assert rel(parts[k][f], o[f]) <= TOL, (k, f, rel(parts[k][f], o[f]))
        s.close()
    b.close()


@pytest.mark.gpu
def test_batch_graph_replay_matches_eager_launches():
    from mpm_b200.solver import Batch
    scenes = small_scenes()
    runs = []
    for graph in (True, False):
        b = Batch(scenes)
        b.upload()
        b.run(64, graph=graph)  # captures a graph of 2 x 32 substeps and launches it
        b.run(64, graph=graph)  # same buffer parity and re-sort phase: replays it
        b.run(5, graph=graph)   # shorter than a graph: eager
        runs.append((b.download(), b.times()[0], b.launch_count()))
        b.close()
    (og, tg, lg), (oe, te, le) = runs
    np.testing.assert_allclose(tg, te, rtol=1e-6)
    for f in ("x", "v", "F"):
        assert rel(og[f], oe[f]) <= 1e-5, (f, rel(og[f], oe[f]))
    assert lg == le  # the graph's kernels are counted like eager launches


@pytest.mark.gpu
def test_material_change_after_a_captured_graph_takes_effect():
    """A material set after the batch captured a graph acts from the next run: the handle-wide
    flags and kernel instances a graph holds (here: no plastic material, so no plastic strain is read
    or written) are rebuilt. Three elastic scenes, one turned into a J2 material after a captured
    run; the graph-replayed batch matches the same sequence run eagerly, and the changed scene
    yields."""
    from mpm_b200.solver import Batch
    scenes = small_scenes()
    # the J2 scenes start elastic (fixed-corotated, same moduli); scene 0 turns J2 after a run
    scenes[0].materials = [Material.from_young(MODEL_FIXED_COROTATED, 1e5, .3, density=1000.)]
    scenes[2].materials = [Material.from_young(MODEL_FIXED_COROTATED, 7e10, .33, density=2700.)]
    # soft enough that its CFL substeps reach the floor within the runs, and it then yields
    soft = Material.from_young(MODEL_J2, 1e5, .3, density=1000., yield_stress=5.0)
    outs = []
    for graph in (True, False):
        b = Batch(scenes)
        b.upload()
        b.run(64, graph=graph)
        b.set_material(0, soft)
        b.run(64, graph=graph)
        outs.append(b.split(b.download(("x", "v", "F", "ep"))))
        assert b.status() == 0
        b.close()
    (og, oe) = outs
    assert np.max(oe[0]["ep"]) > 0 and np.max(og[0]["ep"]) > 0
    for k in range(len(scenes)):
        for f in ("x", "v", "F", "ep"):
            assert rel(og[k][f], oe[k][f]) <= 1e-5, (k, f, rel(og[k][f], oe[k][f]))


@pytest.mark.gpu
def test_batch_scene_one_substep_matches_oracle():
    from mpm_b200.solver import Batch
    from oracle import oracle as orc
    scenes = small_scenes()
    b = Batch(scenes)
    b.upload()
    b.run(1, graph=False)
    t, dt = b.times()
    parts = b.split(b.download())
    for k, sc in enumerate(scenes):
        st = orc.state_from_scene(sc)
        st.step(float(dt[k]))
        assert abs(t[k] - dt[k]) <= 1e-12 * dt[k]
        assert np.max(np.abs(parts[k]["x"] - st.x)) <= 1e-6
        assert rel(parts[k]["v"], st.v) <= TOL, (k, rel(parts[k]["v"], st.v))
        assert np.max(np.abs(parts[k]["F"] - st.F)) <= 1e-6
    b.close()


@pytest.mark.gpu
def test_batch_ledgers_and_grids_are_per_scene():
    from mpm_b200.solver import Batch
    from oracle import oracle as orc
    scenes = small_scenes()
    b = Batch(scenes)
    b.upload()
    whole = b.ledger()
    total = 0.0
    for k, sc in enumerate(scenes):
        L = b.scene_ledger(k)
        R = orc.state_from_scene(sc).ledger()
        assert L.count == sc.n
        assert abs(L.mass - R.mass) <= 1e-6 * R.mass
        assert abs(L.kinetic - R.kinetic) <= 1e-5 * R.kinetic
        total += L.mass
        gm, _ = b.scene_grid_debug(k, 1e-6)
        assert abs(gm.sum() - R.mass) <= 1e-5 * R.mass
    assert abs(total - whole.mass) <= 1e-9 * whole.mass
    b.close()


@pytest.mark.gpu
def test_autotune_keeps_state_and_reports_a_schedule():
    from mpm_b200.solver import Batch
    b = Batch(small_scenes())
    b.upload()
    b.run(3, graph=False)
    before = b.download()
    t0, _ = b.times()
    tune = b.autotune(4)
    after = b.download()
    t1, _ = b.times()
    for f in before:
        assert np.array_equal(before[f], after[f]), f
    assert np.array_equal(t0, t1)
    assert tune["trials"] >= 2 and tune["blocks_per_sm"] >= 1
    assert 0 < tune["ms_per_substep"] <= tune["ms_per_substep_default"]
    b.run(5)  # the tuned schedule steps
    b.close()


@pytest.mark.gpu
def test_reset_and_remove_particle_follow_mpm3():
    from mpm_b200.solver import Solver
    sc = small_scenes()[0]
    s = Solver(sc.domain, sc.n)
    s.upload(sc)
    s.step_cfl(6)
    before = s.download()
    s.reset_particle(5)
    o = s.download()
    assert np.array_equal(o["F"][5], np.eye(3).ravel()) and not o["C"][5].any() and o["ep"][5] == 0
    assert np.array_equal(np.delete(o["x"], 5, 0), np.delete(before["x"], 5, 0))
    n = s.n
    s.remove_particle(3, n - 1)
    r = s.download()
    assert r["x"].shape[0] == n - 1
    assert np.array_equal(r["x"][3], o["x"][n - 1]) and np.array_equal(r["F"][3], o["F"][n - 1])
    keep = [i for i in range(n - 1) if i != 3]
    assert np.array_equal(r["x"][keep], o["x"][keep])
    with pytest.raises(_lib.MpmError):
        s.remove_particle(0, 0)  # last must be count - 1
    s.step_cfl(2)  # the edited state steps
    s.close()
