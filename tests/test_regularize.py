"""Solid position regularisation (regularizeSolids, src/three/solid-sampling.js:5-42).

The FP64 oracle is pinned by restating tests/solid-sampling.test.mjs:7-49 in the reference's units
(spacing 2.8 at volume 1, budget 8 per second, rate 40 per second, the MPM3 default domain): crowded
pairs separate to the target spacing with the centre of mass kept and nothing but positions
touched; other parts and pinned particles do not move; the spacing follows volume loss including
the plastic compaction Jp of snow, soil and foam; coincident particles separate deterministically
within the displacement budget; equal elapsed time gives the same relaxation across substep sizes.
Parts are material indices here. The reference's last case (a six-second drop of a full
Simulation3 with fluids and a press, :50-62) needs that whole simulation and is not restated.

GPU tests (through the C ABI, mpm_regularize): the same cases on the device, and a crowded random
cloud against the oracle (positions within 1e-6 of the spacing after one pass).
"""
import numpy as np
import pytest

from oracle import oracle as orc
from mpm_b200 import scenes
from mpm_b200.params import Domain, Material

DOMAIN = Domain(lower=(-64, -48, -64), upper=(64, 72, 64), H=8.0)  # src/three/mpm.js DEFAULT_DOMAIN


def pair_scene(p0, p1, masses=(1.0, 1.0), models=(0, 0), mats=(0, 0), F=None, jp=None):
    materials = [Material.reference_units(m) for m in models]
    x = np.array([p0, p1], dtype=np.float64)
    sc = scenes._scene("pair", DOMAIN, materials, x, (0, 0, 0))
    sc.m = np.array(masses, dtype=np.float64)
    sc.V = np.ones(2)
    sc.mat = np.array(mats, dtype=np.int32)
    if F is not None:
        sc.F = np.tile(np.asarray(F, dtype=np.float64), (2, 1))
    if jp is not None:
        sc.jp = np.full(2, jp)
    return sc


def oracle_runs(sc, dt, steps, pinned=None):
    st = orc.state_from_scene(sc)
    if pinned is not None:
        st.pinned = np.ascontiguousarray(pinned, dtype=np.uint8)
    for _ in range(steps):
        st.regularize(dt)
    return st


# tests/solid-sampling.test.mjs:7-15
def test_crowded_pair_separates_without_kick_or_history_loss():
    sc = pair_scene((-.5, 0, 0), (.5, 0, 0), masses=(2.7, 3.0))
    sc.v = np.full((2, 3), 7.0)
    sc.C = np.zeros((2, 9))
    sc.C[0, 0] = .2
    sc.ep = np.array([.4, 0.0])
    st = orc.state_from_scene(sc)
    center = sc.m @ sc.x[:, 0]
    F0, C0, v0 = st.F.copy(), st.C.copy(), st.v.copy()
    for _ in range(60):
        st.regularize(1 / 120)
    assert st.x[1, 0] - st.x[0, 0] > 2.79
    assert abs(sc.m @ st.x[:, 0] - center) < 1e-10
    assert np.array_equal(st.v, v0) and np.array_equal(st.F, F0) and np.array_equal(st.C, C0)
    assert st.ep[0] == .4


# tests/solid-sampling.test.mjs:16-25
def test_other_parts_and_pinned_particles_do_not_move():
    st = oracle_runs(pair_scene((0, 0, 0), (1, 0, 0), mats=(0, 1)), 1 / 60, 1)
    assert st.x[0, 0] == 0 and st.x[1, 0] == 1
    st = oracle_runs(pair_scene((0, -46, 0), (0, -45, 0)), 1 / 120, 60, pinned=[1, 0])
    assert st.x[0, 1] == -46
    assert -43.3 < st.x[1, 1] <= -46 + 2.8 + 1e-9


# tests/solid-sampling.test.mjs:26-31: the spacing halves when the volume falls to 1/8 and, for
# snow, soil and foam, falls to a quarter with Jp = 1/8 on top (clamped at 1/64): seen here as the
# distance a pair one unit apart relaxes to
def test_spacing_follows_volume_loss_and_plastic_compaction():
    half = .5 * np.eye(3).ravel()
    st = oracle_runs(pair_scene((0, 0, 0), (1, 0, 0), F=half), 1 / 120, 120)
    assert abs(st.x[1, 0] - st.x[0, 0] - 1.4) < 1e-3  # 2.8 * cbrt(1/8)
    for model in (2, 8, 9):
        st = oracle_runs(pair_scene((0, 0, 0), (.5, 0, 0), models=(model, model), F=half, jp=.125), 1 / 120, 120)
        assert abs(st.x[1, 0] - st.x[0, 0] - .7) < 1e-3  # 2.8 * cbrt(1/64)


# tests/solid-sampling.test.mjs:32-38
def test_coincident_particles_separate_deterministically_within_budget():
    a = oracle_runs(pair_scene((0, 0, 0), (0, 0, 0)), 1 / 240, 1)
    b = oracle_runs(pair_scene((0, 0, 0), (0, 0, 0)), 1 / 240, 1)
    assert np.array_equal(a.x, b.x)
    d = float(np.linalg.norm(a.x[0]))
    assert 0 < d <= 8 / 240 + 1e-12
    assert np.sum(np.abs(a.x[0] + a.x[1])) < 1e-12


# tests/solid-sampling.test.mjs:39-49
def test_equal_elapsed_time_gives_consistent_relaxation():
    distances = []
    for dt in (1 / 120, 1 / 240, 1 / 1200):
        st = oracle_runs(pair_scene((-1, 0, 0), (1, 0, 0)), dt, round(.1 / dt))
        distances.append(st.x[1, 0] - st.x[0, 0])
    assert max(distances) - min(distances) < .01


def crowded_cloud(n=4000, seed=3):
    """A compacted random cloud of two parts in the reference's units (spacing 2.8 at volume 1)."""
    rng = np.random.default_rng(seed)
    x = rng.uniform(-20, 20, (n, 3)) * np.array([1, .5, 1])
    materials = [Material.reference_units(0), Material.reference_units(2)]
    sc = scenes._scene("cloud", DOMAIN, materials, x, (0, 0, 0))
    sc.m = rng.uniform(.5, 2.0, n)
    sc.V = rng.uniform(.5, 1.5, n)
    sc.mat = (rng.uniform(0, 1, n) < .3).astype(np.int32)
    sc.F = np.tile(np.eye(3).ravel(), (n, 1)) + .05 * rng.standard_normal((n, 9))
    sc.jp = rng.uniform(.7, 1.2, n)
    sc.pinned = (rng.uniform(0, 1, n) < .05).astype(np.uint8)
    return sc


def test_oracle_cloud_pass_keeps_pinned_and_the_centre_of_free_mass_bounded():
    sc = crowded_cloud()
    st = orc.state_from_scene(sc)
    x0 = st.x.copy()
    st.regularize(1 / 240)
    moved = np.linalg.norm(st.x - x0, axis=1)
    assert np.all(moved[sc.pinned == 1] == 0)
    assert np.max(moved) <= 8 / 240 + 1e-12  # the budget
    assert np.count_nonzero(moved) > sc.n // 2


# ------------------------------------------------------------------------------ device

def device_runs(sc, dt, steps, pinned=None, enabled=True):
    from mpm_b200.solver import Solver
    if pinned is not None:
        sc.pinned = np.asarray(pinned, dtype=np.uint8)
    sol = Solver(sc.domain, sc.n)
    sol.upload(sc)
    sol.set_regularizer(enabled=enabled)
    for _ in range(steps):
        sol.regularize(dt)
    out = sol.download(("x", "v", "F", "C", "ep"))
    sol.close()
    return out


@pytest.mark.gpu
def test_device_cases_match_the_reference_tests():
    out = device_runs(pair_scene((-.5, 0, 0), (.5, 0, 0), masses=(2.7, 3.0)), 1 / 120, 60)
    assert out["x"][1, 0] - out["x"][0, 0] > 2.79
    # positions are fixed point with resolution H / 2^22: each pass rounds every displacement once, so
    # the centre of mass holds to that resolution (60 passes x total mass x H / 2^22) instead of 1e-10
    assert abs(2.7 * out["x"][0, 0] + 3.0 * out["x"][1, 0] - (-1.35 + 1.5)) <= 60 * 5.7 * DOMAIN.H / 2 ** 22
    out = device_runs(pair_scene((0, 0, 0), (1, 0, 0), mats=(0, 1)), 1 / 60, 1)
    assert out["x"][0, 0] == 0 and out["x"][1, 0] == 1
    out = device_runs(pair_scene((0, 0, 0), (1, 0, 0)), 1 / 60, 1, enabled=False)
    assert out["x"][0, 0] == 0 and out["x"][1, 0] == 1
    out = device_runs(pair_scene((0, -46, 0), (0, -45, 0)), 1 / 120, 60, pinned=[1, 0])
    assert out["x"][0, 1] == -46 and -43.3 < out["x"][1, 1] <= -43.2 + 1e-5
    half = .5 * np.eye(3).ravel()
    out = device_runs(pair_scene((0, 0, 0), (.5, 0, 0), models=(9, 9), F=half, jp=.125), 1 / 120, 120)
    assert abs(out["x"][1, 0] - out["x"][0, 0] - .7) < 1e-3
    a = device_runs(pair_scene((0, 0, 0), (0, 0, 0)), 1 / 240, 1)
    b = device_runs(pair_scene((0, 0, 0), (0, 0, 0)), 1 / 240, 1)
    assert np.array_equal(a["x"], b["x"])
    d = float(np.linalg.norm(a["x"][0]))
    assert 0 < d <= 8 / 240 + 3 ** .5 * .5 * DOMAIN.H / 2 ** 22  # budget, plus one rounding per axis
    assert np.sum(np.abs(a["x"][0] + a["x"][1])) < 1e-6


@pytest.mark.gpu
def test_device_cloud_pass_matches_oracle():
    sc = crowded_cloud()
    st = orc.state_from_scene(sc)
    st.regularize(1 / 240)
    out = device_runs(sc, 1 / 240, 1)
    assert np.max(np.abs(out["x"] - st.x)) <= 1e-6 * 2.8
    assert np.max(np.abs(out["F"] - st.F)) <= 1e-7  # untouched (FP32 storage of F - I)


@pytest.mark.gpu
def test_device_substeps_with_regularisation_match_oracle():
    """mpm_step_fixed with the regulariser on: a gather pass, the regularisation at the substep's dt
    and a re-sorted scatter pass per substep, against oracle step + regularize (x within 1e-6 m)."""
    from mpm_b200.solver import Solver
    sc = scenes.elastic_cube()
    h = sc.domain.H
    kw = dict(spacing=.6 * h, volume_unit=h ** 3 / 8, max_speed=2.0, rate=40.0)
    dt = 1e-4
    st = orc.state_from_scene(sc)
    for _ in range(5):
        st.step(dt)
        st.regularize(dt, **kw)
    sol = Solver(sc.domain, sc.n)
    sol.upload(sc)
    sol.set_regularizer(enabled=True, **kw)
    sol.step_fixed(dt, 5)
    out = sol.download(("x", "v", "F"))
    moved = np.max(np.abs(st.x - orc.state_from_scene(sc).x))
    assert moved > 1e-4  # the regularisation and the step moved the particles
    assert np.max(np.abs(out["x"] - st.x)) <= 1e-6
    assert np.max(np.abs(out["F"] - st.F)) <= 1e-6
    assert sol.status() == 0
    sol.close()
