"""2D elastic solid (SolidMPM, src/solid-mpm.js): the oracle's known answers and GPU parity.

CPU tests restate the reference's own tests (tests/solid-mpm.test.mjs:9-66) on the FP64 oracle,
which pins it. GPU tests run the same cases through the smpm_* C ABI (FP32 state) and compare with
the oracle on the same inputs.

Tolerances for the GPU path. One step, on a smooth and on a rough (independent random particle
velocities) state: velocities and F within 1e-6 relative to their largest magnitude, C within
1e-6 of max|v| * 4 / DX (the scale C is built from), positions within 1e-6 of the grid's extent
(149 x 8 units). After 120 frames: positions within 1e-4 of the grid's extent.
The reference's FP64 bounds on exact invariants (translation 1e-6 absolute, strain 1e-10) are
stated for FP64 arithmetic; the FP32 path meets them at 1e-6 relative and 1e-6 strain.
"""
import math

import numpy as np
import pytest

from mpm_b200.solid_mpm import FIELDS, SolidSim, create_body
from oracle.oracle2d import Oracle2, solid_stress

EXTENT = 149 * 8.0


def empty(capacity=16000):
    # tests/solid-mpm.test.mjs:6: gravity none, thermal off, boundary off
    return SolidSim(capacity, scene="empty", gravity="none", boundary=False)


def width(s):
    return float(s.x[:s.count].max() - s.x[:s.count].min())


def stretched_panel():
    s = empty()
    create_body(s, -18, -18, 18, 18)
    reference = width(s)
    s.x[:s.count] *= 1.25
    return s, reference


def anchored_panel():
    s = empty()
    assert create_body(s, -60, 0, 25, 25, fixed=True)
    # The reference drags the tip with the pointer tool (tests/solid-mpm.test.mjs:44); the pointer
    # is not part of the solid path, so the same load is applied as an upward velocity of the
    # free half of the panel.
    free = (s.x[:s.count] > 0) & (s.pinned[:s.count] == 0)
    s.vy[:s.count][free] = 40
    return s


def random_panel(seed=5, rough=True):
    """A deformed, moving panel. rough: independent random velocities (-10..10) and C (-0.5..0.5)
    per particle, so node sums cancel heavily; smooth: a velocity field varying with position plus
    a little noise, and C within -0.1..0.1."""
    rng = np.random.default_rng(seed)
    s = SolidSim(scene="softbody", gravity="center", boundary=True)
    assert create_body(s, -40, -100, 40, -60)
    n = s.count
    if rough:
        s.vx[:n] = rng.uniform(-10, 10, n)
        s.vy[:n] = rng.uniform(-10, 10, n)
    else:
        x, y = s.x[:n].astype(np.float64), s.y[:n].astype(np.float64)
        s.vx[:n] = 6 + 4 * np.sin(x / 20) + rng.uniform(-.3, .3, n)
        s.vy[:n] = -3 + 4 * np.cos(y / 15) + rng.uniform(-.3, .3, n)
    s.pinned[:n:37] = 1
    fields = np.zeros((8, n))
    fields[0] = 1 + rng.uniform(-.05, .05, n)
    fields[3] = 1 + rng.uniform(-.05, .05, n)
    fields[1] = rng.uniform(-.05, .05, n)
    fields[2] = rng.uniform(-.05, .05, n)
    fields[4:] = rng.uniform(-.5, .5, (4, n)) if rough else rng.uniform(-.1, .1, (4, n))
    return s, fields


def copy_sim(s):
    t = SolidSim(s.capacity, s.scene, **s.settings)
    for k in ("x", "y", "vx", "vy", "mass", "volume", "material", "pinned"):
        getattr(t, k)[:] = getattr(s, k)
    t.count = s.count
    return t


# ---------------------------------------------------------------- oracle known answers (CPU)

def test_oracle_stress_is_rotation_free_and_resists_shear():
    # tests/solid-mpm.test.mjs:9-14
    th = .7
    c, sn = math.cos(th), math.sin(th)
    for tau in (solid_stress(1, 0, 0, 1, 400, 400), solid_stress(c, -sn, sn, c, 400, 400)):
        assert np.all(np.abs(tau) < 1e-10)
    shear = solid_stress(1, .3, 0, 1, 400, 400)
    assert shear[1] > 0 and abs(shear[1] - shear[2]) < 1e-10
    assert solid_stress(1.2, 0, 0, 1, 400, 400)[0] > 0


def test_oracle_ignores_liquid_particles():
    # tests/solid-mpm.test.mjs:15-19
    s = empty()
    for i in range(6):
        s.add(i * 3.5, 0, 2, 3, -2)
    x, vx = s.x.copy(), s.vx.copy()
    o = Oracle2(s.capacity)
    o.step(s, .001)
    assert np.array_equal(s.x, x) and np.array_equal(s.vx, vx)
    assert o.stats(s)["count"] == 0


def test_oracle_panel_preserves_uniform_translation():
    # tests/solid-mpm.test.mjs:22-29
    s = empty()
    assert create_body(s, -15, -15, 15, 15)
    s.vx[:s.count] = 7
    s.vy[:s.count] = -3
    o = Oracle2(s.capacity)
    o.step(s, .001)
    assert np.all(np.abs(s.vx[:s.count] - 7) < 1e-6) and np.all(np.abs(s.vy[:s.count] + 3) < 1e-6)
    assert o.stats(s)["strain"] < 1e-10


def test_oracle_stretched_solid_contracts_after_release():
    # tests/solid-mpm.test.mjs:30-39
    s, reference = stretched_panel()
    o = Oracle2(s.capacity)
    o.fields[0, :s.count] = 1.25
    stretched = width(s)
    lo, speed = math.inf, 0.0
    for _ in range(120):
        o.frame(s)
        lo = min(lo, width(s))
        speed = max(speed, float(np.abs(s.vx[:s.count]).max()))
    assert lo < reference * 1.1 and lo < stretched * .9
    assert speed > 1
    assert o.stats(s)["minJ"] > 0


def test_oracle_anchored_body_deforms_and_recoils():
    # tests/solid-mpm.test.mjs:40-51, with the load applied as an initial velocity
    s = anchored_panel()
    o = Oracle2(s.capacity)
    pins = [(i, s.x[i], s.y[i]) for i in range(s.count) if s.pinned[i]]
    tip = 23
    initial = float(s.y[tip])
    loaded = -math.inf
    for _ in range(120):
        o.frame(s)
        loaded = max(loaded, float(s.y[tip]))
    assert loaded > initial + 8
    assert o.stats(s)["strain"] > .05
    lo = math.inf
    for _ in range(180):
        o.frame(s)
        lo = min(lo, float(s.y[tip]))
    assert lo < loaded - 5
    for i, x, y in pins:
        assert math.hypot(s.x[i] - x, s.y[i] - y) < 1e-5


def test_create_is_atomic_at_capacity_and_rejects_bad_input():
    # tests/solid-mpm.test.mjs:62-66 (capacity part) and src/solid-mpm.js:93-99
    s = empty()
    s.count = s.capacity - 2
    assert create_body(s, 0, 0, 20, 20) is False and s.count == s.capacity - 2
    s = empty()
    assert create_body(s, 0, 0, 5, 20) is False  # narrower than 7
    assert create_body(s, 0, 0, math.nan, 20) is False
    assert create_body(s, 0, 0, 20, 20, material=7) is False  # not an MPM material
    assert s.count == 0
    assert create_body(s, 0, 0, 40, 0, shape="beam")
    assert s.count == 12 * 7


def test_oracle_frame_bounds_substeps_and_time():
    # src/simulation.js:239-255: dt clamped to 0.05, at most 96 substeps, stableStep <= 1/240
    s, _ = stretched_panel()
    o = Oracle2(s.capacity)
    n, adv = o.frame(s, 1.0)
    assert n >= 12 and abs(adv - .05) < 1e-12
    n, adv = o.frame(s, 0.0)
    assert n == 0 and adv == 0


# ---------------------------------------------------------------- GPU parity (smpm_* C ABI)

def gpu_handle(capacity=16000):
    from mpm_b200.solid_mpm import SolidMPM
    return SolidMPM(capacity)


@pytest.mark.gpu
def test_gpu_stress_free_rotation_and_shear_response():
    th = .7
    c, sn = math.cos(th), math.sin(th)
    for F, moves in (((c, -sn, sn, c), False), ((1, .3, 0, 1), True)):
        s = empty()
        create_body(s, -15, -15, 15, 15)
        m = gpu_handle()
        f = np.zeros((8, s.count))
        f[0], f[1], f[2], f[3] = F
        m.set_fields(f)
        m.step(s, .001)
        v = float(np.abs(np.concatenate([s.vx[:s.count], s.vy[:s.count]])).max())
        assert (v > 1e-3) if moves else (v < 1e-4), (F, v)
        m.close()


@pytest.mark.gpu
def test_gpu_ignores_liquid_particles():
    s = empty()
    for i in range(6):
        s.add(i * 3.5, 0, 2, 3, -2)
    x, vx = s.x.copy(), s.vx.copy()
    m = gpu_handle()
    m.step(s, .001)
    assert np.array_equal(s.x, x) and np.array_equal(s.vx, vx)
    assert m.hasParticles(s) is False
    assert m.stats(s)["count"] == 0
    m.close()


@pytest.mark.gpu
def test_gpu_panel_preserves_uniform_translation():
    s = empty()
    create_body(s, -15, -15, 15, 15)
    s.vx[:s.count] = 7
    s.vy[:s.count] = -3
    m = gpu_handle()
    assert m.hasParticles(s)
    m.step(s, .001)
    assert np.all(np.abs(s.vx[:s.count] - 7) <= 7e-6) and np.all(np.abs(s.vy[:s.count] + 3) <= 3e-6)
    assert m.stats(s)["strain"] < 1e-6
    m.close()


@pytest.mark.gpu
@pytest.mark.parametrize("rough", [False, True])
def test_gpu_one_step_matches_oracle(rough):
    tol = 1e-6  # normwise relative
    s, fields = random_panel(rough=rough)
    t = copy_sim(s)
    o = Oracle2(s.capacity)
    o.fields[:, :s.count] = fields
    m = gpu_handle()
    m.set_fields(fields)
    dt = 1e-3
    assert abs(m.stableStep(s) - o.stable_step(t)) <= 1e-6 * o.stable_step(t)
    m.step(s, dt)
    o.step(t, dt)
    n = s.count
    g = m.fields(n)
    vmax = float(np.abs(np.concatenate([t.vx[:n], t.vy[:n]])).max())
    for a, b in ((s.vx, t.vx), (s.vy, t.vy)):
        assert np.abs(a[:n] - b[:n]).max() <= tol * vmax
    for a, b in ((s.x, t.x), (s.y, t.y)):
        assert np.abs(a[:n].astype(np.float64) - b[:n]).max() <= 1e-6 * EXTENT
    assert np.abs(g[:4] - o.fields[:4, :n]).max() <= tol * np.abs(o.fields[:4, :n]).max()
    assert np.abs(g[4:] - o.fields[4:, :n]).max() <= tol * vmax * 4 / 8
    m.close()


@pytest.mark.gpu
def test_gpu_stretched_release_matches_oracle_over_120_frames():
    s, reference = stretched_panel()
    t = copy_sim(s)
    o = Oracle2(s.capacity)
    o.fields[0, :s.count] = 1.25
    m = gpu_handle()
    f = m.fields(s.count)
    f[0] = 1.25
    m.set_fields(f)
    stretched = width(s)
    lo, speed, subs_gpu, subs_cpu = math.inf, 0.0, 0, 0
    for _ in range(120):
        ng, ag = m.frame(s)
        nc, ac = o.frame(t)
        subs_gpu += ng
        subs_cpu += nc
        assert abs(ag - ac) < 1e-9
        lo = min(lo, width(s))
        speed = max(speed, float(np.abs(s.vx[:s.count]).max()))
    n = s.count
    assert np.abs(s.x[:n].astype(np.float64) - t.x[:n]).max() <= 1e-4 * EXTENT
    assert np.abs(s.y[:n].astype(np.float64) - t.y[:n]).max() <= 1e-4 * EXTENT
    assert abs(subs_gpu - subs_cpu) <= 0.02 * subs_cpu
    assert lo < reference * 1.1 and lo < stretched * .9 and speed > 1
    sg, sc = m.stats(s), o.stats(t)
    assert sg["count"] == sc["count"] and sg["minJ"] > 0
    for k in ("minJ", "maxJ"):
        assert abs(sg[k] - sc[k]) <= 1e-3, k
    m.close()


@pytest.mark.gpu
def test_gpu_anchored_body_deforms_recoils_and_keeps_pins():
    s = anchored_panel()
    m = gpu_handle()
    pins = [(i, s.x[i], s.y[i]) for i in range(s.count) if s.pinned[i]]
    tip = 23
    initial = float(s.y[tip])
    loaded = -math.inf
    for _ in range(120):
        m.frame(s)
        loaded = max(loaded, float(s.y[tip]))
    assert loaded > initial + 8 and m.stats(s)["strain"] > .05
    lo = math.inf
    for _ in range(180):
        m.frame(s)
        lo = min(lo, float(s.y[tip]))
    assert lo < loaded - 5
    for i, x, y in pins:
        assert math.hypot(s.x[i] - x, s.y[i] - y) < 1e-5
    m.close()


@pytest.mark.gpu
def test_gpu_frame_with_gravity_and_walls_matches_oracle():
    s, fields = random_panel(9)
    t = copy_sim(s)
    o = Oracle2(s.capacity)
    o.fields[:, :s.count] = fields
    m = gpu_handle()
    m.set_fields(fields)
    for _ in range(30):
        ng, ag = m.frame(s)
        nc, ac = o.frame(t)
    n = s.count
    assert np.abs(s.x[:n].astype(np.float64) - t.x[:n]).max() <= 1e-4 * EXTENT
    assert np.abs(s.y[:n].astype(np.float64) - t.y[:n]).max() <= 1e-4 * EXTENT
    assert np.all(np.abs(s.x[:n]) <= 170) and np.all(np.abs(s.y[:n]) <= 145)
    assert m.stats(s)["nodes"] == o.stats(t)["nodes"]
    m.close()


@pytest.mark.gpu
def test_gpu_delete_reuse_reset_keep_deformation_indices():
    # tests/solid-mpm.test.mjs:62-66
    s = empty()
    m = gpu_handle()
    s.mpm = m
    s.add(0, 0, 11)
    s.add(5, 0, 11)
    f = m.fields(2)
    f[FIELDS.index("f01"), 1] = .3
    m.set_fields(f)
    s.remove_at(0)
    assert abs(m.field("f01", 2)[0] - .3) < 1e-7
    s.add(10, 0, 11)
    assert m.field("f01", 2)[1] == 0 and m.field("f00", 2)[1] == 1
    s.count = s.capacity - 2
    assert m.create(s, 0, 0, 20, 20) is False and s.count == s.capacity - 2
    m.reset()
    assert m.field("f01", 1)[0] == 0 and m.field("f00", 1)[0] == 1
    m.close()


@pytest.mark.gpu
def test_gpu_empty_and_invalid_calls():
    from mpm_b200 import _lib
    s = empty()
    m = gpu_handle(64)
    m.step(s, .001)
    assert m.stats(s) == dict(count=0, minJ=1.0, maxJ=1.0, strain=0.0, nodes=0, substeps=0)
    s2 = empty(128)
    s2.count = 100  # more than the handle's capacity
    with pytest.raises(_lib.MpmError):
        m.step(s2, .001)
    s.settings["gravity"] = "self"
    with pytest.raises(_lib.MpmError):
        m.frame(s)
    m.close()
