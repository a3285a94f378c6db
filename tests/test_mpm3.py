"""MPM3 facade (src/three/mpm.js:7-136): the reference's method names over the C ABI.

One `MPM3.step(s, dt)` with the caller's FP64 arrays must match one FP64 oracle step within the
one-step tolerances of the fused path (x within 1e-6 m, v within 1e-6 relative).
"""
import numpy as np
import pytest

from mpm_b200 import scenes
from mpm_b200.mpm3 import Sim3
from mpm_b200.params import Domain


def sim_from_scene(sc):
    s = Sim3(sc.n + 16)
    for i in range(sc.n):
        s.add(*sc.x[i], mass=sc.m[i], volume=sc.V[i], material=int(sc.mat[i]), v=tuple(sc.v[i]))
    return s


def test_sim3_add_and_remove_follow_simulation3():
    s = Sim3(8)
    for k in range(5):
        assert s.add(k, 2 * k, 3 * k, mass=1 + k, volume=.1)
    last = s.remove(1)
    assert last == 4 and s.count == 4
    assert (s.x[1], s.y[1], s.mass[1]) == (4, 8, 5)
    while s.count < s.capacity:
        s.add(0, 0, 0, mass=1, volume=1)
    assert s.add(0, 0, 0, mass=1, volume=1) is False


def moving_cube():
    sc = scenes.elastic_cube()
    d = sc.domain
    # the reference adds gravity to particle velocities before MPM3.step: zero on the grid here
    dom = Domain(lower=d.lower, upper=d.upper, H=d.H, gravity=(0, 0, 0), sticky_floor=d.sticky_floor)
    sc = scenes.Scene(name="cube", domain=dom, materials=sc.materials, x=sc.x, v=sc.v.copy(), m=sc.m, V=sc.V,
                      mat=sc.mat)
    rng = np.random.default_rng(4)
    sc.v[:] = rng.uniform(-0.5, 0.5, sc.v.shape)
    return sc


@pytest.mark.gpu
def test_mpm3_step_matches_oracle():
    from mpm_b200.mpm3 import MPM3
    from oracle import oracle as orc
    sc = moving_cube()
    s = sim_from_scene(sc)
    m = MPM3(s.capacity, sc.domain, {0: sc.materials[0]})
    dt = 1e-4
    st = orc.state_from_scene(sc)
    assert abs(m.stableStep(s) - st.stable_dt()) <= 1e-6 * st.stable_dt()
    m.step(s, dt)
    st.step(dt)
    n = s.count
    x = np.stack([s.x[:n], s.y[:n], s.z[:n]], 1)
    v = np.stack([s.vx[:n], s.vy[:n], s.vz[:n]], 1)
    assert np.max(np.abs(x - st.x)) <= 1e-6
    assert np.max(np.abs(v - st.v)) <= 1e-6 * np.max(np.abs(st.v))
    m.close()


@pytest.mark.gpu
def test_mpm3_state_methods():
    from mpm_b200.mpm3 import MPM3
    sc = moving_cube()
    s = sim_from_scene(sc)
    m = MPM3(s.capacity, sc.domain, {0: sc.materials[0]})
    assert m.minJ(s) == 1.0
    diag = m.refreshDiagnostics(s)
    assert abs(diag["mass"] - sc.m.sum()) <= 1e-9 * sc.m.sum() and diag["count"] == sc.n
    for _ in range(3):
        m.step(s, 1e-4)
    m.resetParticle(7)
    last = s.remove(2)
    m.remove(2, last)
    m.step(s, 1e-4)
    assert m.refreshDiagnostics(s)["count"] == sc.n - 1
    assert 0.9 < m.minJ(s) <= 1.0 + 1e-3
    assert m.frame(s, 1e-3) >= 1
    m.close()


@pytest.mark.gpu
def test_mpm3_regularize_solids_on_caller_positions():
    """regularizeSolids(s, dt) through the facade: tests/solid-sampling.test.mjs:7-15 on Sim3 arrays."""
    from mpm_b200.mpm3 import MPM3
    from mpm_b200.params import Material
    s = Sim3(8)
    s.add(-.5, 0, 0, mass=2.7, volume=1)
    s.add(.5, 0, 0, mass=3.0, volume=1)
    s.vx[:2] = 7
    m = MPM3(s.capacity, materials={0: Material.reference_units(0)})
    m.setRegularizer(True)
    for _ in range(60):
        m.regularizeSolids(s, 1 / 120)
    assert s.x[1] - s.x[0] > 2.79
    assert list(s.vx[:2]) == [7, 7]
    m.setRegularizer(False)
    x = s.x[:2].copy()
    m.regularizeSolids(s, 1 / 120)
    assert np.array_equal(s.x[:2], x)
    m.close()


@pytest.mark.gpu
def test_mpm3_exchange_heat_updates_caller_temperatures():
    """exchangeHeat through the facade: tests/three.test.mjs:27-31 (contact by 3D distance)."""
    from mpm_b200.mpm3 import MPM3
    from mpm_b200.params import Material
    s = Sim3(8)
    s.add(0, 0, 0, mass=1.0, volume=1, temperature=80.0)
    s.add(0, 0, 20, mass=1.0, volume=1, temperature=20.0)
    water = Material(model=0, mu=.4, lam=.4, specific_heat=4180.0, conductivity=.6)
    m = MPM3(s.capacity, materials={0: water})
    assert m.exchangeHeat(s, 1 / 60) == 0.0
    assert s.temperature[0] == 80 and s.temperature[1] == 20
    m.close()
    s.z[1] = 5
    m = MPM3(s.capacity, materials={0: water})
    e0 = 4180.0 * (80 + 20)
    for _ in range(30):
        m.exchangeHeat(s, 1 / 60)
    assert s.temperature[0] < 80 and s.temperature[1] > 20
    assert abs(float(np.sum(s.enthalpy[:2])) - e0) <= 1e-6 * e0
    m.close()


def oracle_frame(st, dt_frame, max_substeps=48):
    """Simulation3.step's sub-stepping (src/three/simulation.js:305-311) on the oracle: substeps of
    the stable dt, the last one taking exactly what is left."""
    left, n = dt_frame, 0
    while left > 1e-6 * dt_frame and n < max_substeps:
        dt = min(st.stable_dt(), left)
        if left - dt <= 1e-6 * dt_frame:
            dt = left
        st.step(dt)
        left -= dt
        n += 1
    return n


@pytest.mark.gpu
def test_mpm3_frames_match_oracle_substeps():
    """MPM3.frame (mpm_frame_host) over four frames against the oracle's sub-stepping: the same
    substep counts, x within 1e-5 m and v within 1e-5 relative after every frame. The frame's last
    substep skips the scatter the next upload would discard; the third frame multiplies the
    caller's velocities by 30, so the substep count carried over from the previous frame falls
    short and the call scatters the state again and tops the count up."""
    from mpm_b200.mpm3 import MPM3
    from oracle import oracle as orc
    sc = moving_cube()
    s = sim_from_scene(sc)
    m = MPM3(s.capacity, sc.domain, {0: sc.materials[0]})
    st = orc.state_from_scene(sc)
    n = s.count
    dt_frame = 3.5 * st.stable_dt()
    subs = []
    for frame in range(4):
        if frame == 2:
            s.vx[:n] *= 30.0
            s.vy[:n] *= 30.0
            s.vz[:n] *= 30.0
            st.v = np.ascontiguousarray(np.stack([s.vx[:n], s.vy[:n], s.vz[:n]], 1))
        sub = m.frame(s, dt_frame)
        sub_ref = oracle_frame(st, dt_frame)
        assert sub == sub_ref, (frame, sub, sub_ref)
        if frame == 2:
            assert sub > subs[-1]  # more substeps than the carried-over count
        subs.append(sub)
        x = np.stack([s.x[:n], s.y[:n], s.z[:n]], 1)
        v = np.stack([s.vx[:n], s.vy[:n], s.vz[:n]], 1)
        assert np.max(np.abs(x - st.x)) <= 1e-5, frame
        assert np.max(np.abs(v - st.v)) <= 1e-5 * np.max(np.abs(st.v)), frame
        # the device F and C of the frame's final gather-only substep match the oracle too
        out = m.solver.download(("F", "C"))
        assert np.max(np.abs(out["F"] - st.F)) <= 1e-5, frame
    m.close()
