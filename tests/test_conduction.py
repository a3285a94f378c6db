"""Grid heat conduction of the coupled scene (mpm_set_conduction).

The scheme has no counterpart in the reference's solid step, so the FP64 oracle's restatement is
pinned by properties that hold for it: the heat sum m cp T is conserved exactly (the node
conductances are symmetric, and particles take the interpolated node increments plus a relaxation
toward the interpolated node temperature, both of which keep the sum), no particle leaves the
initial temperature range, a uniform field stays stationary, and two bodies at different
temperatures relax to their common temperature. The device (FP32) is checked
against the oracle on the same inputs: temperatures within 1e-5 of the initial temperature range.
"""
import os

import numpy as np
import pytest

from mpm_b200 import scenes
from mpm_b200.params import Domain, Material, MODEL_FIXED_COROTATED
from oracle import oracle as orc

K_TEST = 5e5  # W/m/K: alpha dt / h^2 = 0.05 per step at h = 1/32, dt = 1e-4, rho = cp = 1000


def hot_cold_block(T_hot=400.0, T_cold=300.0):
    d = Domain(lower=(0, 0, 0), upper=(1, 1, 1), H=1 / 32, gravity=(0, 0, 0), sticky_floor=False)
    mat = Material.from_young(MODEL_FIXED_COROTATED, 1e5, 0.3, density=1000.0, specific_heat=1000.0)
    x = scenes.block_particles(d, (10, 10, 10), (22, 16, 16), 3)
    sc = scenes._scene("hot_cold", d, [mat], x, (0, 0, 0),
                       meta=dict(conduction=dict(k=K_TEST, rho=1000.0, cp=1000.0)))
    sc.T = np.where(x[:, 0] < 16 / 32, T_hot, T_cold)
    return sc


def heat(st):
    return float(np.sum(st.m * st.T))


def test_oracle_conserves_heat_and_respects_the_maximum_principle():
    sc = hot_cold_block()
    st = orc.state_from_scene(sc)
    h0 = heat(st)
    spread = [st.T.max() - st.T.min()]
    for _ in range(30):
        st.step(1e-4)
        assert abs(heat(st) - h0) <= 1e-12 * h0
        assert st.T.min() >= 300.0 - 1e-9 and st.T.max() <= 400.0 + 1e-9
        spread.append(st.T.max() - st.T.min())
    # the two halves exchange heat: the hot side cools, the cold side warms
    hot = sc.x[:, 0] < 16 / 32
    assert st.T[hot].mean() < 400.0 - 1.0 and st.T[~hot].mean() > 300.0 + 1.0
    assert spread[-1] <= spread[0]


def test_oracle_relaxes_to_the_common_temperature():
    sc = hot_cold_block()
    st = orc.state_from_scene(sc)
    for _ in range(600):
        st.step(1e-4)
    mean = heat(st) / float(np.sum(st.m))
    assert abs(mean - 350.0) <= 1e-9 and np.max(np.abs(st.T - mean)) <= 0.5


def test_oracle_uniform_field_is_stationary():
    sc = hot_cold_block(350.0, 350.0)
    st = orc.state_from_scene(sc)
    for _ in range(5):
        st.step(1e-4)
    assert np.max(np.abs(st.T - 350.0)) <= 1e-9


def test_oracle_dt_limit_includes_diffusion():
    sc = hot_cold_block()
    st = orc.state_from_scene(sc)
    h = sc.domain.H
    assert st.stable_dt() <= 0.9 * 1000.0 * 1000.0 * h * h / (6 * K_TEST) * (1 + 1e-12)


@pytest.mark.gpu
def test_device_conduction_matches_oracle():
    from mpm_b200.solver import Solver
    sc = hot_cold_block()
    s = Solver(sc.domain, sc.n)
    s.upload(sc)
    st = orc.state_from_scene(sc)
    for _ in range(20):
        st.step(1e-4)
    s.step_fixed(1e-4, 20)
    out = s.download()
    assert np.max(np.abs(out["T"] - st.T)) <= 1e-5 * 100.0
    assert np.max(np.abs(out["x"] - st.x)) <= 1e-6
    assert abs(np.sum(sc.m * out["T"]) - heat(st)) <= 1e-6 * heat(st)
    s.close()


@pytest.mark.gpu
def test_coupled_subsample_prefix_matches_oracle():
    """The coupled scene's seed-matched 1/64 subsample: 100 steps against the FP64 oracle."""
    from mpm_b200.solver import Solver
    sc = scenes.coupled_collision(scale=4)
    dt = sc.meta["dt"]
    s = Solver(sc.domain, sc.n)
    s.upload(sc)
    st = orc.state_from_scene(sc)
    threads = os.cpu_count() or 1
    for _ in range(100):
        st.step(dt, threads=threads)
    s.step_fixed(dt, 100)
    out = s.download()
    assert np.max(np.abs(out["x"] - st.x)) <= 1e-4
    assert np.max(np.abs(out["v"] - st.v)) <= 1e-3 * 20.0
    assert np.max(np.abs(out["T"] - st.T)) <= 1e-3
    assert np.max(np.abs(out["ep"] - st.ep)) <= 1e-5 + 1e-3 * np.max(st.ep)
    assert s.status() == 0
    s.close()
