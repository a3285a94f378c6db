"""Snow (2), sand (3), cohesive Drucker-Prager (8) and Deshpande-Fleck foam (9) through the fused
device step, against the FP64 oracle (GPU tests, through the C ABI).

A soft block (E = 1 MPa, the reference's mu = lambda = 0.4 E and default strengths) drops at 3 m/s
onto a sticky floor while stretching and shearing sideways, so every law yields in the first steps.
Tolerances: grid mass and momentum after one P2G <= 1e-6 normwise; after 10 steps positions within
1e-6 m, F within 2e-6, plastic strain within 2e-6 + 1e-4 of its maximum, Jp and dilation within
1e-5 (FP32 state against FP64).
"""
import numpy as np
import pytest

from oracle import oracle as orc
from mpm_b200 import scenes
from mpm_b200.params import Material
from mpm_b200.solver import Solver

pytestmark = pytest.mark.gpu

MODELS = (2, 3, 8, 9)


def rel(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    s = float(np.max(np.abs(b)))
    return float(np.max(np.abs(a - b)) / (s if s > 0 else 1.0))


def soft_block(model, v0=-3.0, stretch=20.0, jp=None, dilation=None):
    """The block also stretches sideways at `stretch` 1/s and shears, so the laws that do not yield
    in compression (cohesive Drucker-Prager) reach their tension and shear limits."""
    d = scenes.Domain(lower=(0, 0, 0), upper=(1, 1, 1), H=1 / 32, gravity=(0, -9.8, 0), sticky_floor=True)
    mat = Material.reference_units(model, E=1e6, density=1000.0)
    x = scenes.block_particles(d, (10, 1, 10), (22, 7, 22), 5)
    sc = scenes._scene(f"soft_{model}", d, [mat], x, (0, v0, 0))
    r = x - x.mean(axis=0)
    sc.v = sc.v + stretch * np.stack([r[:, 0] + 0.5 * r[:, 1], np.zeros(len(r)), r[:, 2]], axis=1)
    if jp is not None:
        sc.jp = np.full(sc.n, jp)
    if dilation is not None:
        sc.dilation = np.full(sc.n, dilation)
    return sc


@pytest.mark.parametrize("model", MODELS)
def test_impact_matches_oracle(model):
    sc = soft_block(model)
    dt = 1e-4
    sol = Solver(sc.domain, sc.n)
    sol.upload(sc)
    st = orc.state_from_scene(sc)
    gm_ref, gp_ref, _ = st.step(dt, want_grid=True)
    gm, gp = sol.grid_debug(dt)
    assert rel(gm, gm_ref) <= 1e-6
    assert rel(gp, gp_ref) <= 1e-6
    sol.step_fixed(dt, 1)
    for _ in range(9):
        st.step(dt)
    sol.step_fixed(dt, 9)
    out = sol.download(("x", "v", "F", "ep", "jp", "dilation"))
    assert np.max(st.ep) > 0  # the impact yields
    assert np.max(np.abs(out["x"] - st.x)) <= 1e-6
    assert np.max(np.abs(out["F"] - st.F)) <= 2e-6
    assert np.max(np.abs(out["ep"] - st.ep)) <= 2e-6 + 1e-4 * np.max(st.ep)
    np.testing.assert_allclose(out["jp"], st.jp, atol=1e-5, rtol=0)
    np.testing.assert_allclose(out["dilation"], st.dilation, atol=1e-5, rtol=0)
    assert sol.status() == 0
    if model in (2, 8, 9):
        assert np.max(np.abs(st.jp - 1)) > 1e-4  # the history scalar moved
    sol.close()


@pytest.mark.parametrize("model", (2, 9))
def test_uploaded_history_round_trips_and_drives_the_step(model):
    """A non-default Jp is uploaded, read back and used (snow's hardening, foam's J Jp)."""
    sc = soft_block(model, jp=0.8)
    sol = Solver(sc.domain, sc.n)
    sol.upload(sc)
    out = sol.download(("jp", "dilation"))
    np.testing.assert_allclose(out["jp"], 0.8, atol=1e-7)
    assert np.all(out["dilation"] == 0)
    st = orc.state_from_scene(sc)
    assert abs(sol.stable_dt() - st.stable_dt()) <= 1e-5 * st.stable_dt()
    dt = 1e-4
    for _ in range(5):
        st.step(dt)
    sol.step_fixed(dt, 5)
    out = sol.download(("x", "F", "jp"))
    assert np.max(np.abs(out["x"] - st.x)) <= 1e-6
    assert np.max(np.abs(out["F"] - st.F)) <= 2e-6
    np.testing.assert_allclose(out["jp"], st.jp, atol=1e-5, rtol=0)
    sol.close()


def test_sand_dilation_round_trips_and_reset_clears_history():
    sc = soft_block(3, v0=0.0, stretch=0.0, dilation=0.01)
    sol = Solver(sc.domain, sc.n)
    sol.upload(sc)
    out = sol.download(("jp", "dilation"))
    np.testing.assert_allclose(out["dilation"], 0.01, atol=1e-8)
    assert np.all(out["jp"] == 1)
    sol.reset_particle(3)
    out = sol.download(("dilation",))
    assert out["dilation"][3] == 0 and out["dilation"][4] != 0
    sol.close()


def test_ledger_of_snow_matches_oracle():
    sc = soft_block(2)
    dt = 1e-4
    sol = Solver(sc.domain, sc.n)
    sol.upload(sc)
    st = orc.state_from_scene(sc)
    for _ in range(6):
        st.step(dt)
    sol.step_fixed(dt, 6)
    L, R = sol.ledger(), st.ledger()
    assert abs(L.mass - R.mass) <= 1e-6 * R.mass
    assert abs(L.kinetic - R.kinetic) <= 1e-5 * R.kinetic
    assert abs(L.elastic - R.elastic) <= 1e-3 * abs(R.elastic) + 1e-12
    assert abs(L.max_von_mises - R.max_von_mises) <= 1e-3 * R.max_von_mises
    sol.close()
