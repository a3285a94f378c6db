"""The learned return map inside the fused step (mpm_set_return_mode), GPU tests through the C ABI.

A Johnson-Cook network (model 7) is trained on the GPU from the exact bisection's roots, then a
plastic impact steps with it against the FP64 oracle (which runs the reference's 24-halving
bisection, src/three/metal-plasticity.js:28-34). Bounds are those of the exact step's parity tests:
x within 1e-6 m, F within 2e-6, plastic strain within 2e-6 + 1e-4 max ep after ten substeps. The
gate accepts a refined prediction only when its consistency residual is at most gate_tol (1e-5) of
the trial stress, so the learned step carries the same stated stress error as the exact one.
What the trained network gains over the method without it: the share of plastic returns it serves
(the rest run the bisection), against an untrained network of the same shape (about 98% against
about half in the impact). The Newton-gated mode runs the same refinement and gate from a guess
taken from the initial flow stress, with no network, under the same bounds.
"""
import numpy as np
import pytest

from oracle import oracle as orc
from mpm_b200 import scenes
from mpm_b200.solver import Solver
from mpm_b200.surrogate import Surrogate, jc_config

pytestmark = pytest.mark.gpu

GATE_TOL = 1e-5


def impact_scene(model=7):
    return scenes.jc_impact(shape=(12, 6, 12), grid=32, model=model, v0=-60.0)


@pytest.fixture(scope="module")
def trained():
    s = Surrogate(scenes.johnson_cook_metal(7), seed=3)
    hist = s.train(jc_config(samples=2_000_000, steps=6000))
    assert np.all(np.isfinite(hist)) and hist[-100:].mean() < 0.1 * hist[:10].mean()
    yield s
    s.close()


def run(sc, surrogate, substeps=10, dt=1e-6):
    sol = Solver(sc.domain, sc.n)
    sol.upload(sc)
    if surrogate is not None:
        sol.set_return_mode(surrogate, gate_tol=GATE_TOL, newton=4)
    sol.step_fixed(dt, substeps)
    out = sol.download()
    counts = sol.gate_counts()
    assert sol.status() == 0
    sol.close()
    return out, counts


def oracle_run(sc, substeps=10, dt=1e-6):
    st = orc.state_from_scene(sc)
    for _ in range(substeps):
        st.step(dt)
    return st


def check_parity(out, st):
    assert np.max(st.ep) > 0  # the impact yields
    assert np.max(np.abs(out["x"] - st.x)) <= 1e-6
    assert np.max(np.abs(out["F"] - st.F)) <= 2e-6
    assert np.max(np.abs(out["ep"] - st.ep)) <= 2e-6 + 1e-4 * np.max(st.ep)


def test_learned_step_matches_oracle_and_serves_most_returns(trained):
    sc = impact_scene()
    st = oracle_run(sc)
    out, (learned, fallback) = run(sc, trained)
    check_parity(out, st)
    assert learned + fallback > 500
    assert learned >= 0.8 * (learned + fallback), (learned, fallback)


def test_untrained_network_serves_fewer_returns_and_stays_exact(trained):
    """The same gate with an untrained network: the step is still within the oracle bounds (the gate
    sends what it cannot vouch for to the bisection). The Newton refinement alone carries about half
    the returns through the gate from an untrained guess; the trained network raises that share to
    nearly all of them (what the network gains over the method without it)."""
    s = Surrogate(scenes.johnson_cook_metal(7), seed=3)
    sc = impact_scene()
    st = oracle_run(sc)
    out, (learned, fallback) = run(sc, s)
    s.close()
    check_parity(out, st)
    assert learned + fallback > 500
    _, (lt, ft) = run(sc, trained)
    share_untrained, share_trained = learned / (learned + fallback), lt / (lt + ft)
    assert share_trained >= share_untrained + 0.25, (share_untrained, share_trained)


def test_learned_step_on_dense_tiles_matches_oracle(trained):
    """27 particles per cell (three scatter rounds per tile) in learned mode: the oracle bounds
    after ten substeps and most returns served."""
    from test_gpu_parity import dense_j2_scene
    sc = dense_j2_scene(material=scenes.johnson_cook_metal(7))
    st = oracle_run(sc)
    out, (learned, fallback) = run(sc, trained)
    check_parity(out, st)
    assert learned + fallback > 1000
    assert learned >= 0.8 * (learned + fallback), (learned, fallback)


def test_newton_gated_step_without_a_network_matches_oracle():
    """The same refinement and gate started from the initial flow stress's guess, u0 = 1 - flow(ep,
    0, T) / q, with no network (mpm_set_return_mode with MPM_RETURN_NEWTON_GATED): within the oracle
    bounds after ten substeps, and with eight Newton steps it serves nearly every return."""
    sc = impact_scene()
    st = oracle_run(sc)
    sol = Solver(sc.domain, sc.n)
    sol.upload(sc)
    sol.set_return_mode(mode="newton", gate_tol=GATE_TOL, newton=8)
    sol.step_fixed(1e-6, 10)
    out = sol.download()
    served, fallback = sol.gate_counts()
    assert sol.status() == 0
    sol.close()
    check_parity(out, st)
    assert served + fallback > 500
    assert served >= 0.95 * (served + fallback), (served, fallback)


def test_exact_mode_restores_the_reference_map(trained):
    sc = impact_scene()
    sol = Solver(sc.domain, sc.n)
    sol.upload(sc)
    sol.set_return_mode(trained, gate_tol=GATE_TOL)
    sol.set_return_mode(None)
    sol.step_fixed(1e-6, 10)
    out = sol.download()
    assert sol.gate_counts() == (0, 0)
    sol.close()
    check_parity(out, oracle_run(sc))


def test_thermal_johnson_cook_learned_step():
    """Model 6 with thermal softening on a 500 K block: a network trained for model 6."""
    s = Surrogate(scenes.johnson_cook_metal(6), seed=5)
    s.train(jc_config(samples=2_000_000, steps=6000))
    sc = impact_scene(model=6)
    sc.T = np.full(sc.n, 500.0)
    st = oracle_run(sc)
    out, (learned, fallback) = run(sc, s)
    s.close()
    check_parity(out, st)
    np.testing.assert_allclose(out["T"], st.T, rtol=1e-6, atol=1e-3)
    assert learned >= 0.6 * (learned + fallback), (learned, fallback)


def test_learned_mode_on_a_batch_matches_single_handles(trained):
    """A batch of Johnson-Cook scenes in learned mode against each scene's own handle in learned
    mode (same network and gate): x within 1e-6 m."""
    from mpm_b200.solver import Batch
    sc_all = scenes.ensemble(6, model=7)
    b = Batch(sc_all)
    b.upload()
    b.set_return_mode(trained, gate_tol=GATE_TOL)
    b.run(5, graph=True)
    parts = b.split(b.download(("x", "ep")))
    assert b.status() == 0
    b.close()
    for k, sc in enumerate(sc_all):
        sol = Solver(sc.domain, sc.n)
        sol.upload(sc)
        sol.set_return_mode(trained, gate_tol=GATE_TOL)
        sol.step_cfl(5)
        out = sol.download(("x", "ep"))
        sol.close()
        assert np.max(np.abs(parts[k]["x"] - out["x"])) <= 1e-6, k
        assert np.max(np.abs(parts[k]["ep"] - out["ep"])) <= 2e-6 + 1e-4 * max(np.max(out["ep"]), 0.0), k


def test_kernel_level_timing_reports_counts(trained):
    """mpm_surrogate_time on random Johnson-Cook trial states: both maps run, and the gate serves
    most plastic states."""
    r = trained.time(1_000_000, iters=2, gate_tol=GATE_TOL, cfg=jc_config())
    assert r["ms_exact"] > 0 and r["ms_learned"] > 0
    plastic = r["learned"] + r["fallback"]
    assert plastic > 100_000
    assert r["learned"] >= 0.8 * plastic, r


def test_newton_gated_standalone_map_reports_counts(trained):
    """mpm_surrogate_time_newton on the same random Johnson-Cook states: the network-free map runs
    and its gate accepts nearly every plastic state within eight Newton steps."""
    r = trained.time_newton(1_000_000, iters=2, gate_tol=GATE_TOL, cfg=jc_config())
    assert r["ms"] > 0
    plastic = r["accepted"] + r["fallback"]
    assert plastic > 100_000
    assert r["accepted"] >= 0.95 * plastic, r
