"""Parity of the device MLS-MPM step with the FP64 oracle (GPU tests, through the C ABI).

Tolerances (FP32 device state vs FP64 oracle, normwise: max |gpu - oracle| / max |oracle| per field):
  one step          grid mass and momentum <= 1e-6, particle v, C, F, x <= 1e-6 (x: of domain size)
  50 steps          positions within 1e-4 of the domain size
  return map        F within atol 4e-6 / rtol 4e-5 and plastic strain within 1e-5, the tolerances of
                    the reference's own CPU/GPU return-map test (gpu/test_metal_plasticity.py:31-33)
"""
import math

import numpy as np
import pytest

from oracle import oracle as orc
from mpm_b200 import scenes
from mpm_b200.params import Material
from mpm_b200.solver import Solver, return_map_batch

pytestmark = pytest.mark.gpu


def rel(a, b, floor=0.0):
    """max |a - b| / max(max |b|, floor): normwise relative error with an absolute scale floor for
    fields that are pure rounding noise in the FP64 oracle (e.g. C of a uniform velocity field)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = max(float(np.max(np.abs(b))), floor)
    return float(np.max(np.abs(a - b)) / (scale if scale > 0 else 1.0))


def c_scale(v, H):
    """Natural scale of the APIC matrix: a velocity difference of max |v| across a cell (4/h)."""
    return float(np.max(np.abs(v))) * 4.0 / H


def run_pair(scene, dt, steps, capacity=None):
    sol = Solver(scene.domain, capacity or scene.n)
    sol.upload(scene)
    st = orc.state_from_scene(scene)
    for _ in range(steps):
        st.step(dt)
    sol.step_fixed(dt, steps)
    return sol, st


def small_j2_scene(v0=-60.0, model=5, grid=32, block=(12, 6, 12), seed=7):
    d = scenes.Domain(lower=(0, 0, 0), upper=(1, 1, 1), H=1 / grid, gravity=(0, -9.8, 0), sticky_floor=True)
    mat = scenes.aluminium_j2(model)
    x = scenes.block_particles(d, (10, 1, 10), (10 + block[0], 1 + block[1], 10 + block[2]), seed)
    return scenes._scene("j2_small", d, [mat], x, (0, v0, 0))


# ---- constitutive batch: the reference's own GPU parity cases ------------------------------------

def metal_cases():
    # gpu/metal_reference.mjs:1-9: models 4-7 x T x dt
    F = [1.3, .1, 0, 0, .8, 0, 0, 0, 1 / 1.04]
    for model in (4, 5, 6, 7):
        for temp in (20, 650, 1100):
            for dt in (.001, .02):
                yield model, temp, dt, F


def test_return_map_batch_matches_reference_metal_cases():
    for model, temp, dt, F in metal_cases():
        mat = Material.reference_units(model, A=.03, B=.12)
        omat = orc.material_from(mat)
        Fo_ref, inc_ref, tau_ref = orc.project(F, omat, ep=.15, dt=dt, T=temp)
        Fo, dep, tau = return_map_batch(mat, [F], ep=.15, T=temp, dt=dt)
        np.testing.assert_allclose(Fo[0], Fo_ref, atol=4e-6, rtol=4e-5)
        assert abs(.15 + dep[0] - (.15 + inc_ref)) < 1e-5
        np.testing.assert_allclose(tau[0], orc.constitutive_stress(Fo_ref, model, .4, .4), atol=3e-6, rtol=5e-4)


def test_return_map_batch_matches_reference_thermal_cases():
    # gpu/thermal_reference.mjs:1-9 for models 10 and 11
    for model, T, F in [(m, T, F) for m in (10, 11) for T in (-100, 20, 180, 800)
                        for F in ([1, .2, 0, 0, 1, 0, 0, 0, 1], [.9, 0, 0, 0, 1.05, 0, 0, 0, 1])]:
            mat = Material.reference_units(model)
            omat = orc.material_from(mat)
            Fo_ref, inc_ref, _ = orc.project(F, omat, ep=.05, dt=.01, T=T)
            Fo, dep, tau = return_map_batch(mat, [F], ep=.05, T=T, dt=.01)
            np.testing.assert_allclose(Fo[0], Fo_ref, atol=4e-6, rtol=5e-5)
            assert abs(dep[0] - inc_ref) <= 1e-5 + 1e-4 * inc_ref
            vm_ref = orc.von_mises(orc.constitutive_stress(Fo_ref, model, .4, .4), np.linalg.det(np.reshape(Fo_ref, (3, 3))))
            t = tau[0]
            vm = orc.von_mises(t, np.linalg.det(Fo[0].reshape(3, 3)))
            assert abs(vm - vm_ref) < 1e-5


def test_j2_invariants_on_device():
    """tests/metal-plasticity.test.mjs:12-23 on the device map: yield consistency, isochoric flow,
    elastic unloading and hydrostatic loading give no plastic strain."""
    rng = np.random.default_rng(3)
    n = 4096
    F = np.tile(np.eye(3).ravel(), (n, 1)) + 0.05 * rng.standard_normal((n, 9))
    for model in (4, 5):
        mat = Material.reference_units(model)
        Fo, dep, tau = return_map_batch(mat, F, ep=0.0)
        detF = np.linalg.det(F.reshape(-1, 3, 3))
        detFo = np.linalg.det(Fo.reshape(-1, 3, 3))
        np.testing.assert_allclose(detFo, detF, rtol=2e-6)
        yielded = dep > 0
        assert yielded.sum() > 100
        J = detFo[yielded]
        vm = np.array([orc.von_mises(t, j) for t, j in zip(tau[yielded], J)])
        flow = mat.yield_stress + (mat.hardening * dep[yielded] if model == 5 else 0)
        np.testing.assert_allclose(vm, flow, rtol=2e-5)
        _, dep_u, _ = return_map_batch(mat, np.eye(3).ravel()[None], ep=0.1)
        assert dep_u[0] == 0
        Fh, dep_h, _ = return_map_batch(mat, np.diag([.9, .9, .9]).ravel()[None])
        assert dep_h[0] == 0
        assert abs(np.linalg.det(Fh[0].reshape(3, 3)) - .9 ** 3) < 1e-6


# ---- one step and 50 steps against the oracle ------------------------------------------------------

def test_elastic_cube_one_step_grid_and_particles():
    sc = scenes.elastic_cube()
    dt = sc.meta["dt"]
    sol = Solver(sc.domain, sc.n)
    sol.upload(sc)
    st = orc.state_from_scene(sc)
    gm_ref, gp_ref, _ = st.step(dt, want_grid=True)
    gm, gp = sol.grid_debug(dt)
    assert rel(gm, gm_ref) <= 1e-6
    assert rel(gp, gp_ref) <= 1e-6
    sol.step_fixed(dt, 1)
    out = sol.download()
    assert np.max(np.abs(out["x"] - st.x)) <= 1e-6
    assert rel(out["v"], st.v) <= 1e-6
    assert rel(out["C"], st.C, c_scale(st.v, sc.domain.H)) <= 1e-6
    assert np.max(np.abs(out["F"] - st.F)) <= 1e-6


def test_elastic_cube_fifty_steps_positions():
    sc = scenes.elastic_cube()
    dt = sc.meta["dt"]
    sol, st = run_pair(sc, dt, 50)
    out = sol.download()
    assert np.max(np.abs(out["x"] - st.x)) <= 1e-4  # domain size 1 m
    assert rel(out["v"], st.v) <= 1e-3


def test_j2_plastic_one_step_and_ten_steps():
    sc = small_j2_scene()
    dt = 1e-6
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
    out = sol.download()
    assert np.max(st.ep) > 0  # the impact yields
    assert np.max(np.abs(out["x"] - st.x)) <= 1e-6
    assert np.max(np.abs(out["F"] - st.F)) <= 2e-6
    assert np.max(np.abs(out["ep"] - st.ep)) <= 2e-6 + 1e-4 * np.max(st.ep)


def test_johnson_cook_impact_matches_oracle():
    """Model 6 (rate and temperature dependent, bisection return) through the fused step."""
    sc = small_j2_scene(model=6)
    sc.T = np.full(sc.n, 400.0)
    dt = 1e-6
    sol, st = run_pair(sc, dt, 6)
    out = sol.download()
    assert np.max(st.ep) > 0
    assert np.max(np.abs(out["x"] - st.x)) <= 1e-6
    assert np.max(np.abs(out["F"] - st.F)) <= 2e-6
    assert np.max(np.abs(out["ep"] - st.ep)) <= 2e-6 + 1e-4 * np.max(st.ep)


def test_thermal_j2_with_plastic_heating():
    sc = scenes.thermal_j2(grid=32, block=10, v0=-60.0)
    dt = 1e-6
    sol, st = run_pair(sc, dt, 10)
    out = sol.download()
    assert np.max(st.ep) > 0
    assert np.max(np.abs(out["x"] - st.x)) <= 1e-6
    np.testing.assert_allclose(out["T"], st.T, rtol=1e-6, atol=1e-3)
    assert np.max(np.abs(out["ep"] - st.ep)) <= 2e-6 + 1e-4 * np.max(st.ep)


def test_uniform_translation_preserved_on_device():
    """tests/three.test.mjs:14-21 (uniform motion preserved) at FP32 precision."""
    sc = scenes.translation_block(velocity=(3.0, -2.0, 7.0))
    sol = Solver(sc.domain, sc.n)
    sol.upload(sc)
    sol.step_fixed(1e-3, 1)
    out = sol.download()
    np.testing.assert_allclose(out["v"], np.tile([3.0, -2.0, 7.0], (sc.n, 1)), atol=2e-5, rtol=0)
    assert np.max(np.abs(out["F"] - np.eye(3).ravel())) < 1e-6


def test_ledger_matches_oracle():
    sc = small_j2_scene()
    sol, st = run_pair(sc, 2e-7, 3)
    L = sol.ledger()
    R = st.ledger()
    assert abs(L.mass - R.mass) <= 1e-6 * R.mass
    assert abs(L.kinetic - R.kinetic) <= 1e-5 * R.kinetic
    for a in range(3):
        assert abs(L.momentum[a] - R.momentum[a]) <= 1e-5 * max(abs(R.momentum[1]), 1e-30)
    assert abs(L.elastic - R.elastic) <= 1e-3 * abs(R.elastic) + 1e-12
    assert abs(L.min_j - R.min_j) <= 1e-6
    assert L.nonfinite == 0 and L.invalid_j == 0


def test_requested_dt_substeps_to_cfl():
    sc = small_j2_scene(v0=-2.0)
    sol = Solver(sc.domain, sc.n)
    sol.upload(sc)
    st = orc.state_from_scene(sc)
    dt_cfl = st.stable_dt()
    assert abs(sol.stable_dt() - dt_cfl) <= 1e-5 * dt_cfl
    sub, adv = sol.step(2e-6)
    assert sub == math.ceil(2e-6 / dt_cfl - 1e-9) or sub == math.ceil(2e-6 / dt_cfl - 1e-9) + 1
    assert abs(adv - 2e-6) <= 1e-12


def test_tma_and_plain_gather_agree(monkeypatch):
    sc = small_j2_scene()
    a = Solver(sc.domain, sc.n)
    a.upload(sc)
    a.step_fixed(2e-7, 4)
    monkeypatch.setenv("MPM_B200_NO_TMA", "1")
    b = Solver(sc.domain, sc.n)
    b.upload(sc)
    b.step_fixed(2e-7, 4)
    oa, ob = a.download(), b.download()
    for k in ("x", "v", "F"):
        assert rel(oa[k], ob[k]) <= 1e-6
    assert rel(oa["C"], ob["C"], c_scale(ob["v"], sc.domain.H)) <= 1e-6


def test_warp_specialised_pass_matches_oracle(monkeypatch):
    """The producer/consumer scatter pass (an autotuner candidate): the plastic impact case."""
    monkeypatch.setenv("MPM_B200_WS", "1")
    sc = small_j2_scene()
    dt = 1e-6
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
    out = sol.download()
    assert np.max(np.abs(out["x"] - st.x)) <= 1e-6
    assert np.max(np.abs(out["F"] - st.F)) <= 2e-6
    assert np.max(np.abs(out["ep"] - st.ep)) <= 2e-6 + 1e-4 * np.max(st.ep)
    assert sol.status() == 0


def test_step_host_drop_in_matches_resident_step():
    sc = small_j2_scene()
    a = Solver(sc.domain, sc.n)
    a.upload(sc)
    a.step_fixed(2e-7, 1)
    ref = a.download()
    import ctypes
    from mpm_b200 import _lib
    b = Solver(sc.domain, sc.n)
    b.upload(sc)
    x = [np.ascontiguousarray(sc.x[:, k]) for k in range(3)]
    v = [np.ascontiguousarray(sc.v[:, k]) for k in range(3)]
    P = ctypes.c_void_p
    io = _lib.MpmParticles(dtype=0, x=x[0].ctypes.data_as(P), y=x[1].ctypes.data_as(P), z=x[2].ctypes.data_as(P),
                           vx=v[0].ctypes.data_as(P), vy=v[1].ctypes.data_as(P), vz=v[2].ctypes.data_as(P))
    _lib.check(_lib.lib().mpm_step_host(b.h, ctypes.byref(io), 2e-7), b.h)
    np.testing.assert_allclose(np.stack(x, 1), ref["x"], atol=1e-9, rtol=0)
    np.testing.assert_allclose(np.stack(v, 1), ref["v"], atol=1e-6 * np.max(np.abs(ref["v"])), rtol=0)


def test_checkpoint_roundtrip_and_rollback(tmp_path):
    sc = small_j2_scene()
    a = Solver(sc.domain, sc.n)
    a.upload(sc)
    a.step_fixed(2e-7, 3)
    a.save(tmp_path / "ck.bin")
    a.snapshot()
    before = a.download()
    a.step_fixed(2e-7, 2)
    after = a.download()
    a.rollback()
    back = a.download()
    for k in before:
        np.testing.assert_array_equal(before[k], back[k])
    b = Solver(sc.domain, sc.n)
    b.load(tmp_path / "ck.bin")
    b.step_fixed(2e-7, 2)
    again = b.download()
    for k in ("x", "F", "ep"):
        np.testing.assert_allclose(again[k], after[k], atol=1e-7, rtol=0)


def test_nonfinite_input_reports_error():
    """Fault injection on the host: a NaN velocity makes the step return MPM_ERR_NONFINITE."""
    from mpm_b200._lib import MpmError
    sc = small_j2_scene()
    sc.v[5, 1] = float("nan")
    a = Solver(sc.domain, sc.n)
    a.upload(sc)
    with pytest.raises(MpmError) as e:
        a.step_fixed(2e-7, 1)
    assert e.value.code == -4
    assert a.status() & 1


def dense_j2_scene(ppc_axis=3, grid=32, block=(8, 8, 8), v0=-60.0, seed=11, material=None):
    """A block with ppc_axis^3 particles per cell (27 by default): a 4^3-cell tile then holds 1,728
    particles, more than one scatter round of the fused pass takes, so its tiles run several rounds.
    Aluminium J2 (model 5) unless a material is given."""
    d = scenes.Domain(lower=(0, 0, 0), upper=(1, 1, 1), H=1 / grid, gravity=(0, -9.8, 0), sticky_floor=True)
    rng = np.random.default_rng(seed)
    lo = np.array([10, 1, 10])
    cells = np.stack(np.meshgrid(*[np.arange(b) for b in block], indexing="ij"), -1).reshape(-1, 3) + lo
    sub = (np.stack(np.meshgrid(*[np.arange(ppc_axis)] * 3, indexing="ij"), -1).reshape(-1, 3) + 0.5) / ppc_axis
    q = (cells[:, None, :] + sub[None, :, :]).reshape(-1, 3)
    q += rng.uniform(-0.2, 0.2, q.shape) / ppc_axis
    x = np.asarray(d.lower) + q * d.H
    sc = scenes._scene("j2_dense", d, [material or scenes.aluminium_j2(5)], x, (0, v0, 0))
    sc.m = sc.m * 8 / ppc_axis ** 3
    sc.V = sc.V * 8 / ppc_axis ** 3
    return sc


def test_tiles_over_one_scatter_round_match_oracle():
    """27 particles per cell (1,728 per full tile, three scatter rounds of the fused pass per tile):
    grid after the first scatter, then one and ten J2 impact steps, within the one-step bounds."""
    sc = dense_j2_scene()
    dt = 1e-6
    sol = Solver(sc.domain, sc.n)
    sol.upload(sc)
    st = orc.state_from_scene(sc)
    gm_ref, gp_ref, _ = st.step(dt, want_grid=True)
    gm, gp = sol.grid_debug(dt)
    assert rel(gm, gm_ref) <= 1e-6
    assert rel(gp, gp_ref) <= 1e-6
    sol.step_fixed(dt, 1)
    out = sol.download()
    assert np.max(np.abs(out["x"] - st.x)) <= 1e-6
    assert np.max(np.abs(out["F"] - st.F)) <= 1e-6
    for _ in range(9):
        st.step(dt)
    sol.step_fixed(dt, 9)
    out = sol.download()
    assert np.max(st.ep) > 0  # the impact yields
    assert np.max(np.abs(out["x"] - st.x)) <= 1e-6
    assert np.max(np.abs(out["F"] - st.F)) <= 2e-6
    assert np.max(np.abs(out["ep"] - st.ep)) <= 2e-6 + 1e-4 * np.max(st.ep)
    assert sol.status() == 0
    sol.close()


def test_johnson_cook_on_dense_tiles_matches_oracle():
    """Johnson-Cook (model 7) impact with 27 particles per cell, so each tile runs three scatter
    rounds with bisection returns in each. Ten CFL substeps against the oracle's CFL stepping (the
    wave-speed term uses each particle's returned F): time advanced within 1e-5, x within 1e-6 m, F
    within 2e-6, ep within 2e-6 + 1e-4 max ep."""
    sc = dense_j2_scene(material=scenes.johnson_cook_metal(7))
    sol = Solver(sc.domain, sc.n)
    sol.upload(sc)
    st = orc.state_from_scene(sc)
    t_ref = 0.0
    for _ in range(10):
        dt = st.stable_dt()
        st.step(dt)
        t_ref += dt
    t = sol.step_cfl(10)
    out = sol.download()
    assert np.max(st.ep) > 0  # the impact yields
    assert abs(t - t_ref) <= 1e-5 * t_ref
    assert np.max(np.abs(out["x"] - st.x)) <= 1e-6
    assert np.max(np.abs(out["F"] - st.F)) <= 2e-6
    assert np.max(np.abs(out["ep"] - st.ep)) <= 2e-6 + 1e-4 * np.max(st.ep)
    assert sol.status() == 0
    sol.close()
