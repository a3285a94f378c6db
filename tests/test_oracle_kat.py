"""Pins the FP64 oracle against the reference's own known-answer tests (CPU only).

Each test restates one reference test with the same inputs, tolerances and assertions:
tests/metal-plasticity.test.mjs:12-42, tests/thermal-plasticity.test.mjs:12-31,
tests/constitutive.test.mjs:10-25, tests/three.test.mjs:8-21 and tests/vv-mpm.test.mjs:5-17
(src/simulation/vv-mpm.js:7). Reference units: mu = lambda = 0.4, strengths / E.
"""
import math

import numpy as np
import pytest

from oracle import oracle as orc
from mpm_b200 import scenes

F_METAL = [1.3, .1, 0, 0, .8, 0, 0, 0, 1 / 1.04]
I3 = np.eye(3).ravel()


def det(F):
    return float(np.linalg.det(np.asarray(F, dtype=float).reshape(3, 3)))


def close(a, b, tol=1e-7):
    assert abs(a - b) < tol, f"{a} != {b}"


def mm(a, b):
    return (np.asarray(a).reshape(3, 3) @ np.asarray(b).reshape(3, 3)).ravel()


def q_metal(F):
    return orc.von_mises(orc.constitutive_stress(F, 4, .4, .4), det(F))


def project(model, ep=0.0, dt=.01, T=20.0, p=None, F=F_METAL):
    mat = orc.material(model, plasticity=p)
    return orc.project(F, mat, ep=ep, dt=dt, T=T)


# tests/metal-plasticity.test.mjs:12-23
def test_j2_radial_return_consistency_isochoric_unloading():
    for model in (4, 5):
        Fp, inc, _ = project(model)
        assert inc > 0
        close(det(Fp), det(F_METAL))
        close(q_metal(Fp), orc.flow_stress(model, inc, 0, 20, orc.material(model)))
        Fu, inc_u, _ = orc.project(I3, orc.material(model), ep=inc, dt=1 / 240, T=20)
        close(inc_u, 0)
        close(q_metal(Fu), 0)
        Fh, inc_h, _ = orc.project(np.diag([.9, .9, .9]).ravel(), orc.material(model), dt=1 / 240, T=20)
        close(inc_h, 0)
        close(det(Fh), .9 ** 3)
    assert project(5)[1] < project(4)[1]
    assert project(5, .5)[1] < project(5, 0)[1]


# tests/metal-plasticity.test.mjs:25-36
def test_johnson_cook_implicit_rate_and_temperature():
    for model in (6, 7):
        for T in (-20, 20, 650, 1000, 1200):
            for dt in (.0001, .01, .1):
                Fp, inc, _ = project(model, .12, dt, T)
                close(det(Fp), det(F_METAL))
                assert inc >= 0
                close(q_metal(Fp), orc.flow_stress(model, .12 + inc, inc / dt, T, orc.material(model)), 2e-7)
    assert q_metal(project(6, 0, .0001)[0]) > q_metal(project(6, 0, .1)[0])
    assert q_metal(project(6, 0, .01, 650)[0]) < q_metal(project(6, 0, .01, 20)[0])
    close(q_metal(project(6, 0, .01, 1000)[0]), 0)
    close(q_metal(project(7, 0, .01, 650)[0]), q_metal(project(7, 0, .01, 20)[0]))
    close(orc.flow_stress(6, 0, 0, 20, orc.material(6)), orc.PLASTICITY_DEFAULTS["A"])


# tests/metal-plasticity.test.mjs:38-42
def test_limiting_cases_reduce_to_ideal_and_linear_j2():
    close(q_metal(project(6, 0, .01, 20, dict(B=0, C=0))[0]), q_metal(project(4)[0]))
    close(q_metal(project(7, 0, .01, 650, dict(n=1, C=0))[0]), q_metal(project(5)[0]))


F_THERMAL = [1, .2, 0, 0, 1, 0, 0, 0, 1]


def ret(model, T, ep=0.0, p=None, dt=.01, F=F_THERMAL):
    return orc.project(F, orc.material(model, thermal=p), ep=ep, dt=dt, T=T)


def vm(r):
    return orc.von_mises(orc.constitutive_stress(r[0], 10, .4, .4), det(r[0]))


# tests/thermal-plasticity.test.mjs:12-20
def test_thermal_j2_hot_return_on_softened_surface():
    P = orc.material(10)
    cold, hot = ret(10, 20), ret(10, 180)
    assert hot[1] > cold[1]
    assert vm(hot) < vm(cold)
    close(vm(hot), orc.thermal_strength(hot[1], 180, P))
    close(det(hot[0]), det(F_THERMAL))
    cooled = ret(10, 20, hot[1], None, .01, hot[0])
    close(cooled[1], 0)
    close(vm(cooled), vm(hot))
    assert orc.thermal_strength(hot[1], 20, P) > orc.thermal_strength(hot[1], 180, P)
    close(ret(10, 20, 0, dict(hotRatio=1))[1], ret(10, 1000, 0, dict(hotRatio=1))[1])
    for T in (-273.15, 20, 180, 1e6):
        r = ret(10, T)
        assert r[1] >= 0
        close(det(r[0]), 1)


# tests/thermal-plasticity.test.mjs:22-33
def test_norton_creep_known_answers():
    P = orc.material(11)
    cold, hot, long = ret(11, 20), ret(11, 180), ret(11, 180, 0, None, .1)
    assert hot[1] > cold[1] * 5
    assert long[1] > hot[1]
    close(hot[1], .01 * math.exp(orc.creep_log_rate(vm(hot), 180, P)), 1e-8)
    close(det(hot[0]), 1)
    assert ret(11, -100)[1] < cold[1]
    close(ret(11, 180, 0, dict(rate=0))[1], 0)
    close(ret(11, 180, 0, None, 0)[1], 0)
    close(ret(11, 180, 0, None, .01, I3)[1], 0)
    # n = 1 backward-Euler closed form
    p = orc.material(11, thermal=dict(n=1, Q=0, rate=.1))
    sigma = [math.exp(.1), math.exp(-.1), 1]
    q = math.sqrt(6) * .4 * math.sqrt(.02)
    dt = .02
    _, inc = orc.thermal_return(sigma, 11, 0, dt, 20, p)
    expected = dt * .1 * q / .04 / (1 + dt * .1 * 1.2 / .04)
    close(inc, expected, 1e-9)
    for T in (-273.15, 1e6):
        assert np.all(np.isfinite(ret(11, T)[0]))


# tests/constitutive.test.mjs:10-16
def test_svd3_reconstructs_with_orthogonal_factors():
    for F in ([1, .8, .2, 0, .7, .4, .1, 0, 1.2], [.1, 0, 0, 0, .12, 0, 0, 0, 2], [0, -1, 0, 1, 0, 0, 0, 0, 1]):
        u, v, s = orc.svd3(F)
        rec = orc.compose(u, v, s)
        np.testing.assert_allclose(rec, F, atol=1e-8, rtol=0)
        for M in (u, v):
            np.testing.assert_allclose(mm(M, np.asarray(M).reshape(3, 3).T.ravel()), I3, atol=1e-8, rtol=0)


# tests/constitutive.test.mjs:17-25
def test_all_twelve_laws_objective_and_stress_free_under_rotation():
    c, s = math.cos(.7), math.sin(.7)
    R = [c, 0, s, 0, 1, 0, -s, 0, c]
    F = [1.03, .02, 0, 0, .97, 0, 0, 0, .99]
    RT = np.asarray(R).reshape(3, 3).T.ravel()
    for model in range(12):
        np.testing.assert_allclose(orc.constitutive_stress(R, model, 400, 400), 0, atol=1e-8)
        t = orc.constitutive_stress(F, model, 400, 400)
        rotated = orc.constitutive_stress(mm(R, F), model, 400, 400)
        np.testing.assert_allclose(rotated, mm(mm(R, t), RT), atol=1e-8, rtol=0)
    F15 = [1.5, 0, 0, 0, 1, 0, 0, 0, 1]
    assert abs(orc.constitutive_stress(F15, 0, 400, 400)[0] - orc.constitutive_stress(F15, 1, 400, 400)[0]) > 100


# tests/three.test.mjs:8-13
def test_stress3_rotation_invariant_and_restores_shear():
    c, s = math.cos(.8), math.sin(.8)
    r = [1, 0, 0, 0, c, -s, 0, s, c]
    assert np.all(np.abs(orc.stress3(r, 400, 400)) < 1e-8)
    f = list(I3)
    f[2] = .2
    t = orc.stress3(f, 400, 400)
    assert t[2] > 0 and abs(t[2] - t[6]) < 1e-8
    f[5] = .3
    assert orc.stress3(f, 400, 400)[5] > 0


# tests/three.test.mjs:14-21: uniform XYZ motion preserved to 1e-8 by one step
def test_uniform_xyz_motion_preserved_one_step():
    sc = scenes.translation_block(velocity=(3.0, -2.0, 7.0))
    st = orc.state_from_scene(sc)
    st.step(.001)
    np.testing.assert_allclose(st.v, np.tile([3.0, -2.0, 7.0], (sc.n, 1)), atol=1e-8, rtol=0)


# tests/vv-mpm.test.mjs:5-17, src/simulation/vv-mpm.js:7: zero-stress translation across more than
# one cell at grid phases 0, .25, .5 with 1e-8 limits on position, velocity, stress, F deviation
@pytest.mark.parametrize("phase", [0.0, .25, .5])
def test_translation_through_a_cell_at_three_phases(phase):
    sc = scenes.translation_block(phase=phase)
    st = orc.state_from_scene(sc)
    x0 = st.x.copy()
    t, dt_req, duration = 0.0, 1 / 480, .06
    steps = 0
    while t < duration - 1e-12:
        dt = min(dt_req, duration - t, st.stable_dt())
        st.step(dt)
        t += dt
        steps += 1
    assert steps > 1
    assert 2.0 * t / sc.domain.H > 1  # travelled more than one cell
    pos_err = np.max(np.linalg.norm(st.x - x0 - np.array([2.0, 0, 0]) * t, axis=1))
    vel_err = np.max(np.linalg.norm(st.v - np.array([2.0, 0, 0]), axis=1))
    f_dev = np.max(np.abs(st.F - I3))
    assert pos_err < 1e-8 and vel_err < 1e-8 and f_dev < 1e-8
    mats = sc.materials[0]
    tau = orc.constitutive_stress(st.F[0], 0, mats.mu, mats.lam)
    assert orc.von_mises(tau) / (mats.mu * 2.5) < 1e-8


def test_hash_matches_reference_int32_semantics():
    """src/three/sampling.js:8-12 evaluated with explicit 32-bit wraparound (Math.imul, >>>0)."""
    def imul(a, b):
        return (a * b) & 0xFFFFFFFF

    def js_random(seed, index, attempt, axis):
        h = (seed + imul(index + 1, 0x9E3779B9) + imul(attempt * 3 + axis + 1, 0x85EBCA6B)) & 0xFFFFFFFF
        h = imul(h ^ (h >> 16), 0x7FEB352D)
        h = imul(h ^ (h >> 15), 0x846CA68B)
        return ((h ^ (h >> 16)) & 0xFFFFFFFF) / 4294967296 * 2 - 1

    for seed, idx, att, ax in [(42, 0, 0, 0), (1, 13823, 0, 2), (2147483647, 16777215, 7, 1), (3, 5, 1, 0)]:
        assert scenes.hash_random(seed, idx, att, ax) == js_random(seed, idx, att, ax)


def test_oracle_step_conserves_mass_and_momentum_without_walls():
    sc = scenes.translation_block(velocity=(0.5, 0.25, -0.1))
    rng = np.random.default_rng(0)
    sc.F = np.tile(I3, (sc.n, 1)) + 0.01 * rng.standard_normal((sc.n, 9))
    st = orc.state_from_scene(sc)
    before = st.ledger()
    st.step(1e-4)
    after = st.ledger()
    close(after.mass, before.mass, 1e-15)
    for a in range(3):
        close(after.momentum[a], before.momentum[a], 1e-12)
