"""The device constitutive math (mpm_math.h, FP32, centred form) compiled for the host and checked
against the FP64 oracle on CPU: Jacobi eigensolver, fixed-corotated, Neo-Hookean, Hencky stress and
the J2 / thermal J2 return maps, with the tolerances of the reference's own CPU/GPU return-map test
(gpu/test_metal_plasticity.py:31-33: F atol 4e-6 rtol 4e-5)."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle as orc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "summer-particle-lab_b200", "csrc")
P = ctypes.c_void_p


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    out = tmp_path_factory.mktemp("h") / "libharness.so"
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-I", CSRC, "-o", str(out),
                           os.path.join(ROOT, "tests", "native", "math_harness.cpp")])
    L = ctypes.CDLL(str(out))
    d = ctypes.c_double
    L.harness_constitutive.argtypes = [ctypes.c_int, d, d, d, d, d, d, d, ctypes.c_int, P, P, P, ctypes.c_int, P, P, P]
    L.harness_eig.argtypes = [ctypes.c_int, P, P, P]
    return L


def run(L, model, F, ep, T, mu=.4, lam=.4, A=.025, B=.08, Tref=20, Thot=180, hot=.08, do_return=True):
    F = np.ascontiguousarray(np.asarray(F, dtype=np.float64).reshape(-1, 9))
    n = F.shape[0]
    ep = np.ascontiguousarray(np.broadcast_to(np.asarray(ep, dtype=np.float64), (n,)))
    T = np.ascontiguousarray(np.broadcast_to(np.asarray(T, dtype=np.float64), (n,)))
    Fo, dep, tau = np.empty((n, 9)), np.empty(n), np.empty((n, 9))
    c = lambda a: a.ctypes.data_as(P)
    L.harness_constitutive(model, mu, lam, A, B, Tref, Thot, hot, n, c(F), c(ep), c(T), int(do_return), c(Fo), c(dep), c(tau))
    return Fo, dep, tau


def random_F(n, scale, seed):
    rng = np.random.default_rng(seed)
    return np.tile(np.eye(3).ravel(), (n, 1)) + scale * rng.standard_normal((n, 9))


def test_jacobi_eigensolver_reconstructs(harness):
    rng = np.random.default_rng(1)
    for scale in (1e-4, 1e-2, 1.0):
        M = scale * rng.standard_normal((500, 3, 3))
        S = M + M.transpose(0, 2, 1)
        S6 = np.stack([S[:, 0, 0], S[:, 1, 1], S[:, 2, 2], S[:, 0, 1], S[:, 0, 2], S[:, 1, 2]], 1).copy()
        lam, U = np.empty((500, 3)), np.empty((500, 9))
        harness.harness_eig(500, S6.ctypes.data_as(P), lam.ctypes.data_as(P), U.ctypes.data_as(P))
        U = U.reshape(-1, 3, 3)
        rec = U @ (lam[:, :, None] * U.transpose(0, 2, 1))
        err = np.max(np.abs(rec - S), axis=(1, 2)) / np.max(np.abs(S), axis=(1, 2))
        assert np.max(err) < 2e-6, (scale, np.max(err))
        orth = np.max(np.abs(U @ U.transpose(0, 2, 1) - np.eye(3)))
        assert orth < 2e-6


@pytest.mark.parametrize("model", [0, 1])
def test_elastic_stress_matches_oracle(harness, model):
    for scale in (1e-3, 5e-2):
        F = random_F(300, scale, 2 + model)
        _, _, tau = run(harness, model, F, 0, 0, mu=400, lam=300)
        for i in range(F.shape[0]):
            ref = orc.constitutive_stress(F[i], model, 400, 300)
            np.testing.assert_allclose(tau[i], ref, atol=2e-5 * np.max(np.abs(ref)) + 1e-9, rtol=0)


@pytest.mark.parametrize("model", [4, 5])
def test_j2_return_matches_oracle(harness, model):
    F = random_F(400, 0.05, 7 + model)
    Fo, dep, tau = run(harness, model, F, .05, 20)
    mat = orc.material(model)
    n_yield = 0
    for i in range(F.shape[0]):
        Fr, inc, tr = orc.project(F[i], mat, ep=.05, dt=.01, T=20)
        np.testing.assert_allclose(Fo[i], Fr, atol=4e-6, rtol=4e-5)
        assert abs(dep[i] - inc) < 1e-5
        np.testing.assert_allclose(tau[i], tr, atol=3e-6, rtol=5e-4)
        n_yield += inc > 0
    assert n_yield > 50


def test_thermal_j2_return_matches_oracle(harness):
    F = random_F(300, 0.05, 19)
    T = np.linspace(-100, 800, 300)
    Fo, dep, tau = run(harness, 10, F, .05, T, A=.04, B=.04)
    mat = orc.material(10)
    for i in range(F.shape[0]):
        Fr, inc, tr = orc.project(F[i], mat, ep=.05, dt=.01, T=T[i])
        np.testing.assert_allclose(Fo[i], Fr, atol=4e-6, rtol=5e-5)
        assert abs(dep[i] - inc) < 1e-5


def test_small_strain_precision_of_centred_form(harness):
    """Elastic metal strains (~1e-4): the centred form keeps ~1e-6 relative stress accuracy."""
    E = 70e9
    mu, lam = E / 2.66, E * .33 / (1.33 * .34)
    F = random_F(200, 1e-4, 23)
    _, _, tau = run(harness, 5, F, 0, 0, mu=mu, lam=lam, A=250e6, B=1e9)
    for i in range(F.shape[0]):
        ref = orc.constitutive_stress(F[i], 5, mu, lam)
        np.testing.assert_allclose(tau[i], ref, atol=2e-5 * np.max(np.abs(ref)), rtol=0)


def b_norm(F):
    Fm = F.reshape(-1, 3, 3)
    B = Fm @ Fm.transpose(0, 2, 1) - np.eye(3)
    return np.sqrt(np.sum(B * B, axis=(1, 2)))


@pytest.mark.parametrize("scale", [3e-4, 3e-3, 1e-2, 2.5e-2, 0.2])
def test_series_and_eigen_paths_match_oracle_j2(harness, scale):
    """|B| <= 0.15 runs the matrix-series path, larger strains the Jacobi path; both match the
    oracle's SVD-based return map (reference units, yield strain lowered so small strains yield)."""
    F = random_F(400, scale, 31)
    A = 0.002
    Fo, dep, tau = run(harness, 5, F, .01, 20, A=A, B=.08)
    mat = orc.material(5, plasticity=dict(A=A, B=.08))
    series = b_norm(F) <= 0.15
    assert series.all() if scale <= 1e-2 else True
    n_yield = 0
    for i in range(F.shape[0]):
        Fr, inc, tr = orc.project(F[i], mat, ep=.01, dt=.01, T=20)
        np.testing.assert_allclose(Fo[i], Fr, atol=4e-6, rtol=4e-5)
        assert abs(dep[i] - inc) < 1e-5 * max(1.0, inc)
        np.testing.assert_allclose(tau[i], tr, atol=3e-6 * max(1.0, np.max(np.abs(tr))), rtol=5e-4)
        n_yield += inc > 0
    if scale >= 3e-3:
        assert n_yield > 20


@pytest.mark.parametrize("scale", [3e-4, 1e-2, 4e-2, 0.2])
def test_series_and_eigen_paths_fixed_corotated(harness, scale):
    F = random_F(300, scale, 37)
    _, _, tau = run(harness, 0, F, 0, 0, mu=400, lam=300)
    for i in range(F.shape[0]):
        ref = orc.constitutive_stress(F[i], 0, 400, 300)
        np.testing.assert_allclose(tau[i], ref, atol=2e-5 * np.max(np.abs(ref)) + 1e-9, rtol=0)


def test_thermal_series_path_with_softening(harness):
    F = random_F(300, 8e-3, 41)
    T = np.linspace(0, 400, 300)
    Fo, dep, tau = run(harness, 10, F, .02, T, A=.004, B=.04)
    mat = orc.material(10, thermal=dict(A=.004, H=.04))
    n_yield = 0
    for i in range(F.shape[0]):
        Fr, inc, tr = orc.project(F[i], mat, ep=.02, dt=.01, T=T[i])
        np.testing.assert_allclose(Fo[i], Fr, atol=4e-6, rtol=5e-5)
        assert abs(dep[i] - inc) < 1e-5
        n_yield += inc > 0
    assert n_yield > 20


# ---- rate-dependent laws: Johnson-Cook (6, 7) and Norton creep (11), bisection returns ----------

def _full(L, mat, dt, F, ep, T):
    L.harness_constitutive_full.argtypes = [ctypes.c_int, P, ctypes.c_double, ctypes.c_int, P, P, P, P, P, P]
    prm = np.array([mat.mu, mat.lam, mat.yield_stress, mat.hardening, mat.T_ref, mat.T_hot, mat.hot_ratio, mat.jc_n,
                    mat.jc_C, mat.jc_rate0, mat.T_melt, mat.jc_m, mat.creep_rate, mat.creep_Q, mat.creep_n,
                    mat.creep_stress, mat.temperature_offset])
    F = np.ascontiguousarray(np.asarray(F, dtype=np.float64).reshape(-1, 9))
    n = F.shape[0]
    ep = np.ascontiguousarray(np.broadcast_to(np.asarray(ep, dtype=np.float64), (n,)))
    T = np.ascontiguousarray(np.broadcast_to(np.asarray(T, dtype=np.float64), (n,)))
    Fo, dep, tau = np.empty((n, 9)), np.empty(n), np.empty((n, 9))
    c = lambda a: a.ctypes.data_as(P)
    L.harness_constitutive_full(mat.model, c(prm), dt, n, c(F), c(ep), c(T), c(Fo), c(dep), c(tau))
    return Fo, dep, tau


@pytest.mark.parametrize("model", [6, 7])
def test_johnson_cook_matches_oracle(harness, model):
    from mpm_b200.params import Material
    # gpu/metal_reference.mjs:1-9: T in {20, 650, 1100}, dt in {.001, .02}, F preset, ep .15, A .03, B .12
    mat = Material.reference_units(model, A=.03, B=.12)
    omat = orc.material_from(mat)
    F = [1.3, .1, 0, 0, .8, 0, 0, 0, 1 / 1.04]
    for T in (20, 650, 1100):
        for dt in (.001, .02):
            Fo_ref, inc_ref, _ = orc.project(F, omat, ep=.15, dt=dt, T=T)
            Fo, dep, _ = _full(harness, mat, dt, [F], .15, T)
            np.testing.assert_allclose(Fo[0], Fo_ref, atol=4e-6, rtol=4e-5)
            assert abs(dep[0] - inc_ref) < 1e-5, (T, dt, dep[0], inc_ref)
    # random trial states: yielding and elastic, several temperatures and strain rates
    rng = np.random.default_rng(11)
    Fs = random_F(300, .05, 12)
    eps = rng.uniform(0, .3, 300)
    Ts = rng.uniform(0, 900, 300)
    Fo, dep, tau = _full(harness, mat, .005, Fs, eps, Ts)
    yielded = 0
    for i in range(300):
        Fo_ref, inc_ref, _ = orc.project(Fs[i], omat, ep=eps[i], dt=.005, T=Ts[i])
        np.testing.assert_allclose(Fo[i], Fo_ref, atol=4e-6, rtol=4e-5)
        assert abs(dep[i] - inc_ref) < 1e-5
        np.testing.assert_allclose(tau[i], orc.constitutive_stress(Fo_ref, model, mat.mu, mat.lam), atol=3e-6, rtol=5e-4)
        yielded += inc_ref > 0
    assert yielded > 50


def test_norton_creep_matches_oracle(harness):
    from mpm_b200.params import Material
    # gpu/thermal_reference.mjs:1-9 for model 11: T in {-100, 20, 180, 800}, two F, ep .05, dt .01
    mat = Material.reference_units(11)
    omat = orc.material_from(mat)
    for T in (-100, 20, 180, 800):
        for F in ([1, .2, 0, 0, 1, 0, 0, 0, 1], [.9, 0, 0, 0, 1.05, 0, 0, 0, 1]):
            Fo_ref, inc_ref, _ = orc.project(F, omat, ep=.05, dt=.01, T=T)
            Fo, dep, _ = _full(harness, mat, .01, [F], .05, T)
            np.testing.assert_allclose(Fo[0], Fo_ref, atol=4e-6, rtol=5e-5)
            assert abs(dep[0] - inc_ref) <= 1e-5 + 1e-4 * inc_ref, (T, F, dep[0], inc_ref)
    # the n = 1 closed form of tests/thermal-plasticity.test.mjs:28-31 on the device math:
    # dep = dt rate q/s / (1 + dt rate 1.2/s) at T = Tref (activation term zero)
    lin = Material.reference_units(11, thermal=dict(n=1))
    F = [1.02, 0, 0, 0, 1 / 1.02, 0, 0, 0, 1]
    _, dep, _ = _full(harness, lin, .01, [F], 0.0, 20.0)
    Fo_ref, inc_ref, _ = orc.project(F, orc.material_from(lin), ep=0.0, dt=.01, T=20.0)
    assert abs(dep[0] - inc_ref) <= 1e-6 + 1e-4 * inc_ref


def jc_prm(mat):
    return np.array([mat.mu, mat.lam, mat.yield_stress, mat.hardening, mat.T_ref, mat.T_hot, mat.hot_ratio, mat.jc_n,
                     mat.jc_C, mat.jc_rate0, mat.T_melt, mat.jc_m, 0, 0, 1, 1, 0], dtype=np.float64)


@pytest.mark.parametrize("model", [6, 7])
def test_learned_johnson_cook_gate_against_the_oracle(harness, model):
    """The learned Johnson-Cook return's refinement and gate (the device math on the host): from a
    guess within 20% of the root, at most four Newton steps reach the gate (consistency residual
    <= 1e-5 of the trial stress), including roots just past the rate term's kink, and every
    accepted increment satisfies the FP64 oracle's consistency condition
    (src/three/metal-plasticity.js:28-34) to that bound plus FP32 rounding,
    |q - 3 mu / J dep - flow(ep + dep, dep / dt, T)| <= 2e-5 q, and agrees with the exact bisection.
    A guess the gate cannot vouch for (no Newton steps from a wrong root) is rejected. The
    Newton-gated mode's guess from the initial flow stress passes within eight steps, to the same
    bounds."""
    from mpm_b200 import scenes
    mat = scenes.johnson_cook_metal(model)
    om = orc.material_from(mat)
    rng = np.random.default_rng(12)
    n = 400
    J = np.exp(rng.uniform(-0.01, 0.01, n))
    ep = rng.uniform(0, 0.4, n)
    T = rng.uniform(293, 700, n)
    dt = np.exp(rng.uniform(np.log(1e-8), np.log(1e-5), n))
    flow0 = np.array([orc.flow_stress(model, e, 0.0, t, om) for e, t in zip(ep, T)])
    q = flow0 * (1 + np.exp(rng.uniform(np.log(1e-3), np.log(3.0), n)))
    L = harness
    L.harness_jc_refine.argtypes = [ctypes.c_int, P, ctypes.c_int, P, P, P, P, P, P, ctypes.c_double, ctypes.c_int,
                                    P, P, P, P]
    c = lambda a: a.ctypes.data_as(P)
    prm = jc_prm(mat)

    def refine(u, newton):
        ok = np.zeros(n, np.int32)
        dl, de, feat = np.zeros(n), np.zeros(n), np.zeros((n, 8))
        L.harness_jc_refine(model, c(prm), n, c(q), c(J), c(ep), c(T), c(dt), c(np.ascontiguousarray(u)), 1e-5, newton,
                            c(ok), c(dl), c(de), c(feat))
        return ok.astype(bool), dl, de, feat

    s = q * J / (3 * mat.mu)
    _, _, dep_exact, feat = refine(np.full(n, 0.5), 0)
    u_exact = dep_exact / s
    assert np.all((feat[:, 0] > 0) & (feat[:, 0] <= 1))  # A soft / q of a plastic state
    ok, dl, _, _ = refine(u_exact * rng.uniform(0.8, 1.2, n), 4)
    assert ok.mean() >= 0.98, ok.mean()
    for i in np.flatnonzero(ok):
        r = q[i] - 3 * mat.mu / J[i] * dl[i] - orc.flow_stress(model, ep[i] + dl[i], dl[i] / dt[i], T[i], om)
        assert abs(r) <= 2e-5 * q[i], (i, r / q[i])
        assert abs(dl[i] - dep_exact[i]) <= 2e-5 * s[i] + 1e-4 * dep_exact[i], i
    bad, _, _, _ = refine(np.clip(u_exact * 3 + 0.3, 0, 1), 0)
    assert bad.mean() <= 0.05
    # the Newton-gated mode's guess, the root of the rate- and hardening-free condition: within eight
    # Newton steps the gate passes for all but a few states, every accepted increment satisfies the
    # oracle's consistency condition to the gate's bound, and it agrees with the bisection
    u0 = np.clip(1 - flow0 / q, 0, 1)
    ok8, dl8, _, _ = refine(u0, 8)
    assert ok8.mean() >= 0.99, ok8.mean()
    for i in np.flatnonzero(ok8):
        r = q[i] - 3 * mat.mu / J[i] * dl8[i] - orc.flow_stress(model, ep[i] + dl8[i], dl8[i] / dt[i], T[i], om)
        assert abs(r) <= 2e-5 * q[i], (i, r / q[i])
        assert abs(dl8[i] - dep_exact[i]) <= 2e-5 * s[i] + 1e-4 * dep_exact[i], i
