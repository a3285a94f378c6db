"""Snow (2), sand (3), cohesive Drucker-Prager (8) and Deshpande-Fleck foam (9), on the CPU.

The FP64 oracle is pinned by restating the reference's known-answer tests with their inputs,
tolerances and assertions: tests/constitutive.test.mjs:26-43 (snow, sand) and
tests/pressure-plasticity.test.mjs:11-44 (cohesive DP limits, dilatancy and tension cutoff, foam
yield surface, hardening, compaction and associated flow). Reference units: mu = lambda = 0.4,
strengths / E. The reference's parameter validation (pressure-plasticity.test.mjs:36-40) is
restated against mpm_validate_material (the checks of mpm_set_material); its JavaScript-object cases (null, arrays, unknown
keys) have no C counterpart.

Then the device math (mpm_math.h, FP32, compiled for the host) is checked against the oracle on
random deformation gradients with the reference's own CPU/GPU return-map tolerances
(gpu/test_metal_plasticity.py:31-33: F atol 4e-6 rtol 4e-5), the history scalars within 1e-5.
"""
import ctypes
import math
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle as orc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "summer-particle-lab_b200", "csrc")
P = ctypes.c_void_p
I3 = np.eye(3).ravel()
PD = orc.PRESSURE_DEFAULTS


def det(F):
    return float(np.linalg.det(np.asarray(F, dtype=float).reshape(3, 3)))


def close(a, b, tol=1e-7):
    assert abs(a - b) < tol, f"{a} != {b}"


def diag(x, y=None, z=None):
    y = x if y is None else y
    z = x if z is None else z
    return [x, 0, 0, 0, y, 0, 0, 0, z]


def snow_sand(F, model, jp=1.0, dilation=0.0, yield_strain=.025, friction=35.0):
    mat = orc.material(model, yield_strain=yield_strain, friction=friction)
    return orc.project_state(F, mat, jp=jp, dilation=dilation, dt=1 / 240, T=20)


# tests/constitutive.test.mjs:26-34
def test_snow_returns_to_its_asymmetric_yield_surface_and_keeps_compaction():
    F = [.8, 0, 0, 0, .9, 0, 0, 0, 1.2]
    p = snow_sand(F, 2)
    _, _, s = orc.svd3(p["F"])
    assert np.all(s >= .975 - 1e-8) and np.all(s <= 1.0075 + 1e-8)
    close(det(p["F"]) * p["jp"], det(F))
    assert p["jp"] < 1 and orc.hardening(p["jp"]) > 1
    unloaded = snow_sand(I3, 2, jp=p["jp"])
    close(unloaded["jp"], p["jp"])
    r0 = orc.project_state(F, orc.material(0))
    assert np.array_equal(r0["F"], np.asarray(F, dtype=float))  # elastic models keep F
    soft = snow_sand(diag(.96, 1, 1), 2, yield_strain=.01)
    strong = snow_sand(diag(.96, 1, 1), 2, yield_strain=.06)
    assert soft["jp"] < strong["jp"]


# tests/constitutive.test.mjs:35-43
def test_sand_has_no_tensile_stress_and_friction_controls_shear_yield():
    tensile = snow_sand(diag(1.1), 3)
    np.testing.assert_allclose(orc.constitutive_stress(tensile["F"], 3, 400, 400), 0, atol=1e-8)
    assert tensile["dilation"] > 0
    F = [.8, 0, 0, 0, 1.05, 0, 0, 0, 1.05]
    low, high = snow_sand(F, 3, friction=15), snow_sand(F, 3, friction=50)

    def dev_norm(f):
        e = np.log(orc.svd3(f)[2])
        return float(np.linalg.norm(e - e.mean()))

    assert dev_norm(high["F"]) > dev_norm(low["F"])
    close(det(low["F"]), det(F))
    close(det(high["F"]), det(F))
    compressed = snow_sand(diag(.95), 3)
    assert orc.constitutive_stress(compressed["F"], 3, 400, 400)[0] < 0


def pret(F, model=8, p=None, jp=1.0, ep=0.0):
    """ret() of tests/pressure-plasticity.test.mjs:9."""
    mat = orc.material(model, pressure=p)
    return orc.project_state(F, mat, jp=jp, ep=ep, dt=.01, T=20)


def stress(r):
    """stress() of tests/pressure-plasticity.test.mjs:10: Cauchy von Mises and mean over J Jp."""
    J = det(r["F"]) * r["jp"]
    t = orc.constitutive_stress(r["F"], 8, .4, .4)
    return orc.von_mises(t, J), (t[0] + t[4] + t[8]) / (3 * J)


# tests/pressure-plasticity.test.mjs:11-23
def test_cohesive_dp_shear_and_tension_limits_total_j_and_dilatancy():
    for F in (diag(1.1), diag(.8), diag(1.3, .8, 1), [1, .4, 0, 0, 1, 0, 0, 0, 1]):
        r = pret(F)
        q, mean = stress(r)
        assert q / math.sqrt(3) + PD["slope"] * mean <= PD["cohesion"] + 1e-7
        assert mean <= PD["tension"] + 1e-7
        close(det(r["F"]) * r["jp"], det(F))
        assert r["increment"] >= 0
    tension = pret(diag(1.1))
    close(stress(tension)[1], PD["tension"])
    assert tension["jp"] > 1
    compressed = pret(diag(.8))
    close(compressed["increment"], 0)
    close(compressed["jp"], 1)
    F = [1, .5, 0, 0, 1, 0, 0, 0, 1]
    close(pret(F, 8, dict(dilatancy=0))["jp"], 1)
    assert pret(F, 8, dict(dilatancy=.5))["jp"] > 1
    assert stress(pret(F, 8, dict(cohesion=.1)))[0] > stress(pret(F))[0]
    residual = pret(I3, 8, None, tension["jp"], tension["increment"])
    close(residual["jp"], tension["jp"])
    close(residual["increment"], 0)


def foam(ep, p=None):
    return orc.foam_strength(ep, orc.material(9, pressure=p))


# tests/pressure-plasticity.test.mjs:25-35
def test_df_foam_yields_in_hydrostatic_compression_hardens_and_keeps_compaction():
    a2 = PD["alpha"] ** 2
    for F in (diag(.85), diag(1.1), [1, .45, 0, 0, .95, 0, 0, 0, 1.1]):
        for jp in (.6, 1, 1.2):
            r = pret(F, 9, None, jp, .05)
            q, mean = stress(r)
            hat = math.sqrt((q * q + a2 * mean * mean) / (1 + a2 / 9))
            close(det(r["F"]) * r["jp"], det(F) * jp)
            close(hat, foam(.05 + r["increment"]), 2e-7)
            assert .05 + r["increment"] < PD["epsD"]
    p = pret(diag(.85), 9)
    assert p["jp"] < 1 and p["increment"] > 0
    close(stress(p)[0], 0)
    unloaded = pret(I3, 9, None, p["jp"], p["increment"])
    close(unloaded["jp"], p["jp"])
    close(unloaded["increment"], 0)
    close(stress(unloaded)[1], 0)
    assert foam(.65) > foam(.1)
    assert abs(stress(pret(diag(.85), 9, None, 1, .3))[1]) > abs(stress(p)[1])


# tests/pressure-plasticity.test.mjs:37-44
def test_foam_flow_is_associated_and_equivalent_strain_is_work_conjugate():
    a2 = PD["alpha"] ** 2
    F = diag(.85, .97, 1.02)
    p = pret(F, 9)
    q, mean = stress(p)
    hat = math.sqrt((q * q + a2 * mean * mean) / (1 + a2 / 9))
    d = np.log(np.asarray(F)[[0, 4, 8]] / p["F"][[0, 4, 8]])
    tr = d.sum()
    dev = d - tr / 3
    conjugate = math.sqrt((1 + a2 / 9) * (2 / 3 * float(dev @ dev) + tr * tr / a2))
    close(conjugate, p["increment"])
    tau = orc.constitutive_stress(p["F"], 9, .4, .4)
    J = det(p["F"]) * p["jp"]
    work = sum(tau[k] / J * d[i] for i, k in enumerate((0, 4, 8)))
    close(work, hat * p["increment"])


# ---------------------------------------------------------------------------------- ABI checks

def _material(model, **kw):
    from mpm_b200 import _lib
    m = _lib.MpmMaterial(model=model, mu=.4, lam=.4, yield_strain=.025, friction_deg=35.0, dp_cohesion=PD["cohesion"],
                         dp_slope=PD["slope"], dp_dilatancy=PD["dilatancy"], dp_tension=PD["tension"],
                         df_alpha=PD["alpha"], df_plateau=PD["plateau"], df_gamma=PD["gamma"],
                         df_densify=PD["densify"], df_beta=PD["beta"], df_eps_d=PD["epsD"])
    for k, v in kw.items():
        setattr(m, k, v)
    return m


# tests/pressure-plasticity.test.mjs:36-40 (the numeric cases) against the library's checks
# (mpm_validate_material, the checks of mpm_set_material, on the host)
def test_invalid_pressure_parameters_are_rejected():
    from mpm_b200 import _lib
    L = _lib.lib()
    v = L.mpm_validate_material
    assert v(ctypes.byref(_material(8))) == 0
    assert v(ctypes.byref(_material(9))) == 0
    bad = [(9, dict(df_alpha=0.0)), (9, dict(df_eps_d=0.0)), (9, dict(df_densify=0.0)),
           (8, dict(dp_dilatancy=.8)), (8, dict(dp_tension=.2)), (8, dict(dp_cohesion=float("nan"))),
           (9, dict(df_beta=float("inf"))), (2, dict(yield_strain=0.0)), (3, dict(friction_deg=0.0))]
    for model, kw in bad:
        assert v(ctypes.byref(_material(model, **kw))) == -1, (model, kw)


# ---------------------------------------------------------------------------------- device math

@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    out = tmp_path_factory.mktemp("h") / "libharness.so"
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-I", CSRC, "-o", str(out),
                           os.path.join(ROOT, "tests", "native", "math_harness.cpp")])
    L = ctypes.CDLL(str(out))
    L.harness_constitutive_aux.argtypes = [ctypes.c_int, P, ctypes.c_int, P, P, P, ctypes.c_int, P, P, P]
    return L


def prm(mu=.4, lam=.4, yield_strain=.025, friction=35.0, p=None):
    q = dict(PD, **(p or {}))
    return np.array([mu, lam, yield_strain, friction, q["cohesion"], q["slope"], q["dilatancy"], q["tension"],
                     q["alpha"], q["plateau"], q["gamma"], q["densify"], q["beta"], q["epsD"]])


def device(L, model, F, ep, hist, do_return=True, **kw):
    F = np.ascontiguousarray(np.asarray(F, dtype=np.float64).reshape(-1, 9))
    n = F.shape[0]
    ep = np.ascontiguousarray(np.broadcast_to(np.asarray(ep, dtype=np.float64), (n,)))
    h = np.ascontiguousarray(np.broadcast_to(np.asarray(hist, dtype=np.float64), (n,))).copy()
    Fo, dep, tau = np.empty((n, 9)), np.empty(n), np.empty((n, 9))
    c = lambda a: a.ctypes.data_as(P)
    pr = prm(**kw)
    L.harness_constitutive_aux(model, c(pr), n, c(F), c(ep), c(h), int(do_return), c(Fo), c(dep), c(tau))
    return Fo, dep, h, tau


def random_F(n, scale, seed):
    rng = np.random.default_rng(seed)
    return np.tile(I3, (n, 1)) + scale * rng.standard_normal((n, 9))


@pytest.mark.parametrize("model,scale,hist0", [(2, .03, 1.0), (2, .15, .8), (3, .05, 0.0), (3, .1, .02),
                                               (8, .05, 1.0), (8, .15, 1.1), (9, .05, 1.0), (9, .12, .9)])
def test_device_math_matches_oracle(harness, model, scale, hist0):
    F = random_F(300, scale, 11 * model + int(100 * scale))
    F = F[[det(f) > .3 for f in F]]
    ep = .05 if model == 9 else 0.0
    Fo, dep, hist, tau = device(harness, model, F, ep, hist0)
    mat = orc.material(model)
    plastic = 0
    for i in range(F.shape[0]):
        kw = dict(jp=hist0) if model != 3 else dict(dilation=hist0)
        r = orc.project_state(F[i], mat, ep=ep, dt=.01, T=20, **kw)
        np.testing.assert_allclose(Fo[i], r["F"], atol=4e-6, rtol=4e-5)
        t = r["tau"] * (orc.hardening(r["jp"]) if model == 2 else 1.0)
        np.testing.assert_allclose(tau[i], t, atol=4e-6 * max(1.0, np.max(np.abs(t))), rtol=4e-5)
        assert abs(dep[i] - r["increment"]) <= 1e-5 + 1e-4 * r["increment"]
        h = r["dilation"] if model == 3 else r["jp"]
        assert abs(hist[i] - h) <= 1e-5 * max(1.0, abs(h)), (i, hist[i], h)
        plastic += r["increment"] > 0
    assert plastic > F.shape[0] // 10  # the cases exercise the returns


@pytest.mark.parametrize("model", [2, 3, 8, 9])
def test_device_stress_without_return_matches_oracle(harness, model):
    """The stress of a stored state (first P2G, pinned particles): snow scales by its hardening."""
    F = random_F(100, .05, 5 + model)
    jp = .9 if model != 3 else 0.0
    _, dep, hist, tau = device(harness, model, F, 0.0, jp, do_return=False)
    assert np.all(dep == 0) and np.all(np.abs(hist - jp) <= 1e-7)
    for i in range(F.shape[0]):
        t = orc.constitutive_stress(F[i], model, .4, .4) * (orc.hardening(jp) if model == 2 else 1.0)
        np.testing.assert_allclose(tau[i], t, atol=4e-6 * max(1.0, np.max(np.abs(t))), rtol=4e-5)
