"""Particle-pair heat exchange and enthalpy phase change (src/thermal.js:35-56,
src/three/phase-change.js:4-18, with the pairs of src/three/simulation.js:168-174).

The FP64 oracle is pinned by restating the reference's tests with their inputs and tolerances:
tests/material-physics.test.mjs:15-31 (equilibrium of different heat capacities; many contacts
conserve energy without overshoot; iron conducts faster than water), tests/three.test.mjs:27-31
(the contact uses the 3D distance and conserves enthalpy) and tests/phase-change.test.mjs:11-18
and :44-49 (enthalpy with latent heat, switching only at complete melting or freezing, contact
heat melting two custom-material particles with total enthalpy kept). The reference passes a pair
list with explicit weights; here pairs come from positions (weight 1 - r / radius), so a case's
weight w is reproduced by placing the pair at a known distance and scaling heat_rate by w / (1 - r / radius).
Reference units: radius 8, geometry 20, heat_rate 20; water cp 4180, k 0.6, 1 kg per litre
parcel; iron cp 450, k 80, 7.87 kg; custom material cp 1800, k 0.13, 1.1 kg, melting at 120 with
latent heat 120000.

GPU tests: the same cases through mpm_exchange_heat, and a random two-material cloud with phase
change against the oracle (temperatures within 1e-4 K, energy within 1e-6 relative).
"""
import numpy as np
import pytest

from oracle import oracle as orc
from mpm_b200 import scenes
from mpm_b200.params import Domain, Material

DOMAIN = Domain(lower=(-64, -48, -64), upper=(64, 72, 64), H=8.0)
WATER = dict(cp=4180.0, k=.6, m=1.0)
IRON = dict(cp=450.0, k=80.0, m=7.87)
CUSTOM = dict(cp=1800.0, k=.13, m=1.1)


def material(props, latent=0.0, melting=120.0):
    return Material(model=0, mu=.4, lam=.4, specific_heat=props["cp"], conductivity=props["k"], latent_heat=latent,
                    melting_point=melting)


def heat_scene(pos, temps, kinds, latent=0.0):
    """Particles of the given kinds (dicts above) at pos with temperatures; one material per kind."""
    mats, index = [], {}
    for k in kinds:
        key = id(k)
        if key not in index:
            index[key] = len(mats)
            mats.append(material(k, latent))
    x = np.asarray(pos, dtype=np.float64)
    sc = scenes._scene("heat", DOMAIN, mats, x, (0, 0, 0))
    sc.m = np.array([k["m"] for k in kinds])
    sc.V = np.ones(len(kinds))
    sc.mat = np.array([index[id(k)] for k in kinds], dtype=np.int32)
    sc.T = np.asarray(temps, dtype=np.float64)
    return sc


def energy(st):
    return float(np.sum(st.m * st.h))


# tests/material-physics.test.mjs:15-20 (pair weight 100 at r = 4 of 8: heat_rate 20 * 100 / 0.5)
def test_different_capacities_approach_the_energy_weighted_equilibrium():
    sc = heat_scene([(0, 0, 0), (4, 0, 0)], [20, 90], [WATER, IRON])
    st = orc.state_from_scene(sc)
    st.init_enthalpy()
    before = energy(st)
    c0, c1 = 1.0 * 4180, 7.87 * 450
    expected = (20 * c0 + 90 * c1) / (c0 + c1)
    for _ in range(5000):
        st.exchange_heat(.05, heat_rate=20 * 100 / .5)
    assert abs(energy(st) - before) < 1e-5
    assert abs(st.T[0] - expected) < .001 and abs(st.T[1] - expected) < .001


# tests/material-physics.test.mjs:21-31
def test_many_contacts_conserve_energy_without_overshoot_and_iron_conducts_faster():
    for kind in (WATER, IRON):
        rng = np.random.default_rng(1)
        pos = [(0, 0, 0)] + [tuple(rng.uniform(-3, 3, 3)) for _ in range(80)]
        sc = heat_scene(pos, [90] + [20] * 80, [kind] * 81)
        st = orc.state_from_scene(sc)
        st.init_enthalpy()
        before = energy(st)
        st.exchange_heat(1.0, heat_rate=20 * 1000)
        assert abs(energy(st) - before) < .001
        assert np.all(st.T >= 20 - 1e-9) and np.all(st.T <= 90 + 1e-9)
    drops = []
    for kind in (WATER, IRON):  # below the explicit solver's stability cap (heatRate 1, weight 1)
        sc = heat_scene([(0, 0, 0), (4, 0, 0)], [90, 20], [kind, kind])
        st = orc.state_from_scene(sc)
        st.exchange_heat(1.0, heat_rate=1 / .5)
        drops.append(90 - st.T[0])
    assert drops[1] > 20 * drops[0]


# tests/three.test.mjs:27-31
def test_contact_uses_the_3d_distance_and_conserves_enthalpy():
    sc = heat_scene([(0, 0, 0), (0, 0, 20)], [80, 20], [WATER, WATER])
    st = orc.state_from_scene(sc)
    st.init_enthalpy()
    h0 = energy(st)
    st.exchange_heat(1 / 60)
    assert st.T[0] == 80 and st.T[1] == 20
    st.x[1, 2] = 5
    for _ in range(30):
        st.exchange_heat(1 / 60)
    assert st.T[0] < 80 and st.T[1] > 20
    assert abs(energy(st) - h0) < 1e-6


# tests/phase-change.test.mjs:11-18
def test_custom_enthalpy_includes_latent_heat_and_switches_only_at_complete_melting():
    m = orc.material(0, cp=1800.0, melting_point=120.0, latent_heat=120000.0)
    assert orc.lib().oracle_phase_enthalpy(180.0, m) == 444000
    start, end = 216000.0, 336000.0
    for h, was, liquid in (((start + end) / 2, 0, 0), ((start + end) / 2, 1, 1), (start, 1, 0), (end, 0, 1)):
        sc = heat_scene([(0, 0, 0)], [110], [CUSTOM], latent=120000.0)
        st = orc.state_from_scene(sc)
        st.init_enthalpy()
        st.h[0], st.melted[0] = h, was
        st.exchange_heat(1.0)  # a single particle: no pairs, only the decode
        assert st.melted[0] == liquid and abs(st.T[0] - 120.0) < 1e-9
    sc = heat_scene([(0, 0, 0)], [180], [CUSTOM], latent=0.0)  # phase change disabled: stays solid
    st = orc.state_from_scene(sc)
    st.init_enthalpy()
    st.exchange_heat(1.0)
    assert st.melted[0] == 0 and abs(st.T[0] - 180) < 1e-9


# tests/phase-change.test.mjs:44-49: pair weight 0.5 at heatRate 1000 (r = 4 of 8: heat_rate 1000)
def test_contact_heat_melts_custom_material_conserving_enthalpy():
    sc = heat_scene([(0, 0, 0), (4, 0, 0)], [110, 500], [CUSTOM, CUSTOM], latent=120000.0)
    sc.F = np.tile(1.01 * np.eye(3).ravel(), (2, 1))
    st = orc.state_from_scene(sc)
    st.init_enthalpy()
    assert list(st.melted) == [0, 1]
    before = energy(st)
    for _ in range(30):
        st.exchange_heat(1.0, heat_rate=1000)
    assert list(st.melted) == [1, 1]
    assert abs(energy(st) - before) < 1e-7
    assert np.allclose(st.F[0], np.eye(3).ravel())  # reset on melting


def phase_cloud(n=3000, seed=5):
    rng = np.random.default_rng(seed)
    x = rng.uniform(-12, 12, (n, 3))
    mats = [material(CUSTOM, 120000.0), material(IRON)]
    sc = scenes._scene("cloud", DOMAIN, mats, x, (0, 0, 0))
    sc.mat = (rng.uniform(0, 1, n) < .4).astype(np.int32)
    sc.m = np.where(sc.mat == 0, 1.1, 7.87)
    sc.V = np.ones(n)
    sc.T = np.where(x[:, 0] > 0, 300.0, 20.0) + rng.uniform(0, 10, n)
    return sc


def test_oracle_cloud_exchange_conserves_energy():
    sc = phase_cloud()
    st = orc.state_from_scene(sc)
    st.init_enthalpy()
    before = energy(st)
    for _ in range(5):
        st.exchange_heat(1 / 60)
    assert abs(energy(st) - before) <= 1e-9 * abs(before)
    assert 0 < st.melted.sum() < sc.n


# ------------------------------------------------------------------------------ device

def device(sc, runs, dt, radius=8.0, heat_rate=20.0):
    from mpm_b200.solver import Solver
    sol = Solver(sc.domain, sc.n)
    sol.upload(sc)
    q = 0.0
    for _ in range(runs):
        q += sol.exchange_heat(dt, radius, heat_rate=heat_rate)
    out = sol.download(("T", "enthalpy", "melted", "F"))
    sol.close()
    return out, q


@pytest.mark.gpu
def test_device_reference_cases():
    sc = heat_scene([(0, 0, 0), (4, 0, 0)], [20, 90], [WATER, IRON])
    out, _ = device(sc, 500, .05, heat_rate=20 * 100 / .5)
    st = orc.state_from_scene(sc)
    st.init_enthalpy()
    for _ in range(500):
        st.exchange_heat(.05, heat_rate=20 * 100 / .5)
    assert np.max(np.abs(out["T"] - st.T)) < 1e-3
    sc = heat_scene([(0, 0, 0), (0, 0, 20)], [80, 20], [WATER, WATER])
    out, q = device(sc, 1, 1 / 60)
    assert out["T"][0] == 80 and out["T"][1] == 20 and q == 0
    sc = heat_scene([(0, 0, 0), (4, 0, 0)], [110, 500], [CUSTOM, CUSTOM], latent=120000.0)
    sc.F = np.tile(1.01 * np.eye(3).ravel(), (2, 1))
    out, _ = device(sc, 30, 1.0, heat_rate=1000)
    assert list(out["melted"]) == [1, 1]
    assert np.max(np.abs(out["F"][0] - np.eye(3).ravel())) == 0


@pytest.mark.gpu
def test_device_cloud_matches_oracle():
    sc = phase_cloud()
    st = orc.state_from_scene(sc)
    st.init_enthalpy()
    before = energy(st)
    qo = sum(st.exchange_heat(1 / 60) for _ in range(5))
    out, q = device(sc, 5, 1 / 60)
    assert np.max(np.abs(out["T"] - st.T)) <= 1e-4 * 300
    assert np.array_equal(out["melted"], st.melted)
    e = float(np.sum(sc.m * out["enthalpy"]))
    assert abs(e - before) <= 1e-6 * abs(before)
    assert abs(q - qo) <= 1e-4 * qo
