"""Parity at the benchmarked configurations (GPU, through the C ABI, against the FP64 oracle on all host
threads).

The timed workload is the 2,097,152-particle J2 drop on the 128^3 grid (64x64x64-cell block, 8 per
cell, -2 m/s, requested dt 2e-6 s sub-stepped to CFL 0.4), plus its plastic variant (block on the
floor at -60 m/s, so returns run). Same bounds as the small-scene parity tests:
  one substep      grid mass and momentum after P2G <= 1e-6 normwise relative; x <= 1e-6 m, v and C
                   <= 1e-6 relative (C against max|v| 4/h), F <= 1e-6
  ten substeps     (plastic) x <= 1e-6 m, F <= 2e-6, ep <= 2e-6 + 1e-4 max ep
  50 requested     steps through mpm_run, exactly as bench.py times them (about 200 CFL substeps and
                   six physical re-sorts of the particle state): positions within 1e-4 of the domain
                   size, the same substep count within 2%
and the fixed-corotated cube of the first configuration over its full 200 steps (positions within
1e-4 of the domain size).
"""
import os

import numpy as np
import pytest

from oracle import oracle as orc
from mpm_b200 import scenes
from mpm_b200.solver import Solver

pytestmark = pytest.mark.gpu

THREADS = os.cpu_count() or 1


def rel(a, b, floor=0.0):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = max(float(np.max(np.abs(b))), floor)
    return float(np.max(np.abs(a - b)) / (scale if scale > 0 else 1.0))


def c_scale(v, H):
    return float(np.max(np.abs(v))) * 4.0 / H


def requested_step(st, dt_req, max_substeps=48):
    """Simulation3.step's sub-stepping (src/three/simulation.js:305-311) on the oracle."""
    left, n = dt_req, 0
    while left > 1e-6 * dt_req and n < max_substeps:
        dt = min(st.stable_dt(), left)
        if left - dt <= 1e-6 * dt_req:
            dt = left
        st.step(dt, threads=THREADS)
        left -= dt
        n += 1
    return n


def one_substep_checks(sc):
    sol = Solver(sc.domain, sc.n)
    sol.upload(sc)
    st = orc.state_from_scene(sc)
    dt = st.stable_dt()  # the first CFL substep of a requested step
    gm_ref, gp_ref, _ = st.step(dt, threads=THREADS, want_grid=True)
    gm, gp = sol.grid_debug(dt)
    assert rel(gm, gm_ref) <= 1e-6
    assert rel(gp, gp_ref) <= 1e-6
    sol.step_fixed(dt, 1)
    out = sol.download()
    assert np.max(np.abs(out["x"] - st.x)) <= 1e-6
    assert rel(out["v"], st.v) <= 1e-6
    assert rel(out["C"], st.C, c_scale(st.v, sc.domain.H)) <= 1e-6
    assert np.max(np.abs(out["F"] - st.F)) <= 1e-6
    return sol, st, dt


def test_j2_drop_2m_one_substep():
    sc = scenes.j2_drop()
    assert sc.n == 2_097_152
    sol, _, _ = one_substep_checks(sc)
    assert sol.status() == 0
    sol.close()


def test_j2_drop_plastic_2m_one_and_ten_substeps():
    sc = scenes.j2_drop(plastic=True)
    sol, st, dt = one_substep_checks(sc)
    for _ in range(9):
        st.step(dt, threads=THREADS)
    sol.step_fixed(dt, 9)
    out = sol.download()
    assert np.max(st.ep) > 0  # the impact yields
    assert np.max(np.abs(out["x"] - st.x)) <= 1e-6
    assert np.max(np.abs(out["F"] - st.F)) <= 2e-6
    assert np.max(np.abs(out["ep"] - st.ep)) <= 2e-6 + 1e-4 * np.max(st.ep)
    assert sol.status() == 0
    sol.close()


def test_j2_drop_2m_fifty_requested_steps_through_run():
    sc = scenes.j2_drop()
    dt_req = sc.meta["dt"]
    sol = Solver(sc.domain, sc.n)
    sol.upload(sc)
    substeps, advanced = sol.run(dt_req, 50)
    st = orc.state_from_scene(sc)
    ref_substeps = sum(requested_step(st, dt_req) for _ in range(50))
    assert abs(advanced - 50 * dt_req) <= 1e-6 * dt_req
    assert abs(substeps - ref_substeps) <= 0.02 * ref_substeps, (substeps, ref_substeps)
    out = sol.download(("x", "v"))
    assert np.max(np.abs(out["x"] - st.x)) <= 1e-4  # domain size 1 m
    assert sol.status() == 0
    sol.close()


def test_elastic_cube_full_200_steps():
    sc = scenes.elastic_cube()
    dt = sc.meta["dt"]
    steps = sc.meta["steps"]
    assert steps == 200
    sol = Solver(sc.domain, sc.n)
    sol.upload(sc)
    st = orc.state_from_scene(sc)
    for _ in range(steps):
        st.step(dt)
    sol.step_fixed(dt, steps)
    out = sol.download()
    assert np.max(np.abs(out["x"] - st.x)) <= 1e-4  # domain size 1 m
    assert rel(out["v"], st.v) <= 1e-3
    assert np.max(np.abs(out["F"] - st.F)) <= 1e-4
    sol.close()
