"""mpm_run: N requested-dt steps in one call (step boundaries on the device, one host round trip)
against N mpm_step calls on a second handle: the same substep counts and the same state (FP32
atomics sum in a different order between two handles, so x within 1e-6 m and F within 1e-6)."""
import numpy as np
import pytest

from mpm_b200 import scenes
from mpm_b200.solver import Solver

pytestmark = pytest.mark.gpu


def impact_scene():
    d = scenes.Domain(lower=(0, 0, 0), upper=(1, 1, 1), H=1 / 32, gravity=(0, -9.8, 0), sticky_floor=True)
    x = scenes.block_particles(d, (10, 1, 10), (22, 7, 22), 7)
    return scenes._scene("j2_impact", d, [scenes.aluminium_j2(5)], x, (0, -60.0, 0))


def pair(sc):
    a = Solver(sc.domain, sc.n)
    a.upload(sc)
    b = Solver(sc.domain, sc.n)
    b.upload(sc)
    return a, b


@pytest.mark.parametrize("max_substeps", [48, 2])
def test_run_matches_consecutive_steps(max_substeps):
    sc = impact_scene()
    a, b = pair(sc)
    dt_req = 4 * a.stable_dt()  # several CFL substeps per step; with max_substeps 2 every step is cut short
    total, adv = 0, 0.0
    for _ in range(12):
        s, t = a.step(dt_req, max_substeps)
        total += s
        adv += t
    s_run, adv_run = b.run(dt_req, 12, max_substeps)
    assert s_run == total
    assert abs(adv_run - adv) <= 1e-9 * adv
    if max_substeps == 2:
        assert adv < 12 * dt_req  # the cap shortened the steps
    oa, ob = a.download(("x", "F", "ep")), b.download(("x", "F", "ep"))
    assert np.max(ob["ep"]) > 0  # the impact yields
    assert np.max(np.abs(oa["x"] - ob["x"])) <= 1e-6
    assert np.max(np.abs(oa["F"] - ob["F"])) <= 1e-6
    a.close()
    b.close()


def test_run_tops_up_a_short_estimate():
    """A step capped at 2 substeps leaves a per-step estimate of 2 for the same requested dt; the
    next mpm_run of 3 full steps (about 4 substeps each) starts from that estimate and adds substeps
    until all its steps are done."""
    sc = impact_scene()
    a, b = pair(sc)
    dt_req = 4 * a.stable_dt()
    assert a.step(dt_req, 2)[0] == 2 and b.step(dt_req, 2)[0] == 2
    total = sum(a.step(dt_req)[0] for _ in range(3))
    s_run, adv_run = b.run(dt_req, 3)
    assert s_run == total and total > 6
    assert abs(adv_run - 3 * dt_req) <= 1e-6 * dt_req
    oa, ob = a.download(("x",)), b.download(("x",))
    assert np.max(np.abs(oa["x"] - ob["x"])) <= 1e-6
    assert a.status() == 0 and b.status() == 0
    a.close()
    b.close()


def test_run_with_regularisation_matches_consecutive_steps():
    """The regularised branch of mpm_run (solid regularisation after every substep, run step by step
    on the host's schedule) against the same requested steps as single mpm_step calls."""
    sc = impact_scene()
    a, b = pair(sc)
    for s in (a, b):
        s.set_regularizer(True)
    dt_req = 3 * a.stable_dt()
    total = sum(a.step(dt_req)[0] for _ in range(4))
    s_run, adv_run = b.run(dt_req, 4)
    assert s_run == total and total >= 8
    assert abs(adv_run - 4 * dt_req) <= 1e-6 * dt_req
    oa, ob = a.download(("x", "F")), b.download(("x", "F"))
    assert np.max(np.abs(oa["x"] - ob["x"])) <= 1e-6
    assert np.max(np.abs(oa["F"] - ob["F"])) <= 1e-6
    a.close()
    b.close()


def test_run_stops_at_a_nonfinite_state():
    """Fault injection on the host: one particle uploaded with a NaN velocity. mpm_run over 20 steps
    stops with MPM_ERR_NONFINITE and the non-finite flag in the status, and a clean handle stepped
    the same way afterwards is unaffected."""
    from mpm_b200._lib import MpmError
    sc = impact_scene()
    good = Solver(sc.domain, sc.n)
    good.upload(sc)
    sc.v[17, 0] = float("nan")
    a = Solver(sc.domain, sc.n)
    a.upload(sc)
    with pytest.raises(MpmError) as e:
        a.run(2e-7, 20)
    assert e.value.code == -4
    assert a.status() & 1
    sub, _ = good.run(2e-7, 3)
    assert sub >= 3 and good.status() == 0
    a.close()
    good.close()
