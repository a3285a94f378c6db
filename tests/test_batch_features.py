"""Snow, sand and pressure laws, the solid regularisation and the particle-pair heat exchange on a
batch handle: every scene of a batch must get what a single-scene handle gives it (within FP32
rounding of order-dependent sums, 1e-6 relative), and pairs never cross scenes (GPU tests)."""
import numpy as np
import pytest

from mpm_b200.params import Domain, Material
from mpm_b200.scenes import _scene, block_particles

pytestmark = pytest.mark.gpu
TOL = 1e-6


def rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    s = float(np.max(np.abs(b)))
    return float(np.max(np.abs(a - b)) / (s if s > 0 else 1.0))


def law_scenes():
    """One scene per law with history (snow, sand, cohesive Drucker-Prager, foam), stretching on impact."""
    out = []
    for k, model in enumerate((2, 3, 8, 9)):
        g = 16 + 4 * k
        d = Domain(lower=(0, 0, 0), upper=(1, 1, 1), H=1 / g, gravity=(0, -9.8, 0), sticky_floor=True)
        x = block_particles(d, (4, 1, 4), (4 + g // 2, 5, 4 + g // 2), 31 + k)
        sc = _scene(f"law_{model}", d, [Material.reference_units(model, E=1e6, density=1000.0)], x, (0, -3, 0))
        r = x - x.mean(axis=0)
        sc.v = sc.v + 20.0 * np.stack([r[:, 0], np.zeros(len(r)), r[:, 2]], axis=1)
        sc.jp = np.full(sc.n, 0.95) if model != 3 else None
        out.append(sc)
    return out


def test_history_laws_in_a_batch_match_single_handles():
    from mpm_b200.solver import Batch, Solver
    scenes = law_scenes()
    # the batch needs every optional array on every scene or none: give sand a Jp (ignored by it)
    scenes[1].jp = np.ones(scenes[1].n)
    b = Batch(scenes)
    b.upload()
    b.run(7, graph=False)
    parts = b.split(b.download(("x", "v", "F", "ep", "jp", "dilation")))
    for k, sc in enumerate(scenes):
        s = Solver(sc.domain, sc.n)
        s.upload(sc)
        s.step_cfl(7)
        o = s.download(("x", "v", "F", "ep", "jp", "dilation"))
        for f in ("x", "v", "F"):
            assert rel(parts[k][f], o[f]) <= TOL, (k, f, rel(parts[k][f], o[f]))
        for f in ("ep", "jp", "dilation"):
            assert np.max(np.abs(parts[k][f] - o[f])) <= 1e-6, (k, f)
        s.close()
    b.close()


def two_clouds():
    out = []
    for k in range(2):
        d = Domain(lower=(-64, -48, -64), upper=(64, 72, 64), H=8.0)
        rng = np.random.default_rng(40 + k)
        x = rng.uniform(-10, 10, (1500, 3))
        mat = Material(model=0, mu=.4, lam=.4, specific_heat=1800.0, conductivity=.13 + k, latent_heat=120000.0,
                       melting_point=120.0)
        sc = _scene(f"cloud_{k}", d, [mat], x, (0, 0, 0))
        sc.m = rng.uniform(.5, 2.0, sc.n)
        sc.V = np.ones(sc.n)
        sc.T = np.where(x[:, 0] > 0, 300.0, 20.0)
        out.append(sc)
    return out


def test_regularisation_and_heat_exchange_stay_within_scenes():
    from mpm_b200.solver import Batch, Solver
    scenes = two_clouds()  # the two clouds overlap in space: pairs across scenes would show
    b = Batch(scenes)
    b.upload()
    b.set_regularizer(True)
    b.regularize(1 / 240)
    qb = b.exchange_heat(1 / 60, 8.0)
    parts = b.split(b.download(("x", "T", "melted")))
    qs = 0.0
    for k, sc in enumerate(scenes):
        s = Solver(sc.domain, sc.n)
        s.upload(sc)
        s.set_regularizer(True)
        s.regularize(1 / 240)
        qs += s.exchange_heat(1 / 60, 8.0)
        o = s.download(("x", "T", "melted"))
        assert np.max(np.abs(parts[k]["x"] - o["x"])) <= 1e-5, k
        assert np.max(np.abs(parts[k]["T"] - o["T"])) <= 1e-3, k
        assert np.array_equal(parts[k]["melted"], o["melted"]), k
        s.close()
    assert abs(qb - qs) <= 1e-5 * qs
    b.close()
