"""Learned return map: the network's CPU checker, the device gradients, training and the gate.

Pinning. The CPU checker (oracle/mlp_oracle.py) is pinned by central finite differences of its own
FP64 loss. The device forward and backward kernels are then checked against it: with the checker
rounding every tensor-core operand to BF16 where the kernels do, gradients agree within 2e-3
(normwise per parameter block; FP32 accumulation order and rare BF16 tie flips), and within 3e-2
of the unrounded FP64 gradient.

Accuracy of the gated map, against the FP64 restatement of the exact return (oracle_project):
particles below yield and particles the gate rejects take the exact map (stress within 1e-5 of
the initial yield stress of the FP64 result); particles the gate accepts are within
4 * gate_tol * yield (the bound the gate's two residuals imply for a linear-hardening return).
"""
import ctypes
import math

import numpy as np
import pytest

from mpm_b200 import _lib, scenes
from mpm_b200.params import MODEL_THERMAL_J2
from oracle import mlp_oracle as mo

GATE_TOL = 2e-3


def thermal_material():
    # the thermo-elastoplastic scene's law: yield 250 MPa softening 0.3 MPa/K from 293 K
    T_ref, hot = 293.0, 0.001
    return scenes.aluminium_j2(MODEL_THERMAL_J2, T_ref=T_ref, T_hot=T_ref + (1 - hot) * 250e6 / 0.3e6, hot_ratio=hot,
                               heat_fraction=0.9, specific_heat=900.0)


def he_params(seed=0):
    rng = np.random.default_rng(seed)
    w = dict(W1=np.zeros((64, 16)), b1=rng.normal(0, .1, 64), W2=rng.normal(0, math.sqrt(2 / 64), (64, 64)),
             b2=rng.normal(0, .1, 64), W3=np.zeros((8, 64)), b3=np.zeros(8))
    w["W1"][:, :8] = rng.normal(0, math.sqrt(2 / 8), (64, 8))
    w["W3"][:7] = rng.normal(0, math.sqrt(1 / 64), (7, 64))
    w["b3"][:7] = rng.normal(0, .1, 7)
    return mo.pack(w)


def normwise(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-30))


def blocks(g):
    out, k = {}, 0
    for name in mo.ORDER:
        n = int(np.prod(mo.SIZES[name]))
        out[name] = g[k:k + n]
        k += n
    return out


# ------------------------------------------------------------------------------ CPU checker

def test_parameter_layout_matches_header():
    assert mo.NPARAMS == _lib.SURROGATE_PARAMS == 5768


def test_checker_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    p = he_params(2)
    X = rng.normal(0, 1, (32, 8))
    Y = rng.normal(0, 1, (32, 8))
    Y[:, 7] = rng.uniform(0, 1, 32)  # sample weights
    wo = np.array([1, 1, 1, 1, 1, 1, 4, 0.])
    _, g = mo.loss_grad(p, X, Y, wo)
    live = [i for i in range(mo.NPARAMS) if g[i] != 0.0]
    for i in rng.choice(live, 60, replace=False):
        h = 1e-6 * max(1.0, abs(p[i]))
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (mo.loss_grad(pp, X, Y, wo)[0] - mo.loss_grad(pm, X, Y, wo)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])), (i, fd, g[i])


def test_bf16_rounding_is_round_to_nearest_even():
    one = 1.0
    assert mo.bf16(one + 2 ** -8)[()] == 1.0           # tie: rounds to even (1.0)
    assert mo.bf16(one + 3 * 2 ** -8)[()] == 1 + 2 ** -6  # tie: rounds to even (up)
    assert mo.bf16(one + 2 ** -7)[()] == 1 + 2 ** -7     # exact
    assert mo.bf16(-2.5)[()] == -2.5


def test_create_rejects_models_without_a_return_and_null_arguments():
    L = _lib.lib()
    h = ctypes.c_void_p()
    m = _lib.MpmMaterial(model=0, mu=1, lam=1, yield_stress=1)
    assert L.mpm_surrogate_create(ctypes.byref(m), 1, ctypes.byref(h)) == -10
    assert L.mpm_surrogate_create(None, 1, ctypes.byref(h)) == -1
    assert L.mpm_surrogate_destroy(None) == -1


# ------------------------------------------------------------------------------ device

@pytest.mark.gpu
def test_device_gradient_matches_cpu_checker():
    from mpm_b200.surrogate import Surrogate
    s = Surrogate(thermal_material(), seed=3)
    X, Y = s.samples(512)
    p = s.weights().astype(np.float64)
    wo = np.array([1, 1, 1, 1, 1, 1, 4, 0], np.float32)
    loss, g = s.grad(X, Y, wo)
    le, ge = mo.loss_grad(p, X.astype(np.float64), Y.astype(np.float64), wo, emulate_bf16=True)
    lf, gf = mo.loss_grad(p, X.astype(np.float64), Y.astype(np.float64), wo, emulate_bf16=False)
    assert abs(loss - le) <= 1e-3 * le
    gb, eb, fb = blocks(g), blocks(ge), blocks(gf)
    for name in mo.ORDER:
        assert normwise(gb[name], eb[name]) <= 2e-3, (name, normwise(gb[name], eb[name]))
        assert normwise(gb[name], fb[name]) <= 3e-2, (name, normwise(gb[name], fb[name]))
    s.close()


@pytest.mark.gpu
def test_device_forward_matches_cpu_checker():
    from mpm_b200.surrogate import Surrogate
    s = Surrogate(thermal_material(), seed=4)
    X, _ = s.samples(1000)
    y = s.forward(X)
    ye, _ = mo.forward(s.weights().astype(np.float64), X.astype(np.float64), emulate_bf16=True)
    assert normwise(y[:, :7], ye[:, :7]) <= 1e-3
    s.close()


def _fp64_stress(mat, F, ep, T):
    from oracle import oracle as orc
    om = orc.material_from(mat)
    Fo, inc, _ = orc.project(F, om, ep=ep, dt=.01, T=T)
    return orc.constitutive_stress(Fo, mat.model, mat.mu, mat.lam), inc


@pytest.mark.gpu
def test_training_reduces_loss_and_the_gate_bounds_stress_error():
    from mpm_b200.surrogate import Surrogate, config
    mat = thermal_material()
    s = Surrogate(mat, seed=5)
    fresh = Surrogate(mat, seed=5)  # the same network untrained
    hist = s.train(config(samples=1 << 22, batch=16384, steps=12000))
    assert np.all(np.isfinite(hist))
    assert hist[-50:].mean() < 0.1 * hist[:10].mean()
    cfg = config(seed=99)
    _, _, F, ep, T = s.samples(2048, cfg, states=True)
    res = {}
    for name, net in (("trained", s), ("untrained", fresh)):
        Fo, dep, tau, path, counts = net.return_map(F, ep, T, gate_tol=GATE_TOL)
        res[name] = counts
        if name != "trained":
            continue
        Fx, depx, taux, pathx, _ = s.return_map(F, ep, T, use_mlp=False)
        assert np.all((path == 0) == (pathx == 0))  # the elastic decision is the exact one
        for i in range(F.shape[0]):
            soft = 1 - (1 - mat.hot_ratio) * min(1, max(0, (T[i] - mat.T_ref) / (mat.T_hot - mat.T_ref)))
            y0 = mat.yield_stress * soft
            t64, inc64 = _fp64_stress(mat, F[i], ep[i], T[i])
            err = np.max(np.abs(tau[i] - t64)) / y0
            if path[i] == 1:
                assert err <= 4 * GATE_TOL, (i, err)
            else:
                assert err <= 1e-5 * max(1.0, np.max(np.abs(t64)) / y0), (i, path[i], err)
                assert abs(dep[i] - inc64) <= 1e-6
    plastic = res["trained"]["learned"] + res["trained"]["fallback"]
    assert plastic > 100
    # what the trained network gains: the share of plastic returns it serves within the bound
    # (about 18% at this budget and tolerance; the rest fall back to the exact map)
    assert res["trained"]["learned"] >= 0.1 * plastic, res
    assert res["untrained"]["learned"] <= 0.02 * plastic, res
    s.close()
    fresh.close()
