"""Learned return map (mpm_surrogate_* in include/mpm_b200.h): training, inference and the gate.

The network and its training run on the device through the C ABI; this module only moves numpy
arrays across it. Defaults follow the thermo-elastoplastic configuration the map is built for:
trial principal log strains log-uniform in [1e-5, 5e-2] with random principal directions,
temperature uniform in [293, 600] K and plastic strain uniform in [0, 0.2]. Networks for the
Johnson-Cook laws (models 6, 7) train on jc_config() draws and serve the fused step through
Solver.set_return_mode (mpm_set_return_mode).
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import MpmGateCounts, MpmSurrogateConfig, SURROGATE_PARAMS
from .solver import material_struct

_P = ctypes.c_void_p


def config(samples=10_000_000, batch=16384, steps=30000, lr=2e-3, weight_decay=0.0, dep_weight=4.0, cosine=True, seed=31,
           strain_min=1e-5, strain_max=5e-2, T_min=293.0, T_max=600.0, ep_max=0.2, dt_min=0.0, dt_max=0.0, newton=0):
    return MpmSurrogateConfig(samples=samples, batch=batch, steps=steps, lr=lr, weight_decay=weight_decay,
                              dep_weight=dep_weight, cosine=1 if cosine else 0, seed=seed, strain_min=strain_min,
                              strain_max=strain_max, T_min=T_min, T_max=T_max, ep_max=ep_max, dt_min=dt_min,
                              dt_max=dt_max, newton=newton)


def jc_config(samples=4_000_000, batch=16384, steps=8000, lr=2e-3, seed=37, strain_min=1e-4, strain_max=5e-2,
              T_min=293.0, T_max=700.0, ep_max=0.5, dt_min=1e-8, dt_max=1e-5, newton=8):
    """Training and timing draws for a Johnson-Cook network: deviatoric trial log strains log-uniform
    in [strain_min, strain_max] (every other draw a trial stress just above the initial flow stress),
    plastic strain uniform in [0, ep_max], temperature uniform in [T_min, T_max] (model 6 softening),
    substeps log-uniform in [dt_min, dt_max]; the target is the consistency root of the reference's
    bisection (only plastic states weigh in the loss)."""
    return config(samples=samples, batch=batch, steps=steps, lr=lr, seed=seed, strain_min=strain_min,
                  strain_max=strain_max, T_min=T_min, T_max=T_max, ep_max=ep_max, dt_min=dt_min, dt_max=dt_max,
                  newton=newton)


def _f32(a, shape):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32).reshape(shape))


class Surrogate:
    def __init__(self, material, seed=7):
        self.material = material
        h = _P()
        _lib.check(_lib.lib().mpm_surrogate_create(ctypes.byref(material_struct(material)), seed, ctypes.byref(h)))
        self.h = h

    def _check(self, rc):
        if rc != _lib.OK:
            raise _lib.MpmError(rc, _lib.lib().mpm_surrogate_last_error(self.h).decode())

    def close(self):
        if self.h:
            _lib.lib().mpm_surrogate_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def weights(self):
        p = np.empty(SURROGATE_PARAMS, np.float32)
        self._check(_lib.lib().mpm_surrogate_get_weights(self.h, p.ctypes.data))
        return p

    def set_weights(self, p):
        p = _f32(p, (SURROGATE_PARAMS,))
        self._check(_lib.lib().mpm_surrogate_set_weights(self.h, p.ctypes.data))

    def samples(self, n, cfg=None, states=False):
        cfg = cfg or config()
        X = np.empty((n, 8), np.float32)
        Y = np.empty((n, 8), np.float32)
        F = np.empty((n, 9)) if states else None
        ep = np.empty(n) if states else None
        T = np.empty(n) if states else None
        ptr = lambda a: None if a is None else a.ctypes.data
        self._check(_lib.lib().mpm_surrogate_samples(self.h, ctypes.byref(cfg), n, X.ctypes.data, Y.ctypes.data,
                                                     ptr(F), ptr(ep), ptr(T)))
        return (X, Y, F, ep, T) if states else (X, Y)

    def train(self, cfg=None):
        cfg = cfg or config()
        hist = np.empty(cfg.steps, np.float32)
        self._check(_lib.lib().mpm_surrogate_train(self.h, ctypes.byref(cfg), hist.ctypes.data))
        return hist

    def grad(self, X, Y, out_weight=None):
        X = _f32(X, (-1, 8))
        Y = _f32(Y, (-1, 8))
        g = np.empty(SURROGATE_PARAMS, np.float32)
        loss = ctypes.c_double()
        w = None if out_weight is None else _f32(out_weight, (8,))
        self._check(_lib.lib().mpm_surrogate_grad(self.h, X.shape[0], X.ctypes.data, Y.ctypes.data,
                                                  None if w is None else w.ctypes.data, g.ctypes.data,
                                                  ctypes.byref(loss)))
        return loss.value, g

    def forward(self, X):
        X = _f32(X, (-1, 8))
        Y = np.empty((X.shape[0], 8), np.float32)
        self._check(_lib.lib().mpm_surrogate_forward(self.h, X.shape[0], X.ctypes.data, Y.ctypes.data))
        return Y

    def return_map(self, F, ep=None, T=None, gate_tol=2e-3, use_mlp=True):
        F = np.ascontiguousarray(np.asarray(F, dtype=np.float64).reshape(-1, 9))
        n = F.shape[0]
        vec = lambda a: None if a is None else np.ascontiguousarray(np.broadcast_to(np.asarray(a, np.float64), (n,)))
        ep, T = vec(ep), vec(T)
        Fo = np.empty((n, 9))
        dep = np.empty(n)
        tau = np.empty((n, 9))
        path = np.empty(n, np.int8)
        c = MpmGateCounts()
        self._check(_lib.lib().mpm_return_map_learned(self.h, n, F.ctypes.data, None if ep is None else ep.ctypes.data,
                                                      None if T is None else T.ctypes.data, gate_tol,
                                                      1 if use_mlp else 0, Fo.ctypes.data, dep.ctypes.data,
                                                      tau.ctypes.data, path.ctypes.data, ctypes.byref(c)))
        return Fo, dep, tau, path, dict(elastic=c.elastic, learned=c.learned, fallback=c.fallback)

    def time(self, n, iters=10, gate_tol=2e-3, cfg=None):
        cfg = cfg or config()
        me, ml = ctypes.c_double(), ctypes.c_double()
        c = MpmGateCounts()
        self._check(_lib.lib().mpm_surrogate_time(self.h, ctypes.byref(cfg), n, iters, gate_tol, ctypes.byref(me),
                                                  ctypes.byref(ml), ctypes.byref(c)))
        return dict(ms_exact=me.value, ms_learned=ml.value, elastic=c.elastic, learned=c.learned,
                    fallback=c.fallback)

    def time_newton(self, n, iters=10, gate_tol=1e-5, cfg=None):
        """The same Johnson-Cook states through the Newton-gated map without the network
        (mpm_surrogate_time_newton): device ms per call and the gate's counts."""
        cfg = cfg or jc_config()
        ms = ctypes.c_double()
        c = MpmGateCounts()
        self._check(_lib.lib().mpm_surrogate_time_newton(self.h, ctypes.byref(cfg), n, iters, gate_tol, ctypes.byref(ms),
                                                         ctypes.byref(c)))
        return dict(ms=ms.value, elastic=c.elastic, accepted=c.learned, fallback=c.fallback)
