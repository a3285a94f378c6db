"""Host-side handle of the device MLS-MPM step (one scene), over the C ABI.

``Solver`` owns one library handle: it uploads a ``scenes.Scene``, advances it on the device and
downloads the state. It is the Python face of the same entry points a Node N-API addon binds.
"""
import ctypes
import math

import numpy as np

from . import _lib
from ._lib import MpmDomain, MpmMaterial, MpmParticles, MpmLedger, MpmSceneDesc, MpmTuning, check

_P = ctypes.c_void_p


def domain_struct(d):
    s = MpmDomain()
    for a in range(3):
        s.lower[a] = d.lower[a]
        s.upper[a] = d.upper[a]
        s.gravity[a] = d.gravity[a]
    s.cell_size = d.H
    s.sticky_floor = int(d.sticky_floor)
    s.clamp_positions = int(d.clamp_positions)
    s.mass_eps = d.mass_eps
    s.cfl = d.cfl
    s.dt_max = d.dt_max if math.isfinite(d.dt_max) else 0.0
    s.grad_limit = d.grad_limit
    s.cubic = int(d.cubic)
    return s


def material_struct(m):
    return MpmMaterial(model=m.model, mu=m.mu, lam=m.lam, yield_stress=m.yield_stress,
                       hardening=m.hardening, T_ref=m.T_ref, T_hot=m.T_hot, hot_ratio=m.hot_ratio,
                       heat_fraction=m.heat_fraction, specific_heat=m.specific_heat, jc_n=m.jc_n, jc_C=m.jc_C,
                       jc_rate0=m.jc_rate0, T_melt=m.T_melt, jc_m=m.jc_m, creep_rate=m.creep_rate,
                       creep_Q=m.creep_Q, creep_n=m.creep_n, creep_stress=m.creep_stress,
                       temperature_offset=m.temperature_offset, yield_strain=m.yield_strain,
                       friction_deg=m.friction_deg, dp_cohesion=m.dp_cohesion, dp_slope=m.dp_slope,
                       dp_dilatancy=m.dp_dilatancy, dp_tension=m.dp_tension, df_alpha=m.df_alpha,
                       df_plateau=m.df_plateau, df_gamma=m.df_gamma, df_densify=m.df_densify, df_beta=m.df_beta,
                       df_eps_d=m.df_eps_d, conductivity=m.conductivity, melting_point=m.melting_point,
                       latent_heat=m.latent_heat)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_P)


class Solver:
    def __init__(self, domain, capacity):
        self._keep = []
        self.domain = domain
        h = _P()
        check(_lib.lib().mpm_create(ctypes.byref(domain_struct(domain)), int(capacity), ctypes.byref(h)))
        self.h = h
        self.capacity = int(capacity)
        self.n = 0

    def close(self):
        if self.h:
            _lib.lib().mpm_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        return check(rc, self.h)

    def set_material(self, index, m):
        self._check(_lib.lib().mpm_set_material(self.h, index, ctypes.byref(material_struct(m))))

    def upload(self, scene, dtype=np.float64):
        for i, m in enumerate(scene.materials):
            self.set_material(i, m)
        n = scene.n
        f = np.dtype(dtype)
        arr = lambda a: None if a is None else np.ascontiguousarray(a, dtype=f)
        x = np.ascontiguousarray(scene.x, dtype=f)
        v = np.ascontiguousarray(scene.v, dtype=f)
        cols = [np.ascontiguousarray(x[:, a]) for a in range(3)] + [np.ascontiguousarray(v[:, a]) for a in range(3)]
        m, V = arr(scene.m), arr(scene.V)
        T, ep = arr(scene.T), arr(scene.ep)
        jp, dil = arr(getattr(scene, "jp", None)), arr(getattr(scene, "dilation", None))
        enth = arr(getattr(scene, "enthalpy", None))
        mel = None if getattr(scene, "melted", None) is None else np.ascontiguousarray(scene.melted, dtype=np.uint8)
        F = None if scene.F is None else np.ascontiguousarray(np.asarray(scene.F).reshape(n, 9), dtype=f)
        C = None if scene.C is None else np.ascontiguousarray(np.asarray(scene.C).reshape(n, 9), dtype=f)
        mat = np.ascontiguousarray(scene.mat, dtype=np.int32)
        pin = None if scene.pinned is None else np.ascontiguousarray(scene.pinned, dtype=np.uint8)
        p = MpmParticles(dtype=_lib.F64 if f == np.float64 else _lib.F32,
                         x=_ptr(cols[0]), y=_ptr(cols[1]), z=_ptr(cols[2]), vx=_ptr(cols[3]), vy=_ptr(cols[4]),
                         vz=_ptr(cols[5]), mass=_ptr(m), volume=_ptr(V), temperature=_ptr(T), plastic=_ptr(ep),
                         F=_ptr(F), C=_ptr(C), material=_ptr(mat), pinned=_ptr(pin), jp=_ptr(jp), dilation=_ptr(dil),
                         enthalpy=_ptr(enth), melted=_ptr(mel))
        self._check(_lib.lib().mpm_upload_particles(self.h, n, ctypes.byref(p)))
        self.n = n
        cond = scene.meta.get("conduction") if scene.meta else None
        if cond:
            self.set_conduction(cond["k"], cond["rho"], cond["cp"])

    def set_conduction(self, k, rho, cp, scene=0):
        """Grid heat conduction (W/m/K, kg/m^3, J/kg/K); k <= 0 turns it off."""
        self._check(_lib.lib().mpm_set_conduction(self.h, int(scene), float(k), float(rho), float(cp)))

    def download(self, fields=("x", "v", "F", "C", "ep", "T"), dtype=np.float64):
        n = self.n
        f = np.dtype(dtype)
        out = {}
        p = MpmParticles(dtype=_lib.F64 if f == np.float64 else _lib.F32)
        cols = {}
        if "x" in fields:
            for k, a in zip(("x", "y", "z"), range(3)):
                cols[k] = np.empty(n, dtype=f)
                setattr(p, k, _ptr(cols[k]))
        if "v" in fields:
            for k in ("vx", "vy", "vz"):
                cols[k] = np.empty(n, dtype=f)
                setattr(p, k, _ptr(cols[k]))
        one = {"m": "mass", "V": "volume", "T": "temperature", "ep": "plastic", "jp": "jp", "dilation": "dilation",
               "enthalpy": "enthalpy"}
        for k, name in one.items():
            if k in fields:
                out[k] = np.empty(n, dtype=f)
                setattr(p, name, _ptr(out[k]))
        for k in ("F", "C"):
            if k in fields:
                out[k] = np.empty((n, 9), dtype=f)
                setattr(p, k, _ptr(out[k]))
        if "melted" in fields:
            out["melted"] = np.empty(n, dtype=np.uint8)
            p.melted = _ptr(out["melted"])
        self._check(_lib.lib().mpm_download_particles(self.h, ctypes.byref(p)))
        if "x" in fields:
            out["x"] = np.stack([cols["x"], cols["y"], cols["z"]], axis=1)
        if "v" in fields:
            out["v"] = np.stack([cols["vx"], cols["vy"], cols["vz"]], axis=1)
        return out

    def step(self, dt_requested, max_substeps=48):
        sub = ctypes.c_int32()
        adv = ctypes.c_double()
        self._check(_lib.lib().mpm_step(self.h, dt_requested, max_substeps, ctypes.byref(sub), ctypes.byref(adv)))
        return sub.value, adv.value

    def run(self, dt_requested, nsteps, max_substeps=48):
        """nsteps requested-dt steps in one call (mpm_run); returns (total substeps, time advanced)."""
        sub = ctypes.c_int32()
        adv = ctypes.c_double()
        self._check(_lib.lib().mpm_run(self.h, dt_requested, int(nsteps), max_substeps, ctypes.byref(sub),
                                       ctypes.byref(adv)))
        return sub.value, adv.value

    def step_fixed(self, dt, nsteps=1):
        self._check(_lib.lib().mpm_step_fixed(self.h, dt, nsteps))

    def step_cfl(self, nsteps=1):
        t = ctypes.c_double()
        self._check(_lib.lib().mpm_step_cfl(self.h, nsteps, ctypes.byref(t)))
        return t.value

    def stable_dt(self):
        d = ctypes.c_double()
        self._check(_lib.lib().mpm_stable_dt(self.h, ctypes.byref(d)))
        return d.value

    def ledger(self):
        L = MpmLedger()
        self._check(_lib.lib().mpm_ledger_compute(self.h, ctypes.byref(L)))
        return L

    def status(self):
        s = ctypes.c_uint32()
        self._check(_lib.lib().mpm_status(self.h, ctypes.byref(s)))
        return s.value

    def clear_status(self):
        self._check(_lib.lib().mpm_clear_status(self.h))

    def grid_dims(self):
        dims = (ctypes.c_int32 * 3)()
        org = (ctypes.c_double * 3)()
        self._check(_lib.lib().mpm_grid_dims(self.h, dims, org))
        return tuple(dims), tuple(org)

    def grid_debug(self, dt):
        dims, _ = self.grid_dims()
        nodes = int(np.prod(dims))
        m = np.empty(nodes)
        p = np.empty((nodes, 3))
        self._check(_lib.lib().mpm_grid_debug(self.h, dt, _ptr(m), _ptr(p)))
        return m, p

    def snapshot(self):
        self._check(_lib.lib().mpm_snapshot(self.h))

    def rollback(self):
        self._check(_lib.lib().mpm_rollback(self.h))

    def save(self, path):
        self._check(_lib.lib().mpm_checkpoint_save(self.h, str(path).encode()))

    def load(self, path):
        self._check(_lib.lib().mpm_checkpoint_load(self.h, str(path).encode()))
        cnt = ctypes.c_int64()
        self._check(_lib.lib().mpm_count(self.h, ctypes.byref(cnt)))
        self.n = cnt.value

    def profile(self, on=True):
        self._check(_lib.lib().mpm_profile_enable(self.h, 1 if on else 0))

    def profile_read(self):
        n = len(_lib.PROFILE_KERNELS)
        ms = (ctypes.c_double * n)()
        cnt = (ctypes.c_int64 * n)()
        self._check(_lib.lib().mpm_profile_read(self.h, ms, cnt))
        return {k: (ms[i], cnt[i]) for i, k in enumerate(_lib.PROFILE_KERNELS)}

    def launch_count(self):
        c = ctypes.c_int64()
        self._check(_lib.lib().mpm_launch_count(self.h, ctypes.byref(c)))
        return c.value

    def stream(self):
        s = _P()
        self._check(_lib.lib().mpm_get_stream(self.h, ctypes.byref(s)))
        return s.value

    def reset_particle(self, index):
        self._check(_lib.lib().mpm_reset_particle(self.h, int(index)))

    def remove_particle(self, index, last):
        self._check(_lib.lib().mpm_remove_particle(self.h, int(index), int(last)))
        self.n -= 1

    def set_regularizer(self, enabled=True, spacing=2.8, volume_unit=1.0, max_speed=8.0, rate=40.0):
        """Solid position regularisation (regularizeSolids); defaults are the reference's units."""
        r = _lib.MpmRegularizer(enabled=int(bool(enabled)), spacing=spacing, volume_unit=volume_unit,
                                max_speed=max_speed, rate=rate)
        self._check(_lib.lib().mpm_set_regularizer(self.h, ctypes.byref(r)))

    def exchange_heat(self, dt, radius, geometry=20.0, heat_rate=20.0, ambient=False, ambient_T=15.0,
                      ambient_rate=.003):
        """Particle-pair heat exchange (exchangeHeat) over dt; returns the exchanged heat (sum |Q|)."""
        x = _lib.MpmHeatExchange(radius=radius, geometry=geometry, heat_rate=heat_rate, ambient=int(bool(ambient)),
                                 ambient_T=ambient_T, ambient_rate=ambient_rate)
        q = ctypes.c_double()
        self._check(_lib.lib().mpm_exchange_heat(self.h, ctypes.byref(x), float(dt), ctypes.byref(q)))
        return q.value

    def regularize(self, dt):
        """One regularisation pass now (regularizeSolids(s, dt) after a step)."""
        self._check(_lib.lib().mpm_regularize(self.h, float(dt)))

    def set_return_mode(self, surrogate=None, gate_tol=1e-5, newton=8, mode=None):
        """Learned return map inside the step (mpm_set_return_mode) with a Johnson-Cook network, or
        the exact map again with surrogate None. mode="newton": the same refinement and gate from
        the initial flow stress's guess, without a network."""
        if mode == "newton":
            self._check(_lib.lib().mpm_set_return_mode(self.h, _lib.RETURN_NEWTON_GATED, None, float(gate_tol),
                                                       int(newton)))
        elif mode is not None:
            raise ValueError("mode must be None or 'newton'")
        elif surrogate is None:
            self._check(_lib.lib().mpm_set_return_mode(self.h, _lib.RETURN_EXACT, None, 0.0, 0))
        else:
            self._check(_lib.lib().mpm_set_return_mode(self.h, _lib.RETURN_LEARNED_GATED, surrogate.h, float(gate_tol),
                                                       int(newton)))

    def gate_counts(self, reset=False):
        """(returns served by the network, returns sent to the exact map) since the last reset."""
        c = _lib.MpmGateCounts()
        self._check(_lib.lib().mpm_gate_counts_read(self.h, ctypes.byref(c), 1 if reset else 0))
        return c.learned, c.fallback

    def autotune(self, trial_substeps=8):
        t = MpmTuning()
        self._check(_lib.lib().mpm_batch_autotune(self.h, int(trial_substeps), ctypes.byref(t)))
        return dict(warp_specialised=t.warp_specialised, blocks_per_sm=t.blocks_per_sm, reorder_interval=t.reorder_interval, use_tma=t.use_tma,
                    trials=t.trials, ms_per_substep=t.ms_per_substep, ms_per_substep_default=t.ms_per_substep_default)


class Batch(Solver):
    """Many independent scenes on one handle (mpm_batch_*): scene k uses its own domain, grid,
    CFL dt and material (scene.materials[0], stored at material-table index k)."""

    def __init__(self, scenes):
        self._keep = []
        self.scenes = list(scenes)
        descs = (MpmSceneDesc * len(self.scenes))()
        for k, sc in enumerate(self.scenes):
            descs[k].domain = domain_struct(sc.domain)
            descs[k].material = k
            descs[k].count = sc.n
        h = _P()
        check(_lib.lib().mpm_batch_create(descs, len(self.scenes), ctypes.byref(h)))
        self.h = h
        self.domain = self.scenes[0].domain
        self.capacity = sum(sc.n for sc in self.scenes)
        self.n = 0
        self.offsets = np.cumsum([0] + [sc.n for sc in self.scenes])

    def upload(self, scene=None, dtype=np.float64):
        for k, sc in enumerate(self.scenes):
            self.set_material(k, sc.materials[0])
        f = np.dtype(dtype)

        def cat(name, shape=None):
            if any(getattr(sc, name, None) is None for sc in self.scenes):
                return None
            a = np.concatenate([np.asarray(getattr(sc, name)).reshape((sc.n,) + (shape or ())) for sc in self.scenes])
            return np.ascontiguousarray(a, dtype=np.uint8 if name in ("pinned", "melted") else f)

        x, v = cat("x", (3,)), cat("v", (3,))
        cols = [np.ascontiguousarray(x[:, a]) for a in range(3)] + [np.ascontiguousarray(v[:, a]) for a in range(3)]
        m, V, T, ep = cat("m"), cat("V"), cat("T"), cat("ep")
        F, C, pin = cat("F", (9,)), cat("C", (9,)), cat("pinned")
        jp, dil, enth, mel = cat("jp"), cat("dilation"), cat("enthalpy"), cat("melted")
        p = MpmParticles(dtype=_lib.F64 if f == np.float64 else _lib.F32,
                         x=_ptr(cols[0]), y=_ptr(cols[1]), z=_ptr(cols[2]), vx=_ptr(cols[3]), vy=_ptr(cols[4]),
                         vz=_ptr(cols[5]), mass=_ptr(m), volume=_ptr(V), temperature=_ptr(T), plastic=_ptr(ep),
                         F=_ptr(F), C=_ptr(C), material=None, pinned=_ptr(pin), jp=_ptr(jp), dilation=_ptr(dil),
                         enthalpy=_ptr(enth), melted=_ptr(mel))
        self._check(_lib.lib().mpm_upload_particles(self.h, self.capacity, ctypes.byref(p)))
        self.n = self.capacity

    def run(self, nsteps, graph=True):
        self._check(_lib.lib().mpm_batch_run(self.h, int(nsteps), 1 if graph else 0))

    def times(self):
        t = np.empty(len(self.scenes))
        dt = np.empty(len(self.scenes))
        self._check(_lib.lib().mpm_batch_times(self.h, _ptr(t), _ptr(dt)))
        return t, dt

    def scene_ledger(self, k):
        L = MpmLedger()
        self._check(_lib.lib().mpm_batch_ledger(self.h, int(k), ctypes.byref(L)))
        return L

    def scene_grid_debug(self, k, dt):
        nodes = int(np.prod(self.scenes[k].domain.dims))
        m = np.empty(nodes)
        p = np.empty((nodes, 3))
        self._check(_lib.lib().mpm_batch_grid_debug(self.h, int(k), dt, _ptr(m), _ptr(p)))
        return m, p

    def split(self, out):
        """Per-scene views of a download() result."""
        o = self.offsets
        return [{k: v[o[i]:o[i + 1]] for k, v in out.items()} for i in range(len(self.scenes))]


def return_map_batch(material, F, ep=None, T=None, dt=0.01):
    """Device projectPlastic + stress for a batch (n x 9 F): returns (F_out, dep, tau)."""
    F = np.ascontiguousarray(np.asarray(F, dtype=np.float64).reshape(-1, 9))
    n = F.shape[0]
    ep = None if ep is None else np.ascontiguousarray(np.broadcast_to(np.asarray(ep, dtype=np.float64), (n,)))
    T = None if T is None else np.ascontiguousarray(np.broadcast_to(np.asarray(T, dtype=np.float64), (n,)))
    Fo = np.empty((n, 9))
    dep = np.empty(n)
    tau = np.empty((n, 9))
    check(_lib.lib().mpm_return_map_batch(ctypes.byref(material_struct(material)), n, _ptr(F), _ptr(ep),
                                          _ptr(T), dt, _ptr(Fo), _ptr(dep), _ptr(tau)))
    return Fo, dep, tau
