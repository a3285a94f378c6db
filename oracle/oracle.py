"""ctypes binding of the FP64 CPU oracle (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this module, and
only as the checker: the product path (mpm_b200) never calls into it.
The C sources restate src/three/mpm.js:25-134, src/three/constitutive.js:22-106,
src/three/metal-plasticity.js:12-38, src/three/thermal-plasticity.js:12-40,
src/three/pressure-plasticity.js:11-48 and src/three/math.js:9-32 of the reference.
"""
import ctypes
import os

import numpy as np

from . import build_oracle

_D = ctypes.c_double
_P = ctypes.c_void_p


class OracleMaterial(ctypes.Structure):
    _fields_ = [("model", ctypes.c_int32), ("pad", ctypes.c_int32),
                ("mu", _D), ("lam", _D),
                ("A", _D), ("B", _D), ("n", _D), ("C", _D), ("rate0", _D), ("Tref", _D),
                ("Tm", _D), ("m", _D),
                ("tTref", _D), ("tThot", _D), ("tHotRatio", _D), ("tA", _D), ("tH", _D),
                ("tRate", _D), ("tQ", _D), ("tN", _D), ("tStress", _D),
                ("beta", _D), ("cp", _D), ("yieldStrain", _D), ("friction", _D),
                ("cohesion", _D), ("slope", _D), ("dilatancy", _D), ("tension", _D), ("alpha", _D),
                ("plateau", _D), ("gamma", _D), ("densify", _D), ("pbeta", _D), ("epsD", _D),
                ("kcond", _D), ("Tphase", _D), ("latent", _D)]


class OracleScene(ctypes.Structure):
    _fields_ = [("origin", _D * 3), ("H", _D), ("dims", ctypes.c_int32 * 3),
                ("sticky_floor", ctypes.c_int32), ("lower", _D * 3), ("upper", _D * 3),
                ("gravity", _D * 3), ("gravity_on_grid", ctypes.c_int32),
                ("clamp_positions", ctypes.c_int32), ("clamp_lo", _D * 3), ("clamp_hi", _D * 3),
                ("mass_eps", _D), ("cfl", _D), ("dt_max", _D), ("grad_limit", _D),
                ("cond_k", _D), ("cond_rho", _D), ("cond_cp", _D)]


class OracleRegularizer(ctypes.Structure):
    """regularizeSolids parameters (src/three/solid-sampling.js:5-42); reference units: 2.8, 1, 8, 40."""
    _fields_ = [("spacing", _D), ("volume_unit", _D), ("max_speed", _D), ("rate", _D)]


class OracleHeat(ctypes.Structure):
    """exchangeHeat parameters; the reference's units: radius 8, geometry 20, heatRate 20."""
    _fields_ = [("radius", _D), ("geometry", _D), ("heat_rate", _D), ("ambient", ctypes.c_int32),
                ("pad", ctypes.c_int32), ("ambient_T", _D), ("ambient_rate", _D)]


class OracleLedger(ctypes.Structure):
    _fields_ = [("mass", _D), ("kinetic", _D), ("affine", _D), ("potential", _D),
                ("elastic", _D), ("momentum", _D * 3), ("angular", _D * 3), ("min_j", _D),
                ("max_j", _D), ("max_plastic", _D), ("max_von_mises", _D),
                ("nonfinite", ctypes.c_int64), ("invalid_j", ctypes.c_int64),
                ("unsupported_elastic", ctypes.c_int64)]


# Reference defaults (src/three/metal-plasticity.js:3, src/three/thermal-plasticity.js:3)
PLASTICITY_DEFAULTS = dict(A=.025, B=.08, n=.35, C=.025, rate0=1, Tref=20, Tm=1000, m=1)
THERMAL_DEFAULTS = dict(Tref=20, Thot=180, hotRatio=.08, A=.04, H=.04, rate=.0005, Q=35000, n=3,
                        stress=.04)
# src/three/pressure-plasticity.js:2 (strengths / E)
PRESSURE_DEFAULTS = dict(cohesion=.025, slope=.6, dilatancy=.15, tension=.01, alpha=1.5, plateau=.015, gamma=.01,
                         densify=.02, beta=2, epsD=.7)

_lib = None


def use_native():
    """Switch this process to the -march=native build of the oracle (compiled here on first use).
    Only the CPU-baseline timing calls it; the tests use the portable build."""
    global _lib
    _lib = _load(build_oracle.build(native=True))
    return build_oracle.NATIVE_ISA


def lib():
    global _lib
    if _lib is None:
        _lib = _load(build_oracle.build())
    return _lib


def _load(path):
    L = ctypes.CDLL(path)
    P = ctypes.POINTER
    L.oracle_svd3.argtypes = [_P, _P, _P, _P]
    L.oracle_compose.argtypes = [_P, _P, _P, _P]
    L.oracle_rotation.argtypes = [_P, _P]
    L.oracle_stress3.argtypes = [_P, _D, _D, _P]
    L.oracle_von_mises.argtypes = [_P, _D]
    L.oracle_von_mises.restype = _D
    L.oracle_constitutive_stress.argtypes = [_P, ctypes.c_int, _D, _D, _P]
    L.oracle_constitutive_stress.restype = ctypes.c_int
    L.oracle_flow_stress.argtypes = [ctypes.c_int, _D, _D, _D, P(OracleMaterial)]
    L.oracle_flow_stress.restype = _D
    L.oracle_thermal_strength.argtypes = [_D, _D, P(OracleMaterial)]
    L.oracle_thermal_strength.restype = _D
    L.oracle_creep_log_rate.argtypes = [_D, _D, P(OracleMaterial)]
    L.oracle_creep_log_rate.restype = _D
    L.oracle_metal_return.argtypes = [_P, ctypes.c_int, _D, _D, _D, P(OracleMaterial), _P, _P]
    L.oracle_thermal_return.argtypes = [_P, ctypes.c_int, _D, _D, _D, P(OracleMaterial), _P, _P]
    L.oracle_project.argtypes = [_P, P(OracleMaterial), _D, _D, _D, _P, _P, _P, _P, _P]
    L.oracle_project.restype = ctypes.c_int
    L.oracle_hardening.argtypes = [_D]
    L.oracle_hardening.restype = _D
    L.oracle_foam_strength.argtypes = [_D, P(OracleMaterial)]
    L.oracle_foam_strength.restype = _D
    L.oracle_step.argtypes = [P(OracleScene), P(OracleMaterial), ctypes.c_int32, ctypes.c_int64,
                              _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _D, _P, _P, _P,
                              ctypes.c_int32]
    L.oracle_step.restype = ctypes.c_int
    L.oracle_stable_dt.argtypes = [P(OracleScene), P(OracleMaterial), ctypes.c_int64,
                                   _P, _P, _P, _P, _P, _P, _P]
    L.oracle_stable_dt.restype = _D
    L.oracle_ledger.argtypes = [P(OracleScene), P(OracleMaterial), ctypes.c_int64, _P, _P, _P,
                                _P, _P, _P, _P, _P, _P, P(OracleLedger)]
    L.oracle_regularize.argtypes = [P(OracleRegularizer), P(OracleMaterial), ctypes.c_int64, _P, _P, _P, _P, _P,
                                    _P, _P, _D, _P, _P]
    L.oracle_phase_enthalpy.argtypes = [_D, P(OracleMaterial)]
    L.oracle_phase_enthalpy.restype = _D
    L.oracle_exchange_heat.argtypes = [P(OracleHeat), P(OracleMaterial), ctypes.c_int64, _P, _P, _P, _P, _P, _P,
                                       _P, _P, _P, _P, _P, _P, _D]
    L.oracle_exchange_heat.restype = _D
    return L


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _f64(a, shape=None):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
    return a.reshape(shape) if shape is not None else a


def material(model, mu=.4, lam=.4, plasticity=None, thermal=None, beta=0.0, cp=1.0, yield_strain=.025,
             friction=35.0, pressure=None, conductivity=0.0, melting_point=0.0, latent_heat=0.0):
    """Oracle material. Defaults are the reference's units: mu = lambda = 0.4 (E = 1)."""
    p = dict(PLASTICITY_DEFAULTS, **(plasticity or {}))
    t = dict(THERMAL_DEFAULTS, **(thermal or {}))
    q = dict(PRESSURE_DEFAULTS, **(pressure or {}))
    return OracleMaterial(model=model, mu=mu, lam=lam, A=p["A"], B=p["B"], n=p["n"], C=p["C"],
                          rate0=p["rate0"], Tref=p["Tref"], Tm=p["Tm"], m=p["m"],
                          tTref=t["Tref"], tThot=t["Thot"], tHotRatio=t["hotRatio"], tA=t["A"],
                          tH=t["H"], tRate=t["rate"], tQ=t["Q"], tN=t["n"], tStress=t["stress"],
                          beta=beta, cp=cp, yieldStrain=yield_strain, friction=friction,
                          cohesion=q["cohesion"], slope=q["slope"], dilatancy=q["dilatancy"], tension=q["tension"],
                          alpha=q["alpha"], plateau=q["plateau"], gamma=q["gamma"], densify=q["densify"],
                          pbeta=q["beta"], epsD=q["epsD"], kcond=conductivity, Tphase=melting_point,
                          latent=latent_heat)


def hardening(jp):
    return lib().oracle_hardening(jp)


def foam_strength(ep, mat):
    return lib().oracle_foam_strength(ep, ctypes.byref(mat))


def svd3(F):
    F = _f64(F, (9,))
    u, v, s = np.zeros(9), np.zeros(9), np.zeros(3)
    lib().oracle_svd3(_ptr(F), _ptr(u), _ptr(v), _ptr(s))
    return u, v, s


def compose(u, v, sigma):
    out = np.zeros(9)
    lib().oracle_compose(_ptr(_f64(u)), _ptr(_f64(v)), _ptr(_f64(sigma)), _ptr(out))
    return out


def rotation(F):
    out = np.zeros(9)
    lib().oracle_rotation(_ptr(_f64(F, (9,))), _ptr(out))
    return out


def stress3(F, mu, lam):
    out = np.zeros(9)
    lib().oracle_stress3(_ptr(_f64(F, (9,))), mu, lam, _ptr(out))
    return out


def von_mises(tau, J=1.0):
    return lib().oracle_von_mises(_ptr(_f64(tau, (9,))), J)


def constitutive_stress(F, model, mu, lam):
    out = np.zeros(9)
    rc = lib().oracle_constitutive_stress(_ptr(_f64(F, (9,))), model, mu, lam, _ptr(out))
    if rc != 0:
        raise ValueError(f"model {model} is out of scope")
    return out


def flow_stress(model, ep, rate, T, mat):
    return lib().oracle_flow_stress(model, ep, rate, T, ctypes.byref(mat))


def thermal_strength(ep, T, mat):
    return lib().oracle_thermal_strength(ep, T, ctypes.byref(mat))


def creep_log_rate(q, T, mat):
    return lib().oracle_creep_log_rate(q, T, ctypes.byref(mat))


def metal_return(sigma, model, ep, dt, T, mat):
    out, inc = np.zeros(3), np.zeros(1)
    lib().oracle_metal_return(_ptr(_f64(sigma)), model, ep, dt, T, ctypes.byref(mat), _ptr(out), _ptr(inc))
    return out, float(inc[0])


def thermal_return(sigma, model, ep, dt, T, mat):
    out, inc = np.zeros(3), np.zeros(1)
    lib().oracle_thermal_return(_ptr(_f64(sigma)), model, ep, dt, T, ctypes.byref(mat), _ptr(out), _ptr(inc))
    return out, float(inc[0])


def project(F, mat, ep=0.0, dt=.01, T=20.0):
    """projectPlastic (constitutive.js:52-78): returns (F_out, increment, cached tau)."""
    r = project_state(F, mat, ep=ep, dt=dt, T=T)
    return r["F"], r["increment"], r["tau"]


def project_state(F, mat, jp=1.0, dilation=0.0, ep=0.0, dt=.01, T=20.0):
    """projectPlastic with the history scalars: dict(F, jp, dilation, increment, tau)."""
    Fo, inc, tau = np.zeros(9), np.zeros(1), np.zeros(9)
    j, d = np.array([float(jp)]), np.array([float(dilation)])
    rc = lib().oracle_project(_ptr(_f64(F, (9,))), ctypes.byref(mat), ep, dt, T, _ptr(j), _ptr(d), _ptr(Fo),
                              _ptr(inc), _ptr(tau))
    if rc != 0:
        raise ValueError("model out of scope")
    return dict(F=Fo, jp=float(j[0]), dilation=float(d[0]), increment=float(inc[0]), tau=tau)


def scene_struct(domain):
    """OracleScene from a mpm_b200.scenes.Domain-like object."""
    s = OracleScene()
    for a in range(3):
        s.origin[a] = domain.origin[a]
        s.dims[a] = domain.dims[a]
        s.lower[a] = domain.lower[a]
        s.upper[a] = domain.upper[a]
        s.gravity[a] = domain.gravity[a]
        s.clamp_lo[a] = domain.clamp_lo[a]
        s.clamp_hi[a] = domain.clamp_hi[a]
    s.H = domain.H
    s.sticky_floor = int(domain.sticky_floor)
    s.gravity_on_grid = int(getattr(domain, "gravity_on_grid", 0))
    s.clamp_positions = int(domain.clamp_positions)
    s.mass_eps = domain.mass_eps
    s.cfl = domain.cfl
    s.dt_max = domain.dt_max
    s.grad_limit = domain.grad_limit
    return s


class OracleState:
    """FP64 particle state advanced by oracle_step. Arrays are numpy float64 (n,3)/(n,9)/(n,)."""

    def __init__(self, scene, materials):
        self.domain = scene.domain
        self.sc = scene_struct(scene.domain)
        self.mats = (OracleMaterial * len(materials))(*materials)
        self.nmat = len(materials)
        n = scene.n
        self.n = n
        self.x = _f64(scene.x, (n, 3)).copy()
        self.v = _f64(scene.v, (n, 3)).copy()
        self.C = _f64(scene.C, (n, 9)).copy() if scene.C is not None else np.zeros((n, 9))
        self.F = _f64(scene.F, (n, 9)).copy() if scene.F is not None else np.tile(np.eye(3).ravel(), (n, 1))
        self.ep = _f64(scene.ep).copy() if scene.ep is not None else np.zeros(n)
        self.T = _f64(scene.T).copy() if scene.T is not None else np.zeros(n)
        self.jp = _f64(scene.jp).copy() if getattr(scene, "jp", None) is not None else np.ones(n)
        self.dilation = _f64(scene.dilation).copy() if getattr(scene, "dilation", None) is not None else np.zeros(n)
        self.m = _f64(scene.m).copy()
        self.V = _f64(scene.V).copy()
        self.mat = np.ascontiguousarray(np.asarray(scene.mat, dtype=np.int32))
        self.pinned = None if scene.pinned is None else np.ascontiguousarray(scene.pinned, dtype=np.uint8)
        self.tau_cache = np.zeros((n, 9))
        self.cache_valid = np.zeros(n, dtype=np.uint8)

    def step(self, dt, threads=1, want_grid=False):
        nodes = int(np.prod(self.domain.dims))
        gm = np.zeros(nodes) if want_grid else None
        gp = np.zeros((nodes, 3)) if want_grid else None
        gv = np.zeros((nodes, 3)) if want_grid else None
        rc = lib().oracle_step(ctypes.byref(self.sc), self.mats, self.nmat, self.n,
                               _ptr(self.x), _ptr(self.v), _ptr(self.C), _ptr(self.F), _ptr(self.ep),
                               _ptr(self.T), _ptr(self.jp), _ptr(self.dilation), _ptr(self.m), _ptr(self.V),
                               _ptr(self.mat),
                               _ptr(self.pinned), _ptr(self.tau_cache), _ptr(self.cache_valid), dt,
                               _ptr(gm), _ptr(gp), _ptr(gv), threads)
        if rc != 0:
            raise RuntimeError(f"oracle_step failed: {rc}")
        return (gm, gp, gv) if want_grid else None

    def set_conduction(self, k, rho, cp):
        """Grid heat conduction (k W/m/K, density, specific heat); k <= 0 turns it off."""
        self.sc.cond_k, self.sc.cond_rho, self.sc.cond_cp = k, rho, cp

    def stable_dt(self):
        return lib().oracle_stable_dt(ctypes.byref(self.sc), self.mats, self.n, _ptr(self.v),
                                      _ptr(self.C), _ptr(self.F), _ptr(self.m), _ptr(self.V),
                                      _ptr(self.mat), _ptr(self.jp))

    def regularize(self, dt, spacing=2.8, volume_unit=1.0, max_speed=8.0, rate=40.0):
        """regularizeSolids after a step: moves x only, clamped to the domain's clamp box."""
        rg = OracleRegularizer(spacing=spacing, volume_unit=volume_unit, max_speed=max_speed, rate=rate)
        d = self.domain
        lo = np.array(d.clamp_lo if d.clamp_positions else d.origin, dtype=np.float64)
        hi = np.array(d.clamp_hi if d.clamp_positions else
                      [o + (n - 1) * d.H for o, n in zip(d.origin, d.dims)], dtype=np.float64)
        lib().oracle_regularize(ctypes.byref(rg), self.mats, self.n, _ptr(self.x), _ptr(self.F), _ptr(self.jp),
                                _ptr(self.V), _ptr(self.m), _ptr(self.mat), _ptr(self.pinned), dt, _ptr(lo), _ptr(hi))

    def init_enthalpy(self):
        """Simulation3's enthalpy and molten flags from the temperatures (phaseEnthalpy)."""
        L = lib()
        self.h = np.array([L.oracle_phase_enthalpy(float(self.T[i]), ctypes.byref(self.mats[self.mat[i]]))
                           for i in range(self.n)])
        self.melted = np.array([1 if (self.mats[self.mat[i]].latent > 0 and self.T[i] > self.mats[self.mat[i]].Tphase)
                                else 0 for i in range(self.n)], dtype=np.uint8)

    def exchange_heat(self, dt, radius=8.0, geometry=20.0, heat_rate=20.0, ambient=False, ambient_T=15.0,
                      ambient_rate=.003):
        """exchangeHeat over the pairs closer than radius; returns the exchanged heat (sum |Q|)."""
        if not hasattr(self, "h"):
            self.init_enthalpy()
        x = OracleHeat(radius=radius, geometry=geometry, heat_rate=heat_rate, ambient=int(ambient),
                       ambient_T=ambient_T, ambient_rate=ambient_rate)
        if self.pinned is None:
            self.pinned = np.zeros(self.n, dtype=np.uint8)
        return lib().oracle_exchange_heat(ctypes.byref(x), self.mats, self.n, _ptr(self.x), _ptr(self.T), _ptr(self.h),
                                          _ptr(self.melted), _ptr(self.m), _ptr(self.mat), _ptr(self.pinned),
                                          _ptr(self.F), _ptr(self.C), _ptr(self.ep), _ptr(self.jp),
                                          _ptr(self.dilation), dt)

    def ledger(self):
        L = OracleLedger()
        lib().oracle_ledger(ctypes.byref(self.sc), self.mats, self.n, _ptr(self.x), _ptr(self.v),
                            _ptr(self.C), _ptr(self.F), _ptr(self.ep), _ptr(self.m), _ptr(self.V),
                            _ptr(self.mat), _ptr(self.jp), ctypes.byref(L))
        return L


def material_from(mat):
    """Oracle material matching a product Material (SI parameters, read by attribute)."""
    if mat.model in (4, 5):
        return material(mat.model, mu=mat.mu, lam=mat.lam,
                        plasticity=dict(A=mat.yield_stress, B=mat.hardening),
                        beta=mat.heat_fraction, cp=mat.specific_heat)
    if mat.model in (6, 7):
        return material(mat.model, mu=mat.mu, lam=mat.lam,
                        plasticity=dict(A=mat.yield_stress, B=mat.hardening, n=mat.jc_n, C=mat.jc_C,
                                        rate0=mat.jc_rate0, Tref=mat.T_ref, Tm=mat.T_melt, m=mat.jc_m),
                        beta=mat.heat_fraction, cp=mat.specific_heat)
    if mat.model in (10, 11):
        if mat.model == 11 and mat.temperature_offset != 273.15:
            raise ValueError("the restated creep law takes temperatures in deg C (offset 273.15)")
        return material(mat.model, mu=mat.mu, lam=mat.lam,
                        thermal=dict(Tref=mat.T_ref, Thot=mat.T_hot, hotRatio=mat.hot_ratio,
                                     A=mat.yield_stress, H=mat.hardening, rate=mat.creep_rate, Q=mat.creep_Q,
                                     n=mat.creep_n, stress=mat.creep_stress),
                        beta=mat.heat_fraction, cp=mat.specific_heat)
    if mat.model in (2, 3):
        return material(mat.model, mu=mat.mu, lam=mat.lam, yield_strain=mat.yield_strain, friction=mat.friction_deg)
    if mat.model in (8, 9):
        return material(mat.model, mu=mat.mu, lam=mat.lam,
                        pressure=dict(cohesion=mat.dp_cohesion, slope=mat.dp_slope, dilatancy=mat.dp_dilatancy,
                                      tension=mat.dp_tension, alpha=mat.df_alpha, plateau=mat.df_plateau,
                                      gamma=mat.df_gamma, densify=mat.df_densify, beta=mat.df_beta,
                                      epsD=mat.df_eps_d))
    return material(mat.model, mu=mat.mu, lam=mat.lam)


def _with_heat(om, mat):
    om.cp = getattr(mat, "specific_heat", om.cp)
    om.kcond = getattr(mat, "conductivity", 0.0)
    om.Tphase = getattr(mat, "melting_point", 0.0)
    om.latent = getattr(mat, "latent_heat", 0.0)
    return om


def state_from_scene(scene):
    """OracleState for a mpm_b200.scenes.Scene (with its grid heat conduction, if any)."""
    st = OracleState(scene, [_with_heat(material_from(m), m) for m in scene.materials])
    cond = scene.meta.get("conduction") if scene.meta else None
    if cond:
        st.set_conduction(cond["k"], cond["rho"], cond["cp"])
    return st
