"""Domain and material parameters of the MLS-MPM solid step (SI units).

The reference describes its grid by a domain box and a cell size
(src/three/discretization.js:3-15): two guard cells below the box snapped to the world grid,
``origin = floor(lower/h)*h - 2h`` and ``nodes = ceil((upper-origin)/h) + 3``. Walls apply
separating slip on all six faces (src/three/mpm.js:93). The sticky floor is an added option.

Materials follow the reference's model numbering (src/three/constitutive.js:6-19):
0 fixed-corotated, 1 Neo-Hookean, 2 snow, 3 sand (Drucker-Prager), 4 ideal J2, 5 linear-hardening
J2, 6 Johnson-Cook, 7 simplified Johnson-Cook, 8 cohesive Drucker-Prager, 9 Deshpande-Fleck foam,
10 thermal-softening J2, 11 Norton creep.
The reference fixes mu = lambda = 0.4 E and gives strengths as stress / E
(src/three/mpm.js:34-37, src/three/metal-plasticity.js:1-2); here every parameter is SI and
``Material.reference_units`` rebuilds the reference's convention.
"""
from dataclasses import dataclass, field
import math

MODEL_FIXED_COROTATED = 0
MODEL_NEO_HOOKEAN = 1
MODEL_J2 = 4
MODEL_J2_HARDENING = 5
MODEL_THERMAL_J2 = 10
MODEL_JOHNSON_COOK = 6
MODEL_JOHNSON_COOK_SIMPLE = 7
MODEL_NORTON_CREEP = 11
MODEL_SNOW = 2
MODEL_SAND = 3
MODEL_COHESIVE_DP = 8
MODEL_FOAM = 9
SUPPORTED_MODELS = tuple(range(12))
# src/three/pressure-plasticity.js:2, strengths as stress / E
PRESSURE_DEFAULTS = dict(cohesion=.025, slope=.6, dilatancy=.15, tension=.01, alpha=1.5, plateau=.015, gamma=.01,
                         densify=.02, beta=2.0, epsD=.7)

# Positions are held on the device as unsigned 32-bit fixed point in cell units relative to the
# grid origin, with this many fractional bits (grids up to 1023 cells per axis).
FIXED_FRAC_BITS = 22
FIXED_ONE = 1 << FIXED_FRAC_BITS
MAX_NODES_PER_AXIS = 1023


@dataclass
class Domain:
    lower: tuple
    upper: tuple
    H: float
    gravity: tuple = (0.0, 0.0, 0.0)
    sticky_floor: bool = False
    clamp_positions: bool = True
    mass_eps: float = 1e-12
    cfl: float = 0.4
    dt_max: float = math.inf
    grad_limit: float = 0.08
    cubic: bool = False
    origin: tuple = field(init=False)
    dims: tuple = field(init=False)
    clamp_lo: tuple = field(init=False)
    clamp_hi: tuple = field(init=False)

    def __post_init__(self):
        h = float(self.H)
        self.lower = tuple(float(x) for x in self.lower)
        self.upper = tuple(float(x) for x in self.upper)
        self.origin = tuple(math.floor(x / h + 1e-9) * h - 2 * h for x in self.lower)
        dims = [int(math.ceil((u - o) / h - 1e-9)) + 3 for u, o in zip(self.upper, self.origin)]
        if self.cubic:  # the reference sizes every axis by max(nodes) (src/three/mpm.js:18)
            dims = [max(dims)] * 3
        self.dims = tuple(dims)
        if max(self.dims) > MAX_NODES_PER_AXIS:
            raise ValueError(f"grid of {self.dims} nodes exceeds {MAX_NODES_PER_AXIS} per axis")
        # positions are clamped to the box (src/three/simulation.js:358-365 clamps to the box
        # shrunk by a quarter particle spacing); a margin of 1e-6 cells keeps them strictly inside
        eps = 1e-6 * h
        self.clamp_lo = tuple(x + eps for x in self.lower)
        self.clamp_hi = tuple(x - eps for x in self.upper)


@dataclass
class Material:
    model: int
    mu: float
    lam: float
    density: float = 1000.0
    yield_stress: float = 0.0      # A: initial yield (Pa)
    hardening: float = 0.0         # B (models 5) / H (model 10), Pa per unit plastic strain
    T_ref: float = 293.0           # thermal softening starts (model 10)
    T_hot: float = 1293.0          # full softening reached
    hot_ratio: float = 0.08        # strength fraction left at T_hot
    heat_fraction: float = 0.0     # beta: share of plastic work converted to heat
    specific_heat: float = 1.0     # cp (J/kg/K)
    # Johnson-Cook (models 6, 7): (A + B ep^n)(1 + C ln max(1, rate/rate0))(1 - theta^m)
    jc_n: float = 0.35
    jc_C: float = 0.025
    jc_rate0: float = 1.0
    T_melt: float = 1000.0
    jc_m: float = 1.0
    # Norton creep (model 11): rate exp(Q/R (1/T_ref,abs - 1/T_abs)) (q / stress)^n
    creep_rate: float = 0.0
    creep_Q: float = 0.0
    creep_n: float = 1.0
    creep_stress: float = 1.0
    temperature_offset: float = 0.0  # added to T for the Arrhenius term (273.15 for deg C)
    # snow (2): principal stretches clamped to [1 - yield_strain, 1 + 0.3 yield_strain];
    # sand (3): friction angle (degrees)
    yield_strain: float = 0.025
    friction_deg: float = 35.0
    # cohesive Drucker-Prager (8) and Deshpande-Fleck foam (9), strengths in Pa
    dp_cohesion: float = 0.0
    dp_slope: float = 0.6
    dp_dilatancy: float = 0.15
    dp_tension: float = 0.0
    df_alpha: float = 1.5
    df_plateau: float = 1.0
    df_gamma: float = 0.0
    df_densify: float = 1.0
    df_beta: float = 2.0
    df_eps_d: float = 0.7
    # particle-pair heat exchange (W/m/K) and enthalpy phase change (enabled when latent_heat > 0)
    conductivity: float = 0.0
    melting_point: float = 0.0
    latent_heat: float = 0.0

    def __post_init__(self):
        if self.model not in SUPPORTED_MODELS:
            raise ValueError(f"material model {self.model} is not supported")
        if not (self.mu > 0 and self.lam > -2 * self.mu / 3):
            raise ValueError("moduli must satisfy mu > 0 and 3 lambda + 2 mu > 0")
        if self.model == MODEL_THERMAL_J2 and not self.T_hot > self.T_ref:
            raise ValueError("T_hot must exceed T_ref")

    @staticmethod
    def from_young(model, E, nu, **kw):
        mu = E / (2 * (1 + nu))
        lam = E * nu / ((1 + nu) * (1 - 2 * nu))
        return Material(model=model, mu=mu, lam=lam, **kw)

    @staticmethod
    def reference_units(model, E=1.0, A=.025, B=.08, thermal=None, density=1000.0, pressure=None,
                        yield_strain=.025, friction=35.0):
        """The reference's convention: mu = lambda = 0.4 E, strengths given as stress / E."""
        kw = dict(model=model, mu=.4 * E, lam=.4 * E, density=density)
        if model in (2, 3):
            kw.update(yield_strain=yield_strain, friction_deg=friction)
        if model in (8, 9):
            q = dict(PRESSURE_DEFAULTS, **(pressure or {}))
            kw.update(dp_cohesion=q["cohesion"] * E, dp_slope=q["slope"], dp_dilatancy=q["dilatancy"],
                      dp_tension=q["tension"] * E, df_alpha=q["alpha"], df_plateau=q["plateau"] * E,
                      df_gamma=q["gamma"] * E, df_densify=q["densify"] * E, df_beta=q["beta"], df_eps_d=q["epsD"])
        if model in (4, 5):
            kw.update(yield_stress=A * E, hardening=(B * E if model == 5 else 0.0))
        if model in (6, 7):
            # src/three/metal-plasticity.js:3 defaults, temperatures in deg C
            kw.update(yield_stress=A * E, hardening=B * E, jc_n=.35, jc_C=.025, jc_rate0=1.0, T_ref=20.0,
                      T_melt=1000.0, jc_m=1.0)
        if model in (10, 11):
            # src/three/thermal-plasticity.js:3 defaults, temperatures in deg C
            t = dict(Tref=20, Thot=180, hotRatio=.08, A=.04, H=.04, rate=.0005, Q=35000, n=3, stress=.04)
            t.update(thermal or {})
            kw.update(yield_stress=t["A"] * E, hardening=t["H"] * E, T_ref=t["Tref"],
                      T_hot=t["Thot"], hot_ratio=t["hotRatio"])
            if model == 11:
                kw.update(creep_rate=t["rate"], creep_Q=t["Q"], creep_n=t["n"], creep_stress=t["stress"] * E,
                          temperature_offset=273.15)
        return Material(**kw)

    @property
    def wave_speed(self):
        return math.sqrt((self.lam + 2 * self.mu) / self.density)
