"""Seeded synthetic scenes for the MLS-MPM solid step.

Seeding uses the reference's integer hash ``random(seed, index, attempt, axis)``
(src/three/sampling.js:8-12), so a seed gives bit-identical inputs in every consumer.
Particles are sampled 2x2x2 per cell with a uniform in-sub-cell jitter of +-dx/4 per axis,
and positions are rounded to the device's fixed-point lattice (2^-22 cell) so the FP64 oracle
and the device start from exactly the same state.

The named workloads restate the five benchmark configurations of this port with their shapes,
sizes and value distributions (no external dataset is involved):
  elastic_cube         13,824-particle fixed-corotated block on a 32^3 grid
  j2_drop              J2 linear-hardening block (64x32x64 or 64x64x64 cells, 8 ppc) on 128^3
  thermal_j2           thermal-softening J2 block (80^3 cells, 4,096,000 particles) on 160^3
  ensemble             256 independent J2 scenes of uneven particle and grid counts (or Johnson-Cook)
  jc_impact            Johnson-Cook block (64^3 cells, 8 ppc, 2,097,152 particles) hitting the floor at 60 m/s
  coupled_collision    two thermal J2 blocks colliding at +-20 m/s on 256^3 (16.8M particles)
"""
from dataclasses import dataclass, field
import math

import numpy as np

from .params import Domain, Material, FIXED_ONE, MODEL_FIXED_COROTATED, MODEL_J2, \
    MODEL_J2_HARDENING, MODEL_JOHNSON_COOK_SIMPLE, MODEL_THERMAL_J2

_M32 = np.uint64(0xFFFFFFFF)


def hash_random(seed, index, attempt, axis):
    """Uniform value in [-1, 1) from src/three/sampling.js:8-12 (vectorised over numpy arrays)."""
    seed = np.asarray(seed, dtype=np.uint64)
    index = np.asarray(index, dtype=np.uint64)
    attempt = np.asarray(attempt, dtype=np.uint64)
    axis = np.asarray(axis, dtype=np.uint64)
    h = (seed + ((index + np.uint64(1)) * np.uint64(0x9E3779B9) & _M32)
         + ((attempt * np.uint64(3) + axis + np.uint64(1)) * np.uint64(0x85EBCA6B) & _M32)) & _M32
    h = ((h ^ (h >> np.uint64(16))) * np.uint64(0x7FEB352D)) & _M32
    h = ((h ^ (h >> np.uint64(15))) * np.uint64(0x846CA68B)) & _M32
    h = (h ^ (h >> np.uint64(16))) & _M32
    return h.astype(np.float64) / 4294967296.0 * 2 - 1


@dataclass
class Scene:
    name: str
    domain: Domain
    materials: list
    x: np.ndarray            # (n, 3) float64, metres
    v: np.ndarray            # (n, 3) float64, m/s
    m: np.ndarray            # (n,) kg
    V: np.ndarray            # (n,) m^3 (reference volume)
    mat: np.ndarray          # (n,) int32 material index
    T: np.ndarray = None     # (n,) K
    F: np.ndarray = None     # (n, 9) deformation gradient, row-major (default identity)
    C: np.ndarray = None     # (n, 9) APIC affine matrix (default zero)
    ep: np.ndarray = None    # (n,) plastic strain (default zero)
    pinned: np.ndarray = None
    jp: np.ndarray = None    # (n,) plastic volume ratio Jp of snow / pressure materials (default one)
    dilation: np.ndarray = None  # (n,) sand dilation history (default zero)
    enthalpy: np.ndarray = None  # (n,) J/kg; when given it sets T (and the phase of phase-change materials)
    melted: np.ndarray = None    # (n,) u8 molten flags of phase-change materials
    meta: dict = field(default_factory=dict)

    @property
    def n(self):
        return int(self.x.shape[0])


def quantize_positions(x, domain):
    """Round positions to the device lattice: origin + k * H / 2^22 (exact in float64)."""
    o = np.asarray(domain.origin)
    k = np.rint((x - o) / domain.H * FIXED_ONE)
    return o + k * (domain.H / FIXED_ONE)


def block_particles(domain, cell_lo, cell_hi, seed, index0=0):
    """8 particles per cell (2x2x2 sub-lattice) with +-dx/4 jitter from the reference hash.

    cell_lo/cell_hi are integer cell indices relative to ``domain.lower`` (half-open). Particle
    order is x fastest, then y, then z, then the sub-lattice slot.
    """
    h = domain.H
    lo = np.asarray(cell_lo, dtype=np.int64)
    hi = np.asarray(cell_hi, dtype=np.int64)
    ext = hi - lo
    cz, cy, cx = np.meshgrid(np.arange(ext[2]), np.arange(ext[1]), np.arange(ext[0]), indexing="ij")
    cells = np.stack([cx.ravel(), cy.ravel(), cz.ravel()], axis=1) + lo
    sub = np.array([[i, j, k] for k in (0, 1) for j in (0, 1) for i in (0, 1)], dtype=np.float64)
    base = (cells[:, None, :].astype(np.float64) + 0.25 + 0.5 * sub[None, :, :]).reshape(-1, 3)
    n = base.shape[0]
    idx = np.arange(index0, index0 + n, dtype=np.uint64)
    jitter = np.stack([hash_random(seed, idx, 0, a) for a in range(3)], axis=1)
    x = np.asarray(domain.lower) + (base + 0.25 * jitter) * h
    return quantize_positions(x, domain)


def _scene(name, domain, materials, x, v0, mat_index=0, T=None, meta=None):
    n = x.shape[0]
    h = domain.H
    dens = np.array([materials[mat_index].density])
    V = np.full(n, h ** 3 / 8)
    m = V * dens[0]
    v = np.tile(np.asarray(v0, dtype=np.float64), (n, 1))
    return Scene(name=name, domain=domain, materials=list(materials), x=x, v=v, m=m, V=V,
                 mat=np.full(n, mat_index, dtype=np.int32), T=T, meta=dict(meta or {}))


def elastic_cube(seed=1):
    """Unit cube, dx=1/32, 12^3-cell block at the centre (cells 10..21), 8 ppc (13,824),
    fixed-corotated E=1e5 Pa, nu=0.3, rho=1000, gravity -9.8 y, sticky floor and slip walls,
    dt=1e-4 s, 200 steps."""
    d = Domain(lower=(0, 0, 0), upper=(1, 1, 1), H=1 / 32, gravity=(0, -9.8, 0), sticky_floor=True)
    mat = Material.from_young(MODEL_FIXED_COROTATED, 1e5, 0.3, density=1000.0)
    x = block_particles(d, (10, 10, 10), (22, 22, 22), seed)
    return _scene("elastic_cube", d, [mat], x, (0, 0, 0),
                  meta=dict(dt=1e-4, steps=200, workload="elastic_cube_13824"))


def aluminium_j2(model=MODEL_J2_HARDENING, **kw):
    """E=70 GPa, nu=0.33, yield 250 MPa, hardening 1 GPa, rho=2700."""
    return Material.from_young(model, 70e9, 0.33, density=2700.0, yield_stress=250e6,
                               hardening=1e9, **kw)


def j2_drop(shape=(64, 64, 64), seed=2, grid=128, plastic=False):
    """J2 linear-hardening block with 8 ppc on a 128^3 grid, bottom 0.2 m above the floor,
    v0 = -2 m/s (requested dt 2e-6 s, sub-stepped to CFL 0.4; 1000 requested steps).
    ``plastic=True`` starts the block in contact with the floor at -60 m/s (plastic impact)."""
    d = Domain(lower=(0, 0, 0), upper=(1, 1, 1), H=1 / grid, gravity=(0, -9.8, 0), sticky_floor=True)
    sx, sy, sz = shape
    x0 = (grid - sx) // 2
    z0 = (grid - sz) // 2
    y0 = 1 if plastic else int(round(0.2 * grid))
    x = block_particles(d, (x0, y0, z0), (x0 + sx, y0 + sy, z0 + sz), seed)
    # a uniaxial-strain impact at speed u gives a von Mises stress sqrt(6) mu (2/3) u / c_p: at
    # 20 m/s that is ~168 MPa, below the 250 MPa yield, so the plastic variant impacts at 60 m/s
    v0 = (0, -60.0 if plastic else -2.0, 0)
    name = "j2_drop_plastic" if plastic else "j2_drop"
    n = x.shape[0]
    return _scene(name, d, [aluminium_j2()], x, v0,
                  meta=dict(dt=2e-6, steps=1000, workload=f"{name}_{n}_{sx}x{sy}x{sz}_grid{grid}"))


def johnson_cook_metal(model=MODEL_JOHNSON_COOK_SIMPLE, E=70e9, nu=0.33, yield_stress=250e6, density=2700.0, **kw):
    """Johnson-Cook metal: A = yield_stress, B = A, n = 0.35, C = 0.025, rate0 = 1/s (the reference's
    ratios, src/three/metal-plasticity.js:3), temperatures in K for model 6 (T_ref 293, T_melt 933)."""
    kw.setdefault("hardening", yield_stress)
    return Material.from_young(model, E, nu, density=density, yield_stress=yield_stress, jc_n=0.35, jc_C=0.025,
                               jc_rate0=1.0, T_ref=293.0, T_melt=933.0, jc_m=1.0, **kw)


def jc_impact(shape=(64, 64, 64), seed=4, grid=128, model=MODEL_JOHNSON_COOK_SIMPLE, v0=-60.0):
    """Johnson-Cook block of 8 ppc on a 128^3 grid resting on the floor, moving down at 60 m/s: a
    plastic impact whose returns run the reference's 24-halving bisection (the law the learned
    return map is built for). Requested dt 2e-6 s sub-stepped to CFL 0.4."""
    d = Domain(lower=(0, 0, 0), upper=(1, 1, 1), H=1 / grid, gravity=(0, -9.8, 0), sticky_floor=True)
    sx, sy, sz = shape
    x0 = (grid - sx) // 2
    z0 = (grid - sz) // 2
    x = block_particles(d, (x0, 1, z0), (x0 + sx, 1 + sy, z0 + sz), seed)
    n = x.shape[0]
    T = np.full(n, 293.0) if model == 6 else None
    return _scene("jc_impact", d, [johnson_cook_metal(model)], x, (0, v0, 0), T=T,
                  meta=dict(dt=2e-6, steps=1000, workload=f"jc_impact_{n}_{sx}x{sy}x{sz}_grid{grid}"))


def thermal_j2(seed=3, grid=160, block=80, v0=-20.0):
    """Thermal-softening J2: dsigma_y/dT = -0.3 MPa/K from T_ref = 293 K restated as model 10 with
    hot_ratio 0.001 (T_hot = T_ref + 0.999 * 250e6 / 0.3e6), T0 ~ U[293, 600] K from the hash,
    90% of plastic work to heat (cp = 900). Block of block^3 cells resting on the floor moving
    down at v0 (plastic impact)."""
    d = Domain(lower=(0, 0, 0), upper=(1, 1, 1), H=1 / grid, gravity=(0, -9.8, 0), sticky_floor=True)
    T_ref, hot_ratio = 293.0, 0.001
    T_hot = T_ref + (1 - hot_ratio) * 250e6 / 0.3e6
    mat = aluminium_j2(MODEL_THERMAL_J2, T_ref=T_ref, T_hot=T_hot, hot_ratio=hot_ratio,
                       heat_fraction=0.9, specific_heat=900.0)
    c0 = (grid - block) // 2
    x = block_particles(d, (c0, 1, c0), (c0 + block, 1 + block, c0 + block), seed)
    n = x.shape[0]
    T = 293.0 + (600.0 - 293.0) * (hash_random(seed, np.arange(n, dtype=np.uint64), 1, 0) + 1) / 2
    return _scene("thermal_j2", d, [mat], x, (0, v0, 0), T=T,
                  meta=dict(dt=2e-6, steps=1000, workload=f"thermal_j2_{n}_grid{grid}"))


def coupled_collision(scale=1, seed=5):
    """Two thermal J2 blocks moving at +-20 m/s along x toward each other.

    scale=1: 256^3 grid, blocks of 64x128x128 cells x 8 ppc (2 x 8,388,608 particles), 8-cell gap.
    scale=4: the seed-matched 1/64 subsample (64^3 grid, blocks 16x32x32 cells)."""
    grid = 256 // scale
    d = Domain(lower=(0, 0, 0), upper=(1, 1, 1), H=1 / grid, gravity=(0, -9.8, 0), sticky_floor=True)
    T_ref, hot_ratio = 293.0, 0.001
    mat = aluminium_j2(MODEL_THERMAL_J2, T_ref=T_ref, T_hot=T_ref + (1 - hot_ratio) * 250e6 / 0.3e6,
                       hot_ratio=hot_ratio, heat_fraction=0.9, specific_heat=900.0)
    bx, by, bz = 64 // scale, 128 // scale, 128 // scale
    gap = max(2, 8 // scale)
    xa = grid // 2 - gap // 2 - bx
    xb = grid // 2 + gap - gap // 2
    y0 = (grid - by) // 2
    z0 = (grid - bz) // 2
    a = block_particles(d, (xa, y0, z0), (xa + bx, y0 + by, z0 + bz), seed)
    b = block_particles(d, (xb, y0, z0), (xb + bx, y0 + by, z0 + bz), seed, index0=a.shape[0])
    x = np.concatenate([a, b])
    n = x.shape[0]
    v = np.zeros((n, 3))
    v[: a.shape[0], 0] = 20.0
    v[a.shape[0]:, 0] = -20.0
    T = np.full(n, 293.0)
    s = _scene("coupled_collision", d, [mat], x, (0, 0, 0), T=T,
               meta=dict(dt=1e-6, steps=2000, workload=f"coupled_collision_{n}_grid{grid}",
                         conduction=dict(k=150.0, rho=2700.0, cp=900.0)))
    s.v = v
    return s


def ensemble(count=256, seed0=1000, steps=500, model=MODEL_J2):
    """Independent J2 scenes: N_p log-uniform in [5e3, 2e5], grid side U{32..96} cells over a unit
    cube, E log-uniform [1e4, 1e11] Pa, nu U[0.2, 0.45], yield log-uniform [1e3, 5e8] Pa, rho=1000,
    ideal J2. The block is a centred cube of N_p/8 cells (clamped to 3/4 of the grid side) whose
    bottom sits a quarter of the way up, falling at 2 m/s under gravity. dt per scene comes from
    CFL 0.4."""
    scenes = []
    for s in range(count):
        seed = seed0 + s
        r = [float((hash_random(seed, 0, 0, a) + 1) / 2) for a in range(3)]
        r += [float((hash_random(seed, 1, 0, a) + 1) / 2) for a in range(3)]
        n_p = math.exp(math.log(5e3) + r[0] * (math.log(2e5) - math.log(5e3)))
        grid = 32 + min(64, int(r[1] * 65))
        E = math.exp(math.log(1e4) + r[2] * (math.log(1e11) - math.log(1e4)))
        nu = 0.2 + 0.25 * r[3]
        sy = math.exp(math.log(1e3) + r[4] * (math.log(5e8) - math.log(1e3)))
        side = max(4, min(int(round((n_p / 8) ** (1 / 3))), (3 * grid) // 4))
        d = Domain(lower=(0, 0, 0), upper=(1, 1, 1), H=1 / grid, gravity=(0, -9.8, 0),
                   sticky_floor=True)
        if model == MODEL_JOHNSON_COOK_SIMPLE:  # the same draws as a Johnson-Cook law (B = A)
            mat = johnson_cook_metal(model, E, nu, yield_stress=sy, density=1000.0)
        else:
            mat = Material.from_young(model, E, nu, density=1000.0, yield_stress=sy)
        c0 = (grid - side) // 2
        y0 = max(1, min(grid // 4, grid - side - 2))
        x = block_particles(d, (c0, y0, c0), (c0 + side, y0 + side, c0 + side), seed)
        scenes.append(_scene(f"ensemble_{seed}", d, [mat], x, (0, -2.0, 0),
                             meta=dict(steps=steps, seed=seed, grid=grid, E=E, nu=nu, yield_stress=sy)))
    return scenes


def translation_block(phase=0.0, velocity=(2.0, 0.0, 0.0)):
    """Zero-stress translation case of src/simulation/vv-mpm.js:7-8: cell 0.1 m, 2 particles per
    axis, a 0.2 m cube at density 1100 moving at 2 m/s, no gravity; ``phase`` shifts the cloud
    by a fraction of a cell relative to the grid."""
    d = Domain(lower=(-0.4, 0.0, -0.4), upper=(0.8, 1.0, 0.4), H=0.1, sticky_floor=False)
    mat = Material.from_young(MODEL_FIXED_COROTATED, 1e5, 0.25, density=1100.0)
    h = d.H
    pts = []
    for k in range(4):
        for j in range(4):
            for i in range(4):
                pts.append([-0.1 + (i + 0.5) * 0.05 + phase * h, 0.4 + (j + 0.5) * 0.05,
                            -0.1 + (k + 0.5) * 0.05])
    x = quantize_positions(np.array(pts), d)
    s = _scene("translation", d, [mat], x, velocity)
    s.V[:] = 0.05 ** 3
    s.m[:] = 1100.0 * 0.05 ** 3
    return s


WORKLOADS = {
    "elastic_cube": elastic_cube,
    "jc_impact": jc_impact,
    "j2_drop": j2_drop,
    "thermal_j2": thermal_j2,
    "coupled_collision": coupled_collision,
}
