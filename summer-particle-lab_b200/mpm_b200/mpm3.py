"""MPM3: the reference's 3D solid class (src/three/mpm.js:7-136) on the B200 library.

Method names and argument meaning follow the reference: `configure(domain)`, `reset()`,
`resetParticle(p)`, `remove(p, last)`, `stableStep(s)`, `step(s, dt)`, `refreshDiagnostics(s)`,
`minJ(s)`. As in the reference, the caller owns the particle arrays (`Sim3` here, the fields of
Simulation3 that the solid step reads, src/three/simulation.js:27-30) and the class owns F, C, the
plastic strain and the grid, which live on the device. `step(s, dt)` copies the caller's positions
and velocities in, runs one MLS-MPM step and copies them back, exactly where the reference mutates
s.x..s.vz in place; the first call (or a call after particles were added) uploads the whole state.

Gravity: the reference adds gravity to the particle velocities before `mpm.step`
(src/three/simulation.js:337-344), so a domain used with `step` has zero gravity; `frame(s, dt)`
runs the whole Simulation3.step sub-stepping on the device and takes gravity from the domain.
"""
import ctypes

import numpy as np

from . import _lib
from .params import Domain
from .solver import Solver, domain_struct

CAPACITY3 = 20000  # src/three/simulation.js:16


class Sim3:
    """The caller's particle arrays (FP64 like Simulation3's Float64Arrays)."""

    def __init__(self, capacity=CAPACITY3):
        self.capacity = capacity
        for k in ("x", "y", "z", "vx", "vy", "vz", "mass", "volume", "temperature", "enthalpy"):
            setattr(self, k, np.zeros(capacity))
        self.material = np.zeros(capacity, np.int32)
        self.pinned = np.zeros(capacity, np.uint8)
        self.melted = np.zeros(capacity, np.uint8)
        self.count = 0

    def add(self, x, y, z, mass, volume, material=0, v=(0.0, 0.0, 0.0), temperature=0.0):
        if self.count >= self.capacity:
            return False
        i = self.count
        self.count += 1
        self.x[i], self.y[i], self.z[i] = x, y, z
        self.vx[i], self.vy[i], self.vz[i] = v
        self.mass[i], self.volume[i], self.material[i], self.temperature[i] = mass, volume, material, temperature
        self.pinned[i] = 0
        return True

    def remove(self, i):
        """Simulation3.remove(i) for these arrays (src/three/simulation.js:114); pair with MPM3.remove."""
        last = self.count - 1
        for k in ("x", "y", "z", "vx", "vy", "vz", "mass", "volume", "temperature", "enthalpy", "material", "pinned",
                  "melted"):
            a = getattr(self, k)
            a[i] = a[last]
        self.count = last
        return last

    def particles(self, fields="all"):
        """mpm_particles view of the first `count` entries (FP64 arrays, no copies)."""
        d = lambda a: a.ctypes.data_as(ctypes.c_void_p)
        p = _lib.MpmParticles(dtype=_lib.F64, x=d(self.x), y=d(self.y), z=d(self.z), vx=d(self.vx), vy=d(self.vy),
                              vz=d(self.vz))
        if fields == "all":
            p.mass, p.volume, p.temperature = d(self.mass), d(self.volume), d(self.temperature)
            p.material, p.pinned = d(self.material), d(self.pinned)
        return p


class MPM3:
    def __init__(self, capacity=CAPACITY3, domain=None, materials=None):
        self.capacity = capacity
        self.domain = domain or Domain(lower=(-64, -48, -64), upper=(64, 72, 64), H=8.0)  # DEFAULT_DOMAIN
        self.solver = Solver(self.domain, capacity)
        self.materials = dict(materials or {})
        for k, m in self.materials.items():
            self.solver.set_material(k, m)
        self._count = None  # particle count of the last upload

    def _check(self, rc):
        return _lib.check(rc, self.solver.h)

    def close(self):
        self.solver.close()

    def set_material(self, index, material):
        self.materials[index] = material
        self.solver.set_material(index, material)

    def configure(self, domain):
        """MPM3.configure (src/three/mpm.js:19): a new grid; the next step uploads the state again."""
        self.domain = domain
        self._check(_lib.lib().mpm_configure_domain(self.solver.h, ctypes.byref(domain_struct(domain))))
        self._count = None

    def reset(self):
        self._check(_lib.lib().mpm_reset_deformation(self.solver.h))

    def resetParticle(self, p):
        if self._count is not None and p < self._count:
            self.solver.reset_particle(p)

    def remove(self, p, last):
        if self._count is not None and last == self._count - 1:
            self.solver.remove_particle(p, last)
            self._count -= 1

    def _sync(self, s):
        if self._count != s.count:
            self._check(_lib.lib().mpm_upload_particles(self.solver.h, s.count, ctypes.byref(s.particles())))
            self.solver.n = s.count
            self._count = s.count

    def stableStep(self, s):
        self._sync(s)
        return self.solver.stable_dt()

    def step(self, s, dt):
        self._sync(s)
        if s.count == 0:
            return
        self._check(_lib.lib().mpm_step_host(self.solver.h, ctypes.byref(s.particles("xv")), float(dt)))

    def frame(self, s, dt, max_substeps=48):
        """Simulation3.step's sub-stepping (src/three/simulation.js:305-311) on the device."""
        self._sync(s)
        sub = ctypes.c_int32()
        self._check(_lib.lib().mpm_frame_host(self.solver.h, ctypes.byref(s.particles("xv")), float(dt), max_substeps,
                                              ctypes.byref(sub)))
        return sub.value

    def setRegularizer(self, enabled=True, spacing=2.8, volume_unit=1.0, max_speed=8.0, rate=40.0):
        """Parameters of regularizeSolids (the reference's settings.solidAntiClump and its constants,
        src/three/solid-sampling.js:5-42); `frame` then regularises after every substep."""
        self.solver.set_regularizer(enabled, spacing, volume_unit, max_speed, rate)

    def regularizeSolids(self, s, dt):
        """regularizeSolids(s, dt) (src/three/solid-sampling.js:10-42) on the caller's positions,
        in place, as Simulation3.substep runs it after `step`."""
        self._sync(s)
        if s.count == 0:
            return
        self._check(_lib.lib().mpm_regularize_host(self.solver.h, ctypes.byref(s.particles("xv")), float(dt)))

    def exchangeHeat(self, s, dt, radius=8.0, geometry=20.0, heat_rate=20.0, ambient=False):
        """exchangeHeat(s, pairs, dt) (src/thermal.js:35-56) over the pairs closer than `radius`
        (Simulation3.near's H), on the device state; s.temperature, s.enthalpy and s.melted are
        updated from it. Returns the exchanged heat (Simulation3.exchangedHeat)."""
        self._sync(s)
        if s.count == 0:
            return 0.0
        q = self.solver.exchange_heat(dt, radius, geometry, heat_rate, ambient)
        n = s.count
        d = lambda a: a.ctypes.data_as(ctypes.c_void_p)
        p = _lib.MpmParticles(dtype=_lib.F64, temperature=d(s.temperature), enthalpy=d(s.enthalpy),
                              melted=d(s.melted))
        self._check(_lib.lib().mpm_download_particles(self.solver.h, ctypes.byref(p)))
        assert n == s.count
        return q

    def refreshDiagnostics(self, s):
        """The ledger the V&V panel reads (src/simulation/mechanical-diagnostics.js:16-37), FP64."""
        self._sync(s)
        L = self.solver.ledger()
        return {k: (list(getattr(L, k)) if k in ("momentum", "angular") else getattr(L, k)) for k, _ in L._fields_}

    def minJ(self, s):
        self._sync(s)
        v = ctypes.c_double()
        self._check(_lib.lib().mpm_min_j(self.solver.h, ctypes.byref(v)))
        return v.value
