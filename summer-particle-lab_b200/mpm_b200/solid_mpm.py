"""SolidMPM: the reference's 2D elastic MPM class (src/solid-mpm.js:20-116) on the B200 library.

`SolidMPM` keeps the reference's method names and argument meaning; every numeric method runs
through the smpm_* C ABI (include/mpm_b200.h), so F and C live on the device and the caller's
Float32 particle arrays are copied in and out per call, as the reference mutates `s` in place.

`SolidSim` holds the parts of the reference's Simulation (src/simulation.js:14-56) the solid path
reads: Float32 x, y, vx, vy, mass, volume; u8 material and pinned; `count`, `settings` and
`scene`. Its `add` and `pin` follow Simulation.add and Structures.pin for the fields they set.
"""
import ctypes
import math

import numpy as np

from . import _lib

CAPACITY = 16000  # src/simulation.js:7
MPM_MATERIALS = (11,)  # MATERIALS[11].mpm (src/materials.js:15)
DENSITY = {11: 1100.0}  # src/materials.js:19-24, row 11
FIELDS = ("f00", "f01", "f10", "f11", "c00", "c01", "c10", "c11")


class SolidSim:
    def __init__(self, capacity=CAPACITY, scene="empty", **settings):
        self.capacity = capacity
        for k in ("x", "y", "vx", "vy", "mass", "volume"):
            setattr(self, k, np.zeros(capacity, np.float32))
        self.material = np.zeros(capacity, np.uint8)
        self.pinned = np.zeros(capacity, np.uint8)
        self.count = 0
        self.scene = scene
        # src/simulation.js:31 defaults
        self.settings = dict(solidStiffness=1, gravity="center", strength=1, boundary=True)
        self.settings.update(settings)
        self.mpm = None

    def add(self, x, y, material, vx=0.0, vy=0.0):
        """Simulation.add for the fields the solid path reads (src/simulation.js:43-51)."""
        if self.count >= self.capacity or not math.isfinite(x + y + vx + vy):
            return False
        i = self.count
        self.count += 1
        if self.mpm is not None:
            self.mpm.resetParticle(i)
        self.x[i], self.y[i], self.vx[i], self.vy[i] = x, y, vx, vy
        self.material[i] = material
        self.mass[i] = DENSITY.get(material, 1000.0) / 1000
        self.volume[i] = 1
        self.pinned[i] = 0
        return True

    def pin(self, i, value):
        """Structures.pin for the fields the solid path reads (src/structures.js:86-91)."""
        self.pinned[i] = 1 if value else 0
        if value:
            self.vx[i] = self.vy[i] = 0

    def remove_at(self, i):
        """Simulation.removeAt for the particle arrays and the deformation fields (src/simulation.js:167-170)."""
        last = self.count - 1
        self.count = last
        if self.mpm is not None:
            self.mpm.removeParticle(i, last)
        for k in ("x", "y", "vx", "vy", "mass", "volume", "material", "pinned"):
            a = getattr(self, k)
            a[i] = a[last]

    def struct(self):
        s = self.settings
        return _lib.SmpmSim(
            count=self.count, scene=_lib.SMPM_SCENES.get(self.scene, 0), boundary=1 if s.get("boundary") else 0,
            gravity=_lib.SMPM_GRAVITY[s.get("gravity", "none")] if s.get("gravity", "none") in _lib.SMPM_GRAVITY else -1,
            solid_stiffness=float(s.get("solidStiffness", 1) if s.get("solidStiffness") is not None else 1),
            strength=float(s.get("strength", 1)),
            x=self.x.ctypes.data, y=self.y.ctypes.data, vx=self.vx.ctypes.data, vy=self.vy.ctypes.data,
            mass=self.mass.ctypes.data, volume=self.volume.ctypes.data, material=self.material.ctypes.data,
            pinned=self.pinned.ctypes.data)


class SolidMPM:
    """src/solid-mpm.js:20-116 on the device."""

    def __init__(self, capacity=CAPACITY):
        self.capacity = capacity
        h = ctypes.c_void_p()
        _lib.check(_lib.lib().smpm_create(capacity, ctypes.byref(h)))
        self.h = h
        ids = (ctypes.c_uint8 * len(MPM_MATERIALS))(*MPM_MATERIALS)
        self._check(_lib.lib().smpm_set_mpm_materials(self.h, ids, len(MPM_MATERIALS)))

    def _check(self, rc):
        return _lib.check2(rc, self.h)

    def close(self):
        if self.h:
            _lib.lib().smpm_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- state (src/solid-mpm.js:26-29)
    def resetParticle(self, i):
        self._check(_lib.lib().smpm_reset_particle(self.h, i))

    def removeParticle(self, i, last):
        self._check(_lib.lib().smpm_remove_particle(self.h, i, last))

    def reset(self):
        self._check(_lib.lib().smpm_reset(self.h))

    def hasParticles(self, s):
        out = ctypes.c_int32()
        st = s.struct()
        self._check(_lib.lib().smpm_has_particles(self.h, ctypes.byref(st), ctypes.byref(out)))
        return bool(out.value)

    # -- numerics (src/solid-mpm.js:37-91)
    def stableStep(self, s):
        dt = ctypes.c_double()
        st = s.struct()
        self._check(_lib.lib().smpm_stable_step(self.h, ctypes.byref(st), ctypes.byref(dt)))
        return dt.value

    def step(self, s, dt):
        st = s.struct()
        self._check(_lib.lib().smpm_step(self.h, ctypes.byref(st), float(dt)))

    def frame(self, s, dt=1 / 60):
        """The MPM branch of Simulation.step (src/simulation.js:239-255): returns (substeps, advanced)."""
        st = s.struct()
        n = ctypes.c_int32()
        adv = ctypes.c_double()
        self._check(_lib.lib().smpm_frame(self.h, ctypes.byref(st), float(dt), ctypes.byref(n), ctypes.byref(adv)))
        return n.value, adv.value

    def stats(self, s):
        out = _lib.SmpmStats()
        st = s.struct()
        self._check(_lib.lib().smpm_stats_get(self.h, ctypes.byref(st), ctypes.byref(out)))
        return dict(count=out.count, minJ=out.min_j, maxJ=out.max_j, strain=out.strain, nodes=out.nodes,
                    substeps=out.substeps)

    # -- the f00..c11 fields (src/solid-mpm.js:5)
    def fields(self, n=None):
        n = self.capacity if n is None else n
        out = np.zeros((8, n), np.float64)
        self._check(_lib.lib().smpm_get_fields(self.h, n, out.ctypes.data))
        return out

    def set_fields(self, fields):
        fields = np.ascontiguousarray(fields, np.float64)
        self._check(_lib.lib().smpm_set_fields(self.h, fields.shape[1], fields.ctypes.data))

    def field(self, name, n=None):
        return self.fields(n)[FIELDS.index(name)]

    # -- body creation (src/solid-mpm.js:92-107), host-side like the reference
    def create(self, s, x1, y1, x2, y2, material=11, shape="panel", fixed=False):
        return create_body(s, x1, y1, x2, y2, material, shape, fixed)


def create_body(s, x1, y1, x2, y2, material=11, shape="panel", fixed=False):
    """SolidMPM.create (src/solid-mpm.js:92-107): a panel or beam of particles 3.6 apart; False
    (and no particle added) for a non-MPM material, non-finite or degenerate input, or when the
    body does not fit in the remaining capacity."""
    if material not in MPM_MATERIALS or not all(math.isfinite(v) for v in (x1, y1, x2, y2)):
        return False
    c = lambda v: max(-530.0, min(530.0, v))
    x1, x2, y1, y2 = c(x1), c(x2), c(y1), c(y2)
    length = math.hypot(x2 - x1, y2 - y1)
    panel = shape == "panel"
    width = abs(x2 - x1) if panel else length
    height = abs(y2 - y1) if panel else 22
    if width < 7 or height < 7:
        return False
    nx = math.floor(width / 3.6) + 1
    ny = math.floor(height / 3.6) + 1
    if nx * ny + s.count > s.capacity:
        return False
    ux, uy = (x2 - x1) / length, (y2 - y1) / length
    sign = lambda v: (v > 0) - (v < 0)
    for row in range(ny):
        for col in range(nx):
            if panel:
                x = x1 + sign(x2 - x1) * col * 3.6
                y = y1 + sign(y2 - y1) * row * 3.6
            else:
                x = x1 + ux * col * 3.6 - uy * (row * 3.6 - height / 2)
                y = y1 + uy * col * 3.6 + ux * (row * 3.6 - height / 2)
            s.add(x, y, material)
            if fixed and col < 2:
                s.pin(s.count - 1, True)
    return True


def simulation(capacity=CAPACITY, scene="empty", **settings):
    """A SolidSim wired to a SolidMPM of the same capacity (the reference's `new Simulation()` pairing)."""
    s = SolidSim(capacity, scene, **settings)
    s.mpm = SolidMPM(capacity)
    return s
