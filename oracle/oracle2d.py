"""ctypes binding of the FP64 2D solid oracle (oracle/solid_mpm2d_oracle.cpp; test infrastructure only).

Only tests/ import this module, and only as the checker. It restates src/solid-mpm.js:10-116 and the
MPM branch of src/simulation.js:239-298. `Oracle2` owns the eight FP64 deformation fields like the
reference's SolidMPM; the simulation object passed to each call is duck-typed (x, y, vx, vy, mass,
volume as float32 arrays, material and pinned as uint8, count, scene, settings), and the oracle
mutates its float32 arrays in place exactly as the reference mutates its Float32Arrays.
"""
import ctypes

import numpy as np

from .oracle import lib

_D = ctypes.c_double
_P = ctypes.c_void_p


class Oracle2Sim(ctypes.Structure):
    _fields_ = [("count", ctypes.c_int32), ("scene", ctypes.c_int32), ("boundary", ctypes.c_int32),
                ("gravity", ctypes.c_int32), ("stiffness", _D), ("strength", _D),
                ("x", _P), ("y", _P), ("vx", _P), ("vy", _P), ("mass", _P), ("volume", _P),
                ("material", _P), ("pinned", _P), ("mpm_material", _P)]


class Oracle2State(ctypes.Structure):
    _fields_ = [("capacity", ctypes.c_int64), ("f", _P * 8), ("substeps", ctypes.c_int32),
                ("active_nodes", ctypes.c_int32)]


class Oracle2Stats(ctypes.Structure):
    _fields_ = [("count", ctypes.c_int32), ("min_j", _D), ("max_j", _D), ("strain", _D),
                ("nodes", ctypes.c_int32), ("substeps", ctypes.c_int32)]


SCENES = {"softbody": 1, "basin": 2}
GRAVITY = {"none": 0, "center": 1, "uniform": 2}
_bound = False


def _lib():
    global _bound
    L = lib()
    if not _bound:
        L.oracle2_solid_stress.argtypes = [_D, _D, _D, _D, _D, _D, _P]
        L.oracle2_stable_step.restype = _D
        L.oracle2_stable_step.argtypes = [ctypes.POINTER(Oracle2State), ctypes.POINTER(Oracle2Sim)]
        L.oracle2_step.argtypes = [ctypes.POINTER(Oracle2State), ctypes.POINTER(Oracle2Sim), _D, _P]
        L.oracle2_apply_forces.argtypes = [ctypes.POINTER(Oracle2Sim), _D]
        L.oracle2_frame.restype = ctypes.c_int
        L.oracle2_frame.argtypes = [ctypes.POINTER(Oracle2State), ctypes.POINTER(Oracle2Sim), _D, ctypes.POINTER(_D)]
        L.oracle2_stats.argtypes = [ctypes.POINTER(Oracle2State), ctypes.POINTER(Oracle2Sim),
                                    ctypes.POINTER(Oracle2Stats)]
        _bound = True
    return L


def solid_stress(a, b, c, d, mu, lam):
    out = np.zeros(4)
    _lib().oracle2_solid_stress(a, b, c, d, mu, lam, out.ctypes.data)
    return out


class Oracle2:
    """FP64 SolidMPM: fields[8][capacity] = f00 f01 f10 f11 c00 c01 c10 c11."""

    def __init__(self, capacity, mpm_materials=(11,)):
        self.fields = np.zeros((8, capacity))
        self.fields[0] = self.fields[3] = 1
        self.flags = np.zeros(256, np.uint8)
        for m in mpm_materials:
            self.flags[m] = 1
        self.st = Oracle2State(capacity=capacity)
        for k in range(8):
            self.st.f[k] = self.fields[k].ctypes.data

    def reset_particle(self, i):
        self.fields[:, i] = 0
        self.fields[0, i] = self.fields[3, i] = 1

    def remove_particle(self, i, last):
        self.fields[:, i] = self.fields[:, last]

    def _sim(self, s):
        st = s.settings
        for k in ("x", "y", "vx", "vy", "mass", "volume"):
            assert getattr(s, k).dtype == np.float32 and getattr(s, k).flags.c_contiguous
        return Oracle2Sim(count=s.count, scene=SCENES.get(s.scene, 0), boundary=1 if st.get("boundary") else 0,
                          gravity=GRAVITY[st.get("gravity", "none")], stiffness=float(st.get("solidStiffness", 1)),
                          strength=float(st.get("strength", 1)), x=s.x.ctypes.data, y=s.y.ctypes.data,
                          vx=s.vx.ctypes.data, vy=s.vy.ctypes.data, mass=s.mass.ctypes.data,
                          volume=s.volume.ctypes.data, material=s.material.ctypes.data,
                          pinned=s.pinned.ctypes.data, mpm_material=self.flags.ctypes.data)

    def stable_step(self, s):
        sim = self._sim(s)
        return _lib().oracle2_stable_step(ctypes.byref(self.st), ctypes.byref(sim))

    def step(self, s, dt, want_grid=False):
        sim = self._sim(s)
        grid = np.zeros((149 * 149, 3)) if want_grid else None
        _lib().oracle2_step(ctypes.byref(self.st), ctypes.byref(sim), dt, None if grid is None else grid.ctypes.data)
        return grid

    def frame(self, s, dt=1 / 60):
        sim = self._sim(s)
        adv = _D()
        n = _lib().oracle2_frame(ctypes.byref(self.st), ctypes.byref(sim), dt, ctypes.byref(adv))
        return n, adv.value

    def stats(self, s):
        sim = self._sim(s)
        out = Oracle2Stats()
        _lib().oracle2_stats(ctypes.byref(self.st), ctypes.byref(sim), ctypes.byref(out))
        return dict(count=out.count, minJ=out.min_j, maxJ=out.max_j, strain=out.strain, nodes=out.nodes,
                    substeps=out.substeps)
