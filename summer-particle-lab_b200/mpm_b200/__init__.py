"""mpm_b200: B200-native explicit MLS-MPM solid step behind the reference's step/state API.

The compute path is libmpm_b200.so (hand-written sm_100a CUDA behind a C ABI, include/mpm_b200.h).
This package is its host side: ctypes binding (_lib), a one-scene handle (solver), seeded scenes
(scenes), parameters (params) and the MPM3 facade of src/three/mpm.js (mpm3).
"""
from .params import Domain, Material
from .solver import Solver, return_map_batch

__all__ = ["Domain", "Material", "Solver", "return_map_batch"]
