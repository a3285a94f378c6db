"""Viewer frames: the Taichi service's `snapshot` + `packet` (gpu/solver.py:985-1035,
gpu/server.py:17-20) on the B200 library, so the browser's GPU worker (src/three/gpu-worker.js:30-42)
can read frames of this engine unchanged.

A frame is one little-endian u32 header length, the JSON metadata padded with spaces to 4 bytes,
then renderCount rows of 8 float32 (x, y, z, material, temperature, pinned, stress, plastic).
"""
import ctypes
import json
import math
import struct

import numpy as np

from . import _lib

PREVIEW_LIMIT = 100_000  # gpu/solver.py:17
MODEL_COUNT = 12          # gpu/metal_plasticity.py:11


def snapshot(solver, preview_limit=PREVIEW_LIMIT, materials=None, time=0.0, substeps=0):
    """(metadata, data) of the handle's current state. `materials` maps material index -> Material
    (for the per-model counts); by default the solver's scene materials."""
    n = solver.n
    stride = max(1, math.ceil(n / preview_limit)) if n else 1
    rows = math.ceil(n / stride) if n else 0
    data = np.empty((max(rows, 1), 8), np.float32)
    info = _lib.MpmFrameInfo()
    _lib.check(_lib.lib().mpm_pack_frame(solver.h, preview_limit, data.ctypes.data, data.shape[0], ctypes.byref(info)),
               solver.h)
    models = [0] * MODEL_COUNT
    for k in range(256):
        if info.per_material[k]:
            model = materials[k].model if materials and k in materials else 0
            if model < MODEL_COUNT:
                models[model] += info.per_material[k]
    meta = dict(count=info.count, capacity=solver.capacity, renderCount=info.rows, sampleStride=info.stride,
                models=models, time=time, mass=info.mass, energy=info.thermal_energy, solids=info.count, liquids=0,
                min=info.min_T if n else 0.0, max=info.max_T if n else 0.0, substeps=substeps, minJ=info.min_j,
                maxStress=info.max_von_mises, maxPlastic=info.max_plastic)
    return meta, data[:rows]


def packet(metadata, data):
    """gpu/server.py:17-20: u32 header length, JSON header padded to 4 bytes, float32 rows."""
    header = json.dumps(metadata, separators=(",", ":"), ensure_ascii=False, allow_nan=False).encode("utf-8")
    padding = (-len(header)) % 4
    return struct.pack("<I", len(header)) + header + b" " * padding + np.asarray(data, "<f4").tobytes()


def parse_packet(buf):
    """The worker's decoding and validity checks (src/three/gpu-worker.js:36-42)."""
    (length,) = struct.unpack_from("<I", buf, 0)
    offset = 4 + math.ceil(length / 4) * 4
    if length > len(buf) - 4:
        raise ValueError("invalid frame header")
    state = json.loads(buf[4:4 + length].decode("utf-8"))
    rendered = state.get("renderCount", state["count"])
    ok = (isinstance(state["count"], int) and isinstance(rendered, int) and 0 <= rendered <= state["count"]
          and 0 <= state["count"] <= state["capacity"] and offset + rendered * 32 == len(buf))
    if not ok:
        raise ValueError("invalid particle frame")
    state["data"] = np.frombuffer(buf, "<f4", rendered * 8, offset).reshape(rendered, 8)
    return state
