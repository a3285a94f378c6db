"""Viewer frames (gpu/solver.py:985-1035, gpu/server.py:17-20, src/three/gpu-worker.js:36-42)."""
import ctypes
import math

import numpy as np
import pytest

from mpm_b200 import _lib, scenes
from mpm_b200.frame import packet, parse_packet


def preview_pick(row, span):
    """The reference's row hash (gpu/solver.py:995-999) in 32-bit unsigned arithmetic."""
    m = 0xFFFFFFFF
    h = (row * 747796405 + 2891336453) & m
    h = (((h >> ((h >> 28) + 4)) ^ h) * 277803737) & m
    h = (h >> 22) ^ h
    return h % span


def chosen_ids(n, stride):
    rows = math.ceil(n / stride)
    return np.array([r * stride + preview_pick(r, min(stride, n - r * stride)) for r in range(rows)])


def test_preview_hash_picks_one_index_per_block():
    for n, stride in ((10, 1), (1000, 7), (12345, 100), (100_001, 2)):
        ids = chosen_ids(n, stride)
        assert len(ids) == math.ceil(n / stride)
        assert np.all(ids // stride == np.arange(len(ids))) and np.all(ids < n)


def test_packet_roundtrip_and_worker_checks():
    data = np.arange(24, dtype=np.float32).reshape(3, 8)
    meta = dict(count=5, capacity=10, renderCount=3, sampleStride=2, mass=1.5)
    buf = packet(meta, data)
    header = b'{"count":5,"capacity":10,"renderCount":3,"sampleStride":2,"mass":1.5}'
    assert len(buf) == 4 + math.ceil(len(header) / 4) * 4 + data.nbytes
    st = parse_packet(buf)
    assert st["count"] == 5 and np.array_equal(st["data"], data)
    with pytest.raises(ValueError):
        parse_packet(buf[:-4])  # a row cut short
    with pytest.raises(ValueError):
        parse_packet(packet(dict(count=5, capacity=4, renderCount=3), data))  # count above capacity
    with pytest.raises(ValueError):
        packet(dict(count=1, x=float("nan")), data)  # allow_nan=False, like the service


def test_frame_info_layout():
    assert ctypes.sizeof(_lib.MpmFrameInfo) == 3 * 8 + 7 * 8 + 8 + 256 * 8


@pytest.mark.gpu
def test_pack_frame_samples_and_reductions():
    from mpm_b200.frame import snapshot
    from mpm_b200.solver import Solver
    sc = scenes.thermal_j2(grid=32, block=10, v0=-60.0)
    s = Solver(sc.domain, sc.n)
    s.upload(sc)
    s.step_fixed(1e-6, 3)
    out = s.download()
    meta, data = snapshot(s, preview_limit=997, materials={0: sc.materials[0]})
    stride = math.ceil(sc.n / 997)
    ids = chosen_ids(sc.n, stride)
    assert meta["renderCount"] == len(ids) == data.shape[0] and meta["sampleStride"] == stride
    np.testing.assert_allclose(data[:, 0:3], out["x"][ids], rtol=0, atol=1e-6)
    np.testing.assert_allclose(data[:, 4], out["T"][ids], rtol=1e-6)
    np.testing.assert_allclose(data[:, 7], out["ep"][ids], rtol=0, atol=1e-7)
    assert np.all(data[:, 3] == 0) and np.all(data[:, 6] >= 0)
    assert abs(meta["mass"] - sc.m.sum()) <= 1e-6 * sc.m.sum()
    cp = sc.materials[0].specific_heat
    assert abs(meta["energy"] - np.sum(sc.m * cp * out["T"])) <= 1e-5 * np.sum(sc.m * cp * out["T"])
    assert abs(meta["min"] - out["T"].min()) <= 1e-3 and abs(meta["max"] - out["T"].max()) <= 1e-3
    assert meta["models"][10] == sc.n
    st = parse_packet(packet(meta, data))
    assert np.array_equal(st["data"], data)
    s.close()


@pytest.mark.gpu
def test_pack_frame_reports_nonfinite_state():
    from mpm_b200.frame import snapshot
    from mpm_b200.solver import Solver
    sc = scenes.elastic_cube()
    sc.v[5] = np.nan
    s = Solver(sc.domain, sc.n)
    s.upload(sc)
    with pytest.raises(_lib.MpmError):
        snapshot(s)
    s.close()
