"""The C-ABI library loads and exports every symbol include/mpm_b200.h declares (CPU only)."""
import ctypes
import os
import re

import pytest

from mpm_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "mpm_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\**\s+\**(s?mpm_\w+)\s*\(", text, flags=re.M)))


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    names = declared_functions()
    assert len(names) >= 25
    for name in names:
        assert hasattr(L, name), name
        assert name in _lib.SIGNATURES, f"{name} has no ctypes signature"


def test_abi_version_and_error_strings_need_no_gpu():
    L = _lib.lib()
    assert L.mpm_abi_version() == 3
    assert L.mpm_error_string(-4) == b"non-finite particle state"
    assert L.mpm_error_string(0) == b"ok"


def test_struct_layouts_match_header_sizes():
    # sizes follow from the header's field lists (all 8-byte aligned)
    assert ctypes.sizeof(_lib.MpmDomain) == 8 * 3 * 2 + 8 + 24 + 4 + 4 + 8 * 4 + 8
    assert ctypes.sizeof(_lib.MpmMaterial) == 8 + 34 * 8
    assert ctypes.sizeof(_lib.MpmParticles) == 8 + 18 * 8
    assert ctypes.sizeof(_lib.MpmLedger) == 5 * 8 + 6 * 8 + 5 * 8 + 3 * 8
    assert ctypes.sizeof(_lib.SmpmSim) == 4 * 4 + 2 * 8 + 8 * 8
    assert ctypes.sizeof(_lib.SmpmStats) == 4 * 4 + 3 * 8


def test_invalid_arguments_are_rejected_without_touching_a_device():
    L = _lib.lib()
    h = ctypes.c_void_p()
    assert L.mpm_create(None, 10, ctypes.byref(h)) == -1
    assert L.mpm_destroy(None) == -1
    assert L.smpm_create(0, ctypes.byref(h)) == -1
    assert L.smpm_destroy(None) == -1
    m = _lib.MpmMaterial(model=12, mu=1, lam=1)
    assert L.mpm_return_map_batch(ctypes.byref(m), 0, None, None, None, 0.0, None, None, None) == -10
    m = _lib.MpmMaterial(model=2, mu=1, lam=1, yield_strain=.025)  # carries Jp between steps
    assert L.mpm_return_map_batch(ctypes.byref(m), 0, None, None, None, 0.0, None, None, None) == -10
    t = ctypes.c_int32()
    assert L.mpm_check_bounded_wait(None, 1 << 20, ctypes.byref(t)) == -1
