"""The allocation-free P2G entry point against the oracle and the handle path (GPU, through the C ABI).

mpm_p2g_noalloc serves callers that cannot allocate device memory themselves (a host that owns all
device memory through its own pool, or code running where cudaMalloc is not allowed): the caller
passes device inputs and outputs and the library's only intermediate is a fixed device array. This
test allocates the caller's buffers with torch, calls the entry point twice in a row, and checks
both results against the FP64 oracle's grid after P2G of the same state and against mpm_grid_debug
of a handle holding it, within the grid tolerance of the other parity tests (1e-6 normwise
relative). It sits in a file of its own, collected last.
"""
import ctypes

import numpy as np
import pytest

from mpm_b200 import _lib, scenes
from oracle import oracle as orc
from mpm_b200.solver import Solver, domain_struct, material_struct

pytestmark = pytest.mark.gpu


def rel(a, b):
    scale = float(np.max(np.abs(b)))
    return float(np.max(np.abs(a - b)) / (scale if scale > 0 else 1.0))


def deformed_j2_block():
    d = scenes.Domain(lower=(0, 0, 0), upper=(1, 1, 1), H=1 / 32, gravity=(0, -9.8, 0), sticky_floor=True)
    x = scenes.block_particles(d, (8, 2, 8), (20, 10, 20), seed=21)
    sc = scenes._scene("noalloc_j2", d, [scenes.aluminium_j2()], x, (0.5, -3.0, 0.25))
    rng = np.random.default_rng(5)
    sc.F = (np.tile(np.eye(3).ravel(), (sc.n, 1)) + 2e-3 * rng.standard_normal((sc.n, 9)))
    sc.C = 50.0 * rng.standard_normal((sc.n, 9))
    return sc


def test_noalloc_p2g_matches_oracle_and_handle_path_twice():
    import torch
    sc = deformed_j2_block()
    dt = 1e-6
    sol = Solver(sc.domain, sc.n)
    sol.upload(sc)
    gm_dev, gp_dev = sol.grid_debug(dt)
    gm_ref, gp_ref, _ = orc.state_from_scene(sc).step(dt, want_grid=True)
    dims, _ = sol.grid_dims()
    nodes = int(np.prod(dims))
    dev = torch.device("cuda", 0)
    x = torch.tensor(sc.x, dtype=torch.float64, device=dev)
    v = torch.tensor(sc.v, dtype=torch.float32, device=dev)
    F = torch.tensor(sc.F, dtype=torch.float64, device=dev)
    C = torch.tensor(sc.C, dtype=torch.float32, device=dev)
    m = torch.tensor(sc.m, dtype=torch.float32, device=dev)
    V = torch.tensor(sc.V, dtype=torch.float32, device=dev)
    mass = torch.empty(nodes, dtype=torch.float64, device=dev)
    mom = torch.empty(nodes * 3, dtype=torch.float64, device=dev)
    P = ctypes.c_void_p
    dom = domain_struct(sc.domain)
    mat = material_struct(sc.materials[0])
    for call in range(2):
        mass.fill_(-1.0)
        mom.fill_(-1.0)
        torch.cuda.synchronize()
        rc = _lib.lib().mpm_p2g_noalloc(ctypes.byref(dom), ctypes.byref(mat), sc.n, P(x.data_ptr()), P(v.data_ptr()),
                                       P(F.data_ptr()), P(C.data_ptr()), P(m.data_ptr()), P(V.data_ptr()), dt,
                                       P(mass.data_ptr()), P(mom.data_ptr()), None)
        assert rc == 0, _lib.lib().mpm_error_string(rc)
        torch.cuda.synchronize()
        gm = mass.cpu().numpy()
        gp = mom.cpu().numpy().reshape(-1, 3)
        assert rel(gm, gm_ref) <= 1e-6, call
        assert rel(gp, gp_ref) <= 1e-6, call
        assert rel(gm, gm_dev) <= 1e-6, call
        assert rel(gp, gp_dev) <= 1e-6, call
    sol.close()


def test_noalloc_rejects_grids_beyond_the_scratch_size():
    d = scenes.Domain(lower=(0, 0, 0), upper=(1, 1, 1), H=1 / 96)
    dom = domain_struct(d)
    mat = material_struct(scenes.aluminium_j2())
    out = ctypes.c_void_p(1)
    rc = _lib.lib().mpm_p2g_noalloc(ctypes.byref(dom), ctypes.byref(mat), 0, None, None, None, None, None, None, 1e-6,
                                   out, out, None)
    assert rc == -9  # MPM_ERR_CAPACITY: 101^3 nodes exceed 262,144
