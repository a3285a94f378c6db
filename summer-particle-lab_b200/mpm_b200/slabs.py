"""One scene split into slabs along z: on one handle (a batch of slab scenes) or one slab per rank.

Neighbouring slabs hold the same `planes` node planes of the global grid. After every scatter both
copies of a shared node receive the sum of both slabs' contributions (mpm_batch_set_slabs does it on
the device for a batch; ranks export their planes, exchange them and add what they receive), so
both grid updates give the same velocity there and a particle near the seam needs no copy. Every
slab takes the same dt. Particles are assigned to the slab whose own node range holds them and must
stay at least 3 node planes inside their slab's grid; re-partition (download, partition, upload)
before they get closer.
"""
import ctypes
import dataclasses

import numpy as np

from . import _lib
from .params import Domain
from .scenes import Scene

FACE_Z_LOW, FACE_Z_HIGH = 1 << 4, 1 << 5


@dataclasses.dataclass
class Slab:
    domain: Domain   # grid of the slab (own nodes plus the shared planes)
    own: tuple       # [z0, z1) own node range in the global grid
    nodes: tuple     # [g0, g1) global z nodes of the slab's grid


def slab_domains(domain, nslabs, planes):
    """Slab grids aligned with the global grid: slab k's grid starts `planes` nodes before slab
    k-1's grid ends. The seams sit in the middle of the shared planes."""
    if domain.cubic:
        raise ValueError("slabs need a non-cubic domain")
    if planes < 4 or planes % 2:
        raise ValueError("planes must be even and at least 4")
    H = domain.H
    nz = domain.dims[2]
    oz = domain.origin[2]
    cuts = [round(nz * k / nslabs) for k in range(nslabs + 1)]
    out = []
    for k in range(nslabs):
        z0, z1 = cuts[k], cuts[k + 1]
        g0 = 0 if k == 0 else z0 - planes // 2
        g1 = nz if k == nslabs - 1 else z1 + planes // 2
        if g1 - g0 < 2 * planes:
            raise ValueError("slabs too thin for the shared planes")
        lower = list(domain.lower)
        upper = list(domain.upper)
        # build_scene: origin = floor(lower / H) H - 2H, nodes = ceil((upper - origin) / H) + 3
        if k > 0:
            lower[2] = oz + (g0 + 2) * H
        if k < nslabs - 1:
            upper[2] = oz + (g1 - 3) * H
        d = Domain(lower=tuple(lower), upper=tuple(upper), H=H, gravity=domain.gravity,
                   sticky_floor=domain.sticky_floor, clamp_positions=domain.clamp_positions, mass_eps=domain.mass_eps,
                   cfl=domain.cfl, dt_max=domain.dt_max, grad_limit=domain.grad_limit)
        if abs(d.origin[2] - (oz + g0 * H)) > 1e-9 * H or d.dims[2] != g1 - g0:
            raise ValueError("slab grid does not align with the global grid")
        out.append(Slab(domain=d, own=(z0, z1), nodes=(g0, g1)))
    return out


def partition(scene, slabs):
    """Per-slab scenes: each particle goes to the slab whose own node range holds its z."""
    d = scene.domain
    zq = (np.asarray(scene.x)[:, 2] - d.origin[2]) / d.H
    parts = []
    for k, s in enumerate(slabs):
        lo = -np.inf if k == 0 else s.own[0]
        hi = np.inf if k == len(slabs) - 1 else s.own[1]
        sel = (zq >= lo) & (zq < hi)

        def take(a):
            return None if a is None else np.asarray(a)[sel]
        parts.append((Scene(name=f"{scene.name}_slab{k}", domain=s.domain, materials=scene.materials,
                            x=take(scene.x), v=take(scene.v), m=take(scene.m), V=take(scene.V), mat=take(scene.mat),
                            T=take(scene.T), F=take(scene.F), C=take(scene.C), ep=take(scene.ep),
                            pinned=take(scene.pinned), jp=take(scene.jp), dilation=take(scene.dilation),
                            enthalpy=take(scene.enthalpy), melted=take(scene.melted), meta=dict(scene.meta)),
                      np.nonzero(sel)[0]))
    return parts


def slab_batch(scene, nslabs, planes):
    """A Batch handle of the scene's slabs with the on-device overlap sum; returns (batch, index
    arrays mapping each slab's particles to the scene's)."""
    from .solver import Batch
    slabs = slab_domains(scene.domain, nslabs, planes)
    parts = partition(scene, slabs)
    b = Batch([p for p, _ in parts])
    b.upload()
    b._check(_lib.lib().mpm_batch_set_slabs(b.h, int(planes)))
    return b, [idx for _, idx in parts]


def halo_exchange(rank, world, export, add, swap):
    """The overlap sum of one rank with its neighbours along the slab chain: export both seams
    (side 0 low z, side 1 high z) first, so each neighbour receives this rank's own contribution,
    then swap buffers with each neighbour in turn (side 0 first: the chain resolves from rank 0),
    then add what was received. `swap(side, peer)` must send and receive without deadlocking, e.g.
    with batched non-blocking point-to-point operations."""
    sides = [s for s, peer in ((0, rank - 1), (1, rank + 1)) if 0 <= peer < world]
    for s in sides:
        export(s)
    for s in sides:
        swap(s, rank - 1 if s == 0 else rank + 1)
    for s in sides:
        add(s)
    return sides


class SlabRank:
    """One slab on one rank (a single-scene handle with the seam faces open). `transport(send, recv,
    peer)` moves one buffer to and from a neighbour rank (NCCL point-to-point between GPUs); `alloc(n)`
    returns a 16-byte-aligned device buffer of n bytes with a `.ptr` address. Each substep: the
    smallest stable dt over ranks (`reduce_min`), one fixed substep, then the overlap exchange."""

    def __init__(self, scene, slab, rank, world, planes, transport, reduce_min, alloc, start=True):
        from .solver import Solver
        self.rank, self.world, self.planes = rank, world, planes
        self.transport, self.reduce_min = transport, reduce_min
        self.solver = Solver(slab.domain, max(scene.n, 1))
        self.solver.upload(scene)
        faces = (FACE_Z_LOW if rank > 0 else 0) | (FACE_Z_HIGH if rank < world - 1 else 0)
        self._check(_lib.lib().mpm_set_open_faces(self.solver.h, faces))
        nb = ctypes.c_int64()
        self._check(_lib.lib().mpm_halo_bytes(self.solver.h, planes, ctypes.byref(nb)))
        self.nbytes = nb.value
        self.send = {s: alloc(self.nbytes) for s in (0, 1)}
        self.recv = {s: alloc(self.nbytes) for s in (0, 1)}
        self._check(_lib.lib().mpm_prepare(self.solver.h))
        if start:
            self.exchange()

    def _check(self, rc):
        return _lib.check(rc, self.solver.h)

    def export(self, side):
        self._check(_lib.lib().mpm_halo_export(self.solver.h, side, self.planes, ctypes.c_void_p(self.send[side].ptr)))

    def add(self, side):
        self._check(_lib.lib().mpm_halo_add(self.solver.h, side, self.planes, ctypes.c_void_p(self.recv[side].ptr)))

    def exchange(self):
        halo_exchange(self.rank, self.world, self.export, self.add,
                      lambda s, peer: self.transport(self.send[s], self.recv[s], peer))

    def step(self, nsteps=1):
        for _ in range(nsteps):
            dt = self.reduce_min(self.solver.stable_dt())
            self.solver.step_fixed(dt, 1)
            self.exchange()

    def advance(self, duration):
        """Substeps until `duration` seconds have passed, each at the smallest stable dt over ranks
        (cut to the time left), so every rank takes the same substeps; returns their number."""
        t, n = 0.0, 0
        while duration - t > 1e-9 * duration:
            dt = self.reduce_min(min(self.solver.stable_dt(), duration - t))
            self.solver.step_fixed(dt, 1)
            self.exchange()
            t += dt
            n += 1
        return n

    def close(self):
        self.solver.close()
