"""SlabSim -- one scene split along z into slabs, one handle per slab, on one
or several GPUs (lbm_set_slab, lbm_slab_copy_planes).

The reference holds a scene in one set of typed arrays (src/sim.js:30-96).  A
scene too large for one GPU's memory (beyond ~500 M cells at 338 B per cell)
is cut into z slabs: slab s owns the scene's planes g0 .. g1 and keeps two
copied planes of each neighbour (one of the scene's wall planes at the ends).
Every step each slab steps on its own GPU; afterwards the two planes next to
each cut cross it in both directions (device to device, over NVLink between
GPUs).  The sphere keeps the scene's coordinates; each slab counts the
momentum exchange and dead-cell impulses of its own planes only, and the
slabs' impulses are added in slab order, so the solid sees the scene's total.

    scene = SlabSim(256, 256, 512, nslabs=2, devices=[0, 1])
    scene.initFlat(96); scene.tau = 0.6; ...
    solid = RigidSphere(256, 256, 512, cx=128, cy=200, cz=256, r=24, density=2)
    scene.step(solid); solid.absorbDeadCells(scene); solid.step(1.0, scene.gravity)
    phi = scene.field("phi")           # the scene's array, reference layout

Given the same sphere state every cell update is the one a single handle
makes (the fused step's arithmetic does not depend on the tiling, and fresh
cells are filled in the scene's scan order across the cuts, see step); only
the order in which the slabs' impulse sums are added differs from the single
handle's fixed-order reduction.
"""
from __future__ import annotations

import numpy as np

from . import _capi
from ._capi import check, lib
from .sim import Sim

_PARAMS = ("tau", "tauPhi", "sigma", "gravity", "rhoL", "rhoG", "W", "mobility")
HALO = 2  # copied planes on each side of a cut


def slab_plan(nz, nslabs):
    """Cut the interior planes 1 .. nz-2 into nslabs contiguous ranges.
    Returns per slab (g0, g1, lo_halo, hi_halo, zoff, local_nz, own_lo,
    own_hi): owned scene planes g0..g1, copied planes below / above, the
    local frame's offset, size and owned local range."""
    interior = nz - 2
    if nslabs < 1 or interior < HALO * nslabs:
        raise ValueError("every slab needs at least two planes of its own")
    cuts = [1 + interior * s // nslabs for s in range(nslabs + 1)]
    out = []
    for s in range(nslabs):
        g0, g1 = cuts[s], cuts[s + 1] - 1
        lo = 1 if s == 0 else HALO            # the scene's wall plane 0, or two copied planes
        hi = 1 if s == nslabs - 1 else HALO
        nzl = (g1 - g0 + 1) + lo + hi
        out.append((g0, g1, lo, hi, g0 - lo, nzl, lo, lo + g1 - g0))
    return out


def exchange_plan(plan):
    """The plane copies after a step, as (dst slab, dst local plane, src slab,
    src local plane, planes): across each cut, the two owned planes next to it
    go to the neighbour's copied planes, both ways."""
    ops = []
    for s in range(len(plan) - 1):
        lower, upper = plan[s], plan[s + 1]
        ops.append((s + 1, 0, s, lower[7] - (HALO - 1), HALO))    # up: lower's top owned planes
        ops.append((s, lower[7] + 1, s + 1, upper[6], HALO))       # down: upper's bottom owned planes
    return ops


class SlabSim:
    def __init__(self, nx, ny, nz, nslabs=2, storage="f32", devices=None):
        if (nx * ny) % 8:
            raise ValueError("slabs need nx * ny divisible by 8")
        self.nx, self.ny, self.nz = nx, ny, nz
        self.n = nx * ny * nz
        self.storage = storage
        self.plan = slab_plan(nz, nslabs)
        self.slabs = []
        devices = list(devices) if devices else [0]
        for s, (g0, g1, lo, hi, zoff, nzl, own_lo, own_hi) in enumerate(self.plan):
            sim = Sim(nx, ny, nzl, storage=storage, device=devices[s % len(devices)])
            check(sim.handle, lib().lbm_set_slab(sim.handle, zoff, own_lo, own_hi))
            self.slabs.append(sim)
        self._ops = exchange_plan(self.plan)
        self._up = self._ops[0::2]    # per cut: the lower slab's top owned planes go up
        self._down = self._ops[1::2]  # per cut: the upper slab's bottom owned planes go down

    # ------------------------------------------------------------ parameters
    def __getattr__(self, name):
        if name in _PARAMS:
            return getattr(self.__dict__["slabs"][0], name)
        raise AttributeError(name)

    def __setattr__(self, name, value):
        if name in _PARAMS:
            for sim in self.slabs:
                setattr(sim, name, value)
        else:
            object.__setattr__(self, name, value)

    def close(self):
        for sim in self.slabs:
            sim.close()

    # ------------------------------------------------------------ fields
    def _local_planes(self, s):
        """(local plane, scene plane) of every plane slab s holds."""
        zoff, nzl = self.plan[s][4], self.plan[s][5]
        return [(k, k + zoff) for k in range(nzl)]

    def field(self, name):
        """The scene's field in the reference layout, assembled from the owned
        planes of every slab (and the scene's wall planes from the end slabs)."""
        per = {"f": 27, "f2": 27, "h": 7, "h2": 7}.get(name, 1)
        plane = self.nx * self.ny * per
        dtype = np.uint8 if name in ("tag", "tagPrev") else np.float32
        out = np.empty(self.nz * plane, dtype=dtype)
        for s, sim in enumerate(self.slabs):
            g0, g1, lo, hi, zoff, nzl, own_lo, own_hi = self.plan[s]
            a = np.asarray(getattr(sim, name))
            k0 = 0 if s == 0 else own_lo
            k1 = nzl - 1 if s == len(self.slabs) - 1 else own_hi
            out[(k0 + zoff) * plane:(k1 + zoff + 1) * plane] = a[k0 * plane:(k1 + 1) * plane]
        return out

    def set_field(self, name, values):
        """Write a scene-wide field (reference layout) into every slab,
        copied planes included."""
        per = {"f": 27, "f2": 27, "h": 7, "h2": 7}.get(name, 1)
        plane = self.nx * self.ny * per
        values = np.asarray(values)
        for s, sim in enumerate(self.slabs):
            zoff, nzl = self.plan[s][4], self.plan[s][5]
            getattr(sim, name)[:] = values[zoff * plane:(zoff + nzl) * plane]

    # ------------------------------------------------------------ the reference's calls
    def idx(self, x, y, z):
        return ((z * self.ny) + y) * self.nx + x

    def initFlat(self, waterlineY):
        for sim in self.slabs:
            sim.initFlat(waterlineY)

    def seedHydrostatic(self):
        for sim in self.slabs:
            sim.seedHydrostatic()

    def step(self, solid):
        """Sim.step (src/sim.js:202-210) on every slab; the solid collects
        every slab's momentum exchange.  handleFreshCells fills a fresh cell
        from neighbours of which those earlier in the scene's scan order are
        already filled (src/sim.js:257-300), so the slabs begin their steps
        (retag + fill of their own planes) in z order, each handing its two
        top owned planes, filled, to the next slab's copied planes; then each
        slab's two bottom owned planes, filled, go down to the slab below,
        every slab ends its step, and the plane exchange follows."""
        for s, sim in enumerate(self.slabs):
            sim.step_begin(solid)
            if s < len(self._up):
                self._copy(*self._up[s])
        for op in self._down:
            self._copy(*op)
        for sim in self.slabs:
            sim.step_end(solid)
        self.exchange()

    def _absorb_dead(self, spheres):
        # RigidSphere.absorbDeadCells(sim) calls this: every slab's own dead cells
        for sim in self.slabs:
            sim._absorb_dead(spheres)

    def _copy(self, dst, dplane, src, splane, k):
        d, s = self.slabs[dst], self.slabs[src]
        rc = lib().lbm_slab_copy_planes(d.handle, dplane, s.handle, splane, k)
        if rc != _capi.OK:
            raise _capi.LbmError(rc, (lib().lbm_last_error(d.handle) or b"").decode(errors="replace"))
        d._moved()

    def exchange(self):
        for op in self._ops:
            self._copy(*op)
