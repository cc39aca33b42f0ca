"""RigidSphere and the composite solid -- the host side of the reference's
solid interface (src/solid.js:8-211).

The per-cell and per-link work (contains / surfaceVelocity during retagging,
applyImpulseAtCell during streaming, the dead-cell sweep) runs on the GPU; this
class keeps the rigid-body state and its FP64 integrator exactly as the
reference writes them, and accumulates the momentum exchange the device
returns into Fx..Tz just as applyImpulseAtCell would.
"""
from __future__ import annotations

import math

from ._capi import LbmImpulse, LbmSphere, MAX_SPHERES


def _js_max0(v):
    # Math.max(0, v): NaN propagates, +0 wins over -0
    if v != v:
        return v
    if v == 0:
        return 0.0
    return v if v > 0 else 0.0


def _js_min0(v):
    if v != v:
        return v
    if v == 0:
        return v if math.copysign(1.0, v) < 0 else 0.0
    return v if v < 0 else 0.0


class RigidSphere:
    """class RigidSphere (src/solid.js:8-211)."""

    def __init__(self, nx, ny, nz, opts=None, **kw):
        opts = dict(opts or {}, **kw)
        self.nx, self.ny, self.nz = nx, ny, nz
        self.cx = opts.get("cx", nx * 0.5)
        self.cy = opts.get("cy", ny * 0.3)
        self.cz = opts.get("cz", nz * 0.5)
        self.r = opts.get("r", min(nx, ny, nz) * 0.10)
        self.vx = self.vy = self.vz = 0.0
        self.wx = self.wy = self.wz = 0.0
        self.density = opts.get("density", 1.4)
        self.dragging = False
        self.dragTargetX = self.dragTargetY = self.dragTargetZ = 0.0
        self.Fx = self.Fy = self.Fz = 0.0
        self.Tx = self.Ty = self.Tz = 0.0
        self.recomputeMass()

    # src/solid.js:39-47
    def recomputeMass(self):
        V = (4 / 3) * math.pi * self.r * self.r * self.r
        self.volume = V
        self.mass = self.density * V
        self.I = (2 / 5) * self.mass * self.r * self.r

    def setRadius(self, r):
        self.r = r
        self.recomputeMass()

    def setDensity(self, d):
        self.density = d
        self.recomputeMass()

    # src/solid.js:50-66 (host-side; the device evaluates the same FP64 test)
    def contains(self, x, y, z):
        dx = x + 0.5 - self.cx
        dy = y + 0.5 - self.cy
        dz = z + 0.5 - self.cz
        return dx * dx + dy * dy + dz * dz <= self.r * self.r

    def surfaceVelocity(self, x, y, z, out=None):
        rx = x + 0.5 - self.cx
        ry = y + 0.5 - self.cy
        rz = z + 0.5 - self.cz
        out = out if out is not None else [0.0, 0.0, 0.0]
        out[0] = self.vx + (self.wy * rz - self.wz * ry)
        out[1] = self.vy + (self.wz * rx - self.wx * rz)
        out[2] = self.vz + (self.wx * ry - self.wy * rx)
        return out

    # src/solid.js:70-80
    def applyImpulseAtCell(self, x, y, z, px, py, pz):
        self.Fx += px
        self.Fy += py
        self.Fz += pz
        rx = x + 0.5 - self.cx
        ry = y + 0.5 - self.cy
        rz = z + 0.5 - self.cz
        self.Tx += ry * pz - rz * py
        self.Ty += rz * px - rx * pz
        self.Tz += rx * py - ry * px

    def add_impulse(self, imp):
        """Add a device-summed momentum exchange (an LbmImpulse)."""
        self.Fx += imp.Fx
        self.Fy += imp.Fy
        self.Fz += imp.Fz
        self.Tx += imp.Tx
        self.Ty += imp.Ty
        self.Tz += imp.Tz

    # src/solid.js:87-101: the dead-cell sweep runs on the device
    def absorbDeadCells(self, sim):
        sim._absorb_dead([self])

    # src/solid.js:104-210
    def step(self, dt, gravity):
        bodyG = gravity
        self.Fy += self.mass * bodyG
        if self.dragging:
            k = 0.004 * self.mass
            cD = 2.0 * math.sqrt(k * self.mass)
            self.Fx += k * (self.dragTargetX - self.cx) - cD * self.vx
            self.Fy += k * (self.dragTargetY - self.cy) - cD * self.vy
            self.Fz += k * (self.dragTargetZ - self.cz) - cD * self.vz
        g = gravity if (gravity == gravity and gravity != 0) else 0.001  # `gravity || 0.001`
        accCap = 3.5 * abs(g)
        ax = self.Fx / self.mass
        ay = self.Fy / self.mass
        az = self.Fz / self.mass
        a2 = ax * ax + ay * ay + az * az
        c2 = accCap * accCap
        s = accCap / math.sqrt(a2) if a2 > c2 else 1.0
        self.vx += dt * ax * s
        self.vy += dt * ay * s
        self.vz += dt * az * s
        self.wx += dt * self.Tx / self.I
        self.wy += dt * self.Ty / self.I
        self.wz += dt * self.Tz / self.I
        BODY_UMAX = 0.08
        sp2 = self.vx * self.vx + self.vy * self.vy + self.vz * self.vz
        if sp2 > BODY_UMAX * BODY_UMAX:
            s = BODY_UMAX / math.sqrt(sp2)
            self.vx *= s
            self.vy *= s
            self.vz *= s
        self.vx *= 0.98
        self.vy *= 0.98
        self.vz *= 0.98
        self.wx *= 0.95
        self.wy *= 0.95
        self.wz *= 0.95
        SNAP = 0.0001
        if abs(self.vx) < SNAP:
            self.vx = 0
        if abs(self.vy) < SNAP:
            self.vy = 0
        if abs(self.vz) < SNAP:
            self.vz = 0
        if abs(self.wx) < SNAP:
            self.wx = 0
        if abs(self.wy) < SNAP:
            self.wy = 0
        if abs(self.wz) < SNAP:
            self.wz = 0
        self.cx += dt * self.vx
        self.cy += dt * self.vy
        self.cz += dt * self.vz
        m = self.r + 1.5
        if self.cx < m:
            self.cx = m
            self.vx = _js_max0(self.vx)
        if self.cx > self.nx - 1 - m:
            self.cx = self.nx - 1 - m
            self.vx = _js_min0(self.vx)
        if self.cy < m:
            self.cy = m
            self.vy = _js_max0(self.vy)
        if self.cy > self.ny - 1 - m:
            self.cy = self.ny - 1 - m
            self.vy = _js_min0(self.vy)
        if self.cz < m:
            self.cz = m
            self.vz = _js_max0(self.vz)
        if self.cz > self.nz - 1 - m:
            self.cz = self.nz - 1 - m
            self.vz = _js_min0(self.vz)
        self.Fx = self.Fy = self.Fz = 0
        self.Tx = self.Ty = self.Tz = 0

    # ---------------------------------------------------------------- C ABI view
    def to_c(self, out: LbmSphere | None = None) -> LbmSphere:
        s = out if out is not None else LbmSphere()
        for k in ("cx", "cy", "cz", "r", "vx", "vy", "vz", "wx", "wy", "wz", "density", "mass",
                  "I", "dragTargetX", "dragTargetY", "dragTargetZ", "Fx", "Fy", "Fz", "Tx", "Ty",
                  "Tz"):
            setattr(s, k, float(getattr(self, k)))
        s.dragging = 1 if self.dragging else 0
        return s

    def from_c(self, s: LbmSphere):
        for k in ("cx", "cy", "cz", "r", "vx", "vy", "vz", "wx", "wy", "wz", "Fx", "Fy", "Fz",
                  "Tx", "Ty", "Tz"):
            setattr(self, k, getattr(s, k))

    def state(self):
        return {k: getattr(self, k) for k in ("cx", "cy", "cz", "r", "vx", "vy", "vz", "wx", "wy",
                                              "wz", "Fx", "Fy", "Fz", "Tx", "Ty", "Tz")}


class CompositeSolid:
    """Several rigid spheres acting as one solid: a cell is solid when any
    sphere contains it, and the first containing sphere owns it (its surface
    velocity and every impulse applied at it).  Same duck-typed interface as
    RigidSphere (src/solid.js:50-80)."""

    def __init__(self, spheres):
        if len(spheres) > MAX_SPHERES:
            raise ValueError(f"at most {MAX_SPHERES} spheres")
        self.spheres = list(spheres)

    def owner(self, x, y, z):
        for b in self.spheres:
            if b.contains(x, y, z):
                return b
        return None

    def contains(self, x, y, z):
        return self.owner(x, y, z) is not None

    def surfaceVelocity(self, x, y, z, out=None):
        b = self.owner(x, y, z)
        out = out if out is not None else [0.0, 0.0, 0.0]
        if b is None:
            out[0] = out[1] = out[2] = 0.0
            return out
        return b.surfaceVelocity(x, y, z, out)

    def applyImpulseAtCell(self, x, y, z, px, py, pz):
        b = self.owner(x, y, z)
        if b is not None:
            b.applyImpulseAtCell(x, y, z, px, py, pz)

    def absorbDeadCells(self, sim):
        sim._absorb_dead(self.spheres)

    def step(self, dt, gravity):
        for b in self.spheres:
            b.step(dt, gravity)


def is_generic(solid):
    """A duck-typed solid that is not made of RigidSpheres (README.md:69-73:
    any object with contains / surfaceVelocity / applyImpulseAtCell)."""
    return solid is not None and not isinstance(solid, (RigidSphere, CompositeSolid))


def spheres_of(solid):
    """The list of RigidSpheres behind a solid argument (None -> [])."""
    if solid is None:
        return []
    if isinstance(solid, RigidSphere):
        return [solid]
    if isinstance(solid, CompositeSolid):
        return solid.spheres
    raise TypeError(
        "the sphere descriptors take a RigidSphere, a CompositeSolid or None; got " + type(solid).__name__)


def evaluate_generic(solid, nx, ny, nz):
    """retagCells' calls of a duck-typed solid (src/sim.js:214-244), in the
    reference's order: solid.contains(x, y, z) for every interior cell and
    solid.surfaceVelocity for the cells it contains.  Returns the mask (n
    bytes) and the surface velocities (3n float32)."""
    import numpy as np
    n = nx * ny * nz
    mask = np.zeros(n, dtype=np.uint8)
    us = np.zeros(3 * n, dtype=np.float32)
    tmp = [0.0, 0.0, 0.0]
    contains, velocity = solid.contains, solid.surfaceVelocity
    for z in range(1, nz - 1):
        for y in range(1, ny - 1):
            base = (z * ny + y) * nx
            for x in range(1, nx - 1):
                if contains(x, y, z):
                    i = base + x
                    mask[i] = 1
                    velocity(x, y, z, tmp)
                    us[3 * i] = tmp[0]
                    us[3 * i + 1] = tmp[1]
                    us[3 * i + 2] = tmp[2]
    return mask, us


def to_c_array(spheres):
    arr = (LbmSphere * max(1, len(spheres)))()
    for i, b in enumerate(spheres):
        b.to_c(arr[i])
    return arr


def impulse_array(n):
    return (LbmImpulse * max(1, n))()
