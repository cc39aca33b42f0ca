"""MeshSolid -- a rigid body given as a closed triangle mesh, for the solid
interface the reference's fluid code calls: contains / surfaceVelocity /
applyImpulseAtCell and absorbDeadCells (src/solid.js:50-101).  The reference
notes that this interface is mesh-agnostic and that its source paper
rasterises meshes every frame (README.md:65-73); its only body is the
analytic sphere.

On the device path (Sim.step with a MeshSolid) the mesh is voxelised by the
library (lbm_retag_cells_mesh): the cells whose centre lies inside the
closed mesh -- an odd number of crossings of the ray from the centre towards
+x -- become SOLID with the rigid-body surface velocity.  `contains` restates
the same test on the host in double arithmetic, operation for operation, so
both decide every cell the same way (the host loop is the reference's
generic route and the parity check of the device voxeliser).

The body's pose: body-frame vertices `vertices` (relative to nothing in
particular), a rotation `R` (3x3) about the reference point and the point's
position (cx, cy, cz); world vertex = R (v - origin) + c, with origin the
reference point's body-frame position.  Motion is prescribed (kinematic):
`step(dt)` moves the body by its velocity and angular velocity; the momentum
exchange is accumulated in Fx..Tz (FP64, the reference's formulas) for the
caller to use.  The reference has no mesh dynamics to follow, so none is
invented here.
"""
from __future__ import annotations

import math

import numpy as np

from ._capi import LbmRigidMotion


class MeshSolid:
    def __init__(self, vertices, triangles, center, velocity=(0.0, 0.0, 0.0),
                 angular_velocity=(0.0, 0.0, 0.0), origin=None):
        self.v0 = np.asarray(vertices, dtype=np.float64).reshape(-1, 3)
        self.tris = np.asarray(triangles, dtype=np.int64).reshape(-1, 3)
        if self.tris.size and (self.tris.min() < 0 or self.tris.max() >= len(self.v0)):
            raise ValueError("triangle indices out of range")
        self.origin = np.asarray(self.v0.mean(axis=0) if origin is None else origin, dtype=np.float64)
        self.cx, self.cy, self.cz = (float(c) for c in center)
        self.vx, self.vy, self.vz = (float(v) for v in velocity)
        self.wx, self.wy, self.wz = (float(w) for w in angular_velocity)
        self.R = np.eye(3)
        self.Fx = self.Fy = self.Fz = 0.0
        self.Tx = self.Ty = self.Tz = 0.0
        self.use_device = True  # False: Sim evaluates contains / surfaceVelocity per cell on the host
        self._cache = None

    # ------------------------------------------------------------ geometry
    def world_triangles(self):
        """(ntri, 9) world coordinates of the triangles' vertices A, B, C."""
        key = (self.cx, self.cy, self.cz, self.R.tobytes())
        if self._cache is None or self._cache[0] != key:
            c = np.array([self.cx, self.cy, self.cz])
            w = (self.v0 - self.origin) @ self.R.T + c
            tri = np.ascontiguousarray(w[self.tris].reshape(-1, 9))
            self._cache = (key, tri)
        return self._cache[1]

    def motion(self):
        m = LbmRigidMotion()
        for k in ("cx", "cy", "cz", "vx", "vy", "vz", "wx", "wy", "wz"):
            setattr(m, k, float(getattr(self, k)))
        return m

    def crossings(self, px, py, pz):
        """Triangles the +x ray from (px, py, pz) crosses (the device's
        ray_crosses, restated with the same operations in the same order)."""
        t = self.world_triangles()
        ax, ay, az, bx, by, bz, cx, cy, cz = (t[:, j] for j in range(9))
        nx = (by - ay) * (cz - az) - (bz - az) * (cy - ay)
        swap = nx < 0.0
        y1, z1 = np.where(swap, cy, by), np.where(swap, cz, bz)
        y2, z2 = np.where(swap, by, cy), np.where(swap, bz, cz)

        def edge(py_, pz_, qy, qz):
            return (qy - py_) * (pz - pz_) - (qz - pz_) * (py - py_)

        def top_left(py_, pz_, qy, qz):
            dy, dz = qy - py_, qz - pz_
            return ((dz == 0.0) & (dy < 0.0)) | (dz < 0.0)

        e0, e1, e2 = edge(ay, az, y1, z1), edge(y1, z1, y2, z2), edge(y2, z2, ay, az)
        inside = ((e0 > 0.0) | ((e0 == 0.0) & top_left(ay, az, y1, z1))) \
            & ((e1 > 0.0) | ((e1 == 0.0) & top_left(y1, z1, y2, z2))) \
            & ((e2 > 0.0) | ((e2 == 0.0) & top_left(y2, z2, ay, az))) & (nx != 0.0)
        ny = (bz - az) * (cx - ax) - (bx - ax) * (cz - az)
        nz = (bx - ax) * (cy - ay) - (by - ay) * (cx - ax)
        with np.errstate(divide="ignore", invalid="ignore"):
            xh = ax - (ny * (py - ay) + nz * (pz - az)) / nx
        return int(np.count_nonzero(inside & (xh > px)))

    # ------------------------------------------------------------ the solid interface
    def contains(self, x, y, z):
        return (self.crossings(x + 0.5, y + 0.5, z + 0.5) & 1) == 1

    def surfaceVelocity(self, x, y, z, out):
        # u_body + omega x r (src/solid.js:57-66)
        rx = x + 0.5 - self.cx
        ry = y + 0.5 - self.cy
        rz = z + 0.5 - self.cz
        out[0] = self.vx + (self.wy * rz - self.wz * ry)
        out[1] = self.vy + (self.wz * rx - self.wx * rz)
        out[2] = self.vz + (self.wx * ry - self.wy * rx)
        return out

    def applyImpulseAtCell(self, x, y, z, px, py, pz):
        # src/solid.js:70-80
        self.Fx += px
        self.Fy += py
        self.Fz += pz
        rx = x + 0.5 - self.cx
        ry = y + 0.5 - self.cy
        rz = z + 0.5 - self.cz
        self.Tx += ry * pz - rz * py
        self.Ty += rz * px - rx * pz
        self.Tz += rx * py - ry * px

    def absorbDeadCells(self, sim):
        """src/solid.js:87-101 over the scene's fields, in scan order."""
        nx, ny, nz = sim.nx, sim.ny, sim.nz
        tag = np.asarray(sim.tag).reshape(nz, ny, nx)
        prev = np.asarray(sim.tagPrev).reshape(nz, ny, nx)
        dead = np.argwhere((tag == 1) & (prev == 0))
        if not len(dead):
            return
        phi, ux, uy, uz = (np.asarray(getattr(sim, k)) for k in ("phi", "ux", "uy", "uz"))
        dRho = sim.rhoL - sim.rhoG
        for z, y, x in dead.tolist():  # argwhere is in scan order (z, y, x)
            if not (0 < x < nx - 1 and 0 < y < ny - 1 and 0 < z < nz - 1):
                continue
            i = (z * ny + y) * nx + x
            rho_phase = sim.rhoG + float(phi[i]) * dRho
            self.applyImpulseAtCell(x, y, z, rho_phase * float(ux[i]), rho_phase * float(uy[i]),
                                    rho_phase * float(uz[i]))

    def step(self, dt=1.0, gravity=None):
        """Prescribed motion: the reference point moves by v dt and the body
        turns by w dt about it (a rotation by |w| dt about w / |w|)."""
        self.cx += self.vx * dt
        self.cy += self.vy * dt
        self.cz += self.vz * dt
        w = math.sqrt(self.wx * self.wx + self.wy * self.wy + self.wz * self.wz)
        if w > 0.0:
            k = np.array([self.wx, self.wy, self.wz]) / w
            a = w * dt
            K = np.array([[0.0, -k[2], k[1]], [k[2], 0.0, -k[0]], [-k[1], k[0], 0.0]])
            self.R = (np.eye(3) + math.sin(a) * K + (1.0 - math.cos(a)) * (K @ K)) @ self.R
        self.Fx = self.Fy = self.Fz = 0.0
        self.Tx = self.Ty = self.Tz = 0.0


def box_mesh(lo, hi):
    """A closed axis-aligned box: 8 vertices, 12 triangles (outward normals)."""
    (x0, y0, z0), (x1, y1, z1) = lo, hi
    v = [(x0, y0, z0), (x1, y0, z0), (x1, y1, z0), (x0, y1, z0),
         (x0, y0, z1), (x1, y0, z1), (x1, y1, z1), (x0, y1, z1)]
    t = [(0, 2, 1), (0, 3, 2), (4, 5, 6), (4, 6, 7), (0, 1, 5), (0, 5, 4),
         (2, 3, 7), (2, 7, 6), (1, 2, 6), (1, 6, 5), (0, 4, 7), (0, 7, 3)]
    return np.array(v, dtype=np.float64), np.array(t, dtype=np.int64)


def icosphere(center, r, subdivisions=2):
    """A closed triangulated sphere (subdivided icosahedron)."""
    p = (1.0 + math.sqrt(5.0)) / 2.0
    v = [(-1, p, 0), (1, p, 0), (-1, -p, 0), (1, -p, 0), (0, -1, p), (0, 1, p),
         (0, -1, -p), (0, 1, -p), (p, 0, -1), (p, 0, 1), (-p, 0, -1), (-p, 0, 1)]
    v = [np.array(a, dtype=np.float64) / np.linalg.norm(a) for a in v]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
         (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5),
         (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(subdivisions):
        mid = {}

        def m(a, b):
            key = (min(a, b), max(a, b))
            if key not in mid:
                c = v[a] + v[b]
                v.append(c / np.linalg.norm(c))
                mid[key] = len(v) - 1
            return mid[key]

        f = [t for a, b, c in f for t in ((a, m(a, b), m(c, a)), (b, m(b, c), m(a, b)),
                                           (c, m(c, a), m(b, c)), (m(a, b), m(b, c), m(c, a)))]
    verts = np.array(v) * r + np.asarray(center, dtype=np.float64)
    return verts, np.array(f, dtype=np.int64)


def torus(center, R, r, nu=24, nv=12):
    """A closed triangulated torus about the z axis."""
    cx, cy, cz = center
    verts = []
    for i in range(nu):
        u = 2 * math.pi * i / nu
        for j in range(nv):
            w = 2 * math.pi * j / nv
            verts.append((cx + (R + r * math.cos(w)) * math.cos(u), cy + (R + r * math.cos(w)) * math.sin(u),
                          cz + r * math.sin(w)))
    tris = []
    for i in range(nu):
        for j in range(nv):
            a = i * nv + j
            b = ((i + 1) % nu) * nv + j
            c = ((i + 1) % nu) * nv + (j + 1) % nv
            d = i * nv + (j + 1) % nv
            tris += [(a, b, c), (a, c, d)]
    return np.array(verts, dtype=np.float64), np.array(tris, dtype=np.int64)
