"""Scene builders shared by the oracle (CPU checker) and the CUDA path.

Each builder takes the Sim class and the sphere class, so the same setup code
(plain property writes and direct field writes, as the reference's test/*.mjs
and src/worker.js do) runs against both.  Returns (sim, solid).
"""
import math

import numpy as np

W7 = np.array([1 / 4, 1 / 8, 1 / 8, 1 / 8, 1 / 8, 1 / 8, 1 / 8])


def _params(sim, tau, tauPhi, sigma, gravity, rhoL=1.0, rhoG=0.1, W=4.0):
    sim.tau = tau
    sim.tauPhi = tauPhi
    sim.sigma = sigma
    sim.gravity = gravity
    sim.rhoL = rhoL
    sim.rhoG = rhoG
    sim.W = W


def smoke(SimC, SphC):
    """test/smoke.mjs:7-19 (12^3, 80 steps)."""
    sim = SimC(12, 12, 12)
    sim.initFlat(6)
    _params(sim, 0.7, 0.7, 0.012, 0.0012)
    solid = SphC(12, 12, 12, cx=6, cy=3, cz=6, r=2.0, density=1.5)
    return sim, solid


def profile(SimC, SphC):
    """test/profile.mjs:4-12 (8x12x8, no solid)."""
    sim = SimC(8, 12, 8)
    sim.initFlat(6)
    _params(sim, 0.7, 0.7, 0.012, 0.0012)
    return sim, None


def bench(SimC, SphC):
    """test/bench.mjs:6-11 (40x28x40)."""
    sim = SimC(40, 28, 40)
    sim.initFlat(14)
    _params(sim, 0.7, 0.7, 0.012, 0.00135)
    solid = SphC(40, 28, 40, cx=20, cy=6, cz=20, r=4, density=1.6)
    return sim, solid


def drop(SimC, SphC, sigma=0.008, gravity=0.0015):
    """src/worker.js:23-53 'drop' preset (heavy ball falling into the pool)."""
    NX, NY, NZ = 40, 28, 40
    sim = SimC(NX, NY, NZ)
    _params(sim, 0.85, 0.7, sigma, gravity)
    solid = SphC(NX, NY, NZ, cx=NX * 0.5, cy=NY * 0.20, cz=NZ * 0.5, r=4.0, density=1.6)
    sim.initFlat(NY * 0.25)
    solid.cx, solid.cy, solid.cz = NX * 0.5, NY * 0.35, NZ * 0.5
    solid.setRadius(4.0)
    solid.setDensity(2.0)
    return sim, solid


def dam(SimC, SphC):
    """src/worker.js:54-79 'dam' preset: direct phi/phiPrev/h writes, then seedHydrostatic."""
    NX, NY, NZ = 40, 28, 40
    sim = SimC(NX, NY, NZ)
    _params(sim, 0.85, 0.7, 0.008, 0.0015)
    solid = SphC(NX, NY, NZ, cx=NX * 0.5, cy=NY * 0.20, cz=NZ * 0.5, r=4.0, density=1.6)
    sim.initFlat(NY + 1)
    phi = np.array(sim.phi, dtype=np.float32)
    h = np.array(sim.h, dtype=np.float32).reshape(-1, 7)
    for z in range(1, NZ - 1):
        for y in range(1, NY - 1):
            p = 1.0 if y > NY * 0.35 else 0.0
            xs = [x for x in range(1, NX - 1) if x < NX * 0.35]
            for x in range(1, NX - 1):
                i = sim.idx(x, y, z)
                pv = p if x in xs else 0.0
                phi[i] = pv
                h[i, :] = (W7 * pv).astype(np.float32)
    sim.phi[:] = phi
    sim.phiPrev[:] = phi
    sim.h[:] = h.reshape(-1)
    sim.seedHydrostatic()
    solid.cx, solid.cy, solid.cz = NX * 0.7, NY * 0.6, NZ * 0.5
    solid.setRadius(3.5)
    solid.setDensity(0.5)
    return sim, solid


def rise(SimC, SphC):
    """src/worker.js:81-90 'rise' preset: a buoyant ball (density 0.5) below the surface."""
    NX, NY, NZ = 40, 28, 40
    sim = SimC(NX, NY, NZ)
    _params(sim, 0.85, 0.7, 0.008, 0.0015)
    solid = SphC(NX, NY, NZ, cx=NX * 0.5, cy=NY * 0.20, cz=NZ * 0.5, r=4.0, density=1.6)
    sim.initFlat(NY * 0.25)
    solid.cx, solid.cy, solid.cz = NX * 0.5, NY * 0.65, NZ * 0.5
    solid.setRadius(4.0)
    solid.setDensity(0.5)
    return sim, solid


def drag(SimC, SphC):
    """test/drag_stress.mjs:6-18: a density-1.4 sphere dragged by its spring
    (RigidSphere.step, src/solid.js:118-131) along DRAG_PATH."""
    NX, NY, NZ = 40, 28, 40
    sim = SimC(NX, NY, NZ)
    _params(sim, 0.8, 0.7, 0.008, 0.0015)
    sim.initFlat(NY * 0.25)
    solid = SphC(NX, NY, NZ, cx=NX * 0.5, cy=NY * 0.65, cz=NZ * 0.5, r=4, density=1.4)
    solid.dragging = True
    return sim, solid


# (steps, target) legs of test/drag_stress.mjs:20-26: to the floor, along it,
# up through the interface, along the top, back down through the interface
DRAG_PATH = [(100, (20, 24, 20)), (100, (30, 24, 20)), (200, (30, 4, 20)), (100, (20, 4, 20)),
             (200, (20, 18, 20))]


def drag_target(solid, step, path=DRAG_PATH):
    """Set the drag target for (0-based) step `step` of the path."""
    for n, t in path:
        if step < n:
            solid.dragTargetX, solid.dragTargetY, solid.dragTargetZ = t
            return
        step -= n
    solid.dragTargetX, solid.dragTargetY, solid.dragTargetZ = path[-1][1]


def mirrored_pool(sim, level, W):
    """Liquid below y = level (phi = 1/2 (1 + tanh(2 (level - y)/W))) on every
    cell, h = w7 * phi, then seedHydrostatic -- the dam-preset pattern
    (src/worker.js:57-73) used for the gravity-down scenes."""
    nx, ny, nz = sim.nx, sim.ny, sim.nz
    ys = np.arange(ny, dtype=np.float64)
    col = 0.5 * (1 + np.tanh(2 * (level - ys) / W))
    phi = np.broadcast_to(col[None, :, None], (nz, ny, nx)).reshape(-1)
    sim.phi[:] = phi.astype(np.float32)
    sim.phiPrev[:] = phi.astype(np.float32)
    sim.h[:] = (phi[:, None] * W7[None, :]).astype(np.float32).reshape(-1)
    sim.seedHydrostatic()


def cfg1(SimC, SphC):
    """40x28x40, liquid below y = 10, tau 0.6, tauPhi 0.8, sigma 1e-3, g = -1e-5,
    sphere r = 5, density 2 at (20, 21, 20), 80 steps."""
    sim = SimC(40, 28, 40)
    _params(sim, 0.6, 0.8, 1e-3, -1e-5)
    sim.initFlat(10)
    mirrored_pool(sim, 10.0, 4.0)
    solid = SphC(40, 28, 40, cx=20, cy=21, cz=20, r=5, density=2.0)
    return sim, solid


def cfg2_interface(nx, nz, seed=0, level=96.0, amp=0.5, wavelength=64.0):
    """Seeded interface height y_w(x, z) = level + amp sin(2 pi x/L + tx) cos(2 pi z/L + tz)."""
    rng = np.random.default_rng(seed)
    tx, tz = rng.uniform(0, 2 * math.pi, size=2)
    xs = np.arange(nx)[None, :]
    zs = np.arange(nz)[:, None]
    return level + amp * np.sin(2 * math.pi * xs / wavelength + tx) * np.cos(2 * math.pi * zs / wavelength + tz)


def wavy_pool(sim, yw, W):
    """phi = 1/2 (1 + tanh(2 (y_w(x,z) - y)/W)) per column, h = w7 phi, seedHydrostatic."""
    nx, ny, nz = sim.nx, sim.ny, sim.nz
    ys = np.arange(ny, dtype=np.float64)[None, :, None]
    phi = 0.5 * (1 + np.tanh(2 * (yw[:, None, :] - ys) / W))  # (nz, ny, nx)
    phi = phi.reshape(-1)
    sim.phi[:] = phi.astype(np.float32)
    sim.phiPrev[:] = phi.astype(np.float32)
    sim.h[:] = (phi[:, None] * W7[None, :]).astype(np.float32).reshape(-1)
    sim.seedHydrostatic()


def cfg2(SimC, SphC, n=256, seed=0):
    """n^3 (256^3 by default), liquid below a seeded +-0.5 cell sinusoidal interface at
    y = 96 n/256, sphere r = 24 n/256, density 2 at (n/2, 200 n/256, n/2)."""
    s = n / 256.0
    sim = SimC(n, n, n)
    _params(sim, 0.6, 0.8, 1e-3, -1e-5)
    sim.initFlat(96 * s)
    wavy_pool(sim, cfg2_interface(n, n, seed, level=96 * s, wavelength=64 * s), 4.0)
    solid = SphC(n, n, n, cx=128 * s, cy=200 * s, cz=128 * s, r=24 * s, density=2.0)
    return sim, solid


SCENES = {"smoke": smoke, "profile": profile, "bench": bench, "drop": drop, "dam": dam,
          "cfg1": cfg1, "rise": rise, "drag": drag}


def substep(sim, solid):
    """One worker tick (src/worker.js:96-100)."""
    sim.step(solid)
    if solid is not None:
        solid.absorbDeadCells(sim)
        solid.step(1.0, sim.gravity)


def field_err(a, b, norm=None):
    """(rel-L2, Linf) of a against reference b; Linf scaled by `norm` if given."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    d = a - b
    nb = np.linalg.norm(b)
    rel = np.linalg.norm(d) / (nb if nb > 0 else 1.0)
    linf = np.abs(d).max() if d.size else 0.0
    if norm:
        linf /= norm
    return rel, linf


class Crate:
    """A duck-typed solid that is not a sphere (README.md:69-73: any object
    with contains / surfaceVelocity / applyImpulseAtCell works): an
    axis-aligned box moving at a fixed velocity, kinematically (its step only
    moves it), accumulating the force and torque the fluid exerts.  Its
    absorbDeadCells follows src/solid.js:87-101 for this body."""

    def __init__(self, lo, hi, vel):
        self.lo = [float(v) for v in lo]
        self.hi = [float(v) for v in hi]
        self.vx, self.vy, self.vz = (float(v) for v in vel)
        self.Fx = self.Fy = self.Fz = 0.0
        self.Tx = self.Ty = self.Tz = 0.0

    def centre(self):
        return [(a + b) * 0.5 for a, b in zip(self.lo, self.hi)]

    def contains(self, x, y, z):
        p = (x + 0.5, y + 0.5, z + 0.5)
        return all(self.lo[a] <= p[a] <= self.hi[a] for a in range(3))

    def surfaceVelocity(self, x, y, z, out):
        out[0] = self.vx
        out[1] = self.vy
        out[2] = self.vz

    def applyImpulseAtCell(self, x, y, z, px, py, pz):
        cx, cy, cz = self.centre()
        rx, ry, rz = x + 0.5 - cx, y + 0.5 - cy, z + 0.5 - cz
        self.Fx += px
        self.Fy += py
        self.Fz += pz
        self.Tx += ry * pz - rz * py
        self.Ty += rz * px - rx * pz
        self.Tz += rx * py - ry * px

    def absorbDeadCells(self, sim):
        nx, ny, nz = sim.nx, sim.ny, sim.nz
        tag, prev, phi = sim.tag, sim.tagPrev, sim.phi
        ux, uy, uz = sim.ux, sim.uy, sim.uz
        dRho = sim.rhoL - sim.rhoG
        # dead cells are inside the box: scan its cells (in the reference's order)
        rng = [range(max(1, int(self.lo[a] - 1)), min(n - 1, int(self.hi[a]) + 2))
               for a, n in enumerate((nx, ny, nz))]
        for z in rng[2]:
            for y in rng[1]:
                for x in rng[0]:
                    i = (z * ny + y) * nx + x
                    if tag[i] != 1 or prev[i] != 0:
                        continue
                    rhoPhase = sim.rhoG + float(phi[i]) * dRho
                    self.applyImpulseAtCell(x, y, z, rhoPhase * float(ux[i]), rhoPhase * float(uy[i]),
                                            rhoPhase * float(uz[i]))

    def step(self, dt, gravity):
        for a, v in enumerate((self.vx, self.vy, self.vz)):
            self.lo[a] += dt * v
            self.hi[a] += dt * v
        self.Fx = self.Fy = self.Fz = 0.0
        self.Tx = self.Ty = self.Tz = 0.0


def crate(SimC, SphC=None):
    """The drop preset's pool (src/worker.js:23-53; sigma 0.012, g 0.0012) with
    a moving box instead of the sphere: 6.2 x 5.5 x 6.5 cells, not aligned to
    the lattice, sliding down and sideways through the liquid."""
    sim = SimC(40, 28, 40)
    _params(sim, 0.85, 0.7, 0.012, 0.0012)
    sim.initFlat(7)
    return sim, Crate((14.2, 15.6, 17.3), (20.4, 21.1, 23.8), (0.03, -0.05, 0.02))
