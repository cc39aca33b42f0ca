"""Seeded synthetic workloads: many-scene batches and a served request stream.

The reference has one hard-coded scene per preset (src/worker.js:23-79) and no
dataset.  These generators produce the multi-scene workloads the batch and the
server are measured on, from a seed:

  * scene_specs(n, seed): n scenes with grid edges uniform integers in
    [32, 160] per axis, a liquid pool filling a uniform 30-60% of ny (liquid
    below, gravity -y, as in the gravity-down scenes), and 1-3 spheres each
    with r ~ U[3, 12], density ~ U[1.2, 4.0], speed <= 0.02 in a uniform
    direction, centred above the interface, inside RigidSphere.step's clamp
    margin r + 1.5 (src/solid.js:199-205) and not overlapping each other.
    Placement rule: each sphere is drawn (r, density, position) until it fits,
    up to 200 draws; a sphere that still does not fit is dropped, and a scene
    left with none gets one sphere of r = 3 (which always fits for ny >= 32
    and a fill <= 60%).
  * request_stream(n, seed): Poisson arrivals at a given rate; each request
    is a scene from the same distribution, or with probability 0.1 the 256^3
    benchmark scene; 500-5000 steps (a multiple of the frame cadence), one RG8
    frame every 20 steps (the worker's frame cadence, src/worker.js:94-111,
    generalised).
"""
from __future__ import annotations

import math

import numpy as np

from .sim import Sim
from .solid import CompositeSolid, RigidSphere

# physics of the gravity-down scenes: liquid below, g along -y
PHYSICS = dict(tau=0.6, tauPhi=0.8, sigma=1e-3, gravity=-1e-5, rhoL=1.0, rhoG=0.1, W=4.0)
W7 = np.array([1 / 4, 1 / 8, 1 / 8, 1 / 8, 1 / 8, 1 / 8, 1 / 8])


def _sphere(rng, nx, ny, nz, level, placed, r=None):
    for _ in range(200):
        rr = float(rng.uniform(3.0, 12.0)) if r is None else r
        dens = float(rng.uniform(1.2, 4.0))
        m = rr + 1.5
        ylo = max(m, level + rr)
        yhi = ny - 1 - m
        if ylo > yhi or m > nx - 1 - m or m > nz - 1 - m:
            continue
        c = (float(rng.uniform(m, nx - 1 - m)), float(rng.uniform(ylo, yhi)),
             float(rng.uniform(m, nz - 1 - m)))
        if any(math.dist(c, (p["cx"], p["cy"], p["cz"])) <= rr + p["r"] for p in placed):
            continue
        speed = float(rng.uniform(0.0, 0.02))
        d = rng.normal(size=3)
        d /= np.linalg.norm(d) or 1.0
        return dict(cx=c[0], cy=c[1], cz=c[2], r=rr, density=dens,
                    vx=float(speed * d[0]), vy=float(speed * d[1]), vz=float(speed * d[2]))
    return None


def scene_spec(rng):
    nx, ny, nz = (int(v) for v in rng.integers(32, 161, size=3))
    level = float(rng.uniform(0.3, 0.6)) * ny
    placed = []
    for _ in range(int(rng.integers(1, 4))):
        s = _sphere(rng, nx, ny, nz, level, placed)
        if s is not None:
            placed.append(s)
    if not placed:
        placed.append(_sphere(rng, nx, ny, nz, level, placed, r=3.0))
    return dict(dims=(nx, ny, nz), level=level, spheres=placed)


def scene_specs(n=64, seed=0):
    rng = np.random.default_rng(seed)
    return [scene_spec(rng) for _ in range(n)]


def big_spec(n=256):
    """The n^3 benchmark scene: pool below y = 96 n/256, one density-2 sphere
    of radius 24 n/256 at (n/2, 200 n/256, n/2)."""
    s = n / 256.0
    return dict(dims=(n, n, n), level=96 * s,
                spheres=[dict(cx=128 * s, cy=200 * s, cz=128 * s, r=24 * s, density=2.0,
                              vx=0.0, vy=0.0, vz=0.0)])


def pool_column(ny, level, W=4.0):
    """phi of a pool below `level`: 1/2 (1 + tanh(2 (level - y) / W)) per row."""
    ys = np.arange(ny, dtype=np.float64)
    return 0.5 * (1 + np.tanh(2 * (level - ys) / W))


def pool_below_host(sim, level, W=4.0):
    """phi = pool_column on every cell, h = w7 phi, then seedHydrostatic,
    written from the host as the dam preset does (src/worker.js:57-73)."""
    nx, ny, nz = sim.nx, sim.ny, sim.nz
    col = pool_column(ny, level, W)
    phi = np.broadcast_to(col[None, :, None], (nz, ny, nx)).reshape(-1)
    sim.phi[:] = phi.astype(np.float32)
    sim.phiPrev[:] = phi.astype(np.float32)
    sim.h[:] = (phi[:, None] * W7[None, :]).astype(np.float32).reshape(-1)
    sim.seedHydrostatic()


def pool_below(sim, level, W=4.0):
    """The same state as pool_below_host, initialised on the device from the
    column profile (Sim.initProfile): nothing crosses the host link."""
    sim.initProfile(pool_column(sim.ny, level, W))


def build(spec, storage="f16", device=0):
    """A Sim and its solid (a RigidSphere, or a CompositeSolid for several)."""
    nx, ny, nz = spec["dims"]
    sim = Sim(nx, ny, nz, storage=storage, device=device)
    for k, v in PHYSICS.items():
        setattr(sim, k, v)
    pool_below(sim, spec["level"], PHYSICS["W"])
    spheres = []
    for p in spec["spheres"]:
        b = RigidSphere(nx, ny, nz, cx=p["cx"], cy=p["cy"], cz=p["cz"], r=p["r"], density=p["density"])
        b.vx, b.vy, b.vz = p["vx"], p["vy"], p["vz"]
        spheres.append(b)
    solid = spheres[0] if len(spheres) == 1 else CompositeSolid(spheres)
    return sim, solid


def request_stream(n=24, seed=0, rate=20.0, frame_every=20, min_steps=500, max_steps=5000, big_frac=0.1,
                   big_n=256):
    """Seeded request trace: dicts (rid, arrival in s, spec, steps, frame_every)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n):
        t += float(rng.exponential(1.0 / rate))
        spec = big_spec(big_n) if rng.uniform() < big_frac else scene_spec(rng)
        steps = int(rng.integers(min_steps, max_steps + 1))
        steps = max(frame_every, steps // frame_every * frame_every)
        out.append(dict(rid=i, arrival=t, spec=spec, steps=steps, frame_every=frame_every))
    return out


def cells(spec):
    nx, ny, nz = spec["dims"]
    return nx * ny * nz
