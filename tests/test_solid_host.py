"""Host-side RigidSphere (src/solid.js) against the oracle's C restatement:
the FP64 integrator, contains / surfaceVelocity / applyImpulseAtCell agree
bit for bit."""
import math
import random

import pytest


def _pair(oracle_mod, **kw):
    from b200lbm.solid import RigidSphere
    return RigidSphere(40, 28, 40, **kw), oracle_mod.OracleSphere(40, 28, 40, **kw)


FIELDS = ("cx", "cy", "cz", "vx", "vy", "vz", "wx", "wy", "wz", "Fx", "Fy", "Fz", "Tx", "Ty", "Tz")


@pytest.mark.parametrize("seed", range(6))
def test_step_bit_exact(oracle_mod, seed):
    rnd = random.Random(seed)
    a, b = _pair(oracle_mod, cx=20, cy=9.8, cz=20, r=4, density=2.0)
    for t in range(300):
        imp = [rnd.uniform(-1, 1) * 10 ** rnd.uniform(-4, 1) for _ in range(3)]
        x, y, z = rnd.randrange(1, 39), rnd.randrange(1, 27), rnd.randrange(1, 39)
        a.applyImpulseAtCell(x, y, z, *imp)
        b.applyImpulseAtCell(x, y, z, *imp)
        if t % 50 == 10:
            for s in (a, b):
                s.dragging = not s.dragging
                s.dragTargetX, s.dragTargetY, s.dragTargetZ = 30, 4, 20
        g = rnd.choice([0.0012, -1e-5, 0.0015, 0.0])
        a.step(1.0, g)
        b.step(1.0, g)
        for k in FIELDS:
            assert getattr(a, k) == getattr(b, k), (t, k)


def test_contains_and_surface_velocity(oracle_mod):
    a, b = _pair(oracle_mod, cx=20.3, cy=11.7, cz=19.1, r=4.6, density=1.3)
    for s in (a, b):
        s.vx, s.vy, s.vz, s.wx, s.wy, s.wz = 0.01, -0.02, 0.003, 0.001, 0.002, -0.004
    for x in range(14, 27):
        for y in range(6, 18):
            for z in range(13, 26):
                assert a.contains(x, y, z) == b.contains(x, y, z)
                assert a.surfaceVelocity(x, y, z) == b.surfaceVelocity(x, y, z)


def test_mass_and_inertia(oracle_mod):
    a, b = _pair(oracle_mod, r=3.5, density=0.5)
    assert a.mass == b.mass and a.I == b.I
    a.setRadius(4.25)
    b.setRadius(4.25)
    a.setDensity(2.5)
    b.setDensity(2.5)
    assert a.mass == b.mass == 2.5 * (4 / 3) * math.pi * 4.25 ** 3
