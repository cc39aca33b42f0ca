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


def test_host_integrator_entry_matches_oracle(oracle_mod):
    """lbm_sphere_step_host (the C ABI's FP64 RigidSphere.step, the same code
    the device-resident loop runs) against the oracle's or_sphere_step, bit for
    bit, over random states that reach every branch: drag spring, acceleration
    and speed caps, damping, snap, wall clamps, zero and NaN gravity."""
    import math
    import random

    from b200lbm._capi import LbmSphere, lib
    rnd = random.Random(5)
    L = lib()
    keys = ("cx", "cy", "cz", "vx", "vy", "vz", "wx", "wy", "wz", "Fx", "Fy", "Fz", "Tx", "Ty", "Tz")
    for t in range(400):
        nx, ny, nz = 40, 28, 40
        o = oracle_mod.OracleSphere(nx, ny, nz, cx=rnd.uniform(2, 38), cy=rnd.uniform(2, 26), cz=rnd.uniform(2, 38),
                                    r=rnd.uniform(2, 6), density=rnd.uniform(0.4, 3.0))
        for k in ("vx", "vy", "vz"):
            setattr(o, k, rnd.choice([0.0, rnd.uniform(-0.12, 0.12), rnd.uniform(-2e-4, 2e-4)]))
        for k in ("wx", "wy", "wz"):
            setattr(o, k, rnd.choice([0.0, rnd.uniform(-0.05, 0.05), rnd.uniform(-2e-4, 2e-4)]))
        for k in ("Fx", "Fy", "Fz", "Tx", "Ty", "Tz"):
            setattr(o, k, rnd.uniform(-2, 2) * 10 ** rnd.uniform(-4, 1))
        o.dragging = rnd.random() < 0.3
        o.dragTargetX, o.dragTargetY, o.dragTargetZ = rnd.uniform(0, 40), rnd.uniform(0, 28), rnd.uniform(0, 40)
        g = rnd.choice([0.0, float("nan"), -1e-5, 0.0012, -0.0015])
        c = LbmSphere()
        for k in keys + ("r", "density", "mass", "I", "dragTargetX", "dragTargetY", "dragTargetZ"):
            setattr(c, k, getattr(o, k))
        c.dragging = int(o.dragging)
        assert L.lbm_sphere_step_host(c, 1, 1.0, g, nx, ny, nz) == 0
        o.step(1.0, g)
        for k in keys:
            a, b = getattr(c, k), getattr(o, k)
            assert a == b or (math.isnan(a) and math.isnan(b)), (t, k, a, b)
            assert math.copysign(1.0, a) == math.copysign(1.0, b), (t, k, a, b)
