"""lbm_step also computes absorbDeadCells (src/solid.js:87-101), which the
worker calls right after every step (src/worker.js:96-100), and fetches it with
the step's impulses; lbm_absorb_dead_cells then returns that result without a
launch or a wait of its own.  Any call on the handle in between makes it
compute anew, so the result is always the one a fresh computation gives, bit
for bit, including after the fields were changed between the two calls."""
import numpy as np
import pytest

import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import b200lbm
    return b200lbm


def _falling(SimC, SphC):
    """48 x 30 x 26, a sphere moving down through the interface: cells turn
    SOLID (dead) at most steps."""
    sim = SimC(48, 30, 26)
    scenes._params(sim, 0.7, 0.75, 0.01, 0.001)
    sim.initFlat(12.5)
    sol = SphC(48, 30, 26, cx=20.3, cy=17.2, cz=12.7, r=4.1, density=2.5)
    sol.vy = -0.08
    sol.vx = 0.02
    return sim, sol


def _absorb(sim, sol):
    """lbm_absorb_dead_cells through the C ABI: the six impulse terms."""
    from b200lbm._capi import check, lib
    from b200lbm.solid import impulse_array, to_c_array
    out = impulse_array(1)
    check(sim.handle, lib().lbm_absorb_dead_cells(sim.handle, to_c_array([sol]), 1, out))
    o = out[0]
    return (o.Fx, o.Fy, o.Fz, o.Tx, o.Ty, o.Tz)


def _touch(sim):
    """A call on the handle that moves nothing (it drops the result computed
    ahead, so the next absorbDeadCells computes anew)."""
    import ctypes as C

    from b200lbm._capi import check, lib
    buf = np.empty(sim.n, dtype=np.float32)
    check(sim.handle, lib().lbm_download_field(sim.handle, 8, buf.ctypes.data_as(C.c_void_p), sim.n))


@pytest.mark.parametrize("storage", ["f32", "f16"])
def test_absorb_ahead_equals_fresh(gpu, storage):
    import functools
    SimS = functools.partial(gpu.Sim, storage=storage)
    a, sa = _falling(SimS, gpu.RigidSphere)
    b, sb = _falling(SimS, gpu.RigidSphere)
    nonzero = 0
    for t in range(30):
        a.step(sa)
        b.step(sb)
        n0 = a.launch_count()
        ia = _absorb(a, sa)  # the result computed with the step
        assert a.launch_count() == n0, "absorbDeadCells after a step launched a kernel"
        _touch(b)
        n1 = b.launch_count()
        ib = _absorb(b, sb)  # computed anew
        assert b.launch_count() > n1
        assert ia == ib, (storage, t)
        nonzero += any(v != 0 for v in ia)
        for s, imp in ((sa, ia), (sb, ib)):
            s.Fx += imp[0]
            s.Fy += imp[1]
            s.Fz += imp[2]
            s.Tx += imp[3]
            s.Ty += imp[4]
            s.Tz += imp[5]
            s.step(1.0, a.gravity)
        # a second call computes anew and agrees
        assert _absorb(a, sa) == _absorb(b, sb)
    assert nonzero >= 5, "the scene should have dead cells at several steps"
    a.close()
    b.close()


def test_absorb_after_a_field_change_sees_it(gpu):
    """A field written between the step and absorbDeadCells is seen: the
    result differs from the one computed with the step and equals a fresh
    computation on a twin that got the same write."""
    a, sa = _falling(gpu.Sim, gpu.RigidSphere)
    b, sb = _falling(gpu.Sim, gpu.RigidSphere)
    c, sc = _falling(gpu.Sim, gpu.RigidSphere)
    seen = 0
    for t in range(30):
        for sim, sol in ((a, sa), (b, sb), (c, sc)):
            sim.step(sol)
        ic = _absorb(c, sc)  # the result computed with the step
        if not any(v != 0 for v in ic):
            for sim, sol in ((a, sa), (b, sb), (c, sc)):
                sol.step(1.0, sim.gravity)
            continue
        for sim in (a, b):
            sim.phi[...] = np.asarray(sim.phi) * np.float32(0.5)
            sim._sync()  # the write goes to the device (lbm_upload_field)
        _touch(b)
        ia, ib = _absorb(a, sa), _absorb(b, sb)
        assert ia == ib
        assert ia != ic
        seen += 1
        break
    assert seen == 1, "no step with dead cells in 30 steps"
    for sim in (a, b, c):
        sim.close()
