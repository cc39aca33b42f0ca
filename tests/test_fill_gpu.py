"""The fresh-cell fill in parallel rounds (k_fresh_fill / kb_fresh_fill)
against the reference's loop -- one thread in scan order
(lbm_test_sequential_fill) -- on scenes whose spheres uncover many cells per
step, alone (host-driven and device-resident steps) and in a batch: every
field bit for bit."""
import functools

import numpy as np
import pytest

import scenes

pytestmark = pytest.mark.gpu

FIELDS = ("phi", "phiPrev", "rho", "ux", "uy", "uz", "f", "h", "tag")


@pytest.fixture(scope="module")
def gpu():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import b200lbm
    return b200lbm


def _fast(SimC, SphC):
    """46 x 40 x 38, a large sphere moving diagonally: dozens of fresh cells
    per step, in chains along x, y and z."""
    sim = SimC(46, 40, 38)
    scenes._params(sim, 0.8, 0.7, 0.008, 0.0015)
    sim.initFlat(15)
    sol = SphC(46, 40, 38, cx=20.3, cy=22.6, cz=17.9, r=7.4, density=2.5)
    sol.vx, sol.vy, sol.vz = 0.06, -0.05, 0.045
    return sim, sol


def _pair(SimC, SphC):
    from b200lbm import CompositeSolid
    sim = SimC(40, 34, 36)
    scenes._params(sim, 0.8, 0.7, 0.008, 0.0015)
    sim.initFlat(12)
    a = SphC(40, 34, 36, cx=13, cy=21, cz=18, r=5.0, density=2.5)
    b = SphC(40, 34, 36, cx=27, cy=23, cz=17, r=4.5, density=1.8)
    a.vx, a.vy = 0.05, -0.04
    b.vx, b.vz = -0.04, 0.05
    return sim, CompositeSolid([a, b])


BUILDERS = [_fast, _pair, lambda S, R: scenes.drop(S, R, sigma=0.012, gravity=0.0012)]


def _state(sim):
    return {k: np.array(getattr(sim, k)) for k in FIELDS}


def _sequential(sim, on=True):
    from b200lbm import _capi
    _capi.check(sim.handle, _capi.lib().lbm_test_sequential_fill(sim.handle, 1 if on else 0))


@pytest.mark.parametrize("storage", ["f32", "f16", "f64"])
def test_parallel_fill_equals_sequential(gpu, storage):
    SimS = functools.partial(gpu.Sim, storage=storage)
    for bi, bld in enumerate(BUILDERS):
        runs = []
        fresh_seen = 0
        for seq in (True, False):
            sim, sol = bld(SimS, gpu.RigidSphere)
            _sequential(sim, seq)
            for _ in range(12):  # host-driven steps
                scenes.substep(sim, sol)
                tag, prev = np.asarray(sim.tag), np.asarray(sim.tagPrev)
                fresh_seen += int(np.count_nonzero((tag == 0) & (prev == 1)))
            sim.run_coupled(sol, 12)  # device-resident steps
            runs.append(_state(sim))
            sim.close()
        if bi < 2:  # the drop preset starts at rest: its fresh cells come later
            assert fresh_seen > 40, (bi, fresh_seen)
        for k in FIELDS:
            assert np.array_equal(runs[0][k], runs[1][k]), (storage, bi, k)


def test_batch_parallel_fill_equals_sequential_alone(gpu):
    SimS = functools.partial(gpu.Sim, storage="f16")
    ref = []
    for bld in BUILDERS:
        sim, sol = bld(SimS, gpu.RigidSphere)
        _sequential(sim, True)
        sim.run_coupled(sol, 10)
        ref.append(_state(sim))
        sim.close()
    mixed = [bld(SimS, gpu.RigidSphere) for bld in BUILDERS]
    with gpu.Batch(mixed) as batch:
        batch.run(10)
    for i, (sim, _) in enumerate(mixed):
        got = _state(sim)
        for k in FIELDS:
            assert np.array_equal(got[k], ref[i][k]), (i, k)
        sim.close()
