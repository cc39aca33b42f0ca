"""The compact-ring forms of the fused step -- register loads (4 or 6 |
LBM_FUSED_COMPACT), per-thread asynchronous copies one plane ahead (4 or 6 |
LBM_FUSED_ASYNC), tile rows staged by bulk asynchronous copies (4 or 6 |
LBM_FUSED_STAGED) -- give, bit for bit, what the plain 4-row form gives --
for FP32, FP16 and BF16 storage, on grids whose rows start inside an 8-cell
block (odd nx), with partial tiles in x and y, with moving spheres (SOLID
links, fresh and dead cells) and a composite solid.  Run alone (lbm_step,
lbm_run_coupled) and in a batch."""
import functools

import numpy as np
import pytest

import scenes

pytestmark = pytest.mark.gpu

STAGED = 0x100
COMPACT = 0x400
ASYNC = 0x800
PIPE_SHAPES = ((4 | STAGED, 32), (6 | STAGED, 32), (4 | STAGED, 5), (6 | STAGED, 9), (4 | COMPACT, 32),
               (6 | COMPACT, 7), (6 | ASYNC, 32), (4 | ASYNC, 6), (6 | ASYNC, 5))


@pytest.fixture(scope="module")
def gpu():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import b200lbm
    return b200lbm


def _odd(SimC, SphC):
    """33 x 17 x 29: rows start off the 8-cell blocks, partial tiles, a sphere."""
    sim = SimC(33, 17, 29)
    scenes._params(sim, 0.7, 0.75, 0.01, 0.001)
    sim.initFlat(8.5)
    return sim, SphC(33, 17, 29, cx=15.3, cy=11.2, cz=13.7, r=3.1, density=2.2)


def _wide(SimC, SphC):
    """70 x 40 x 50 with a falling sphere: three x tiles (the last partial),
    y tiles that do not divide ny."""
    sim = SimC(70, 40, 50)
    scenes._params(sim, 0.8, 0.7, 0.008, 0.0015)
    sim.initFlat(12)
    sol = SphC(70, 40, 50, cx=33.5, cy=24.0, cz=25.2, r=5.5, density=2.5)
    sol.vy = -0.03
    return sim, sol


def _pair(SimC, SphC):
    from b200lbm import CompositeSolid
    sim = SimC(36, 30, 36)
    scenes._params(sim, 0.8, 0.7, 0.008, 0.0015)
    sim.initFlat(12)
    a = SphC(36, 30, 36, cx=12, cy=20, cz=18, r=3.5, density=2.5)
    b = SphC(36, 30, 36, cx=25, cy=22, cz=17, r=3.0, density=1.8)
    return sim, CompositeSolid([a, b])


BUILDERS = [lambda S, R: scenes.drop(S, R, sigma=0.012, gravity=0.0012), scenes.smoke, _odd, _wide, _pair]


def _state(sim, solid):
    from b200lbm.solid import spheres_of
    fields = {k: np.array(getattr(sim, k)) for k in ("phi", "rho", "ux", "uy", "uz", "f", "h", "tag")}
    return fields, [b.state() for b in spheres_of(solid)]


def _set_shape(sim, rows, zchunk):
    from b200lbm import _capi
    sim._sync()
    _capi.check(sim.handle, _capi.lib().lbm_set_fused_config(sim.handle, rows, zchunk))


@pytest.mark.parametrize("storage", ["f32", "f16", "bf16"])
def test_pipelined_equals_plain_alone(gpu, storage):
    SimS = functools.partial(gpu.Sim, storage=storage)
    for bi, bld in enumerate(BUILDERS):
        ref_sim, ref_sol = bld(SimS, gpu.RigidSphere)
        ref_sim.run_coupled(ref_sol, 9)
        for _ in range(3):  # the host-driven step as well
            scenes.substep(ref_sim, ref_sol)
        want = _state(ref_sim, ref_sol)
        for rows, zchunk in PIPE_SHAPES:
            sim, sol = bld(SimS, gpu.RigidSphere)
            _set_shape(sim, rows, zchunk)
            sim.run_coupled(sol, 9)
            for _ in range(3):
                scenes.substep(sim, sol)
            got = _state(sim, sol)
            for k in want[0]:
                assert np.array_equal(got[0][k], want[0][k]), (storage, bi, rows, zchunk, k)
            assert got[1] == want[1], (storage, bi, rows, zchunk)
            sim.close()
        ref_sim.close()


@pytest.mark.parametrize("storage", ["f32", "f16"])
def test_pipelined_batch_equals_alone(gpu, storage):
    SimS = functools.partial(gpu.Sim, storage=storage)
    ref = [bld(SimS, gpu.RigidSphere) for bld in BUILDERS]
    for sim, solid in ref:
        sim.run_coupled(solid, 10)
    mixed = [bld(SimS, gpu.RigidSphere) for bld in BUILDERS]
    with gpu.Batch(mixed) as batch:
        batch.set_config(6 | STAGED, 32)
        batch.run(4)
        batch.set_config(4 | STAGED, 16)
        batch.run(2, use_graph=False)
        batch.set_config(4 | COMPACT, 32)
        batch.run(2)
        batch.set_config(6 | ASYNC, 32)
        batch.run(2)
    for i, ((sim, solid), (rsim, rsolid)) in enumerate(zip(mixed, ref)):
        a, sa = _state(sim, solid)
        b, sb = _state(rsim, rsolid)
        for k in a:
            assert np.array_equal(a[k], b[k]), f"scene {i}: {k} differs"
        assert sa == sb, f"scene {i}: sphere state differs"


TMA = 0x1000
L2PF = 0x2000
# the two forms that use the scene's tensor maps: rows staged by tensor copies
# (TMA) and register loads behind tensor prefetches into L2 (L2PF)
TMA_SHAPES = ((6 | TMA, 32), (6 | TMA, 5), (6 | TMA, 9), (6 | TMA, 1), (6 | L2PF, 24), (6 | L2PF, 5),
              (6 | L2PF, 2), (6 | L2PF, 1))


def _tma16(SimC, SphC):
    """16 x 22 x 19: one x tile half outside the grid (its last two blocks
    arrive as zeros), y tiles that do not divide ny, a sphere."""
    sim = SimC(16, 22, 19)
    scenes._params(sim, 0.7, 0.75, 0.01, 0.001)
    sim.initFlat(7.5)
    return sim, SphC(16, 22, 19, cx=8.2, cy=12.5, cz=9.4, r=3.0, density=2.0)


def _tma48(SimC, SphC):
    """48 x 40 x 36, a falling sphere: two x tiles, the second partial."""
    sim = SimC(48, 40, 36)
    scenes._params(sim, 0.8, 0.7, 0.008, 0.0015)
    sim.initFlat(12)
    sol = SphC(48, 40, 36, cx=30.5, cy=24.0, cz=17.2, r=5.0, density=2.5)
    sol.vy = -0.03
    return sim, sol


def _tma64(SimC, SphC):
    from b200lbm import CompositeSolid
    sim = SimC(64, 26, 30)
    scenes._params(sim, 0.8, 0.7, 0.008, 0.0015)
    sim.initFlat(9)
    a = SphC(64, 26, 30, cx=20, cy=15, cz=14, r=3.5, density=2.5)
    b = SphC(64, 26, 30, cx=41, cy=17, cz=16, r=3.0, density=1.8)
    return sim, CompositeSolid([a, b])


TMA_BUILDERS = [_tma16, _tma48, _tma64]


@pytest.mark.parametrize("storage", ["f32", "f16", "bf16"])
def test_tma_equals_plain_alone(gpu, storage):
    """6 | LBM_FUSED_TMA (tensor-map copies of each plane's tile rows) and 6 |
    LBM_FUSED_L2PF (tensor prefetches of the rows two planes ahead into L2)
    give what the plain 4-row form gives, bit for bit, on grids with nx a
    multiple of 16; on others they run the compact form (and still agree)."""
    SimS = functools.partial(gpu.Sim, storage=storage)
    for bi, bld in enumerate(TMA_BUILDERS + [_odd]):
        ref_sim, ref_sol = bld(SimS, gpu.RigidSphere)
        _set_shape(ref_sim, 4, 32)
        ref_sim.run_coupled(ref_sol, 9)
        for _ in range(3):
            scenes.substep(ref_sim, ref_sol)
        want = _state(ref_sim, ref_sol)
        for rows, zchunk in TMA_SHAPES:
            sim, sol = bld(SimS, gpu.RigidSphere)
            _set_shape(sim, rows, zchunk)
            staged = sim.nx % 16 == 0
            assert sim.launch_shape() == (rows if staged else 6 | COMPACT), (storage, bi)
            sim.run_coupled(sol, 9)
            for _ in range(3):
                scenes.substep(sim, sol)
            got = _state(sim, sol)
            for k in want[0]:
                assert np.array_equal(got[0][k], want[0][k]), (storage, bi, rows, zchunk, k)
            assert got[1] == want[1], (storage, bi, rows, zchunk)
            sim.close()
        ref_sim.close()


@pytest.mark.parametrize("storage,form", [("f32", TMA), ("f16", TMA), ("f32", L2PF), ("bf16", L2PF)])
def test_tma_batch_equals_alone(gpu, storage, form):
    """A batch of scenes with tensor maps runs the TMA (or L2PF) form; a batch
    with one scene whose nx is not a multiple of 16 runs the compact form;
    both equal the scenes run alone."""
    SimS = functools.partial(gpu.Sim, storage=storage)
    for builders in (TMA_BUILDERS, TMA_BUILDERS + [_odd]):
        ref = [bld(SimS, gpu.RigidSphere) for bld in builders]
        for sim, solid in ref:
            sim.run_coupled(solid, 8)
        mixed = [bld(SimS, gpu.RigidSphere) for bld in builders]
        with gpu.Batch(mixed) as batch:
            batch.set_config(6 | form, 32)
            batch.run(4)
            batch.set_config(6 | form, 7)
            batch.run(2, use_graph=False)
            batch.run(2)
        for i, ((sim, solid), (rsim, rsolid)) in enumerate(zip(mixed, ref)):
            a, sa = _state(sim, solid)
            b, sb = _state(rsim, rsolid)
            for k in a:
                assert np.array_equal(a[k], b[k]), f"scene {i}: {k} differs"
            assert sa == sb, f"scene {i}: sphere state differs"
        for sim, _ in ref + mixed:
            sim.close()
