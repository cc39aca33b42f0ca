"""Page-locked frame buffers (lbm_host_alloc / Sim.frameBuffer): packVolume
into one gives the same bytes as into a plain numpy buffer, frame after frame,
and the memory stays valid while any view of the array is alive."""
import gc

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


def test_pinned_frames_match_pageable(gpu):
    sim, solid = scenes.drop(gpu.Sim, gpu.RigidSphere)
    pinned = sim.frameBuffer()
    assert pinned.dtype == np.uint8 and pinned.size == 2 * sim.n and pinned.flags.c_contiguous
    view = pinned[: sim.n]  # a view keeps the block alive on its own
    del pinned
    gc.collect()
    for _ in range(3):
        for _ in range(4):
            sim.step(solid)
            solid.absorbDeadCells(sim)
            solid.step(1.0, sim.gravity)
        plain = sim.packVolume()
        got = sim.packVolume(sim.frameBuffer())
        assert np.array_equal(got, plain)
    buf = sim.frameBuffer()
    sim.packVolume(buf)
    assert np.array_equal(buf[: sim.n], sim.packVolume()[: sim.n])
    assert view.size == sim.n and int(view.sum()) >= 0  # still readable


def test_async_frames_match_sync(gpu):
    """packVolumeAsync frames, taken while later steps are already queued, are
    the frames packVolume gives at the same steps (two runs of one scene)."""
    want = []
    sim, solid = scenes.drop(gpu.Sim, gpu.RigidSphere)
    for _ in range(5):
        for _ in range(3):
            sim.step(solid)
            solid.absorbDeadCells(sim)
            solid.step(1.0, sim.gravity)
        want.append(sim.packVolume().copy())
    sim2, solid2 = scenes.drop(gpu.Sim, gpu.RigidSphere)
    bufs = [sim2.frameBuffer() for _ in range(5)]
    for f in range(5):
        for _ in range(3):
            sim2.step(solid2)
            solid2.absorbDeadCells(sim2)
            solid2.step(1.0, sim2.gravity)
        sim2.packVolumeAsync(bufs[f])
    sim2.waitFrames()
    for f in range(5):
        assert np.array_equal(bufs[f], want[f]), f


SHAPES = ((4, 32), (0x406, 32), (0x806, 9), (0x104, 7), (2, 5))


def _set_shape(sim, rows, zchunk):
    from b200lbm import _capi
    sim._sync()
    _capi.check(sim.handle, _capi.lib().lbm_set_fused_config(sim.handle, rows, zchunk))


def _odd_falling(SimC, SphC):
    """35 x 21 x 26 (partial tiles, rows off the 8-cell blocks) with a sphere
    moving down through the interface: SOLID cells, fresh and dead cells."""
    sim = SimC(35, 21, 26)
    scenes._params(sim, 0.7, 0.75, 0.01, 0.001)
    sim.initFlat(8.5)
    sol = SphC(35, 21, 26, cx=16.3, cy=12.2, cz=12.7, r=3.6, density=2.5)
    sol.vy = -0.03
    return sim, sol


@pytest.mark.parametrize("storage", ["f32", "f16", "bf16", "f64"])
def test_fused_pack_equals_pack(gpu, storage):
    """The RG8 volume written by the fused step on a frame step (stepFrame,
    and run_coupled with frames) is byte for byte packVolume after the step,
    for every launch form, with SOLID, wall and end-plane cells; the fields
    are those of plain steps."""
    import functools
    SimS = functools.partial(gpu.Sim, storage=storage)
    ref, rsol = _odd_falling(SimS, gpu.RigidSphere)
    want = []
    for t in range(6):
        scenes.substep(ref, rsol)
        want.append(ref.packVolume().copy())
    assert any((w[1::2] == 255).any() for w in want)  # SOLID cells in the frames
    dref, dsol = _odd_falling(SimS, gpu.RigidSphere)  # the device-resident loop, one step per call
    want_dev = []
    for t in range(6):
        dref.run_coupled(dsol, 1)
        want_dev.append(dref.packVolume().copy())
    dref.close()
    shapes = SHAPES if storage != "f64" else ((4, 32), (2, 5), (8, 16))
    for rows, zchunk in shapes:
        sim, sol = _odd_falling(SimS, gpu.RigidSphere)
        _set_shape(sim, rows, zchunk)
        bufs = [sim.frameBuffer(), sim.frameBuffer()]
        for t in range(6):
            out = bufs[t % 2]
            sim.waitFrames()
            sim.stepFrame(sol, out)
            sol.absorbDeadCells(sim)
            sol.step(1.0, sim.gravity)
            sim.waitFrames()
            assert np.array_equal(out, want[t]), (storage, hex(rows), zchunk, t)
        for k in ("phi", "rho", "f", "h", "tag"):
            assert np.array_equal(np.asarray(getattr(sim, k)), np.asarray(getattr(ref, k))), (storage, hex(rows), k)
        sim.close()
        # the device-resident loop with frames every 2 steps
        sim, sol = _odd_falling(SimS, gpu.RigidSphere)
        _set_shape(sim, rows, zchunk)
        frames = sim.run_coupled(sol, 6, frame_every=2)
        for j in range(3):
            assert np.array_equal(frames[j], want_dev[2 * j + 1]), (storage, hex(rows), "run_coupled", j)
        sim.close()
    ref.close()


def _falling48(SimC, SphC):
    """48 x 21 x 26: nx a multiple of 16 (the tensor-map forms run), the last
    x tile partial, a sphere moving down through the interface."""
    sim = SimC(48, 21, 26)
    scenes._params(sim, 0.7, 0.75, 0.01, 0.001)
    sim.initFlat(8.5)
    sol = SphC(48, 21, 26, cx=20.3, cy=12.2, cz=12.7, r=3.6, density=2.5)
    sol.vy = -0.03
    return sim, sol


@pytest.mark.parametrize("storage", ["f32", "f16"])
def test_fused_pack_tensor_map_forms(gpu, storage):
    """On a scene with tensor maps, the frame-step instances of the TMA-staged
    form (6 | 0x1000) and of the L2-prefetch form (6 | 0x2000) write, byte
    for byte, packVolume after the step, and the fields of plain steps."""
    import functools
    SimS = functools.partial(gpu.Sim, storage=storage)
    ref, rsol = _falling48(SimS, gpu.RigidSphere)
    _set_shape(ref, 4, 32)
    want = []
    for t in range(6):
        scenes.substep(ref, rsol)
        want.append(ref.packVolume().copy())
    for rows, zchunk in ((0x1006, 32), (0x2006, 24), (0x2006, 5), (0x2006, 3)):
        sim, sol = _falling48(SimS, gpu.RigidSphere)
        _set_shape(sim, rows, zchunk)
        assert sim.launch_shape() == rows
        bufs = [sim.frameBuffer(), sim.frameBuffer()]
        for t in range(6):
            out = bufs[t % 2]
            sim.waitFrames()
            sim.stepFrame(sol, out)
            sol.absorbDeadCells(sim)
            sol.step(1.0, sim.gravity)
            sim.waitFrames()
            assert np.array_equal(out, want[t]), (storage, hex(rows), zchunk, t)
        for k in ("phi", "rho", "f", "h", "tag"):
            assert np.array_equal(np.asarray(getattr(sim, k)), np.asarray(getattr(ref, k))), (storage, hex(rows), k)
        sim.close()
    ref.close()
