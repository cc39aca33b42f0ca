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
