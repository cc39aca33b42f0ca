"""Batches (lbm_batch_*): several scenes of uneven sizes advanced together by
one persistent fused launch per step, with and without CUDA-graph replay,
give every scene exactly the results of running it alone (Sim.run_coupled):
fields, sphere states and RG8 frames bit for bit -- the per-cell arithmetic
does not depend on which CTA or launch processes a tile, and every reduction
has a fixed order."""
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


def _odd(SimC, SphC):
    """33 x 17 x 29: rows start off the 8-cell blocks, partial tiles, no solid."""
    sim = SimC(33, 17, 29)
    scenes._params(sim, 0.7, 0.75, 0.01, 0.001)
    sim.initFlat(8.5)
    return sim, None


def _pair(SimC, SphC):
    """Two spheres (a composite solid) in 36 x 30 x 36."""
    from b200lbm import CompositeSolid
    sim = SimC(36, 30, 36)
    scenes._params(sim, 0.8, 0.7, 0.008, 0.0015)
    sim.initFlat(12)
    a = SphC(36, 30, 36, cx=12, cy=20, cz=18, r=3.5, density=2.5)
    b = SphC(36, 30, 36, cx=25, cy=22, cz=17, r=3.0, density=1.8)
    return sim, CompositeSolid([a, b])


BUILDERS = [scenes.drop, scenes.smoke, _odd, _pair]


def _build(gpu):
    return [bld(gpu.Sim, gpu.RigidSphere) for bld in BUILDERS]


def _state(sim, solid):
    from b200lbm.solid import spheres_of
    fields = {k: np.array(getattr(sim, k)) for k in ("phi", "rho", "ux", "uy", "uz", "f", "h", "tag")}
    return fields, [b.state() for b in spheres_of(solid)]


@pytest.mark.parametrize("use_graph,nsteps,every", [(True, 24, 4), (True, 17, 4), (False, 13, 5),
                                                    (True, 13, 5)])
def test_batch_equals_scenes_alone(gpu, use_graph, nsteps, every):
    """Graph replay (2-step chunks, frames between chunks), a trailing eager
    step, eager mode, and an odd frame cadence (which runs eagerly)."""
    alone = _build(gpu)
    want = []
    for sim, solid in alone:
        frames = sim.run_coupled(solid, nsteps, frame_every=every)
        want.append((frames, _state(sim, solid)))
    mixed = _build(gpu)
    with gpu.Batch(mixed) as batch:
        got = batch.run(nsteps, frame_every=every, use_graph=use_graph)
        assert batch.launch_count() == nsteps
    for i, ((sim, solid), (wframes, (wf, ws))) in enumerate(zip(mixed, want)):
        assert np.array_equal(got[i], wframes), f"scene {i}: frames differ"
        gf, gs = _state(sim, solid)
        for k in wf:
            assert np.array_equal(gf[k], wf[k]), f"scene {i}: {k} differs"
        assert gs == ws, f"scene {i}: sphere state differs"


def test_batch_continues_across_runs_and_configs(gpu):
    """Two runs with different tile shapes continue a scene exactly like one run."""
    ref = _build(gpu)
    for sim, solid in ref:
        sim.run_coupled(solid, 10)
    mixed = _build(gpu)
    with gpu.Batch(mixed) as batch:
        batch.set_config(8, 16)
        batch.run(4)
        batch.run(2)  # the cached graph is replayed
        batch.set_config(2, 7)
        batch.run(4)
        ms = batch.time_fused(4, 32, reps=2)
        assert ms > 0
    for (sim, solid), (rsim, rsolid) in zip(mixed, ref):
        a, sa = _state(sim, solid)
        b, sb = _state(rsim, rsolid)
        for k in ("phi", "rho", "ux", "f"):
            assert np.array_equal(a[k], b[k]), k
        assert sa == sb


@pytest.mark.parametrize("storage", ["f16", "bf16"])
def test_reduced_storage_independent_of_tile_shape(gpu, storage):
    """Reduced storage has a staged form of the fused kernel (4 | STAGED:
    populations brought in by bulk asynchronous copies) beside the plain 2, 4
    and 8 row forms; a scene stepped through all of them, in a batch, ends bit
    for bit where the same scene run alone with the default shape ends."""
    import functools
    SimS = functools.partial(gpu.Sim, storage=storage)
    shapes = ((8, 16), (4 | 0x100, 32), (2, 7), (4 | 0x100, 5), (4, 9))
    ref = [bld(SimS, gpu.RigidSphere) for bld in BUILDERS]
    for sim, solid in ref:
        sim.run_coupled(solid, 3 * len(shapes))
    mixed = [bld(SimS, gpu.RigidSphere) for bld in BUILDERS]
    with gpu.Batch(mixed) as batch:
        for rows, zchunk in shapes:
            batch.set_config(rows, zchunk)
            batch.run(3, use_graph=False)
    for i, ((sim, solid), (rsim, rsolid)) in enumerate(zip(mixed, ref)):
        a, sa = _state(sim, solid)
        b, sb = _state(rsim, rsolid)
        for k in a:
            assert np.array_equal(a[k], b[k]), f"scene {i}: {k} differs"
        assert sa == sb, f"scene {i}: sphere state differs"
