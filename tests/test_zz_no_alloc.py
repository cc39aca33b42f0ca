"""The allocation-free dead-cell sweep, lbm_absorb_dead_cells_noalloc, checked
through the C ABI against the handle-based lbm_absorb_dead_cells.

That entry point serves callers that cannot allocate device memory where they
need the sweep -- an engine that hands out all device memory from its own pool,
or a host whose allocator belongs to another runtime.  It takes the fields as
device arrays the caller owns and keeps its scratch in one fixed array inside
the library, shared by every call.  Two calls in a row, a large sphere and then
a small one on different fields, check that the second call does not pick up
what the first left in that array.  The file is named to be collected last; it
passes alone in a fresh process as well.
"""
import ctypes as C

import numpy as np
import pytest

import scenes

pytestmark = pytest.mark.gpu

TOL = 1e-12  # relative, the bar of the FP64 impulse parity tests
KEYS = ("Fx", "Fy", "Fz", "Tx", "Ty", "Tz")


@pytest.fixture(scope="module")
def gpu():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import b200lbm
    return b200lbm


def _large(SimC, SphC):
    """110^3 pool for a sphere whose search box nearly fills the array."""
    sim = SimC(110, 110, 110)
    scenes._params(sim, 0.7, 0.7, 0.012, 0.00135)
    sim.initFlat(30)
    return sim, SphC(110, 110, 110, cx=55, cy=55, cz=55, r=10, density=1.6)


def _scene(gpu, centre, r, seed, build=scenes.bench):
    """A scene with random fields and a sphere placed on them: the first retag
    turns every cell of the sphere FLUID -> SOLID (all of them dead)."""
    sim, sol = build(gpu.Sim, gpu.RigidSphere)
    rng = np.random.default_rng(seed)
    sim.phi[:] = rng.uniform(-0.1, 1.1, sim.n).astype(np.float32)
    for name in ("ux", "uy", "uz"):
        getattr(sim, name)[:] = rng.normal(0, 0.02, sim.n).astype(np.float32)
    sol.cx, sol.cy, sol.cz = centre
    sol.setRadius(r)
    sim.retagCells(sol)
    return sim, sol


def _handle_based(gpu, sim, sol):
    from b200lbm._capi import check, lib
    from b200lbm.solid import impulse_array, to_c_array
    out = impulse_array(1)
    check(sim.handle, lib().lbm_absorb_dead_cells(sim.handle, to_c_array([sol]), 1, out))
    return np.array([getattr(out[0], k) for k in KEYS])


def _no_alloc(gpu, sim, sol):
    import torch
    from b200lbm._capi import OK, lib
    from b200lbm.solid import to_c_array
    dev = torch.device("cuda", 0)
    arrays = [torch.from_numpy(np.array(getattr(sim, name))).to(dev)
              for name in ("tag", "tagPrev", "phi", "ux", "uy", "uz")]
    out = torch.full((6,), float("nan"), dtype=torch.float64, device=dev)
    err = C.create_string_buffer(256)
    stream = torch.cuda.current_stream(dev)
    rc = lib().lbm_absorb_dead_cells_noalloc(
        sim.nx, sim.ny, sim.nz, sim.rhoL, sim.rhoG, *[a.data_ptr() for a in arrays],
        to_c_array([sol]), 1, out.data_ptr(), stream.cuda_stream, err, len(err))
    assert rc == OK, err.value.decode()
    stream.synchronize()
    return out.cpu().numpy()


def test_no_alloc_matches_handle_based_two_calls(gpu):
    cases = [((19.3, 13.6, 20.4), 8.5, 11), ((9.7, 20.2, 27.1), 3.2, 12)]
    for n, (centre, r, seed) in enumerate(cases):
        sim, sol = _scene(gpu, centre, r, seed)
        tag, prev = np.array(sim.tag), np.array(sim.tagPrev)
        assert np.count_nonzero((tag == 1) & (prev == 0)) > 100
        want = _handle_based(gpu, sim, sol)
        got = _no_alloc(gpu, sim, sol)
        assert np.all(np.isfinite(got)), (n, got)
        for k, a, b in zip(KEYS, got, want):
            assert abs(a - b) <= TOL * max(1.0, abs(b)), (n, k, a, b)
        sim.close()


def test_no_alloc_near_capacity(gpu):
    """A sphere of radius 49 in a 110^3 grid: its search box is 101^3 =
    1,030,301 cells (98% of the 2^20 limit) with ~490,000 dead cells, then a
    small sphere on other fields right after it."""
    cases = [((55.3, 55.6, 54.8), 49.0, 21, _large), ((20.6, 9.4, 19.9), 4.1, 22, scenes.bench)]
    for n, (centre, r, seed, build) in enumerate(cases):
        sim, sol = _scene(gpu, centre, r, seed, build)
        tag, prev = np.array(sim.tag), np.array(sim.tagPrev)
        ndead = np.count_nonzero((tag == 1) & (prev == 0))
        assert ndead > (400000 if n == 0 else 100), ndead
        want = _handle_based(gpu, sim, sol)
        got = _no_alloc(gpu, sim, sol)
        assert np.all(np.isfinite(got)), (n, got)
        for k, a, b in zip(KEYS, got, want):
            assert abs(a - b) <= TOL * max(1.0, abs(b)), (n, k, a, b)
        sim.close()


def test_no_alloc_rejects_oversized_box(gpu):
    import torch
    from b200lbm._capi import ERR_CAPACITY, LbmSphere, lib
    dev = torch.device("cuda", 0)
    dummy = torch.zeros(16, dtype=torch.float64, device=dev)
    sph = (LbmSphere * 1)()
    sph[0].cx = sph[0].cy = sph[0].cz = 100.0
    sph[0].r = 60.0  # box of ~121^3 cells > 2^20
    err = C.create_string_buffer(256)
    p = dummy.data_ptr()
    rc = lib().lbm_absorb_dead_cells_noalloc(200, 200, 200, 1.0, 0.05, p, p, p, p, p, p, sph, 1, p,
                                             None, err, len(err))
    assert rc == ERR_CAPACITY
    assert b"at most 1048576" in err.value
