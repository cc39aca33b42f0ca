"""Grids whose population offsets exceed 2^31 elements (more than ~76.7 M
cells) run the fused step, with 64-bit population offsets.  A 64 x 64 x 20000
flat pool (81.9 M cells) with no solid is the same in every z plane away from
the two end walls, and influence travels one plane per step, so after 5 steps
a plane near the bottom (small offsets) and one near the top (offsets beyond
2^31) must hold the same phi, rho and u bit for bit."""
import ctypes as C

import numpy as np
import pytest

import scenes

pytestmark = pytest.mark.gpu

NX, NY, NZ, STEPS = 64, 64, 20000, 5


@pytest.fixture(scope="module")
def gpu():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import b200lbm
    return b200lbm


def test_fused_step_beyond_32bit_population_offsets(gpu):
    from b200lbm import _capi
    L = _capi.lib()
    sim = gpu.Sim(NX, NY, NZ)
    assert sim.n * 28 > 2 ** 31
    scenes._params(sim, 0.7, 0.75, 0.01, 0.001)
    sim.initFlat(NY / 2 + 0.25)
    sim._sync()
    h = sim.handle
    _capi.check(h, L.lbm_fused_timing(h, 1))
    sim.run_coupled(None, STEPS)
    ms, n = C.c_double(), C.c_int64()
    _capi.check(h, L.lbm_fused_timing_query(h, C.byref(ms), C.byref(n)))
    _capi.check(h, L.lbm_fused_timing(h, 0))
    assert n.value == STEPS  # the fused kernel ran (no fallback to the phase path)
    plane = NX * NY
    lo, hi = STEPS + 3, NZ - STEPS - 4
    assert (hi * plane) * 28 > 2 ** 31
    for name in ("phi", "rho", "ux", "uy", "uz"):
        a = np.asarray(getattr(sim, name))
        assert np.all(np.isfinite(a)), name
        assert np.array_equal(a[lo * plane:(lo + 1) * plane], a[hi * plane:(hi + 1) * plane]), name
    sim.close()
