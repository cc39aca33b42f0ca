"""Bounded device waits of the fused step.

The staged forms of the fused kernel (tile shapes 4 | LBM_FUSED_STAGED and
6 | LBM_FUSED_TMA) wait on an mbarrier for each plane's bulk or tensor copy.  Every
such wait is bounded: when it runs out the tile stops, the step is abandoned,
the library returns LBM_ERR_TIMEOUT and the fault record holds location code
90.  The test makes the wait run out by withholding the copy it waits for
(lbm_test_withhold_stage_copy), so nothing faults or hangs, and then shows
the handle and the CUDA context still work: the same scene re-initialised
steps bit for bit like a fresh one.
"""
import ctypes as C

import numpy as np
import pytest

import scenes

pytestmark = pytest.mark.gpu

FAULT_STAGE_WAIT = 90
STAGED = 0x100
TMA = 0x1000


@pytest.fixture(scope="module")
def gpu():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import b200lbm
    return b200lbm


def _scene(gpu, storage):
    sim = gpu.Sim(16, 16, 16, storage=storage)
    scenes._params(sim, 0.7, 0.75, 0.01, 0.001)
    sim.initFlat(7.5)
    return sim


@pytest.mark.parametrize("storage,shape", [("f16", 4 | STAGED), ("bf16", 4 | STAGED), ("f32", 6 | TMA),
                                           ("f16", 6 | TMA)])
def test_withheld_copy_times_out_and_handle_recovers(gpu, storage, shape):
    from b200lbm import _capi
    L = _capi.lib()
    sim = _scene(gpu, storage)
    sim._sync()
    h = sim.handle
    _capi.check(h, L.lbm_set_fused_config(h, shape, 32))
    assert sim.launch_shape() == shape
    rec = (C.c_int64 * 4)()
    _capi.check(h, L.lbm_fault_record(h, rec))  # clear any earlier record

    _capi.check(h, L.lbm_test_withhold_stage_copy(h, 1))
    with pytest.raises(_capi.LbmError) as err:
        sim.run_coupled(None, 1)
    assert err.value.code == _capi.ERR_TIMEOUT, err.value
    _capi.check(h, L.lbm_fault_record(h, rec))
    assert rec[0] == FAULT_STAGE_WAIT, list(rec)
    _capi.check(h, L.lbm_test_withhold_stage_copy(h, 0))
    assert L.lbm_synchronize(h) == _capi.OK  # the status was cleared when reported

    sim.initFlat(7.5)
    sim.run_coupled(None, 6)
    fresh = _scene(gpu, storage)
    fresh._sync()
    _capi.check(fresh.handle, L.lbm_set_fused_config(fresh.handle, shape, 32))
    fresh.run_coupled(None, 6)
    for k in ("phi", "rho", "ux", "f", "h"):
        a, b = np.array(getattr(sim, k)), np.array(getattr(fresh, k))
        assert np.all(np.isfinite(np.asarray(a, np.float64))), k
        assert np.array_equal(a, b), k
