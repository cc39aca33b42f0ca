"""NaN/Inf watchdog (lbm_set_nan_watchdog).

The reference raises nothing on a numerical blow-up: NaN simply appears in
the fields (its macro update even turns a NaN density sum into 0.01,
src/sim.js:546).  The drop-in keeps that as the default and offers an opt-in
scan of phi, rho and u that turns a blow-up into LBM_ERR_NAN.  The blow-up is
made on the host: one fluid cell's phi is written as NaN through the field
mirror, and the next step spreads it.  No device fault is involved.
"""
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


def _scene(gpu, storage="f32"):
    sim = gpu.Sim(20, 16, 18, storage=storage)
    scenes._params(sim, 0.7, 0.75, 0.01, 0.001)
    sim.initFlat(7.5)
    return sim


def _poison(sim):
    i = sim.idx(9, 4, 8)  # a fluid cell below the waterline
    assert sim.tag[i] == 0
    sim.phi[i] = np.float32(np.nan)
    return i


def _first_bad(sim):
    bad = ~np.isfinite(sim.phi) | ~np.isfinite(sim.rho)
    for f in (sim.ux, sim.uy, sim.uz):
        bad |= ~np.isfinite(f)
    idx = np.flatnonzero(bad)
    return int(idx[0]) if idx.size else None


def test_off_by_default_like_the_reference(gpu):
    sim = _scene(gpu)
    _poison(sim)
    sim.step(None)
    sim.step(None)
    assert _first_bad(sim) is not None


@pytest.mark.parametrize("storage", ["f32", "f16", "f64"])
def test_step_reports_the_first_non_finite_cell(gpu, storage):
    from b200lbm import _capi
    sim = _scene(gpu, storage)
    sim.setNanWatchdog(1)
    sim.step(None)
    sim.step(None)  # finite fields: no error
    assert _first_bad(sim) is None
    _poison(sim)
    with pytest.raises(_capi.LbmError) as err:
        sim.step(None)
    assert err.value.code == _capi.ERR_NAN, err.value
    first = _first_bad(sim)  # the step completed: the mirror shows its fields
    assert first is not None
    x, y, z = first % sim.nx, (first // sim.nx) % sim.ny, first // (sim.nx * sim.ny)
    assert f"cell {first} (x {x}, y {y}, z {z})" in str(err.value), err.value


def test_every_n_steps_and_off_again(gpu):
    from b200lbm import _capi
    sim = _scene(gpu)
    sim.setNanWatchdog(3)
    sim.step(None)
    _poison(sim)
    sim.step(None)  # 2 steps since the watchdog was set: no scan yet
    with pytest.raises(_capi.LbmError) as err:
        sim.step(None)  # the third step scans
    assert err.value.code == _capi.ERR_NAN
    sim.setNanWatchdog(0)
    sim.step(None)  # off: the fields stay non-finite and nothing is raised
    assert _first_bad(sim) is not None
    with pytest.raises(_capi.LbmError):
        sim.setNanWatchdog(-1)


def test_coupled_run_and_batch_report_it(gpu):
    from b200lbm import Batch, RigidSphere, _capi
    sim = _scene(gpu)
    sol = RigidSphere(20, 16, 18, cx=14, cy=10, cz=12, r=2.5, density=1.6)  # clear of the poisoned cell
    sim.setNanWatchdog(4)
    sim.run_coupled(sol, 4)  # finite: scanned at the end, no error
    _poison(sim)
    with pytest.raises(_capi.LbmError) as err:
        sim.run_coupled(sol, 4)
    assert err.value.code == _capi.ERR_NAN

    good = _scene(gpu)
    good.setNanWatchdog(2)
    bad = _scene(gpu)
    bad.setNanWatchdog(2)
    _poison(bad)
    bad._sync()
    with Batch([(good, None), (bad, None)]) as batch:
        with pytest.raises(_capi.LbmError) as err:
            batch.run(2)
    assert "non-finite" in str(err.value)
    assert _first_bad(good) is None and _first_bad(bad) is not None
