"""lbm_init_profile (Sim.initProfile) against the host pattern it replaces:
initFlat, then phi, phiPrev and h = w7 phi written cell by cell from the host,
then seedHydrostatic (the dam preset's pattern, src/worker.js:57-73; the
served scenes' pool below the interface).  Every field bit for bit, for every
storage form that holds FP32 values or less, and the next steps too.  The
FP64 form keeps the profile's doubles unrounded (as its initFlat does), where
the host pattern goes through the float32 field upload; it is checked against
the profile itself."""
import numpy as np
import pytest

import scenes

pytestmark = pytest.mark.gpu

FIELDS = ("phi", "phiPrev", "rho", "ux", "uy", "uz", "f", "h", "tag", "tagPrev")


@pytest.fixture(scope="module")
def gpu():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import b200lbm
    return b200lbm


@pytest.mark.parametrize("storage", ["f32", "f16", "bf16"])
@pytest.mark.parametrize("dims,level", [((40, 33, 24), 13.3), ((67, 52, 45), 24.7)])
def test_profile_equals_host_writes(gpu, storage, dims, level):
    from b200lbm import workloads
    sims = []
    for mode in ("host", "device"):
        sim = gpu.Sim(*dims, storage=storage)
        for k, v in workloads.PHYSICS.items():
            setattr(sim, k, v)
        if mode == "host":
            sim.initFlat(level)
            workloads.pool_below_host(sim, level, workloads.PHYSICS["W"])
        else:
            workloads.pool_below(sim, level, workloads.PHYSICS["W"])
        sims.append(sim)
    a, b = sims
    for k in FIELDS:
        assert np.array_equal(np.asarray(getattr(a, k)), np.asarray(getattr(b, k))), (storage, k)
    nx, ny, nz = dims
    sa = gpu.RigidSphere(nx, ny, nz, cx=nx / 2, cy=ny * 0.7, cz=nz / 2, r=4.2, density=2.0)
    sb = gpu.RigidSphere(nx, ny, nz, cx=nx / 2, cy=ny * 0.7, cz=nz / 2, r=4.2, density=2.0)
    for _ in range(5):
        scenes.substep(a, sa)
        scenes.substep(b, sb)
    for k in ("phi", "rho", "f", "h"):
        assert np.array_equal(np.asarray(getattr(a, k)), np.asarray(getattr(b, k))), (storage, "stepped", k)
    assert sa.state() == sb.state()
    a.close()
    b.close()


def test_profile_f64_keeps_doubles(gpu):
    from b200lbm import workloads
    nx, ny, nz = 24, 30, 20
    sim = gpu.Sim(nx, ny, nz, storage="f64")
    for k, v in workloads.PHYSICS.items():
        setattr(sim, k, v)
    workloads.pool_below(sim, 11.6, workloads.PHYSICS["W"])
    col = workloads.pool_column(ny, 11.6, workloads.PHYSICS["W"])
    want = np.broadcast_to(col[None, :, None], (nz, ny, nx)).reshape(-1)
    assert np.array_equal(sim.field64("phi"), want)
    sim.close()


def test_profile_rejects_wrong_length(gpu):
    sim = gpu.Sim(16, 20, 16)
    with pytest.raises(ValueError):
        sim.initProfile(np.zeros(19))
    sim.close()
