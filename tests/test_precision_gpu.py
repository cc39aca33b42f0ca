"""Error bars of the reduced storage forms, under test.

Populations stored as FP16 or BF16 offsets f - w_k, h - w7_k phi (all
arithmetic FP32) against the FP64 storage form -- the GPU error reference,
itself held to the FP64 oracle at 1e-10 (tests/test_parity_gpu.py) -- on two
scenes, through the timed path (Sim.run_coupled, one tick per call so the
trajectory is compared at every tick):

  * the drop preset (src/worker.js:23-53, sigma 0.012, g 0.0012), 300 ticks:
    the sphere falls 2.9 cells through the interface, so the moving-wall
    term, fresh and dead cells and the FP64 sphere integration all act;
  * the 256^3 benchmark scene scaled to 64^3, 200 ticks.

Asserted per form: rel-L2 and L-inf of phi and rho, of u as one vector field
(L-inf over max|u|), the largest sphere-centre difference over the run, and
the relative difference of the FP64 sums of rho and phi (mass and phase)
from the FP64 run's.  Bars are about 2-3x the values measured on a B200
(written beside each); FP32 storage is held to the same table as a check of
the harness.  A second test pins every field bit for bit to committed SHA-256
digests (tests/golden/device_digests.json, made by
tests/golden/make_device_digests.py), so a change of the FP16 / BF16 encode
or of the arithmetic that stays inside these bars still fails.
"""
import functools
import json
import os
import sys

import numpy as np
import pytest

import scenes

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))

# scene -> storage -> bars: (phi rel, phi inf, rho rel, rho inf, u rel, u inf/umax,
#                            sphere drift [cells], mass vs FP64, phase vs FP64)
# measured (drop, 300 ticks): f32 2.3e-5 3.3e-4 6.3e-7 1.4e-6 8.4e-5 8.5e-5 2.4e-6 5.6e-7 2.3e-8
#                             f16 6.2e-5 6.4e-4 4.0e-6 1.0e-5 7.6e-4 2.5e-4 1.0e-4 3.4e-6 2.5e-6
#                             bf16 1.8e-4 1.6e-3 3.7e-5 7.5e-5 8.9e-3 4.2e-3 7.6e-4 3.3e-5 9.7e-6
# measured (64^3, 200 ticks): f32 1.0e-5 1.2e-4 1.0e-6 2.2e-6 5.6e-3 3.3e-3 0 9.4e-7 1.6e-7
#                             f16 1.2e-5 1.4e-4 9.5e-7 2.5e-6 6.5e-3 3.9e-3 0 8.6e-7 2.9e-7
#                             bf16 1.2e-5 1.3e-4 6.0e-7 2.6e-6 1.5e-2 7.5e-3 0 1.7e-7 5.4e-8
BARS = {
    "drop300": {
        "f32": (6e-5, 1e-3, 2e-6, 4e-6, 3e-4, 3e-4, 1e-5, 2e-6, 1e-7),
        "f16": (1.5e-4, 1.5e-3, 1e-5, 3e-5, 2e-3, 8e-4, 3e-4, 1e-5, 8e-6),
        "bf16": (5e-4, 4e-3, 1e-4, 2e-4, 2.5e-2, 1.2e-2, 2e-3, 1e-4, 3e-5),
    },
    "cfg2_64_200": {
        "f32": (3e-5, 3e-4, 3e-6, 6e-6, 1.5e-2, 1e-2, 1e-6, 3e-6, 5e-7),
        "f16": (3e-5, 3e-4, 3e-6, 6e-6, 1.5e-2, 1e-2, 1e-6, 3e-6, 1e-6),
        "bf16": (3e-5, 3e-4, 2e-6, 7e-6, 4e-2, 2e-2, 1e-6, 1e-6, 2e-7),
    },
}
SCENES = {
    "drop300": (lambda S, R: scenes.drop(S, R, sigma=0.012, gravity=0.0012), 300),
    "cfg2_64_200": (lambda S, R: scenes.cfg2(S, R, n=64), 200),
}


@pytest.fixture(scope="module")
def gpu():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import b200lbm
    return b200lbm


def _run(gpu, build, steps, storage):
    sim, sol = build(functools.partial(gpu.Sim, storage=storage), gpu.RigidSphere)
    traj = []
    for _ in range(steps):
        sim.run_coupled(sol, 1)
        traj.append((sol.cx, sol.cy, sol.cz))
    f = {k: sim.field64(k) for k in ("phi", "rho", "ux", "uy", "uz")}
    sums = (float(np.sum(f["rho"])), float(np.sum(f["phi"])))
    sim.close()
    return f, np.array(traj), sums


@pytest.fixture(scope="module")
def reference_runs(gpu):
    return {name: _run(gpu, build, steps, "f64") for name, (build, steps) in SCENES.items()}


@pytest.mark.parametrize("scene", list(SCENES))
@pytest.mark.parametrize("storage", ["f32", "f16", "bf16"])
def test_storage_form_error_bars(gpu, reference_runs, scene, storage):
    build, steps = SCENES[scene]
    ref, tref, sref = reference_runs[scene]
    got, tgot, sgot = _run(gpu, build, steps, storage)
    b = BARS[scene][storage]
    meas = []
    for i, k in enumerate(("phi", "rho")):
        d = got[k] - ref[k]
        rel = np.linalg.norm(d) / np.linalg.norm(ref[k])
        inf = np.abs(d).max()
        meas += [rel, inf]
        assert rel <= b[2 * i] and inf <= b[2 * i + 1], (scene, storage, k, rel, inf)
    u = np.concatenate([got["ux"], got["uy"], got["uz"]])
    uref = np.concatenate([ref["ux"], ref["uy"], ref["uz"]])
    rel = np.linalg.norm(u - uref) / np.linalg.norm(uref)
    inf = np.abs(u - uref).max() / np.abs(uref).max()
    drift = np.abs(tgot - tref).max()
    mass = abs(sgot[0] - sref[0]) / abs(sref[0])
    phase = abs(sgot[1] - sref[1]) / abs(sref[1])
    meas += [rel, inf, drift, mass, phase]
    print(scene, storage, " ".join(f"{v:.2e}" for v in meas))
    assert rel <= b[4] and inf <= b[5], (scene, storage, "u", rel, inf)
    assert drift <= b[6], (scene, storage, "sphere drift", drift)
    assert mass <= b[7] and phase <= b[8], (scene, storage, "sums", mass, phase)
    if scene == "drop300":
        assert np.abs(tref[-1] - tref[0]).max() > 2.5  # the sphere moved


def test_fields_match_committed_digests(gpu):
    """Every field after fixed runs, in every storage form, bit for bit as
    recorded in tests/golden/device_digests.json."""
    sys.path.insert(0, os.path.join(HERE, "golden"))
    import make_device_digests as mdd
    want = json.load(open(os.path.join(HERE, "golden", "device_digests.json")))
    for name, (build, steps) in mdd.cases().items():
        for st in mdd.STORAGES:
            got = mdd.digest_run(build, steps, st)
            assert got == want[f"{name}/{st}"], (name, st, [k for k in got if got[k] != want[f"{name}/{st}"][k]])
