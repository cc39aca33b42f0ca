"""The CUDA path against golden vectors of the reference's own code
(tests/golden/*.npz, made by tests/golden/make_golden.py from the reference's
src/*.js; see test_golden_cpu.py for how the oracle matches them bit for bit).

Bars, as in test_parity_gpu.py (the plain CUDA path computes in FP32 where the
reference computes in double and stores float32):
  * fresh / dead sets and tags: exact, given the reference's sphere state at
    the start of every step (the sphere is set from the golden trajectory);
  * phi, rho: rel-L2 <= 2e-5, Linf <= 2e-4 (1e-3 where the sphere crosses
    the interface: rise, drag, dam); u (the vector field): rel-L2
    <= 1e-2 and Linf <= 2e-2 of max|u| (u is a small difference of O(w_k)
    populations), or |du| <= 1e-7 where max|u| is below 5e-6;
  * sphere state after RigidSphere.step: within 1e-6 cells (cell units);
  * dead-cell impulse on identical fields: 1e-12 relative (FP64, summation
    order only); RG8 pack of identical phi: exact.
"""
import json
import os

import numpy as np
import pytest

from golden import scenarios
from scenes import field_err

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL_REL, TOL_INF = 2e-5, 2e-4
# scenes where the sphere crosses the interface: fresh cells are filled with
# averages of FP32 neighbours (src/sim.js:260-293), so single cells carry a
# larger error; rel-L2 keeps the tight bar
TOL_INF_CROSSING = 1e-3
CROSSING = ("rise", "drag", "dam")
TOL_REL_U, TOL_INF_U = 1e-2, 2e-2
TOL_SPHERE = 1e-6
U_ABS_FLOOR = 1e-7


@pytest.fixture(scope="module")
def gpu():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import b200lbm
    return b200lbm


def _load(name):
    return np.load(os.path.join(GOLDEN, f"{name}.npz"))


def _check_fields(tag, got, want, stride=1, tol_inf=TOL_INF):
    """got: full GPU fields; want: golden arrays (full or strided samples).

    u is compared as one vector field (ux, uy, uz stacked): its components can
    differ by orders of magnitude (cfg1 at step 1: |ux| ~ 6e-6, |uy| ~ 2e-4),
    and FP32 round-off (~1e-8 per step in u) would dominate a per-component
    relative norm of the small one.  Where max|u| itself is below
    U_ABS_FLOOR / TOL_INF_U the bar is |du| <= U_ABS_FLOOR."""
    for k in ("phi", "rho"):
        rel, linf = field_err(got[k][::stride], want[k])
        assert rel <= TOL_REL and linf <= tol_inf, f"{tag} {k}: rel {rel:.3e} linf {linf:.3e}"
    gu = np.concatenate([np.asarray(got[k][::stride], np.float64) for k in ("ux", "uy", "uz")])
    wu = np.concatenate([np.asarray(want[k], np.float64) for k in ("ux", "uy", "uz")])
    umax = np.abs(wu).max() or 1e-30
    rel, linf = field_err(gu, wu, norm=umax)
    if umax * TOL_INF_U >= U_ABS_FLOOR:
        assert rel <= TOL_REL_U and linf <= TOL_INF_U, f"{tag} u: rel {rel:.3e} linf {linf:.3e}"
    else:
        assert linf * umax <= U_ABS_FLOOR, f"{tag} u: |du| {linf * umax:.3e}"


@pytest.mark.parametrize("name", list(scenarios.PLAN))
def test_gpu_matches_reference_golden(name, gpu):
    g = _load(name)
    meta = json.loads(str(g["meta"]))
    sph = g["sphere"] if "sphere" in g else None

    def on_step(s, sim, sol):
        # the reference's sphere state at the start of step s
        if sol is not None and s > 1:
            for k, v in zip(scenarios.SPHERE_KEYS, sph[s - 2]):
                setattr(sol, k, float(v))

    rec = scenarios.run_scene(name, gpu.Sim, gpu.RigidSphere, on_step=on_step)
    stride = meta["sample_stride"] if meta["digest_only"] else 1
    for s in meta["checkpoints"]:
        got = {k: rec["fields"][(k, s)] for k in scenarios.FIELDS}
        key = (lambda k: f"sample_{k}_{s}") if meta["digest_only"] else (lambda k: f"{k}_{s}")
        want = {k: g[key(k)] for k in scenarios.FIELDS}
        _check_fields(f"{name} step {s}", got, want, stride,
                      TOL_INF_CROSSING if name in CROSSING else TOL_INF)
        assert np.array_equal(rec["fields"][("tag", s)][::stride], g[key("tag")]), (name, s)
    assert np.array_equal(np.concatenate(rec["fresh"]), g["fresh"]), name
    assert np.array_equal(np.concatenate(rec["dead"]), g["dead"]), name
    if sph is not None:
        drift = np.abs(np.array(rec["sphere"])[:, :3] - sph[:, :3]).max()
        assert drift <= TOL_SPHERE, (name, drift)


def test_gpu_phases_match_reference_golden(gpu):
    g = _load("phases")
    fields, sphere = scenarios.run_phases(gpu.Sim, gpu.RigidSphere)
    stride = scenarios.SAMPLE_STRIDE
    _check_fields("phases", fields, {k: g[f"sample_{k}"] for k in scenarios.FIELDS}, stride)
    assert np.array_equal(fields["tag"][::stride], g["sample_tag"])
    for k in ("gx", "gy", "gz", "lap"):
        rel, _ = field_err(fields[k][::stride], g[f"sample_{k}"])
        assert rel <= 1e-4, (k, rel)
    assert np.abs(sphere[:3] - g["sphere"][:3]).max() <= TOL_SPHERE


def test_gpu_absorb_and_pack_match_reference_golden(gpu):
    g = _load("absorb_pack")
    imp, dead = scenarios.run_absorb(gpu.Sim, gpu.RigidSphere)
    assert np.array_equal(dead, g["absorb_dead"])
    want = g["absorb_impulse"]
    assert np.all(np.abs(imp - want) <= 1e-12 * np.maximum(1.0, np.abs(want))), (imp, want)
    packed = scenarios.run_pack(gpu.Sim, gpu.RigidSphere, lambda sim: sim.packVolume())
    assert np.array_equal(packed, g["pack_bytes"])
