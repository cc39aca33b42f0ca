"""The Node-API addon driving the CUDA step on the GPU, through the C
stand-in for Node (tests/napi/harness.c): test/smoke.mjs's scene for 10
worker ticks (src/worker.js:96-100) -- create, setParams, initFlat, then
step / absorbDeadCells / sphereStep with the impulses added as
applyImpulseAtCell would -- ends bit for bit where the Python drop-in (the
same library, through ctypes) ends, and a destroyed handle throws."""
import os
import subprocess

import numpy as np
import pytest

import scenes

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ADDON = os.path.join(ROOT, "claude-vibe-code-raytracing_b200", "napi", "build", "lbm_b200.node")
HARNESS = os.path.join(ROOT, "tests", "napi", "build", "harness")


def test_addon_smoke_scene_matches_python_path():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import b200lbm
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "claude-vibe-code-raytracing_b200", "napi")], check=True)
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "tests", "napi")], check=True)
    r = subprocess.run([HARNESS, ADDON, "gpu"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    out = {ln.split()[0]: ln.split()[1:] for ln in r.stdout.splitlines() if not ln.startswith("threw")}
    assert "threw destroyed handle: LBM_ERR_1" in r.stdout

    sim, sol = scenes.smoke(b200lbm.Sim, b200lbm.RigidSphere)
    sim.rhoG, sim.mobility = 0.1, 0.02
    for _ in range(10):
        scenes.substep(sim, sol)
    phi = np.asarray(sim.phi)
    total = 0.0
    for v in phi.astype(np.float64):  # the harness's order: cell 0 first, in double
        total += float(v)
    assert float(out["phisum"][0]) == total
    assert np.float32(out["phi777"][0]) == phi[sim.idx(7, 7, 7)]
    keys = ("cx", "cy", "cz", "vx", "vy", "vz", "wx", "wy", "wz")
    assert [float(v) for v in out["sphere"]] == [getattr(sol, k) for k in keys]
