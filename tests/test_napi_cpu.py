"""The Node-API addon (claude-vibe-code-raytracing_b200/napi/binding.c) built and
driven from C through a stand-in for Node's side of Node-API
(tests/napi/napi_stub.c), as Node would load it: dlopen, then
napi_register_module_v1.  There is no Node on this machine or the GPU box, so
the reference's JavaScript itself is not run.  Here, without a GPU: every
C-ABI entry with a JavaScript caller is exported, the host RigidSphere.step
behind sphereStep matches the oracle bit for bit, and bad arguments throw
JavaScript errors with the library's codes instead of crashing."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ADDON = os.path.join(ROOT, "claude-vibe-code-raytracing_b200", "napi", "build", "lbm_b200.node")
HARNESS = os.path.join(ROOT, "tests", "napi", "build", "harness")

EXPECTED = """create destroy lastError getDims deviceBytes footprintBytes setParams getParams uploadField retagCellsMask retagCellsMesh voxelizeMesh solidLinks
downloadField downloadFieldF64 initFlat seedHydrostatic retagCells handleFreshCells computePhiGradients
collidePhase streamPhase collideHydro streamHydroAndMacro step absorbDeadCells packVolume packVolumeAsync
waitFrames waitFrameSlot stepFrame initProfile runCoupled sphereStep synchronize setNanWatchdog lastSets launchCount checkedBuild faultRecord
transferBytes fusedTiming fusedTimingQuery setFusedConfig getFusedConfig testWithholdStageCopy cameraDefault render
batchCreate batchDestroy batchSetConfig batchRun batchTimeFused batchLaunchCount""".split()


@pytest.fixture(scope="module")
def built():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "claude-vibe-code-raytracing_b200", "napi")], check=True)
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "tests", "napi")], check=True)
    return ADDON, HARNESS


def _run(built, mode):
    addon, harness = built
    r = subprocess.run([harness, addon, mode], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout


def test_exports(built):
    names = _run(built, "exports").split()
    assert sorted(names) == sorted(EXPECTED)


def test_sphere_step_and_argument_errors(built, oracle_mod):
    out = _run(built, "cpu")
    got = {ln.split()[0]: [float(v) for v in ln.split()[1:]] for ln in out.splitlines() if ln.startswith("sphere")}
    a = oracle_mod.OracleSphere(40, 28, 40, cx=20.0, cy=14.0, cz=20.0, r=4.0, density=2.0)
    a.Fy, a.Tx = -0.3, 0.02
    b = oracle_mod.OracleSphere(40, 28, 40, cx=10.0, cy=8.0, cz=30.0, r=3.0, density=1.4)
    b.dragging = True
    b.dragTargetX, b.dragTargetY, b.dragTargetZ = 30.0, 20.0, 10.0
    for _ in range(3):
        a.step(1.0, -0.001)
        b.step(1.0, -0.001)
    keys = ("cx", "cy", "cz", "vx", "vy", "vz", "wx", "wy", "wz")
    assert got["sphere0"] == [getattr(a, k) for k in keys]
    assert got["sphere1"] == [getattr(b, k) for k in keys]
    for what in ("float32 spheres", "22 numbers", "number as handle", "too few arguments", "2x2x2 grid"):
        assert f"threw {what}: LBM_ERR_" in out, what
