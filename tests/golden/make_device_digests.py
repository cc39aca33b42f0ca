"""Bit-level pins of the CUDA path's own output, one per storage form.

The FP32 path is held to the oracle within FP32 rounding, and the reduced forms
(FP16 / BF16 offsets) to the FP64 storage form within their error bars; neither
bar notices a change that moves bits inside the bar (a different rounding of
the encode, a pad slot written differently, an operation reassociated).  This
script records SHA-256 digests of every field after a fixed run of two scenes
in each storage form; tests/test_precision_gpu.py recomputes them and must
match bit for bit.  A deliberate change of the arithmetic regenerates the file
(on a GPU) and says why in its commit.

Scenes: the drop preset of src/worker.js:23-53 with sigma 0.012 and g 0.0012
(the sphere falls through the interface, so moving-wall links, fresh and dead
cells all occur), 60 ticks through Sim.run_coupled; and the 256^3 benchmark
scene scaled to 48^3, 30 ticks.

Usage (needs a CUDA device):  python tests/golden/make_device_digests.py
writes tests/golden/device_digests.json.
"""
import hashlib
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (ROOT, os.path.join(ROOT, "claude-vibe-code-raytracing_b200"), os.path.dirname(HERE)):
    if p not in sys.path:
        sys.path.insert(0, p)

import numpy as np  # noqa: E402

FIELDS = ("f", "h", "phi", "rho", "ux", "uy", "uz", "tag")
STORAGES = ("f32", "f16", "bf16", "f64")


def cases():
    import scenes
    return {
        "drop60": (lambda S, R: scenes.drop(S, R, sigma=0.012, gravity=0.0012), 60),
        "cfg2_48_30": (lambda S, R: scenes.cfg2(S, R, n=48), 30),
    }


def digest_run(build, steps, storage):
    """Digests of every field (float32 bits as downloaded; FP64 storage as
    float64 bits) and of the sphere state after `steps` ticks."""
    import functools

    import b200lbm
    sim, sol = build(functools.partial(b200lbm.Sim, storage=storage), b200lbm.RigidSphere)
    sim.run_coupled(sol, steps)
    out = {}
    for k in FIELDS:
        a = sim.field64(k) if storage == "f64" and k != "tag" else np.asarray(getattr(sim, k))
        out[k] = hashlib.sha256(np.ascontiguousarray(a).view(np.uint8)).hexdigest()
    st = sol.state()
    out["sphere"] = hashlib.sha256(np.array([st[k] for k in sorted(st)], np.float64).view(np.uint8)).hexdigest()
    sim.close()
    return out


def main():
    table = {}
    for name, (build, steps) in cases().items():
        for st in STORAGES:
            table[f"{name}/{st}"] = digest_run(build, steps, st)
            print(name, st, table[f"{name}/{st}"]["phi"][:16], flush=True)
    path = os.path.join(HERE, "device_digests.json")
    with open(path, "w") as fh:
        json.dump(table, fh, indent=1, sort_keys=True)
    print("wrote", path)


if __name__ == "__main__":
    main()
