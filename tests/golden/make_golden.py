"""Golden vectors from the reference solver's own code.

There is no JavaScript engine on this machine, so this script translates the
reference's src/lattices.js, src/solid.js and src/sim.js with jsmini (a
translator for the small JS subset those files use; see jsmini.py), executes
them, drives the scenarios of scenarios.py through the reference's own classes
in the worker's order (src/worker.js:96-100: sim.step(solid);
solid.absorbDeadCells(sim); solid.step(1.0, sim.gravity)), and writes the
results to tests/golden/<name>.npz.

The fixtures hold, per scene: the sphere state and the impulses of every step,
the fresh / dead cell sets of every step, and the fields at checkpoints -- in
full for the 12^3 and 8x12x8 scenes, and as SHA-256 digests plus a strided
sample for the 40x28x40 scenes (keeps the files small; the oracle must match
the digests bit for bit, the GPU compares against the samples).

Usage (needs the reference sources; runs in about three minutes):
    python tests/golden/make_golden.py --ref <reference checkout> [--only smoke ...]
(or set LBM_REFERENCE_DIR to the reference checkout instead of --ref).
"""
import argparse
import array
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import jsmini  # noqa: E402
import scenarios  # noqa: E402


def load_reference(ref):
    srcs = []
    for name in ("lattices.js", "solid.js", "sim.js"):
        with open(os.path.join(ref, "src", name)) as fh:
            srcs.append((name, fh.read()))
    return jsmini.load(srcs)


class _HostWrites:
    """Field writes from the scene builders (`sim.phi[:] = numpy_array`) on the
    translated typed arrays, which only take array.array slices."""

    def __setitem__(self, key, value):
        if isinstance(key, slice) and not isinstance(value, array.array):
            value = array.array(self.typecode, np.ascontiguousarray(
                np.asarray(value), dtype=np.dtype(self.typecode)).tobytes())
        super().__setitem__(key, value)


def reference_classes(ns):
    """(Sim factory, sphere factory, built hook) over the translated classes."""
    writable = {}

    def sim_factory(nx, ny, nz):
        sim = ns["Sim"](nx, ny, nz)
        for v in vars(sim).values():
            if isinstance(v, array.array):
                cls = type(v)
                if cls not in writable:
                    writable[cls] = type(cls.__name__, (_HostWrites, cls), {})
                v.__class__ = writable[cls]
        return sim

    def sphere(nx, ny, nz, **kw):
        return ns["RigidSphere"](nx, ny, nz, jsmini._JSObject(kw))

    def built(sim):
        # back to the plain typed arrays (C-speed element access) for the run
        for v in vars(sim).values():
            if isinstance(v, _HostWrites):
                v.__class__ = type(v).__mro__[2]

    return sim_factory, sphere, built


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("LBM_REFERENCE_DIR"),
                    help="root of the reference checkout (holds src/sim.js); default $LBM_REFERENCE_DIR")
    ap.add_argument("--only", nargs="*")
    args = ap.parse_args()
    if not args.ref:
        ap.error("give --ref <reference checkout> or set LBM_REFERENCE_DIR")
    ns = load_reference(args.ref)
    SimC, SphC, built = reference_classes(ns)

    def pack(sim):
        buf = jsmini.Uint8Array(2 * sim.n)
        sim.packVolume(buf, None)
        return buf

    jobs = {k: (lambda k=k: scenarios.to_fixture(k, scenarios.run_scene(k, SimC, SphC, built)))
            for k in scenarios.PLAN}
    jobs["phases"] = lambda: scenarios.phases_fixture(*scenarios.run_phases(SimC, SphC, built))

    def absorb_pack():
        imp, dead = scenarios.run_absorb(SimC, SphC, built)
        return {"absorb_impulse": imp, "absorb_dead": dead,
                "pack_bytes": scenarios.run_pack(SimC, SphC, pack, built)}

    jobs["absorb_pack"] = absorb_pack
    jobs["crate"] = lambda: scenarios.crate_fixture(scenarios.run_crate(SimC, built))
    for name, job in jobs.items():
        if args.only and name not in args.only:
            continue
        t = time.time()
        data = job()
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **data)
        print(f"{name}: {time.time() - t:.1f} s -> {os.path.relpath(path)} "
              f"({os.path.getsize(path) / 1024:.0f} KiB)")


if __name__ == "__main__":
    main()
