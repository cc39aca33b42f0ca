"""The golden scenarios: one driver shared by the fixture generator (which runs
it on the reference's own code, translated by jsmini) and by the tests (which
run it on the oracle and on the CUDA path), so all three see exactly the same
sequence of calls.

Each driver takes the Sim class, the sphere class and a hook run once the
scene is built (the generator uses it to switch the translated typed arrays
back to their fast form).  Field arrays come back as numpy copies.
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

import scenes  # noqa: E402

FIELDS = ("phi", "rho", "ux", "uy", "uz")
SPHERE_KEYS = ("cx", "cy", "cz", "vx", "vy", "vz", "wx", "wy", "wz")
IMPULSE_KEYS = ("Fx", "Fy", "Fz", "Tx", "Ty", "Tz")
SAMPLE_STRIDE = 13

# scene -> (steps, checkpoints, populations kept in full, fields as digest + sample)
PLAN = {
    "smoke": (80, (1, 2, 10, 80), True, False),
    "profile": (40, (1, 40), True, False),
    "cfg1": (80, (1, 80), False, True),
    "drop": (60, (60,), False, True),
    "dam": (120, (120,), False, True),
    "rise": (120, (120,), False, True),
    "drag": (220, (220,), False, True),
}

# test/drag_stress.mjs's path with shorter legs (the same targets), so the
# translated reference finishes in minutes
SHORT_DRAG_PATH = [(40, (20, 24, 20)), (40, (30, 24, 20)), (60, (30, 4, 20)), (30, (20, 4, 20)),
                   (50, (20, 18, 20))]


def _drag_prestep(s, sim, sol):
    scenes.drag_target(sol, s - 1, SHORT_DRAG_PATH)


# called before step s (1-based) of a scene
PRESTEP = {"drag": _drag_prestep}


def digest(arr):
    return hashlib.sha256(np.ascontiguousarray(arr).tobytes()).hexdigest()


def as_np(field):
    return np.array(field, copy=True)


def sets_of(sim):
    tag, prev = as_np(sim.tag), as_np(sim.tagPrev)
    fresh = np.nonzero((tag == 0) & (prev == 1))[0].astype(np.int32)
    dead = np.nonzero((tag == 1) & (prev == 0))[0].astype(np.int32)
    return fresh, dead


def _noop(sim):
    pass


def run_scene(name, SimC, SphC, built=_noop, on_step=None):
    """`steps` worker ticks (src/worker.js:96-100) of a scenes.py scene.

    Returns the raw record: per-step sphere state, the impulse of the stream
    (momentum exchange) and of absorbDeadCells, the fresh / dead sets, and the
    fields at the checkpoints (plus f, h at the end)."""
    steps, checkpoints, _, _ = PLAN[name]
    sim, sol = scenes.SCENES[name](SimC, SphC)
    built(sim)
    rec = {"fields": {}, "sphere": [], "impulse_stream": [], "impulse_dead": [],
           "fresh": [], "dead": []}
    pre = PRESTEP.get(name)
    for s in range(1, steps + 1):
        if pre is not None:
            pre(s, sim, sol)
        if on_step is not None:
            on_step(s, sim, sol)
        sim.step(sol)
        fr, de = sets_of(sim)
        rec["fresh"].append(fr)
        rec["dead"].append(de)
        if sol is not None:
            rec["impulse_stream"].append([getattr(sol, k) for k in IMPULSE_KEYS])
            f0 = [getattr(sol, k) for k in IMPULSE_KEYS]
            sol.absorbDeadCells(sim)
            rec["impulse_dead"].append([getattr(sol, k) - a for k, a in zip(IMPULSE_KEYS, f0)])
            sol.step(1.0, sim.gravity)
            rec["sphere"].append([getattr(sol, k) for k in SPHERE_KEYS])
        if s in checkpoints:
            for fld in FIELDS + ("tag",):
                rec["fields"][(fld, s)] = as_np(getattr(sim, fld))
    rec["f_final"] = as_np(sim.f)
    rec["h_final"] = as_np(sim.h)
    return rec


def to_fixture(name, rec):
    steps, checkpoints, full_pops, digest_only = PLAN[name]
    out = {}
    for (fld, s), a in rec["fields"].items():
        if digest_only:
            out[f"sha_{fld}_{s}"] = np.array(digest(a))
            out[f"sample_{fld}_{s}"] = a[::SAMPLE_STRIDE].copy()
        else:
            out[f"{fld}_{s}"] = a
    for k in ("f_final", "h_final"):
        if full_pops:
            out[k] = rec[k]
        else:
            out["sha_" + k] = np.array(digest(rec[k]))
    if rec["sphere"]:
        for k in ("sphere", "impulse_stream", "impulse_dead"):
            out[k] = np.array(rec[k], dtype=np.float64)
    out["n_fresh"] = np.array([len(x) for x in rec["fresh"]], dtype=np.int32)
    out["n_dead"] = np.array([len(x) for x in rec["dead"]], dtype=np.int32)
    out["fresh"] = np.concatenate(rec["fresh"]).astype(np.int32)
    out["dead"] = np.concatenate(rec["dead"]).astype(np.int32)
    out["meta"] = np.array(json.dumps({"scene": name, "steps": steps,
                                       "checkpoints": list(checkpoints),
                                       "sample_stride": SAMPLE_STRIDE,
                                       "digest_only": digest_only}))
    return out


def run_phases(SimC, SphC, built=_noop):
    """The seven Sim phases called one by one (test/bench_phases.mjs) on the
    bench scene for 6 steps; returns the fields and the gradient scratch."""
    sim, sol = scenes.bench(SimC, SphC)
    built(sim)
    for _ in range(6):
        sim.retagCells(sol)
        sim.handleFreshCells(sol)
        sim.computePhiGradients()
        sim.collidePhase()
        sim.streamPhase()
        sim.collideHydro()
        sim.streamHydroAndMacro(sol)
        sol.absorbDeadCells(sim)
        sol.step(1.0, sim.gravity)
    fields = {fld: as_np(getattr(sim, fld)) for fld in FIELDS + ("gx", "gy", "gz", "lap", "tag")}
    return fields, np.array([getattr(sol, k) for k in SPHERE_KEYS])


def phases_fixture(fields, sphere):
    out = {}
    for fld, a in fields.items():
        out[f"sha_{fld}"] = np.array(digest(a))
        out[f"sample_{fld}"] = a[::SAMPLE_STRIDE].copy()
    out["sphere"] = sphere
    return out


def absorb_fields(n):
    rng = np.random.default_rng(11)
    return {"phi": rng.uniform(-0.1, 1.1, n).astype(np.float32),
            "ux": rng.normal(0, 0.02, n).astype(np.float32),
            "uy": rng.normal(0, 0.02, n).astype(np.float32),
            "uz": rng.normal(0, 0.02, n).astype(np.float32)}


def run_absorb(SimC, SphC, built=_noop):
    """absorbDeadCells (src/solid.js:87-101) over a whole sphere of dead cells
    (the first retag after placing it) on seeded fields of the bench scene."""
    sim, sol = scenes.bench(SimC, SphC)
    for k, v in absorb_fields(sim.n).items():
        getattr(sim, k)[:] = v
    built(sim)
    sol.cx, sol.cy, sol.cz = 19.3, 13.6, 20.4
    sol.setRadius(8.5)
    sim.retagCells(sol)
    sol.absorbDeadCells(sim)
    _, dead = sets_of(sim)
    return np.array([getattr(sol, k) for k in IMPULSE_KEYS]), dead


def pack_phi(n):
    rng = np.random.default_rng(3)
    phi = rng.uniform(-0.2, 1.2, size=n).astype(np.float32)
    phi[::97] = np.float32(np.nan)
    phi[1::89] = np.float32(254.5 / 255)
    phi[2::83] = np.float32(1.0)
    phi[3::79] = np.float32(0.0)
    return phi


def run_pack(SimC, SphC, pack, built=_noop):
    """packVolume (src/sim.js:586-600) of seeded phi with NaN and edge values on
    the smoke scene after one retag (so SOLID cells set the G channel)."""
    sim, sol = scenes.smoke(SimC, SphC)
    sim.retagCells(sol)
    sim.phi[:] = pack_phi(sim.n)
    built(sim)
    return np.asarray(pack(sim), dtype=np.uint8).copy()


CRATE_STEPS = 40


def run_crate(SimC, built=_noop):
    """A duck-typed solid that is not a sphere (scenes.Crate: a moving box)
    in the drop preset's pool, CRATE_STEPS worker ticks: per step the force and
    torque the stream gave it (through its applyImpulseAtCell), the dead-cell
    impulse, the fresh / dead sets; the fields at the end."""
    sim, box = scenes.crate(SimC)
    built(sim)
    rec = {"impulse_stream": [], "impulse_dead": [], "fresh": [], "dead": []}
    for s in range(CRATE_STEPS):
        sim.step(box)
        fr, de = sets_of(sim)
        rec["fresh"].append(fr)
        rec["dead"].append(de)
        rec["impulse_stream"].append([getattr(box, k) for k in IMPULSE_KEYS])
        f0 = [getattr(box, k) for k in IMPULSE_KEYS]
        box.absorbDeadCells(sim)
        rec["impulse_dead"].append([getattr(box, k) - a for k, a in zip(IMPULSE_KEYS, f0)])
        box.step(1.0, sim.gravity)
    rec["fields"] = {fld: as_np(getattr(sim, fld)) for fld in FIELDS + ("tag",)}
    return rec


def crate_fixture(rec):
    out = {}
    for fld, a in rec["fields"].items():
        out[f"sha_{fld}"] = np.array(digest(a))
        out[f"sample_{fld}"] = a[::SAMPLE_STRIDE].copy()
    for k in ("impulse_stream", "impulse_dead"):
        out[k] = np.array(rec[k], dtype=np.float64)
    out["n_fresh"] = np.array([len(x) for x in rec["fresh"]], dtype=np.int32)
    out["n_dead"] = np.array([len(x) for x in rec["dead"]], dtype=np.int32)
    out["fresh"] = np.concatenate(rec["fresh"]).astype(np.int32)
    out["dead"] = np.concatenate(rec["dead"]).astype(np.int32)
    return out
