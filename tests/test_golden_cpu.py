"""The oracle pinned against golden vectors of the reference's own code.

tests/golden/*.npz were produced by tests/golden/make_golden.py, which runs the
reference's src/lattices.js, src/solid.js and src/sim.js (translated
mechanically into Python by tests/golden/jsmini.py, since no JavaScript engine
exists here) through the scenarios of tests/golden/scenarios.py.  The oracle
replays the same scenarios and must agree BIT FOR BIT: every field, tag, set,
sphere state and impulse.  Both evaluate in double and round to float32 only
on stores, in the same order, without contraction.
"""
import json
import os

import numpy as np
import pytest

from golden import scenarios

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load(name):
    return np.load(os.path.join(GOLDEN, f"{name}.npz"))


def _bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint32) if a.dtype == np.float32 else a


def assert_record_matches(name, rec, g):
    meta = json.loads(str(g["meta"]))
    for (fld, s), a in rec["fields"].items():
        if meta["digest_only"]:
            assert scenarios.digest(a) == str(g[f"sha_{fld}_{s}"]), f"{name}: {fld} at step {s}"
        else:
            assert np.array_equal(_bits(a), _bits(g[f"{fld}_{s}"])), f"{name}: {fld} at step {s}"
    for k in ("f_final", "h_final"):
        if k in g:
            assert np.array_equal(_bits(rec[k]), _bits(g[k])), f"{name}: {k}"
        else:
            assert scenarios.digest(rec[k]) == str(g["sha_" + k]), f"{name}: {k}"
    nf = np.array([len(x) for x in rec["fresh"]])
    nd = np.array([len(x) for x in rec["dead"]])
    assert np.array_equal(nf, g["n_fresh"]) and np.array_equal(nd, g["n_dead"]), name
    assert np.array_equal(np.concatenate(rec["fresh"]), g["fresh"]), name
    assert np.array_equal(np.concatenate(rec["dead"]), g["dead"]), name
    if "sphere" in g:
        for k in ("sphere", "impulse_stream", "impulse_dead"):
            assert np.array_equal(np.array(rec[k]), g[k]), f"{name}: {k}"


@pytest.mark.parametrize("name", list(scenarios.PLAN))
def test_oracle_matches_reference_golden(name, oracle_mod):
    g = _load(name)
    rec = scenarios.run_scene(name, oracle_mod.OracleSim, oracle_mod.OracleSphere)
    assert_record_matches(name, rec, g)


def test_oracle_phases_match_reference_golden(oracle_mod):
    g = _load("phases")
    fields, sphere = scenarios.run_phases(oracle_mod.OracleSim, oracle_mod.OracleSphere)
    for fld, a in fields.items():
        assert scenarios.digest(a) == str(g[f"sha_{fld}"]), fld
    assert np.array_equal(sphere, g["sphere"])


def test_oracle_absorb_and_pack_match_reference_golden(oracle_mod):
    g = _load("absorb_pack")
    imp, dead = scenarios.run_absorb(oracle_mod.OracleSim, oracle_mod.OracleSphere)
    assert np.array_equal(dead, g["absorb_dead"])
    assert np.array_equal(imp, g["absorb_impulse"])
    packed = scenarios.run_pack(oracle_mod.OracleSim, oracle_mod.OracleSphere,
                                lambda sim: sim.packVolume())
    assert np.array_equal(packed, g["pack_bytes"])


def test_golden_fixtures_exercise_the_edge_cases():
    """The fixtures cover what the reference's path branches on: fresh and dead
    cells (moving sphere), a scene without a solid, NaN / edge pack inputs."""
    for name in ("smoke", "cfg1", "drop"):
        g = _load(name)
        assert g["n_dead"].sum() > 0 and g["n_fresh"].sum() > 0, name
    assert "sphere" not in _load("profile")
    pk = _load("absorb_pack")["pack_bytes"]
    assert set(np.unique(pk[1::2])) == {0, 255} and pk[0::2].max() == 255 and pk[0::2].min() == 0
