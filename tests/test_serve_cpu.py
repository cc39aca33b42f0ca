"""Host logic of batching and serving that needs no GPU: admission order and
budget, the seeded workload generators, the autotuner's signature."""
import numpy as np

from b200lbm import autotune, serve, workloads


def _req(rid, arrival, size):
    return dict(rid=rid, arrival=arrival, spec=dict(dims=(size, size, size)), steps=40, frame_every=20)


def test_admission_within_budget_with_aging():
    q = [_req(0, 0.0, 10), _req(1, 0.1, 20), _req(2, 0.2, 10), _req(3, 5.0, 10)]
    fp = lambda r: r["spec"]["dims"][0]  # noqa: E731
    # all arrived but the last; the second does not fit, the third does
    assert [r["rid"] for r in serve.admit(q, 0, 25, 1.0, fp)] == [0, 2]
    assert [r["rid"] for r in serve.admit(q, 0, 40, 1.0, fp)] == [0, 1, 2]
    # a request that does not fit is passed over by smaller later ones ...
    assert [r["rid"] for r in serve.admit(q[1:], 10, 25, 1.0, fp)] == [2]
    # ... until it has waited the aging bound; then nothing goes ahead of it
    assert [r["rid"] for r in serve.admit(q[1:], 10, 25, 0.1 + serve.AGE_LIMIT_S, fp)] == []
    # nothing arrived yet
    assert serve.admit(q, 0, 100, -1.0, fp) == []
    # an oversized request runs alone when the device is idle
    assert [r["rid"] for r in serve.admit([_req(9, 0.0, 99)], 0, 50, 1.0, fp)] == [9]
    assert serve.admit([_req(9, 0.0, 99)], 1, 50, 1.0, fp) == []


def test_scene_specs_follow_the_stated_distribution():
    specs = workloads.scene_specs(64, seed=0)
    assert specs == workloads.scene_specs(64, seed=0)  # seeded
    for s in specs:
        nx, ny, nz = s["dims"]
        assert all(32 <= d <= 160 for d in (nx, ny, nz))
        assert 0.3 * ny <= s["level"] <= 0.6 * ny
        assert 1 <= len(s["spheres"]) <= 3
        for i, p in enumerate(s["spheres"]):
            m = p["r"] + 1.5
            assert 3.0 <= p["r"] <= 12.0 and 1.2 <= p["density"] <= 4.0
            assert m <= p["cx"] <= nx - 1 - m and m <= p["cz"] <= nz - 1 - m
            assert max(m, s["level"] + p["r"]) <= p["cy"] <= ny - 1 - m
            assert np.hypot(np.hypot(p["vx"], p["vy"]), p["vz"]) <= 0.02 + 1e-12
            for q in s["spheres"][:i]:
                d = np.linalg.norm([p["cx"] - q["cx"], p["cy"] - q["cy"], p["cz"] - q["cz"]])
                assert d > p["r"] + q["r"]


def test_request_stream():
    rs = workloads.request_stream(200, seed=1)
    arr = np.array([r["arrival"] for r in rs])
    assert np.all(np.diff(arr) > 0)
    assert 10 < 200 / arr[-1] < 30  # Poisson at 20/s
    assert all(500 <= r["steps"] <= 5000 and r["steps"] % 20 == 0 for r in rs)
    big = sum(r["spec"]["dims"] == (256, 256, 256) for r in rs)
    assert 5 <= big <= 40


def test_autotune_signature_buckets():
    a = autotune.signature([(64, 64, 64)] * 3, "f16")
    b = autotune.signature([(60, 64, 64)] * 4, "f16")
    assert a == b
    assert autotune.signature([(64, 64, 64)] * 5, "f16") != a
    assert autotune.signature([(64, 64, 64)] * 3, "f32") != a


class _FakeBatch:
    """time_fused returns a fixed time per shape; set_config records the shape."""

    def __init__(self, times):
        self.times = times
        self.timed = []
        self.shape = None

    def time_fused(self, rows, zchunk, reps=3):
        self.timed.append((rows, zchunk))
        return self.times[(rows, zchunk)]

    def set_config(self, rows, zchunk):
        self.shape = (rows, zchunk)


def test_incremental_tuner_times_one_candidate_per_step():
    autotune.clear()
    cands = [(4, 32), (4, 16), (8, 16)]
    times = {(4, 32): 7.1, (4, 16): 6.9, (8, 16): 7.5}
    b = _FakeBatch(times)
    t = autotune.Incremental(b, [(64, 64, 64)] * 3, "f16", candidates=cands)
    assert not t.done and b.shape is None
    assert t.step() is False and b.timed == [(4, 32)] and b.shape is None
    assert t.step() is False and len(b.timed) == 2
    assert t.step() is True and b.shape == (4, 16)  # the fastest, set after the last candidate
    assert t.step() is True and len(b.timed) == 3   # nothing more is timed
    # timings of one signature accumulate across batches (members changed)
    autotune.clear()
    b4, b5 = _FakeBatch(times), _FakeBatch(times)
    t4 = autotune.Incremental(b4, [(64, 64, 64)] * 3, "f16", candidates=cands)
    t4.step()
    t5 = autotune.Incremental(b5, [(62, 64, 64)] * 4, "f16", candidates=cands)
    assert t5.step() is False and b5.timed == [(4, 16)]
    assert t5.step() is True and b5.shape == (4, 16) and b5.timed == [(4, 16), (8, 16)]
    assert t4.step() is True and b4.shape == (4, 16) and b4.timed == [(4, 32)]
    # the same signature later is answered from the cache at once, like tune()
    b2 = _FakeBatch(times)
    t2 = autotune.Incremental(b2, [(60, 64, 64)] * 4, "f16", candidates=cands)
    assert t2.done and b2.shape == (4, 16) and b2.timed == []
    b3 = _FakeBatch(times)
    assert autotune.tune(b3, [(64, 64, 64)] * 3, "f16", candidates=cands)[:2] == (4, 16)
    assert b3.timed == []
    autotune.clear()
