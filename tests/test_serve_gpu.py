"""Serving (b200lbm.serve.Server): continuous batching of scene requests on
one GPU.  Each request's frames, final fields and sphere state are the same
whether it is served alone or in a mix with others, and whether the memory
budget lets all run at once or forces them to take turns -- bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import b200lbm
    return b200lbm


def _trace():
    from b200lbm import workloads
    specs = workloads.scene_specs(4, seed=3)
    # small grids keep the test short; arrival order and lengths differ
    for s in specs:
        s["dims"] = tuple(min(d, 48) for d in s["dims"])
        nx, ny, nz = s["dims"]
        s["level"] = min(s["level"], 0.5 * ny)
        kept = []
        for p in s["spheres"]:
            m = p["r"] + 1.5
            if p["r"] <= 6 and m <= p["cx"] <= nx - 1 - m and m <= p["cz"] <= nz - 1 - m \
                    and max(m, s["level"] + p["r"]) <= p["cy"] <= ny - 1 - m:
                kept.append(p)
        s["spheres"] = kept or [dict(cx=nx / 2, cy=ny - 6.0, cz=nz / 2, r=3.0, density=2.0,
                                     vx=0.0, vy=0.0, vz=0.0)]
    steps = [60, 40, 80, 40]
    return [dict(rid=i, arrival=0.01 * i, spec=s, steps=steps[i], frame_every=20)
            for i, s in enumerate(specs)]


def _serve(gpu, reqs, claims=None, **kw):
    from b200lbm.serve import Server
    from b200lbm.solid import spheres_of
    frames, final = {}, {}

    def on_frame(rid, j, vol):
        frames.setdefault(rid, []).append(vol.copy())

    def on_finish(rid, sim, solid):
        final[rid] = ({k: np.array(getattr(sim, k)) for k in ("phi", "rho", "ux", "f", "h")},
                      [b.state() for b in spheres_of(solid)])

    rep = Server(**kw).run(reqs, realtime=False, on_frame=on_frame, on_finish=on_finish, claims=claims)
    return rep, frames, final


def test_served_alone_equals_in_mix(gpu):
    reqs = _trace()
    rep, frames, final = _serve(gpu, reqs, storage="f16")
    # scenes are built on worker threads, so a short request may finish before
    # the last one joins: at least three run together
    assert rep["max_active"] >= len(reqs) - 1
    assert rep["frames"] == sum(r["steps"] // 20 for r in reqs)
    assert rep["scene_steps"] == sum(r["steps"] for r in reqs)
    for r in reqs:
        _, fa, ga = _serve(gpu, [r], storage="f16")
        rid = r["rid"]
        assert len(frames[rid]) == r["steps"] // 20
        for a, b in zip(frames[rid], fa[rid]):
            assert np.array_equal(a, b), rid
        for k in ga[rid][0]:
            assert np.array_equal(final[rid][0][k], ga[rid][0][k]), (rid, k)
        assert final[rid][1] == ga[rid][1]


def test_budget_serialises_without_changing_results(gpu):
    from b200lbm.serve import footprint
    reqs = _trace()
    biggest = max(footprint(r["spec"], "f16") for r in reqs)
    _, frames_all, final_all = _serve(gpu, reqs, storage="f16")
    rep, frames, final = _serve(gpu, reqs, storage="f16", budget_bytes=int(1.5 * biggest))
    assert rep["max_active"] < len(reqs)
    for r in reqs:
        rid = r["rid"]
        for a, b in zip(frames[rid], frames_all[rid]):
            assert np.array_equal(a, b)
        for k in final[rid][0]:
            assert np.array_equal(final[rid][0][k], final_all[rid][0][k]), (rid, k)


def test_claimed_stream_equals_listed(gpu):
    """The same requests taken through a claim queue (as several serving
    processes share one stream), here one process under a tight budget:
    every request is claimed once and served bit for bit as from the list."""
    from b200lbm import placement
    from b200lbm.serve import footprint
    reqs = _trace()
    biggest = max(footprint(r["spec"], "f16") for r in reqs)
    _, frames_all, final_all = _serve(gpu, reqs, storage="f16")
    q = placement.ClaimQueue(reqs)
    rep, frames, final = _serve(gpu, None, claims=q, storage="f16", budget_bytes=int(1.5 * biggest))
    assert sorted(rep["claimed"]) == [r["rid"] for r in reqs]
    for r in reqs:
        rid = r["rid"]
        for a, b in zip(frames[rid], frames_all[rid]):
            assert np.array_equal(a, b), rid
        for k in final_all[rid][0]:
            assert np.array_equal(final[rid][0][k], final_all[rid][0][k]), (rid, k)
