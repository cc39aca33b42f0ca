"""The z-slab partition and exchange schedule (b200lbm.slab), without a GPU:
every interior plane is owned by exactly one slab, each slab holds two
copied planes per cut, and the exchange fills every copied plane from the
neighbour that owns it."""
import pytest

from b200lbm.slab import HALO, exchange_plan, slab_plan


@pytest.mark.parametrize("nz,ns", [(48, 2), (48, 3), (256, 4), (11, 4), (40, 1)])
def test_partition_and_exchange(nz, ns):
    plan = slab_plan(nz, ns)
    owned = []
    for s, (g0, g1, lo, hi, zoff, nzl, own_lo, own_hi) in enumerate(plan):
        assert own_hi - own_lo == g1 - g0 and own_lo + zoff == g0 and own_hi + zoff == g1
        assert g1 - g0 + 1 >= HALO
        assert zoff >= 0 and zoff + nzl <= nz
        assert lo == (1 if s == 0 else HALO) and hi == (1 if s == ns - 1 else HALO)
        owned += list(range(g0, g1 + 1))
    assert owned == list(range(1, nz - 1))
    filled = {}
    for dst, dplane, src, splane, k in exchange_plan(plan):
        for j in range(k):
            scene_dst = plan[dst][4] + dplane + j
            scene_src = plan[src][4] + splane + j
            assert scene_dst == scene_src  # the same scene plane
            assert plan[src][6] <= splane + j <= plan[src][7]  # copied from its owner
            filled[(dst, dplane + j)] = True
    for s, (g0, g1, lo, hi, zoff, nzl, own_lo, own_hi) in enumerate(plan):
        for k in range(nzl):
            scene = k + zoff
            if scene in (0, nz - 1) or own_lo <= k <= own_hi:
                continue
            assert (s, k) in filled, (s, k)


def test_too_many_slabs():
    with pytest.raises(ValueError):
        slab_plan(7, 4)


def test_step_order_fills_in_scan_order(monkeypatch):
    """SlabSim.step's protocol with stand-ins for the handles: slab s + 1
    begins (retag + fresh fill) only after slab s began and its top owned
    planes were copied up; every bottom-plane copy down comes after all begins
    and before any end; the post-step exchange comes last."""
    import b200lbm.slab as slab
    log, made = [], []

    class FakeSim:
        def __init__(self, nx, ny, nz, storage="f32", device=0):
            self.handle = len(made)
            made.append(self)

        def step_begin(self, solid):
            log.append(("begin", self.handle))

        def step_end(self, solid):
            log.append(("end", self.handle))

        def _moved(self):
            pass

    class FakeLib:
        def lbm_set_slab(self, *a):
            return 0

        def lbm_slab_copy_planes(self, d, dp, s, sp, k):
            log.append(("copy", d, dp, s, sp, k))
            return 0

        def lbm_last_error(self, h):
            return b""

    monkeypatch.setattr(slab, "Sim", FakeSim)
    monkeypatch.setattr(slab, "lib", lambda: FakeLib())
    monkeypatch.setattr(slab, "check", lambda h, rc: None)
    ns = 3
    scene = slab.SlabSim(8, 8, 48, nslabs=ns)
    scene.step(None)
    plan = scene.plan
    up = [("copy", s + 1, 0, s, plan[s][7] - 1, 2) for s in range(ns - 1)]
    down = [("copy", s, plan[s][7] + 1, s + 1, plan[s + 1][6], 2) for s in range(ns - 1)]
    expect = []
    for s in range(ns):
        expect.append(("begin", s))
        if s < ns - 1:
            expect.append(up[s])
    expect += down
    expect += [("end", s) for s in range(ns)]
    for u, d in zip(up, down):
        expect += [u, d]
    assert log == expect
