"""The launch-shape autotuner's search and cache, against a fake context
whose probe cost is a known function of the knobs (no GPU)."""
import json

from retrocam_b200 import autotune


class FakeCtx:
    def __init__(self, cost):
        self.t = {"engine": 1, "chunk_paths": 0, "wide_bvh": 0, "trace_block": 128, "shade_block": 128,
                  "photon_block": 128, "photon_full_first": 0, "refill_lanes": 20, "leaf_quarters": 2,
                  "material_queues": 0, "interior_steps": 1}
        self.cost = cost
        self.calls = 0

    def tuning(self):
        return dict(self.t)

    def set_tuning(self, **k):
        self.t.update(k)

    def synchronize(self):
        pass


def test_coordinate_descent_finds_separable_optimum():
    want = {"engine": 2, "chunk_paths": 32 << 20, "wide_bvh": 3, "trace_block": 64, "shade_block": 256,
            "photon_block": 64, "photon_full_first": 1, "refill_lanes": 28, "leaf_quarters": 3,
            "material_queues": 1, "interior_steps": 4}

    def cost(t):
        return 100.0 + sum(10.0 for k in want if t[k] != want[k])

    ctx = FakeCtx(cost)
    best, ms = autotune.tune(ctx, None, timer=lambda: cost(ctx.t))
    assert best == want and ms == 100.0
    assert ctx.tuning() == want


def test_small_gains_do_not_move_the_incumbent():
    ctx = FakeCtx(None)
    start = ctx.tuning()
    best, _ = autotune.tune(ctx, None, timer=lambda: 100.0 - (0.5 if ctx.t["trace_block"] == 256 else 0.0),
                            min_gain=0.01)
    assert best == start


def test_engine_specific_knobs_searched_per_engine():
    # wide_bvh helps only with the megakernel (engine 0); engine is searched first
    def cost(t):
        if t["engine"] == 0:
            return 80.0 if t["wide_bvh"] & 1 else 120.0
        return 100.0

    ctx = FakeCtx(cost)
    best, ms = autotune.tune(ctx, None, knobs={"engine": (1, 0), "wide_bvh": (0, 1)}, max_passes=3,
                             timer=lambda: cost(ctx.t))
    # plain coordinate descent would stop at engine 1 (120 > 100 before wide
    # is tried); each engine gets its own descent, so engine 0 + wide 1 wins
    assert (best["engine"], best["wide_bvh"]) == (0, 1) and ms == 80.0


def test_cache_roundtrip(tmp_path):
    path = tmp_path / "t.json"
    cache = autotune.TuningCache(str(path))
    key = autotune.cache_key("B200", 854, 480, 0, "t1-n1-l1-x")
    assert cache.get(key) is None
    calls = []
    ctx = FakeCtx(None)

    def timer():
        calls.append(1)
        return 50.0 if ctx.t["photon_block"] == 64 else 60.0

    t = autotune.tuned(ctx, key, None, cache=cache, timer=timer, knobs={"photon_block": (64, 128)})
    assert t["photon_block"] == 64 and calls
    assert json.loads(path.read_text())[key]["ms"] == 50.0
    # second use: from the cache, no probe
    calls.clear()
    ctx2 = FakeCtx(None)
    t2 = autotune.tuned(ctx2, key, None, cache=autotune.TuningCache(str(path)), timer=timer)
    assert t2 == t and ctx2.tuning() == t and not calls
