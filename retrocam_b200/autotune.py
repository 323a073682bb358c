"""Autotuner for the launch shape of the render path (rc_tuning).

The reference's shaders have fixed local sizes and nothing to tune; this
module picks, per GPU, resolution and scene, the knobs of
`rc_set_tuning`: the path-tracer engine, the wavefront queue capacity
(paths in flight per chunk), which ray classes walk the 4-wide BVH, and the
block sizes of the trace, shade and photon kernels.

Search: for each engine, coordinate descent over the other knobs from the
best tuning so far.  Each knob in turn is set to each of its candidate
values with the others held, a probe (one caller-supplied step of the real
workload) is timed, and the fastest value is kept when it beats the
incumbent by more than `min_gain`.  Passes repeat until one changes nothing
(at most `max_passes`); the engine whose descent ends fastest wins.  A probe
is timed by wall clock around a device synchronize, min over `repeats` after
one untimed warm-up, so launch overhead counts as it does for the caller.

Results are cached as JSON keyed by device name, resolution, math mode and a
scene signature; the cache file is `$RETROCAM_TUNING_CACHE` or
`~/.cache/retrocam_b200/tuning.json`.  Entries tuned on a B200 for the
project's workloads ship in `tuning_b200.json` beside this module and are
read when the user cache has no entry for a key.
"""
from __future__ import annotations

import json
import os
import time
from typing import Callable

# candidate values per knob, in search order
KNOBS: dict[str, tuple[int, ...]] = {
    "engine": (1, 2, 0),                           # wavefront, wavefront static, megakernel
    "chunk_paths": (8 << 20, 16 << 20, 32 << 20),
    "wide_bvh": (0, 1, 2, 3),
    "trace_block": (64, 128, 256),
    "shade_block": (64, 128, 256),
    "photon_block": (64, 128, 256),
    "photon_full_first": (0, 1),
    "refill_lanes": (12, 16, 20, 24, 28),
    "leaf_quarters": (1, 2, 3, 4),
    "material_queues": (0, 1),
    "interior_steps": (2, 4, 6, 8),
}


def default_cache_path() -> str:
    return os.environ.get("RETROCAM_TUNING_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "retrocam_b200", "tuning.json"))


def cache_key(device_name: str, width: int, height: int, math_mode: int, scene_signature: str) -> str:
    return f"{device_name}|{width}x{height}|math{math_mode}|{scene_signature}"


def scene_signature(scene: dict) -> str:
    """Triangle, node and light counts plus a hash of the node boxes: the
    traversal cost depends on the tree, not on materials."""
    import hashlib
    nodes = scene["nodes"]
    h = hashlib.sha1(nodes.tobytes()).hexdigest()[:12]
    return f"t{len(scene['tris'])}-n{len(nodes)}-l{int(scene['light_count'])}-{h}"


SHIPPED = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning_b200.json")


def _load(path: str) -> dict:
    if path and os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    return {}


class TuningCache:
    def __init__(self, path: str | None = None, shipped: str | None = SHIPPED):
        self.path = path or default_cache_path()
        self.entries: dict[str, dict] = _load(self.path)
        self.shipped: dict[str, dict] = _load(shipped) if shipped else {}

    def get(self, key: str) -> dict | None:
        e = self.entries.get(key) or self.shipped.get(key)
        return dict(e["tuning"]) if e else None

    def put(self, key: str, tuning: dict, ms: float) -> None:
        self.entries[key] = {"tuning": dict(tuning), "ms": ms}
        os.makedirs(os.path.dirname(self.path) or ".", exist_ok=True)
        tmp = self.path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(self.entries, f, indent=1, sort_keys=True)
        os.replace(tmp, self.path)


def time_probe(ctx, probe: Callable[[], None], repeats: int) -> float:
    """Milliseconds of one probe: min over `repeats` after one warm-up."""
    probe()
    ctx.synchronize()
    best = float("inf")
    for _ in range(repeats):
        t0 = time.perf_counter()
        probe()
        ctx.synchronize()
        best = min(best, (time.perf_counter() - t0) * 1e3)
    return best


def _descend(ctx, timer, knobs, best, best_ms, min_gain, max_passes, log):
    for _ in range(max_passes):
        changed = False
        for name, values in knobs.items():
            for v in values:
                if v == best[name]:
                    continue
                trial = dict(best)
                trial[name] = v
                ctx.set_tuning(**trial)
                ms = timer()
                if log:
                    log(f"{trial}: {ms:.2f} ms (best {best_ms:.2f})")
                if ms < best_ms * (1.0 - min_gain):
                    best, best_ms, changed = trial, ms, True
            ctx.set_tuning(**best)
        if not changed:
            break
    return best, best_ms


def tune(ctx, probe: Callable[[], None], knobs: dict[str, tuple[int, ...]] | None = None, repeats: int = 3,
         min_gain: float = 0.01, max_passes: int = 2, timer: Callable | None = None, log=None) -> tuple[dict, float]:
    """Searches `knobs`, leaves the best tuning set on `ctx` and returns
    (tuning, ms).  The engine changes which other knobs matter (the
    megakernel has no shade kernel; the persistent wavefront trace ignores
    the 4-wide paths bit), so each engine gets its own coordinate descent
    over the remaining knobs and the best engine wins."""
    knobs = KNOBS if knobs is None else knobs
    timer = timer or (lambda: time_probe(ctx, probe, repeats))
    start = ctx.tuning()
    rest = {k: v for k, v in knobs.items() if k != "engine"}
    engines = knobs.get("engine", (start["engine"],))
    engines = (start["engine"],) + tuple(e for e in engines if e != start["engine"])
    best, best_ms = None, float("inf")
    for e in engines:
        t = dict(start if best is None else best)
        t["engine"] = e
        ctx.set_tuning(**t)
        ms = timer()
        t, ms = _descend(ctx, timer, rest, t, ms, min_gain, max_passes, log)
        if best is None or ms < best_ms * (1.0 - min_gain):
            best, best_ms = t, ms
    ctx.set_tuning(**best)
    return best, best_ms


def tuned(ctx, key: str, probe: Callable[[], None], cache: TuningCache | None = None, retune: bool = False,
          **kw) -> dict:
    """Applies the cached tuning for `key`, tuning (and caching) it first
    when absent or when `retune` is set."""
    cache = cache or TuningCache()
    t = None if retune else cache.get(key)
    if t is None:
        t, ms = tune(ctx, probe, **kw)
        cache.put(key, t, ms)
    ctx.set_tuning(**t)
    return t


def _main(argv=None) -> int:
    """Tunes the named workloads' frame step (render + SPPM + à-trous) on GPU 0
    and writes the entries to --out (the shipped table by default)."""
    import argparse
    import torch
    from retrocam_b200 import api, scenes
    ap = argparse.ArgumentParser(description=_main.__doc__)
    ap.add_argument("--workloads", default="export_frame,cornell_small")
    ap.add_argument("--math", default="fast", choices=["fast", "exact"])
    ap.add_argument("--out", default=SHIPPED)
    args = ap.parse_args(argv)
    mode = api.RC_MATH_EXACT if args.math == "exact" else api.RC_MATH_FAST
    cache = TuningCache(args.out, shipped=None)
    for name in args.workloads.split(","):
        w = scenes.WORKLOADS[name]()
        sc = api.build_scene(w.scene)
        cam = api.workload_camera(w)
        sppm = api.rc_sppm_params(w.sppm.photons, w.sppm.hash_size, w.sppm.alpha) if w.sppm else None
        atrous = api.atrous_params(w.atrous if w.atrous is not None else scenes.AtrousDesc(enabled=0))
        iters = w.sppm.iterations if w.sppm else 0
        r0 = w.sppm.r0 if w.sppm else 0.05
        with api.Context(w.width, w.height, 0, mode) as ctx:
            ctx.upload(sc)
            key = cache_key(torch.cuda.get_device_name(0), w.width, w.height, mode, scene_signature(sc))
            t = tuned(ctx, key, lambda: ctx.render_frame(cam, (w.nee_enabled, w.nee_firefly_clamp), w.spp, sppm,
                                                         r0, iters, atrous, read=False),
                      cache=cache, retune=True, log=print)
            print(name, key, t, cache.entries[key]["ms"], "ms", flush=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(_main())
