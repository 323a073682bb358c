"""The VHS chain's host side: pass names in PostProcessStack order
(render/PostProcessStack.java:149-277 runs p01..p16 over a ping-pong pair,
each pass behind its settings toggle) and a timing entry point.

    python -m retrocam_b200.post_stack --time      # all passes, 854x480

p05/p06 (AGC, white balance) have no shaders in the reference: AGC is a
uniform (TemporalState.agcGain) that p04 and p07 read.
"""
from __future__ import annotations

import argparse
import json
import time

from . import api, scenes

PASS_NAMES = {1: "downsample", 2: "chroma_res", 3: "color_matrix", 4: "dynamic_range", 7: "ccd_noise",
              8: "ccd_smear", 9: "chroma_bleed", 10: "timebase", 11: "dot_crawl", 12: "dropout",
              13: "headswitch", 14: "tracking", 15: "edge_enhance", 16: "interlace"}
assert tuple(PASS_NAMES) == api.VHS_PASSES


def time_chain(width=854, height=480, passes=api.VHS_PASSES, calls=50) -> dict:
    """CUDA-event milliseconds of rc_post_vhs (the given passes) on a
    denoised 1-spp frame of the export scene resident on the device; 3
    untimed calls first."""
    w = scenes.export_frame()
    p = api.vhs_defaults(passes=passes, frame_index=90, time_s=3.0, tape_age=0.5, dropout_burst_rate=0.5)
    with api.Context(width, height, 0, api.RC_MATH_FAST) as ctx:
        ctx.upload(api.build_scene(w.scene))
        ctx.render(api.workload_camera(w), (w.nee_enabled, w.nee_firefly_clamp), 0, 1)
        ctx.denoise(api.atrous_params(scenes.AtrousDesc()), read=False)
        for _ in range(3):
            ctx.post_vhs(p)
        ctx.synchronize()
        ctx.set_kernel_timing(True)
        ctx.kernel_times()
        t0 = time.perf_counter()
        for _ in range(calls):
            ctx.post_vhs(p)
        ctx.synchronize()
        wall = (time.perf_counter() - t0) * 1e3 / calls
        ms, n = ctx.kernel_times()["vhs"]
    px = width * height
    return {"width": width, "height": height, "passes": len(passes), "calls": calls,
            "chain_ms": ms / calls, "wall_ms": wall, "launches_per_call": n // calls,
            "ns_per_pixel_pass": ms / calls * 1e6 / (px * len(passes))}


def _main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--time", action="store_true", help="time the whole chain at 854x480")
    ap.add_argument("--each", action="store_true", help="also time each pass alone")
    args = ap.parse_args(argv)
    if args.time or args.each:
        print(json.dumps(time_chain()))
    if args.each:
        for k, name in PASS_NAMES.items():
            r = time_chain(passes=(k,))
            print(json.dumps({"pass": k, "name": name, "ms": r["chain_ms"]}))
    return 0


if __name__ == "__main__":
    raise SystemExit(_main())
