#!/usr/bin/env python
"""Benchmark of the B200 render hot path: Msamples/s of one export frame.

A step is one export frame of the `export_frame` workload (854x480, 128 spp
with per-channel lens offsets, i.e. 3 paths per sample; 16 SPPM iterations of
2,000,000 photons on a 2^22-cell hash; 5 à-trous passes), the call sequence
of export/RenderPipeline.java:209-239, issued through rc_render_frame.

  value  samples/s with the scene resident in HBM (rc_render_frame alone),
         timed with CUDA events on the stream the kernels run on
  e2e    the same metric through the C ABI with host buffers, as the
         export path ends: per step the scene upload (host -> device, pinned
         staging), the frame, the display pass (rc_display: ACES + sRGB to
         RGBA8, RenderPipeline.applyDisplayPass) and the read-back of that
         RGBA8 image (device -> host, FrameExporter) are inside the timed region
  roofline  the dominant kernel (render_kernel): algorithmic bytes per launch
         from the kernel's own work counters, divided by its CUDA-event time
  cpu_baseline  the reference's own shaders compiled for the host
         (oracle/_ref, OpenMP over all host cores) on a bounded sample of the
         same workload, extrapolated to a full frame

Multi-GPU: one process per GPU (torchrun); each rank renders its own frame
(independent replicas, no collective on the data path); timing is the max over
ranks and value counts the samples of all ranks (weak scaling).

`--impl reference` times the reference's own CPU shaders on this host and
prints the same line with "impl": "reference" (rank 0 only).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

HBM_FALLBACK_GBS = 6650.0
METRIC = "Msamples/s at 854x480; time to relMSE<=1e-2, learned vs plain, one B200"
UNIT = "Msamples/s"

# algorithmic bytes of the render path (per unit of work, minimal layouts):
BYTES_NODE_TEST = 32      # 6 floats of AABB + 2 ints
BYTES_TRI_TEST = 36       # v0, e1, e2
BYTES_SURFACE_HIT = 40 + 64  # 3 normals + material index, + the 64-B material
BYTES_LIGHT_SAMPLE = 80   # one light record
BYTES_SAMPLE_RMW = 20     # accum RGBA32F (16) + variance R32F (4) per pixel sample


KERNEL_SYMBOL = {"render": "render_kernel", "wf_trace": "wf_trace", "wf_shade": "wf_shade",
                 "photon_trace": "photon_trace_kernel", "photon_gather": "photon_gather_kernel",
                 "atrous": "atrous_kernel", "wf_generate": "wf_generate", "wf_accumulate": "wf_accumulate"}


def algorithmic_bytes(kernel: str, ctr: dict, samples: int) -> float:
    """Bytes the kernel must move at minimum for the work its counters record:
    32 B per ray-box test (6 floats + 2 ints), 36 B per ray-triangle test
    (v0, e1, e2), 104 B per shaded hit (3 normals + material index + the 64-B
    material), 80 B per light record, 20 B per pixel sample (accum + variance
    read-modify-write), and for the wavefront stages the path state they must
    read and write (48 B per closest-hit ray, 96 B per shadow ray)."""
    trav = BYTES_NODE_TEST * ctr["node_tests"] + BYTES_TRI_TEST * ctr["tri_tests"]
    if kernel == "render":
        return (trav + BYTES_SURFACE_HIT * ctr["surface_hits"] + BYTES_LIGHT_SAMPLE * ctr["light_samples"]
                + BYTES_SAMPLE_RMW * samples)
    if kernel == "wf_trace":
        return trav + 48 * ctr["closest_rays"] + 96 * ctr["shadow_rays"]
    if kernel == "wf_shade":
        return (BYTES_SURFACE_HIT + 160) * ctr["surface_hits"] + BYTES_LIGHT_SAMPLE * ctr["light_samples"]
    if kernel in ("photon_trace", "photon_gather"):
        return BYTES_NODE_TEST * ctr["photon_node_tests"] + BYTES_TRI_TEST * ctr["photon_tri_tests"]
    return 0.0


FLOP_NODE_TEST = 22       # 6 sub + 6 mul + 10 min/max
FLOP_TRI_TEST = 40        # Moller-Trumbore


def fp32_roofline(kernel: str, ctr: dict, launches: int, avg_launch_s: float, device: int):
    """FP32 fraction of a traversal kernel: its box and triangle tests as
    FLOPs per launch over its average launch time, against the FMA
    throughput measured on this GPU (rc_measure_fp32_peak).  The scene of
    the export frame is cache-resident, so the traversal is bound by issue
    rate rather than HBM."""
    if kernel == "wf_trace" or kernel == "render":
        flops = FLOP_NODE_TEST * ctr["node_tests"] + FLOP_TRI_TEST * ctr["tri_tests"]
    elif kernel in ("photon_trace", "photon_gather"):
        flops = FLOP_NODE_TEST * ctr["photon_node_tests"] + FLOP_TRI_TEST * ctr["photon_tri_tests"]
    else:
        return None
    import ctypes
    from retrocam_b200 import api
    peak = ctypes.c_double(0.0)
    if api.lib().rc_measure_fp32_peak(device, ctypes.byref(peak)) != 0 or peak.value <= 0 or avg_launch_s <= 0:
        return None
    achieved = flops / max(1, launches) / avg_launch_s / 1e12
    return {"achieved": achieved, "peak": peak.value, "unit": "TFLOP/s", "frac": achieved / peak.value,
            "flops_per_launch": flops / max(1, launches), "peak_source": "measured FMA microbenchmark"}


def parse_args(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="export_frame")
    ap.add_argument("--math", default="fast", choices=["fast", "exact"])
    ap.add_argument("--engine", default="auto", choices=["auto", "wavefront", "wavefront_static", "megakernel"],
                    help="auto: the autotuner's launch shape for this GPU and workload (cached)")
    ap.add_argument("--retune", action="store_true", help="with --engine auto: tune again, ignore the cache")
    ap.add_argument("--chunk-paths", type=int, default=0, help="wavefront paths in flight (0: default)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-quality", action="store_true", help="skip the time-to-relMSE comparison")
    ap.add_argument("--quality-variants", type=int, default=8, help="held-out Cornell variants for time-to-relMSE")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="budget of the CPU-baseline sample")
    ap.add_argument("--spp", type=int, default=0, help="override spp (profiling of a small case)")
    ap.add_argument("--sppm-iterations", type=int, default=-1, help="override SPPM iterations")
    return ap.parse_args(argv)


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0")), \
        int(os.environ.get("WORLD_SIZE", "1"))


def init_dist(world, backend):
    if world <= 1:
        return None
    import datetime

    import torch.distributed as dist
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return dist


def max_over_ranks(value: float, dist, device=None) -> float:
    """Max of a per-rank scalar (timing) over all ranks."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist, device=None):
    if dist is None:
        return
    if device is not None:
        dist.barrier(device_ids=[device.index])
    else:
        dist.barrier()


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            if len(r) < 9:
                continue
            for name, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(name)
        power = [float(r[3]) for r in self.rows if len(r) >= 9 and r[3].replace(".", "").isdigit()]
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm),
                "power_w_max": max(power) if power else None}


# ---------------------------------------------------------------------------
# workload
# ---------------------------------------------------------------------------
def workload_setup(name, args=None):
    from retrocam_b200 import api, scenes
    w = scenes.WORKLOADS[name]()
    if args is not None and args.spp > 0:
        w.spp = args.spp
    if args is not None and args.sppm_iterations >= 0 and w.sppm is not None:
        if args.sppm_iterations == 0:
            w.sppm = None
        else:
            w.sppm.iterations = args.sppm_iterations
    sppm = None
    if w.sppm is not None:
        sppm = api.rc_sppm_params(w.sppm.photons, w.sppm.hash_size, w.sppm.alpha)
    atrous = api.atrous_params(w.atrous if w.atrous is not None else scenes.AtrousDesc(enabled=0))
    return w, sppm, atrous


def read_traffic(kernel: str, workload: str):
    """DRAM bytes per launch of `kernel` from the committed ncu summary
    (profiles/ncu_<kernel>_<workload>.md, line 'traffic_bytes_per_launch: N')."""
    path = os.path.join(REPO, "profiles", f"ncu_{kernel}_{workload}.md")
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.strip().startswith("traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].strip().split()[0])
            except ValueError:
                return None
    return None


def hbm_peak():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return HBM_FALLBACK_GBS, "fallback"


# ---------------------------------------------------------------------------
# CPU baseline: the reference shaders compiled for the host (oracle/_ref)
# ---------------------------------------------------------------------------
def cpu_reference_sample(w, budget_s: float, threads: int = 0):
    """Times the reference's own shaders (pathtrace, photon trace, gather,
    à-trous) on a bounded sample of the workload on all host cores and
    extrapolates the time of one full frame.  Returns (frame_seconds, info)."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import pyoracle as po
    from retrocam_b200 import scenes
    orc, ref = po.load(build=False)
    kind = "reference"
    if ref is None:
        kind = "port"
    sc = scenes.build_scene(w.scene, orc, po.MAT)
    cam = scenes.camera(w.orbit, w.lens, orc)
    W, H, spp = w.width, w.height, w.spp
    cores = threads or os.cpu_count()
    bufs = po.alloc_images(W, H)
    settings = (w.nee_enabled, w.nee_firefly_clamp)

    def render_rows(rows, frame):
        if ref is not None:
            ref.pathtrace(sc, cam, settings, W, H, frame, bufs, threads=cores, rows=rows)
        else:
            orc.render(sc, cam, settings, W, H, frame, 1, buffers=bufs, rows=rows, threads=cores)

    # path tracer: grow the row count until ~40% of the budget is spent
    render_rows((0, 16), 0)  # frame 0 (writes the G-buffer); warm
    rows, t = 16, 0.0
    while True:
        t0 = time.perf_counter()
        render_rows((H // 2 - rows // 2, H // 2 + rows // 2), 1)
        t = time.perf_counter() - t0
        if t > 0.4 * budget_s / 2 or rows >= H:
            break
        rows = min(H, rows * 2)
    t_sample = t / (rows * W)             # seconds per pixel-sample (centre rows)
    t_render = t_sample * W * H * spp
    info = {"render_rows": rows, "render_s": t}
    t_frame = t_render
    if w.sppm is not None and sc["light_count"] > 0:
        n_ph = 50_000
        while True:
            t0 = time.perf_counter()
            if ref is not None:
                ph, hd, nx, cnt = ref.photon_trace(sc, n_ph, w.sppm.r0, 6271, w.sppm.hash_size, threads=cores)
            else:
                ph, hd, nx, cnt, _ = orc.photon_trace(sc, n_ph, w.sppm.r0, 6271, w.sppm.hash_size, threads=cores)
            tp = time.perf_counter() - t0
            if tp > 0.15 * budget_s / 2 or n_ph >= w.sppm.photons:
                break
            n_ph = min(w.sppm.photons, n_ph * 4)
        t_trace = tp / n_ph * w.sppm.photons * w.sppm.iterations
        g_rows = max(8, rows // 2)
        t0 = time.perf_counter()
        if ref is not None:
            ref.photon_gather(sc, cam, W, H, w.sppm.r0, n_ph, w.sppm.hash_size, 0, ph, hd, nx, bufs[0],
                              threads=cores, rows=(H // 2 - g_rows // 2, H // 2 + g_rows // 2))
        else:
            orc.photon_gather(sc, cam, W, H, w.sppm.r0, w.sppm.hash_size, ph, hd, nx, bufs[0], threads=cores)
            g_rows = H
        tg = time.perf_counter() - t0
        t_gather = tg / (g_rows * W) * W * H * w.sppm.iterations
        t_frame += t_trace + t_gather
        info.update({"photons": n_ph, "photon_s": tp, "gather_rows": g_rows, "gather_s": tg})
    if w.atrous is not None and w.atrous.enabled:
        a_rows = max(8, rows // 2)
        out = np.zeros((H, W, 4), np.float32)
        col = orc.p00(bufs[0], W, H, 1, 1.0)
        t0 = time.perf_counter()
        if ref is not None:
            ref.atrous_pass(col, bufs[1], bufs[2], bufs[3], W, H, 16, w.atrous.sigma_color, w.atrous.sigma_normal,
                            w.atrous.sigma_depth, 1, 1.0, out, rows=(H // 2 - a_rows // 2, H // 2 + a_rows // 2),
                            threads=cores)
        else:
            orc.atrous_pass(col, bufs[1], bufs[2], bufs[3], W, H, 16, w.atrous.sigma_color, w.atrous.sigma_normal,
                            w.atrous.sigma_depth, 1, 1.0, threads=cores)
            a_rows = H
        ta = time.perf_counter() - t0
        t_frame += ta / (a_rows * W) * W * H * w.atrous.iterations
        info.update({"atrous_rows": a_rows, "atrous_s": ta})
    desc = (f"{kind} shaders on {cores} host threads: pathtrace {rows} centre rows x {W} px x 1 spp "
            f"({'3 LCA paths/sample' if any(w.lens.lca_delta) else '1 path/sample'})")
    if "photons" in info:
        desc += f"; photon trace {info['photons']} photons; gather {info['gather_rows']} rows"
    if "atrous_rows" in info:
        desc += f"; a-trous {info['atrous_rows']} rows x 1 pass"
    desc += f"; extrapolated to {W}x{H}x{spp} spp" + (
        f" + {w.sppm.iterations} SPPM iterations" if w.sppm is not None else "") + " + full denoise"
    return t_frame, {"kind": kind, "cores": cores, "sample": desc, "detail": info}


# ---------------------------------------------------------------------------
# reference arm
# ---------------------------------------------------------------------------
def run_reference(args):
    rank, _, world = dist_env()
    if rank != 0:
        return 0
    w, _, _ = workload_setup(args.workload, args)
    samples = w.width * w.height * w.spp
    budget = max(2.0, min(args.cpu_seconds, 240.0 / max(1, args.steps + args.warmup)))
    for _ in range(args.warmup):
        cpu_reference_sample(w, budget)
    times, info = [], None
    for _ in range(args.steps):
        t, info = cpu_reference_sample(w, budget)
        times.append(t)
    t_frame = statistics.mean(times)
    value = samples / t_frame / 1e6
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_frame * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": workload_config(w, args),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": info["cores"], "kind": info["kind"],
                             "sample": info["sample"]},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def time_to_relmse(args) -> dict:
    """The metric's second half: wall time (render + denoise, one frame at
    854x480) to reach mean relMSE <= 1e-2 against a 4096-spp render, path
    tracer + à-trous vs path tracer + the shipped learned denoiser, on
    held-out seeded Cornell variants (no dataset exists for this scene)."""
    from retrocam_b200 import kpcnn
    seeds = list(range(5000, 5000 + args.quality_variants))
    rep = kpcnn.evaluate(kpcnn.load(), seeds, spps=(1, 2, 4, 8, 16, 32, 64), ref_spp=4096, log=None)
    t = rep["time_to_threshold"]
    return {"threshold": rep["threshold"], "ref_spp": rep["ref_spp"], "variants": seeds,
            "plain_atrous": t["atrous"], "learned": t["learned"], "plain_no_denoiser": t["noisy"],
            "learned_speedup": rep["speedup_learned_vs_atrous"],
            "relmse_at_spp": {"spp": rep["spp"], "atrous": rep["relmse"]["atrous"],
                              "learned": rep["relmse"]["learned"]}}


def workload_config(w, args):
    cfg = {"workload": w.name, "width": w.width, "height": w.height, "spp": w.spp,
           "paths_per_sample": 3 if any(w.lens.lca_delta) else 1, "max_bounces": 6,
           "lens": f"{w.lens.focal_length_mm:g}mm f/{w.lens.f_stop:g} focus {w.lens.focus_dist_m:g} "
                   f"{w.lens.blades} blades",
           "math": args.math, "engine": args.engine, "parallelism": f"replicas x{args.gpus}",
           "l2": "scene (BVH + triangles) is L2-resident by design; the 854x480 images (6.6 MB accum) are "
                 "rewritten every step"}
    if w.sppm is not None:
        cfg["sppm"] = {"photons": w.sppm.photons, "hash": w.sppm.hash_size, "r0": w.sppm.r0,
                       "alpha": w.sppm.alpha, "iterations": w.sppm.iterations}
    if w.atrous is not None:
        cfg["atrous"] = {"passes": w.atrous.iterations, "sigma_n": w.atrous.sigma_normal,
                         "sigma_d": w.atrous.sigma_depth, "sigma_c": w.atrous.sigma_color}
    return cfg


# ---------------------------------------------------------------------------
# B200 arm
# ---------------------------------------------------------------------------
def run_b200(args):
    import torch
    from retrocam_b200 import api, build
    rank, local_rank, world = dist_env()
    build.build()
    torch.cuda.set_device(local_rank)
    device = torch.device("cuda", local_rank)
    dist = init_dist(world, "nccl")
    w, sppm, atrous = workload_setup(args.workload, args)
    sc = api.build_scene(w.scene)
    cam = api.workload_camera(w)
    mode = api.RC_MATH_EXACT if args.math == "exact" else api.RC_MATH_FAST
    ctx = api.Context(w.width, w.height, local_rank, mode)
    stream = torch.cuda.Stream(device=device)
    ctx.set_stream(stream.cuda_stream)
    ctx.upload(sc)
    settings = (w.nee_enabled, w.nee_firefly_clamp)
    iters = w.sppm.iterations if w.sppm is not None else 0
    r0 = w.sppm.r0 if w.sppm is not None else 0.05
    samples_per_step = w.width * w.height * w.spp
    if args.engine == "auto":
        from retrocam_b200 import autotune
        key = autotune.cache_key(torch.cuda.get_device_name(device), w.width, w.height, mode,
                                 autotune.scene_signature(sc))
        autotune.tuned(ctx, key, lambda: ctx.render_frame(cam, settings, w.spp, sppm, r0, iters, atrous,
                                                          read=False), retune=args.retune)
    else:
        ctx.set_engine({"wavefront": api.RC_ENGINE_WAVEFRONT, "wavefront_static": api.RC_ENGINE_WAVEFRONT_STATIC,
                        "megakernel": api.RC_ENGINE_MEGAKERNEL}[args.engine], args.chunk_paths)
    tuning = ctx.tuning()

    def step():
        ctx.render_frame(cam, settings, w.spp, sppm, r0, iters, atrous, read=False)

    # ---- device-resident timing ----
    for _ in range(args.warmup):
        step()
    ctx.synchronize()
    ctx.reset_counters()
    ctx.set_kernel_timing(True)
    ctx.kernel_times()
    barrier(dist, device)
    torch.cuda.synchronize()
    clocks = ClockSampler(local_rank)
    clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        step()
    ev1.record(stream)
    ev1.synchronize()
    torch.cuda.synchronize()
    clock_info = clocks.stop()
    barrier(dist, device)
    t_ms = ev0.elapsed_time(ev1)
    ctr = ctx.counters()
    ktimes = ctx.kernel_times()
    ctx.set_kernel_timing(False)
    t_ms_max = max_over_ranks(t_ms, dist, device)
    ms_per_step = t_ms_max / args.steps
    value = samples_per_step * world / (ms_per_step / 1e3) / 1e6
    if ctr["error_word"]:
        raise RuntimeError(f"kernel guard raised: {ctr['error_word']:#x}")

    # ---- end to end through the C ABI with host buffers (the export path:
    # scene upload, frame, display pass, RGBA8 read-back) ----
    out_pinned = torch.empty((w.height, w.width, 4), dtype=torch.uint8, pin_memory=True)

    def export_step():
        ctx.upload(sc)
        step()
        ctx.check(api.lib().rc_display(ctx.h, 1, 1.0, api.C.c_void_p(out_pinned.data_ptr())))

    for _ in range(max(1, args.warmup)):
        export_step()
    ctx.reset_counters()
    barrier(dist, device)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        export_step()
    e1.record(stream)
    e1.synchronize()
    e_ms = max_over_ranks(e0.elapsed_time(e1), dist, device)
    ectr = ctx.counters()
    e2e = {"value": samples_per_step * world / (e_ms / args.steps / 1e3) / 1e6, "unit": UNIT,
           "h2d_bytes_per_step": ectr["h2d_bytes"] // args.steps,
           "d2h_bytes_per_step": ectr["d2h_bytes"] // args.steps,
           "includes": "rc_scene_upload (host layout conversion + validation + H2D), rc_render_frame, "
                       "rc_display (ACES + sRGB to RGBA8) and the RGBA8 frame read back into pinned host "
                       "memory (the export path's result)"}

    # ---- roofline of the dominant kernel ----
    kernel, (k_ms, k_launches) = max(ktimes.items(), key=lambda kv: kv[1][0])
    per_launch_bytes = algorithmic_bytes(kernel, ctr, samples_per_step * args.steps) / max(1, k_launches)
    avg_launch_s = (k_ms / max(1, k_launches)) / 1e3
    peak, peak_kind = hbm_peak()
    achieved = per_launch_bytes / avg_launch_s / 1e9 if avg_launch_s > 0 else 0.0
    traffic = read_traffic(KERNEL_SYMBOL.get(kernel, kernel), w.name)
    fp32 = fp32_roofline(kernel, ctr, k_launches, avg_launch_s, local_rank)
    rays = ctr["closest_rays"] + ctr["shadow_rays"] + ctr["photon_rays"] + ctr["gather_rays"]
    kernels_total_ms = sum(v[0] for v in ktimes.values())
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural scene, no dataset)",
        "config": dict(workload_config(w, args), tuning=tuning),
        "e2e": e2e,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                     "kernel": KERNEL_SYMBOL.get(kernel, kernel), "algorithmic_bytes_per_launch": per_launch_bytes,
                     "avg_launch_ms": avg_launch_s * 1e3, "launches": k_launches, "fp32": fp32},
        "mrays_per_s": rays / (t_ms / 1e3) / 1e6,
        "kernel_ms": {k: v[0] / args.steps for k, v in ktimes.items()},
        "kernel_share": {k: (v[0] / kernels_total_ms if kernels_total_ms else 0.0) for k, v in ktimes.items()},
        "gpu_launches": int(ctr["kernel_launches"]),
        "clocks": clock_info,
        "counters_per_step": {k: ctr[k] / args.steps for k in
                              ("camera_paths", "closest_rays", "shadow_rays", "photon_rays", "gather_rays",
                               "node_tests", "tri_tests", "surface_hits", "light_samples")},
    }
    if rank == 0 and not args.no_quality:
        line["time_to_relmse"] = time_to_relmse(args)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        t_frame, info = cpu_reference_sample(w, args.cpu_seconds)
        line["cpu_baseline"] = {"value": samples_per_step / t_frame / 1e6, "unit": UNIT, "cores": info["cores"],
                                "kind": info["kind"], "sample": info["sample"]}
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))
    return 0


def run_keyframes(args):
    """The batched keyframe export: 64 frames of the export frame's scene on a
    keyframed orbit (spp U{8..128}, SPPM iterations U{4..16}), one
    rc_render_frames call per step under a CUDA graph.  value = samples of
    all frames / device time of the batch; e2e adds the read-back of every
    finished frame to host memory."""
    import torch
    from retrocam_b200 import api, autotune, build, scenes
    rank, local_rank, world = dist_env()
    build.build()
    torch.cuda.set_device(local_rank)
    device = torch.device("cuda", local_rank)
    dist = init_dist(world, "nccl")
    w = scenes.export_frame()
    sc = api.build_scene(w.scene)
    frames = scenes.keyframe_batch(api.HOST, 64, 1)
    sppm = api.rc_sppm_params(w.sppm.photons, w.sppm.hash_size, w.sppm.alpha)
    atrous = api.atrous_params(w.atrous)
    settings = (w.nee_enabled, w.nee_firefly_clamp)
    ctx = api.Context(w.width, w.height, local_rank, api.RC_MATH_FAST)
    stream = torch.cuda.Stream(device=device)
    ctx.set_stream(stream.cuda_stream)
    ctx.upload(sc)
    key = autotune.cache_key(torch.cuda.get_device_name(device), w.width, w.height, api.RC_MATH_FAST,
                             autotune.scene_signature(sc))
    t = autotune.TuningCache().get(key)
    if t:
        ctx.set_tuning(**t)
    samples = sum(s for _, s, _ in frames) * w.width * w.height

    def step(read=False):
        return ctx.render_frames(frames, settings, sppm, w.sppm.r0, atrous, use_graph=True, read=read)

    for _ in range(args.warmup):
        step()
    ctx.synchronize()
    ctx.reset_counters()
    barrier(dist, device)
    torch.cuda.synchronize()
    clocks = ClockSampler(local_rank)
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        step()
    ev1.record(stream)
    ev1.synchronize()
    clock_info = clocks.stop()
    t_ms = max_over_ranks(ev0.elapsed_time(ev1), dist, device) / args.steps
    ctr = ctx.counters()
    if ctr["error_word"]:
        raise RuntimeError(f"kernel guard raised: {ctr['error_word']:#x}")
    launches = int(ctr["kernel_launches"]) // args.steps
    ctx.reset_counters()
    barrier(dist, device)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step(read=True)
    e_ms = max_over_ranks((time.perf_counter() - t0) * 1e3, dist, device) / args.steps
    ectr = ctx.counters()
    line = {"metric": METRIC, "value": samples * world / (t_ms / 1e3) / 1e6, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded procedural scene and keyframes, no dataset)",
            "config": {"workload": "keyframes", "frames": len(frames), "width": w.width, "height": w.height,
                       "spp_total": sum(s for _, s, _ in frames),
                       "sppm_iterations_total": sum(i for _, _, i in frames),
                       "photon_maps_traced_per_batch": max(i for _, _, i in frames),
                       "graph": True, "tuning": ctx.tuning(), "parallelism": f"replicas x{world}"},
            "e2e": {"value": samples * world / (e_ms / 1e3) / 1e6, "unit": UNIT,
                    "h2d_bytes_per_step": ectr["h2d_bytes"] // args.steps,
                    "d2h_bytes_per_step": ectr["d2h_bytes"] // args.steps,
                    "includes": "rc_render_frames with all 64 finished frames read back to host memory"},
            "gpu_launches": launches, "clocks": clock_info}
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))
    return 0


def main(argv=None):
    args = parse_args(argv)
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "keyframes":
        return run_keyframes(args)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
