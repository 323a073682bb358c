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
  roofline  the dominant kernel (the wavefront trace): algorithmic bytes per
         launch from the kernel's own work counters (32 B per box test, 36 B
         per triangle test), divided by its CUDA-event time, against the
         measured HBM copy bandwidth; `bound` and `limiter` come from the
         committed ncu summary of the same kernel (the scene is cache-resident,
         so the kernel is issue-bound, not HBM-bound), `traffic` its DRAM
         bytes per launch
  exact_math  the same frame in the bit-exact build, and how many pixels of
         the fast build agree with it within 1e-4 at 1 spp
  cornell_small  the small Cornell box (256x256 x 16 spp) on the B200
  bvh_stress  the 1M-triangle scene (854x480 x 32 spp), device-resident
  keyframes  the 64-frame keyframed batch under one CUDA graph
  time_to_relmse  the metric's second half (64 held-out Cornell variants,
         every integer spp to 16, a 5x5 box filter as control); one GPU only
  cpu_baseline  the reference's own shaders compiled for the host
         (oracle/_ref, OpenMP over all host cores) on a bounded sample of the
         same workload: 1/16 of the frame (its centre eighth of rows at half
         the spp, with the SPPM and à-trous work in proportion), timed whole

Multi-GPU: one process per GPU (torchrun); the ranks split one export frame
(retrocam_b200/frame_split.py: each renders a contiguous share of the SPPM
iterations and their samples with rc_render_frame_part, then the
accumulation and variance images -- 20 bytes per pixel -- are summed onto
rank 0 with NCCL, which denoises and, for e2e, displays and reads back);
timing is the max over ranks and value is one frame's samples over that
time (strong scaling).

`--impl reference` times the reference's own CPU shaders on this host and
prints the same line with "impl": "reference" (rank 0 only): each step is
the 1/16 sample above, timed whole; the line adds the same sample with the
host C library's transcendental functions and a whole small-Cornell frame.
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
                 "photon_trace": "photon_bounce_kernel", "photon_gather": "photon_gather_kernel",
                 "atrous": "atrous_kernel", "wf_generate": "wf_generate", "wf_accumulate": "wf_accumulate",
                 "wf_sort": "wf_sort"}


def algorithmic_bytes(kernel: str, ctr: dict, samples: int) -> float:
    """Bytes the kernel must move at minimum for the work its counters record,
    in the path's own units: 32 B per ray-box test (6 floats + 2 ints), 36 B
    per ray-triangle test (v0, e1, e2), 104 B per shaded hit (3 normals +
    material index + the 64-B material), 80 B per light record, 20 B per
    pixel sample (accum + variance read-modify-write).  The wavefront's own
    path-state traffic (a design choice, not the algorithm's) is reported
    apart by `state_bytes`."""
    trav = BYTES_NODE_TEST * ctr["node_tests"] + BYTES_TRI_TEST * ctr["tri_tests"]
    if kernel == "render":
        return (trav + BYTES_SURFACE_HIT * ctr["surface_hits"] + BYTES_LIGHT_SAMPLE * ctr["light_samples"]
                + BYTES_SAMPLE_RMW * samples)
    if kernel == "wf_trace":
        return trav
    if kernel == "wf_shade":
        return (BYTES_SURFACE_HIT + 160) * ctr["surface_hits"] + BYTES_LIGHT_SAMPLE * ctr["light_samples"]
    if kernel in ("photon_trace", "photon_gather"):
        return BYTES_NODE_TEST * ctr["photon_node_tests"] + BYTES_TRI_TEST * ctr["photon_tri_tests"]
    return 0.0


def state_bytes(kernel: str, ctr: dict) -> float:
    """Path state the wavefront trace reads and writes per ray (origin and
    direction in, hit record out: 48 B per closest ray; the 48-B shadow
    record in, radiance read-modify-write: 80 B per shadow ray)."""
    if kernel == "wf_trace":
        return 48 * ctr["closest_rays"] + 80 * ctr["shadow_rays"]
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
    ap.add_argument("--material-queues", action="store_true",
                    help="shade each bounce's hits from material queues (rc_tuning.material_queues)")
    ap.add_argument("--tune", action="append", default=[], metavar="KNOB=VALUE",
                    help="set an rc_tuning knob after the autotuned shape (repeatable)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-quality", action="store_true", help="skip the time-to-relMSE comparison")
    ap.add_argument("--quality-variants", type=int, default=64, help="held-out Cornell variants for time-to-relMSE")
    ap.add_argument("--no-exact", action="store_true", help="skip the exact-math line")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the 1M-triangle and keyframed-batch lines")
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


PROFILE_FIELDS = ("traffic_bytes_per_launch", "bound", "simt_efficiency", "issue_active", "dram_throughput",
                  "l1_hit_rate", "warps_active")


def read_profile(kernel: str, workload: str) -> dict:
    """The machine-readable lines ('key: value') of the committed ncu summary
    profiles/ncu_<kernel>_<workload>.md: DRAM bytes per launch and the
    limiter counters of the same kernel."""
    path = os.path.join(REPO, "profiles", f"ncu_{kernel}_{workload}.md")
    out = {}
    if not os.path.exists(path):
        return out
    for line in open(path):
        key, _, val = line.strip().partition(":")
        if key in PROFILE_FIELDS and val.strip():
            v = val.strip().split()[0]
            try:
                out[key] = float(v)
            except ValueError:
                out[key] = v
    return out


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
class ReferenceFrame:
    """A bounded sample of a workload on the reference's own shaders compiled
    for the host (oracle/_ref; the oracle's restatement where that library
    is absent), OpenMP over the host's cores: the frame restricted to its
    `H/8` centre rows and `spp/2` samples -- 1/16 of the frame -- with the
    SPPM work in the same proportion (one iteration of the full photon count
    for the export frame's 16 iterations per 128 spp: same hash density and
    chain lengths) and the à-trous passes over those rows.  Per sample it
    does the export path's work in its order (trace photons, render the
    iteration's samples, gather, shrink the radius; denoise), so samples/s
    of the sample is samples/s of the frame."""

    def __init__(self, w, threads: int = 0, libm: bool = False):
        sys.path.insert(0, os.path.join(REPO, "oracle"))
        import pyoracle as po
        from retrocam_b200 import scenes
        self.po = po
        self.orc, self.ref = po.load(build=False)
        if libm:
            self.ref = po.load_reference_libm()
            if self.ref is None:
                raise RuntimeError("oracle/_ref/libretrocam_ref_libm.so is missing")
        self.kind = "reference" if self.ref is not None else "port"
        self.w = w
        self.sc = scenes.build_scene(w.scene, self.orc, po.MAT)
        self.cam = scenes.camera(w.orbit, w.lens, self.orc)
        self.cores = threads or os.cpu_count()
        W, H = w.width, w.height
        self.rows = max(8, H // 8)
        self.r0 = H // 2 - self.rows // 2
        self.spp = max(1, w.spp // 2)
        self.frac = (self.rows / H) * (self.spp / w.spp)
        self.iters, self.photons = 0, 0
        if w.sppm is not None and self.sc["light_count"] > 0:
            total = w.sppm.photons * w.sppm.iterations * self.frac
            self.iters = max(1, round(w.sppm.iterations * self.frac))
            self.photons = int(round(total / self.iters))
        self.bufs = po.alloc_images(W, H)
        self.samples = self.rows * W * self.spp

    def describe(self) -> str:
        w = self.w
        d = (f"{self.kind} shaders on {self.cores} host threads: {self.rows} centre rows x {w.width} px x "
             f"{self.spp} spp ({'3 LCA paths' if any(w.lens.lca_delta) else '1 path'} per sample)")
        if self.iters:
            d += f", {self.iters} SPPM iteration(s) of {self.photons} photons with the gather over those rows"
        if w.atrous is not None and w.atrous.enabled:
            d += f", {w.atrous.iterations} a-trous passes over those rows"
        return d + f" = 1/{round(1 / self.frac)} of one {w.width}x{w.height}x{w.spp}-spp frame, timed in full"

    def step(self) -> float:
        """Runs the sample once; returns its wall seconds."""
        w, sc, cam, ref, orc = self.w, self.sc, self.cam, self.ref, self.orc
        W, H = w.width, w.height
        rows = (self.r0, self.r0 + self.rows)
        settings = (w.nee_enabled, w.nee_firefly_clamp)
        acc = self.bufs[0]
        t0 = time.perf_counter()
        radius = w.sppm.r0 if w.sppm is not None else 0.0
        blocks = self.iters if self.iters else 1
        for k in range(blocks):
            s0, s1 = k * self.spp // blocks, (k + 1) * self.spp // blocks
            if self.iters:
                seed = k * 7919 + 6271
                if ref is not None:
                    ph, hd, nx, _ = ref.photon_trace(sc, self.photons, radius, seed, w.sppm.hash_size,
                                                     threads=self.cores)
                else:
                    ph, hd, nx, _, _ = orc.photon_trace(sc, self.photons, radius, seed, w.sppm.hash_size,
                                                        threads=self.cores)
            for f in range(s0, s1):
                if ref is not None:
                    ref.pathtrace(sc, cam, settings, W, H, f, self.bufs, threads=self.cores, rows=rows)
                else:
                    orc.render(sc, cam, settings, W, H, f, 1, buffers=self.bufs, rows=rows, threads=self.cores)
            if self.iters:
                if ref is not None:
                    ref.photon_gather(sc, cam, W, H, radius, self.photons, w.sppm.hash_size, 0, ph, hd, nx, acc,
                                      threads=self.cores, rows=rows)
                else:
                    orc.photon_gather(sc, cam, W, H, radius, w.sppm.hash_size, ph, hd, nx, acc,
                                      threads=self.cores)
                radius = orc.lib.or_sppm_next_radius(radius, k, w.sppm.alpha)
        if w.atrous is not None and w.atrous.enabled:
            a = orc.p00(acc, W, H, self.spp, w.atrous.exposure)
            out = np.zeros((H, W, 4), np.float32)
            for i in range(w.atrous.iterations):
                if ref is not None:
                    ref.atrous_pass(a, self.bufs[1], self.bufs[2], self.bufs[3], W, H, 1 << i,
                                    w.atrous.sigma_color, w.atrous.sigma_normal, w.atrous.sigma_depth, self.spp,
                                    w.atrous.exposure, out, rows=rows, threads=self.cores)
                else:
                    out = orc.atrous_pass(a, self.bufs[1], self.bufs[2], self.bufs[3], W, H, 1 << i,
                                          w.atrous.sigma_color, w.atrous.sigma_normal, w.atrous.sigma_depth,
                                          self.spp, w.atrous.exposure, threads=self.cores)
                a, out = out, a
        return time.perf_counter() - t0


def cpu_full_frame(name: str, threads: int = 0) -> dict:
    """A whole frame of a small workload on the compiled reference (the
    small Cornell box: 256x256 x 16 spp, no SPPM, no denoiser), timed once
    after one untimed frame."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import pyoracle as po
    from retrocam_b200 import scenes
    orc, ref = po.load(build=False)
    w = scenes.WORKLOADS[name]()
    sc = scenes.build_scene(w.scene, orc, po.MAT)
    cam = scenes.camera(w.orbit, w.lens, orc)
    cores = threads or os.cpu_count()
    settings = (w.nee_enabled, w.nee_firefly_clamp)

    def frame():
        bufs = po.alloc_images(w.width, w.height)
        t0 = time.perf_counter()
        if ref is not None:
            ref.render(sc, cam, settings, w.width, w.height, 0, w.spp, buffers=bufs, threads=cores)
        else:
            orc.render(sc, cam, settings, w.width, w.height, 0, w.spp, buffers=bufs, threads=cores)
        return time.perf_counter() - t0

    frame()
    t = frame()
    n = w.width * w.height * w.spp
    return {"workload": name, "value": n / t / 1e6, "unit": UNIT, "ms_per_frame": t * 1e3, "samples": n,
            "kind": "reference" if ref is not None else "port", "cores": cores,
            "sample": f"the whole {w.width}x{w.height}x{w.spp}-spp frame"}


# ---------------------------------------------------------------------------
# reference arm
# ---------------------------------------------------------------------------
def run_reference(args):
    rank, _, world = dist_env()
    if rank != 0:
        return 0
    w, _, _ = workload_setup(args.workload, args)
    rf = ReferenceFrame(w)
    for _ in range(args.warmup):
        rf.step()
    times = [rf.step() for _ in range(args.steps)]
    t = statistics.mean(times)
    value = rf.samples / t / 1e6
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": workload_config(w, args),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": rf.cores, "kind": rf.kind,
                             "sample": rf.describe()},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    try:
        lm = ReferenceFrame(w, libm=True)
        lm.step()
        tl = statistics.mean(lm.step() for _ in range(min(3, args.steps)))
        line["host_libm"] = {"value": lm.samples / tl / 1e6, "unit": UNIT, "ms_per_step": tl * 1e3,
                             "sample": "the same sample on the reference shaders built with the host C "
                                       "library's sinf/cosf/expf/logf/powf (a GL driver would use its own "
                                       "fast functions) instead of the correctly rounded ones parity uses"}
    except RuntimeError as e:
        line["host_libm"] = {"unavailable": str(e)}
    if w.name != "cornell_small":
        line["cornell_small_full_frame"] = cpu_full_frame("cornell_small")
    print(json.dumps(line))
    return 0


# every integer spp up to 32 (over the 64 held-out variants the à-trous path
# crosses 1e-2 between 16 and 32 spp), then 48 and 64
QUALITY_SPPS = tuple(range(1, 33)) + (48, 64)


def time_to_relmse(args) -> dict:
    """The metric's second half: wall time (render + denoise, one frame at
    854x480) to reach mean relMSE <= 1e-2 against a 4096-spp render, path
    tracer + à-trous vs path tracer + the shipped learned denoiser, on
    held-out seeded Cornell variants (no dataset exists for this scene), at
    every integer spp from 1 to 32.  The speed-up is reported against the
    path tracer + à-trous (the comparison the brief names) and against the
    faster of that and the path tracer alone (à-trous at low spp has no
    variance estimate and at high spp adds bias, so the undenoised image
    reaches 1e-2 first).  A plain 5x5 box average of the noisy image is
    evaluated beside them as a control."""
    from retrocam_b200 import kpcnn
    seeds = list(range(5000, 5000 + args.quality_variants))
    rep = kpcnn.evaluate(kpcnn.load(), seeds, spps=QUALITY_SPPS, ref_spp=4096, log=None)
    t = rep["time_to_threshold"]
    box_hit = [s for s, v in zip(rep["spp"], rep["relmse"]["box5"]) if v <= rep["threshold"]]
    return {"threshold": rep["threshold"], "ref_spp": rep["ref_spp"], "variants": len(seeds),
            "variant_seeds": [seeds[0], seeds[-1]],
            "plain_atrous": t["atrous"], "learned": t["learned"], "plain_no_denoiser": t["noisy"],
            "box5_control_spp": box_hit[0] if box_hit else None,
            "learned_speedup": rep["speedup_learned_vs_atrous"],
            "learned_speedup_vs_best_plain": (min(x["ms"] for x in (t["atrous"], t["noisy"]) if x) / t["learned"]["ms"]
                                              if t["learned"] and (t["atrous"] or t["noisy"]) else None),
            "relmse_at_spp": {"spp": rep["spp"], "noisy": rep["relmse"]["noisy"],
                              "atrous": rep["relmse"]["atrous"], "learned": rep["relmse"]["learned"],
                              "box5": rep["relmse"]["box5"]},
            "ms_at_spp": {"render": rep["ms"]["render"], "atrous": rep["ms"]["atrous"],
                          "learned": rep["ms"]["learned"]}}


def workload_config(w, args):
    cfg = {"workload": w.name, "width": w.width, "height": w.height, "spp": w.spp,
           "paths_per_sample": 3 if any(w.lens.lca_delta) else 1, "max_bounces": 6,
           "lens": f"{w.lens.focal_length_mm:g}mm f/{w.lens.f_stop:g} focus {w.lens.focus_dist_m:g} "
                   f"{w.lens.blades} blades",
           "math": args.math, "engine": args.engine,
           "parallelism": ("one frame split over %d GPUs by SPPM iterations, accum + variance summed onto rank 0"
                           % args.gpus) if args.gpus > 1 else "one GPU",
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
def device_timed(step, steps: int, warmup: int, stream) -> float:
    """Milliseconds per step on `stream` (CUDA events, synchronize on both
    sides) after `warmup` untimed steps."""
    import torch
    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        step()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / steps


def exact_math_line(args, w, sc, cam, sppm, atrous, fast_ctx, stream, device) -> dict:
    """The same frame in the exact build (no contraction, IEEE divide and
    square root, correctly rounded transcendentals, the reference's
    traversal order: the oracle's bits, so per-pixel agreement with the
    reference's shaders at any spp), timed like the headline; and, at 1 spp,
    how many pixels of the benchmarked fast build agree with it within
    1e-4 relative."""
    from retrocam_b200 import api
    settings = (w.nee_enabled, w.nee_firefly_clamp)
    iters = w.sppm.iterations if w.sppm is not None else 0
    r0 = w.sppm.r0 if w.sppm is not None else 0.05
    import torch
    from retrocam_b200 import autotune
    with api.Context(w.width, w.height, device.index, api.RC_MATH_EXACT) as ex:
        ex.set_stream(stream.cuda_stream)
        ex.upload(sc)
        # the autotuned shape for exact math when the table has one
        t = autotune.TuningCache().get(autotune.cache_key(torch.cuda.get_device_name(device), w.width, w.height,
                                                          api.RC_MATH_EXACT, autotune.scene_signature(sc)))
        if t:
            ex.set_tuning(**t)
        steps = max(1, min(args.steps, 5))
        ms = device_timed(lambda: ex.render_frame(cam, settings, w.spp, sppm, r0, iters, atrous, read=False),
                          steps, max(3, min(args.warmup, 3)), stream)
        if ex.counters()["error_word"]:
            raise RuntimeError("kernel guard raised in the exact build")
        # one more frame with per-kernel CUDA events: where the exact frame's time goes
        ex.set_kernel_timing(True)
        ex.kernel_times()
        ex.render_frame(cam, settings, w.spp, sppm, r0, iters, atrous, read=False)
        ex.synchronize()
        kt = {k: v[0] for k, v in ex.kernel_times().items() if v[1]}
        ex.set_kernel_timing(False)
        ex.reset()
        ex.render(cam, settings, 0, 1)
        a_ex = ex.read_buffers()[0]
        tuning = ex.tuning()
    fast_ctx.reset()
    fast_ctx.render(cam, settings, 0, 1)
    a_fa = fast_ctx.read_buffers()[0]
    rel = np.abs(a_fa[..., :3] - a_ex[..., :3]) / np.maximum(np.abs(a_ex[..., :3]), 1e-3)
    within = np.all(rel <= 1e-4, axis=-1)
    return {"value": w.width * w.height * w.spp / (ms / 1e3) / 1e6, "unit": UNIT, "ms_per_step": ms,
            "steps": steps, "tuning": tuning, "kernel_ms": kt,
            "fast_vs_exact_1spp": {"pixels_within_1e-4_rel": float(within.mean()),
                                   "pixels_bit_identical": float(np.all(a_fa[..., :3].view(np.uint32) ==
                                                                        a_ex[..., :3].view(np.uint32),
                                                                        axis=-1).mean()),
                                   "image_mean_rel_diff": float(abs(a_fa[..., :3].mean() - a_ex[..., :3].mean()) /
                                                                a_ex[..., :3].mean())}}


def converged_line(w, sc, cam, device, width=427, height=240) -> dict:
    """The path tracer's converged image (the export scene and lens, path
    tracing alone, half resolution): relMSE of the fast build at 1024 spp
    and of the exact build at the same samples, against an exact 4096-spp
    render on independent frame indices (2^20 on)."""
    from retrocam_b200 import api, kpcnn
    settings = (w.nee_enabled, w.nee_firefly_clamp)

    def mean_image(mode, first, spp):
        with api.Context(width, height, device.index, mode) as c:
            c.upload(sc)
            c.reset()
            c.render(cam, settings, first, spp)
            acc = c.read_buffers()[0]
        return acc[..., :3] / acc[..., 3:4]

    ref = mean_image(api.RC_MATH_EXACT, 1 << 20, 4096)
    fast = kpcnn.relmse(mean_image(api.RC_MATH_FAST, 0, 1024), ref)
    exact = kpcnn.relmse(mean_image(api.RC_MATH_EXACT, 0, 1024), ref)
    return {"relmse_fast_1024spp": fast, "relmse_exact_1024spp": exact, "bound": 1e-3,
            "reference": f"exact build, 4096 spp, independent seeds, {width}x{height}, path tracer alone"}


def small_cornell_line(args, stream, device) -> dict:
    """The small Cornell box (256x256, 16 spp, no SPPM, no denoiser) on the
    B200, device-resident, autotuned shape; the reference arm times the
    same whole frame on the host."""
    from retrocam_b200 import api, autotune, scenes
    w = scenes.cornell_small()
    sc = api.build_scene(w.scene)
    cam = api.workload_camera(w)
    settings = (w.nee_enabled, w.nee_firefly_clamp)
    with api.Context(w.width, w.height, device.index, api.RC_MATH_FAST) as c:
        c.set_stream(stream.cuda_stream)
        c.upload(sc)
        import torch
        key = autotune.cache_key(torch.cuda.get_device_name(device), w.width, w.height, api.RC_MATH_FAST,
                                 autotune.scene_signature(sc))
        t = autotune.TuningCache().get(key)
        if t:
            c.set_tuning(**t)
        ms = device_timed(lambda: c.render(cam, settings, 0, w.spp), max(args.steps, 10), max(args.warmup, 3), stream)
    return {"value": w.width * w.height * w.spp / (ms / 1e3) / 1e6, "unit": UNIT, "ms_per_frame": ms,
            "config": "256x256, 16 spp, 6 bounces, 35 mm f/16, 36 triangles"}


def stress_line(args, stream, device) -> dict:
    """The 1M-triangle scene (854x480, 32 spp, no SPPM, no denoiser; about
    160 MB of BVH and triangles, larger than L2), device-resident frames,
    autotuned shape (warm-up 3, then the timed frames)."""
    import torch
    from retrocam_b200 import api, autotune, scenes
    w = scenes.bvh_stress()
    t0 = time.perf_counter()
    sc = api.build_scene(w.scene)
    build_s = time.perf_counter() - t0
    cam = api.workload_camera(w)
    settings = (w.nee_enabled, w.nee_firefly_clamp)
    atrous = api.atrous_params(scenes.AtrousDesc(enabled=0))
    with api.Context(w.width, w.height, device.index, api.RC_MATH_FAST) as c:
        c.set_stream(stream.cuda_stream)
        c.upload(sc)
        key = autotune.cache_key(torch.cuda.get_device_name(device), w.width, w.height, api.RC_MATH_FAST,
                                 autotune.scene_signature(sc))
        t = autotune.TuningCache().get(key)
        if t:
            c.set_tuning(**t)
        ms = device_timed(lambda: c.render_frame(cam, settings, w.spp, None, 0.05, 0, atrous, read=False),
                          max(1, min(args.steps, 5)), 3, stream)
        ctr = c.counters()
    return {"value": w.width * w.height * w.spp / (ms / 1e3) / 1e6, "unit": UNIT, "ms_per_frame": ms,
            "triangles": len(sc["tris"]), "nodes": len(sc["nodes"]), "bvh_depth": int(ctr["bvh_depth"]),
            "host_bvh_build_s": build_s, "config": "854x480, 32 spp, 6 bounces, no SPPM, no denoiser"}


def keyframes_line(args, stream, device) -> dict:
    """The 64-frame keyframed batch (spp U{8..128}, SPPM iterations U{4..16})
    as one rc_render_frames call under a CUDA graph: samples of all frames
    over the device time of the batch (one warm-up batch, which also
    captures the graph, then two timed)."""
    from retrocam_b200 import api, autotune, scenes
    import torch
    w = scenes.export_frame()
    sc = api.build_scene(w.scene)
    frames = scenes.keyframe_batch(api.HOST, 64, 1)
    sppm = api.rc_sppm_params(w.sppm.photons, w.sppm.hash_size, w.sppm.alpha)
    atrous = api.atrous_params(w.atrous)
    settings = (w.nee_enabled, w.nee_firefly_clamp)
    with api.Context(w.width, w.height, device.index, api.RC_MATH_FAST) as c:
        c.set_stream(stream.cuda_stream)
        c.upload(sc)
        key = autotune.cache_key(torch.cuda.get_device_name(device), w.width, w.height, api.RC_MATH_FAST,
                                 autotune.scene_signature(sc))
        t = autotune.TuningCache().get(key)
        if t:
            c.set_tuning(**t)
        ms = device_timed(lambda: c.render_frames(frames, settings, sppm, w.sppm.r0, atrous, use_graph=True,
                                                  read=False), 2, 1, stream)
        if c.counters()["error_word"]:
            raise RuntimeError("kernel guard raised in the keyframed batch")
    samples = sum(s for _, s, _ in frames) * w.width * w.height
    return {"value": samples / (ms / 1e3) / 1e6, "unit": UNIT, "ms_per_batch": ms, "frames": len(frames),
            "spp_total": sum(s for _, s, _ in frames), "sppm_iterations_total": sum(i for _, _, i in frames),
            "config": "64 keyframed export frames, one rc_render_frames call under a CUDA graph"}


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
    if args.material_queues:
        ctx.set_tuning(material_queues=1)
    for kv in args.tune:
        k, _, v = kv.partition("=")
        ctx.set_tuning(**{k: int(v)})
    tuning = ctx.tuning()

    if world > 1:
        from retrocam_b200 import frame_split

        def step():
            # one frame over all ranks: a share of the SPPM iterations each,
            # then accum + variance summed onto rank 0 (NCCL), denoised there
            frame_split.render_frame_split(ctx, dist, stream, cam, settings, w.spp, sppm, r0, iters, atrous)
    else:
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
    # one frame per step on any number of GPUs (strong scaling)
    value = samples_per_step / (ms_per_step / 1e3) / 1e6
    if ctr["error_word"]:
        raise RuntimeError(f"kernel guard raised: {ctr['error_word']:#x}")

    # ---- end to end through the C ABI with host buffers (the export path:
    # scene upload, frame, display pass, RGBA8 read-back) ----
    out_pinned = torch.empty((w.height, w.width, 4), dtype=torch.uint8, pin_memory=True)

    def export_step():
        ctx.upload(sc)
        step()
        if rank == 0:
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
    e2e = {"value": samples_per_step / (e_ms / args.steps / 1e3) / 1e6, "unit": UNIT,
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
    prof = read_profile(KERNEL_SYMBOL.get(kernel, kernel), w.name)
    traffic = prof.get("traffic_bytes_per_launch")
    fp32 = fp32_roofline(kernel, ctr, k_launches, avg_launch_s, local_rank)
    rays = ctr["closest_rays"] + ctr["shadow_rays"] + ctr["photon_rays"] + ctr["gather_rays"]
    kernels_total_ms = sum(v[0] for v in ktimes.values())
    roofline = {"bound": prof.get("bound", "hbm"), "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                "kernel": KERNEL_SYMBOL.get(kernel, kernel), "algorithmic_bytes_per_launch": per_launch_bytes,
                "state_bytes_per_launch": state_bytes(kernel, ctr) / max(1, k_launches),
                "traffic_over_algorithmic": (traffic / per_launch_bytes) if traffic and per_launch_bytes else None,
                "avg_launch_ms": avg_launch_s * 1e3, "launches": k_launches,
                "limiter": {k: prof[k] for k in ("simt_efficiency", "issue_active", "dram_throughput",
                                                 "l1_hit_rate", "warps_active") if k in prof},
                "fp32": fp32}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural scene, no dataset)",
        "config": dict(workload_config(w, args), tuning=tuning),
        "e2e": e2e,
        "roofline": roofline,
        "mrays_per_s": rays / (t_ms / 1e3) / 1e6,
        "kernel_ms": {k: v[0] / args.steps for k, v in ktimes.items()},
        "kernel_share": {k: (v[0] / kernels_total_ms if kernels_total_ms else 0.0) for k, v in ktimes.items()},
        "gpu_launches": int(ctr["kernel_launches"]),
        "clocks": clock_info,
        "counters_per_step": {k: ctr[k] / args.steps for k in
                              ("camera_paths", "closest_rays", "shadow_rays", "photon_rays", "gather_rays",
                               "node_tests", "tri_tests", "surface_hits", "light_samples")},
    }
    if world == 1 and not args.no_exact:
        line["exact_math"] = exact_math_line(args, w, sc, cam, sppm, atrous, ctx, stream, device)
    if world == 1 and args.workload != "cornell_small":
        line["cornell_small"] = small_cornell_line(args, stream, device)
    if world == 1 and not args.no_exact:
        line["converged"] = converged_line(w, sc, cam, device)
    if world == 1 and args.workload == "export_frame" and not args.no_configs:
        line["bvh_stress"] = stress_line(args, stream, device)
        line["keyframes"] = keyframes_line(args, stream, device)
    if rank == 0 and world == 1 and not args.no_quality:
        line["time_to_relmse"] = time_to_relmse(args)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rf = ReferenceFrame(w)
        rf.step()
        t_cpu = rf.step()
        line["cpu_baseline"] = {"value": rf.samples / t_cpu / 1e6, "unit": UNIT, "cores": rf.cores,
                                "kind": rf.kind, "sample": rf.describe(), "ms": t_cpu * 1e3}
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
