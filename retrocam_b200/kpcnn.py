"""The learned denoiser: parameters, training driver, data and evaluation.

The network and its kernels are in csrc/kpcnn.cu (BF16 tcgen05
convolutions, FP32 accumulation); this module drives them through the C ABI
(`rc_kp_*` building blocks on device buffers, `rc_denoise_learned` for
inference on a context).  PyTorch provides device memory and the stream
only; no torch operator runs on the training or inference path.

Data: the path tracer renders randomised Cornell boxes
(`scenes.cornell_variant`) at 854x480; each variant gives noisy inputs at
1, 4 and 16 spp (nested sample sets) and an independent high-spp target
(different frame indices, hence independent PCG streams).

Loss: the evaluation metric itself, relMSE = mean (x - r)^2 / (r^2 + 0.01)
over pixels and channels, on random 128x128 crops; Adam.
"""
from __future__ import annotations

import ctypes as C
import os
import time

import numpy as np

from retrocam_b200 import api, scenes

P = api.RC_KPCNN_PARAMS
# offsets into the parameter vector (layer: W[tap][co][ci], then bias[32])
W1, B1 = 0, 9 * 32 * 16
W2, B2 = B1 + 32, B1 + 32 + 9 * 32 * 32
W3, B3 = B2 + 32, B2 + 32 + 9 * 32 * 32
WH, BH = B3 + 32, B3 + 32 + 9 * 32 * 32
assert BH + 32 == P
PACKED_ELEMS = (9 * 32 * 16,) + (9 * 32 * 32,) * 6
IN_CHANNELS = 10
TAPS = 25

WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "kpcnn_weights.npz")


def init_params(seed: int = 0) -> np.ndarray:
    """He-normal hidden layers; a small head so the first filters are close
    to a uniform 5x5 average."""
    rng = np.random.default_rng(seed)
    p = np.zeros(P, np.float32)
    w1 = rng.normal(0, np.sqrt(2.0 / (9 * IN_CHANNELS)), (9, 32, 16)).astype(np.float32)
    w1[:, :, IN_CHANNELS:] = 0
    p[W1:B1] = w1.ravel()
    for w in (W2, W3):
        p[w:w + 9 * 32 * 32] = rng.normal(0, np.sqrt(2.0 / (9 * 32)), 9 * 32 * 32).astype(np.float32)
    wh = rng.normal(0, 0.01, (9, 32, 32)).astype(np.float32)
    wh[:, TAPS:, :] = 0
    p[WH:BH] = wh.ravel()
    return p


def save(path: str, params: np.ndarray, **meta) -> None:
    np.savez(path, params=params.astype(np.float32), **{k: np.asarray(v) for k, v in meta.items()})


def load(path: str = WEIGHTS) -> np.ndarray:
    with np.load(path) as z:
        p = z["params"].astype(np.float32)
    if p.size != P:
        raise ValueError(f"{path}: {p.size} parameters, expected {P}")
    return p


def relmse(x: np.ndarray, ref: np.ndarray) -> float:
    """mean over pixels and RGB of (x - ref)^2 / (ref^2 + 1e-2)."""
    x = x[..., :3].astype(np.float64)
    r = ref[..., :3].astype(np.float64)
    return float(np.mean((x - r) ** 2 / (r * r + 1e-2)))


def _ptr(t) -> C.c_void_p:
    return C.c_void_p(t.data_ptr())


def _ck(code: int, what: str) -> None:
    if code != api.RC_OK:
        raise api.RetroCamError(code, what)


class Network:
    """Device state of one network: fp32 parameters and their bf16 packed
    copies, with the forward and backward passes over NHWC batches."""

    def __init__(self, params: np.ndarray, device, stream):
        import torch
        self.torch = torch
        self.dev = device
        self.stream = stream
        self.params = torch.from_numpy(np.ascontiguousarray(params, np.float32)).to(device)
        self.packed = [torch.zeros(n, dtype=torch.bfloat16, device=device) for n in PACKED_ELEMS]
        self.err = torch.zeros(1, dtype=torch.int32, device=device)
        self.pack()

    @property
    def sptr(self):
        return C.c_void_p(self.stream.cuda_stream)

    def pack(self):
        arr = (C.c_void_p * 7)(*[t.data_ptr() for t in self.packed])
        _ck(api.lib().rc_kp_pack(_ptr(self.params), arr, self.sptr), "rc_kp_pack")

    def conv(self, x, cin, layer, out, relu, out_f32=False, mask=None, backward=False, n=1, h=1, w=1):
        """layer: 0..3 (1, 2, 3, head); backward uses the flipped/transposed
        copy (layers 1..3 only) and no bias."""
        wpk = self.packed[4 + layer - 1] if backward else self.packed[layer]
        bias = None if backward else C.c_void_p(self.params.data_ptr() + 4 * (B1, B2, B3, BH)[layer])
        _ck(api.lib().rc_kp_conv3x3(_ptr(x), cin, _ptr(wpk), bias, _ptr(out), int(out_f32), int(relu),
                                    _ptr(mask) if mask is not None else None, n, h, w, _ptr(self.err), self.sptr),
            "rc_kp_conv3x3")

    def check(self):
        self.stream.synchronize()
        e = int(self.err.item())
        if e:
            raise api.RetroCamError(api.RC_ERR_DEVICE_GUARD, f"kpcnn kernel guard {e:#x}")


class Trainer:
    """Adam on random crops of a device-resident data set."""

    def __init__(self, params: np.ndarray, batch: int = 16, crop: int = 128, lr: float = 2e-3, device=None):
        import torch
        self.torch = torch
        self.dev = device or torch.device("cuda", 0)
        self.stream = torch.cuda.Stream(device=self.dev)
        self.net = Network(params, self.dev, self.stream)
        self.B, self.S, self.lr = batch, crop, lr
        B, S = batch, crop
        z = lambda *shape, dt=torch.float32: torch.zeros(*shape, dtype=dt, device=self.dev)  # noqa: E731
        bf = torch.bfloat16
        self.x = z(B, S, S, 16, dt=bf)
        self.color, self.target, self.out = z(B, S, S, 4), z(B, S, S, 4), z(B, S, S, 4)
        self.a1, self.a2, self.a3 = z(B, S, S, 32, dt=bf), z(B, S, S, 32, dt=bf), z(B, S, S, 32, dt=bf)
        self.logits = z(B, S, S, 32)
        self.dlog, self.d3, self.d2, self.d1 = (z(B, S, S, 32, dt=bf) for _ in range(4))
        self.grads, self.m, self.v = z(P), z(P), z(P)
        self.loss = z(1, dt=torch.float64)
        self.idx = torch.zeros(4, B, dtype=torch.int32, device=self.dev)
        self.step_count = 0

    def forward(self, n, h, w, x, a1, a2, a3, logits):
        net = self.net
        net.conv(x, 16, 0, a1, relu=True, n=n, h=h, w=w)
        net.conv(a1, 32, 1, a2, relu=True, n=n, h=h, w=w)
        net.conv(a2, 32, 2, a3, relu=True, n=n, h=h, w=w)
        net.conv(a3, 32, 3, logits, relu=False, out_f32=True, n=n, h=h, w=w)

    def backward(self, n, h, w):
        L, net, e = api.lib(), self.net, _ptr(self.net.err)
        g = self.grads.data_ptr()
        s = net.sptr
        wg = lambda x, cin, dy, wo, bo: _ck(L.rc_kp_wgrad(_ptr(x), cin, _ptr(dy), C.c_void_p(g + 4 * wo),  # noqa: E731
                                                          C.c_void_p(g + 4 * bo), n, h, w, e, s), "rc_kp_wgrad")
        wg(self.a3, 32, self.dlog, WH, BH)
        net.conv(self.dlog, 32, 3, self.d3, relu=False, mask=self.a3, backward=True, n=n, h=h, w=w)
        wg(self.a2, 32, self.d3, W3, B3)
        net.conv(self.d3, 32, 2, self.d2, relu=False, mask=self.a2, backward=True, n=n, h=h, w=w)
        wg(self.a1, 32, self.d2, W2, B2)
        net.conv(self.d2, 32, 1, self.d1, relu=False, mask=self.a1, backward=True, n=n, h=h, w=w)
        wg(self.x, 16, self.d1, W1, B1)

    def step(self, data: "Dataset", rng: np.random.Generator, lr: float) -> None:
        torch, B, S = self.torch, self.B, self.S
        src = rng.integers(0, data.n_inputs, B)
        idx = np.stack([src, data.target_of[src], rng.integers(0, data.H - S + 1, B),
                        rng.integers(0, data.W - S + 1, B)]).astype(np.int32)
        with torch.cuda.stream(self.stream):
            self.idx.copy_(torch.from_numpy(idx), non_blocking=False)
        L, s = api.lib(), self.net.sptr
        _ck(L.rc_kp_crop(_ptr(data.feat), _ptr(data.color), _ptr(data.target), _ptr(self.idx[0]), _ptr(self.idx[1]),
                         _ptr(self.idx[2]), _ptr(self.idx[3]), B, data.H, data.W, S, _ptr(self.x), _ptr(self.color),
                         _ptr(self.target), s), "rc_kp_crop")
        self.forward(B, S, S, self.x, self.a1, self.a2, self.a3, self.logits)
        _ck(L.rc_kp_head(_ptr(self.logits), _ptr(self.color), _ptr(self.target), _ptr(self.out), _ptr(self.dlog),
                         _ptr(self.loss), 1.0 / (B * S * S * 3), B, S, S, s), "rc_kp_head")
        self.backward(B, S, S)
        self.step_count += 1
        _ck(L.rc_kp_adam(_ptr(self.net.params), _ptr(self.grads), _ptr(self.m), _ptr(self.v), P, lr, 0.9, 0.999,
                         1e-8, self.step_count, s), "rc_kp_adam")
        self.net.pack()

    def train(self, data: "Dataset", steps: int, seed: int = 0, log_every: int = 250, log=print) -> list:
        rng = np.random.default_rng(seed)
        hist = []
        t0 = time.perf_counter()
        for i in range(steps):
            lr = self.lr * 0.5 * (1.0 + np.cos(np.pi * i / steps)) + 1e-5
            self.step(data, rng, lr)
            if (i + 1) % log_every == 0 or i + 1 == steps:
                self.net.check()
                loss = float(self.loss.item()) / (log_every * self.B * self.S * self.S * 3)
                self.loss.zero_()
                hist.append((i + 1, loss))
                if log:
                    log(f"step {i + 1}: train relMSE {loss:.5f} ({time.perf_counter() - t0:.1f} s)")
        self.net.check()
        return hist

    def params(self) -> np.ndarray:
        self.stream.synchronize()
        return self.net.params.cpu().numpy()


class Dataset:
    """Device-resident inputs (features + noisy radiance) and targets."""

    def __init__(self, n_inputs, n_targets, H, W, device):
        import torch
        self.H, self.W, self.n_inputs = H, W, n_inputs
        self.feat = torch.zeros(n_inputs, H, W, 16, dtype=torch.bfloat16, device=device)
        self.color = torch.zeros(n_inputs, H, W, 4, dtype=torch.float32, device=device)
        self.target = torch.zeros(n_targets, H, W, 4, dtype=torch.float32, device=device)
        self.target_of = np.zeros(n_inputs, np.int64)


def render_dataset(seeds, input_spps=(1, 4, 16), target_spp=1024, width=854, height=480, device=None,
                   log=print) -> Dataset:
    """Renders each seed's Cornell variant: nested noisy inputs at
    `input_spps` and an independent `target_spp` target."""
    import torch
    device = device or torch.device("cuda", 0)
    data = Dataset(len(seeds) * len(input_spps), len(seeds), height, width, device)
    scratch = torch.zeros(height, width, 16, dtype=torch.bfloat16, device=device)
    t0 = time.perf_counter()
    with api.Context(width, height, device.index or 0, api.RC_MATH_FAST) as ctx:
        for vi, seed in enumerate(seeds):
            w = scenes.cornell_variant(seed, width, height)
            ctx.upload(api.build_scene(w.scene))
            cam = api.workload_camera(w)
            settings = (w.nee_enabled, w.nee_firefly_clamp)
            ctx.reset()
            done = 0
            for li, spp in enumerate(input_spps):
                ctx.render(cam, settings, done, spp - done)
                done = spp
                k = vi * len(input_spps) + li
                ctx.kp_features(data.feat[k].data_ptr(), data.color[k].data_ptr())
                data.target_of[k] = vi
            ctx.reset()
            ctx.render(cam, settings, 1 << 20, target_spp)
            ctx.kp_features(scratch.data_ptr(), data.target[vi].data_ptr())
            ctx.synchronize()
            if log and (vi + 1) % 32 == 0:
                log(f"rendered {vi + 1}/{len(seeds)} variants ({time.perf_counter() - t0:.1f} s)")
    return data


def _timed(ctx, fn) -> float:
    """Milliseconds of fn() on the context's stream (synchronize on both sides)."""
    ctx.synchronize()
    t0 = time.perf_counter()
    fn()
    ctx.synchronize()
    return (time.perf_counter() - t0) * 1e3


def box5(img: np.ndarray) -> np.ndarray:
    """5x5 box average with edge clamping (the control filter: equal weights
    over the learned filter's footprint, no features)."""
    p = np.pad(img.astype(np.float64), ((2, 2), (2, 2), (0, 0)), mode="edge")
    c = np.cumsum(np.cumsum(p, axis=0), axis=1)
    c = np.pad(c, ((1, 0), (1, 0), (0, 0)))
    H, W = img.shape[:2]
    s = c[5:5 + H, 5:5 + W] - c[0:H, 5:5 + W] - c[5:5 + H, 0:W] + c[0:H, 0:W]
    return (s / 25.0).astype(np.float32)


def evaluate(params: np.ndarray, seeds, spps=(1, 2, 4, 8, 16, 32, 64, 128, 256), ref_spp=4096, width=854,
             height=480, threshold=1e-2, log=print) -> dict:
    """relMSE against an independent `ref_spp` render, for the path tracer
    plus à-trous (5 passes, sigma_n 128, sigma_d 1, sigma_c 1), plus the
    learned denoiser, and plus a plain 5x5 box average (a control: what the
    learned filter's footprint gives with equal weights) at equal spp; wall
    time of render + denoise per frame.  `time_to_threshold` is, per
    method, the time at the smallest spp of `spps` whose mean relMSE over
    the variants is <= threshold (None if none is)."""
    atrous = api.atrous_params(scenes.AtrousDesc(max_spp=0))
    res = {"spp": list(spps), "ref_spp": ref_spp, "variants": list(seeds), "width": width, "height": height,
           "relmse": {"noisy": [], "atrous": [], "learned": [], "box5": []},
           "ms": {"render": [], "atrous": [], "learned": []}}
    per = {k: np.zeros((len(seeds), len(spps))) for k in ("noisy", "atrous", "learned", "box5", "render",
                                                           "t_atrous", "t_learned")}
    with api.Context(width, height, 0, api.RC_MATH_FAST) as ctx:
        for vi, seed in enumerate(seeds):
            w = scenes.cornell_variant(seed, width, height)
            ctx.upload(api.build_scene(w.scene))
            cam = api.workload_camera(w)
            st = (w.nee_enabled, w.nee_firefly_clamp)
            ctx.reset()
            ctx.render(cam, st, 1 << 21, ref_spp)
            acc = ctx.read_buffers()[0]
            ref = acc[..., :3] / np.maximum(acc[..., 3:4], 1)
            # first calls allocate their scratch: keep that out of the timings
            ctx.denoise(atrous, read=False)
            ctx.denoise_learned(params, read=False)
            for si, k in enumerate(spps):
                ctx.reset()
                per["render"][vi, si] = _timed(ctx, lambda: ctx.render(cam, st, 0, k))
                acc = ctx.read_buffers()[0]
                noisy = acc[..., :3] / np.maximum(acc[..., 3:4], 1)
                per["noisy"][vi, si] = relmse(noisy, ref)
                per["box5"][vi, si] = relmse(box5(noisy), ref)
                per["t_atrous"][vi, si] = _timed(ctx, lambda: ctx.denoise(atrous, read=False))
                per["atrous"][vi, si] = relmse(ctx.read_output(), ref)
                per["t_learned"][vi, si] = _timed(ctx, lambda: ctx.denoise_learned(params, read=False))
                per["learned"][vi, si] = relmse(ctx.read_output(), ref)
                if ctx.counters()["error_word"]:
                    raise api.RetroCamError(api.RC_ERR_DEVICE_GUARD, "kernel guard during evaluation")
            if log:
                log(f"variant {seed}: atrous {np.round(per['atrous'][vi], 4).tolist()} "
                    f"learned {np.round(per['learned'][vi], 4).tolist()}")
    for k in ("noisy", "atrous", "learned", "box5"):
        res["relmse"][k] = per[k].mean(axis=0).tolist()
    res["ms"]["render"] = per["render"].mean(axis=0).tolist()
    res["ms"]["atrous"] = per["t_atrous"].mean(axis=0).tolist()
    res["ms"]["learned"] = per["t_learned"].mean(axis=0).tolist()
    ttt = {}
    for k, tk in (("noisy", None), ("atrous", "atrous"), ("learned", "learned")):
        hit = [i for i, v in enumerate(res["relmse"][k]) if v <= threshold]
        if hit:
            i = hit[0]
            t = res["ms"]["render"][i] + (res["ms"][tk][i] if tk else 0.0)
            ttt[k] = {"spp": spps[i], "ms": t}
        else:
            ttt[k] = None
    res["threshold"] = threshold
    res["time_to_threshold"] = ttt
    a, l_ = ttt.get("atrous"), ttt.get("learned")
    res["speedup_learned_vs_atrous"] = (a["ms"] / l_["ms"]) if (a and l_) else None
    return res


def time_inference(params: np.ndarray, width=854, height=480, calls=20) -> dict:
    """Wall and CUDA-event milliseconds of one rc_denoise_learned call on a
    1-spp render of a held-out Cornell variant (3 untimed calls first)."""
    w = scenes.cornell_variant(5000, width, height)
    with api.Context(width, height, 0, api.RC_MATH_FAST) as ctx:
        ctx.upload(api.build_scene(w.scene))
        ctx.render(api.workload_camera(w), (w.nee_enabled, w.nee_firefly_clamp), 0, 1)
        for _ in range(3):
            ctx.denoise_learned(params, read=False)
        ctx.synchronize()
        ctx.set_kernel_timing(True)
        ctx.kernel_times()
        n0 = ctx.counters()["kernel_launches"]
        t0 = time.perf_counter()
        for _ in range(calls):
            ctx.denoise_learned(params, read=False)
        ctx.synchronize()
        wall = (time.perf_counter() - t0) / calls * 1e3
        kt = ctx.kernel_times()
        launches = (ctx.counters()["kernel_launches"] - n0) // calls
        ctx.set_kernel_timing(False)
    # one call = features and four convolutions (the head in the last); the
    # weights were packed by the first call
    return {"wall_ms": wall, "kernel_ms": kt["kpcnn"][0] / calls, "launches_per_call": launches}


def _main(argv=None) -> int:
    """Renders the training set, trains, saves the weights, evaluates."""
    import argparse
    import json
    ap = argparse.ArgumentParser(description=_main.__doc__)
    ap.add_argument("--variants", type=int, default=192)
    ap.add_argument("--target-spp", type=int, default=1024)
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--eval-variants", type=int, default=8)
    ap.add_argument("--ref-spp", type=int, default=4096)
    ap.add_argument("--out", default=WEIGHTS)
    ap.add_argument("--report", default="")
    ap.add_argument("--eval-only", action="store_true")
    ap.add_argument("--time-inference", action="store_true",
                    help="time rc_denoise_learned on a 1-spp 854x480 frame (3 warm-up + 20 timed calls)")
    args = ap.parse_args(argv)
    if args.time_inference:
        print(json.dumps(time_inference(load(args.out))))
        return 0
    if args.eval_only:
        params = load(args.out)
    else:
        data = render_dataset(range(1000, 1000 + args.variants), target_spp=args.target_spp)
        tr = Trainer(init_params(0), batch=args.batch, lr=args.lr)
        t0 = time.perf_counter()
        hist = tr.train(data, args.steps)
        train_s = time.perf_counter() - t0
        params = tr.params()
        del data
        save(args.out, params, steps=args.steps, variants=args.variants, target_spp=args.target_spp,
             batch=args.batch, train_seconds=train_s, final_train_relmse=hist[-1][1])
        print(f"trained {args.steps} steps in {train_s:.1f} s; saved {args.out}")
    rep = evaluate(params, range(5000, 5000 + args.eval_variants), ref_spp=args.ref_spp)
    print(json.dumps({k: rep[k] for k in ("relmse", "time_to_threshold", "speedup_learned_vs_atrous")}))
    if args.report:
        with open(args.report, "w") as f:
            json.dump(rep, f, indent=1)
    return 0


if __name__ == "__main__":
    raise SystemExit(_main())
