"""The learned denoiser's tensor-core kernels against plain PyTorch fp32
references of the same operations (conv2d, its weight and input gradients,
softmax filtering), on BF16-representable inputs.

Tolerances: products of BF16 operands are exact in FP32, so FP32 outputs
differ from torch only by summation order (rel 1e-4 of the sum of |terms|);
BF16 outputs are additionally rounded once (2^-8 relative).
"""
import ctypes as C

import numpy as np
import pytest

from conftest import bits

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def T(product, cuda_ok):
    import torch
    return torch


def _p(t):
    return C.c_void_p(t.data_ptr())


def _pack_fwd(T, W, cin):
    """[9][32][cin] -> packed [9][cin/8][32][8] bf16."""
    return W.reshape(9, 32, cin // 8, 8).permute(0, 2, 1, 3).contiguous().to(T.bfloat16)


def _pack_bwd(T, W):
    """Flipped/transposed copy [tap'][co/8][ci][8] of W[8 - tap'][co][ci]."""
    Wf = W.flip(0)                                    # [tap'][co][ci]
    return Wf.reshape(9, 4, 8, 32).permute(0, 1, 3, 2).contiguous().to(T.bfloat16)


def _tw(T, W, cin):
    """torch conv2d weight [co][ci][3][3] of W[tap][co][ci]."""
    return W.reshape(3, 3, 32, cin).permute(2, 3, 0, 1).contiguous()


def _nchw(x):
    return x.permute(0, 3, 1, 2)


def _close_bf16(got, ref):
    got, ref = got.float(), ref.float()
    tol = 2.0 ** -7 * ref.abs() + 1e-3
    bad = (got - ref).abs() > tol
    assert not bool(bad.any()), f"{int(bad.sum())} of {bad.numel()} differ; max {float((got - ref).abs().max())}"


@pytest.mark.parametrize("cin", [16, 32])
@pytest.mark.parametrize("mode", ["relu_bf16", "f32", "mask_bf16"])
def test_conv3x3_matches_torch(product, T, cin, mode):
    g = T.Generator(device="cuda").manual_seed(cin)
    n, h, w = 2, 5, 300            # three 128-pixel tiles per row, the last partial
    x = T.randn(n, h, w, cin, device="cuda", generator=g).to(T.bfloat16)
    W = (T.randn(9, 32, cin, device="cuda", generator=g) * 0.2).to(T.bfloat16).float()
    bias = T.randn(32, device="cuda", generator=g)
    mask = T.randn(n, h, w, 32, device="cuda", generator=g).to(T.bfloat16) if mode == "mask_bf16" else None
    out = T.zeros(n, h, w, 32, device="cuda", dtype=T.float32 if mode == "f32" else T.bfloat16)
    err = T.zeros(1, dtype=T.int32, device="cuda")
    wpk = _pack_fwd(T, W, cin)
    rc = product.lib().rc_kp_conv3x3(_p(x), cin, _p(wpk), _p(bias), _p(out), int(mode == "f32"),
                                     int(mode == "relu_bf16"), _p(mask) if mask is not None else None, n, h, w,
                                     _p(err), None)
    assert rc == 0
    T.cuda.synchronize()
    assert int(err.item()) == 0
    ref = T.nn.functional.conv2d(_nchw(x.float()), _tw(T, W, cin), bias, padding=1).permute(0, 2, 3, 1)
    if mode == "relu_bf16":
        ref = T.relu(ref)
    if mode == "mask_bf16":
        ref = ref * (mask.float() > 0)
    if mode == "f32":
        scale = T.nn.functional.conv2d(_nchw(x.float().abs()), _tw(T, W.abs(), cin), bias.abs(),
                                       padding=1).permute(0, 2, 3, 1)
        assert bool(((out - ref).abs() <= 1e-4 * scale + 1e-6).all())
    else:
        _close_bf16(out, ref)


@pytest.mark.parametrize("cin", [16, 32])
def test_wgrad_matches_torch(product, T, cin):
    g = T.Generator(device="cuda").manual_seed(100 + cin)
    n, h, w = 2, 7, 200
    x = T.randn(n, h, w, cin, device="cuda", generator=g).to(T.bfloat16)
    dy = T.randn(n, h, w, 32, device="cuda", generator=g).to(T.bfloat16)
    dw = T.zeros(9, 32, cin, device="cuda")
    db = T.zeros(32, device="cuda")
    err = T.zeros(1, dtype=T.int32, device="cuda")
    assert product.lib().rc_kp_wgrad(_p(x), cin, _p(dy), _p(dw), _p(db), n, h, w, _p(err), None) == 0
    T.cuda.synchronize()
    assert int(err.item()) == 0
    ref = T.nn.grad.conv2d_weight(_nchw(x.float()), (32, cin, 3, 3), _nchw(dy.float()), padding=1)
    ref = ref.permute(2, 3, 0, 1).reshape(9, 32, cin)
    scale = T.nn.grad.conv2d_weight(_nchw(x.float().abs()), (32, cin, 3, 3), _nchw(dy.float().abs()), padding=1)
    scale = scale.permute(2, 3, 0, 1).reshape(9, 32, cin)
    assert bool(((dw - ref).abs() <= 1e-4 * scale + 1e-5).all()), float((dw - ref).abs().max())
    dbr = dy.float().sum(dim=(0, 1, 2))
    assert bool(((db - dbr).abs() <= 1e-4 * dy.float().abs().sum(dim=(0, 1, 2)) + 1e-5).all())


def test_backward_data_conv_matches_torch(product, T):
    g = T.Generator(device="cuda").manual_seed(7)
    n, h, w = 1, 6, 260
    W = (T.randn(9, 32, 32, device="cuda", generator=g) * 0.2).to(T.bfloat16).float()
    dy = T.randn(n, h, w, 32, device="cuda", generator=g).to(T.bfloat16)
    act = T.randn(n, h, w, 32, device="cuda", generator=g).to(T.bfloat16)
    out = T.zeros(n, h, w, 32, device="cuda", dtype=T.bfloat16)
    err = T.zeros(1, dtype=T.int32, device="cuda")
    assert product.lib().rc_kp_conv3x3(_p(dy), 32, _p(_pack_bwd(T, W)), None, _p(out), 0, 0, _p(act), n, h, w,
                                       _p(err), None) == 0
    T.cuda.synchronize()
    ref = T.nn.grad.conv2d_input((n, 32, h, w), _tw(T, W, 32), _nchw(dy.float()), padding=1).permute(0, 2, 3, 1)
    _close_bf16(out, ref * (act.float() > 0))


def test_pack_layouts(product, T):
    from retrocam_b200 import kpcnn
    p = np.random.default_rng(3).normal(size=kpcnn.P).astype(np.float32)
    params = T.from_numpy(p).cuda()
    packed = [T.zeros(k, dtype=T.bfloat16, device="cuda") for k in kpcnn.PACKED_ELEMS]
    arr = (C.c_void_p * 7)(*[t.data_ptr() for t in packed])
    assert product.lib().rc_kp_pack(_p(params), arr, None) == 0
    T.cuda.synchronize()
    W1 = params[kpcnn.W1:kpcnn.B1].reshape(9, 32, 16)
    assert T.equal(packed[0].view(-1), _pack_fwd(T, W1, 16).view(-1))
    for i, off in enumerate((kpcnn.W2, kpcnn.W3, kpcnn.WH)):
        Wl = params[off:off + 9 * 32 * 32].reshape(9, 32, 32)
        assert T.equal(packed[1 + i].view(-1), _pack_fwd(T, Wl, 32).view(-1))
        assert T.equal(packed[4 + i].view(-1), _pack_bwd(T, Wl).view(-1))


def _head_ref(T, logits, color, target):
    n, h, w, _ = logits.shape
    lg = logits[..., :25].clone().requires_grad_(True)
    wts = T.softmax(lg, dim=-1)
    c = _nchw(color[..., :3])
    cp = T.nn.functional.pad(c, (2, 2, 2, 2), mode="replicate")
    patches = cp.unfold(2, 5, 1).unfold(3, 5, 1)           # n, 3, h, w, 5, 5
    patches = patches.reshape(n, 3, h, w, 25).permute(0, 2, 3, 4, 1)   # n h w 25 3
    out = (wts[..., None] * patches).sum(dim=-2)
    r = target[..., :3]
    terms = (out - r) ** 2 / (r * r + 0.01)
    loss = terms.sum()
    loss.backward()
    return out.detach(), float(loss), lg.grad


def test_head_forward_and_gradient(product, T):
    g = T.Generator(device="cuda").manual_seed(11)
    n, h, w = 2, 9, 140
    logits = T.randn(n, h, w, 32, device="cuda", generator=g) * 2
    color = T.rand(n, h, w, 4, device="cuda", generator=g) * 3
    target = T.rand(n, h, w, 4, device="cuda", generator=g) * 3
    out = T.zeros(n, h, w, 4, device="cuda")
    dlog = T.zeros(n, h, w, 32, device="cuda", dtype=T.bfloat16)
    loss = T.zeros(1, device="cuda", dtype=T.float64)
    scale = 0.5
    assert product.lib().rc_kp_head(_p(logits), _p(color), _p(target), _p(out), _p(dlog), _p(loss),
                                    C.c_float(scale), n, h, w, None) == 0
    T.cuda.synchronize()
    ro, rl, rg = _head_ref(T, logits, color, target)
    assert T.allclose(out[..., :3], ro, rtol=1e-5, atol=1e-5)
    assert abs(float(loss.item()) - rl) <= 1e-5 * abs(rl)
    _close_bf16(dlog[..., :25], rg * scale)
    assert not bool(dlog[..., 25:].float().any())


def test_adam_step(product, T):
    rng = np.random.default_rng(5)
    p, gr = rng.normal(size=1000).astype(np.float32), rng.normal(size=1000).astype(np.float32)
    m, v = rng.normal(size=1000).astype(np.float32) * 0.1, rng.random(1000).astype(np.float32) * 0.1
    tp, tg, tm, tv = (T.from_numpy(a.copy()).cuda() for a in (p, gr, m, v))
    assert product.lib().rc_kp_adam(_p(tp), _p(tg), _p(tm), _p(tv), 1000, C.c_float(1e-3), C.c_float(0.9),
                                    C.c_float(0.999), C.c_float(1e-8), 3, None) == 0
    T.cuda.synchronize()
    m2 = 0.9 * m + 0.1 * gr
    v2 = 0.999 * v + 0.001 * gr * gr
    p2 = p - 1e-3 * (m2 / (1 - 0.9 ** 3)) / (np.sqrt(v2 / (1 - 0.999 ** 3)) + 1e-8)
    np.testing.assert_allclose(tp.cpu().numpy(), p2, rtol=1e-5, atol=1e-6)
    assert not tg.any()


def _net_ref(T, params, feat, color):
    """Torch fp32 forward with the kernels' BF16 rounding points."""
    from retrocam_b200 import kpcnn
    P = T.from_numpy(params).cuda()
    x = _nchw(feat.float())

    def conv(x, w0, b0, cin, relu):
        W = P[w0:w0 + 9 * 32 * cin].reshape(9, 32, cin).to(T.bfloat16).float()
        y = T.nn.functional.conv2d(x, _tw(T, W, cin), P[b0:b0 + 32], padding=1)
        return T.relu(y).to(T.bfloat16).float() if relu else y

    a = conv(x, kpcnn.W1, kpcnn.B1, 16, True)
    a = conv(a, kpcnn.W2, kpcnn.B2, 32, True)
    a = conv(a, kpcnn.W3, kpcnn.B3, 32, True)
    lg = conv(a, kpcnn.WH, kpcnn.BH, 32, False).permute(0, 2, 3, 1)
    out, _, _ = _head_ref(T, lg, color, T.zeros_like(color))
    return out


def test_denoise_learned_matches_torch_network(product, T):
    """rc_denoise_learned on a rendered frame: features from the context's
    images, four convolutions and the filter, against the same network in
    torch fp32 (BF16 at the same points)."""
    from retrocam_b200 import kpcnn, scenes
    w = scenes.cornell_variant(3, 200, 96)
    sc = product.build_scene(w.scene)
    cam = product.workload_camera(w)
    params = kpcnn.init_params(1)
    params[kpcnn.WH:kpcnn.BH] *= 30.0    # peaked filters, so a wrong tap shows
    with product.Context(200, 96, 0, product.RC_MATH_FAST) as ctx:
        ctx.upload(sc)
        ctx.render(cam, (1, 1.0), 0, 4)
        feat = T.zeros(1, 96, 200, 16, dtype=T.bfloat16, device="cuda")
        color = T.zeros(1, 96, 200, 4, device="cuda")
        ctx.kp_features(feat.data_ptr(), color.data_ptr())
        out = ctx.denoise_learned(params)
        assert ctx.counters()["error_word"] == 0
    ref = _net_ref(T, params, feat, color)[0].cpu().numpy()
    got = out[..., :3]
    # a few logits straddle a bf16 rounding boundary differently: per-pixel
    # agreement for nearly all pixels, and the frame mean
    close = np.abs(got - ref) <= 2e-2 * np.abs(ref) + 1e-3
    assert np.mean(np.all(close, axis=-1)) > 0.995
    assert abs(got.mean() - ref.mean()) <= 1e-3 * abs(ref.mean())


def test_fused_head_equals_separate_head(product, T):
    """Inference applies the head in the last convolution's epilogue; the
    same four convolutions with the logits written out and the separate
    head kernel (the training path) give the same bits."""
    import ctypes as C
    from retrocam_b200 import kpcnn, scenes
    H, W = 96, 200
    w = scenes.cornell_variant(4, W, H)
    params = kpcnn.init_params(2)
    params[kpcnn.WH:kpcnn.BH] *= 30.0
    with product.Context(W, H, 0, product.RC_MATH_FAST) as ctx:
        ctx.upload(product.build_scene(w.scene))
        ctx.render(product.workload_camera(w), (1, 1.0), 0, 2)
        feat = T.zeros(1, H, W, 16, dtype=T.bfloat16, device="cuda")
        color = T.zeros(1, H, W, 4, device="cuda")
        ctx.kp_features(feat.data_ptr(), color.data_ptr())
        fused = ctx.denoise_learned(params)
        ctx.synchronize()
    stream = T.cuda.current_stream()
    net = kpcnn.Network(params, T.device("cuda", 0), stream)
    bf = T.bfloat16
    a1, a2, a3 = (T.zeros(1, H, W, 32, dtype=bf, device="cuda") for _ in range(3))
    logits = T.zeros(1, H, W, 32, device="cuda")
    out = T.zeros(1, H, W, 4, device="cuda")
    net.conv(feat, 16, 0, a1, relu=True, n=1, h=H, w=W)
    net.conv(a1, 32, 1, a2, relu=True, n=1, h=H, w=W)
    net.conv(a2, 32, 2, a3, relu=True, n=1, h=H, w=W)
    net.conv(a3, 32, 3, logits, relu=False, out_f32=True, n=1, h=H, w=W)
    assert product.lib().rc_kp_head(_p(logits), _p(color), None, _p(out), None, None, C.c_float(0.0), 1, H, W,
                                    C.c_void_p(stream.cuda_stream)) == 0
    net.check()
    np.testing.assert_array_equal(bits(fused), bits(out[0].cpu().numpy()))


def test_features_layout(product, T):
    from retrocam_b200 import scenes
    w = scenes.cornell_variant(5, 64, 48)
    with product.Context(64, 48, 0, product.RC_MATH_FAST) as ctx:
        ctx.upload(product.build_scene(w.scene))
        ctx.render(product.workload_camera(w), (1, 1.0), 0, 2)
        feat = T.zeros(48, 64, 16, dtype=T.bfloat16, device="cuda")
        color = T.zeros(48, 64, 4, device="cuda")
        ctx.kp_features(feat.data_ptr(), color.data_ptr())
        ctx.synchronize()
        acc, gb, ga, _ = ctx.read_buffers()
    c = acc[..., :3] / np.maximum(acc[..., 3:4], 1)
    np.testing.assert_allclose(color.cpu().numpy()[..., :3], c, rtol=1e-6)
    f = feat.float().cpu().numpy()
    np.testing.assert_allclose(f[..., :3], np.log1p(np.maximum(c, 0)), rtol=1e-2, atol=1e-2)
    np.testing.assert_allclose(f[..., 3:6], ga.view(np.float16)[..., :3].astype(np.float32), rtol=1e-2, atol=1e-3)
    np.testing.assert_allclose(f[..., 6:9], gb.view(np.float16)[..., :3].astype(np.float32), rtol=1e-2, atol=1e-3)
    t = gb.view(np.float16)[..., 3].astype(np.float32)
    np.testing.assert_allclose(f[..., 9], t / (1 + np.abs(t)), rtol=1e-2, atol=1e-3)
    assert not f[..., 10:].any()


def test_shipped_weights_beat_atrous_on_held_out_variant(product, T):
    """The shipped network, on a Cornell variant outside its training seeds
    at 4 spp, lands under relMSE 1e-2 and well under the à-trous filter."""
    from retrocam_b200 import kpcnn, scenes
    params = kpcnn.load()
    W, H = 320, 180
    w = scenes.cornell_variant(6001, W, H)
    cam = product.workload_camera(w)
    with product.Context(W, H, 0, product.RC_MATH_FAST) as ctx:
        ctx.upload(product.build_scene(w.scene))
        ctx.render(cam, (1, 1.0), 1 << 21, 1024)
        acc = ctx.read_buffers()[0]
        ref = acc[..., :3] / acc[..., 3:4]
        ctx.reset()
        ctx.render(cam, (1, 1.0), 0, 4)
        a = kpcnn.relmse(ctx.denoise(product.atrous_params(scenes.AtrousDesc())), ref)
        l_ = kpcnn.relmse(ctx.denoise_learned(params), ref)
    assert l_ < 1e-2 and l_ < 0.5 * a, (l_, a)


def test_weights_repacked_only_when_they_change(product, T):
    """A context keeps the packed weights between calls with the same
    parameters (one launch fewer) and repacks when they change: alternating
    two parameter vectors on one context gives each vector's own output."""
    from retrocam_b200 import kpcnn, scenes
    H, W = 64, 160
    w = scenes.cornell_variant(6, W, H)
    pa, pb = kpcnn.init_params(3), kpcnn.init_params(4)
    pa[kpcnn.WH:kpcnn.BH] *= 30.0
    pb[kpcnn.WH:kpcnn.BH] *= 30.0
    outs = {}
    for name, p in (("a", pa), ("b", pb)):
        with product.Context(W, H, 0, product.RC_MATH_FAST) as ctx:
            ctx.upload(product.build_scene(w.scene))
            ctx.render(product.workload_camera(w), (1, 1.0), 0, 2)
            outs[name] = ctx.denoise_learned(p)
    with product.Context(W, H, 0, product.RC_MATH_FAST) as ctx:
        ctx.upload(product.build_scene(w.scene))
        ctx.render(product.workload_camera(w), (1, 1.0), 0, 2)
        seq = []
        for p in (pa, pa, pb, pb, pa):
            n0 = ctx.counters()["kernel_launches"]
            seq.append((ctx.denoise_learned(p), ctx.counters()["kernel_launches"] - n0))
    assert [n for _, n in seq] == [6, 5, 6, 5, 6]
    for (img, _), name in zip(seq, "aabba"):
        np.testing.assert_array_equal(bits(img), bits(outs[name]))
    assert not np.array_equal(bits(outs["a"]), bits(outs["b"]))
