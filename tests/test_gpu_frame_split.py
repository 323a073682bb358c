"""A frame split into parts on the GPU (rc_render_frame_part), merged through
the contexts' device images as retrocam_b200/frame_split.py merges them
across ranks -- here two contexts on one device stand in for two ranks, and
the sum is a torch add on zero-copy views of the images instead of a NCCL
reduce (this run has one GPU).

One part of one is the whole frame: bit for bit rc_render_frame's images
and denoised frame in exact math without SPPM (with it, within the gather's
insertion-order tolerance).  Two parts summed: the G-buffer and albedo bit
for bit, the sums within the tolerance of another float addition order,
the denoised frame within the tolerance of the CPU split test
(test_frame_split.py).
"""
import numpy as np
import pytest

from conftest import bits

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def frame(product, cuda_ok):
    from retrocam_b200 import scenes
    w = scenes.export_frame()
    return w, product.build_scene(w.scene), product.workload_camera(w)


ARGS = dict(W=96, H=54, spp=8, iters=4, N=50_000, hs=1 << 18, r0=0.02)


def _whole(product, sc, cam, atrous, iters):
    a = ARGS
    sppm = product.rc_sppm_params(a["N"], a["hs"], 0.7)
    with product.Context(a["W"], a["H"], 0, product.RC_MATH_EXACT) as ctx:
        ctx.upload(sc)
        out = ctx.render_frame(cam, (1, 1.0), a["spp"], sppm, a["r0"], iters, atrous)
        return ctx.read_buffers(), out


@pytest.mark.parametrize("iters", [0, 4])
def test_one_part_is_the_whole_frame(product, frame, iters):
    """Without SPPM bit for bit; with it the gather sums each cell's photons
    in the order GPU atomics inserted them, so accum agrees within the
    gather tolerance of the other tests (2e-5) and the rest bit for bit."""
    from retrocam_b200 import scenes
    w, sc, cam = frame
    a = ARGS
    atrous = product.atrous_params(scenes.AtrousDesc())
    sppm = product.rc_sppm_params(a["N"], a["hs"], 0.7)
    bufs, out = _whole(product, sc, cam, atrous, iters)
    with product.Context(a["W"], a["H"], 0, product.RC_MATH_EXACT) as ctx:
        ctx.upload(sc)
        ctx.render_frame_part(cam, (1, 1.0), a["spp"], sppm, a["r0"], iters, 0, 1)
        assert ctx.total_samples == a["spp"]
        part = ctx.read_buffers()
        ctx.set_total_samples(a["spp"])
        got = ctx.denoise(atrous)
    if iters == 0:
        for g, c in zip(part, bufs):
            assert np.array_equal(bits(g), bits(c))
        assert np.array_equal(bits(got), bits(out))
    else:
        np.testing.assert_allclose(part[0], bufs[0], rtol=2e-5, atol=1e-6)
        for g, c in zip(part[1:], bufs[1:]):
            assert np.array_equal(bits(g), bits(c))
        np.testing.assert_allclose(got, out, rtol=1e-3, atol=1e-4)


@pytest.mark.parametrize("mode", ["exact", "fast"])
def test_two_parts_merged_in_place(product, frame, mode):
    import torch
    from retrocam_b200 import frame_split, scenes
    w, sc, cam = frame
    a = ARGS
    m = product.RC_MATH_EXACT if mode == "exact" else product.RC_MATH_FAST
    atrous = product.atrous_params(scenes.AtrousDesc())
    sppm = product.rc_sppm_params(a["N"], a["hs"], 0.7)
    dev = torch.device("cuda", 0)
    ctxs = [product.Context(a["W"], a["H"], 0, m) for _ in range(2)]
    try:
        for p, ctx in enumerate(ctxs):
            ctx.upload(sc)
            ctx.render_frame_part(cam, (1, 1.0), a["spp"], sppm, a["r0"], a["iters"], p, 2)
            ctx.synchronize()
        assert [c.total_samples for c in ctxs] == [4, 4]
        acc0, var0 = frame_split.image_tensors(ctxs[0], dev)
        acc1, var1 = frame_split.image_tensors(ctxs[1], dev)
        acc0 += acc1
        var0 += var1
        torch.cuda.synchronize()
        ctxs[0].set_total_samples(a["spp"])
        merged = ctxs[0].read_buffers()
        got = ctxs[0].denoise(atrous)
        for c in ctxs:
            assert c.counters()["error_word"] == 0
    finally:
        for c in ctxs:
            c.close()
    with product.Context(a["W"], a["H"], 0, m) as ctx:
        ctx.upload(sc)
        want = ctx.render_frame(cam, (1, 1.0), a["spp"], sppm, a["r0"], a["iters"], atrous)
        whole = ctx.read_buffers()
    np.testing.assert_array_equal(merged[0][..., 3], whole[0][..., 3])
    assert np.array_equal(merged[1], whole[1]) and np.array_equal(merged[2], whole[2])
    if mode == "exact":
        # the same terms, summed as two part sums (and the gather in
        # insertion order): only the rounding differs
        np.testing.assert_allclose(merged[0], whole[0], rtol=2e-5, atol=1e-6)
        np.testing.assert_allclose(merged[3], whole[3], rtol=1e-5, atol=1e-6)
        np.testing.assert_allclose(got, want, rtol=1e-3, atol=1e-4)
    else:
        # fast math: the gather sums photons in insertion order (GPU
        # atomics), so the two runs of one part already differ by rounding
        np.testing.assert_allclose(merged[0], whole[0], rtol=1e-3, atol=1e-4)
        assert abs(got.mean() - want.mean()) <= 1e-4 * abs(want.mean())
