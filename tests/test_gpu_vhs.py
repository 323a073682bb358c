"""The VHS chain on the GPU against the reference's own pass shaders
compiled for the host (oracle/_ref): every pass bit for bit, at several
frame indices (the dropout and tracking events depend on them) and with
the default and a heavy setting; the whole chain through rc_post_vhs on a
denoised frame, then displayed."""
import ctypes as C

import numpy as np
import pytest

from conftest import bits

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def T(product, cuda_ok):
    import torch
    return torch


@pytest.fixture(scope="module")
def c1(product, orc, cuda_ok):
    import pyoracle as po
    from retrocam_b200 import scenes
    w = scenes.export_frame()
    return w, scenes.build_scene(w.scene, orc, po.MAT), scenes.camera(w.orbit, w.lens, orc)


def _image(W, H, seed):
    rng = np.random.default_rng(seed)
    img = (rng.random((H, W, 4)) * 1.05).astype(np.float32)
    # bright spots (CCD smear threshold), a dark stripe, a hard vertical edge
    img[rng.integers(0, H, 12), rng.integers(0, W, 12), :3] = 3.0
    img[H // 3:H // 3 + 2] *= 0.02
    img[:, W // 2:, :3] *= 0.3
    return img


HEAVY = dict(tape_age=1.0, dropout_burst_rate=1.0, dropout_bright=1.0, tracking_severity=1.0,
             agc_gain=4.0, ccd_smear_intensity=0.5, ccd_smear_length=60, head_switch_lines=20,
             color_hue_rot=12.0, color_temp_bias=0.6, edge_enhance_amount=2.5, interlace_comb_strength=4.0)


@pytest.mark.parametrize("setting", ["default", "heavy"])
@pytest.mark.parametrize("frame", [0, 57, 1001, 40000])
def test_every_pass_bit_identical(product, ref, T, setting, frame):
    W, H = 97, 61
    img = _image(W, H, frame)
    p = product.vhs_defaults(frame_index=frame, time_s=frame / 29.97, **(HEAVY if setting == "heavy" else {}))
    src = T.from_numpy(img).cuda()
    dst = T.zeros_like(src)
    for k in product.VHS_PASSES:
        assert product.lib().rc_vhs_pass(k, C.c_void_p(src.data_ptr()), C.c_void_p(dst.data_ptr()), W, H,
                                         C.byref(p), None) == 0
        T.cuda.synchronize()
        got = dst.cpu().numpy()
        want = ref.post_pass(k, img, W, H, p)
        if not np.array_equal(bits(got), bits(want)):
            bad = np.argwhere(bits(got) != bits(want))
            raise AssertionError(f"pass {k}: {len(bad)} words differ, first {bad[:3].tolist()}")


def test_chain_on_a_denoised_frame_then_display(product, ref, orc, c1):
    w, sc, cam = c1
    W, H = 96, 64
    p = product.vhs_defaults(passes=product.VHS_PASSES, frame_index=90, time_s=3.0, **HEAVY)
    a = product.rc_atrous_params(1, 5, 1.0, 128.0, 1.0, 0, 1.0)
    with product.Context(W, H, 0, product.RC_MATH_EXACT) as ctx:
        ctx.upload(sc)
        ctx.render(cam, (1, 1.0), 0, 2)
        den = ctx.denoise(a)
        out = ctx.post_vhs(p, read=True)
        img = ctx.display()
        again = ctx.post_vhs(product.vhs_defaults(), read=True)   # nothing enabled: unchanged
    want = den
    for k in product.VHS_PASSES:
        want = ref.post_pass(k, want, W, H, p)
    np.testing.assert_array_equal(bits(out), bits(want))
    np.testing.assert_array_equal(bits(again), bits(out))
    np.testing.assert_array_equal(img, orc.display(want, W, H, 1, 1.0))
