"""The VHS chain's host side: rc_vhs_defaults gives RenderSettings' values
(core/RenderSettings.java:49-191) with every pass off, and the ctypes mirror
has the C layout; bad arguments are refused without a GPU."""
import ctypes as C

import numpy as np


def test_defaults_are_render_settings(product):
    p = product.vhs_defaults()
    f32 = lambda v: float(np.float32(v))   # noqa: E731
    want = {"enabled": 0, "frame_index": 0, "agc_gain": 1.0, "luma_blur_sigma": 1.5, "chroma_res_sigma": 7.0,
            "color_saturation": f32(0.95), "color_drift_speed": f32(0.05), "dr_black_lift": f32(0.01),
            "dr_shadow_crush": f32(0.03), "dr_highlight_knee": f32(0.78), "dr_highlight_clip": f32(0.95),
            "ccd_noise_luma_base": f32(0.015), "ccd_noise_chroma_scale": f32(1.6), "ccd_smear_threshold": f32(0.85),
            "ccd_smear_intensity": f32(0.009), "ccd_smear_length": 20, "chroma_bleed_factor": f32(0.35),
            "timebase_amplitude_px": 1.5, "timebase_freq": f32(0.02), "timebase_speed": f32(0.7),
            "dot_crawl_intensity": 0.25, "dot_crawl_subcarrier": f32(0.14), "dot_crawl_edge_thresh": f32(0.04),
            "tape_age": f32(0.3), "dropout_bright": f32(0.92), "dropout_burst_rate": f32(0.45),
            "head_switch_lines": 12, "head_switch_jitter": 4.0, "head_switch_ripple": f32(0.1),
            "head_switch_chroma": f32(0.35), "tracking_severity": f32(0.1), "tracking_max_displace_px": 28.0,
            "tracking_fringe_width_px": 4.0, "edge_enhance_amount": 1.5, "edge_enhance_core_threshold": f32(0.025),
            "interlace_field_offset_px": 0.5, "interlace_comb_strength": 1.5,
            "interlace_comb_edge_thresh": f32(0.04), "interlace_line_weighting": f32(0.05)}
    for k, v in want.items():
        assert getattr(p, k) == v, k
    assert C.sizeof(product.rc_vhs_params) == 4 * 42
    q = product.vhs_defaults(passes=(1, 3, 16), tape_age=1.0)
    assert q.enabled == (1 | 4 | 1 << 15) and q.tape_age == 1.0


def test_bad_pass_arguments(product):
    p = product.vhs_defaults()
    L = product.lib()
    buf = (C.c_float * 16)()
    for pass_ in (0, 5, 6, 17):
        assert L.rc_vhs_pass(pass_, buf, C.byref(buf, 32), 1, 1, C.byref(p), None) == product.RC_ERR_INVALID_ARG
    assert L.rc_vhs_pass(1, buf, buf, 1, 1, C.byref(p), None) == product.RC_ERR_INVALID_ARG   # in place
    assert L.rc_vhs_pass(1, buf, C.byref(buf, 32), 0, 1, C.byref(p), None) == product.RC_ERR_INVALID_ARG
    assert L.rc_post_vhs(None, C.byref(p)) == product.RC_ERR_INVALID_ARG
