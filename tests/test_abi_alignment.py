"""Entry points that take raw device pointers refuse misaligned ones (their
kernels use 16-, 8- or 4-byte vector accesses; a misaligned address would
fault the device) and out-of-range sizes, before touching the device, so
these checks run without a GPU.  The pointers below are never dereferenced:
validation fails first."""
import ctypes as C

import pytest

A16 = C.c_void_p(1 << 20)          # 16-byte aligned stand-ins
BAD = C.c_void_p((1 << 20) + 4)    # 4-byte aligned only
ERR = C.c_void_p((1 << 20) + 64)


def test_vhs_pass_alignment_and_size(product):
    L = product.lib()
    p = product.vhs_defaults()
    inv = product.RC_ERR_INVALID_ARG
    assert L.rc_vhs_pass(1, BAD, A16, 8, 8, C.byref(p), None) == inv
    assert L.rc_vhs_pass(1, A16, BAD, 8, 8, C.byref(p), None) == inv
    assert L.rc_vhs_pass(1, A16, C.c_void_p((1 << 20) + 4096), 16385, 8, C.byref(p), None) == inv
    assert L.rc_vhs_pass(1, A16, C.c_void_p((1 << 20) + 4096), 8, 16385, C.byref(p), None) == inv


@pytest.mark.parametrize("which", ["in", "wpk", "out", "mask"])
def test_conv_alignment(product, which):
    args = {"in": A16, "wpk": A16, "out": A16, "mask": None}
    args[which] = BAD
    rc = product.lib().rc_kp_conv3x3(args["in"], 32, args["wpk"], None, args["out"], 0, 1, args["mask"],
                                     1, 4, 4, ERR, None)
    assert rc == product.RC_ERR_INVALID_ARG


def test_head_wgrad_crop_pack_adam_alignment(product):
    L = product.lib()
    inv = product.RC_ERR_INVALID_ARG
    assert L.rc_kp_wgrad(BAD, 32, A16, A16, A16, 1, 4, 4, ERR, None) == inv
    assert L.rc_kp_head(BAD, A16, None, A16, None, None, C.c_float(0.0), 1, 4, 4, None) == inv
    assert L.rc_kp_head(A16, A16, None, BAD, None, None, C.c_float(0.0), 1, 4, 4, None) == inv
    packed = (C.c_void_p * 7)(*([A16] * 6 + [BAD]))
    assert L.rc_kp_pack(A16, packed, None) == inv
    assert L.rc_kp_adam(C.c_void_p((1 << 20) + 2), A16, A16, A16, 16, C.c_float(1e-3), C.c_float(0.9),
                        C.c_float(0.999), C.c_float(1e-8), 1, None) == inv
    i4 = C.c_void_p((1 << 20) + 8)
    assert L.rc_kp_crop(A16, A16, A16, i4, i4, i4, i4, 1, 8, 8, 4, BAD, A16, A16, None) == inv


def test_noalloc_alignment(product):
    a = product.rc_atrous_params(1, 5, 1.0, 128.0, 1.0, 0, 1.0)
    rc = product.lib().rc_denoise_atrous_noalloc(BAD, A16, A16, A16, C.c_void_p((1 << 20) + 4096), 4, 4, 1,
                                                 C.byref(a), product.RC_MATH_FAST, None)
    assert rc == product.RC_ERR_INVALID_ARG
    rc = product.lib().rc_denoise_atrous_noalloc(A16, C.c_void_p((1 << 20) + 4), A16, A16,
                                                 C.c_void_p((1 << 20) + 4096), 4, 4, 1, C.byref(a),
                                                 product.RC_MATH_FAST, None)
    assert rc == product.RC_ERR_INVALID_ARG


@pytest.mark.parametrize("which", [0, 1, 2, 3])
def test_noalloc_rejects_output_overlapping_an_input(product, which):
    """The output image may share no byte with any of the four inputs: a pass
    reads neighbouring pixels of its inputs while other threads write the
    output.  Each input in turn is placed so that it ends inside the output's
    first bytes (16x16 pixels: 4 KiB of output)."""
    a = product.rc_atrous_params(1, 5, 1.0, 128.0, 1.0, 0, 1.0)
    base = 1 << 24
    out = C.c_void_p(base)
    sizes = [16 * 256, 8 * 256, 8 * 256, 4 * 256]
    args = [C.c_void_p(base + (1 << 20) * (k + 1)) for k in range(4)]
    args[which] = C.c_void_p(base - sizes[which] + 16)
    rc = product.lib().rc_denoise_atrous_noalloc(*args, out, 16, 16, 1, C.byref(a), product.RC_MATH_FAST, None)
    assert rc == product.RC_ERR_INVALID_ARG
    buf = C.create_string_buffer(256)
    product.lib().rc_last_error(None, buf, len(buf))
    assert b"overlaps" in buf.value
