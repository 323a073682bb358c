"""The allocation-free denoiser entry point, checked against the context's own.

rc_denoise_atrous_noalloc exists for callers that cannot let a library call
cudaMalloc: hosts that pool and budget every byte of device memory
themselves, and frame loops that must not stall on the synchronisation an
allocation can bring.  It reads and writes only caller-owned device buffers
plus one static device array inside the library.

The test renders a frame through a context, copies the four renderer images
into device buffers it owns, and makes no-alloc calls in a row (exact math
with several settings -- five passes, the denoiser disabled, a sample count
above max_spp, one pass, seven passes clamped to five -- then fast math with
other settings, so each call reuses the static array the one before left
behind).  Each result must equal what rc_denoise_atrous produced for the same
images: bit for bit in exact math, within the fast-math tolerance of the
other denoiser tests otherwise.  This file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bind(api):
    fn = api.lib().rc_denoise_atrous_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p] * 5 + [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p]
    return fn


def _device_images(torch, dev, acc, gb, ga, var):
    return (torch.from_numpy(acc).to(dev), torch.from_numpy(gb.view(np.int16)).to(dev),
            torch.from_numpy(ga.view(np.int16)).to(dev), torch.from_numpy(var).to(dev))


# (math mode, spp, parameter cases).  Exact math: the full five passes, the
# normalise-only branch (denoiser disabled; sample count above max_spp) and
# pass counts the reference clamps (1 and 7 -> 5); fast math: other sigmas.
CASES = [
    (0, 3, [(1, 5, 1.0, 128.0, 1.0, 0, 1.0), (0, 5, 1.0, 128.0, 1.0, 0, 1.0), (1, 5, 1.0, 128.0, 1.0, 2, 1.0),
            (1, 1, 1.0, 128.0, 1.0, 0, 1.0), (1, 7, 1.0, 128.0, 1.0, 0, 1.3)]),
    (1, 5, [(1, 4, 1.0, 64.0, 0.15, 0, 1.5)]),
]


def test_noalloc_denoise_matches_context_denoise(product, cuda_ok):
    import torch
    from retrocam_b200 import scenes
    api = product
    fn = _bind(api)
    w = scenes.export_frame()
    sc = api.build_scene(w.scene)
    cam = api.workload_camera(w)
    W, H = 200, 120
    dev = torch.device("cuda", 0)
    for fast, spp, plist in CASES:
        mode = api.RC_MATH_FAST if fast else api.RC_MATH_EXACT
        with api.Context(W, H, 0, mode) as ctx:
            ctx.upload(sc)
            ctx.render(cam, (1, 1.0), 0, spp)
            acc, gb, ga, var = ctx.read_buffers()
            wants = [ctx.denoise(api.rc_atrous_params(*pv)) for pv in plist]
        d_acc, d_gb, d_ga, d_var = _device_images(torch, dev, acc, gb, ga, var)
        for pv, want in zip(plist, wants):
            params = api.rc_atrous_params(*pv)
            d_out = torch.full((H, W, 4), float("nan"), dtype=torch.float32, device=dev)
            torch.cuda.synchronize()
            rc = fn(d_acc.data_ptr(), d_gb.data_ptr(), d_ga.data_ptr(), d_var.data_ptr(), d_out.data_ptr(), W, H,
                    spp, C.byref(params), mode, None)
            assert rc == api.RC_OK, pv
            torch.cuda.synchronize()
            got = d_out.cpu().numpy()
            if mode == api.RC_MATH_EXACT:
                assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), pv
            else:
                np.testing.assert_allclose(got, want, rtol=2e-3, atol=2e-4)


def test_noalloc_rejects_images_over_its_limit(product, cuda_ok):
    api = product
    fn = _bind(api)
    p = api.rc_atrous_params(1, 5, 1.0, 128.0, 1.0, 0, 1.0)
    fake = C.c_void_p(16)  # never dereferenced: the size check comes first
    rc = fn(fake, C.c_void_p(32), C.c_void_p(48), C.c_void_p(64), C.c_void_p(80), 2048, 1024, 1, C.byref(p),
            api.RC_MATH_FAST, None)
    assert rc == api.RC_ERR_CAPACITY
    buf = C.create_string_buffer(256)
    api.lib().rc_last_error(None, buf, len(buf))
    assert b"RC_NOALLOC_MAX_PIXELS" in buf.value
