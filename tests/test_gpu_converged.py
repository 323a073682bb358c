"""The path tracer's converged image against a 4096-spp reference.

The reference image is the exact build (the oracle's bits, so the
reference shaders' arithmetic) at 4096 spp on frame indices 2^20 onwards
(independent PCG streams); the images under test use frames 0..1023.
relMSE = mean over pixels and RGB of (x - ref)^2 / (ref^2 + 1e-2), the
project's quality metric.

Bounds: relMSE <= 1e-3 for the benchmarked fast build at 1024 spp, and
the fast build's relMSE within 5% of the exact build's at the same 1024
samples -- i.e. the fast arithmetic adds no error of its own beyond the
Monte Carlo noise both share.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BOUND = 1e-3


def _relmse(x, ref):
    x = x[..., :3].astype(np.float64)
    r = ref[..., :3].astype(np.float64)
    return float(np.mean((x - r) ** 2 / (r * r + 1e-2)))


def _mean_image(product, sc, cam, W, H, mode, first, spp, settings):
    with product.Context(W, H, 0, mode) as ctx:
        ctx.upload(sc)
        ctx.reset()
        ctx.render(cam, settings, first, spp)
        acc = ctx.read_buffers()[0]
        assert ctx.counters()["error_word"] == 0
    return acc[..., :3] / acc[..., 3:4]


@pytest.mark.parametrize("workload,W,H", [("cornell_small", 128, 128), ("export_frame", 160, 90)])
def test_converged_image_within_bound(product, cuda_ok, workload, W, H):
    from retrocam_b200 import scenes
    w = scenes.WORKLOADS[workload]()
    sc = product.build_scene(w.scene)
    cam = product.workload_camera(w)
    st = (w.nee_enabled, w.nee_firefly_clamp)
    ref = _mean_image(product, sc, cam, W, H, product.RC_MATH_EXACT, 1 << 20, 4096, st)
    fast = _mean_image(product, sc, cam, W, H, product.RC_MATH_FAST, 0, 1024, st)
    exact = _mean_image(product, sc, cam, W, H, product.RC_MATH_EXACT, 0, 1024, st)
    e_fast, e_exact = _relmse(fast, ref), _relmse(exact, ref)
    assert e_fast <= BOUND, (e_fast, e_exact)
    assert abs(e_fast - e_exact) <= 0.05 * e_exact, (e_fast, e_exact)
