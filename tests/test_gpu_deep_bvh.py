"""Traversal parity on BVHs deep enough that the reference's stacks overflow,
and on the 1,000,014-triangle stress scene.

The reference's shaders drop pushes once a stack is full: the closest-hit
walk keeps a node's children only while top < 62 (pathtrace.comp:176), the
shadow walk while top < 30 (pathtrace.comp:235), the photon trace and gather
walks while top < 62 (photon_trace.comp:102-128, photon_gather.comp).  Which
subtrees are lost depends on each walk's own visiting order.  The chained
tree of tests/deep_bvh.py (87 levels over the export frame's 7,972
triangles) fills all three stacks, so every traversal here runs its
deep-tree form: the `<false>` instantiations of the megakernel, the
wavefront trace, the photon trace and the gather, in both math builds
(rc_counters.bvh_depth > 60 is asserted).  Exact math must give the
oracle's bits -- the oracle itself is pinned to the compiled reference
shaders on the same tree (test_oracle_vs_ref.py); fast math keeps the
reference's visiting order on such trees and is compared by tolerance.
"""
import numpy as np
import pytest

from conftest import bits

pytestmark = pytest.mark.gpu

ENGINES = ("megakernel", "wavefront", "wavefront_small_chunks", "wavefront_static")


def _ctx(product, W, H, mode, engine="wavefront"):
    ctx = product.Context(W, H, 0, mode)
    if engine == "megakernel":
        ctx.set_engine(product.RC_ENGINE_MEGAKERNEL)
    elif engine == "wavefront_small_chunks":
        ctx.set_engine(product.RC_ENGINE_WAVEFRONT, 5000)
        ctx.set_tuning(refill_min_paths=1)
    elif engine == "wavefront_static":
        ctx.set_engine(product.RC_ENGINE_WAVEFRONT_STATIC)
    else:
        ctx.set_engine(product.RC_ENGINE_WAVEFRONT)
        ctx.set_tuning(refill_min_paths=1)
    return ctx


@pytest.fixture(scope="module")
def deep(product, orc, cuda_ok):
    import deep_bvh
    import pyoracle as po
    from retrocam_b200 import scenes
    w = scenes.export_frame()
    sc = deep_bvh.chain_scene(w.scene, orc, po.MAT, groups=80)
    cam = scenes.camera(w.orbit, w.lens, orc)
    assert deep_bvh.bvh_depth(sc["nodes"]) > 60
    return w, sc, cam


@pytest.fixture(scope="module")
def stress(product, cuda_ok):
    """The 1M-triangle scene, built once by the product's host builder (bit
    for bit the oracle's, tests/test_host_scene.py).  The triangle cloud is
    about 25 mean free paths deep, so from the benchmark's camera outside
    the box almost no light reaches what it sees (the image is black); the
    tests look down into the cloud from just under a ceiling light, where
    about half the pixels receive light."""
    import math
    from retrocam_b200 import scenes
    w = scenes.bvh_stress()
    orbit = scenes.OrbitDesc(theta=-math.pi / 2, phi=0.3, radius=0.14, target=(0.3, 0.85, 0.3))
    cam = scenes.camera(orbit, scenes.LensDesc(focal_length_mm=24.0, f_stop=16.0, focus_dist_m=0.2), product.HOST)
    return w, product.build_scene(w.scene), cam


def _same_images(gpu, cpu):
    for n, g, c in zip(("accum", "gbuffer", "albedo", "variance"), gpu, cpu):
        if not np.array_equal(bits(g), bits(c)):
            bad = np.argwhere(bits(g) != bits(c))
            raise AssertionError(f"{n}: {len(bad)} words differ, first at {bad[:3].tolist()}")


def _photon_records(ph, n):
    r = ph[:n].view(np.float32).reshape(n, 12)
    return r[np.lexsort(r.view(np.uint32).T[::-1])]


def test_depth_reported(product, deep):
    import deep_bvh
    w, sc, cam = deep
    with product.Context(16, 16, 0, product.RC_MATH_FAST) as ctx:
        assert ctx.counters()["bvh_depth"] == 0
        ctx.upload(sc)
        assert ctx.counters()["bvh_depth"] == deep_bvh.bvh_depth(sc["nodes"]) > 60


@pytest.mark.parametrize("engine", ENGINES)
def test_render_exact_bit_identical_deep(product, orc, deep, engine):
    w, sc, cam = deep
    W, H, spp = 96, 54, 2
    with _ctx(product, W, H, product.RC_MATH_EXACT, engine) as ctx:
        ctx.upload(sc)
        ctx.render(cam, (1, 1.0), 0, spp)
        gpu = ctx.read_buffers()
        cnt = ctx.counters()
    cpu, st = orc.render(sc, cam, (1, 1.0), W, H, 0, spp)
    _same_images(gpu, cpu)
    assert (cnt["camera_paths"], cnt["closest_rays"], cnt["shadow_rays"]) == tuple(st[:3])
    assert cnt["error_word"] == 0 and cnt["bvh_depth"] > 60


def test_render_exact_deep_nee_off_and_clamp(product, orc, deep):
    w, sc, cam = deep
    W, H = 48, 32
    for settings in ((0, 1.0), (1, 20.0)):
        with _ctx(product, W, H, product.RC_MATH_EXACT, "wavefront_static") as ctx:
            ctx.upload(sc)
            ctx.render(cam, settings, 0, 2)
            gpu = ctx.read_buffers()
        cpu, _ = orc.render(sc, cam, settings, W, H, 0, 2)
        _same_images(gpu, cpu)


def test_photon_map_exact_deep(product, orc, deep):
    w, sc, cam = deep
    N, r0, hs = 100_000, 0.02, 1 << 18
    with _ctx(product, 32, 32, product.RC_MATH_EXACT) as ctx:
        ctx.upload(sc)
        ctx.sppm_reset(r0)
        ctx.sppm_trace(N, hs)
        ph, heads, nxt, cnt = ctx.read_photon_map(N, hs)
        counters = ctx.counters()
    cph, cheads, cnxt, ccnt, st = orc.photon_trace(sc, N, r0, 6271, hs)
    assert cnt == ccnt > 1000
    assert counters["photon_rays"] == st[3] and counters["error_word"] == 0
    np.testing.assert_array_equal(_photon_records(ph, cnt).view(np.uint32),
                                  _photon_records(cph, ccnt).view(np.uint32))
    np.testing.assert_array_equal(heads < 0, cheads < 0)


def test_gather_exact_deep(product, orc, deep):
    """Gather rays walk the deep tree with the reference's photon-walk order;
    sums agree within the summation-order tolerance of the other gather
    tests (chains stay below the 512 cap at this photon count)."""
    w, sc, cam = deep
    W, H, N, r0, hs = 96, 64, 100_000, 0.02, 1 << 20
    with _ctx(product, W, H, product.RC_MATH_EXACT) as ctx:
        ctx.upload(sc)
        ctx.render(cam, (1, 1.0), 0, 1)
        before = ctx.read_buffers()[0]
        ctx.sppm_reset(r0)
        ctx.sppm_trace(N, hs)
        ctx.sppm_gather(cam, N, hs, 1.0)
        after = ctx.read_buffers()[0]
        assert ctx.counters()["error_word"] == 0
    cph, cheads, cnxt, ccnt, _ = orc.photon_trace(sc, N, r0, 6271, hs)
    cacc = before.copy()
    orc.photon_gather(sc, cam, W, H, r0, hs, cph, cheads, cnxt, cacc)
    assert np.abs(after - before).max() > 0
    np.testing.assert_allclose(after, cacc, rtol=2e-5, atol=1e-6)


@pytest.mark.parametrize("engine", ("megakernel", "wavefront", "wavefront_static"))
def test_render_fast_close_to_oracle_deep(product, orc, deep, engine):
    """Fast math on the deep tree: the reference's stack policies, FMA
    rounding.  Same statistical bar as on the builder's tree: >= 97% of
    pixels within 1e-4 relative, image mean within 1%."""
    w, sc, cam = deep
    W, H, spp = 160, 90, 4
    with _ctx(product, W, H, product.RC_MATH_FAST, engine) as ctx:
        ctx.upload(sc)
        ctx.render(cam, (1, 1.0), 0, spp)
        acc = ctx.read_buffers()[0]
        assert ctx.counters()["error_word"] == 0
    (cacc, _, _, _), _ = orc.render(sc, cam, (1, 1.0), W, H, 0, spp)
    rel = np.abs(acc[..., :3] - cacc[..., :3]) / np.maximum(np.abs(cacc[..., :3]), 1e-3)
    frac_close = np.mean(np.all(rel <= 1e-4, axis=-1))
    assert frac_close >= 0.97, frac_close
    assert abs(acc[..., :3].mean() - cacc[..., :3].mean()) / cacc[..., :3].mean() < 0.01


def test_photon_and_gather_fast_deep(product, orc, deep):
    """Fast build on the deep tree: no first-segment split (it walks other
    trees), the photon walk in the reference's order.  The stored photons
    agree with the oracle's in count and power; the gather over the
    product's own map agrees with the oracle's gather over that map."""
    w, sc, cam = deep
    W, H, N, r0, hs = 96, 64, 100_000, 0.02, 1 << 20
    with _ctx(product, W, H, product.RC_MATH_FAST) as ctx:
        ctx.upload(sc)
        ctx.render(cam, (1, 1.0), 0, 1)
        before = ctx.read_buffers()[0]
        ctx.sppm_reset(r0)
        ctx.sppm_trace(N, hs)
        ph, heads, nxt, cnt = ctx.read_photon_map(N, hs)
        ctx.sppm_gather(cam, N, hs, 1.0)
        after = ctx.read_buffers()[0]
        assert ctx.counters()["error_word"] == 0
    cph, _, _, ccnt, _ = orc.photon_trace(sc, N, r0, 6271, hs)
    assert abs(cnt - ccnt) <= max(2, ccnt // 200), (cnt, ccnt)
    p_gpu = ph[:cnt]["power"].astype(np.float64).sum(0)
    p_cpu = cph[:ccnt]["power"].astype(np.float64).sum(0)
    np.testing.assert_allclose(p_gpu, p_cpu, rtol=1e-2)
    cacc = before.copy()
    orc.photon_gather(sc, cam, W, H, r0, hs, ph, heads, nxt, cacc)
    g, c = (after - before)[..., :3], (cacc - before)[..., :3]
    assert np.abs(c).max() > 0
    close = np.all(np.abs(g - c) <= 1e-3 * np.abs(c) + 1e-5, axis=-1)
    assert close.mean() > 0.99, close.mean()


@pytest.mark.parametrize("engine", ("megakernel", "wavefront_static"))
def test_render_exact_bit_identical_stress_scene(product, orc, stress, engine):
    """The 1M-triangle scene (679,169 nodes, 27 levels; 160 MB of BVH and
    triangles, larger than L2) at a small image: the oracle's bits."""
    w, sc, cam = stress
    W, H, spp = 64, 36, 1
    with _ctx(product, W, H, product.RC_MATH_EXACT, engine) as ctx:
        ctx.upload(sc)
        ctx.render(cam, (w.nee_enabled, w.nee_firefly_clamp), 0, spp)
        gpu = ctx.read_buffers()
        cnt = ctx.counters()
    cpu, st = orc.render(sc, cam, (w.nee_enabled, w.nee_firefly_clamp), W, H, 0, spp)
    _same_images(gpu, cpu)
    assert (cnt["closest_rays"], cnt["shadow_rays"]) == tuple(st[1:3]) and cnt["error_word"] == 0
    assert (cpu[0][..., :3].max(axis=-1) > 0).mean() > 0.2   # not a black image


def test_render_fast_close_stress_scene(product, orc, stress):
    """The stress scene in the benchmarked build (the refill trace over the
    packed-reference records)."""
    w, sc, cam = stress
    W, H, spp = 96, 54, 2
    settings = (w.nee_enabled, w.nee_firefly_clamp)
    with _ctx(product, W, H, product.RC_MATH_FAST, "wavefront") as ctx:
        ctx.upload(sc)
        ctx.render(cam, settings, 0, spp)
        acc = ctx.read_buffers()[0]
        c = ctx.counters()
        assert c["error_word"] == 0 and c["bvh_depth"] <= 28
    (cacc, _, _, _), _ = orc.render(sc, cam, settings, W, H, 0, spp)
    assert (cacc[..., :3].max(axis=-1) > 0).mean() > 0.2   # not a black image
    rel = np.abs(acc[..., :3] - cacc[..., :3]) / np.maximum(np.abs(cacc[..., :3]), 1e-3)
    frac_close = np.mean(np.all(rel <= 1e-4, axis=-1))
    assert frac_close >= 0.97, frac_close
    assert abs(acc[..., :3].mean() - cacc[..., :3].mean()) / cacc[..., :3].mean() < 0.01
