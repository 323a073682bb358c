"""The oracle against the reference's own shaders compiled for the host
(oracle/_ref, built from the reference checkout by oracle/build_ref.py).

Every comparison is bit for bit.  Skipped where the compiled reference is not
available (no reference checkout and no prebuilt library); the committed
golden fixtures (test_golden.py) cover that case.
"""
import numpy as np
import pytest

from conftest import bits


@pytest.fixture(scope="module")
def scenes_built(orc):
    import pyoracle as po
    from retrocam_b200 import scenes
    out = {}
    for name in ("cornell_small", "export_frame"):
        w = scenes.WORKLOADS[name]()
        out[name] = (w, scenes.build_scene(w.scene, orc, po.MAT), scenes.camera(w.orbit, w.lens, orc))
    return out


def _eq(a, b):
    return np.array_equal(bits(a), bits(b))


@pytest.mark.parametrize("name,W,H,spp,lca,settings", [
    ("cornell_small", 64, 64, 3, False, (1, 1.0)),
    ("cornell_small", 48, 40, 2, True, (1, 1.0)),
    ("cornell_small", 32, 32, 2, False, (0, 1.0)),
    ("export_frame", 96, 54, 3, True, (1, 1.0)),
    ("export_frame", 64, 36, 2, False, (1, 20.0)),
])
def test_render_bit_identical(orc, ref, scenes_built, name, W, H, spp, lca, settings):
    w, sc, cam = scenes_built[name]
    cam = dict(cam)
    cam["lca_delta"] = (-0.009, 0.0, 0.009) if lca else (0.0, 0.0, 0.0)
    mine, _ = orc.render(sc, cam, settings, W, H, 0, spp)
    theirs = ref.render(sc, cam, settings, W, H, 0, spp)
    for a, b in zip(mine, theirs):
        assert _eq(a, b)


def test_render_lens_variants(orc, ref, scenes_built):
    """Pinhole (lens radius 0), 5/6/8 blades, spherical aberration off."""
    w, sc, cam = scenes_built["export_frame"]
    for lr, blades, sa in ((0.0, 5, 0.04), (5e-3, 8, 0.0), (1e-2, 5, 0.1)):
        c = dict(cam, lens_radius=lr, aperture_blades=blades, sa_strength=sa)
        mine, _ = orc.render(sc, c, (1, 1.0), 40, 30, 0, 2)
        theirs = ref.render(sc, c, (1, 1.0), 40, 30, 0, 2)
        for a, b in zip(mine, theirs):
            assert _eq(a, b)


def test_photon_trace_and_gather_bit_identical(orc, ref, scenes_built):
    w, sc, cam = scenes_built["export_frame"]
    N, r, hs = 120_000, 0.02, 1 << 18
    ph, hd, nx, cnt, _ = orc.photon_trace(sc, N, r, 3 * 7919 + 6271, hs)
    ph2, hd2, nx2, cnt2 = ref.photon_trace(sc, N, r, 3 * 7919 + 6271, hs, threads=1)
    assert cnt == cnt2 > 0
    assert _eq(ph[:cnt].view(np.float32), ph2[:cnt].view(np.float32))
    assert np.array_equal(hd, hd2) and np.array_equal(nx[:cnt], nx2[:cnt])
    W, H = 80, 48
    a1 = np.ones((H, W, 4), np.float32)
    a2 = a1.copy()
    orc.photon_gather(sc, cam, W, H, r, hs, ph, hd, nx, a1)
    ref.photon_gather(sc, cam, W, H, r, N, hs, 0, ph2, hd2, nx2, a2)
    assert _eq(a1, a2) and (a1 != 1.0).any()


def test_photon_trace_small_hash(orc, ref, scenes_built):
    """A 4096-cell hash and a wide radius: many cells share one chain."""
    w, sc, cam = scenes_built["export_frame"]
    N = 40_000
    ph, hd, nx, cnt, _ = orc.photon_trace(sc, N, 0.05, 6271, 1 << 12)
    ph2, hd2, nx2, cnt2 = ref.photon_trace(sc, N, 0.05, 6271, 1 << 12, threads=1)
    assert cnt == cnt2 and np.array_equal(hd, hd2)


@pytest.mark.parametrize("W,H,iters,sn,sd,sc_,exposure", [
    (96, 54, 5, 128.0, 1.0, 1.0, 1.0),
    (40, 24, 5, 64.0, 0.15, 1.0, 1.0),    # steps 8 and 16 wrap past the borders
    (33, 17, 3, 16.0, 0.5, 2.0, 1.7),
])
def test_atrous_bit_identical(orc, ref, scenes_built, W, H, iters, sn, sd, sc_, exposure):
    import pyoracle as po
    w, sc, cam = scenes_built["export_frame"]
    bufs, _ = orc.render(sc, cam, (1, 1.0), W, H, 0, 3)
    p = po.AtrousParams(1, iters, sc_, sn, sd, 0, exposure)
    assert _eq(orc.denoise(*bufs, W, H, 3, p), ref.denoise(*bufs, W, H, 3, p))


def test_atrous_gating(orc, ref, scenes_built):
    import pyoracle as po
    w, sc, cam = scenes_built["cornell_small"]
    bufs, _ = orc.render(sc, cam, (1, 1.0), 32, 32, 0, 4)
    for p in (po.AtrousParams(0, 4, 1.0, 64.0, 0.15, 0, 1.0),   # disabled: p00 only
              po.AtrousParams(1, 4, 1.0, 64.0, 0.15, 3, 1.0),   # over max_spp: p00 only
              po.AtrousParams(1, 9, 1.0, 64.0, 0.15, 0, 1.0),   # iterations clamp to 5
              po.AtrousParams(1, 0, 1.0, 64.0, 0.15, 0, 1.0)):  # and to 1
        assert _eq(orc.denoise(*bufs, 32, 32, 4, p), ref.denoise(*bufs, 32, 32, 4, p))


@pytest.mark.parametrize("total,exposure", [(1, 1.0), (16, 1.3), (0, 0.7)])
def test_display_bit_identical(orc, ref, total, exposure):
    """display.frag (ACES fit, sRGB encode) and the RGBA8 export store, on
    log-normal HDR values plus the edges: zero, the sRGB knee 0.0031308 and
    its neighbour, 1, half-float max, a negative value."""
    rng = np.random.default_rng(3)
    W, H = 97, 61
    c = np.exp(rng.normal(-1.5, 2.0, (H, W, 4))).astype(np.float32)
    c[0, :8, 0] = [0.0, 1e-6, 0.0031308, 0.0031307, 1.0, 65504.0, -0.5, 3.0]
    a = orc.display(c, W, H, total, exposure)
    assert np.array_equal(a, ref.display(c, W, H, total, exposure))
    assert (a[..., 3] == 255).all()
    # rows top first: flipping the buffer flips the image
    assert np.array_equal(a[::-1], orc.display(np.ascontiguousarray(c[::-1]), W, H, total, exposure))


@pytest.fixture(scope="module")
def deep_scene(orc):
    """The export frame's triangles under the chained 87-level tree of
    tests/deep_bvh.py, where the shaders' stacks overflow."""
    import deep_bvh
    import pyoracle as po
    from retrocam_b200 import scenes
    w = scenes.export_frame()
    sc = deep_bvh.chain_scene(w.scene, orc, po.MAT, groups=80)
    assert deep_bvh.bvh_depth(sc["nodes"]) > 60
    return w, sc, scenes.camera(w.orbit, w.lens, orc)


@pytest.mark.parametrize("lca,settings", [(True, (1, 1.0)), (False, (0, 1.0)), (False, (1, 20.0))])
def test_render_bit_identical_deep_tree(orc, ref, deep_scene, scenes_built, lca, settings):
    """Closest-hit (top < 62) and shadow (top < 30) stack overflow as the
    shaders have it.  With NEE on, the deep tree must change the image
    against the builder's tree (shadow rays lose subtrees), or no overflow
    happened; with NEE off only the few closest-hit rays travelling against
    the chain's order overflow."""
    w, sc, cam = deep_scene
    cam = dict(cam)
    cam["lca_delta"] = (-0.009, 0.0, 0.009) if lca else (0.0, 0.0, 0.0)
    W, H = 64, 36
    mine, _ = orc.render(sc, cam, settings, W, H, 0, 2)
    theirs = ref.render(sc, cam, settings, W, H, 0, 2)
    for a, b in zip(mine, theirs):
        assert _eq(a, b)
    shallow, _ = orc.render(scenes_built["export_frame"][1], cam, settings, W, H, 0, 2)
    changed = (np.abs(shallow[0] - mine[0]).max(axis=-1) > 1e-3).mean()
    assert changed > (0.02 if settings[0] else 0.0), changed


def test_photon_trace_and_gather_bit_identical_deep_tree(orc, ref, deep_scene, scenes_built):
    w, sc, cam = deep_scene
    N, r, hs = 100_000, 0.02, 1 << 18
    ph, hd, nx, cnt, _ = orc.photon_trace(sc, N, r, 6271, hs)
    ph2, hd2, nx2, cnt2 = ref.photon_trace(sc, N, r, 6271, hs, threads=1)
    assert cnt == cnt2 > 1000
    assert _eq(ph[:cnt].view(np.float32), ph2[:cnt].view(np.float32))
    assert np.array_equal(hd, hd2) and np.array_equal(nx[:cnt], nx2[:cnt])
    # the photon walk's 64-entry stack overflowed: fewer photons stored
    _, _, _, cnt_shallow, _ = orc.photon_trace(scenes_built["export_frame"][1], N, r, 6271, hs)
    assert cnt < 0.9 * cnt_shallow
    W, H = 80, 48
    a1 = np.ones((H, W, 4), np.float32)
    a2 = a1.copy()
    orc.photon_gather(sc, cam, W, H, r, hs, ph, hd, nx, a1)
    ref.photon_gather(sc, cam, W, H, r, N, hs, 0, ph2, hd2, nx2, a2)
    assert _eq(a1, a2) and (a1 != 1.0).any()
