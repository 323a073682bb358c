"""Parity of the CUDA path tracer, photon passes and denoiser with the CPU
oracle, through the C ABI.

Exact math mode (RC_MATH_EXACT) must be bit-identical to the oracle for
every deterministic output (accumulation, variance, G-buffer, albedo,
photon records and cells, à-trous).  The gather sums photons in hash-chain
order, which the GPU's atomic insertion leaves unordered, so it is compared
within 2e-5 relative.  Fast mode is compared by tolerance (see each test).
"""
import numpy as np
import pytest

from conftest import bits

pytestmark = pytest.mark.gpu


def _scene(product, orc, workload):
    import pyoracle as po
    from retrocam_b200 import scenes
    w = workload()
    sc = scenes.build_scene(w.scene, orc, po.MAT)
    cam = scenes.camera(w.orbit, w.lens, orc)
    return w, sc, cam


ENGINES = ("megakernel", "wavefront", "wavefront_small_chunks", "wavefront_static")


def _ctx(product, W, H, mode, engine="wavefront"):
    ctx = product.Context(W, H, 0, mode)
    if engine == "megakernel":
        ctx.set_engine(product.RC_ENGINE_MEGAKERNEL)
    elif engine == "wavefront_small_chunks":
        ctx.set_engine(product.RC_ENGINE_WAVEFRONT, 5000)   # several chunks per call
        ctx.set_tuning(refill_min_paths=1)
    elif engine == "wavefront_static":
        ctx.set_engine(product.RC_ENGINE_WAVEFRONT_STATIC)
    else:
        # the refill trace even for the tests' small chunks (by default
        # chunks below 2^20 paths are traced grid-stride)
        ctx.set_engine(product.RC_ENGINE_WAVEFRONT)
        ctx.set_tuning(refill_min_paths=1)
    return ctx


def test_fast_dynamic_fetch_matches_static_schedule(product, c1):
    """The persistent refill trace (fast build) visits the same rays as the
    grid-stride one; only exact ties between triangles may resolve another
    way, so almost every pixel is bit-identical."""
    w, sc, cam = c1
    out = []
    for engine in ("wavefront", "wavefront_static"):
        with _ctx(product, 160, 90, product.RC_MATH_FAST, engine) as ctx:
            ctx.upload(sc)
            ctx.render(cam, (1, 1.0), 0, 4)
            out.append(ctx.read_buffers()[0])
            assert ctx.counters()["error_word"] == 0
    same = np.all(bits(out[0]) == bits(out[1]), axis=-1).mean()
    assert same > 0.995, same


def test_refill_interior_steps_change_nothing(product, c1):
    """The refill trace's per-round budget of tree moves changes only when a
    lane moves, not where: every budget gives the same hits, bit for bit."""
    w, sc, cam = c1
    out = []
    for steps in (1, 2, 6, 8):
        with _ctx(product, 160, 90, product.RC_MATH_FAST, "wavefront") as ctx:
            ctx.set_tuning(interior_steps=steps)
            ctx.upload(sc)
            ctx.render(cam, (1, 1.0), 0, 4)
            out.append(ctx.read_buffers())
            assert ctx.counters()["error_word"] == 0
    for o in out[1:]:
        _same_images(o, out[0])


def test_tuning_roundtrip_and_validation(product):
    with product.Context(64, 64, 0, product.RC_MATH_FAST) as ctx:
        t = ctx.tuning()
        assert t == {"engine": product.RC_ENGINE_WAVEFRONT, "chunk_paths": 0, "wide_bvh": 0,
                     "trace_block": 128, "shade_block": 128, "photon_block": 128, "photon_full_first": 0,
                     "refill_lanes": 16, "leaf_quarters": 2, "refill_min_paths": 1 << 20, "material_queues": 0,
                     "interior_steps": 6}
        ctx.set_tuning(engine=product.RC_ENGINE_WAVEFRONT_STATIC, wide_bvh=3, trace_block=256, shade_block=64)
        t = ctx.tuning()
        assert (t["engine"], t["wide_bvh"], t["trace_block"], t["shade_block"]) == (2, 3, 256, 64)
        for bad in ({"engine": 7}, {"chunk_paths": -1}, {"wide_bvh": 4}, {"trace_block": 96},
                    {"photon_block": 512}, {"photon_full_first": 2},
                    {"refill_lanes": 33}, {"leaf_quarters": 5}, {"refill_min_paths": -1},
                    {"material_queues": 2}, {"interior_steps": 9}):
            with pytest.raises(product.RetroCamError) as e:
                ctx.set_tuning(**bad)
            assert e.value.code == product.RC_ERR_INVALID_ARG
        assert ctx.tuning() == t   # a rejected call changes nothing


@pytest.mark.parametrize("mode", ["exact", "fast"])
@pytest.mark.parametrize("engine", ("wavefront", "wavefront_static"))
def test_material_queues_change_nothing(product, orc, c1, mode, engine):
    """Shading each bounce's hits from material queues (misses finished by
    the sort kernel) only reorders independent paths: bit-identical images
    in both builds, and in exact math the oracle's."""
    w, sc, cam = c1
    cam = dict(cam)
    W, H, spp = 96, 64, 3
    m = product.RC_MATH_EXACT if mode == "exact" else product.RC_MATH_FAST
    out = []
    for mq in (0, 1):
        with _ctx(product, W, H, m, engine) as ctx:
            ctx.set_tuning(material_queues=mq)
            ctx.set_kernel_timing(True)
            ctx.upload(sc)
            ctx.render(cam, (1, 1.0), 0, spp)
            out.append(ctx.read_buffers())
            sorted_launches = ctx.kernel_times()["wf_sort"][1]
            assert (sorted_launches > 0) == (mq == 1)
            assert ctx.counters()["error_word"] == 0
    _same_images(out[1], out[0])
    if mode == "exact":
        cpu, _ = orc.render(sc, cam, (1, 1.0), W, H, 0, spp)
        _same_images(out[1], cpu)


def test_exact_results_independent_of_tuning(product, orc, c1):
    """Exact math walks the binary tree in the reference's order whatever the
    knobs say, so every launch shape gives the oracle's bits."""
    w, sc, cam = c1
    W, H = 96, 64
    cpu, _ = orc.render(sc, cam, (1, 1.0), W, H, 0, 2)
    for knobs in ({"wide_bvh": 3, "trace_block": 64, "shade_block": 256},
                  {"engine": product.RC_ENGINE_WAVEFRONT_STATIC, "trace_block": 256, "shade_block": 64},
                  {"engine": product.RC_ENGINE_MEGAKERNEL, "wide_bvh": 3}):
        with product.Context(W, H, 0, product.RC_MATH_EXACT) as ctx:
            ctx.set_tuning(**knobs)
            ctx.upload(sc)
            ctx.render(cam, (1, 1.0), 0, 2)
            _same_images(ctx.read_buffers(), cpu)


@pytest.mark.parametrize("engine", ("megakernel", "wavefront", "wavefront_static"))
def test_fast_wide_bvh_matches_binary(product, c1, engine):
    """The 4-wide traversal finds the same nearest triangle as the binary one
    (ties between triangles at one distance aside), so nearly every pixel is
    bit-identical; block sizes change nothing."""
    w, sc, cam = c1
    out = []
    for wide, block in ((0, 128), (product.RC_WIDE_PATHS, 128), (product.RC_WIDE_PATHS, 256), (0, 64)):
        with _ctx(product, 160, 90, product.RC_MATH_FAST, engine) as ctx:
            ctx.set_tuning(wide_bvh=wide, trace_block=block, shade_block=block)
            ctx.upload(sc)
            ctx.render(cam, (1, 1.0), 0, 4)
            out.append(ctx.read_buffers()[0])
            assert ctx.counters()["error_word"] == 0
    for o in out[1:]:
        same = np.all(bits(o) == bits(out[0]), axis=-1).mean()
        assert same > 0.995, same


def test_fast_wide_bvh_photon_map(product, c1):
    """Photon trace through the 4-wide tree stores the same photons as
    through the binary tree (compared as sorted records)."""
    w, sc, cam = c1
    maps = []
    for wide in (0, product.RC_WIDE_PHOTONS):
        with product.Context(64, 64, 0, product.RC_MATH_FAST) as ctx:
            ctx.set_tuning(wide_bvh=wide, photon_block=64 if wide else 256)
            ctx.upload(sc)
            ctx.sppm_reset(0.02)
            ctx.sppm_trace(200_000, 1 << 18)
            ph, heads, nxt, n = ctx.read_photon_map(200_000, 1 << 18)
            maps.append(_photon_records(ph, n))
            assert ctx.counters()["error_word"] == 0
    a, b = maps
    assert abs(len(a) - len(b)) <= max(2, len(a) // 1000)
    k = min(len(a), len(b))
    assert np.mean(np.all(bits(a[:k]) == bits(b[:k]), axis=-1)) > 0.99


def test_fast_photon_first_segment_split(product, c1):
    """Tracing a photon's first segment against the specular triangles and
    then testing the others up to that hit stores the same photons as
    tracing the whole scene (ties between triangles at one distance aside)."""
    w, sc, cam = c1
    maps, rays = [], []
    for full in (1, 0):
        with product.Context(64, 64, 0, product.RC_MATH_FAST) as ctx:
            ctx.set_tuning(photon_full_first=full)
            ctx.upload(sc)
            ctx.sppm_reset(0.02)
            ctx.sppm_trace(300_000, 1 << 18)
            ph, heads, nxt, n = ctx.read_photon_map(300_000, 1 << 18)
            maps.append(_photon_records(ph, n))
            c = ctx.counters()
            rays.append((c["photon_rays"], c["photon_node_tests"]))
            assert c["error_word"] == 0
    a, b = maps
    assert len(a) > 1000 and abs(len(a) - len(b)) <= max(2, len(a) // 1000)
    k = min(len(a), len(b))
    assert np.mean(np.all(bits(a[:k]) == bits(b[:k]), axis=-1)) > 0.99
    assert rays[0][0] == rays[1][0]          # one traversal per segment either way
    assert rays[1][1] < 0.5 * rays[0][1]     # far fewer box tests with the split


def test_empty_scene_renders_black(product):
    """A scene without triangles: every ray misses, no guard is raised."""
    from retrocam_b200 import scenes
    w = scenes.cornell_small()
    sc = product.build_scene(w.scene)
    sc = dict(sc)
    sc["tris"] = sc["tris"][:0]
    sc["nodes"] = sc["nodes"][:1].copy()
    sc["nodes"]["prim_count"] = 0
    sc["nodes"]["left_child"] = 0
    sc["nodes"]["right_child"] = 0
    sc["light_count"] = 0
    with product.Context(32, 32, 0, product.RC_MATH_FAST) as ctx:
        ctx.upload(sc)
        ctx.render(product.workload_camera(w), (1, 1.0), 0, 2)
        acc = ctx.read_buffers()[0]
        assert ctx.counters()["error_word"] == 0
    assert not acc[..., :3].any() and (acc[..., 3] == 2).all()


@pytest.fixture(scope="module")
def c0(product, orc, cuda_ok):
    from retrocam_b200 import scenes
    return _scene(product, orc, scenes.cornell_small)


@pytest.fixture(scope="module")
def c1(product, orc, cuda_ok):
    from retrocam_b200 import scenes
    return _scene(product, orc, scenes.export_frame)


def _same_images(gpu, cpu):
    names = ("accum", "gbuffer", "albedo", "variance")
    for n, g, c in zip(names, gpu, cpu):
        if not np.array_equal(bits(g), bits(c)):
            bad = np.argwhere(bits(g) != bits(c))
            raise AssertionError(f"{n}: {len(bad)} words differ, first at {bad[:3].tolist()}")


@pytest.mark.parametrize("engine", ENGINES)
@pytest.mark.parametrize("size,spp,lca", [((64, 64), 1, False), ((256, 256), 1, False), ((256, 256), 4, True),
                                          ((97, 61), 3, False)])
def test_render_exact_bit_identical_cornell(product, orc, c0, size, spp, lca, engine):
    w, sc, cam = c0
    cam = dict(cam)
    if lca:
        cam["lca_delta"] = (-0.009, 0.0, 0.009)
    W, H = size
    with _ctx(product, W, H, product.RC_MATH_EXACT, engine) as ctx:
        ctx.upload(sc)
        ctx.render(cam, (1, 1.0), 0, spp)
        gpu = ctx.read_buffers()
    cpu, _ = orc.render(sc, cam, (1, 1.0), W, H, 0, spp)
    _same_images(gpu, cpu)


@pytest.mark.parametrize("engine", ENGINES)
def test_render_exact_bit_identical_export_scene(product, orc, c1, engine):
    w, sc, cam = c1
    W, H = 160, 90
    with _ctx(product, W, H, product.RC_MATH_EXACT, engine) as ctx:
        ctx.upload(sc)
        ctx.render(cam, (1, 1.0), 0, 3)
        gpu = ctx.read_buffers()
        cnt = ctx.counters()
    cpu, st = orc.render(sc, cam, (1, 1.0), W, H, 0, 3)
    _same_images(gpu, cpu)
    # the device counters count the same traversals as the oracle
    assert cnt["camera_paths"] == st[0]
    assert cnt["closest_rays"] == st[1]
    assert cnt["shadow_rays"] == st[2]
    assert cnt["error_word"] == 0


@pytest.mark.parametrize("engine", ENGINES)
def test_render_split_launches_equal_one_launch(product, c1, engine):
    """n_spp frames in one launch == one launch per frame (same additions)."""
    w, sc, cam = c1
    W, H = 64, 48
    out = []
    for split in (False, True):
        with _ctx(product, W, H, product.RC_MATH_EXACT, engine) as ctx:
            ctx.upload(sc)
            if split:
                for f in range(5):
                    ctx.render(cam, (1, 1.0), f, 1)
            else:
                ctx.render(cam, (1, 1.0), 0, 5)
            out.append(ctx.read_buffers())
            assert ctx.total_samples == 5
    _same_images(out[0], out[1])


@pytest.mark.parametrize("engine", ENGINES[:2])
def test_render_nee_off_and_clamp(product, orc, c1, engine):
    w, sc, cam = c1
    W, H = 48, 32
    for settings in ((0, 1.0), (1, 20.0)):
        with _ctx(product, W, H, product.RC_MATH_EXACT, engine) as ctx:
            ctx.upload(sc)
            ctx.render(cam, settings, 0, 2)
            gpu = ctx.read_buffers()
        cpu, _ = orc.render(sc, cam, settings, W, H, 0, 2)
        _same_images(gpu, cpu)


@pytest.mark.parametrize("engine", ("megakernel", "wavefront", "wavefront_static"))
def test_render_fast_close_to_oracle(product, orc, c1, engine):
    """Fast math reorders rounding, so a few paths take another branch; the
    per-pixel check is statistical and the image mean must agree."""
    w, sc, cam = c1
    W, H, spp = 160, 90, 4
    with _ctx(product, W, H, product.RC_MATH_FAST, engine) as ctx:
        ctx.upload(sc)
        ctx.render(cam, (1, 1.0), 0, spp)
        acc, gb, ga, var = ctx.read_buffers()
    (cacc, cgb, cga, cvar), _ = orc.render(sc, cam, (1, 1.0), W, H, 0, spp)
    rel = np.abs(acc[..., :3] - cacc[..., :3]) / np.maximum(np.abs(cacc[..., :3]), 1e-3)
    frac_close = np.mean(np.all(rel <= 1e-4, axis=-1))
    assert frac_close >= 0.97, frac_close
    m_gpu, m_cpu = acc[..., :3].mean(), cacc[..., :3].mean()
    assert abs(m_gpu - m_cpu) / m_cpu < 0.01
    np.testing.assert_array_equal(acc[..., 3], cacc[..., 3])
    # G-buffer: same surfaces; values within half precision of the oracle's
    g, c = gb.view(np.float16).astype(np.float32), cgb.view(np.float16).astype(np.float32)
    assert np.mean(np.all(np.abs(g - c) <= 2e-3 * np.maximum(np.abs(c), 1.0), axis=-1)) >= 0.99


def _photon_records(ph, n):
    r = ph[:n].view(np.float32).reshape(n, 12)
    u = r.view(np.uint32)
    return r[np.lexsort(u.T[::-1])]


def test_photon_map_exact(product, orc, c1):
    w, sc, cam = c1
    N, r0, hs = 300_000, 0.02, 1 << 20
    with _ctx(product, 64, 64, product.RC_MATH_EXACT) as ctx:
        ctx.upload(sc)
        ctx.sppm_reset(r0)
        ctx.sppm_trace(N, hs)
        ph, heads, nxt, cnt = ctx.read_photon_map(N, hs)
        counters = ctx.counters()
    cph, cheads, cnxt, ccnt, st = orc.photon_trace(sc, N, r0, 0 * 7919 + 6271, hs)
    assert cnt == ccnt > 1000
    assert counters["photon_rays"] == st[3]
    # same set of photon records (insertion order differs: GPU atomics)
    g = _photon_records(ph, cnt)
    c = _photon_records(cph, ccnt)
    np.testing.assert_array_equal(g.view(np.uint32), c.view(np.uint32))
    # chains: every photon sits in exactly one chain, the one of its own cell
    pos = ph[:cnt]["position"]
    cells = np.floor(pos / np.float32(r0)).astype(np.int64)
    h = ((cells[:, 0] * 73856093) ^ (cells[:, 1] * 19349663) ^ (cells[:, 2] * 83492791)) & (hs - 1)
    seen = np.zeros(cnt, bool)
    for cell in np.unique(h):
        i = heads[cell]
        while i >= 0:
            assert not seen[i]
            seen[i] = True
            assert h[i] == cell
            i = nxt[i]
    assert seen.all()
    # heads hold -1 exactly where the oracle's do
    np.testing.assert_array_equal(heads < 0, cheads < 0)


def _max_chain(ph, n, r, hs):
    cells = np.floor(ph[:n]["position"] / np.float32(r)).astype(np.int64)
    h = ((cells[:, 0] * 73856093) ^ (cells[:, 1] * 19349663) ^ (cells[:, 2] * 83492791)) & (hs - 1)
    return np.bincount(h).max()


def _gather_pair(product, orc, sc, cam, W, H, N, r0, hs):
    with _ctx(product, W, H, product.RC_MATH_EXACT) as ctx:
        ctx.upload(sc)
        ctx.render(cam, (1, 1.0), 0, 1)
        before = ctx.read_buffers()[0]
        ctx.sppm_reset(r0)
        ctx.sppm_trace(N, hs)
        ctx.sppm_gather(cam, N, hs, 1.0)
        after = ctx.read_buffers()[0]
    cph, cheads, cnxt, ccnt, _ = orc.photon_trace(sc, N, r0, 6271, hs)
    cacc = before.copy()
    orc.photon_gather(sc, cam, W, H, r0, hs, cph, cheads, cnxt, cacc)
    return before, after, cacc, _max_chain(cph, ccnt, r0, hs)


def test_gather_matches_oracle(product, orc, c1):
    """Chains below the reference's 512-step walk cap: every photon in range
    is summed, only the summation order differs (GPU insertion order)."""
    w, sc, cam = c1
    before, after, cacc, longest = _gather_pair(product, orc, sc, cam, 96, 64, 100_000, 0.02, 1 << 20)
    assert longest < 512
    assert np.abs(after - before).max() > 0  # caustics landed somewhere
    np.testing.assert_allclose(after, cacc, rtol=2e-5, atol=1e-6)
    np.testing.assert_array_equal(after[..., 3], before[..., 3])


@pytest.mark.parametrize("mode", ["exact", "fast"])
def test_gather_hits_reused_across_iterations(product, c1, mode):
    """The pixel-centre gather rays and their specular walks are traced once
    per camera: a second gather with the same camera and photon map adds the
    same amounts (bit for bit) without tracing, and a new camera traces
    again."""
    w, sc, cam = c1
    W, H, N, hs = 96, 64, 100_000, 1 << 18
    m = product.RC_MATH_EXACT if mode == "exact" else product.RC_MATH_FAST
    with product.Context(W, H, 0, m) as ctx:
        ctx.upload(sc)
        ctx.sppm_reset(0.02)
        ctx.sppm_trace(N, hs)
        ctx.reset_counters()
        a0 = ctx.read_buffers()[0]
        ctx.sppm_gather(cam, N, hs)
        a1 = ctx.read_buffers()[0]
        traced = ctx.counters()["gather_rays"]
        ctx.reset_counters()
        ctx.sppm_gather(cam, N, hs)
        a2 = ctx.read_buffers()[0]
        assert ctx.counters()["gather_rays"] == 0 and traced >= W * H
        cam2 = dict(cam)
        cam2["cam_pos"] = np.asarray(cam["cam_pos"], np.float32) + np.float32(0.01)
        ctx.reset_counters()
        ctx.sppm_gather(cam2, N, hs)
        assert ctx.counters()["gather_rays"] >= W * H
    d1, d2 = a1 - a0, a2 - a1
    assert np.abs(d1).max() > 0
    # the same per-pixel amounts, added onto a different running sum
    np.testing.assert_allclose(d2, d1, rtol=1e-5, atol=1e-7)


def test_gather_with_capped_chains(product, orc, c1):
    """Chains longer than 512 are cut by the reference's `safety < 512` walk
    cap (photon_gather.comp:193), so which photons count depends on insertion
    order -- on the reference's own GPU too.  Pixels agree statistically."""
    w, sc, cam = c1
    before, after, cacc, longest = _gather_pair(product, orc, sc, cam, 96, 64, 300_000, 0.02, 1 << 20)
    assert longest > 512
    g, c = (after - before)[..., :3], (cacc - before)[..., :3]
    close = np.all(np.abs(g - c) <= 2e-5 * np.abs(c) + 1e-6, axis=-1)
    assert close.mean() > 0.98, close.mean()
    assert abs(g.sum() - c.sum()) / c.sum() < 0.02


@pytest.mark.parametrize("photons", [100_000, 300_000])
def test_gather_fast_matches_oracle_on_its_map(product, orc, c1, photons):
    """Fast build: pixels whose 27 cells hold more than 64 photons are
    gathered one warp per pixel with lanes striding the photons.  Against
    the oracle's gather over the product's own photon map (same chains, so
    the same first 512 photons of a long chain), only the summation order
    and the fast-math gather hit points differ.  300k photons make chains
    longer than the 512 cap, so those pixels take the warp-per-pixel path."""
    w, sc, cam = c1
    W, H, hs, r0 = 96, 64, 1 << 20, 0.02
    with _ctx(product, W, H, product.RC_MATH_FAST) as ctx:
        ctx.upload(sc)
        ctx.render(cam, (1, 1.0), 0, 1)
        before = ctx.read_buffers()[0]
        ctx.sppm_reset(r0)
        ctx.sppm_trace(photons, hs)
        ph, heads, nxt, stored = ctx.read_photon_map(photons, hs)
        ctx.sppm_gather(cam, photons, hs, 1.0)
        after = ctx.read_buffers()[0]
    longest = _max_chain(ph, min(stored, photons), r0, hs)
    assert (longest > 512) == (photons == 300_000), longest
    cacc = before.copy()
    orc.photon_gather(sc, cam, W, H, r0, hs, ph, heads, nxt, cacc)
    g, c = (after - before)[..., :3], (cacc - before)[..., :3]
    assert np.abs(c).max() > 0
    close = np.all(np.abs(g - c) <= 1e-3 * np.abs(c) + 1e-5, axis=-1)
    assert close.mean() > 0.995, close.mean()
    # the brightest caustic pixels (the densest cells: the warp-per-pixel
    # path at 300k photons) agree as well as the rest
    lum = c.sum(axis=-1)
    bright = lum >= np.quantile(lum[lum > 0], 0.9)
    assert close[bright].mean() > 0.98, close[bright].mean()
    # a few gather rays refract differently under fast math (glass walks)
    assert abs(g.sum() - c.sum()) / c.sum() < 5e-3
    np.testing.assert_array_equal(after[..., 3], before[..., 3])


def test_scene_file_render_matches_oracle(product, orc):
    """A scene read from a file in the reference's scene format (boxes,
    rotated boxes, spheres, an emissive box) renders with the oracle's bits
    under exact math."""
    import pyoracle as po
    from retrocam_b200 import scene_json as sj
    from retrocam_b200 import scenes
    text = """{"materials": [
      {"name": "White", "albedo": [0.73, 0.73, 0.73], "roughness": 0.5, "ior": 1.5},
      {"name": "Lamp", "albedo": [1.0, 0.95, 0.85], "emission": [1.0, 0.95, 0.85], "emissionStrength": 15,
       "roughness": 0.5, "ior": 1.5},
      {"name": "Gold", "albedo": [0.95, 0.85, 0.55], "metallic": 1, "roughness": 0.1, "ior": 1.5},
      {"name": "Glass", "albedo": [1, 1, 1], "roughness": 0, "ior": 1.5, "transmission": 1}],
     "objects": [
      {"name": "Floor", "type": "BOX", "px": 0.5, "py": 0, "pz": 0.5, "sx": 1, "sy": 0.02, "sz": 1, "materialIndex": 0},
      {"name": "Back", "type": "BOX", "px": 0.5, "py": 0.5, "pz": 1.2, "sx": 1, "sy": 1, "sz": 0.02, "materialIndex": 0},
      {"name": "Light", "type": "BOX", "px": 0.5, "py": 1.1, "pz": 0.5, "sx": 0.2, "sy": 0.02, "sz": 0.2, "materialIndex": 1},
      {"name": "Block", "type": "BOX", "px": 0.3, "py": 0.25, "pz": 0.6, "sx": 0.15, "sy": 0.25, "sz": 0.15,
       "ry": 22.5, "materialIndex": 2},
      {"name": "Ball", "type": "SPHERE", "px": 0.7, "py": 0.2, "pz": 0.4, "sx": 0.2, "stacks": 12, "slices": 20,
       "materialIndex": 3}]}"""
    desc = sj.loads(text).to_scene_desc()
    cam = scenes.camera(scenes.CORNELL_ORBIT, scenes.LensDesc(), orc)
    W, H = 48, 32
    cpu, _ = orc.render(scenes.build_scene(desc, orc, po.MAT), cam, (1, 1.0), W, H, 0, 2)
    with _ctx(product, W, H, product.RC_MATH_EXACT) as ctx:
        ctx.upload(product.build_scene(desc))
        ctx.render(cam, (1, 1.0), 0, 2)
        _same_images(ctx.read_buffers(), cpu)
        assert ctx.counters()["error_word"] == 0


def test_display_exact_matches_oracle(product, orc, c1):
    """rc_display (the export path's display pass and RGBA8 read-back):
    exact math gives the oracle's bytes for the denoised frame, with the
    export path's uniforms (1 sample, exposure 1) and with others; the image
    is written rows top first, and a call that keeps the image on the device
    leaves the next read unchanged."""
    w, sc, cam = c1
    W, H = 96, 64
    p = product.rc_atrous_params(1, 5, 1.0, 128.0, 1.0, 0, 1.0)
    with _ctx(product, W, H, product.RC_MATH_EXACT) as ctx:
        ctx.upload(sc)
        ctx.render(cam, (1, 1.0), 0, 4)
        out = ctx.denoise(p)
        img = ctx.display()
        assert img.shape == (H, W, 4) and img.dtype == np.uint8
        np.testing.assert_array_equal(img, orc.display(out, W, H, 1, 1.0))
        assert (img[..., 3] == 255).all() and img[..., :3].std() > 10
        np.testing.assert_array_equal(ctx.display(4, 1.5), orc.display(out, W, H, 4, 1.5))
        assert ctx.display(read=False) is None
        np.testing.assert_array_equal(ctx.display(), img)
        assert ctx.counters()["error_word"] == 0


def test_display_fast_close_and_exported_png(product, orc, c1, tmp_path):
    """Fast math (approximate divide and pow) stays within one step of the
    8-bit code; export_frame writes the same bytes as a PNG."""
    from retrocam_b200 import export
    w, sc, cam = c1
    W, H = 96, 64
    p = product.rc_atrous_params(1, 3, 1.0, 64.0, 1.0, 0, 1.0)
    with _ctx(product, W, H, product.RC_MATH_FAST) as ctx:
        ctx.upload(sc)
        ctx.render(cam, (1, 1.0), 0, 4)
        out = ctx.denoise(p)
        img = export.export_frame(ctx, str(tmp_path / "out" / "frame.png"))
    ref = orc.display(out, W, H, 1, 1.0)
    d = np.abs(img.astype(np.int32) - ref.astype(np.int32))
    assert d.max() <= 1 and (d == 0).mean() > 0.99, (d.max(), (d == 0).mean())
    np.testing.assert_array_equal(export.read_png(str(tmp_path / "out" / "frame.png")), img)


def test_atrous_exact_bit_identical(product, orc, c1):
    import pyoracle as po
    w, sc, cam = c1
    W, H, spp = 128, 72, 4
    p = product.rc_atrous_params(1, 5, 1.0, 128.0, 1.0, 0, 1.0)
    with _ctx(product, W, H, product.RC_MATH_EXACT) as ctx:
        ctx.upload(sc)
        ctx.render(cam, (1, 1.0), 0, spp)
        acc, gb, ga, var = ctx.read_buffers()
        out = ctx.denoise(p)
        # disabled denoiser = p00 only
        p_off = product.rc_atrous_params(0, 5, 1.0, 128.0, 1.0, 0, 1.5)
        out_off = ctx.denoise(p_off)
    ref_out = orc.denoise(acc, gb, ga, var, W, H, spp, po.AtrousParams(1, 5, 1.0, 128.0, 1.0, 0, 1.0))
    assert np.array_equal(bits(out), bits(ref_out))
    ref_off = orc.p00(acc, W, H, spp, 1.5)
    assert np.array_equal(bits(out_off), bits(ref_off))


@pytest.mark.parametrize("iters,step_sigma", [(1, 64.0), (3, 16.0)])
def test_atrous_fast_close(product, orc, c1, iters, step_sigma):
    import pyoracle as po
    w, sc, cam = c1
    W, H, spp = 128, 72, 4
    p = product.rc_atrous_params(1, iters, 1.0, step_sigma, 0.15, 0, 1.0)
    with _ctx(product, W, H, product.RC_MATH_EXACT) as ctx:
        ctx.upload(sc)
        ctx.render(cam, (1, 1.0), 0, spp)
        acc, gb, ga, var = ctx.read_buffers()
        ctx.set_math_mode(product.RC_MATH_FAST)
        out = ctx.denoise(p)
    ref_out = orc.denoise(acc, gb, ga, var, W, H, spp, po.AtrousParams(1, iters, 1.0, step_sigma, 0.15, 0, 1.0))
    np.testing.assert_allclose(out, ref_out, rtol=2e-3, atol=2e-4)


def test_render_frame_matches_reference_sequence(product, orc, c1):
    """rc_render_frame with SPPM iterations == spp is the reference export
    loop: trace -> render 1 spp -> gather -> shrink radius, then p00+à-trous."""
    import pyoracle as po
    w, sc, cam = c1
    W, H, spp, N, hs, r0, alpha = 96, 64, 3, 100_000, 1 << 18, 0.02, 0.7
    p = product.rc_atrous_params(1, 5, 1.0, 128.0, 1.0, 0, 1.0)
    with _ctx(product, W, H, product.RC_MATH_EXACT) as ctx:
        ctx.upload(sc)
        out = ctx.render_frame(cam, (1, 1.0), spp, product.rc_sppm_params(N, hs, alpha), r0, spp, p)
        acc = ctx.read_buffers()[0]
        r_end, it_end = ctx.sppm_state()
    bufs = po.alloc_images(W, H)
    r = r0
    for i in range(spp):
        ph, hd, nx, cnt, _ = orc.photon_trace(sc, N, r, i * 7919 + 6271, hs)
        orc.render(sc, cam, (1, 1.0), W, H, i, 1, buffers=bufs)
        orc.photon_gather(sc, cam, W, H, r, hs, ph, hd, nx, bufs[0])
        r = orc.lib.or_sppm_next_radius(r, i, alpha)
    assert it_end == spp and np.float32(r_end) == np.float32(r)
    np.testing.assert_allclose(acc, bufs[0], rtol=2e-5, atol=1e-6)
    ref_out = orc.denoise(*bufs, W, H, spp, po.AtrousParams(1, 5, 1.0, 128.0, 1.0, 0, 1.0))
    np.testing.assert_allclose(out, ref_out, rtol=1e-3, atol=1e-5)


def _batch_frames(product, n, spps, iters):
    from retrocam_b200 import scenes
    frames = scenes.keyframe_batch(product.HOST, n_frames=n)
    return [(cam, s, it) for (cam, _, _), s, it in zip(frames, spps, iters)]


@pytest.mark.parametrize("use_graph", [False, True])
def test_batch_without_sppm_bit_identical_to_frames(product, c1, use_graph):
    """A batch packs slices of several frames into shared chunks (here split
    across many small chunks); without SPPM every frame is bit-identical to
    its own rc_render_frame, with and without the CUDA graph."""
    w, sc, cam = c1
    W, H = 96, 64
    frames = _batch_frames(product, 4, (3, 5, 2, 4), (0, 0, 0, 0))
    p = product.rc_atrous_params(1, 5, 1.0, 128.0, 1.0, 0, 1.0)
    with _ctx(product, W, H, product.RC_MATH_EXACT) as ctx:
        ctx.set_tuning(chunk_paths=30_000)
        ctx.upload(sc)
        single = [ctx.render_frame(c, (1, 1.0), s, None, 0.02, 0, p) for c, s, _ in frames]
        batch = ctx.render_frames(frames, (1, 1.0), None, 0.02, p, use_graph=use_graph)
        again = ctx.render_frames(frames, (1, 1.0), None, 0.02, p, use_graph=use_graph)
        assert ctx.counters()["error_word"] == 0
    for f in range(len(frames)):
        assert np.array_equal(bits(batch[f]), bits(single[f])), f
    assert np.array_equal(bits(again), bits(batch))


def test_batch_with_sppm_matches_frames(product, c1):
    """With SPPM, iteration k's photon map is traced once for all frames;
    each frame's slices, gathers and radius schedule follow rc_render_frame.
    Only the hash-chain order of the gather sums differs (GPU atomics)."""
    w, sc, cam = c1
    W, H, N, hs = 96, 64, 100_000, 1 << 18
    frames = _batch_frames(product, 3, (6, 4, 5), (3, 4, 0))
    p = product.rc_atrous_params(1, 5, 1.0, 128.0, 1.0, 0, 1.0)
    sp = product.rc_sppm_params(N, hs, 0.7)
    with _ctx(product, W, H, product.RC_MATH_EXACT) as ctx:
        ctx.upload(sc)
        single = [ctx.render_frame(c, (1, 1.0), s, sp, 0.02, it, p) for c, s, it in frames]
        batch = ctx.render_frames(frames, (1, 1.0), sp, 0.02, p, use_graph=True)
        assert ctx.counters()["error_word"] == 0
    for f in range(len(frames)):
        close = np.abs(batch[f] - single[f]) <= 1e-3 * np.abs(single[f]) + 1e-5
        assert np.mean(close) > 0.999, (f, np.mean(close))
        np.testing.assert_allclose(batch[f].mean(axis=(0, 1)), single[f].mean(axis=(0, 1)), rtol=1e-4)
    # frame 2 has no SPPM: bit-identical
    assert np.array_equal(bits(batch[2]), bits(single[2]))


def test_errors_are_codes_not_crashes(product, c0):
    w, sc, cam = c0
    with _ctx(product, 32, 32, product.RC_MATH_FAST) as ctx:
        with pytest.raises(product.RetroCamError) as e:
            ctx.render(cam)
        assert e.value.code == product.RC_ERR_NO_SCENE
        bad = dict(sc)
        nodes = sc["nodes"].copy()
        interior = np.nonzero(nodes["prim_count"] == 0)[0]
        nodes[interior[0]]["left_child"] = len(nodes) + 5
        bad["nodes"] = nodes
        with pytest.raises(product.RetroCamError) as e:
            ctx.upload(bad)
        assert e.value.code == product.RC_ERR_BAD_SCENE
        cyc = sc["nodes"].copy()
        cyc[interior[-1]]["left_child"] = 0       # a cycle back to the root
        bad["nodes"] = cyc
        with pytest.raises(product.RetroCamError) as e:
            ctx.upload(bad)
        assert e.value.code == product.RC_ERR_BAD_SCENE
        ctx.upload(sc)
        with pytest.raises(product.RetroCamError) as e:
            ctx.sppm_trace(1000, 1000)               # not a power of two
        assert e.value.code == product.RC_ERR_INVALID_ARG
        with pytest.raises(product.RetroCamError) as e:
            ctx.render(cam, (1, 1.0), -1, 1)
        assert e.value.code == product.RC_ERR_INVALID_ARG
        ctx.render(cam, (1, 1.0), 0, 1)             # still usable
        ctx.synchronize()
