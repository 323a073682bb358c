"""Known-answer tests of the oracle (CPU only).

The reference ships no tests or golden data for this path, so the answers
here are computed independently in Python from the constants and formulas
the reference states (pathtrace.comp:80-98, photon_trace.comp:60-72,140-143,
SPPMManager.java:170-173, KeyframeTrack.java:102-178, Sphere.java:57-58,
SceneUploader.java:199-205) and compared with the oracle's C++ restatement.
"""
import ctypes as C
import math

import numpy as np
import pytest

M32 = 0xFFFFFFFF


def pcg_py(state):
    state = (state * 747796405 + 2891336453) & M32
    w = (((state >> ((state >> 28) + 4)) ^ state) * 277803737) & M32
    return state, (w >> 22) ^ w


def test_pcg_stream_known_answers(orc):
    for seed in (0, 1, 12345, 0xDEADBEEF, M32):
        s_py, s_c = seed, C.c_uint32(seed)
        for _ in range(500):
            s_py, out = pcg_py(s_py)
            assert orc.lib.or_pcg_next(C.byref(s_c)) == out
        assert s_c.value == s_py


def test_rand_is_u32_over_2_pow_32_in_float(orc):
    rng = np.random.default_rng(0)
    for seed in rng.integers(0, 2**32, 2000, dtype=np.uint64).tolist():
        _, out = pcg_py(seed)
        want = np.float32(np.float32(out) / np.float32(4294967296.0))
        assert orc.lib.or_rand(C.byref(C.c_uint32(seed))) == want
    # float(u32) rounds to 2^32 for the top 128 values, so rand() can be 1.0
    assert np.float32(np.float32(M32) / np.float32(4294967296.0)) == 1.0


def init_seed_py(px, py, frame):
    s = (px + py * 7919 + frame * 6271) & M32  # GLSL int arithmetic wraps
    s, _ = pcg_py(s)
    s, _ = pcg_py(s)
    return s


def test_init_seed_and_photon_seed(orc):
    rng = np.random.default_rng(1)
    for px, py, f in [(0, 0, 0), (853, 479, 127), (5, 7, 99991), (1, 2, 2**29), (3, 4, -5)]:
        assert orc.lib.or_init_seed(px, py, f) == init_seed_py(px, py, f)
    for idx, seed in zip(rng.integers(0, 2_000_000, 100).tolist(), rng.integers(0, 200_000, 100).tolist()):
        s = (idx * 1664525 + seed * 1013904223 + 2531011) & M32
        s, _ = pcg_py(s)
        s, _ = pcg_py(s)
        assert orc.lib.or_photon_seed(idx, seed) == s


def test_cell_hash_wraps_like_glsl_int(orc):
    def h(cx, cy, cz, size):
        v = ((cx * 73856093) ^ (cy * 19349663) ^ (cz * 83492791)) & M32
        return v & (size - 1)
    for c in [(0, 0, 0), (1, 2, 3), (-1, -1, -1), (50, -3, 49), (2**20, -2**20, 12345), (-7, 400, -90000)]:
        for size in (1 << 22, 1 << 16, 1):
            assert orc.lib.or_cell_hash(*c, size) == h(*c, size)


def _tri(orc, v0, v1, v2):
    return orc.flat_triangles(np.array([v0 + v1 + v2], np.float32), 0)


def _isect(orc, tri, ro, rd):
    ro = np.array(ro, np.float32)
    rd = np.array(rd, np.float32)
    out = np.zeros(3, np.float32)
    hit = orc.lib.or_intersect_triangle(ro.ctypes.data, rd.ctypes.data, tri.ctypes.data, out.ctypes.data)
    return bool(hit), out


def test_moller_trumbore_edge_cases(orc):
    tri = _tri(orc, (0, 0, 0), (1, 0, 0), (0, 1, 0))
    hit, tuv = _isect(orc, tri, (0.25, 0.25, 1.0), (0, 0, -1))
    assert hit and tuv[0] == np.float32(1.0)
    # edges are inclusive: u = 0 and u + v = 1 both hit
    assert _isect(orc, tri, (0.0, 0.5, 1.0), (0, 0, -1))[0]
    assert _isect(orc, tri, (0.5, 0.5, 1.0), (0, 0, -1))[0]
    assert not _isect(orc, tri, (0.6, 0.6, 1.0), (0, 0, -1))[0]
    # parallel ray: |a| < 1e-8 rejects
    assert not _isect(orc, tri, (0.25, 0.25, 1.0), (1, 0, 0))[0]
    # hits closer than t = 1e-4 are rejected (self-intersection guard)
    assert not _isect(orc, tri, (0.25, 0.25, 5e-5), (0, 0, -1))[0]
    assert _isect(orc, tri, (0.25, 0.25, 2e-4), (0, 0, -1))[0]
    # behind the origin
    assert not _isect(orc, tri, (0.25, 0.25, -1.0), (0, 0, -1))[0]
    # degenerate triangle never hits
    deg = _tri(orc, (0, 0, 0), (1, 1, 1), (2, 2, 2))
    assert not _isect(orc, deg, (0.5, 0.5, 1.0), (0, 0, -1))[0]


def test_slab_test_with_infinite_inverse_direction(orc):
    import pyoracle as po
    node = np.zeros(1, po.NODE)
    node["aabb_min"] = (0, 0, 0)
    node["aabb_max"] = (1, 1, 1)
    t = C.c_float(0)

    def hit(ro, rd):
        ro = np.array(ro, np.float32)
        rd = np.array(rd, np.float32)
        return orc.lib.or_intersect_aabb(ro.ctypes.data, rd.ctypes.data, node.ctypes.data, C.byref(t))

    assert hit((0.5, 0.5, -1), (0, 0, 1)) == 1 and t.value == 1.0   # 1/0 = inf on x and y
    assert hit((2.0, 0.5, -1), (0, 0, 1)) == 0                      # outside the x slab
    assert hit((0.5, 0.5, 0.5), (0, 0, 1)) == 1 and t.value < 0     # origin inside: tmin < 0 still hits
    assert hit((0.5, 0.5, 2.0), (0, 0, 1)) == 0                     # box behind the ray


@pytest.mark.parametrize("fn,ref", [("or_sinf", math.sin), ("or_cosf", math.cos), ("or_expf", math.exp),
                                    ("or_logf", math.log)])
def test_exact_math_is_correctly_rounded(orc, fn, ref):
    rng = np.random.default_rng(2)
    if fn in ("or_sinf", "or_cosf"):
        xs = rng.uniform(-7, 7, 20000).astype(np.float32)
    elif fn == "or_expf":
        xs = rng.uniform(-100, 80, 20000).astype(np.float32)
    else:
        xs = (rng.uniform(0.5, 1, 20000) * 2.0 ** rng.integers(-120, 120, 20000)).astype(np.float32)
    f = getattr(orc.lib, fn)
    got = np.array([f(float(x)) for x in xs], np.float32)
    want = np.array([ref(float(x)) for x in xs]).astype(np.float32)
    assert np.mean(got == want) > 0.9999
    assert np.max(np.abs(got.astype(np.float64) - want) / np.maximum(np.abs(want), 1e-30)) < 1.2e-7


def test_exact_pow_specials(orc):
    p = orc.lib.or_powf
    assert p(0.0, 5.0) == 0.0 and p(2.0, 0.0) == 1.0 and p(1.0, 123.0) == 1.0
    assert p(0.5, 5.0) == np.float32(0.03125)
    assert p(0.9, 128.0) == np.float32(float(np.float32(0.9)) ** 128)
    assert math.isinf(p(0.0, -1.0))


def test_half_conversion_matches_ieee(orc):
    rng = np.random.default_rng(3)
    xs = np.concatenate([rng.normal(0, 10, 5000), rng.normal(0, 1e-5, 2000), [0.0, -0.0, 65504, 65520, 1e5, -1e5,
                                                                              6e-8, 3e-8, 1e4, 5.96e-8]])
    xs = xs.astype(np.float32)
    for x in xs:
        h = orc.lib.or_float_to_half(float(x))
        assert h == np.array([x], np.float32).astype(np.float16).view(np.uint16)[0]
        assert orc.lib.or_half_to_float(h) == np.uint16(h).view(np.float16).astype(np.float32)


def test_sphere_skips_pole_triangles(orc):
    t = orc.tess_sphere((0, 0, 0), 1.0, 0, 32, 64)
    assert len(t) == 2 * 32 * 64 - 2 * 64 == 3968
    t = orc.tess_sphere((0, 0, 0), 1.0, 0, 24, 24)
    assert len(t) == 24 * 24 * 2 - 48
    n = np.linalg.norm(t["n0"], axis=1)
    assert np.allclose(n, 1.0, atol=1e-6)


def test_box_and_rotation(orc):
    b = orc.tess_box((0.5, 0.5, 0.5), (0.1, 0.2, 0.3), 7)
    assert len(b) == 12 and (b["mat_index"] == 7).all()
    assert np.allclose(np.linalg.norm(b["n0"], axis=1), 1.0)
    r = orc.tess_box((0.5, 0.5, 0.5), (0.1, 0.2, 0.3), 7, rot=(0.0, 90.0, 0.0))
    # a quarter turn about y swaps the x and z extents
    v = np.concatenate([r["v0"], r["v1"], r["v2"]])
    assert np.allclose(v[:, 0].max() - v[:, 0].min(), 0.6, atol=1e-6)
    assert np.allclose(v[:, 2].max() - v[:, 2].min(), 0.2, atol=1e-6)


def _check_bvh(tris, nodes):
    n = len(tris)
    covered = np.zeros(n, int)
    stack = [0]
    order = []
    while stack:
        i = stack.pop()
        order.append(i)
        nd = nodes[i]
        if nd["prim_count"] > 0:
            s, c = nd["prim_start"], nd["prim_count"]
            covered[s:s + c] += 1
            v = np.concatenate([tris["v0"][s:s + c], tris["v1"][s:s + c], tris["v2"][s:s + c]])
            assert (v >= nd["aabb_min"] - 0).all() and (v <= nd["aabb_max"] + 0).all()
        else:
            l, r = nd["left_child"], nd["right_child"]
            assert l == i + 1  # depth-first pre-order: left child follows its parent
            for ch in (l, r):
                assert (nodes[ch]["aabb_min"] >= nd["aabb_min"]).all()
                assert (nodes[ch]["aabb_max"] <= nd["aabb_max"]).all()
            stack += [r, l]
    assert (covered == 1).all()
    assert sorted(order) == list(range(len(nodes)))


def test_bvh_invariants_and_determinism(orc):
    import pyoracle as po
    from retrocam_b200 import scenes
    for wl in (scenes.cornell_small, scenes.export_frame):
        w = wl()
        sc = scenes.build_scene(w.scene, orc, po.MAT)
        _check_bvh(sc["tris"], sc["nodes"])
        again = scenes.build_scene(w.scene, orc, po.MAT)
        assert np.array_equal(sc["nodes"].view(np.uint32), again["nodes"].view(np.uint32))
        assert np.array_equal(sc["tris"].view(np.uint32), again["tris"].view(np.uint32))
    assert len(scenes.build_scene(scenes.cornell_small().scene, orc, po.MAT)["tris"]) == 36
    assert len(scenes.build_scene(scenes.export_frame().scene, orc, po.MAT)["tris"]) == 36 + 2 * 3968


def test_light_list_and_cdf(orc):
    import pyoracle as po
    from retrocam_b200 import scenes
    sc = scenes.build_scene(scenes.export_frame().scene, orc, po.MAT)
    L = sc["lights"][:sc["light_count"]]
    assert sc["light_count"] == 2
    assert L["cdf_weight"][-1] == np.float32(1.0)
    assert (np.diff(L["cdf_weight"]) >= 0).all()
    assert np.isclose(L["power"].sum(), sc["total_power"], rtol=1e-6)
    # emission (17,12,4): power = luma601 * area * pi with the 0.25^2 quad split in two
    lum = 0.299 * 17 + 0.587 * 12 + 0.114 * 4
    assert np.isclose(sc["total_power"], lum * 0.0625 * math.pi, rtol=1e-5)
    assert (L["normal"][:, 1] < 0).all()  # the quad faces down into the box


def test_scene_without_lights_gets_stub(orc):
    import pyoracle as po
    from retrocam_b200 import scenes
    desc = scenes.SceneDesc([scenes.diffuse(0.5, 0.5, 0.5)], [scenes.Box((0, 0, 0), (1, 1, 1), 0)])
    sc = scenes.build_scene(desc, orc, po.MAT)
    assert sc["light_count"] == 0 and len(sc["lights"]) == 1 and sc["total_power"] == 0.0


def test_sppm_radius_schedule(orc):
    r = np.float32(0.02)
    for n in range(40):
        num = np.float32(np.float32(n) + np.float32(0.7))
        want = np.float32(r * np.float32(math.sqrt(float(num) / (n + 1.0))))
        got = np.float32(orc.lib.or_sppm_next_radius(float(r), n, 0.7))
        assert got == want
        r = got


def test_keyframe_interpolation(orc):
    t = np.array([0.0, 1.0, 2.0, 4.0], np.float32)
    v = np.array([0.0, 10.0, 5.0, 7.0], np.float32)
    f = np.float32
    for interp_mode in (0, 1, 2):
        ip = np.full(4, interp_mode, np.int32)
        ev = lambda x: orc.lib.or_keyframe_eval(t.ctypes.data, v.ctypes.data, ip.ctypes.data, 4, x, -1.0)  # noqa
        assert ev(-1.0) == 0.0 and ev(5.0) == 7.0
        x = f(1.5)
        lt = f((x - t[1]) / (t[2] - t[1]))
        if interp_mode == 0:
            assert ev(1.5) == 10.0
        elif interp_mode == 1:
            assert ev(1.5) == f(v[1] + f(v[2] - v[1]) * lt)
        else:
            dt = f(t[2] - t[1])
            m0 = f(f(v[2] - v[0]) / f(t[2] - t[0]))
            m1 = f(f(v[3] - v[1]) / f(t[3] - t[1]))
            t2, t3 = f(lt * lt), f(f(lt * lt) * lt)
            h00 = f(f(f(f(2) * t3) - f(f(3) * t2)) + f(1))
            h10 = f(f(t3 - f(f(2) * t2)) + lt)
            h01 = f(f(f(-2) * t3) + f(f(3) * t2))
            h11 = f(t3 - t2)
            want = f(f(f(f(h00 * v[1]) + f(f(h10 * dt) * m0)) + f(h01 * v[2])) + f(f(h11 * dt) * m1))
            assert ev(1.5) == want
    assert orc.lib.or_keyframe_eval(t.ctypes.data, v.ctypes.data, np.zeros(4, np.int32).ctypes.data, 0,
                                    1.0, -3.0) == -3.0
