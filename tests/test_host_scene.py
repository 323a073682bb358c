"""The C ABI's host half against the oracle (CPU only): tessellation, the SAH
BVH builder, the light list, camera helpers, the SPPM radius schedule and
keyframes must equal the oracle's restatement of the reference's Java bit for
bit.  Also: the library loads without a GPU and exports every function that
include/retrocam.h declares; host functions report bad arguments as codes.
"""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import REPO, bits


@pytest.fixture(scope="module")
def host(product):
    return product.HOST


def test_library_exports_every_declared_function(product):
    header = open(os.path.join(REPO, "include", "retrocam.h")).read()
    names = set(re.findall(r"^\s*(?:int|float|void)\s+(rc_\w+)\s*\(", header, flags=re.M))
    assert len(names) >= 35
    L = product.lib()
    missing = [n for n in sorted(names) if not hasattr(L, n)]
    assert not missing, missing
    assert L.rc_abi_version() == 1


def test_record_layouts_match_oracle(product):
    import pyoracle as po
    for a, b in ((product.TRIANGLE, po.TRI), (product.BVH_NODE, po.NODE), (product.MATERIAL, po.MAT),
                 (product.LIGHT, po.LIGHT), (product.PHOTON, po.PHOTON)):
        assert a.itemsize == b.itemsize and a.names == b.names
    assert C.sizeof(product.rc_camera) == 4 * 20


@pytest.mark.parametrize("rot", [(0.0, 0.0, 0.0), (0.0, 15.0, 0.0), (0.0, -18.0, 0.0), (33.0, -71.5, 190.0)])
def test_box_bit_identical(host, orc, rot):
    for c, h in (((0.66, 0.3, 0.62), (0.15, 0.3, 0.15)), ((0.0, 0.0, 0.0), (1.0, 0.05, 1.0)),
                 ((-1.5, 1.5, -1.0), (1.0, 1.5, 1.0))):
        assert np.array_equal(bits(host.tess_box(c, h, 3, rot).view(np.float32)),
                              bits(orc.tess_box(c, h, 3, rot).view(np.float32)))


@pytest.mark.parametrize("stacks,slices,rot", [(32, 64, (0.0, 0.0, 0.0)), (24, 24, (0.0, 0.0, 0.0)),
                                               (7, 5, (10.0, 20.0, 30.0)), (2, 3, (0.0, 0.0, 0.0))])
def test_sphere_bit_identical(host, orc, stacks, slices, rot):
    a = host.tess_sphere((0.34, 0.45, 0.35), 0.15, 4, stacks, slices, rot)
    b = orc.tess_sphere((0.34, 0.45, 0.35), 0.15, 4, stacks, slices, rot)
    assert len(a) == len(b) == 2 * stacks * slices - 2 * slices
    assert np.array_equal(bits(a.view(np.float32)), bits(b.view(np.float32)))


def _scene_both(product, orc, desc):
    import pyoracle as po
    from retrocam_b200 import scenes
    return product.build_scene(desc), scenes.build_scene(desc, orc, po.MAT)


@pytest.mark.parametrize("name", ["cornell_small", "export_frame"])
def test_scene_build_bit_identical(product, orc, name):
    from retrocam_b200 import scenes
    a, b = _scene_both(product, orc, scenes.WORKLOADS[name]().scene)
    for k in ("tris", "nodes", "mats"):
        assert np.array_equal(a[k].view(np.uint8), b[k].view(np.uint8)), k
    assert a["light_count"] == b["light_count"]
    assert np.array_equal(a["lights"].view(np.uint8), b["lights"].view(np.uint8))
    assert np.float32(a["total_power"]) == np.float32(b["total_power"])


def test_bvh_stress_million_triangles_bit_identical(product, orc):
    """The 1,000,000-triangle scene: node order, primitive order and boxes."""
    from retrocam_b200 import scenes
    w = scenes.bvh_stress()
    a, b = _scene_both(product, orc, w.scene)
    assert len(a["tris"]) == 1_000_000 + 10 + 8
    assert np.array_equal(a["nodes"].view(np.uint8), b["nodes"].view(np.uint8))
    assert np.array_equal(a["tris"].view(np.uint8), b["tris"].view(np.uint8))
    assert a["light_count"] == b["light_count"] == 8


def test_bvh_degenerate_inputs(host, orc):
    # all triangles at one point: SAH finds no split -> a single leaf
    tris = host.flat_triangles(np.zeros((9, 9), np.float32), 0)
    ta, na = host.build_bvh(tris)
    tb, nb = orc.build_bvh(tris)
    assert len(na) == len(nb) == 1 and na[0]["prim_count"] == 9
    # duplicated coordinates and signed zeros keep Java's min/max semantics
    p = np.array([[0, 0, 0, -0.0, 1, 0, 0, 0, 1]] * 3 + [[-0.0, 0, 0, 0, 1, 0, 0, -0.0, 1]] * 4 +
                 [[5, 5, 5, 6, 5, 5, 5, 6, 5]] * 6, np.float32)
    tris = host.flat_triangles(p, 1)
    ta, na = host.build_bvh(tris)
    tb, nb = orc.build_bvh(orc.flat_triangles(p, 1))
    assert np.array_equal(na.view(np.uint8), nb.view(np.uint8))
    assert np.array_equal(ta.view(np.uint8), tb.view(np.uint8))


def test_camera_helpers_bit_identical(host, orc):
    import math
    for f, n in ((35.0, 16.0), (28.0, 2.8), (20.0, 1.8), (80.0, 16.0)):
        assert host.thin_lens(f, n) == orc.thin_lens(f, n)
    for th, ph, r, t in ((-math.pi / 2, math.pi / 2, 1.9, (0.5, 0.5, 0.5)), (math.pi / 2, 1.2, 10.0, (0, 5, 0)),
                         (0.3, 0.02, 3.0, (1, 2, 3))):
        assert np.array_equal(bits(host.orbit_basis(th, ph, r, t)), bits(orc.orbit_basis(th, ph, r, t)))


def test_radius_and_keyframes_bit_identical(product, orc):
    L = product.lib()
    r1 = r2 = 0.02
    for n in range(30):
        r1 = L.rc_sppm_next_radius(r1, n, 0.7)
        r2 = orc.lib.or_sppm_next_radius(r2, n, 0.7)
        assert np.float32(r1) == np.float32(r2)
    t = np.array([0.0, 0.3, 1.1, 2.0, 3.5], np.float32)
    v = np.array([0.0, 90.0, 20.0, 80.0, 16.0], np.float32)
    for mode in (0, 1, 2):
        ip = np.full(5, mode, np.int32)
        for x in np.linspace(-0.5, 4.0, 37, dtype=np.float32):
            a = L.rc_keyframe_evaluate(t.ctypes.data, v.ctypes.data, ip.ctypes.data, 5, float(x), -1.0)
            b = orc.lib.or_keyframe_eval(t.ctypes.data, v.ctypes.data, ip.ctypes.data, 5, float(x), -1.0)
            assert np.float32(a) == np.float32(b)


def test_host_functions_return_codes(product):
    L = product.lib()
    assert L.rc_tessellate_box(0, 0, 0, 1, 1, 1, 0, 0, 0, 0, None) == product.RC_ERR_INVALID_ARG
    out = np.zeros(4, product.TRIANGLE)
    n = C.c_int(0)
    assert L.rc_tessellate_sphere(0, 0, 0, 1, 0, 8, 8, 0, 0, 0, out.ctypes.data, 4, C.byref(n)) == \
        product.RC_ERR_CAPACITY
    tris = product.HOST.flat_triangles(np.random.default_rng(0).random((50, 9)).astype(np.float32), 0)
    nodes = np.zeros(3, product.BVH_NODE)
    assert L.rc_build_bvh(tris.ctypes.data, 50, np.zeros_like(tris).ctypes.data, nodes.ctypes.data, 3,
                          C.byref(n)) == product.RC_ERR_CAPACITY
    assert L.rc_build_bvh(None, 0, None, None, 0, C.byref(n)) == product.RC_ERR_INVALID_ARG
    mats = np.zeros(1, product.MATERIAL)
    tris["mat_index"][3] = 5  # out of range
    lights = np.zeros(50, product.LIGHT)
    tp = C.c_float(0)
    assert L.rc_build_lights(tris.ctypes.data, 50, mats.ctypes.data, 1, lights.ctypes.data, 50, C.byref(n),
                             C.byref(tp)) == product.RC_ERR_INVALID_ARG


def test_context_creation_without_gpu_is_an_error_code(product):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    code = product.lib().rc_ctx_create(64, 64, 0, C.byref(h))
    assert code == product.RC_ERR_CUDA
    buf = C.create_string_buffer(256)
    product.lib().rc_last_error(None, buf, 256)
    assert b"device" in buf.value
