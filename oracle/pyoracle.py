"""TEST INFRASTRUCTURE (oracle): ctypes bindings for the CPU oracle
(oracle/_build/liboracle.so) and the compiled reference shaders
(oracle/_ref/libretrocam_ref.so).  Only tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg import this module.

Record dtypes below restate the std430 layouts of the reference SSBOs
(scene/GpuTriangle.java:68-78, BVHNode.java:32-41, Material.java:61-69,
SceneUploader.java:18-23, PhotonMap.java:16-21) independently of the
product's own definitions.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "_build", "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libretrocam_ref.so")
# the same shaders with the host C library's sin/cos/exp/log/pow: a timing
# variant of the CPU baseline, not a parity reference
REF_LIB_LIBM = os.path.join(HERE, "_ref", "libretrocam_ref_libm.so")

F3 = ("<f4", 3)
TRI = np.dtype([("v0",) + F3, ("pad0", "<f4"), ("v1",) + F3, ("pad1", "<f4"), ("v2",) + F3, ("pad2", "<f4"),
                ("n0",) + F3, ("pad3", "<f4"), ("n1",) + F3, ("pad4", "<f4"), ("n2",) + F3, ("pad5", "<f4"),
                ("uv0", "<f4", 2), ("uv1", "<f4", 2), ("uv2", "<f4", 2), ("mat_index", "<i4"), ("pad6", "<f4")])
NODE = np.dtype([("aabb_min",) + F3, ("pad0", "<f4"), ("aabb_max",) + F3, ("pad1", "<f4"),
                 ("left_child", "<i4"), ("right_child", "<i4"), ("prim_start", "<i4"), ("prim_count", "<i4")])
MAT = np.dtype([("albedo",) + F3, ("metallic", "<f4"), ("emission",) + F3, ("emission_strength", "<f4"),
                ("roughness", "<f4"), ("ior", "<f4"), ("transmission", "<f4"), ("albedo_tex", "<i4"),
                ("pad", "<f4", 4)])
LIGHT = np.dtype([("v0",) + F3, ("area", "<f4"), ("v1",) + F3, ("pad1", "<f4"), ("v2",) + F3, ("pad2", "<f4"),
                  ("emission",) + F3, ("power", "<f4"), ("normal",) + F3, ("cdf_weight", "<f4")])
PHOTON = np.dtype([("position",) + F3, ("pad0", "<f4"), ("power",) + F3, ("pad1", "<f4"),
                   ("dir",) + F3, ("pad2", "<f4")])
assert TRI.itemsize == 128 and NODE.itemsize == 48 and MAT.itemsize == 64
assert LIGHT.itemsize == 80 and PHOTON.itemsize == 48


class Camera(C.Structure):
    _fields_ = [("cam_pos", C.c_float * 3), ("cam_right", C.c_float * 3), ("cam_up", C.c_float * 3),
                ("cam_forward", C.c_float * 3), ("focal_dist", C.c_float), ("lens_radius", C.c_float),
                ("fov_tan_half", C.c_float), ("aperture_blades", C.c_int32), ("sa_strength", C.c_float),
                ("lca_delta", C.c_float * 3)]


class Settings(C.Structure):
    _fields_ = [("nee_enabled", C.c_int32), ("nee_firefly_clamp", C.c_float)]


class AtrousParams(C.Structure):
    _fields_ = [("enabled", C.c_int32), ("iterations", C.c_int32), ("sigma_color", C.c_float),
                ("sigma_normal", C.c_float), ("sigma_depth", C.c_float), ("max_spp", C.c_int32),
                ("exposure", C.c_float)]


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def camera_struct(cam: dict) -> Camera:
    c = Camera()
    for k in ("cam_pos", "cam_right", "cam_up", "cam_forward", "lca_delta"):
        getattr(c, k)[:] = [float(x) for x in cam[k]]
    c.focal_dist = cam["focal_dist"]
    c.lens_radius = cam["lens_radius"]
    c.fov_tan_half = cam["fov_tan_half"]
    c.aperture_blades = int(cam["aperture_blades"])
    c.sa_strength = cam["sa_strength"]
    return c


_VP, _I, _F, _U32 = C.c_void_p, C.c_int, C.c_float, C.c_uint32


class Oracle:
    """The hand-written restatement (oracle/oracle.cpp, oracle_host.cpp)."""

    def __init__(self, path: str = ORACLE_LIB):
        self.lib = lib = C.CDLL(path)
        sig = {
            "or_pcg_next": (_U32, [C.POINTER(_U32)]),
            "or_rand": (_F, [C.POINTER(_U32)]),
            "or_init_seed": (_U32, [_I, _I, _I]),
            "or_photon_seed": (_U32, [_U32, _I]),
            "or_cell_hash": (_I, [_I, _I, _I, _I]),
            "or_intersect_triangle": (_I, [_VP, _VP, _VP, _VP]),
            "or_intersect_aabb": (_I, [_VP, _VP, _VP, _VP]),
            "or_sinf": (_F, [_F]), "or_cosf": (_F, [_F]), "or_expf": (_F, [_F]), "or_logf": (_F, [_F]),
            "or_powf": (_F, [_F, _F]),
            "or_float_to_half": (C.c_uint16, [_F]), "or_half_to_float": (_F, [C.c_uint16]),
            "or_tess_box": (_I, [_F] * 6 + [_I] + [_F] * 3 + [_VP]),
            "or_tess_sphere": (_I, [_F] * 4 + [_I, _I, _I] + [_F] * 3 + [_VP, _I]),
            "or_flat_triangles": (_I, [_VP, _I, _I, _VP]),
            "or_build_bvh": (_I, [_VP, _I, _VP, _VP, _I]),
            "or_build_lights": (_I, [_VP, _I, _VP, _VP, _I, C.POINTER(_F)]),
            "or_thin_lens": (None, [_F, _F, C.POINTER(_F), C.POINTER(_F)]),
            "or_orbit_basis": (None, [_F] * 6 + [_VP]),
            "or_sppm_next_radius": (_F, [_F, _I, _F]),
            "or_keyframe_eval": (_F, [_VP, _VP, _VP, _I, _F, _F]),
            "or_render": (_I, [_VP, _VP, _VP, _VP, _I, _F, _VP, _VP, _I, _I, _I, _I, _I, _I,
                               _VP, _VP, _VP, _VP, _VP, _I]),
            "or_photon_trace": (_I, [_VP, _VP, _VP, _VP, _I, _F, _I, _F, _I, _I, _VP, _VP, _VP, _VP, _VP, _I]),
            "or_photon_gather": (_I, [_VP, _VP, _VP, _VP, _I, _I, _F, _I, _VP, _VP, _VP, _F, _VP, _VP, _I]),
            "or_p00": (_I, [_VP, _I, _I, _I, _F, _VP, _I]),
            "or_atrous_pass": (_I, [_VP, _VP, _VP, _VP, _I, _I, _I, _F, _F, _F, _I, _F, _VP, _I]),
            "or_denoise": (_I, [_VP, _VP, _VP, _VP, _I, _I, _I, _VP, _VP, _I]),
            "or_display": (_I, [_VP, _I, _I, _I, _F, _VP, _I]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args

    # ---- scene building (Java host restated) ----
    def tess_box(self, c, h, mat, rot=(0.0, 0.0, 0.0)):
        out = np.zeros(12, TRI)
        n = self.lib.or_tess_box(*map(float, c), *map(float, h), int(mat), *map(float, rot), _p(out))
        return out[:n]

    def tess_sphere(self, c, r, mat, stacks, slices, rot=(0.0, 0.0, 0.0)):
        out = np.zeros(2 * stacks * slices, TRI)
        n = self.lib.or_tess_sphere(*map(float, c), float(r), int(mat), int(stacks), int(slices),
                                    *map(float, rot), _p(out), len(out))
        assert n >= 0
        return out[:n]

    def flat_triangles(self, positions, mat):
        pos = np.ascontiguousarray(positions, dtype=np.float32).reshape(-1, 9)
        out = np.zeros(len(pos), TRI)
        self.lib.or_flat_triangles(_p(pos), len(pos), int(mat), _p(out))
        return out

    def build_bvh(self, tris):
        tris = np.ascontiguousarray(tris)
        out_t = np.zeros_like(tris)
        cap = max(1, 2 * len(tris))
        out_n = np.zeros(cap, NODE)
        n = self.lib.or_build_bvh(_p(tris), len(tris), _p(out_t), _p(out_n), cap)
        assert n > 0
        return out_t, out_n[:n]

    def build_lights(self, tris, mats):
        tris = np.ascontiguousarray(tris)
        out = np.zeros(max(1, len(tris)), LIGHT)
        tp = C.c_float(0)
        n = self.lib.or_build_lights(_p(tris), len(tris), _p(np.ascontiguousarray(mats)), _p(out), len(out),
                                     C.byref(tp))
        return out[:n], tp.value

    def thin_lens(self, focal_mm, fstop):
        a, b = C.c_float(0), C.c_float(0)
        self.lib.or_thin_lens(focal_mm, fstop, C.byref(a), C.byref(b))
        return a.value, b.value

    def orbit_basis(self, theta, phi, radius, target):
        out = np.zeros(12, np.float32)
        self.lib.or_orbit_basis(theta, phi, radius, *map(float, target), _p(out))
        return out

    # ---- shaders restated ----
    def render(self, scene, cam, settings, W, H, first, nspp, buffers=None, rows=(0, 0), threads=0):
        acc, gb, ga, var = buffers if buffers is not None else alloc_images(W, H)
        st = np.zeros(10, np.uint64)
        self.lib.or_render(_p(scene["tris"]), _p(scene["nodes"]), _p(scene["mats"]), _p(scene["lights"]),
                           scene["light_count"], scene["total_power"], C.byref(camera_struct(cam)),
                           C.byref(Settings(*settings)), W, H, first, nspp, rows[0], rows[1],
                           _p(acc), _p(gb), _p(ga), _p(var), _p(st), threads)
        return (acc, gb, ga, var), st

    def photon_trace(self, scene, N, radius, seed, hash_size, threads=0):
        ph = np.zeros(max(N, 1), PHOTON)
        heads = np.zeros(hash_size, np.int32)
        nxt = np.zeros(max(N, 1), np.int32)
        cnt = np.zeros(1, np.uint32)
        st = np.zeros(10, np.uint64)
        self.lib.or_photon_trace(_p(scene["tris"]), _p(scene["nodes"]), _p(scene["mats"]), _p(scene["lights"]),
                                 scene["light_count"], scene["total_power"], N, radius, seed, hash_size,
                                 _p(ph), _p(heads), _p(nxt), _p(cnt), _p(st), threads)
        return ph, heads, nxt, int(cnt[0]), st

    def photon_gather(self, scene, cam, W, H, radius, hash_size, ph, heads, nxt, accum, weight=1.0, threads=0):
        st = np.zeros(10, np.uint64)
        self.lib.or_photon_gather(_p(scene["tris"]), _p(scene["nodes"]), _p(scene["mats"]),
                                  C.byref(camera_struct(cam)), W, H, radius, hash_size, _p(ph), _p(heads),
                                  _p(nxt), weight, _p(accum), _p(st), threads)
        return st

    def p00(self, accum, W, H, total, exposure, threads=0):
        out = np.zeros((H, W, 4), np.float32)
        self.lib.or_p00(_p(accum), W, H, total, exposure, _p(out), threads)
        return out

    def display(self, color, W, H, total=1, exposure=1.0, threads=0):
        """RGBA8 export image (rows top first) of an RGBA32F frame."""
        out = np.zeros((H, W, 4), np.uint8)
        self.lib.or_display(_p(np.ascontiguousarray(color, np.float32)), W, H, total, exposure, _p(out), threads)
        return out

    def atrous_pass(self, col, gb, ga, var, W, H, step, sc, sn, sd, N, exposure, threads=0):
        out = np.zeros((H, W, 4), np.float32)
        self.lib.or_atrous_pass(_p(col), _p(gb), _p(ga), _p(var), W, H, step, sc, sn, sd, N, exposure,
                                _p(out), threads)
        return out

    def denoise(self, acc, gb, ga, var, W, H, total, params: AtrousParams, threads=0):
        out = np.zeros((H, W, 4), np.float32)
        self.lib.or_denoise(_p(acc), _p(gb), _p(ga), _p(var), W, H, total, C.byref(params), _p(out), threads)
        return out


class Reference:
    """The reference's own shaders compiled for the host (oracle/_ref)."""

    def __init__(self, path: str = REF_LIB):
        self.lib = lib = C.CDLL(path)
        lib.ref_pathtrace.argtypes = [_VP, _VP, _VP, _VP, _I, _F, _VP, _VP, _I, _I, _I, _VP, _VP, _VP, _VP,
                                      _I, _I, _I]
        lib.ref_photon_trace.argtypes = [_VP, _VP, _VP, _VP, _I, _F, _I, _F, _I, _I, _VP, _VP, _VP, _VP, _I]
        lib.ref_photon_gather.argtypes = [_VP, _VP, _VP, _VP, _I, _I, _F, _I, _I, _I, _VP, _VP, _VP, _VP,
                                          _I, _I, _I]
        lib.ref_p00.argtypes = [_VP, _I, _I, _I, _F, _VP, _I]
        lib.ref_atrous_pass.argtypes = [_VP, _VP, _VP, _VP, _I, _I, _I, _F, _F, _F, _I, _F, _VP, _I, _I, _I]
        lib.ref_display.argtypes = [_VP, _I, _I, _I, _F, _VP, _I]
        lib.ref_post_pass.argtypes = [_I, _VP, _I, _I, _VP, _VP, _I]

    def pathtrace(self, scene, cam, settings, W, H, frame, buffers, threads=0, rows=(0, 0)):
        acc, gb, ga, var = buffers
        self.lib.ref_pathtrace(_p(scene["tris"]), _p(scene["nodes"]), _p(scene["mats"]), _p(scene["lights"]),
                               scene["light_count"], scene["total_power"], C.byref(camera_struct(cam)),
                               C.byref(Settings(*settings)), W, H, frame, _p(acc), _p(gb), _p(ga), _p(var),
                               rows[0], rows[1], threads)

    def render(self, scene, cam, settings, W, H, first, nspp, buffers=None, threads=0):
        bufs = buffers if buffers is not None else alloc_images(W, H)
        for f in range(first, first + nspp):
            self.pathtrace(scene, cam, settings, W, H, f, bufs, threads)
        return bufs

    def photon_trace(self, scene, N, radius, seed, hash_size, threads=1):
        ph = np.zeros(max(N, 1), PHOTON)
        heads = np.full(hash_size, -1, np.int32)
        nxt = np.zeros(max(N, 1), np.int32)
        cnt = np.zeros(1, np.uint32)
        self.lib.ref_photon_trace(_p(scene["tris"]), _p(scene["nodes"]), _p(scene["mats"]), _p(scene["lights"]),
                                  scene["light_count"], scene["total_power"], N, radius, seed, hash_size,
                                  _p(ph), _p(heads), _p(nxt), _p(cnt), threads)
        return ph, heads, nxt, int(cnt[0])

    def photon_gather(self, scene, cam, W, H, radius, N, hash_size, frame, ph, heads, nxt, accum, threads=0,
                      rows=(0, 0)):
        self.lib.ref_photon_gather(_p(scene["tris"]), _p(scene["nodes"]), _p(scene["mats"]),
                                   C.byref(camera_struct(cam)), W, H, radius, N, hash_size, frame, _p(ph),
                                   _p(heads), _p(nxt), _p(accum), rows[0], rows[1], threads)

    def post_pass(self, pass_, color, W, H, params, threads=0):
        """One VHS pass of the reference's own shader (params: the product's
        rc_vhs_params ctypes struct, the same layout)."""
        out = np.zeros((H, W, 4), np.float32)
        r = self.lib.ref_post_pass(pass_, _p(np.ascontiguousarray(color, np.float32)), W, H, C.byref(params),
                                   _p(out), threads)
        assert r == 0, pass_
        return out

    def display(self, color, W, H, total=1, exposure=1.0, threads=0):
        out = np.zeros((H, W, 4), np.uint8)
        self.lib.ref_display(_p(np.ascontiguousarray(color, np.float32)), W, H, total, exposure, _p(out), threads)
        return out

    def atrous_pass(self, col, gb, ga, var, W, H, step, sc, sn, sd, N, exposure, out, rows=(0, 0), threads=0):
        self.lib.ref_atrous_pass(_p(col), _p(gb), _p(ga), _p(var), W, H, step, sc, sn, sd, N, exposure, _p(out),
                                 rows[0], rows[1], threads)

    def denoise(self, acc, gb, ga, var, W, H, total, params: AtrousParams, threads=0):
        a = np.zeros((H, W, 4), np.float32)
        self.lib.ref_p00(_p(acc), W, H, total, params.exposure, _p(a), threads)
        if params.enabled and not (params.max_spp > 0 and total > params.max_spp):
            passes = max(1, min(params.iterations, 5))
            for i in range(passes):
                b = np.zeros_like(a)
                self.lib.ref_atrous_pass(_p(a), _p(gb), _p(ga), _p(var), W, H, 1 << i, params.sigma_color,
                                         params.sigma_normal, params.sigma_depth, max(total, 1),
                                         params.exposure, _p(b), 0, 0, threads)
                a = b
        return a


def alloc_images(W, H):
    return (np.zeros((H, W, 4), np.float32), np.zeros((H, W, 4), np.uint16),
            np.zeros((H, W, 4), np.uint16), np.zeros((H, W), np.float32))


def load(build: bool = True):
    """Returns (Oracle, Reference or None)."""
    if build:
        import sys
        sys.path.insert(0, HERE)
        try:
            import build as _b  # noqa
            _b.build_all()
        finally:
            sys.path.pop(0)
    ref = Reference() if os.path.exists(REF_LIB) else None
    return Oracle(), ref


def load_reference_libm():
    """The timing variant of the compiled reference, or None."""
    return Reference(REF_LIB_LIBM) if os.path.exists(REF_LIB_LIBM) else None
