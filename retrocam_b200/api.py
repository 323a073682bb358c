"""ctypes bindings of the C ABI (include/retrocam.h) and a Python mirror of
the reference's render-path classes.

The mirror keeps the reference's names and call order so code written
against the Java classes maps one to one:

  SceneUploader.upload(scene)          scene/SceneUploader.java:54
  Renderer.render(...) / reset()       core/Renderer.java:72,120
  SPPMManager.trace_photons / gather_radiance / update_radius / reset
                                       scene/SPPMManager.java:76,118,170,182
  AtrousDenoiser.denoise(...)          post/AtrousDenoiser.java:60

Every call goes through libretrocam.so; there is no CPU fallback.  Loading
fails loudly when the library has not been built.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import scenes

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "_lib", "libretrocam.so")

RC_OK = 0
RC_ERR_INVALID_ARG = -1
RC_ERR_CUDA = -2
RC_ERR_OUT_OF_MEMORY = -3
RC_ERR_NO_SCENE = -4
RC_ERR_DEVICE_GUARD = -5
RC_ERR_CAPACITY = -6
RC_ERR_BAD_SCENE = -7
RC_MATH_FAST = 0
RC_MATH_EXACT = 1
RC_GUARD_TRAVERSAL_CAP = 0x1

# ---- record dtypes: the std430 layouts of include/retrocam.h ----
_F3 = ("<f4", 3)
TRIANGLE = np.dtype([("v0",) + _F3, ("pad0", "<f4"), ("v1",) + _F3, ("pad1", "<f4"), ("v2",) + _F3,
                     ("pad2", "<f4"), ("n0",) + _F3, ("pad3", "<f4"), ("n1",) + _F3, ("pad4", "<f4"),
                     ("n2",) + _F3, ("pad5", "<f4"), ("uv0", "<f4", 2), ("uv1", "<f4", 2), ("uv2", "<f4", 2),
                     ("mat_index", "<i4"), ("pad6", "<f4")])
BVH_NODE = np.dtype([("aabb_min",) + _F3, ("pad0", "<f4"), ("aabb_max",) + _F3, ("pad1", "<f4"),
                     ("left_child", "<i4"), ("right_child", "<i4"), ("prim_start", "<i4"), ("prim_count", "<i4")])
MATERIAL = np.dtype([("albedo",) + _F3, ("metallic", "<f4"), ("emission",) + _F3, ("emission_strength", "<f4"),
                     ("roughness", "<f4"), ("ior", "<f4"), ("transmission", "<f4"), ("albedo_tex", "<i4"),
                     ("pad", "<f4", 4)])
LIGHT = np.dtype([("v0",) + _F3, ("area", "<f4"), ("v1",) + _F3, ("pad1", "<f4"), ("v2",) + _F3, ("pad2", "<f4"),
                  ("emission",) + _F3, ("power", "<f4"), ("normal",) + _F3, ("cdf_weight", "<f4")])
PHOTON = np.dtype([("position",) + _F3, ("pad0", "<f4"), ("power",) + _F3, ("pad1", "<f4"), ("dir",) + _F3,
                   ("pad2", "<f4")])


class rc_camera(C.Structure):
    _fields_ = [("cam_pos", C.c_float * 3), ("cam_right", C.c_float * 3), ("cam_up", C.c_float * 3),
                ("cam_forward", C.c_float * 3), ("focal_dist", C.c_float), ("lens_radius", C.c_float),
                ("fov_tan_half", C.c_float), ("aperture_blades", C.c_int32), ("sa_strength", C.c_float),
                ("lca_delta", C.c_float * 3)]


class rc_settings(C.Structure):
    _fields_ = [("nee_enabled", C.c_int32), ("nee_firefly_clamp", C.c_float)]


class rc_frame_desc(C.Structure):
    _fields_ = [("camera", rc_camera), ("spp", C.c_int32), ("sppm_iterations", C.c_int32)]


class rc_sppm_params(C.Structure):
    _fields_ = [("photon_count", C.c_int32), ("hash_size", C.c_int32), ("alpha", C.c_float)]


class rc_atrous_params(C.Structure):
    _fields_ = [("enabled", C.c_int32), ("iterations", C.c_int32), ("sigma_color", C.c_float),
                ("sigma_normal", C.c_float), ("sigma_depth", C.c_float), ("max_spp", C.c_int32),
                ("exposure", C.c_float)]


_VHS_FIELDS = [("enabled", "i"), ("frame_index", "i"), ("time_s", "f"), ("agc_gain", "f"),
               ("luma_blur_sigma", "f"), ("chroma_res_sigma", "f"),
               ("color_temp_bias", "f"), ("color_hue_rot", "f"), ("color_saturation", "f"),
               ("color_drift_speed", "f"), ("dr_black_lift", "f"), ("dr_shadow_crush", "f"),
               ("dr_highlight_knee", "f"), ("dr_highlight_clip", "f"), ("ccd_noise_luma_base", "f"),
               ("ccd_noise_chroma_scale", "f"), ("ccd_smear_threshold", "f"), ("ccd_smear_intensity", "f"),
               ("ccd_smear_length", "i"), ("chroma_bleed_factor", "f"), ("timebase_amplitude_px", "f"),
               ("timebase_freq", "f"), ("timebase_speed", "f"), ("dot_crawl_intensity", "f"),
               ("dot_crawl_subcarrier", "f"), ("dot_crawl_edge_thresh", "f"), ("tape_age", "f"),
               ("dropout_bright", "f"), ("dropout_burst_rate", "f"), ("head_switch_lines", "i"),
               ("head_switch_jitter", "f"), ("head_switch_ripple", "f"), ("head_switch_chroma", "f"),
               ("tracking_severity", "f"), ("tracking_max_displace_px", "f"), ("tracking_fringe_width_px", "f"),
               ("edge_enhance_amount", "f"), ("edge_enhance_core_threshold", "f"),
               ("interlace_field_offset_px", "f"), ("interlace_comb_strength", "f"),
               ("interlace_comb_edge_thresh", "f"), ("interlace_line_weighting", "f")]


class rc_vhs_params(C.Structure):
    """The VHS chain's knobs (include/retrocam.h rc_vhs_params)."""
    _fields_ = [(n, C.c_int32 if t == "i" else C.c_float) for n, t in _VHS_FIELDS]


VHS_PASSES = (1, 2, 3, 4, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16)


def vhs_defaults(**overrides) -> rc_vhs_params:
    """RenderSettings' defaults (every pass off), with overrides by field name;
    `passes=(1, 3, ...)` sets the enabled mask."""
    p = rc_vhs_params()
    lib().rc_vhs_defaults(C.byref(p))
    for k, v in overrides.items():
        if k == "passes":
            p.enabled = sum(1 << (i - 1) for i in v)
        else:
            setattr(p, k, v)
    return p


class rc_tuning(C.Structure):
    _fields_ = [("engine", C.c_int32), ("chunk_paths", C.c_int32), ("wide_bvh", C.c_int32),
                ("trace_block", C.c_int32), ("shade_block", C.c_int32), ("photon_block", C.c_int32),
                ("photon_full_first", C.c_int32), ("refill_lanes", C.c_int32), ("leaf_quarters", C.c_int32),
                ("refill_min_paths", C.c_int32), ("material_queues", C.c_int32),
                ("interior_steps", C.c_int32)]

    def as_dict(self) -> dict:
        return {k: int(getattr(self, k)) for k, _ in self._fields_}


class rc_counters(C.Structure):
    _fields_ = [("camera_paths", C.c_uint64), ("closest_rays", C.c_uint64), ("shadow_rays", C.c_uint64),
                ("photon_rays", C.c_uint64), ("gather_rays", C.c_uint64), ("photons_stored", C.c_uint64),
                ("node_tests", C.c_uint64), ("tri_tests", C.c_uint64), ("surface_hits", C.c_uint64),
                ("light_samples", C.c_uint64), ("photon_node_tests", C.c_uint64),
                ("photon_tri_tests", C.c_uint64), ("kernel_launches", C.c_uint64), ("h2d_bytes", C.c_uint64), ("d2h_bytes", C.c_uint64),
                ("error_word", C.c_uint32), ("bvh_depth", C.c_uint32)]


KERNEL_KINDS = ("render", "photon_trace", "photon_gather", "atrous", "normalize", "wf_generate", "wf_trace",
                "wf_shade", "wf_accumulate", "photon_layout", "kpcnn", "display", "vhs", "wf_sort")
RC_ENGINE_MEGAKERNEL = 0
RC_ENGINE_WAVEFRONT = 1
RC_ENGINE_WAVEFRONT_STATIC = 2
RC_WIDE_PATHS = 0x1
RC_WIDE_PHOTONS = 0x2


_VP, _I, _F = C.c_void_p, C.c_int, C.c_float
_SIGNATURES = {
    "rc_abi_version": (_I, []),
    "rc_ctx_create": (_I, [_I, _I, _I, C.POINTER(_VP)]),
    "rc_ctx_destroy": (_I, [_VP]),
    "rc_last_error": (_I, [_VP, C.c_char_p, C.c_size_t]),
    "rc_set_math_mode": (_I, [_VP, _I]),
    "rc_synchronize": (_I, [_VP]),
    "rc_ctx_set_stream": (_I, [_VP, _VP]),
    "rc_set_kernel_timing": (_I, [_VP, _I]),
    "rc_get_kernel_times": (_I, [_VP, _VP, _VP]),
    "rc_set_engine": (_I, [_VP, _I, _I]),
    "rc_set_tuning": (_I, [_VP, _VP]),
    "rc_get_tuning": (_I, [_VP, _VP]),
    "rc_render_frames": (_I, [_VP, _VP, _I, _VP, _VP, _F, _VP, _VP, _I]),
    "rc_tessellate_box": (_I, [_F] * 6 + [_I] + [_F] * 3 + [_VP]),
    "rc_tessellate_sphere": (_I, [_F] * 4 + [_I, _I, _I] + [_F] * 3 + [_VP, _I, C.POINTER(_I)]),
    "rc_triangles_from_positions": (_I, [_VP, _I, _I, _VP]),
    "rc_build_bvh": (_I, [_VP, _I, _VP, _VP, _I, C.POINTER(_I)]),
    "rc_build_lights": (_I, [_VP, _I, _VP, _I, _VP, _I, C.POINTER(_I), C.POINTER(_F)]),
    "rc_thin_lens": (_I, [_F, _F, C.POINTER(_F), C.POINTER(_F)]),
    "rc_orbit_basis": (_I, [_F] * 6 + [_VP]),
    "rc_sppm_next_radius": (_F, [_F, _I, _F]),
    "rc_keyframe_evaluate": (_F, [_VP, _VP, _VP, _I, _F, _F]),
    "rc_scene_upload": (_I, [_VP, _VP, _I, _VP, _I, _VP, _I, _VP, _I, _F]),
    "rc_render": (_I, [_VP, _VP, _VP, _I, _I]),
    "rc_reset": (_I, [_VP]),
    "rc_total_samples": (_I, [_VP]),
    "rc_sppm_reset": (_I, [_VP, _F]),
    "rc_sppm_trace": (_I, [_VP, _VP]),
    "rc_sppm_gather": (_I, [_VP, _VP, _VP, _F]),
    "rc_sppm_update_radius": (_I, [_VP, _F]),
    "rc_sppm_state": (_I, [_VP, C.POINTER(_F), C.POINTER(_I)]),
    "rc_denoise_atrous": (_I, [_VP, _VP, _VP]),
    "rc_render_frame": (_I, [_VP, _VP, _VP, _I, _VP, _F, _I, _VP, _VP]),
    "rc_frame_part_range": (_I, [_I, _I, _I, _I] + [C.POINTER(_I)] * 4),
    "rc_render_frame_part": (_I, [_VP, _VP, _VP, _I, _VP, _F, _I, _I, _I]),
    "rc_set_total_samples": (_I, [_VP, _I]),
    "rc_get_images": (_I, [_VP] + [C.POINTER(_VP)] * 5),
    "rc_read_buffers": (_I, [_VP, _VP, _VP, _VP, _VP]),
    "rc_read_output": (_I, [_VP, _VP]),
    "rc_display": (_I, [_VP, _I, _F, _VP]),
    "rc_display_frame": (_I, [_VP, _I, _I, _F, _VP]),
    "rc_vhs_defaults": (None, [_VP]),
    "rc_post_vhs": (_I, [_VP, _VP]),
    "rc_vhs_pass": (_I, [_I, _VP, _VP, _I, _I, _VP, _VP]),
    "rc_read_photon_map": (_I, [_VP, _VP, _I, _VP, _I, _VP, _VP]),
    "rc_get_counters": (_I, [_VP, _VP]),
    "rc_reset_counters": (_I, [_VP]),
    "rc_measure_fp32_peak": (_I, [_I, C.POINTER(C.c_double)]),
    "rc_denoise_learned": (_I, [_VP, _VP, _VP]),
    "rc_kp_features": (_I, [_VP, _VP, _VP]),
    "rc_kp_conv3x3": (_I, [_VP, _I, _VP, _VP, _VP, _I, _I, _VP, _I, _I, _I, _VP, _VP]),
    "rc_kp_wgrad": (_I, [_VP, _I, _VP, _VP, _VP, _I, _I, _I, _VP, _VP]),
    "rc_kp_head": (_I, [_VP, _VP, _VP, _VP, _VP, _VP, _F, _I, _I, _I, _VP]),
    "rc_kp_pack": (_I, [_VP, _VP, _VP]),
    "rc_kp_adam": (_I, [_VP, _VP, _VP, _VP, _I, _F, _F, _F, _F, _I, _VP]),
    "rc_kp_crop": (_I, [_VP, _VP, _VP, _VP, _VP, _VP, _VP, _I, _I, _I, _I, _VP, _VP, _VP, _VP]),
}

RC_KPCNN_PARAMS = 32384
RC_GUARD_MMA_WAIT = 0x8


class rc_kpcnn(C.Structure):
    _fields_ = [("params", C.c_void_p), ("param_count", C.c_int32)]

_lib = None


def lib():
    """The loaded libretrocam.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with retrocam_b200.build.build()")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


class RetroCamError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _check(code, ctx=None):
    if code != RC_OK:
        buf = C.create_string_buffer(1024)
        lib().rc_last_error(ctx, buf, len(buf))
        raise RetroCamError(code, buf.value.decode(errors="replace"))


# ---------------------------------------------------------------------------
# host scene logic (scene builder backend for scenes.build_scene)
# ---------------------------------------------------------------------------
class HostScene:
    """Bit-exact restatements of the reference's Java scene code, in C++."""

    def tess_box(self, c, h, mat, rot=(0.0, 0.0, 0.0)):
        out = np.zeros(12, TRIANGLE)
        _check(lib().rc_tessellate_box(*map(float, c), *map(float, h), int(mat), *map(float, rot), _p(out)))
        return out

    def tess_sphere(self, c, r, mat, stacks, slices, rot=(0.0, 0.0, 0.0)):
        out = np.zeros(2 * stacks * slices, TRIANGLE)
        n = C.c_int(0)
        _check(lib().rc_tessellate_sphere(*map(float, c), float(r), int(mat), int(stacks), int(slices),
                                          *map(float, rot), _p(out), len(out), C.byref(n)))
        return out[:n.value]

    def flat_triangles(self, positions, mat):
        pos = np.ascontiguousarray(positions, dtype=np.float32).reshape(-1, 9)
        out = np.zeros(len(pos), TRIANGLE)
        _check(lib().rc_triangles_from_positions(_p(pos), len(pos), int(mat), _p(out)))
        return out

    def build_bvh(self, tris):
        tris = np.ascontiguousarray(tris, dtype=TRIANGLE)
        out_t = np.zeros_like(tris)
        cap = 2 * len(tris) + 1
        nodes = np.zeros(cap, BVH_NODE)
        n = C.c_int(0)
        _check(lib().rc_build_bvh(_p(tris), len(tris), _p(out_t), _p(nodes), cap, C.byref(n)))
        return out_t, nodes[:n.value]

    def build_lights(self, tris, mats):
        tris = np.ascontiguousarray(tris, dtype=TRIANGLE)
        mats = np.ascontiguousarray(mats, dtype=MATERIAL)
        out = np.zeros(max(1, len(tris)), LIGHT)
        n, tp = C.c_int(0), C.c_float(0)
        _check(lib().rc_build_lights(_p(tris), len(tris), _p(mats), len(mats), _p(out), len(out), C.byref(n),
                                     C.byref(tp)))
        return out[:n.value], tp.value

    def thin_lens(self, focal_mm, fstop):
        a, b = C.c_float(0), C.c_float(0)
        _check(lib().rc_thin_lens(focal_mm, fstop, C.byref(a), C.byref(b)))
        return a.value, b.value

    def orbit_basis(self, theta, phi, radius, target):
        out = np.zeros(12, np.float32)
        _check(lib().rc_orbit_basis(theta, phi, radius, *map(float, target), _p(out)))
        return out

    def keyframe(self, times, values, interp, t, default=0.0):
        """KeyframeTrack.evaluate: interp 0 STEP, 1 LINEAR, 2 BEZIER."""
        tt = np.ascontiguousarray(times, np.float32)
        vv = np.ascontiguousarray(values, np.float32)
        ii = np.ascontiguousarray(interp, np.int32)
        return float(lib().rc_keyframe_evaluate(_p(tt), _p(vv), _p(ii), len(tt), float(t), float(default)))


HOST = HostScene()


def build_scene(desc: scenes.SceneDesc) -> dict:
    return scenes.build_scene(desc, HOST, MATERIAL)


def camera_struct(cam: dict) -> rc_camera:
    c = rc_camera()
    for k in ("cam_pos", "cam_right", "cam_up", "cam_forward", "lca_delta"):
        getattr(c, k)[:] = [float(x) for x in cam[k]]
    c.focal_dist = cam["focal_dist"]
    c.lens_radius = cam["lens_radius"]
    c.fov_tan_half = cam["fov_tan_half"]
    c.aperture_blades = int(cam["aperture_blades"])
    c.sa_strength = cam["sa_strength"]
    return c


# ---------------------------------------------------------------------------
# context
# ---------------------------------------------------------------------------
class Context:
    """One rc_ctx: a device, a stream, the renderer images, a scene."""

    def __init__(self, width: int, height: int, device: int = 0, math_mode: int = RC_MATH_FAST):
        L = lib()
        h = C.c_void_p()
        _check(L.rc_ctx_create(width, height, device, C.byref(h)))
        self.h = h
        self.width, self.height = width, height
        self.set_math_mode(math_mode)

    def close(self):
        if self.h:
            lib().rc_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def check(self, code):
        _check(code, self.h)

    def set_math_mode(self, mode):
        self.check(lib().rc_set_math_mode(self.h, mode))

    def upload(self, sc: dict):
        lights = sc["lights"] if sc["light_count"] > 0 else None
        self.check(lib().rc_scene_upload(self.h, _p(sc["tris"]), len(sc["tris"]), _p(sc["nodes"]),
                                         len(sc["nodes"]), _p(sc["mats"]), len(sc["mats"]), _p(lights),
                                         sc["light_count"], sc["total_power"]))

    def render(self, cam: dict, settings=(1, 1.0), first_frame=0, n_spp=1):
        self.check(lib().rc_render(self.h, C.byref(camera_struct(cam)), C.byref(rc_settings(*settings)),
                                   first_frame, n_spp))

    def reset(self):
        self.check(lib().rc_reset(self.h))

    @property
    def total_samples(self):
        return lib().rc_total_samples(self.h)

    def sppm_reset(self, r0):
        self.check(lib().rc_sppm_reset(self.h, r0))

    def sppm_trace(self, photons, hash_size, alpha=0.7):
        self.check(lib().rc_sppm_trace(self.h, C.byref(rc_sppm_params(photons, hash_size, alpha))))

    def sppm_gather(self, cam, photons, hash_size, weight=1.0, alpha=0.7):
        self.check(lib().rc_sppm_gather(self.h, C.byref(camera_struct(cam)),
                                        C.byref(rc_sppm_params(photons, hash_size, alpha)), weight))

    def sppm_update_radius(self, alpha):
        self.check(lib().rc_sppm_update_radius(self.h, alpha))

    def sppm_state(self):
        r, i = C.c_float(0), C.c_int(0)
        self.check(lib().rc_sppm_state(self.h, C.byref(r), C.byref(i)))
        return r.value, i.value

    def denoise(self, params: rc_atrous_params, read=True):
        out = np.zeros((self.height, self.width, 4), np.float32) if read else None
        self.check(lib().rc_denoise_atrous(self.h, C.byref(params), _p(out)))
        return out

    def render_frames(self, frames, settings, sppm: rc_sppm_params | None, r0, atrous: rc_atrous_params,
                      use_graph=True, read=True):
        """rc_render_frames over [(camera dict, spp, sppm_iterations), ...];
        returns the (n, H, W, 4) finished frames when `read`."""
        n = len(frames)
        arr = (rc_frame_desc * n)()
        for i, (cam, spp, iters) in enumerate(frames):
            arr[i] = rc_frame_desc(camera_struct(cam), int(spp), int(iters))
        out = np.zeros((n, self.height, self.width, 4), np.float32) if read else None
        self.check(lib().rc_render_frames(self.h, arr, n, C.byref(rc_settings(*settings)),
                                          C.byref(sppm) if sppm is not None else None, r0, C.byref(atrous),
                                          _p(out), 1 if use_graph else 0))
        return out

    def denoise_learned(self, params: np.ndarray, read=True):
        """rc_denoise_learned with a float32 parameter vector (RC_KPCNN_PARAMS)."""
        params = np.ascontiguousarray(params, np.float32)
        out = np.zeros((self.height, self.width, 4), np.float32) if read else None
        w = rc_kpcnn(params.ctypes.data, params.size)
        self.check(lib().rc_denoise_learned(self.h, C.byref(w), _p(out)))
        return out

    def kp_features(self, feat_ptr: int, color_ptr: int):
        """Network input of the current images into device buffers."""
        self.check(lib().rc_kp_features(self.h, C.c_void_p(feat_ptr), C.c_void_p(color_ptr)))

    def render_frame(self, cam, settings, spp, sppm: rc_sppm_params | None, r0, sppm_iters,
                     atrous: rc_atrous_params, read=True):
        out = np.zeros((self.height, self.width, 4), np.float32) if read else None
        self.check(lib().rc_render_frame(self.h, C.byref(camera_struct(cam)), C.byref(rc_settings(*settings)),
                                         spp, C.byref(sppm) if sppm is not None else None, r0, sppm_iters,
                                         C.byref(atrous), _p(out)))
        return out

    def render_frame_part(self, cam, settings, spp, sppm: rc_sppm_params | None, r0, sppm_iters, part, parts):
        """rc_render_frame_part: this context's share of a frame split
        `parts` ways (no denoise; images hold the part's sums)."""
        self.check(lib().rc_render_frame_part(self.h, C.byref(camera_struct(cam)), C.byref(rc_settings(*settings)),
                                              spp, C.byref(sppm) if sppm is not None else None, r0, sppm_iters,
                                              part, parts))

    def set_total_samples(self, n: int):
        self.check(lib().rc_set_total_samples(self.h, int(n)))

    def image_pointers(self) -> dict:
        """Device addresses of the images and the context's stream handle."""
        p = [C.c_void_p() for _ in range(5)]
        self.check(lib().rc_get_images(self.h, *[C.byref(x) for x in p]))
        return dict(zip(("accum", "gbuffer", "albedo", "variance", "stream"), (x.value or 0 for x in p)))

    def read_buffers(self):
        H, W = self.height, self.width
        acc = np.zeros((H, W, 4), np.float32)
        gb = np.zeros((H, W, 4), np.uint16)
        ga = np.zeros((H, W, 4), np.uint16)
        var = np.zeros((H, W), np.float32)
        self.check(lib().rc_read_buffers(self.h, _p(acc), _p(gb), _p(ga), _p(var)))
        return acc, gb, ga, var

    def read_output(self):
        out = np.zeros((self.height, self.width, 4), np.float32)
        self.check(lib().rc_read_output(self.h, _p(out)))
        return out

    def display(self, total_samples=1, exposure=1.0, read=True):
        """RenderPipeline.applyDisplayPass + FrameExporter's read-back: the
        last output ACES-tonemapped, sRGB-encoded and stored as RGBA8, rows
        top first (an (H, W, 4) uint8 array; None with read=False)."""
        if not read:
            self.check(lib().rc_display(self.h, total_samples, exposure, None))
            return None
        out = np.zeros((self.height, self.width, 4), np.uint8)
        self.check(lib().rc_display(self.h, total_samples, exposure, _p(out)))
        return out

    def post_vhs(self, params: rc_vhs_params, read=False):
        """rc_post_vhs: the enabled VHS passes on the last output (which they
        replace); returns it when `read`."""
        self.check(lib().rc_post_vhs(self.h, C.byref(params)))
        return self.read_output() if read else None

    def display_frame(self, frame, total_samples=1, exposure=1.0):
        """display() on frame `frame` of the last render_frames batch."""
        out = np.zeros((self.height, self.width, 4), np.uint8)
        self.check(lib().rc_display_frame(self.h, frame, total_samples, exposure, _p(out)))
        return out

    def read_photon_map(self, capacity, hash_size):
        ph = np.zeros(capacity, PHOTON)
        heads = np.zeros(hash_size, np.int32)
        nxt = np.zeros(capacity, np.int32)
        cnt = np.zeros(1, np.uint32)
        self.check(lib().rc_read_photon_map(self.h, _p(ph), capacity, _p(heads), hash_size, _p(nxt), _p(cnt)))
        return ph, heads, nxt, int(cnt[0])

    def counters(self):
        c = rc_counters()
        self.check(lib().rc_get_counters(self.h, C.byref(c)))
        return {k: getattr(c, k) for k, _ in rc_counters._fields_}

    def reset_counters(self):
        self.check(lib().rc_reset_counters(self.h))

    def synchronize(self):
        self.check(lib().rc_synchronize(self.h))

    def set_stream(self, cuda_stream_handle: int | None):
        """Run on a caller-owned cudaStream_t (e.g. torch.cuda.Stream().cuda_stream)."""
        self.check(lib().rc_ctx_set_stream(self.h, C.c_void_p(cuda_stream_handle or 0)))

    def set_engine(self, engine: int, chunk_paths: int = 0):
        self.check(lib().rc_set_engine(self.h, engine, chunk_paths))

    def set_tuning(self, **knobs):
        """Sets launch-shape knobs (rc_tuning field names); unnamed ones keep
        their current values."""
        t = self.tuning()
        for k, v in knobs.items():
            if k not in t:
                raise KeyError(k)
            t[k] = int(v)
        self.check(lib().rc_set_tuning(self.h, C.byref(rc_tuning(**t))))

    def tuning(self) -> dict:
        t = rc_tuning()
        self.check(lib().rc_get_tuning(self.h, C.byref(t)))
        return t.as_dict()

    def set_kernel_timing(self, on: bool):
        self.check(lib().rc_set_kernel_timing(self.h, 1 if on else 0))

    def kernel_times(self):
        """{kind: (milliseconds, launches)} since the previous call."""
        ms = np.zeros(len(KERNEL_KINDS), np.float64)
        n = np.zeros(len(KERNEL_KINDS), np.uint64)
        self.check(lib().rc_get_kernel_times(self.h, _p(ms), _p(n)))
        return {k: (float(ms[i]), int(n[i])) for i, k in enumerate(KERNEL_KINDS)}


# ---------------------------------------------------------------------------
# mirror of the reference's Java classes on the render path
# ---------------------------------------------------------------------------
class SceneUploader:
    """scene/SceneUploader.java: builds the BVH and lights, uploads."""

    def __init__(self, ctx: Context):
        self.ctx = ctx
        self.triangle_count = self.node_count = self.light_count = 0
        self.total_light_power = 0.0

    def upload(self, desc: scenes.SceneDesc):
        sc = build_scene(desc)
        self.ctx.upload(sc)
        self.triangle_count, self.node_count = len(sc["tris"]), len(sc["nodes"])
        self.light_count, self.total_light_power = sc["light_count"], sc["total_power"]
        return sc


class Renderer:
    """core/Renderer.java: one render() = one sample per pixel."""

    def __init__(self, ctx: Context):
        self.ctx = ctx

    def render(self, cam: dict, settings=(1, 1.0)):
        self.ctx.render(cam, settings, first_frame=self.ctx.total_samples, n_spp=1)

    def reset(self):
        self.ctx.reset()

    def get_total_samples(self):
        return self.ctx.total_samples


class SPPMManager:
    """scene/SPPMManager.java over the context's photon map."""

    def __init__(self, ctx: Context, photons=500_000, hash_size=1 << 22, init_radius=0.05):
        self.ctx, self.photons, self.hash_size = ctx, photons, hash_size
        ctx.sppm_reset(init_radius)

    def trace_photons(self):
        self.ctx.sppm_trace(self.photons, self.hash_size)

    def gather_radiance(self, cam: dict, weight=1.0):
        self.ctx.sppm_gather(cam, self.photons, self.hash_size, weight)

    def update_radius(self, alpha):
        self.ctx.sppm_update_radius(alpha)

    def reset(self, init_radius):
        self.ctx.sppm_reset(init_radius)

    def get_search_radius(self):
        return self.ctx.sppm_state()[0]

    def get_iteration(self):
        return self.ctx.sppm_state()[1]


class AtrousDenoiser:
    """post/AtrousDenoiser.java with the PostProcessStack gate and p00."""

    def __init__(self, ctx: Context):
        self.ctx = ctx

    def denoise(self, params: rc_atrous_params, read=True):
        return self.ctx.denoise(params, read)


def frame_part_range(spp: int, sppm_iterations: int, part: int, parts: int) -> tuple:
    """rc_frame_part_range: (k0, k1, s0, s1) of one part of a split frame."""
    v = [C.c_int() for _ in range(4)]
    _check(lib().rc_frame_part_range(spp, sppm_iterations, part, parts, *[C.byref(x) for x in v]))
    return tuple(x.value for x in v)


def atrous_params(a: scenes.AtrousDesc) -> rc_atrous_params:
    return rc_atrous_params(a.enabled, a.iterations, a.sigma_color, a.sigma_normal, a.sigma_depth, a.max_spp,
                            a.exposure)


def workload_camera(w: scenes.Workload) -> dict:
    return scenes.camera(w.orbit, w.lens, HOST)
