"""The keyframed export loop: export/RenderPipeline.java:63-185 with
keyframe/KeyframeTimeline.java and KeyframeTrack.java.

A RenderJob renders a photo (one frame at t = 0) or an image sequence
(frame f at t = f * (1 / fps), `round(duration * fps)` frames, written to
`<output>_frames/frame_%05d.png`).  Before each frame the timeline writes
every track's value at t into its target -- the orbit camera ("cam.theta",
"cam.phi", "cam.radius", "cam.targetX/Y/Z", "cam.fovY"), the render settings
("lens.focalLength", "lens.aperture", "lens.focusDist", "lens.saStrength",
"post.exposure", ...) or a scene object ("pos.x" ... "rot.z") -- with the
setters' clamps; tracks on scene objects re-upload the scene.  Each frame
is then the export path of `rc_render_frame` (SPPM iterations = samples per
frame, as accumulateFrame runs them), the display pass and a PNG file.

With `batched` (the default) and no scene-object or exposure tracks, the
frames of a job are rendered together by `rc_render_frames` (one CUDA graph
per batch of up to `batch_frames` frames) and each is displayed with
`rc_display_frame`; the images are those of the frame-by-frame loop (exact
math: the same bits without SPPM, and up to the photon-hash insertion order
with it).

With `vhs`, each frame runs the VHS chain (rc_post_vhs) between the
denoiser and the display pass, as PostProcessStack.runChain does.

Not built: MP4/MOV encoding through ffmpeg (RenderFormat.VIDEO_*), JPEG
files, the free camera, and TemporalState's autofocus hunting and AGC
dynamics (the lens focuses at exactly lens.focusDist; the AGC gain is the
value given) -- all outside the render path.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field, replace

import numpy as np

from . import api, export, scenes
from .scene_json import SceneFile

f32 = np.float32


# ---------------------------------------------------------------------------
# timeline (keyframe/KeyframeTimeline.java, KeyframeTrack.java)
# ---------------------------------------------------------------------------
@dataclass
class Track:
    """One (target, property) track: keyframe times in seconds (sorted),
    values and per-key interpolation (0 step, 1 linear, 2 Bezier).
    target: "camera", "settings" or ("object", index)."""
    target: object
    prop: str
    times: tuple = ()
    values: tuple = ()
    interp: tuple = ()

    def evaluate(self, time: float, current: float) -> float:
        """KeyframeTrack.evaluate (the library's rc_keyframe_evaluate);
        a track without keys keeps the current value."""
        if not self.times:
            return current
        interp = self.interp or (2,) * len(self.times)
        return api.HOST.keyframe(self.times, self.values, interp, time, current)


@dataclass
class Orbit:
    """camera/OrbitCamera.java's keyframeable state (radians, metres)."""
    theta: float = -math.pi / 2
    phi: float = math.pi / 2
    radius: float = 1.9
    target: tuple = (0.5, 0.5, 0.5)
    fov_y: float = 45.0   # the raster preview's field of view; the lens sets the traced one


@dataclass
class Lens:
    """The keyframeable part of core/RenderSettings.java (lens and post)."""
    focal_length_mm: float = 35.0
    f_stop: float = 2.0
    focus_dist_m: float = 2.0
    sa_strength: float = 0.04
    exposure: float = 1.0
    saturation: float = 1.0       # VHS chain (not rendered here)
    color_temp: float = 0.0
    tape_age: float = 0.0
    blades: int = 5
    lca_scale: float = 0.0        # LCA offsets (-s * focus, 0, +s * focus); 0 = off


def _clamp(v, lo, hi):
    return max(f32(lo), min(f32(hi), f32(v)))


def _set_camera(o: Orbit, prop: str, v: float) -> Orbit:
    """OrbitCamera.setKeyframeableProperty (OrbitCamera.java:216-226)."""
    v = float(f32(v))
    if prop == "cam.theta":
        return replace(o, theta=v)
    if prop == "cam.phi":
        return replace(o, phi=float(max(f32(0.02), min(f32(f32(math.pi) - f32(0.02)), f32(v)))))
    if prop == "cam.radius":
        return replace(o, radius=float(max(f32(0.5), f32(v))))
    if prop in ("cam.targetX", "cam.targetY", "cam.targetZ"):
        t = list(o.target)
        t["XYZ".index(prop[-1])] = v
        return replace(o, target=tuple(t))
    if prop == "cam.fovY":
        return replace(o, fov_y=float(_clamp(v, 5.0, 150.0)))
    return o


def _get_camera(o: Orbit, prop: str) -> float:
    return {"cam.theta": o.theta, "cam.phi": o.phi, "cam.radius": o.radius, "cam.targetX": o.target[0],
            "cam.targetY": o.target[1], "cam.targetZ": o.target[2], "cam.fovY": o.fov_y}.get(prop, 0.0)


_LENS = {"lens.focalLength": ("focal_length_mm", 1.0, None), "lens.aperture": ("f_stop", 0.7, None),
         "lens.focusDist": ("focus_dist_m", 0.1, None), "lens.saStrength": ("sa_strength", None, None),
         "post.exposure": ("exposure", 0.0, None), "post.saturation": ("saturation", 0.0, None),
         "post.colorTemp": ("color_temp", None, None), "post.tapeAge": ("tape_age", 0.0, 1.0)}


def _set_settings(s: Lens, prop: str, v: float) -> Lens:
    """RenderSettings.setKeyframeableProperty (RenderSettings.java:237-248)."""
    if prop not in _LENS:
        return s
    name, lo, hi = _LENS[prop]
    v = f32(v)
    if lo is not None:
        v = max(f32(lo), v)
    if hi is not None:
        v = min(f32(hi), v)
    return replace(s, **{name: float(v)})


_OBJ = {"pos.x": "px", "pos.y": "py", "pos.z": "pz", "scl.x": "sx", "scl.y": "sy", "scl.z": "sz",
        "rot.x": "rx", "rot.y": "ry", "rot.z": "rz"}


@dataclass
class Timeline:
    duration_s: float = 5.0
    tracks: list = field(default_factory=list)

    def has_scene_object_tracks(self) -> bool:
        return any(isinstance(t.target, tuple) and t.target[0] == "object" for t in self.tracks)

    def has_track(self, prop: str) -> bool:
        return any(t.prop == prop and t.times for t in self.tracks)

    def apply(self, time: float, orbit: Orbit, lens: Lens, scene: SceneFile | None):
        """KeyframeTimeline.apply: every track in order writes its value at
        `time` (the current value where it has no keys).  Returns the new
        (orbit, lens, scene)."""
        for t in self.tracks:
            if t.target == "camera":
                orbit = _set_camera(orbit, t.prop, t.evaluate(time, _get_camera(orbit, t.prop)))
            elif t.target == "settings":
                cur = getattr(lens, _LENS[t.prop][0]) if t.prop in _LENS else 0.0
                lens = _set_settings(lens, t.prop, t.evaluate(time, cur))
            elif isinstance(t.target, tuple) and t.target[0] == "object" and scene is not None:
                idx = t.target[1]
                if 0 <= idx < len(scene.objects) and t.prop in _OBJ:
                    o = scene.objects[idx]
                    name = _OBJ[t.prop]
                    objs = list(scene.objects)
                    objs[idx] = replace(o, **{name: float(f32(t.evaluate(time, getattr(o, name))))})
                    scene = replace(scene, objects=objs)
        return orbit, lens, scene


# ---------------------------------------------------------------------------
# job (export/RenderJob.java) and the loop (RenderPipeline.tickPhoto /
# tickVideoFrame / accumulateFrame)
# ---------------------------------------------------------------------------
@dataclass
class RenderJob:
    """output_path without extension; a photo (PHOTO_PNG) or a PNG image
    sequence (IMAGE_SEQUENCE)."""
    output_path: str
    image_sequence: bool = False
    samples_per_frame: int = 64
    duration_s: float = 5.0
    fps: float = 29.97
    timeline: Timeline | None = None

    def total_frames(self) -> int:
        """getTotalFrames: max(1, Math.round(duration * fps)) in float."""
        if not self.image_sequence:
            return 1
        return max(1, int(math.floor(float(f32(self.duration_s) * f32(self.fps)) + 0.5)))

    def frame_dt(self) -> float:
        return float(f32(1.0) / f32(self.fps if self.fps > 0 else 29.97))

    def frame_time(self, frame: int) -> float:
        """tickVideoFrame's canonical time: currentFrame * getFrameDt()."""
        return float(f32(frame) * f32(self.frame_dt())) if self.image_sequence else 0.0

    def frame_path(self, frame: int) -> str:
        if not self.image_sequence:
            return self.output_path + ".png"
        return f"{self.output_path}_frames/frame_{frame:05d}.png"


def camera_of(orbit: Orbit, lens: Lens) -> dict:
    """The rc_camera of an orbit and lens state (ThinLensCamera.uploadTo)."""
    focus = lens.focus_dist_m
    s = lens.lca_scale
    ld = scenes.LensDesc(focal_length_mm=lens.focal_length_mm, f_stop=lens.f_stop, focus_dist_m=focus,
                         blades=lens.blades, sa_strength=lens.sa_strength, lca_delta=(-s * focus, 0.0, s * focus))
    return scenes.camera(scenes.OrbitDesc(orbit.theta, orbit.phi, orbit.radius, tuple(orbit.target)), ld, api.HOST)


def plan(job: RenderJob, orbit: Orbit, lens: Lens, scene: SceneFile):
    """Per frame: (time, orbit, lens, scene) after the timeline's apply."""
    out = []
    for f in range(job.total_frames()):
        t = job.frame_time(f)
        if job.timeline is not None:
            orbit, lens, scene = job.timeline.apply(t, orbit, lens, scene)
        out.append((t, orbit, lens, scene))
    return out


def vhs_for_frame(vhs, frame: int, time_s: float, lens: Lens):
    """The chain's per-frame knobs: frame index (the caller's start plus the
    frame), TemporalState.time (the canonical frame time) and the keyframed
    post settings (saturation, colour temperature, tape age)."""
    import ctypes as C
    p = api.rc_vhs_params()
    C.memmove(C.byref(p), C.byref(vhs), C.sizeof(p))
    p.frame_index = vhs.frame_index + frame
    p.time_s = time_s
    p.color_saturation = lens.saturation
    p.color_temp_bias = lens.color_temp
    p.tape_age = lens.tape_age
    return p


def run_job(ctx, job: RenderJob, scene: SceneFile, orbit: Orbit | None = None, lens: Lens | None = None,
            settings=(1, 1.0), sppm: scenes.SppmDesc | None = scenes.SppmDesc(), r0: float = 0.02,
            atrous: scenes.AtrousDesc = scenes.AtrousDesc(), batched: bool = True, batch_frames: int = 32,
            vhs=None):
    """Renders the job through the context and writes its PNG files;
    returns their paths.  SPPM (when given and the scene has lights) runs one
    photon pass per sample, as accumulateFrame does.  `vhs` (an
    api.rc_vhs_params with passes enabled) runs the VHS chain on each
    denoised frame before the display pass, as PostProcessStack.runChain
    does (frame by frame; its AGC gain stays the value given)."""
    orbit = orbit or Orbit()
    lens = lens or Lens()
    frames = plan(job, orbit, lens, scene)
    spp = int(job.samples_per_frame)
    uploaded = None
    paths = []

    def upload(sf):
        nonlocal uploaded
        sc = api.build_scene(sf.to_scene_desc())
        ctx.upload(sc)
        uploaded = sf
        return sc

    sc = upload(frames[0][3])
    sp = api.rc_sppm_params(sppm.photons, sppm.hash_size, sppm.alpha) if sppm and sc["light_count"] > 0 else None
    iters = spp if sp is not None else 0
    tl = job.timeline
    use_vhs = vhs is not None and vhs.enabled != 0
    can_batch = batched and not use_vhs and not (tl and (tl.has_scene_object_tracks() or
                                                          tl.has_track("post.exposure")))
    if can_batch:
        ap = api.atrous_params(replace(atrous, exposure=lens.exposure if not tl else frames[0][2].exposure))
        for b0 in range(0, len(frames), batch_frames):
            chunk = frames[b0:b0 + batch_frames]
            ctx.render_frames([(camera_of(o, ln), spp, iters) for _, o, ln, _ in chunk], settings, sp, r0, ap,
                              use_graph=True, read=False)
            for i in range(len(chunk)):
                path = job.frame_path(b0 + i)
                export.write_png(path, ctx.display_frame(i))
                paths.append(path)
        return paths
    for f, (t, o, ln, sf) in enumerate(frames):
        if sf is not uploaded:
            upload(sf)
        ap = api.atrous_params(replace(atrous, exposure=ln.exposure))
        ctx.render_frame(camera_of(o, ln), settings, spp, sp, r0, iters, ap, read=False)
        if use_vhs:
            ctx.post_vhs(vhs_for_frame(vhs, f, t, ln))
        path = job.frame_path(f)
        export.write_png(path, ctx.display())
        paths.append(path)
    return paths
