"""The keyframed export loop's host logic (export/RenderJob.java,
keyframe/KeyframeTimeline.java): frame counts, frame times and paths in
float arithmetic, track application with the setters' clamps, scene-object
tracks."""
import math

import numpy as np

from retrocam_b200 import export_loop as el
from retrocam_b200 import scene_json as sj

f32 = np.float32


def test_job_frames_times_and_paths():
    j = el.RenderJob("out/clip", image_sequence=True, samples_per_frame=4, duration_s=5.0, fps=29.97)
    assert j.total_frames() == 150                       # round(149.85)
    assert el.RenderJob("c", True, duration_s=0.5, fps=29.97).total_frames() == 15   # round(14.985)
    assert el.RenderJob("c", True, duration_s=1.0, fps=24.0).total_frames() == 24
    assert el.RenderJob("c", True, duration_s=0.01, fps=24.0).total_frames() == 1    # at least one
    assert j.frame_dt() == float(f32(1.0) / f32(29.97))
    assert el.RenderJob("c", True, fps=0.0).frame_dt() == float(f32(1.0) / f32(29.97))
    assert j.frame_time(7) == float(f32(7) * f32(j.frame_dt()))
    assert j.frame_path(7) == "out/clip_frames/frame_00007.png"
    photo = el.RenderJob("shots/still")
    assert (photo.total_frames(), photo.frame_time(0), photo.frame_path(0)) == (1, 0.0, "shots/still.png")


def test_timeline_applies_tracks_with_the_setters_clamps():
    tl = el.Timeline(1.0, [
        el.Track("camera", "cam.theta", (0.0, 1.0), (0.0, 2.0), (1, 1)),
        el.Track("camera", "cam.phi", (0.0,), (9.0,)),
        el.Track("camera", "cam.radius", (0.0,), (0.1,)),
        el.Track("camera", "cam.fovY", (0.0,), (400.0,)),
        el.Track("camera", "cam.targetY", (0.0, 1.0), (0.0, 1.0), (0, 0)),
        el.Track("settings", "lens.aperture", (0.0, 1.0), (0.1, 0.3), (1, 1)),
        el.Track("settings", "post.tapeAge", (0.0,), (3.0,)),
        el.Track("settings", "lens.focusDist"),                     # no keys: value kept
    ])
    o, lens, _ = tl.apply(0.5, el.Orbit(), el.Lens(focus_dist_m=2.5), None)
    assert o.theta == 1.0
    assert o.phi == float(f32(f32(math.pi) - f32(0.02)))
    assert o.radius == 0.5 and o.fov_y == 150.0
    assert o.target[1] == 0.0                                   # step: the earlier key
    assert lens.f_stop == float(f32(0.7)) and lens.tape_age == 1.0 and lens.focus_dist_m == 2.5
    assert not tl.has_scene_object_tracks() and tl.has_track("lens.aperture")
    assert not tl.has_track("lens.focusDist")


def test_scene_object_tracks_and_plan():
    scene = sj.SceneFile([sj.MaterialEntry("m")], [sj.ObjectEntry("box"), sj.ObjectEntry("ball", "SPHERE", sx=0.2)])
    tl = el.Timeline(1.0, [el.Track(("object", 1), "pos.x", (0.0, 1.0), (0.0, 1.0), (1, 1)),
                           el.Track(("object", 7), "pos.x", (0.0,), (5.0,))])   # no such object: ignored
    assert tl.has_scene_object_tracks()
    job = el.RenderJob("x", True, 1, duration_s=3 / 24.0, fps=24.0, timeline=tl)
    frames = el.plan(job, el.Orbit(), el.Lens(), scene)
    assert [round(f[0], 6) for f in frames] == [0.0, round(float(f32(1) * f32(1 / 24.0)), 6),
                                                 round(float(f32(2) * f32(f32(1) / f32(24))), 6)]
    xs = [f[3].objects[1].px for f in frames]
    assert xs[0] == 0.0 and 0.0 < xs[1] < xs[2] < 0.1
    assert all(f[3].objects[0] == scene.objects[0] for f in frames)
    assert scene.objects[1].px == 0.0                           # the input scene is left as it was
