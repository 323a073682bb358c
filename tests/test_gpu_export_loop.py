"""The keyframed export loop on the GPU: batched (rc_render_frames +
rc_display_frame) and frame-by-frame (rc_render_frame + rc_display) runs of
the same job write the same PNG bytes under exact math; a photo job writes
one file; tracks on a scene object re-upload the scene per frame."""
import numpy as np
import pytest

from retrocam_b200 import export, scenes
from retrocam_b200 import export_loop as el
from retrocam_b200 import scene_json as sj

pytestmark = pytest.mark.gpu

W, H = 64, 48


def _scene():
    mats = [scenes.diffuse(0.73, 0.73, 0.73), scenes.emissive(1.0, 0.95, 0.85, 15.0),
            scenes.metal(0.95, 0.85, 0.55, 0.1), scenes.glass(1.5)]
    objs = [scenes.Box((0.5, 0.0, 0.5), (1.0, 0.02, 1.0), 0),
            scenes.Box((0.5, 0.5, 1.2), (1.0, 1.0, 0.02), 0),
            scenes.Box((0.5, 1.1, 0.5), (0.2, 0.02, 0.2), 1),
            scenes.Box((0.3, 0.25, 0.6), (0.15, 0.25, 0.15), 2, (0.0, 22.5, 0.0)),
            scenes.Sphere((0.7, 0.2, 0.4), 0.2, 3, 12, 20)]
    return sj.from_scene_desc(scenes.SceneDesc(mats, objs))


def _camera_timeline():
    return el.Timeline(0.25, [el.Track("camera", "cam.theta", (0.0, 0.125), (-1.70, -1.45), (2, 2)),
                              el.Track("settings", "lens.focusDist", (0.0, 0.125), (1.4, 2.2), (1, 1))])


def test_batched_and_frame_by_frame_write_the_same_files(product, tmp_path):
    job_a = el.RenderJob(str(tmp_path / "a" / "clip"), True, 2, duration_s=0.125, fps=24.0,
                         timeline=_camera_timeline())
    job_b = el.RenderJob(str(tmp_path / "b" / "clip"), True, 2, duration_s=0.125, fps=24.0,
                         timeline=_camera_timeline())
    assert job_a.total_frames() == 3
    with product.Context(W, H, 0, product.RC_MATH_EXACT) as ctx:
        pa = el.run_job(ctx, job_a, _scene(), sppm=None, batched=True, batch_frames=2)
        pb = el.run_job(ctx, job_b, _scene(), sppm=None, batched=False)
        assert ctx.counters()["error_word"] == 0
    assert [p.split("/")[-1] for p in pa] == ["frame_00000.png", "frame_00001.png", "frame_00002.png"]
    imgs = [export.read_png(p) for p in pa]
    for a, b in zip(pa, pb):
        assert open(a, "rb").read() == open(b, "rb").read()
    assert not np.array_equal(imgs[0], imgs[2])           # the camera moved
    assert imgs[0][..., :3].std() > 5


def test_photo_job_matches_a_direct_frame(product, tmp_path):
    job = el.RenderJob(str(tmp_path / "still"), samples_per_frame=2)
    lens = el.Lens(focus_dist_m=1.8)
    with product.Context(W, H, 0, product.RC_MATH_EXACT) as ctx:
        (path,) = el.run_job(ctx, job, _scene(), lens=lens, sppm=scenes.SppmDesc(photons=50_000, hash_size=1 << 16))
        img = export.read_png(path)
        ctx.upload(product.build_scene(_scene().to_scene_desc()))
        cam = el.camera_of(el.Orbit(), lens)
        ctx.render_frame(cam, (1, 1.0), 2, product.rc_sppm_params(50_000, 1 << 16, 0.7), 0.02, 2,
                         product.atrous_params(scenes.AtrousDesc()), read=False)
        direct = ctx.display()
    assert path.endswith("still.png")
    # the photon map's insertion order may differ between the two runs
    d = np.abs(img.astype(np.int32) - direct.astype(np.int32))
    assert d.max() <= 2 and (d == 0).mean() > 0.99


def test_scene_object_track_moves_the_object(product, tmp_path):
    tl = el.Timeline(0.125, [el.Track(("object", 4), "pos.x", (0.0, 0.125), (0.3, 0.8), (1, 1))])
    job = el.RenderJob(str(tmp_path / "m" / "clip"), True, 2, duration_s=0.125, fps=24.0, timeline=tl)
    with product.Context(W, H, 0, product.RC_MATH_EXACT) as ctx:
        paths = el.run_job(ctx, job, _scene(), sppm=None)     # falls back to frame by frame
        first = export.read_png(paths[0])
        moved = _scene()
        moved.objects[4].px = 0.3
        ctx.upload(product.build_scene(moved.to_scene_desc()))
        ctx.render_frame(el.camera_of(el.Orbit(), el.Lens()), (1, 1.0), 2, None, 0.02, 0,
                         product.atrous_params(scenes.AtrousDesc()), read=False)
        np.testing.assert_array_equal(first, ctx.display())
    assert not np.array_equal(first, export.read_png(paths[-1]))


def test_vhs_chain_in_the_loop(product, ref, orc, tmp_path):
    """With the VHS chain, each frame is render -> denoise -> chain (frame
    index and time of that frame) -> display; frame 1 equals the chain of the
    reference's pass shaders on that frame's denoised image."""
    vhs = product.vhs_defaults(passes=(3, 7, 10, 16), frame_index=100, agc_gain=2.0)
    job = el.RenderJob(str(tmp_path / "v" / "clip"), True, 2, duration_s=0.125, fps=24.0)
    with product.Context(W, H, 0, product.RC_MATH_EXACT) as ctx:
        paths = el.run_job(ctx, job, _scene(), sppm=None, vhs=vhs)
        ctx.render_frame(el.camera_of(el.Orbit(), el.Lens()), (1, 1.0), 2, None, 0.02, 0,
                         product.atrous_params(scenes.AtrousDesc()), read=False)
        den = ctx.read_output()
    p = el.vhs_for_frame(vhs, 1, job.frame_time(1), el.Lens())
    assert (p.frame_index, p.time_s) == (101, job.frame_time(1))
    want = den
    for k in (3, 7, 10, 16):
        want = ref.post_pass(k, want, W, H, p)
    np.testing.assert_array_equal(export.read_png(paths[1]), orc.display(want, W, H, 1, 1.0))
    assert not np.array_equal(export.read_png(paths[0]), export.read_png(paths[1]))   # the noise moved
