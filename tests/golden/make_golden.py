"""Generates tests/golden/*.npz from the reference's own shaders compiled for
the host (oracle/_ref/libretrocam_ref.so, built by oracle/build_ref.py from a
reference checkout).  Run from the repository root:

    python tests/golden/make_golden.py

Scenes, cameras and settings come from retrocam_b200/scenes.py, tessellated
and BVH-built by the oracle's restatement of the reference's Java host code;
the images, photon maps and denoised frames are outputs of the reference
shader code.  tests/test_golden.py recomputes each case with the oracle and
compares bit for bit.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "oracle"))

CASES = {
    # name: (workload, W, H, spp, lca)
    "render_cornell_64x64_3spp": ("cornell_small", 64, 64, 3, False),
    "render_cornell_lca_48x40_2spp": ("cornell_small", 48, 40, 2, True),
    "render_export_96x54_3spp": ("export_frame", 96, 54, 3, True),
}
PHOTONS = dict(N=120_000, radius=0.02, seed=3 * 7919 + 6271, hash_size=1 << 18)
GATHER_SIZE = (80, 48)


def setup(name):
    import pyoracle as po
    from retrocam_b200 import scenes
    orc, _ = po.load(build=False)
    w = scenes.WORKLOADS[name]()
    sc = scenes.build_scene(w.scene, orc, po.MAT)
    cam = scenes.camera(w.orbit, w.lens, orc)
    return orc, w, sc, cam


def main():
    import pyoracle as po
    _, ref = po.load(build=True)
    if ref is None:
        raise SystemExit("the compiled reference (oracle/_ref) is required")
    for case, (wl, W, H, spp, lca) in CASES.items():
        orc, w, sc, cam = setup(wl)
        cam = dict(cam, lca_delta=(-0.009, 0.0, 0.009) if lca else (0.0, 0.0, 0.0))
        acc, gb, ga, var = ref.render(sc, cam, (1, 1.0), W, H, 0, spp)
        out = {"accum": acc, "gbuffer": gb, "albedo": ga, "variance": var}
        if case == "render_export_96x54_3spp":
            p = po.AtrousParams(1, 5, 1.0, 128.0, 1.0, 0, 1.0)
            out["atrous_5pass"] = ref.denoise(acc, gb, ga, var, W, H, spp, p)
        np.savez_compressed(os.path.join(HERE, case + ".npz"), **out)
    orc, w, sc, cam = setup("export_frame")
    ph, heads, nxt, cnt = ref.photon_trace(sc, PHOTONS["N"], PHOTONS["radius"], PHOTONS["seed"],
                                           PHOTONS["hash_size"], threads=1)
    used = np.nonzero(heads >= 0)[0].astype(np.int32)
    W, H = GATHER_SIZE
    acc = np.ones((H, W, 4), np.float32)
    ref.photon_gather(sc, cam, W, H, PHOTONS["radius"], PHOTONS["N"], PHOTONS["hash_size"], 0, ph, heads, nxt, acc)
    np.savez_compressed(os.path.join(HERE, "photons_export.npz"), count=np.int64(cnt),
                        photons=ph[:cnt].view(np.float32).reshape(cnt, 12), next=nxt[:cnt],
                        head_cells=used, head_values=heads[used], gather_80x48=acc)
    print("wrote", sorted(f for f in os.listdir(HERE) if f.endswith(".npz")))


if __name__ == "__main__":
    main()
