"""The oracle against committed golden outputs of the reference's own shader
code (tests/golden/*.npz, written by tests/golden/make_golden.py from the
compiled reference).  Bit-for-bit comparisons; needs no reference checkout.
"""
import os
import sys

import numpy as np
import pytest

from conftest import bits

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
sys.path.insert(0, GOLDEN)
import make_golden as mg  # noqa: E402


def _load(name):
    path = os.path.join(GOLDEN, name + ".npz")
    if not os.path.exists(path):
        pytest.fail(f"missing golden fixture {path}")
    return np.load(path)


@pytest.mark.parametrize("case", sorted(mg.CASES))
def test_render_matches_golden(orc, case):
    import pyoracle as po
    wl, W, H, spp, lca = mg.CASES[case]
    _, w, sc, cam = mg.setup(wl)
    cam = dict(cam, lca_delta=(-0.009, 0.0, 0.009) if lca else (0.0, 0.0, 0.0))
    (acc, gb, ga, var), _ = orc.render(sc, cam, (1, 1.0), W, H, 0, spp)
    g = _load(case)
    for name, mine in (("accum", acc), ("gbuffer", gb), ("albedo", ga), ("variance", var)):
        assert np.array_equal(bits(mine), bits(g[name])), name
    if "atrous_5pass" in g:
        p = po.AtrousParams(1, 5, 1.0, 128.0, 1.0, 0, 1.0)
        assert np.array_equal(bits(orc.denoise(acc, gb, ga, var, W, H, spp, p)), bits(g["atrous_5pass"]))


def test_photon_map_and_gather_match_golden(orc):
    P = mg.PHOTONS
    _, w, sc, cam = mg.setup("export_frame")
    ph, heads, nxt, cnt, _ = orc.photon_trace(sc, P["N"], P["radius"], P["seed"], P["hash_size"])
    g = _load("photons_export")
    assert cnt == int(g["count"])
    assert np.array_equal(bits(ph[:cnt].view(np.float32).reshape(cnt, 12)), bits(g["photons"]))
    assert np.array_equal(nxt[:cnt], g["next"])
    used = np.nonzero(heads >= 0)[0]
    assert np.array_equal(used, g["head_cells"]) and np.array_equal(heads[used], g["head_values"])
    W, H = mg.GATHER_SIZE
    acc = np.ones((H, W, 4), np.float32)
    orc.photon_gather(sc, cam, W, H, P["radius"], P["hash_size"], ph, heads, nxt, acc)
    assert np.array_equal(bits(acc), bits(g["gather_80x48"]))
