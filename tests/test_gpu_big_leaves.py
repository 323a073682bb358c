"""The refill trace over the plain node records.

Scenes whose leaves all hold 1..31 triangles are traced by the refill
kernel over a copy of the node records with packed child references
(wf_trace_dynp); any other tree of at most 28 levels is traced by the same
state machine over the plain records (wf_trace_dyn), whose stack entries
pack a leaf's triangle count into 16 bits.  The reference's builder never
makes leaves that large, but the shaders take any tree the host uploads, so
this file makes one: the export frame's tree with every subtree of at most
`LIMIT` triangles collapsed into a single leaf.  Exact math must give the
oracle's bits and work counts; fast math is held to the statistical bar of
the other fast tests.
"""
import numpy as np
import pytest

from conftest import bits

pytestmark = pytest.mark.gpu

LIMIT = 40   # triangles in the largest collapsed leaf's subtree


def collapse(nodes, limit):
    """The tree with each subtree of at most `limit` triangles as one leaf
    (its triangles are contiguous in the builder's order), in pre-order."""
    count = np.zeros(len(nodes), np.int64)
    lo = np.zeros(len(nodes), np.int64)

    def size(i):
        n = nodes[i]
        if n["prim_count"] > 0:
            count[i], lo[i] = n["prim_count"], n["prim_start"]
        else:
            size(int(n["left_child"]))
            size(int(n["right_child"]))
            a, b = int(n["left_child"]), int(n["right_child"])
            count[i], lo[i] = count[a] + count[b], min(lo[a], lo[b])

    size(0)
    out = []

    def emit(i):
        k = len(out)
        rec = nodes[i].copy()
        out.append(rec)
        if nodes[i]["prim_count"] > 0 or count[i] <= limit:
            rec["left_child"] = rec["right_child"] = -1
            rec["prim_start"], rec["prim_count"] = lo[i], count[i]
            return k
        rec["prim_count"] = 0
        rec["left_child"] = emit(int(nodes[i]["left_child"]))
        rec["right_child"] = emit(int(nodes[i]["right_child"]))
        out[k] = rec
        return k

    emit(0)
    return np.array(out, dtype=nodes.dtype)


@pytest.fixture(scope="module")
def big(product, orc, cuda_ok):
    import deep_bvh
    from retrocam_b200 import scenes
    w = scenes.export_frame()
    sc = dict(product.build_scene(w.scene))
    sc["nodes"] = collapse(sc["nodes"], LIMIT)
    leaves = sc["nodes"][sc["nodes"]["prim_count"] > 0]
    # every triangle in exactly one leaf, some leaves past the packed limit
    covered = np.zeros(len(sc["tris"]), np.int64)
    for s, c in zip(leaves["prim_start"], leaves["prim_count"]):
        covered[s:s + c] += 1
    assert (covered == 1).all()
    assert leaves["prim_count"].max() > 31
    assert deep_bvh.bvh_depth(sc["nodes"]) <= 28
    cam = scenes.camera(w.orbit, w.lens, orc)
    return w, sc, cam


def _ctx(product, W, H, mode):
    ctx = product.Context(W, H, 0, mode)
    ctx.set_engine(product.RC_ENGINE_WAVEFRONT)
    ctx.set_tuning(refill_min_paths=1)   # the refill trace even for this small image
    return ctx


def test_render_exact_bit_identical_big_leaves(product, orc, big):
    w, sc, cam = big
    W, H, spp = 64, 36, 2
    with _ctx(product, W, H, product.RC_MATH_EXACT) as ctx:
        ctx.upload(sc)
        ctx.render(cam, (1, 1.0), 0, spp)
        gpu = ctx.read_buffers()
        cnt = ctx.counters()
    cpu, st = orc.render(sc, cam, (1, 1.0), W, H, 0, spp)
    for name, g, c in zip(("accum", "gbuffer", "albedo", "variance"), gpu, cpu):
        assert np.array_equal(bits(g), bits(c)), name
    assert (cnt["camera_paths"], cnt["closest_rays"], cnt["shadow_rays"]) == tuple(st[:3])
    assert cnt["error_word"] == 0


def test_render_fast_close_big_leaves(product, orc, big):
    """>= 97% of pixels within 1e-4 relative, image mean within 1%."""
    w, sc, cam = big
    W, H, spp = 96, 54, 4
    with _ctx(product, W, H, product.RC_MATH_FAST) as ctx:
        ctx.upload(sc)
        ctx.render(cam, (1, 1.0), 0, spp)
        acc = ctx.read_buffers()[0]
        assert ctx.counters()["error_word"] == 0
    (cacc, _, _, _), _ = orc.render(sc, cam, (1, 1.0), W, H, 0, spp)
    rel = np.abs(acc[..., :3] - cacc[..., :3]) / np.maximum(np.abs(cacc[..., :3]), 1e-3)
    frac_close = np.mean(np.all(rel <= 1e-4, axis=-1))
    assert frac_close >= 0.97, frac_close
    assert abs(acc[..., :3].mean() - cacc[..., :3].mean()) / cacc[..., :3].mean() < 0.01
