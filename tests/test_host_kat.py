"""Known answers for the Java host logic, derived by hand from the reference.

The product's host code (retrocam_b200/csrc/host_scene.cpp, behind the C ABI)
and the oracle's (oracle/oracle_host.cpp) are two restatements by one author
of scene/BVHBuilder.java, scene/Box.java and scene/Sphere.java; comparing them
with each other cannot catch a misreading they share.  The answers below
were worked out from the Java by hand (the derivations are in the comments)
on inputs whose arithmetic is exact in float, and both implementations must
reproduce them bit for bit.

BVHBuilder.java, the rules exercised:
  * node bounds = union of the triangles' AABBs (fromTriangles, :56-62); the
    bucketing range of an axis is the NODE's extent, lo = axisMin(parent),
    hi = axisMax(parent) (:107-109), not the centroids' extent;
  * b = min(7, (int)(8 * (c - lo) / (hi - lo))) with c = (v0+v1+v2)/3f (:116-118);
    an axis with hi - lo < 1e-6 is skipped (:109);
  * cost = 1 + SA_L*n_L*1.5/SA_P + SA_R*n_R*1.5/SA_P for s = 0..6, axes x, y,
    z in order, first strict minimum wins (:124-142);
  * leaf when count <= 4, when best cost >= 1.5*count (:76-80);
  * partition: while lo <= hi, keep tris[lo] if c < splitPos else swap with
    tris[hi--] (:150-164); splitPos = lo + (hi - lo) * (s + 1) / 8 (:138);
  * nodes in pre-order, leaves have children -1 (BVHNode.java:22-25).
"""
import numpy as np
import pytest

INF = None


# ---------------------------------------------------------------------------
# triangle families with exact centroids
# ---------------------------------------------------------------------------
def _x_tri(c):
    """X(c): v0 (c-.5, 0, 0), v1 (c, 1, 0), v2 (c+.5, 0, 1).  cx = 3c/3 = c
    exactly; cy = cz = 1/3f for every such triangle (one bucket: y and z
    never split); AABB x [c-.5, c+.5], y [0, 1], z [0, 1]."""
    return [c - 0.5, 0, 0, c, 1, 0, c + 0.5, 0, 1]


def _xz_tri(cx, cz):
    """T(cx, cz): v0 (cx-.5, 0, cz-.5), v1 (cx, 1, cz), v2 (cx+.5, 0, cz+.5):
    centroid (cx, 1/3f, cz) exactly in x and z; the set {T(a,b)} is mapped
    onto itself by swapping x and z."""
    return [cx - 0.5, 0, cz - 0.5, cx, 1, cz, cx + 0.5, 0, cz + 0.5]


def _wide_tri(c):
    """W(c): v0 (0, 0, 0), v1 (3c-8, 1, 0), v2 (8, 0, 1): cx = c exactly,
    AABB x [0, 8] for 8/3 <= c <= 16/3 -- every W has the same box."""
    return [0, 0, 0, 3 * c - 8, 1, 0, 8, 0, 1]


def _tris(backend, rows):
    return backend.flat_triangles(np.asarray(rows, np.float32), 0)


def _node(lo, hi, left=-1, right=-1, start=0, count=0):
    return (tuple(map(float, lo)), tuple(map(float, hi)), left, right, start, count)


def _nodes_as_tuples(nodes):
    return [(tuple(map(float, n["aabb_min"])), tuple(map(float, n["aabb_max"])), int(n["left_child"]),
             int(n["right_child"]), int(n["prim_start"]), int(n["prim_count"])) for n in nodes]


def _backends(product, orc):
    return {"product": product.HOST, "oracle": orc}


# ---------------------------------------------------------------------------
# BVH scenario 1: recursion, ties between splits, the partition's swap order
# ---------------------------------------------------------------------------
# Input order of centroids: 16, 1, 15, 2, 14, 3, 13, 4, 30, 29 (indices 0-9).
#
# Root, 10 triangles: x [0.5, 30.5], hi-lo = 30.  b = (int)(8(c-.5)/30):
#   c=1,2,3,4 -> 0.13,0.4,0.67,0.93 -> 0;  13,14,15 -> 3.33,3.6,3.87 -> 3;
#   16 -> 4.13 -> 4;  29,30 -> 7.6,7.87 -> 7.
#   SA = 2(dx*1 + 1*1 + 1*dx) = 4dx + 2 (y and z extents are 1); SA_P = 122.
#   s=0,1,2: L {1..4} dx 4 SA 18 n 4, R dx 18 SA 74 n 6:
#            1 + 108/122 + 666/122 = 7.34
#   s=3:     L dx 15 SA 62 n 7, R dx 15 SA 62 n 3: 1 + 651/122 + 279/122 = 8.62
#   s=4..6:  L dx 16 SA 66 n 8, R dx 2 SA 10 n 2: 1 + 792/122 + 30/122 = 7.74
#   best s=0 (s=1,2 tie with it, not strictly less), 7.34 < 15 = 1.5*10;
#   splitPos = 0.5 + 30*1/8 = 4.25.
# Partition [16,1,15,2,14,3,13,4,30,29] at 4.25 (lo=0, hi=9):
#   16 -> swap(0,9) [29,1,15,2,14,3,13,4,30,16] hi 8
#   29 -> swap(0,8) [30,1,15,2,14,3,13,4,29,16] hi 7
#   30 -> swap(0,7) [4,1,15,2,14,3,13,30,29,16] hi 6
#   4 keep, 1 keep, 15 -> swap(2,6) [4,1,13,2,14,3,15,30,29,16] hi 5
#   13 -> swap(2,5) [4,1,3,2,14,13,15,30,29,16] hi 4
#   3 keep, 2 keep, 14 -> swap(4,4) hi 3; mid = 4.
# Node 1 = leaf [0,4) {4,1,3,2}, x [0.5, 4.5].
# Node 2, [4,10) = {14,13,15,30,29,16}: x [12.5, 30.5], hi-lo 18, SA_P 74.
#   b = (int)(8(c-12.5)/18): 14 -> .67 -> 0; 13 -> .22 -> 0; 15 -> 1.11 -> 1;
#   30 -> 7.78 -> 7; 29 -> 7.33 -> 7; 16 -> 1.56 -> 1.
#   s=0: L {13,14} SA 10 n 2, R dx 16 SA 66 n 4: 1 + 30/74 + 396/74 = 6.76
#   s=1..6: L {13..16} dx 4 SA 18 n 4, R {29,30} SA 10 n 2: 1 + 108/74 + 30/74 = 2.86
#   best s=1 (< 9 = 1.5*6); splitPos = 12.5 + 18*2/8 = 17.
#   Partition [14,13,15,30,29,16] at 17: 14,13,15 keep; 30 -> swap with 16
#   [14,13,15,16,29,30] hi 8; 16 keep; 29 -> swap(8,8) hi 7; mid = 8.
# Node 3 = leaf [4,8) {14,13,15,16} x [12.5,16.5]; node 4 = leaf [8,10) {29,30}.
S1_INPUT = [16, 1, 15, 2, 14, 3, 13, 4, 30, 29]
S1_ORDER = [4, 1, 3, 2, 14, 13, 15, 16, 29, 30]
S1_NODES = [
    _node((0.5, 0, 0), (30.5, 1, 1), left=1, right=2),
    _node((0.5, 0, 0), (4.5, 1, 1), start=0, count=4),
    _node((12.5, 0, 0), (30.5, 1, 1), left=3, right=4),
    _node((12.5, 0, 0), (16.5, 1, 1), start=4, count=4),
    _node((28.5, 0, 0), (30.5, 1, 1), start=8, count=2),
]


@pytest.mark.parametrize("which", ["product", "oracle"])
def test_bvh_scenario_recursion_and_partition_order(product, orc, which):
    be = _backends(product, orc)[which]
    tris, nodes = be.build_bvh(_tris(be, [_x_tri(c) for c in S1_INPUT]))
    got_order = [float((t["v0"][0] + t["v1"][0] + t["v2"][0]) / np.float32(3)) for t in tris]
    assert got_order == [float(c) for c in S1_ORDER]
    assert _nodes_as_tuples(nodes) == S1_NODES


# ---------------------------------------------------------------------------
# BVH scenario 2: a tie between axes -- x wins
# ---------------------------------------------------------------------------
# Five T(cx, cz), input order (9,9), (1,9), (8,8), (9,1), (1,1): a set mapped
# onto itself by swapping x and z, so the x and z bucket costs are the same
# float operations on the same values -- an exact tie -- and x, searched
# first, must win (cost < best.cost is strict).
# Node: x [0.5, 9.5], y [0, 1], z [0.5, 9.5]; SA_P = 2(9*1 + 1*9 + 9*9) = 198.
#   y: every cy = 1/3f -> one bucket -> no split.
#   x: b = (int)(8(cx-.5)/9): 1 -> .44 -> 0; 8 -> 6.67 -> 6; 9 -> 7.56 -> 7.
#   s=0..5: L {(1,9),(1,1)} box x [.5,1.5] z [.5,9.5]: SA 2(1+9+9) = 38, n 2;
#           R {(8,8),(9,9),(9,1)} x [7.5,9.5] z [.5,9.5]: SA 2(2+9+18) = 58, n 3:
#           1 + 114/198 + 261/198 = 2.89
#   s=6:    L x [.5,8.5]: SA 2(8+9+72) = 178, n 3; R x [8.5,9.5]: SA 38, n 2: 5.62
#   best x: s=0, splitPos = 0.5 + 9/8 = 1.625; z gives the same cost, not less.
# Partition along x at 1.625 over [(9,9),(1,9),(8,8),(9,1),(1,1)]:
#   (9,9) -> swap(0,4) [(1,1),(1,9),(8,8),(9,1),(9,9)] hi 3
#   (1,1) keep, (1,9) keep, (8,8) -> swap(2,3) [(1,1),(1,9),(9,1),(8,8),(9,9)] hi 2
#   (9,1) -> swap(2,2) hi 1; mid = 2.   (Along z the left leaf would hold
#   (1,1) and (9,1) instead.)
S2_INPUT = [(9, 9), (1, 9), (8, 8), (9, 1), (1, 1)]
S2_ORDER = [(1, 1), (1, 9), (9, 1), (8, 8), (9, 9)]
S2_NODES = [
    _node((0.5, 0, 0.5), (9.5, 1, 9.5), left=1, right=2),
    _node((0.5, 0, 0.5), (1.5, 1, 9.5), start=0, count=2),
    _node((7.5, 0, 0.5), (9.5, 1, 9.5), start=2, count=3),
]


@pytest.mark.parametrize("which", ["product", "oracle"])
def test_bvh_scenario_axis_tie_takes_x(product, orc, which):
    be = _backends(product, orc)[which]
    tris, nodes = be.build_bvh(_tris(be, [_xz_tri(a, b) for a, b in S2_INPUT]))
    got = [(float(t["v1"][0]), float(t["v1"][2])) for t in tris]   # v1 = (cx, 1, cz)
    assert got == [(float(a), float(b)) for a, b in S2_ORDER]
    assert _nodes_as_tuples(nodes) == S2_NODES


# ---------------------------------------------------------------------------
# BVH scenario 3: the cost rule makes a leaf of more than four triangles
# ---------------------------------------------------------------------------
# Five W(c), c = 3, 4, 5, 4, 3: every AABB is x [0, 8], y [0, 1], z [0, 1],
# so SA_L = SA_R = SA_P = 2(8 + 1 + 8) = 34 whatever the split.
#   x: lo 0, hi 8, b = (int)(8c/8) = c: buckets 3 {3,3}, 4 {4,4}, 5 {5}.
#   s=3: 1 + 34*2*1.5/34 + 34*3*1.5/34 = 1 + 3 + 4.5 = 8.5
#   s=4: 1 + 34*4*1.5/34 + 34*1*1.5/34 = 1 + 6 + 1.5 = 8.5
#   (all exact); 8.5 >= 7.5 = 1.5*5 -> one leaf of 5, input order kept.
S3_INPUT = [3, 4, 5, 4, 3]


@pytest.mark.parametrize("which", ["product", "oracle"])
def test_bvh_scenario_cost_rule_leaf(product, orc, which):
    be = _backends(product, orc)[which]
    src = _tris(be, [_wide_tri(c) for c in S3_INPUT])
    tris, nodes = be.build_bvh(src)
    assert np.array_equal(tris.view(np.uint8), src.view(np.uint8))
    assert _nodes_as_tuples(nodes) == [_node((0, 0, 0), (8, 1, 1), start=0, count=5)]


# ---------------------------------------------------------------------------
# Box.java:25-76 -- twelve triangles, vertex order, flat normals, UVs
# ---------------------------------------------------------------------------
# Box centre (1, 2, 3), half extents (0.5, 1, 1.5): x0 .5, x1 1.5, y0 1,
# y1 3, z0 1.5, z1 4.5 (all exact).  Faces in order +X, -X, +Y, -Y, +Z, -Z;
# each quad (a, b, c, d) gives t1 = (a, b, c), UVs (0,0) (0,1) (1,1), and
# t2 = (a, c, d), UVs (0,0) (1,1) (1,0).
# GpuTriangle.withFlatNormal (:38-50): A = v1 - v0, B = v2 - v0,
#   n = (Ay*Bz - Az*By, Az*Bx - Ax*Bz, Ax*By - Ay*Bx) / |n|; the signs of the
#   zero components follow IEEE: 0*(-k) = -0, (-0) - (+0) = -0,
#   (+0) - (-0) = +0, (-0) - (-0) = +0.
#   +X t1: A (0,2,0) B (0,2,-3): (2(-3) - 0*2, 0*0 - 0(-3), 0*2 - 2*0)
#          = (-6, +0 - -0 = +0, +0) -> (-1, +0, +0)
#   +X t2: A (0,2,-3) B (0,0,-3): (-6 - (-3)0 = -6, (-3)0 - 0(-3) = -0 - -0 = +0, +0)
#   -X t1: A (0,2,0) B (0,2,3): (6, +0, +0);  -X t2: A (0,2,3) B (0,0,3): (6, +0, +0)
#   +Y t1: A (0,0,-3) B (1,0,-3): (0(-3) - (-3)0 = -0 - -0 = +0, -3 - 0(-3) = -3, +0)
#   +Y t2: A (1,0,-3) B (1,0,0): (0*0 - (-3)0 = +0 - -0 = +0, -3*1 - 1*0 = -3, +0)
#   -Y t1: A (0,0,3) B (1,0,3): (+0, 3, +0);  -Y t2: A (1,0,3) B (1,0,0): (+0, 3, +0)
#   +Z t1: A (0,2,0) B (1,2,0): (+0, +0, 0*2 - 2*1 = -2)
#   +Z t2: A (1,2,0) B (1,0,0): (+0, +0, 1*0 - 2*1 = -2)
#   -Z t1: A (0,2,0) B (-1,2,0): (+0, 0(-1) - 0*0 = -0 - +0 = -0, 0*2 - 2(-1) = 2)
#   -Z t2: A (-1,2,0) B (-1,0,0): (+0, 0(-1) - (-1)0 = -0 - -0 = +0, (-1)0 - 2(-1) = 2)
#   each divided by its length (6, 6, 6, 6, 3, 3, 3, 3, 2, 2, 2, 2).
_X0, _X1, _Y0, _Y1, _Z0, _Z1 = 0.5, 1.5, 1.0, 3.0, 1.5, 4.5
_QUADS = [
    ((_X1, _Y0, _Z1), (_X1, _Y1, _Z1), (_X1, _Y1, _Z0), (_X1, _Y0, _Z0)),   # +X
    ((_X0, _Y0, _Z0), (_X0, _Y1, _Z0), (_X0, _Y1, _Z1), (_X0, _Y0, _Z1)),   # -X
    ((_X0, _Y1, _Z1), (_X0, _Y1, _Z0), (_X1, _Y1, _Z0), (_X1, _Y1, _Z1)),   # +Y
    ((_X0, _Y0, _Z0), (_X0, _Y0, _Z1), (_X1, _Y0, _Z1), (_X1, _Y0, _Z0)),   # -Y
    ((_X0, _Y0, _Z1), (_X0, _Y1, _Z1), (_X1, _Y1, _Z1), (_X1, _Y0, _Z1)),   # +Z
    ((_X1, _Y0, _Z0), (_X1, _Y1, _Z0), (_X0, _Y1, _Z0), (_X0, _Y0, _Z0)),   # -Z
]
_NORMALS = [(-1.0, 0.0, 0.0), (-1.0, 0.0, 0.0), (1.0, 0.0, 0.0), (1.0, 0.0, 0.0),
            (0.0, -1.0, 0.0), (0.0, -1.0, 0.0), (0.0, 1.0, 0.0), (0.0, 1.0, 0.0),
            (0.0, 0.0, -1.0), (0.0, 0.0, -1.0), (0.0, -0.0, 1.0), (0.0, 0.0, 1.0)]


def _box_expected():
    out = []
    for k, (a, b, c, d) in enumerate(_QUADS):
        out.append(((a, b, c), ((0, 0), (0, 1), (1, 1)), _NORMALS[2 * k]))
        out.append(((a, c, d), ((0, 0), (1, 1), (1, 0)), _NORMALS[2 * k + 1]))
    return out


def _bits(x):
    return np.asarray(x, np.float32).view(np.uint32).tolist()


@pytest.mark.parametrize("which", ["product", "oracle"])
def test_box_tessellation(product, orc, which):
    be = _backends(product, orc)[which]
    tris = be.tess_box((1.0, 2.0, 3.0), (0.5, 1.0, 1.5), 7)
    assert len(tris) == 12
    for t, (verts, uvs, n) in zip(tris, _box_expected()):
        assert [tuple(map(float, t[k])) for k in ("v0", "v1", "v2")] == list(verts)
        assert [tuple(map(float, t[k])) for k in ("uv0", "uv1", "uv2")] == [tuple(map(float, u)) for u in uvs]
        for k in ("n0", "n1", "n2"):
            assert _bits(t[k]) == _bits(n), (k, t[k], n)   # signs of zero included
        assert int(t["mat_index"]) == 7


# ---------------------------------------------------------------------------
# Sphere.java:34-101 -- triangle order and pole skipping (3 stacks x 4 slices)
# ---------------------------------------------------------------------------
# Grid point P(i, j) = spherePt(phi_i, theta_j) with phi_i = (float)(pi*i/3),
# theta_j = (float)(2*pi*j/4).  For i in 0..2 (outer), j in 0..3 (inner) the
# quad is A = P(i,j), B = P(i,j+1), C = P(i+1,j+1), D = P(i+1,j); the
# triangle (A, B, C) is skipped at i == 0 and (A, C, D) at i == stacks-1, so
# 2*3*4 - 2*4 = 16 triangles, in this order:
SPHERE_ORDER = (
    [((0, j), (1, j + 1), (1, j)) for j in range(4)] +                          # i = 0: ACD only
    [t for j in range(4) for t in (((1, j), (1, j + 1), (2, j + 1)),            # i = 1: ABC, ACD
                                    ((1, j), (2, j + 1), (2, j)))] +
    [((2, j), (2, j + 1), (3, j + 1)) for j in range(4)]                        # i = 2: ABC only
)


def _sphere_point(c, r, i, j, stacks=3, slices=4):
    """spherePt with Java's casts: phi, theta rounded to float; sin/cos in
    double of the float angle, rounded to float; float products left to
    right: cx + (radius * sinP) * cos(theta)."""
    f = np.float32
    phi = f(np.pi * i / stacks)
    theta = f(2 * np.pi * j / slices)
    sinp = f(np.sin(np.float64(phi)))
    return (f(f(c[0]) + f(f(f(r) * sinp) * f(np.cos(np.float64(theta))))),
            f(f(c[1]) + f(f(r) * f(np.cos(np.float64(phi))))),
            f(f(c[2]) + f(f(f(r) * sinp) * f(np.sin(np.float64(theta))))))


@pytest.mark.parametrize("which", ["product", "oracle"])
def test_sphere_triangle_order(product, orc, which):
    be = _backends(product, orc)[which]
    c, r = (0.25, 0.5, 0.75), 2.0
    tris = be.tess_sphere(c, r, 3, 3, 4)
    assert len(tris) == len(SPHERE_ORDER) == 16
    for t, corners in zip(tris, SPHERE_ORDER):
        for k, (i, j) in zip(("v0", "v1", "v2"), corners):
            assert _bits(t[k]) == _bits(_sphere_point(c, r, i, j)), (k, i, j)
        # uv of corner (i, j) is ((float)j/4, (float)i/3)
        for k, (i, j) in zip(("uv0", "uv1", "uv2"), corners):
            assert _bits(t[k]) == _bits((np.float32(j) / np.float32(4), np.float32(i) / np.float32(3)))
        assert int(t["mat_index"]) == 3
