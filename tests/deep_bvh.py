"""Deep BVHs for the traversal tests.

The reference's builder (scene/BVHBuilder.java) gives the test scenes 10 to
27 levels, where none of pathtrace.comp's or photon_trace.comp's stacks can
overflow.  The shaders take any tree the host uploads, though, and their
stack policies -- closest hit: 64 entries, a node's children pushed only
while top < 62 (pathtrace.comp:176); shadow: 32 entries, top < 30
(pathtrace.comp:235); photon trace and gather: 64 entries, top < 62
(photon_trace.comp:102-128) -- decide which subtrees a walk skips once the
stack is full.  `chain_scene` makes a tree where they matter:

  * the scene's triangles are sorted by centroid along a fixed direction and
    cut into `groups` consecutive groups;
  * each group gets its own BVH from the backend's builder (the reference's
    binned SAH), its triangles in that builder's order;
  * the group trees hang off a chain: chain node k has the chain's rest as
    its LEFT child and group k's tree as its RIGHT child, the last chain
    node being group K-1's tree itself.

Depth is (groups - 1) + the deepest group tree.  The push-untested walks
(shadow, photon, gather) push right then left and pop left first, so they
leave one group tree on the stack per chain level: the 32-entry shadow
stack fills at chain level 30 and the 64-entry photon stack at level 62.
The closest-hit walk pushes the farther child, so rays that meet the
chain's rest before its group (those travelling against the sort
direction) fill its stack too.  Nodes are stored in pre-order (parent, left
subtree, right subtree), as the reference's builder stores them.
"""
from __future__ import annotations

import numpy as np

SORT_DIRECTION = np.array([0.62, 0.31, 0.72], np.float64)


def _depth(nodes) -> int:
    best, todo = 0, [(0, 0)]
    while todo:
        i, d = todo.pop()
        n = nodes[i]
        if n["prim_count"] > 0:
            best = max(best, d)
        else:
            todo.append((int(n["left_child"]), d + 1))
            todo.append((int(n["right_child"]), d + 1))
    return best


def bvh_depth(nodes) -> int:
    """Levels below the root (0 for a root leaf), as rc_counters.bvh_depth."""
    return _depth(nodes)


def chain_bvh(tris: np.ndarray, groups: int, backend):
    """(triangles in the new order, nodes) of the chained tree over `tris`."""
    c = (tris["v0"].astype(np.float64) + tris["v1"] + tris["v2"]) / 3.0
    order = np.argsort(c @ SORT_DIRECTION, kind="stable")
    cuts = np.linspace(0, len(tris), groups + 1).round().astype(int)
    parts, subtrees, offset = [], [], 0
    for g in range(groups):
        sub = tris[order[cuts[g]:cuts[g + 1]]]
        t, n = backend.build_bvh(sub)
        n = n.copy()
        leaf = n["prim_count"] > 0
        n["prim_start"][leaf] += offset
        parts.append(t)
        subtrees.append(n)
        offset += len(t)
    node_dtype = subtrees[0].dtype
    # pre-order: chain node k, chain node k+1 ... (left), then group k (right)
    # -- i.e. all chain nodes first, then the group trees from the last
    # group back to the first.
    n_chain = groups - 1
    out = []

    def box_of(n):
        return np.asarray(n["aabb_min"], np.float32), np.asarray(n["aabb_max"], np.float32)

    # boxes of the chain nodes: union of their groups' roots
    lo = [None] * groups
    hi = [None] * groups
    run_lo, run_hi = box_of(subtrees[-1][0])
    for k in range(groups - 2, -1, -1):
        glo, ghi = box_of(subtrees[k][0])
        run_lo, run_hi = np.minimum(run_lo, glo), np.maximum(run_hi, ghi)
        lo[k], hi[k] = run_lo.copy(), run_hi.copy()
    # positions: chain nodes 0..n_chain-1 at 0..n_chain-1, then the group
    # trees in pre-order of the whole tree (the deepest chain node's left
    # child is group K-1's tree, its right child group K-2's tree, ...)
    base = {}
    pos = n_chain
    for g in [groups - 1] + list(range(groups - 2, -1, -1)):
        base[g] = pos
        pos += len(subtrees[g])
    for k in range(n_chain):
        rec = np.zeros(1, node_dtype)[0]
        rec["aabb_min"], rec["aabb_max"] = lo[k], hi[k]
        left = k + 1 if k + 1 < n_chain else base[groups - 1]
        rec["left_child"], rec["right_child"] = left, base[k]
        out.append(rec)
    for g in [groups - 1] + list(range(groups - 2, -1, -1)):
        n = subtrees[g].copy()
        inner = n["prim_count"] <= 0
        n["left_child"][inner] += base[g]
        n["right_child"][inner] += base[g]
        out.extend(list(n))
    nodes = np.array(out, dtype=node_dtype)
    return np.concatenate(parts), nodes


def chain_scene(desc, backend, mat_dtype, groups: int = 80) -> dict:
    """scenes.build_scene with the chained tree in place of the builder's
    BVH (the light list follows the new triangle order, as SceneUploader
    builds it after the BVH)."""
    from retrocam_b200 import scenes
    tris = scenes.tessellate(desc, backend)
    mats = scenes.material_array(desc.materials, mat_dtype)
    tris, nodes = chain_bvh(tris, groups, backend)
    lights, total = backend.build_lights(tris, mats)
    light_count = len(lights)
    if light_count == 0:
        lights = np.zeros(1, lights.dtype)
    return {"tris": tris, "nodes": nodes, "mats": mats, "lights": lights, "light_count": light_count,
            "total_power": total}
