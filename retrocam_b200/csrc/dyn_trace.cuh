// dyn_trace.cuh -- the per-lane traversal state machine of the refill
// kernels (camera / shadow rays in wavefront.cu, both builds; photon first
// segments in kernels.cu: the fast build's split walk, the exact build's
// full-scene walk in the reference's photon order).
//
// A lane owns one ray at a time and advances it per loop iteration of its
// warp: interior nodes, parking a reached leaf, or the triangles of a parked
// leaf.  Leaf tests and interior steps never share an iteration: the warp
// tests leaves (every lane with one parked, together) once all busy lanes
// have one parked or `leaf_quarters` quarters of them are blocked (a leaf
// parked and no interior node to go on with); otherwise the unblocked lanes
// take up to `interior_steps` interior moves each.  A kernel refills lanes
// whose ray finished from its own work list when fewer than `refill_lanes`
// lanes are busy, so a warp is not held by its slowest ray.
//
// Fast build: a lane walks on past a parked leaf (its triangles are tested
// later, with the warp); the hits are the plain traversal's, ties aside.
// Exact build: a closest-hit lane stops at a reached leaf until the warp
// tests it, and pops the next stack entry only then, with the entry distance
// kept exactly -- trace_closest's visits in trace_closest's order, so the
// same hit bit for bit; shadow lanes walk on as in the fast build (a yes/no
// that does not depend on the order).
//
// Node references come in two encodings: (ref, count) pairs from the plain
// records, or one packed word per child from DeviceScene::nodes_packed
// (kPacked), whose stack entries keep the full entry distance.
#ifndef RC_DYN_TRACE_CUH
#define RC_DYN_TRACE_CUH

#include "device_common.cuh"

namespace rc {
namespace RC_NS {

#if !RC_EXACT
// Stack entries: the binary walk pushes at most one per level (guarded at
// 62, as the reference, where the tree can be that deep), the 4-wide walk
// up to three.  An entry is 8 bytes: over the plain records (ref, count |
// entry distance truncated to its top 16 bits) -- truncation rounds a
// positive distance down, so the cull `t > hit` never drops a needed
// entry; over the packed records (reference, entry distance).
constexpr int kDynStack = 96;
struct DynStack {
    int2 e[kDynStack];
};

// Pops the next stack entry not culled by the current hit distance.
DI bool pop_entry(DynStack& stk, int& top, float cull, TravNode& n) {
    while (top > 0) {
        const int2 e = stk.e[--top];
        if (__int_as_float(e.y & (int)0xffff0000) > cull) continue;
        n.ref = e.x;
        n.cnt = e.y & 0xffff;
        return true;
    }
    return false;
}

#else
// Exact build: (ref, count) and the exact entry distance the parent
// computed (what the reference's re-test on pop returns); at most 61
// entries on trees of up to 60 levels, the only ones this walk serves.
constexpr int kDynStack = 64;
struct DynStack {
    int2 e[kDynStack];
    float t[kDynStack];
};

DI bool pop_entry(DynStack& stk, int& top, float cull, TravNode& n) {
    while (top > 0) {
        --top;
        if (stk.t[top] > cull) continue;
        n.ref = stk.e[top].x;
        n.cnt = stk.e[top].y;
        return true;
    }
    return false;
}
#endif

// Packed child references (DeviceScene::nodes_packed): a TravNode's ref
// alone names a child -- a node index, or for a leaf INT_MIN | prim_start
// << 5 | count -- so choosing a child is one select, and a stack entry is
// (reference, the full entry distance bits) in both builds.
DI int pk_start(int p) { return (int)(((unsigned int)p >> 5) & 0x3ffffffu); }
DI int pk_count(int p) { return p & 31; }

DI bool pop_packed(DynStack& stk, int& top, float cull, TravNode& n) {
    while (top > 0) {
        const int2 e = stk.e[--top];
        if (__int_as_float(e.y) > cull) continue;
        n.ref = e.x;
        return true;
    }
    return false;
}
// The members of a DeviceScene that dyn_step reads, for walks whose scene
// is chosen per lane (a select of four values instead of a whole scene).
struct StepScene {
    const NodeRec* nodes;
    const Node4* nodes4;
    const float4* tri_isect;
    int node_count;
};

DI StepScene step_scene(bool second, const DeviceScene& a, const DeviceScene& b) {
    StepScene s;
    s.nodes = second ? b.nodes : a.nodes;
    s.nodes4 = second ? b.nodes4 : a.nodes4;
    s.tri_isect = second ? b.tri_isect : a.tri_isect;
    s.node_count = second ? b.node_count : a.node_count;
    return s;
}

struct LaneRay {
    Ray r;
    Hit h;
    TravNode node, leaf;
    bool have_node;
    bool any;      // any hit below h.t (visibility), else closest hit
    int item;      // the kernel's work index, -1 idle, -2 no more work
    int top;
    int steps;     // moves and leaf tests so far, checked against the
                   // traversal cap once per dyn_step call (a call makes at
                   // most interior_steps moves, so the cap is overshot by
                   // fewer than 8; counting per move cost 2.3 ms of a
                   // 61.4 ms trace per export frame)
};

// Starts L's walk of S (a DeviceScene, or any type with the same root and
// array members) for ray r up to tmax.
template <class Scn>
DI void dyn_start(const Scn& S, LaneRay& L, float tmax, bool any, Guard& g) {
    L.any = any;
    L.h.t = tmax;
    L.h.prim = -1;
    L.h.u = L.h.v = 0.0f;
    L.top = 0;
    L.leaf.cnt = 0;
    L.leaf.ref = 0;
    L.node.ref = S.root_ref;
    L.node.cnt = S.root_count;
    L.steps = 0;
    float tmin;
    L.have_node = S.tri_count > 0 &&
                  tslab(g, L.r, S.root_min[0], S.root_min[1], S.root_min[2], S.root_max[0], S.root_max[1],
                        S.root_max[2], tmin) &&
                  !(tmin > L.h.t);
}

// Whether n is a leaf, and whether L has a leaf parked, in either encoding.
template <bool kPacked>
DI bool is_leaf(const TravNode& n) {
    return kPacked ? n.ref < 0 : n.cnt > 0;
}
template <bool kPacked>
DI bool parked_leaf(const LaneRay& L) {
    return is_leaf<kPacked>(L.leaf);
}

// The warp's choice for this iteration; every lane of the warp calls it with
// the warp's busy mask `act` (the caller's ballot of `busy`).  Returns
// whether this lane steps, and the phase.
template <bool kPacked = false>
DI bool dyn_schedule(const LaneRay& L, bool busy, unsigned int act, int leaf_quarters, bool& leaf_phase) {
    const unsigned int FULL = 0xffffffffu;
    const bool has = parked_leaf<kPacked>(L);
    const bool blocked = busy && has && (!L.have_node || is_leaf<kPacked>(L.node));
    const unsigned int parked = __ballot_sync(FULL, busy && has);
    const unsigned int blk = __ballot_sync(FULL, blocked);
    leaf_phase = parked == act || 4 * __popc(blk) >= leaf_quarters * __popc(act);
    return busy && (leaf_phase ? has : !blocked);
}

#if !RC_EXACT
// One step of L (kWide: interior nodes from S.nodes4): in the leaf phase the
// parked leaf's triangles; otherwise up to `interior_steps` moves through
// the tree -- interior nodes, or parking a reached leaf -- while the lane is
// not blocked (a leaf parked and the next node a leaf too, or none), so the
// warp's scheduling work is shared by several moves.  Returns true when the
// ray is finished: its walk ended, an any-hit ray hit, or the step cap.
// kDeep: keep the reference's push guard (no push once 62 entries are on
// the stack); the wavefront trace clears it, since it only runs on trees of
// at most 28 levels, whose walks never hold more than 28 entries (0.8 ms of
// a 59 ms trace per export frame).  kUnordered is the exact build's.
template <bool kWide, bool kUnordered = false, bool kDeep = true, bool kPacked = false, class Scn>
DI bool dyn_step(const Scn& S, LaneRay& L, DynStack& stk, bool leaf_phase, Guard& g, int interior_steps = 1) {
    bool done = false;
    if (leaf_phase) {
        const int first = kPacked ? pk_start(L.leaf.ref) : L.leaf.ref;
        const int end = first + (kPacked ? pk_count(L.leaf.ref) : L.leaf.cnt);
        for (int i = first; i < end; ++i) {
            float t, u, v;
            if (thit(g, L.r, S.tri_isect, i, L.h.t, t, u, v) && t < L.h.t) {
                L.h.t = t;
                L.h.u = u;
                L.h.v = v;
                L.h.prim = i;
                if (L.any) {
                    done = true;
                    break;
                }
            }
        }
        if (kPacked)
            L.leaf.ref = 0;
        else
            L.leaf.cnt = 0;
    } else {
        int m = 0;
        for (; m < interior_steps && L.have_node; ++m) {
            if (is_leaf<kPacked>(L.node)) {
                if (parked_leaf<kPacked>(L)) break;   // blocked: a leaf is parked already
                L.leaf = L.node;
                L.have_node = kPacked ? pop_packed(stk, L.top, L.h.t, L.node) : pop_entry(stk, L.top, L.h.t, L.node);
            } else if (kWide) {
                // 4-wide node: hit children ordered by entry distance, the
                // nearest entered, the others pushed far to near
                const Node4* n4 = S.nodes4 + L.node.ref;
                const float4 lx = __ldg(&n4->lox), hx = __ldg(&n4->hix), ly = __ldg(&n4->loy);
                const float4 hy = __ldg(&n4->hiy), lz = __ldg(&n4->loz), hz = __ldg(&n4->hiz);
                const int4 cr = __ldg(&n4->ref), cc = __ldg(&n4->cnt);
                const float LX[4] = {lx.x, lx.y, lx.z, lx.w}, HX[4] = {hx.x, hx.y, hx.z, hx.w};
                const float LY[4] = {ly.x, ly.y, ly.z, ly.w}, HY[4] = {hy.x, hy.y, hy.z, hy.w};
                const float LZ[4] = {lz.x, lz.y, lz.z, lz.w}, HZ[4] = {hz.x, hz.y, hz.z, hz.w};
                const int CR[4] = {cr.x, cr.y, cr.z, cr.w}, CC[4] = {cc.x, cc.y, cc.z, cc.w};
                float t4[4];
                unsigned int key[4];
    #pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const bool hit = CC[k] >= 0 && tslab(g, L.r, LX[k], LY[k], LZ[k], HX[k], HY[k], HZ[k], t4[k]) &&
                                     !(t4[k] > L.h.t);
                    key[k] = hit ? ((__float_as_uint(fmaxf(t4[k], 0.0f)) & ~3u) | (unsigned int)k) : 0xffffffffu;
                }
                cswap(key[0], key[1]);
                cswap(key[2], key[3]);
                cswap(key[0], key[2]);
                cswap(key[1], key[3]);
                cswap(key[1], key[2]);
                if (key[0] == 0xffffffffu) {
                    L.have_node = pop_entry(stk, L.top, L.h.t, L.node);
                } else {
    #pragma unroll
                    for (int k = 3; k >= 1; --k) {
                        if (key[k] != 0xffffffffu) {
                            if (L.top < kDynStack) {
                                const int s = key[k] & 3u;
                                stk.e[L.top++] =
                                    make_int2(CR[s], (CC[s] & 0xffff) | (__float_as_int(t4[s]) & (int)0xffff0000));
                            } else {
                                g.flags |= RC_GUARD_TRAVERSAL_CAP;
                            }
                        }
                    }
                    const int s0 = key[0] & 3u;
                    L.node.ref = CR[s0];
                    L.node.cnt = CC[s0];
                }
            } else {
                const NodeRec* nrec = S.nodes + L.node.ref;
                const float4 a = __ldg(&nrec->a), b = __ldg(&nrec->b), c = __ldg(&nrec->c);
                const int4 d = __ldg(&nrec->d);
                float tl, tr;
                const bool hl = tslab_left(g, L.r, a, b, c, tl) && !(tl > L.h.t);
                const bool hr = tslab_right(g, L.r, a, b, c, tr) && !(tr > L.h.t);
                if (kPacked) {
                    // d = (left, right) packed references
                    if (hl && hr) {
                        const bool left_first = tl < tr;
                        if (!kDeep || L.top < 62)
                            stk.e[L.top++] = make_int2(left_first ? d.y : d.x, __float_as_int(left_first ? tr : tl));
                        L.node.ref = left_first ? d.x : d.y;
                    } else if (hl || hr) {
                        L.node.ref = hl ? d.x : d.y;
                    } else {
                        L.have_node = pop_packed(stk, L.top, L.h.t, L.node);
                    }
                } else if (hl && hr) {
                    const bool left_first = tl < tr;
                    if (!kDeep || L.top < 62) {
                        const float tf = left_first ? tr : tl;
                        const int cf = left_first ? d.w : d.y;
                        stk.e[L.top++] =
                            make_int2(left_first ? d.z : d.x, (cf & 0xffff) | (__float_as_int(tf) & (int)0xffff0000));
                    }
                    L.node.ref = left_first ? d.x : d.z;
                    L.node.cnt = left_first ? d.y : d.w;
                } else if (hl) {
                    L.node.ref = d.x;
                    L.node.cnt = d.y;
                } else if (hr) {
                    L.node.ref = d.z;
                    L.node.cnt = d.w;
                } else {
                    L.have_node = pop_entry(stk, L.top, L.h.t, L.node);
                }
            }
        }
        L.steps += m;
    }
    if (!L.have_node && !parked_leaf<kPacked>(L)) done = true;
    if (++L.steps > 4 * S.node_count + 64) {
        g.flags |= RC_GUARD_TRAVERSAL_CAP;
        done = true;
    }
    return done;
}

#else
// Exact build: one step of L with trace_closest's order for closest-hit
// lanes (see the file comment); shadow lanes park and walk on.
// kUnordered: trace_unordered's order instead (the photon walks,
// photon_trace.comp:102-128): the left child first whatever the distances,
// and a node met with 62 or more entries on the stack has neither child
// tested nor visited.
// kDeep as in the fast build (the closest-hit walk's guard; the unordered
// walk keeps its own).
template <bool kWide, bool kUnordered = false, bool kDeep = true, bool kPacked = false, class Scn>
DI bool dyn_step(const Scn& S, LaneRay& L, DynStack& stk, bool leaf_phase, Guard& g, int interior_steps = 1) {
    bool done = false;
    if (leaf_phase) {
        const int first = kPacked ? pk_start(L.leaf.ref) : L.leaf.ref;
        const int end = first + (kPacked ? pk_count(L.leaf.ref) : L.leaf.cnt);
        for (int i = first; i < end; ++i) {
            float t, u, v;
            if (thit(g, L.r, S.tri_isect, i, L.h.t, t, u, v) && t < L.h.t) {
                L.h.t = t;
                L.h.u = u;
                L.h.v = v;
                L.h.prim = i;
                if (L.any) {
                    done = true;
                    break;
                }
            }
        }
        if (kPacked)
            L.leaf.ref = 0;
        else
            L.leaf.cnt = 0;
    } else {
        int m = 0;
        for (; m < interior_steps; ++m) {
            if (!L.have_node) {
                // a closest-hit lane pops only after its parked leaf was
                // tested, against the distance that leaf may have lowered
                if (parked_leaf<kPacked>(L) || L.top == 0) break;
                L.have_node = kPacked ? pop_packed(stk, L.top, L.h.t, L.node) : pop_entry(stk, L.top, L.h.t, L.node);
                if (!L.have_node) break;
            }
            if (is_leaf<kPacked>(L.node)) {
                if (parked_leaf<kPacked>(L)) break;   // blocked: a leaf is parked already
                L.leaf = L.node;
                if (L.any) {
                    L.have_node =
                        kPacked ? pop_packed(stk, L.top, L.h.t, L.node) : pop_entry(stk, L.top, L.h.t, L.node);
                } else {
                    L.have_node = false;
                    break;
                }
            } else if (kUnordered && L.top >= 62) {
                L.have_node = false;
            } else {
                const NodeRec* nrec = S.nodes + L.node.ref;
                const float4 a = __ldg(&nrec->a), b = __ldg(&nrec->b), c = __ldg(&nrec->c);
                const int4 d = __ldg(&nrec->d);
                float tl, tr;
                // a child whose entry lies past the current hit is the one
                // the reference's walk would push and then drop when popping it
                const bool hl = tslab_left(g, L.r, a, b, c, tl) && !(tl > L.h.t);
                const bool hr = tslab_right(g, L.r, a, b, c, tr) && !(tr > L.h.t);
                if (kPacked) {
                    // d = (left, right) packed references; the entry
                    // distance rides in the stack entry
                    if (hl && hr) {
                        const bool left_first = kUnordered || tl < tr;
                        if (kUnordered || !kDeep || L.top < 62)
                            stk.e[L.top++] = make_int2(left_first ? d.y : d.x, __float_as_int(left_first ? tr : tl));
                        L.node.ref = left_first ? d.x : d.y;
                    } else if (hl || hr) {
                        L.node.ref = hl ? d.x : d.y;
                    } else {
                        L.have_node = false;
                    }
                } else if (hl && hr) {
                    const bool left_first = kUnordered || tl < tr;
                    if (kUnordered || !kDeep || L.top < 62) {
                        stk.e[L.top] = left_first ? make_int2(d.z, d.w) : make_int2(d.x, d.y);
                        stk.t[L.top++] = left_first ? tr : tl;
                    }
                    L.node.ref = left_first ? d.x : d.z;
                    L.node.cnt = left_first ? d.y : d.w;
                } else if (hl) {
                    L.node.ref = d.x;
                    L.node.cnt = d.y;
                } else if (hr) {
                    L.node.ref = d.z;
                    L.node.cnt = d.w;
                } else {
                    L.have_node = false;
                }
            }
        }
        L.steps += m;
    }
    if (!L.have_node && !parked_leaf<kPacked>(L) && L.top == 0) done = true;
    if (++L.steps > 4 * S.node_count + 64) {
        g.flags |= RC_GUARD_TRAVERSAL_CAP;
        done = true;
    }
    return done;
}
#endif

}  // namespace RC_NS
}  // namespace rc

#endif
