// dyn_trace.cuh -- the per-lane traversal state machine of the fast build's
// refill kernels (camera / shadow rays in wavefront.cu, photon segments in
// kernels.cu).
//
// A lane owns one ray at a time and advances it one step per loop iteration
// of its warp: an interior node, parking a reached leaf, or the triangles of
// a parked leaf.  Leaf tests and interior steps never share an iteration:
// the warp tests leaves (every lane with one parked, together) once all busy
// lanes have one parked or `leaf_quarters` quarters of them are blocked (a
// leaf parked and no interior node to go on with); otherwise the unblocked
// lanes take interior steps.  A kernel refills lanes whose ray finished from
// its own work list when fewer than `refill_lanes` lanes are busy, so a warp
// is not held by its slowest ray.  The rays, the visit order of each ray and
// the hits are the plain traversal's; only the schedule differs.
#ifndef RC_DYN_TRACE_CUH
#define RC_DYN_TRACE_CUH

#include "device_common.cuh"

#if !RC_EXACT
namespace rc {
namespace RC_NS {

// Stack entries: the binary walk pushes at most one per level (guarded at
// 62, as the reference), the 4-wide walk up to three.
constexpr int kDynStack = 96;

// Pops the next stack entry not culled by the current hit distance.  An
// entry is 8 bytes: (ref, count | entry distance truncated to its top 16
// bits); truncation rounds a positive distance down, so the cull `t > hit`
// never drops a needed entry.
DI bool pop_packed(const int2* stk, int& top, float cull, TravNode& n) {
    while (top > 0) {
        const int2 e = stk[--top];
        if (__int_as_float(e.y & (int)0xffff0000) > cull) continue;
        n.ref = e.x;
        n.cnt = e.y & 0xffff;
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
    int steps;
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
    L.node.ref = S.root_ref;
    L.node.cnt = S.root_count;
    L.steps = 0;
    float tmin;
    L.have_node = S.tri_count > 0 &&
                  tslab(g, L.r, S.root_min[0], S.root_min[1], S.root_min[2], S.root_max[0], S.root_max[1],
                        S.root_max[2], tmin) &&
                  !(tmin > L.h.t);
}

// The warp's choice for this iteration; every lane of the warp calls it with
// the warp's busy mask `act` (the caller's ballot of `busy`).  Returns
// whether this lane steps, and the phase.
DI bool dyn_schedule(const LaneRay& L, bool busy, unsigned int act, int leaf_quarters, bool& leaf_phase) {
    const unsigned int FULL = 0xffffffffu;
    const bool blocked = busy && L.leaf.cnt > 0 && (!L.have_node || L.node.cnt > 0);
    const unsigned int parked = __ballot_sync(FULL, busy && L.leaf.cnt > 0);
    const unsigned int blk = __ballot_sync(FULL, blocked);
    leaf_phase = parked == act || 4 * __popc(blk) >= leaf_quarters * __popc(act);
    return busy && (leaf_phase ? L.leaf.cnt > 0 : !blocked);
}

// One step of L (kWide: interior nodes from S.nodes4): in the leaf phase the
// parked leaf's triangles; otherwise up to `interior_steps` moves through
// the tree -- interior nodes, or parking a reached leaf -- while the lane is
// not blocked (a leaf parked and the next node a leaf too, or none), so the
// warp's scheduling work is shared by several moves.  Returns true when the
// ray is finished: its walk ended, an any-hit ray hit, or the step cap.
template <bool kWide, class Scn>
DI bool dyn_step(const Scn& S, LaneRay& L, int2* stk, bool leaf_phase, Guard& g, int interior_steps = 1) {
    bool done = false;
    if (leaf_phase) {
        for (int i = L.leaf.ref; i < L.leaf.ref + L.leaf.cnt; ++i) {
            float t, u, v;
            if (thit(g, L.r, S.tri_isect, i, t, u, v) && t < L.h.t) {
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
        L.leaf.cnt = 0;
    } else {
        for (int m = 0; m < interior_steps && L.have_node; ++m) {
            if (L.node.cnt > 0) {
                if (L.leaf.cnt > 0) break;   // blocked: a leaf is parked already
                L.leaf = L.node;
                L.have_node = pop_packed(stk, L.top, L.h.t, L.node);
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
                    L.have_node = pop_packed(stk, L.top, L.h.t, L.node);
                } else {
    #pragma unroll
                    for (int k = 3; k >= 1; --k) {
                        if (key[k] != 0xffffffffu) {
                            if (L.top < kDynStack) {
                                const int s = key[k] & 3u;
                                stk[L.top++] =
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
                const bool hl = tslab(g, L.r, a.x, a.y, a.z, a.w, b.x, b.y, tl) && !(tl > L.h.t);
                const bool hr = tslab(g, L.r, b.z, b.w, c.x, c.y, c.z, c.w, tr) && !(tr > L.h.t);
                if (hl && hr) {
                    const bool left_first = tl < tr;
                    if (L.top < 62) {
                        const float tf = left_first ? tr : tl;
                        const int cf = left_first ? d.w : d.y;
                        stk[L.top++] =
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
                    L.have_node = pop_packed(stk, L.top, L.h.t, L.node);
                }
            }
            if (m + 1 < interior_steps && ++L.steps > 4 * S.node_count + 64) break;
        }
    }
    if (!L.have_node && L.leaf.cnt == 0) done = true;
    if (++L.steps > 4 * S.node_count + 64) {
        g.flags |= RC_GUARD_TRAVERSAL_CAP;
        done = true;
    }
    return done;
}

}  // namespace RC_NS
}  // namespace rc
#endif  // !RC_EXACT

#endif
