// device_common.cuh -- device functions shared by the megakernel
// (kernels.cu) and the wavefront kernels (wavefront.cu): scalar math of the
// build's mode, float3 helpers, PCG, intersection, the three traversals,
// materials and sampling.  Each includer is compiled twice (RC_EXACT 0/1),
// and everything here lands in namespace rc::exact or rc::fast.
#ifndef RC_DEVICE_COMMON_CUH
#define RC_DEVICE_COMMON_CUH

#include <cuda_fp16.h>
#include <stdint.h>

#include "device_scene.h"
#include "rc_exact_math.h"
#include "retrocam.h"

#ifndef RC_EXACT
#error "RC_EXACT must be 0 or 1"
#endif

#if RC_EXACT
#define RC_NS exact
#else
#define RC_NS fast
#endif

namespace rc {
namespace RC_NS {

#define DI __device__ __forceinline__

// ---------------------------------------------------------------------------
// scalar math of the chosen mode
// ---------------------------------------------------------------------------
#if RC_EXACT
DI float gmin(float x, float y) { return (y < x) ? y : x; }
DI float gmax(float x, float y) { return (x < y) ? y : x; }
DI void sincos_(float x, float* s, float* c) { *s = rcx_sinf(x); *c = rcx_cosf(x); }
DI float pow5(float x) { return rcx_powf(x, 5.0f); }
DI float powf_(float x, float y) { return rcx_powf(x, y); }
DI float expf_(float x) { return rcx_expf(x); }
DI float logf_(float x) { return rcx_logf(x); }
#else
DI float gmin(float x, float y) { return fminf(x, y); }
DI float gmax(float x, float y) { return fmaxf(x, y); }
DI void sincos_(float x, float* s, float* c) {
    // The arguments here lie in [0, 2*pi]; fold to [-pi, pi] where the SFU
    // approximation is specified.
    const float PI_F = 3.14159265358979f;
    if (x > PI_F) x -= 2.0f * PI_F;
    __sincosf(x, s, c);
}
DI float pow5(float x) { const float x2 = x * x; return x2 * x2 * x; }
DI float powf_(float x, float y) { return x <= 0.0f ? (y == 0.0f ? 1.0f : 0.0f) : exp2f(y * __log2f(x)); }
DI float expf_(float x) { return __expf(x); }
DI float logf_(float x) { return __logf(x); }
#endif
DI float gclamp(float x, float a, float b) { return gmin(gmax(x, a), b); }
DI float fabs_(float x) { return __uint_as_float(__float_as_uint(x) & 0x7fffffffu); }
DI bool bad(float x) { return (__float_as_uint(x) & 0x7f800000u) == 0x7f800000u; }

// ---------------------------------------------------------------------------
// float3 helpers
// ---------------------------------------------------------------------------
DI float3 f3(float a, float b, float c) { return make_float3(a, b, c); }
DI float3 operator+(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
DI float3 operator-(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
DI float3 operator*(float3 a, float3 b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
DI float3 operator*(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
DI float3 operator*(float s, float3 a) { return f3(s * a.x, s * a.y, s * a.z); }
DI float3 operator/(float3 a, float s) { return f3(a.x / s, a.y / s, a.z / s); }
DI float3 operator/(float3 a, float3 b) { return f3(a.x / b.x, a.y / b.y, a.z / b.z); }
DI float3 operator-(float3 a) { return f3(-a.x, -a.y, -a.z); }
DI float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
DI float3 cross(float3 a, float3 b) {
    return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
DI float3 vmin(float3 a, float3 b) { return f3(gmin(a.x, b.x), gmin(a.y, b.y), gmin(a.z, b.z)); }
DI float3 vmax(float3 a, float3 b) { return f3(gmax(a.x, b.x), gmax(a.y, b.y), gmax(a.z, b.z)); }
#if RC_EXACT
DI float3 normalize(float3 v) { return v / sqrtf(dot(v, v)); }
#else
DI float3 normalize(float3 v) { return v * rsqrtf(dot(v, v)); }
#endif
DI float3 reflect(float3 I, float3 N) { return I - (2.0f * dot(N, I)) * N; }
DI float3 refract(float3 I, float3 N, float eta) {
    const float d = dot(N, I);
    const float k = 1.0f - eta * eta * (1.0f - d * d);
    if (k < 0.0f) return f3(0.0f, 0.0f, 0.0f);
    return eta * I - (eta * d + sqrtf(k)) * N;
}
DI float3 xyz(float4 v) { return f3(v.x, v.y, v.z); }
DI float luma709(float3 c) { return dot(c, f3(0.2126f, 0.7152f, 0.0722f)); }

// ---------------------------------------------------------------------------
// RNG (pathtrace.comp:80-98, photon_trace.comp:60-72)
// ---------------------------------------------------------------------------
DI uint32_t pcg(uint32_t& s) {
    s = s * 747796405u + 2891336453u;
    const uint32_t w = ((s >> ((s >> 28u) + 4u)) ^ s) * 277803737u;
    return (w >> 22u) ^ w;
}
DI float rnd(uint32_t& s) { return (float)pcg(s) / 4294967296.0f; }
DI uint32_t init_seed(int px, int py, int frame) {
    uint32_t s = (uint32_t)px + (uint32_t)py * 7919u + (uint32_t)frame * 6271u;
    pcg(s);
    pcg(s);
    return s;
}
DI uint32_t photon_seed(uint32_t idx, int seed) {
    uint32_t s = idx * 1664525u + (uint32_t)seed * 1013904223u + 2531011u;
    pcg(s);
    pcg(s);
    return s;
}
DI int cell_hash(int cx, int cy, int cz, int hash_size) {
    const uint32_t h = ((uint32_t)cx * 73856093u) ^ ((uint32_t)cy * 19349663u) ^ ((uint32_t)cz * 83492791u);
    return (int)(h & (uint32_t)(hash_size - 1));
}

// ---------------------------------------------------------------------------
// intersection (pathtrace.comp:102-130)
// ---------------------------------------------------------------------------
struct Ray {
    float3 o, d;
#if RC_EXACT
    float3 inv;
#else
    // 1/d and -o/d for the FMA form of the slab test, x and y side by side
    // so that one paired FMA (__ffma2_rn) covers both axes
    float2 ixy, nxy;
    float iz, nz;
#endif
};

DI Ray make_ray(float3 o, float3 d) {
    Ray r;
    r.o = o;
    r.d = d;
#if RC_EXACT
    r.inv = f3(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
#else
    r.ixy = make_float2(1.0f / d.x, 1.0f / d.y);
    r.iz = 1.0f / d.z;
    r.nxy = make_float2(-(o.x * r.ixy.x), -(o.y * r.ixy.y));
    r.nz = -(o.z * r.iz);
#endif
    return r;
}

// The slab test from the six plane distances (pathtrace.comp:102-110).
DI bool slab_from(float t0x, float t0y, float t0z, float t1x, float t1y, float t1z, float& tmin) {
    const float lox = gmin(t0x, t1x), loy = gmin(t0y, t1y), loz = gmin(t0z, t1z);
    const float hix = gmax(t0x, t1x), hiy = gmax(t0y, t1y), hiz = gmax(t0z, t1z);
    tmin = gmax(gmax(lox, loy), loz);
    const float tmax = gmin(gmin(hix, hiy), hiz);
    return tmax >= gmax(tmin, 0.0f);
}

DI bool slab(const Ray& r, float nx, float ny, float nz, float xx, float xy, float xz, float& tmin) {
#if RC_EXACT
    const float t0x = (nx - r.o.x) * r.inv.x, t0y = (ny - r.o.y) * r.inv.y, t0z = (nz - r.o.z) * r.inv.z;
    const float t1x = (xx - r.o.x) * r.inv.x, t1y = (xy - r.o.y) * r.inv.y, t1z = (xz - r.o.z) * r.inv.z;
#else
    const float t0x = fmaf(nx, r.ixy.x, r.nxy.x), t0y = fmaf(ny, r.ixy.y, r.nxy.y), t0z = fmaf(nz, r.iz, r.nz);
    const float t1x = fmaf(xx, r.ixy.x, r.nxy.x), t1y = fmaf(xy, r.ixy.y, r.nxy.y), t1z = fmaf(xz, r.iz, r.nz);
#endif
    return slab_from(t0x, t0y, t0z, t1x, t1y, t1z, tmin);
}

// A box given as (min x, min y), min z, (max x, max y), max z.  The fast
// build forms the x and y plane distances with one paired FMA per corner
// (each lane rounded as fmaf rounds it: the same distances as slab()).
DI bool slab_xy(const Ray& r, float2 lo, float loz, float2 hi, float hiz, float& tmin) {
#if RC_EXACT
    return slab(r, lo.x, lo.y, loz, hi.x, hi.y, hiz, tmin);
#else
    const float2 t0 = __ffma2_rn(lo, r.ixy, r.nxy);
    const float2 t1 = __ffma2_rn(hi, r.ixy, r.nxy);
    return slab_from(t0.x, t0.y, fmaf(loz, r.iz, r.nz), t1.x, t1.y, fmaf(hiz, r.iz, r.nz), tmin);
#endif
}

#if !RC_EXACT
// Fast build: Moller-Trumbore with the triangle's normal n = e1 x e2 from the
// record's w components.  The same determinant and barycentrics as scalar
// triple products -- a = -d.n, t = f s.n, u = f e2.(s x d), v = -f e1.(s x d)
// -- so one cross product instead of two, and the distance first: a
// triangle at or beyond `tmax` (the caller's current hit) is refused before
// its barycentrics.  Accepts what the reference's test accepts, up to
// rounding.
DI bool hit_triangle(const Ray& r, const float4* __restrict__ tri_isect, int i, float tmax, float& t, float& u,
                     float& v) {
    const float4 A = __ldg(tri_isect + 3 * i + 0);
    const float4 B = __ldg(tri_isect + 3 * i + 1);
    const float4 Cc = __ldg(tri_isect + 3 * i + 2);
    const float3 v0 = xyz(A), e1 = xyz(B), e2 = xyz(Cc), n = f3(A.w, B.w, Cc.w);
    const float a = -dot(r.d, n);
    if (fabs_(a) < 1e-8f) return false;
    const float f = 1.0f / a;
    const float3 s = r.o - v0;
    const float tt = f * dot(s, n);
    if (tt < 1e-4f || !(tt < tmax)) return false;
    const float3 c = cross(s, r.d);
    const float uu = f * dot(e2, c);
    if (uu < 0.0f || uu > 1.0f) return false;
    const float vv = -f * dot(e1, c);
    if (vv < 0.0f || uu + vv > 1.0f) return false;
    t = tt;
    u = uu;
    v = vv;
    return true;
}
#else
// pathtrace.comp's Moller-Trumbore, operation for operation (tmax unused:
// the caller compares the distance).
DI bool hit_triangle(const Ray& r, const float4* __restrict__ tri_isect, int i, float tmax, float& t, float& u,
                     float& v) {
    const float4 A = __ldg(tri_isect + 3 * i + 0);
    const float4 B = __ldg(tri_isect + 3 * i + 1);
    const float4 Cc = __ldg(tri_isect + 3 * i + 2);
    const float3 v0 = xyz(A), e1 = xyz(B), e2 = xyz(Cc);
    const float3 h = cross(r.d, e2);
    const float a = dot(e1, h);
    if (fabs_(a) < 1e-8f) return false;
    const float f = 1.0f / a;
    const float3 s = r.o - v0;
    const float uu = f * dot(s, h);
    if (uu < 0.0f || uu > 1.0f) return false;
    const float3 q = cross(s, e1);
    const float vv = f * dot(r.d, q);
    if (vv < 0.0f || uu + vv > 1.0f) return false;
    const float tt = f * dot(e2, q);
    if (tt < 1e-4f) return false;
    t = tt;
    u = uu;
    v = vv;
    return true;
}
#endif

struct Hit {
    float t, u, v;
    int prim;
};

struct Surf {
    float3 pos, normal;
    int mat;
};

// Position, interpolated normal and material of an accepted hit, computed
// as the reference computes them at acceptance (pathtrace.comp:166-172).
DI Surf surface(const DeviceScene& S, const Ray& r, const Hit& h) {
    Surf s;
    s.pos = r.o + r.d * h.t;
    const float4 n0 = __ldg(S.tri_shade + 3 * h.prim + 0);
    const float4 n1 = __ldg(S.tri_shade + 3 * h.prim + 1);
    const float4 n2 = __ldg(S.tri_shade + 3 * h.prim + 2);
    const float w = 1.0f - h.u - h.v;
    s.normal = normalize(xyz(n0) * w + xyz(n1) * h.u + xyz(n2) * h.v);
    s.mat = __float_as_int(n0.w);
    return s;
}

// Per-thread guard flags and work counts (ray-box and ray-triangle tests),
// flushed once per warp at the end of a kernel.
struct Guard {
    unsigned int flags;
    unsigned int nodes;
    unsigned int tris;
};

DI bool tslab(Guard& g, const Ray& r, float nx, float ny, float nz, float xx, float xy, float xz, float& tmin) {
    ++g.nodes;
    return slab(r, nx, ny, nz, xx, xy, xz, tmin);
}

// The two child boxes of a node record (NodeRec: a = left (min x, min y,
// max x, max y), b = the same for the right child, c = (left min z, left
// max z, right min z, right max z)).
DI bool tslab_left(Guard& g, const Ray& r, const float4& a, const float4& b, const float4& c, float& tmin) {
    ++g.nodes;
    return slab_xy(r, make_float2(a.x, a.y), c.x, make_float2(a.z, a.w), c.y, tmin);
}
DI bool tslab_right(Guard& g, const Ray& r, const float4& a, const float4& b, const float4& c, float& tmin) {
    ++g.nodes;
    return slab_xy(r, make_float2(b.x, b.y), c.z, make_float2(b.z, b.w), c.w, tmin);
}

// The root box test; a scene without triangles has no root to enter.
DI bool enter_root(const DeviceScene& S, Guard& g, const Ray& r, float& tmin) {
    return S.tri_count > 0 &&
           tslab(g, r, S.root_min[0], S.root_min[1], S.root_min[2], S.root_max[0], S.root_max[1], S.root_max[2], tmin);
}

// tmax: the caller's current hit distance (or shadow length), which it
// compares the returned distance against; the fast test may stop early.
DI bool thit(Guard& g, const Ray& r, const float4* __restrict__ tri_isect, int i, float tmax, float& t, float& u,
             float& v) {
    ++g.tris;
    return hit_triangle(r, tri_isect, i, tmax, t, u, v);
}

// A node to visit: cnt > 0 a leaf with primitives [ref, ref+cnt), else the
// interior node `ref`.
struct TravNode {
    int ref, cnt;
};

// Closest hit, near child first (pathtrace.comp:142-203).  A stack entry
// holds the child's (ref, count) and the entry distance the parent computed;
// the reference re-tests the same box with the same ray on pop, which gives
// the same answer, so only the aabbT > rec.t cull is repeated.
DI Hit trace_closest(const DeviceScene& S, const Ray& r, Guard& g) {
    Hit h;
    h.t = 1e30f;
    h.prim = -1;
    h.u = h.v = 0.0f;
    float tmin;
    if (!enter_root(S, g, r, tmin))
        return h;
    if (tmin > h.t) return h;
    int2 stk[64];
    float stt[64];
    int top = 0;
    int ref = S.root_ref, cnt = S.root_count;
    int pops = 0;
    while (true) {
        if (cnt > 0) {
            for (int i = ref; i < ref + cnt; ++i) {
                float t, u, v;
                if (thit(g, r, S.tri_isect, i, h.t, t, u, v) && t < h.t) {
                    h.t = t;
                    h.u = u;
                    h.v = v;
                    h.prim = i;
                }
            }
        } else if (top < 62) {
            const NodeRec* nr = S.nodes + ref;
            const float4 a = __ldg(&nr->a), b = __ldg(&nr->b), c = __ldg(&nr->c);
            const int4 d = __ldg(&nr->d);
            float tl, tr;
            const bool hl = tslab_left(g, r, a, b, c, tl);
            const bool hr = tslab_right(g, r, a, b, c, tr);
            if (hl && hr) {
                if (tl < tr) {
                    stk[top] = make_int2(d.z, d.w); stt[top++] = tr;
                    stk[top] = make_int2(d.x, d.y); stt[top++] = tl;
                } else {
                    stk[top] = make_int2(d.x, d.y); stt[top++] = tl;
                    stk[top] = make_int2(d.z, d.w); stt[top++] = tr;
                }
            } else if (hl) {
                stk[top] = make_int2(d.x, d.y); stt[top++] = tl;
            } else if (hr) {
                stk[top] = make_int2(d.z, d.w); stt[top++] = tr;
            }
        }
        // pop the next entry that survives the aabbT > rec.t cull
        bool found = false;
        while (top > 0) {
            --top;
            if (stt[top] > h.t) continue;
            ref = stk[top].x;
            cnt = stk[top].y;
            found = true;
            break;
        }
        if (!found) break;
        if (++pops > S.node_count) { g.flags |= RC_GUARD_TRAVERSAL_CAP; break; }
    }
    return h;
}

// Closest hit with the photon passes' order: children pushed right then
// left with no ordering (photon_trace.comp:102-128, photon_gather.comp).
// kTestAtParent: test both child boxes at the parent and push only hits
// (identical results whenever the reference's 64-entry stack cannot
// overflow, i.e. BVH depth <= 60); otherwise the reference's own policy:
// push untested children and test each box when it is popped.
template <bool kTestAtParent>
DI Hit trace_unordered(const DeviceScene& S, const Ray& r, Guard& g) {
    Hit h;
    h.t = 1e30f;
    h.prim = -1;
    h.u = h.v = 0.0f;
    float tmin;
    if (!enter_root(S, g, r, tmin))
        return h;
    if (tmin > h.t) return h;
    int2 stk[64];
    float stt[64];
    int top = 0;
    int ref = S.root_ref, cnt = S.root_count;
    int pops = 0;
    while (true) {
        if (cnt > 0) {
            for (int i = ref; i < ref + cnt; ++i) {
                float t, u, v;
                if (thit(g, r, S.tri_isect, i, h.t, t, u, v) && t < h.t) {
                    h.t = t;
                    h.u = u;
                    h.v = v;
                    h.prim = i;
                }
            }
        } else if (top < 62) {
            if (kTestAtParent) {
                const NodeRec* nr = S.nodes + ref;
                const float4 a = __ldg(&nr->a), b = __ldg(&nr->b), c = __ldg(&nr->c);
                const int4 d = __ldg(&nr->d);
                float tl, tr;
                const bool hl = tslab_left(g, r, a, b, c, tl);
                const bool hr = tslab_right(g, r, a, b, c, tr);
                if (hr) { stk[top] = make_int2(d.z, d.w); stt[top++] = tr; }
                if (hl) { stk[top] = make_int2(d.x, d.y); stt[top++] = tl; }
            } else {
                // (parent node, side) of each untested child
                stk[top++] = make_int2(ref, 1);
                stk[top++] = make_int2(ref, 0);
            }
        }
        bool found = false;
        while (top > 0) {
            --top;
            if (kTestAtParent) {
                if (stt[top] > h.t) continue;
                ref = stk[top].x;
                cnt = stk[top].y;
            } else {
                const NodeRec* nr = S.nodes + stk[top].x;
                const float4 a = __ldg(&nr->a), b = __ldg(&nr->b), c = __ldg(&nr->c);
                const int4 d = __ldg(&nr->d);
                float tc;
                const bool right = stk[top].y != 0;
                const bool hit = right ? tslab_right(g, r, a, b, c, tc)
                                       : tslab_left(g, r, a, b, c, tc);
                if (!hit || tc > h.t) continue;
                ref = right ? d.z : d.x;
                cnt = right ? d.w : d.y;
            }
            found = true;
            break;
        }
        if (!found) break;
        if (++pops > 2 * S.node_count) { g.flags |= RC_GUARD_TRAVERSAL_CAP; break; }
    }
    return h;
}

// Any hit closer than max_dist (pathtrace.comp:211-242); true = unoccluded.
// Same two policies as above; test-at-parent is exact for BVH depth <= 28
// (the reference's 32-entry stack cannot overflow) because the answer is a
// yes/no that does not depend on visiting order.
template <bool kTestAtParent>
DI bool trace_shadow(const DeviceScene& S, const Ray& r, float max_dist, Guard& g) {
    float tmin;
    if (!enter_root(S, g, r, tmin))
        return true;
    if (tmin > max_dist) return true;
    int2 stk[32];
    int top = 0;
    int ref = S.root_ref, cnt = S.root_count;
    int pops = 0;
    while (true) {
        if (cnt > 0) {
            for (int i = ref; i < ref + cnt; ++i) {
                float t, u, v;
                if (thit(g, r, S.tri_isect, i, max_dist, t, u, v) && t < max_dist) return false;
            }
        } else if (top < 30) {
            if (kTestAtParent) {
                const NodeRec* nr = S.nodes + ref;
                const float4 a = __ldg(&nr->a), b = __ldg(&nr->b), c = __ldg(&nr->c);
                const int4 d = __ldg(&nr->d);
                float tl, tr;
                const bool hl = tslab_left(g, r, a, b, c, tl) && !(tl > max_dist);
                const bool hr = tslab_right(g, r, a, b, c, tr) && !(tr > max_dist);
                if (hr) stk[top++] = make_int2(d.z, d.w);
                if (hl) stk[top++] = make_int2(d.x, d.y);
            } else {
                stk[top++] = make_int2(ref, 1);
                stk[top++] = make_int2(ref, 0);
            }
        }
        bool found = false;
        while (top > 0) {
            --top;
            if (kTestAtParent) {
                ref = stk[top].x;
                cnt = stk[top].y;
            } else {
                const NodeRec* nr = S.nodes + stk[top].x;
                const float4 a = __ldg(&nr->a), b = __ldg(&nr->b), c = __ldg(&nr->c);
                const int4 d = __ldg(&nr->d);
                float tc;
                const bool right = stk[top].y != 0;
                const bool hit = right ? tslab_right(g, r, a, b, c, tc)
                                       : tslab_left(g, r, a, b, c, tc);
                if (!hit || tc > max_dist) continue;
                ref = right ? d.z : d.x;
                cnt = right ? d.w : d.y;
            }
            found = true;
            break;
        }
        if (!found) break;
        if (++pops > 2 * S.node_count) { g.flags |= RC_GUARD_TRAVERSAL_CAP; break; }
    }
    return true;
}

#if !RC_EXACT
// Fast-build traversals.  Interior steps and triangle tests run in separate
// loops; a lane that reaches a leaf parks it and keeps descending until every
// lane of the warp still descending holds a parked leaf, then the warp tests
// triangles together, so interior and leaf work are not interleaved lane by
// lane.  The nearer hit child is entered directly and only the farther one is
// pushed.  The closest hit equals trace_closest's except where two triangles
// tie exactly; the shadow answer is the same yes/no.

DI bool pop_entry(const int2* stk, const float* stt, int& top, float cull, TravNode& n) {
    while (top > 0) {
        --top;
        if (stt[top] > cull) continue;
        n.ref = stk[top].x;
        n.cnt = stk[top].y;
        return true;
    }
    return false;
}

template <bool kAnyHit>
DI bool traverse_ww(const DeviceScene& S, const Ray& r, float max_t, Guard& g, Hit& h) {
    h.t = max_t;
    h.prim = -1;
    h.u = h.v = 0.0f;
    float tmin;
    if (!enter_root(S, g, r, tmin) ||
        tmin > h.t)
        return false;
    int2 stk[64];
    float stt[64];
    int top = 0;
    TravNode node = {S.root_ref, S.root_count};
    bool have_node = true;
    TravNode leaf = {0, 0};
    int steps = 0;
    while (have_node || leaf.cnt > 0) {
        while (have_node) {
            if (node.cnt > 0) {
                if (leaf.cnt > 0) break;  // already parked one: test it first
                leaf = node;
                have_node = pop_entry(stk, stt, top, h.t, node);
            } else {
                const NodeRec* nr = S.nodes + node.ref;
                const float4 a = __ldg(&nr->a), b = __ldg(&nr->b), c = __ldg(&nr->c);
                const int4 d = __ldg(&nr->d);
                float tl, tr;
                const bool hl = tslab_left(g, r, a, b, c, tl) && !(tl > h.t);
                const bool hr = tslab_right(g, r, a, b, c, tr) && !(tr > h.t);
                if (hl && hr) {
                    const bool left_first = tl < tr;
                    if (top < 62) {
                        stk[top] = left_first ? make_int2(d.z, d.w) : make_int2(d.x, d.y);
                        stt[top++] = left_first ? tr : tl;
                    }
                    node.ref = left_first ? d.x : d.z;
                    node.cnt = left_first ? d.y : d.w;
                } else if (hl) {
                    node.ref = d.x;
                    node.cnt = d.y;
                } else if (hr) {
                    node.ref = d.z;
                    node.cnt = d.w;
                } else {
                    have_node = pop_entry(stk, stt, top, h.t, node);
                }
            }
            if (++steps > 2 * S.node_count) {
                g.flags |= RC_GUARD_TRAVERSAL_CAP;
                return h.prim >= 0;
            }
            if (__all_sync(__activemask(), leaf.cnt > 0)) break;
        }
        if (leaf.cnt > 0) {
            for (int i = leaf.ref; i < leaf.ref + leaf.cnt; ++i) {
                float t, u, v;
                if (thit(g, r, S.tri_isect, i, h.t, t, u, v) && t < h.t) {
                    if (kAnyHit) return true;
                    h.t = t;
                    h.u = u;
                    h.v = v;
                    h.prim = i;
                }
            }
            leaf.cnt = 0;
        }
    }
    return h.prim >= 0;
}

DI void cswap(unsigned int& a, unsigned int& b) {
    const unsigned int lo = min(a, b), hi = max(a, b);
    a = lo;
    b = hi;
}

// 4-wide traversal over Node4 (same leaf parking as traverse_ww).  The hit
// children of a node are ordered by entry distance with a 5-comparator
// network on keys (distance bits with the slot in the low two bits; misses
// and empty slots, count < 0, sort last); the nearest is entered and the rest
// pushed far to near.  Up to three pushes per level: the stack holds 96
// entries, and a push that would overflow it raises RC_GUARD_TRAVERSAL_CAP.
constexpr int kStack4 = 96;

template <bool kAnyHit>
DI bool traverse4(const DeviceScene& S, const Ray& r, float max_t, Guard& g, Hit& h) {
    h.t = max_t;
    h.prim = -1;
    h.u = h.v = 0.0f;
    float tmin;
    if (!enter_root(S, g, r, tmin) ||
        tmin > h.t)
        return false;
    int2 stk[kStack4];
    float stt[kStack4];
    int top = 0;
    TravNode node = {S.root_count > 0 ? S.root_ref : 0, S.root_count};
    bool have_node = true;
    TravNode leaf = {0, 0};
    int steps = 0;
    while (have_node || leaf.cnt > 0) {
        while (have_node) {
            if (node.cnt > 0) {
                if (leaf.cnt > 0) break;
                leaf = node;
                have_node = pop_entry(stk, stt, top, h.t, node);
            } else {
                const Node4* n4 = S.nodes4 + node.ref;
                const float4 lx = __ldg(&n4->lox), hx = __ldg(&n4->hix), ly = __ldg(&n4->loy);
                const float4 hy = __ldg(&n4->hiy), lz = __ldg(&n4->loz), hz = __ldg(&n4->hiz);
                const int4 cr = __ldg(&n4->ref), cc = __ldg(&n4->cnt);
                float t[4];
                unsigned int key[4];
                const float LX[4] = {lx.x, lx.y, lx.z, lx.w}, HX[4] = {hx.x, hx.y, hx.z, hx.w};
                const float LY[4] = {ly.x, ly.y, ly.z, ly.w}, HY[4] = {hy.x, hy.y, hy.z, hy.w};
                const float LZ[4] = {lz.x, lz.y, lz.z, lz.w}, HZ[4] = {hz.x, hz.y, hz.z, hz.w};
                const int CR[4] = {cr.x, cr.y, cr.z, cr.w}, CC[4] = {cc.x, cc.y, cc.z, cc.w};
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const bool hit = CC[k] >= 0 && tslab(g, r, LX[k], LY[k], LZ[k], HX[k], HY[k], HZ[k], t[k]) &&
                                     !(t[k] > h.t);
                    const float tk = fmaxf(t[k], 0.0f);
                    key[k] = hit ? ((__float_as_uint(tk) & ~3u) | (unsigned int)k) : 0xffffffffu;
                }
                cswap(key[0], key[1]);
                cswap(key[2], key[3]);
                cswap(key[0], key[2]);
                cswap(key[1], key[3]);
                cswap(key[1], key[2]);
                if (key[0] == 0xffffffffu) {
                    have_node = pop_entry(stk, stt, top, h.t, node);
                } else {
#pragma unroll
                    for (int k = 3; k >= 1; --k) {
                        if (key[k] != 0xffffffffu) {
                            if (top < kStack4) {
                                const int s = key[k] & 3u;
                                stk[top] = make_int2(CR[s], CC[s]);
                                stt[top++] = t[s];
                            } else {
                                g.flags |= RC_GUARD_TRAVERSAL_CAP;
                            }
                        }
                    }
                    const int s0 = key[0] & 3u;
                    node.ref = CR[s0];
                    node.cnt = CC[s0];
                }
            }
            if (++steps > 2 * S.node_count + 64) {
                g.flags |= RC_GUARD_TRAVERSAL_CAP;
                return h.prim >= 0;
            }
            if (__all_sync(__activemask(), leaf.cnt > 0)) break;
        }
        if (leaf.cnt > 0) {
            for (int i = leaf.ref; i < leaf.ref + leaf.cnt; ++i) {
                float tt, u, v;
                if (thit(g, r, S.tri_isect, i, h.t, tt, u, v) && tt < h.t) {
                    if (kAnyHit) return true;
                    h.t = tt;
                    h.u = u;
                    h.v = v;
                    h.prim = i;
                }
            }
            leaf.cnt = 0;
        }
    }
    return h.prim >= 0;
}
#endif

// Closest hit and visibility as used by the kernels: the reference's
// traversal order in the exact build; in the fast build the 4-wide
// traversal when the scene has 4-wide nodes, else the binary one -- except
// on BVHs deep enough that the reference's stacks can overflow (closest hit
// and photon walks past 60 levels, shadow walks past 28): there the
// reference drops pushes, which ones depends on its own visiting order, and
// the fast build keeps that order so that it drops the same ones.
// kShallow: the caller runs only on BVHs of at most 60 levels (the
// shallow-tree instantiations of its kernel: 28 levels for the path tracer's,
// 60 for the photon passes'), where the reference's closest-hit stack cannot
// overflow, so the deep-tree branch is compiled out.
template <bool kShallow>
DI Hit closest_hit(const DeviceScene& S, const Ray& r, Guard& g) {
#if RC_EXACT
    return trace_closest(S, r, g);
#else
    if (!kShallow && S.depth > 60) return trace_closest(S, r, g);
    Hit h;
    if (S.nodes4)
        traverse4<false>(S, r, 1e30f, g, h);
    else
        traverse_ww<false>(S, r, 1e30f, g, h);
    return h;
#endif
}

template <bool kTestAtParent>
DI bool unoccluded(const DeviceScene& S, const Ray& r, float max_dist, Guard& g) {
#if RC_EXACT
    return trace_shadow<kTestAtParent>(S, r, max_dist, g);
#else
    if (!kTestAtParent) return trace_shadow<false>(S, r, max_dist, g);
    Hit h;
    if (S.nodes4) return !traverse4<true>(S, r, max_dist, g, h);
    return !traverse_ww<true>(S, r, max_dist, g, h);
#endif
}

// The photon passes' closest hit: the reference's unordered push order in
// the exact build (it decides ties), the fast traversal otherwise.
template <bool kTestAtParent>
DI Hit photon_hit(const DeviceScene& S, const Ray& r, Guard& g) {
#if RC_EXACT
    return trace_unordered<kTestAtParent>(S, r, g);
#else
    if (!kTestAtParent) return trace_unordered<false>(S, r, g);
    return closest_hit<true>(S, r, g);
#endif
}

// ---------------------------------------------------------------------------
// materials and sampling
// ---------------------------------------------------------------------------
struct Mat {
    float3 albedo;
    float metallic;
    float3 emission;
    float strength;
    float roughness, ior, transmission;
};

DI Mat load_mat(const DeviceScene& S, int m) {
    const float4 a = __ldg(S.materials + 4 * m + 0);
    const float4 b = __ldg(S.materials + 4 * m + 1);
    const float4 c = __ldg(S.materials + 4 * m + 2);
    Mat M;
    M.albedo = xyz(a);
    M.metallic = a.w;
    M.emission = xyz(b);
    M.strength = b.w;
    M.roughness = c.x;
    M.ior = c.y;
    M.transmission = c.z;
    return M;
}

// pathtrace.comp:252-276
DI float3 sample_ggx_vndf(float3 wo, float alpha, float ux, float uy) {
    const float3 v = normalize(f3(wo.x * alpha, wo.y, wo.z * alpha));
    const float3 t1 = (v.y < 0.9999f) ? normalize(cross(v, f3(0.0f, 1.0f, 0.0f))) : f3(1.0f, 0.0f, 0.0f);
    const float3 t2 = cross(t1, v);
    const float a = 1.0f / (1.0f + v.y);
    const float r = sqrtf(ux);
    const float phi = (uy < a) ? (uy / a) * 3.14159265359f : 3.14159265359f + (uy - a) / (1.0f - a) * 3.14159265359f;
    float sp, cp;
    sincos_(phi, &sp, &cp);
    const float p1 = r * cp;
    const float p2 = r * sp * ((uy < a) ? 1.0f : v.y);
    const float3 n = p1 * t1 + p2 * t2 + sqrtf(gmax(0.0f, 1.0f - p1 * p1 - p2 * p2)) * v;
    return normalize(f3(alpha * n.x, gmax(0.0f, n.y), alpha * n.z));
}

// pathtrace.comp:279-292
DI float smith_g1(float NdotV, float alpha) {
    const float a2 = alpha * alpha;
    const float denom = NdotV + sqrtf(a2 + (1.0f - a2) * NdotV * NdotV);
    return 2.0f * NdotV / gmax(denom, 1e-7f);
}
DI float smith_g2(float NdotL, float NdotV, float alpha) {
    const float a2 = alpha * alpha;
    const float dA = NdotV * sqrtf(a2 + (1.0f - a2) * NdotL * NdotL);
    const float dB = NdotL * sqrtf(a2 + (1.0f - a2) * NdotV * NdotV);
    return 2.0f * NdotL * NdotV / gmax(dA + dB, 1e-7f);
}

// pathtrace.comp:296-306 (= photon_trace.comp:131-137)
DI float3 cosine_hemisphere(float ux, float uy, float3 n) {
    const float r = sqrtf(ux);
    const float phi = 6.28318530718f * uy;
    float sp, cp;
    sincos_(phi, &sp, &cp);
    const float3 local = f3(r * cp, r * sp, sqrtf(gmax(0.0f, 1.0f - ux)));
    const float3 up = fabs_(n.y) < 0.9999f ? f3(0.0f, 1.0f, 0.0f) : f3(1.0f, 0.0f, 0.0f);
    const float3 t = normalize(cross(up, n));
    const float3 b = cross(n, t);
    return normalize(t * local.x + b * local.y + n * local.z);
}

// pathtrace.comp:310-321
// The aperture polygon's corner directions: (sin, cos) of
// 6.28318530718f * k / N for k = 0..N+1, each computed as sample_ngon
// computes it, so a sample read from the table is the sample computed
// directly, bit for bit.  A kernel whose paths share a blade count fills
// one per block (kNgonTab entries at most) and skips four sin/cos
// evaluations per camera ray -- the exact build's correctly rounded ones
// cost most of its ray generation.
constexpr int kNgonTab = 34;
DI void fill_ngon_table(float2* tab, int N) {
    if (N < 1 || N + 2 > kNgonTab) return;
    for (int k = threadIdx.x; k <= N + 1; k += blockDim.x) {
        float s, c;
        sincos_(6.28318530718f * (float)k / (float)N, &s, &c);
        tab[k] = make_float2(s, c);
    }
}
DI bool ngon_table_ok(int N) { return N >= 1 && N + 2 <= kNgonTab; }

// tab: fill_ngon_table(tab, N)'s table for this N, or null.
DI float2 sample_ngon(uint32_t& seed, float radius, int N, const float2* tab = nullptr) {
    float r1 = rnd(seed);
    float r2 = rnd(seed);
    if (r1 + r2 > 1.0f) {
        r1 = 1.0f - r1;
        r2 = 1.0f - r2;
    }
    const int sector = (int)(rnd(seed) * (float)N);
    float s0, c0, s1, c1;
    if (tab && sector >= 0 && sector <= N) {
        const float2 e0 = tab[sector], e1 = tab[sector + 1];
        s0 = e0.x;
        c0 = e0.y;
        s1 = e1.x;
        c1 = e1.y;
    } else {
        const float a0 = 6.28318530718f * (float)sector / (float)N;
        const float a1 = 6.28318530718f * (float)(sector + 1) / (float)N;
        sincos_(a0, &s0, &c0);
        sincos_(a1, &s1, &c1);
    }
    return make_float2((r1 * c0 + r2 * c1) * radius, (r1 * s0 + r2 * s1) * radius);
}

struct Counts {
    uint32_t paths, closest, shadow, hits, lights;
};

// pathtrace.comp:401-439
// ngon: the corner table for cam.blades (fill_ngon_table), or null.
DI Ray generate_ray(const CamParams& cam, int W, int H, int px, int py, uint32_t& seed, float offset,
                    const float2* ngon = nullptr) {
    const float aspect = (float)W / (float)H;
    const float jx = rnd(seed) - 0.5f;
    const float jy = rnd(seed) - 0.5f;
    const float nx = ((float)px + 0.5f + jx) / (float)W;
    const float ny = ((float)py + 0.5f + jy) / (float)H;
    const float sx = nx * 2.0f - 1.0f;
    const float sy = ny * 2.0f - 1.0f;
    const float3 F = f3(cam.fwd[0], cam.fwd[1], cam.fwd[2]);
    const float3 R = f3(cam.right[0], cam.right[1], cam.right[2]);
    const float3 U = f3(cam.up[0], cam.up[1], cam.up[2]);
    const float3 P = f3(cam.pos[0], cam.pos[1], cam.pos[2]);
    const float3 pin = normalize(F + R * (sx * aspect * cam.tan_half) + U * (sy * cam.tan_half));
    float2 lens = make_float2(0.0f, 0.0f);
    if (cam.lens_radius > 0.0f) lens = sample_ngon(seed, cam.lens_radius, cam.blades, ngon);
    const float nr2 = (cam.lens_radius > 1e-6f)
        ? gclamp((lens.x * lens.x + lens.y * lens.y) / (cam.lens_radius * cam.lens_radius), 0.0f, 1.0f)
        : 0.0f;
    float eff = cam.focal + offset + cam.sa * nr2;
    eff = gmax(eff, 0.01f);
    const float tf = eff / dot(pin, F);
    const float3 focal_pt = P + pin * tf;
    const float3 ro = P + R * lens.x + U * lens.y;
    return make_ray(ro, normalize(focal_pt - ro));
}

// pathtrace.comp:341-395
template <bool kShadowAtParent>
DI float3 sample_direct_light(const DeviceScene& S, float3 hp, float3 n, float3 albedo, float clampk,
                              uint32_t& seed, Guard& g, Counts& cn) {
    if (S.light_count <= 0 || S.total_light_power <= 0.0f) return f3(0, 0, 0);
    const float u = rnd(seed);
    int sel = S.light_count - 1;
    for (int i = 0; i < S.light_count; ++i)
        if (u < __ldg(S.light_cdf + i)) {
            sel = i;
            break;
        }
    const float4* L = S.lights + 5 * sel;
    const float4 l0 = __ldg(L + 0), l1 = __ldg(L + 1), l2 = __ldg(L + 2), l3 = __ldg(L + 3), l4 = __ldg(L + 4);
    cn.lights++;
    const float pick = l3.w / S.total_light_power;
    if (pick <= 0.0f) return f3(0, 0, 0);
    float r1 = rnd(seed);
    float r2 = rnd(seed);
    if (r1 + r2 > 1.0f) {
        r1 = 1.0f - r1;
        r2 = 1.0f - r2;
    }
    const float3 lv0 = xyz(l0);
    const float3 lp = lv0 + r1 * (xyz(l1) - lv0) + r2 * (xyz(l2) - lv0);
    const float3 to = lp - hp;
    const float dist2 = dot(to, to);
    const float dist = sqrtf(dist2);
    const float3 sd = to / dist;
    const float cos_hit = dot(n, sd);
    if (cos_hit <= 0.0f) return f3(0, 0, 0);
    const float cos_light = fabs_(dot(xyz(l4), sd));
    if (cos_light <= 0.0f) return f3(0, 0, 0);
    const float area = l0.w;
    const float dist2_safe = gmax(dist2, area);
    cn.shadow++;
    if (!unoccluded<kShadowAtParent>(S, make_ray(hp + n * 2e-3f, sd), dist - 4e-3f, g)) return f3(0, 0, 0);
    const float pdf = pick * (dist2_safe / (area * cos_light));
    if (pdf <= 0.0f) return f3(0, 0, 0);
    const float3 em = xyz(l3);
    const float3 contrib = (((albedo / 3.14159265359f) * em) * cos_hit) / pdf;
    const float cap = dot(em, f3(0.299f, 0.587f, 0.114f)) * clampk;
    return vmin(contrib, f3(cap, cap, cap));
}

// pathtrace.comp:454-585
template <bool kShadowAtParent>
DI float3 trace_radiance(const DeviceScene& S, Ray ray, uint32_t& seed, int nee, float clampk, float3& first_alb,
                         Guard& g, Counts& cn) {
    first_alb = f3(1.0f, 1.0f, 1.0f);
    float3 rad = f3(0, 0, 0);
    float3 thr = f3(1.0f, 1.0f, 1.0f);
    bool last_diffuse = false;
    cn.paths++;
    for (int bounce = 0; bounce < 6; ++bounce) {
        cn.closest++;
        const Hit hit = closest_hit<kShadowAtParent>(S, ray, g);
        if (hit.prim < 0) break;
        cn.hits++;
        const Surf sf = surface(S, ray, hit);
        const Mat m = load_mat(S, sf.mat);
        const float3 rd = ray.d;
        const float3 n = dot(rd, sf.normal) < 0.0f ? sf.normal : -sf.normal;
        if (bounce == 0) first_alb = (m.transmission > 0.5f) ? f3(1.0f, 1.0f, 1.0f) : m.albedo;
        if (!last_diffuse) rad = rad + (thr * m.emission) * m.strength;
        if (bounce >= 2) {
            float survive = gmax(m.albedo.x, gmax(m.albedo.y, m.albedo.z));
            if (m.metallic > 0.5f || m.transmission > 0.5f) survive = 0.95f;
            survive = gclamp(survive, 0.01f, 0.95f);
            if (rnd(seed) > survive) break;
            thr = thr / survive;
        }
        if (m.transmission > 0.5f) {
            const bool entering = dot(rd, sf.normal) < 0.0f;
            const float eta = entering ? (1.0f / m.ior) : m.ior;
            const float cosI = fabs_(dot(rd, n));
            float r0 = (1.0f - m.ior) / (1.0f + m.ior);
            r0 *= r0;
            const float F = r0 + (1.0f - r0) * pow5(gclamp(1.0f - cosI, 0.0f, 1.0f));
            float3 nd;
            if (rnd(seed) < F) {
                nd = reflect(rd, n);
            } else {
                float3 refr = refract(rd, n, eta);
                if (dot(refr, refr) < 0.001f) refr = reflect(rd, n);
                nd = normalize(refr);
            }
            ray = make_ray(sf.pos + nd * 2e-3f, nd);
            thr = thr * m.albedo;
            last_diffuse = false;
        } else if (m.metallic > 0.5f) {
            const float3 wo = -rd;
            const float alpha = gmax(m.roughness, 1e-3f);
            const float3 up3 = fabs_(n.y) < 0.9999f ? f3(0.0f, 1.0f, 0.0f) : f3(1.0f, 0.0f, 0.0f);
            const float3 T = normalize(cross(up3, n));
            const float3 B = cross(n, T);
            const float3 wol = f3(dot(wo, T), dot(wo, n), dot(wo, B));
            const float u1 = rnd(seed);
            const float u2 = rnd(seed);
            const float3 hl = sample_ggx_vndf(wol, alpha, u1, u2);
            const float3 h = normalize(T * hl.x + n * hl.y + B * hl.z);
            float3 nd = reflect(-wo, h);
            if (dot(nd, n) <= 0.0f) nd = reflect(-wo, n);
            const float NdotL = gmax(dot(n, nd), 1e-4f);
            const float NdotV = gmax(dot(n, wo), 1e-4f);
            const float HdotV = gmax(dot(h, wo), 1e-4f);
            const float p5 = pow5(1.0f - HdotV);
            const float3 F = m.albedo + f3(1.0f - m.albedo.x, 1.0f - m.albedo.y, 1.0f - m.albedo.z) * p5;
            const float G1 = smith_g1(NdotV, alpha);
            const float G2 = smith_g2(NdotL, NdotV, alpha);
            thr = thr * (F * (G2 / gmax(G1, 1e-7f)));
            ray = make_ray(sf.pos + n * 2e-3f, nd);
            last_diffuse = false;
        } else {
            if (nee != 0)
                rad = rad + thr * sample_direct_light<kShadowAtParent>(S, sf.pos, n, m.albedo, clampk, seed, g, cn);
            const float u1 = rnd(seed);
            const float u2 = rnd(seed);
            const float3 nd = cosine_hemisphere(u1, u2, n);
            thr = thr * m.albedo;
            ray = make_ray(sf.pos + n * 1e-3f, nd);
            last_diffuse = true;
        }
    }
    return rad;
}

// Warp-level sums of the work counts; one 64-bit atomic per counter per warp.
DI void flush_work(const Guard& g, unsigned int hits, unsigned int lights, DevCounters* ctr,
                   bool photon_pass = false) {
    const unsigned int lane = threadIdx.x & 31u;
    const unsigned int n = __reduce_add_sync(0xffffffffu, g.nodes);
    const unsigned int t = __reduce_add_sync(0xffffffffu, g.tris);
    const unsigned int h = __reduce_add_sync(0xffffffffu, hits);
    const unsigned int l = __reduce_add_sync(0xffffffffu, lights);
    const unsigned int gf = __reduce_or_sync(0xffffffffu, g.flags);
    if (lane == 0) {
        if (n) atomicAdd(photon_pass ? &ctr->photon_node_tests : &ctr->node_tests, (unsigned long long)n);
        if (t) atomicAdd(photon_pass ? &ctr->photon_tri_tests : &ctr->tri_tests, (unsigned long long)t);
        if (h) atomicAdd(&ctr->surface_hits, (unsigned long long)h);
        if (l) atomicAdd(&ctr->light_samples, (unsigned long long)l);
        if (gf) atomicOr(&ctr->error_word, gf);
    }
}

DI void flush_counts(const Counts& cn, const Guard& g, DevCounters* ctr) {
    const unsigned int lane = threadIdx.x & 31u;
    const unsigned int p = __reduce_add_sync(0xffffffffu, cn.paths);
    const unsigned int c = __reduce_add_sync(0xffffffffu, cn.closest);
    const unsigned int s = __reduce_add_sync(0xffffffffu, cn.shadow);
    if (lane == 0) {
        if (p) atomicAdd(&ctr->camera_paths, (unsigned long long)p);
        if (c) atomicAdd(&ctr->closest_rays, (unsigned long long)c);
        if (s) atomicAdd(&ctr->shadow_rays, (unsigned long long)s);
    }
    flush_work(g, cn.hits, cn.lights, ctr);
}

DI ushort4 to_half4(float a, float b, float c, float d) {
    return make_ushort4(__half_as_ushort(__float2half_rn(a)), __half_as_ushort(__float2half_rn(b)),
                        __half_as_ushort(__float2half_rn(c)), __half_as_ushort(__float2half_rn(d)));
}

}  // namespace RC_NS
}  // namespace rc

#endif
