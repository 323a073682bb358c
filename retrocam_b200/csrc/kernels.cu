// kernels.cu -- sm_100a kernels of the render hot path.
//
// Compiled twice into the library:
//   RC_EXACT=1, -fmad=false: IEEE single operations in the order the GLSL
//     reads, GLSL min/max definitions, transcendentals from
//     include/rc_exact_math.h.  Results are bit-identical to the CPU oracle
//     (namespace rc::exact).
//   RC_EXACT=0, -fmad=true: FMA contraction, hardware min/max, SFU
//     intrinsics, rsqrt-based normalisation (namespace rc::fast); checked
//     against the oracle by tolerance and by converged-image error.
//
// Kernels (reference shader each replaces):
//   render_kernel         pathtrace.comp main()   (Renderer.render x n_spp)
//   photon_trace_kernel   photon_trace.comp main()
//   photon_gather_kernel  photon_gather.comp main()
//   atrous_kernel         post/atrous_denoise.frag (p00_normalize fused
//                         into the first pass)
//   normalize_kernel      post/p00_normalize.frag  (denoiser disabled)
//
// Every traversal loop is bounded: a traversal that pops more stack
// entries than the scene has nodes (impossible for a validated tree) sets
// RC_GUARD_TRAVERSAL_CAP in the context's error word and stops.
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
    float3 o, d, inv;
#if !RC_EXACT
    float3 oinv;   // o * inv, for the FMA form of the slab test
#endif
};

DI Ray make_ray(float3 o, float3 d) {
    Ray r;
    r.o = o;
    r.d = d;
    r.inv = f3(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
#if !RC_EXACT
    r.oinv = o * r.inv;
#endif
    return r;
}

DI bool slab(const Ray& r, float nx, float ny, float nz, float xx, float xy, float xz, float& tmin) {
#if RC_EXACT
    const float t0x = (nx - r.o.x) * r.inv.x, t0y = (ny - r.o.y) * r.inv.y, t0z = (nz - r.o.z) * r.inv.z;
    const float t1x = (xx - r.o.x) * r.inv.x, t1y = (xy - r.o.y) * r.inv.y, t1z = (xz - r.o.z) * r.inv.z;
#else
    const float t0x = fmaf(nx, r.inv.x, -r.oinv.x), t0y = fmaf(ny, r.inv.y, -r.oinv.y), t0z = fmaf(nz, r.inv.z, -r.oinv.z);
    const float t1x = fmaf(xx, r.inv.x, -r.oinv.x), t1y = fmaf(xy, r.inv.y, -r.oinv.y), t1z = fmaf(xz, r.inv.z, -r.oinv.z);
#endif
    const float lox = gmin(t0x, t1x), loy = gmin(t0y, t1y), loz = gmin(t0z, t1z);
    const float hix = gmax(t0x, t1x), hiy = gmax(t0y, t1y), hiz = gmax(t0z, t1z);
    tmin = gmax(gmax(lox, loy), loz);
    const float tmax = gmin(gmin(hix, hiy), hiz);
    return tmax >= gmax(tmin, 0.0f);
}

DI bool hit_triangle(const Ray& r, const float4* __restrict__ tri_isect, int i, float& t, float& u, float& v) {
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

DI bool thit(Guard& g, const Ray& r, const float4* __restrict__ tri_isect, int i, float& t, float& u, float& v) {
    ++g.tris;
    return hit_triangle(r, tri_isect, i, t, u, v);
}

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
    if (!tslab(g, r, S.root_min[0], S.root_min[1], S.root_min[2], S.root_max[0], S.root_max[1], S.root_max[2], tmin))
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
                if (thit(g, r, S.tri_isect, i, t, u, v) && t < h.t) {
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
            const bool hl = tslab(g, r, a.x, a.y, a.z, a.w, b.x, b.y, tl);
            const bool hr = tslab(g, r, b.z, b.w, c.x, c.y, c.z, c.w, tr);
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
    if (!tslab(g, r, S.root_min[0], S.root_min[1], S.root_min[2], S.root_max[0], S.root_max[1], S.root_max[2], tmin))
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
                if (thit(g, r, S.tri_isect, i, t, u, v) && t < h.t) {
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
                const bool hl = tslab(g, r, a.x, a.y, a.z, a.w, b.x, b.y, tl);
                const bool hr = tslab(g, r, b.z, b.w, c.x, c.y, c.z, c.w, tr);
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
                const bool hit = right ? tslab(g, r, b.z, b.w, c.x, c.y, c.z, c.w, tc)
                                       : tslab(g, r, a.x, a.y, a.z, a.w, b.x, b.y, tc);
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
    if (!tslab(g, r, S.root_min[0], S.root_min[1], S.root_min[2], S.root_max[0], S.root_max[1], S.root_max[2], tmin))
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
                if (thit(g, r, S.tri_isect, i, t, u, v) && t < max_dist) return false;
            }
        } else if (top < 30) {
            if (kTestAtParent) {
                const NodeRec* nr = S.nodes + ref;
                const float4 a = __ldg(&nr->a), b = __ldg(&nr->b), c = __ldg(&nr->c);
                const int4 d = __ldg(&nr->d);
                float tl, tr;
                const bool hl = tslab(g, r, a.x, a.y, a.z, a.w, b.x, b.y, tl) && !(tl > max_dist);
                const bool hr = tslab(g, r, b.z, b.w, c.x, c.y, c.z, c.w, tr) && !(tr > max_dist);
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
                const bool hit = right ? tslab(g, r, b.z, b.w, c.x, c.y, c.z, c.w, tc)
                                       : tslab(g, r, a.x, a.y, a.z, a.w, b.x, b.y, tc);
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
DI float2 sample_ngon(uint32_t& seed, float radius, int N) {
    float r1 = rnd(seed);
    float r2 = rnd(seed);
    if (r1 + r2 > 1.0f) {
        r1 = 1.0f - r1;
        r2 = 1.0f - r2;
    }
    const int sector = (int)(rnd(seed) * (float)N);
    const float a0 = 6.28318530718f * (float)sector / (float)N;
    const float a1 = 6.28318530718f * (float)(sector + 1) / (float)N;
    float s0, c0, s1, c1;
    sincos_(a0, &s0, &c0);
    sincos_(a1, &s1, &c1);
    return make_float2((r1 * c0 + r2 * c1) * radius, (r1 * s0 + r2 * s1) * radius);
}

struct Counts {
    uint32_t paths, closest, shadow, hits, lights;
};

// pathtrace.comp:401-439
DI Ray generate_ray(const CamParams& cam, int W, int H, int px, int py, uint32_t& seed, float offset) {
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
    if (cam.lens_radius > 0.0f) lens = sample_ngon(seed, cam.lens_radius, cam.blades);
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
    if (!trace_shadow<kShadowAtParent>(S, make_ray(hp + n * 2e-3f, sd), dist - 4e-3f, g)) return f3(0, 0, 0);
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
        const Hit hit = trace_closest(S, ray, g);
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

DI ushort4 to_half4(float a, float b, float c, float d) {
    return make_ushort4(__half_as_ushort(__float2half_rn(a)), __half_as_ushort(__float2half_rn(b)),
                        __half_as_ushort(__float2half_rn(c)), __half_as_ushort(__float2half_rn(d)));
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

// pathtrace.comp:601-655 for frames first .. first+n_spp-1.  A 128-thread
// block covers a 16x8 pixel tile; each warp an 8x4 sub-tile, so primary rays
// of a warp are spatially coherent.  The running sums stay in registers
// across the frames and are stored once, which gives the same float
// additions in the same order as one dispatch per frame.
template <bool kShadowAtParent>
__global__ void __launch_bounds__(128) render_kernel(RenderArgs A) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int px = blockIdx.x * 16 + (warp & 1) * 8 + (lane & 7);
    const int py = blockIdx.y * 8 + (warp >> 1) * 4 + (lane >> 3);
    const int W = A.img.width, H = A.img.height;
    const bool inside = px < W && py < H;
    Counts cn = {0u, 0u, 0u, 0u, 0u};
    Guard g = {0u, 0u, 0u};
    if (inside) {
        const long i = (long)py * W + px;
        const DeviceScene& S = A.scene;
        const CamParams& cam = A.cam;
        const bool lca = (fabs_(cam.lca[0]) + fabs_(cam.lca[2])) > 1e-4f;
        float4 acc = make_float4(0, 0, 0, 0);
        float var = 0.0f;
        if (A.first_frame > 0) {
            acc = A.img.accum[i];
            var = A.img.var[i];
        }
        for (int f = A.first_frame; f < A.first_frame + A.n_spp; ++f) {
            float3 rad, alb;
            if (lca) {
                float ch[3];
                for (int c = 0; c < 3; ++c) {
                    uint32_t s = init_seed(px, py, f * 3 + c);
                    const Ray ray = generate_ray(cam, W, H, px, py, s, cam.lca[c]);
                    float3 a;
                    const float3 r = trace_radiance<kShadowAtParent>(S, ray, s, A.nee_enabled, A.firefly_clamp, a, g, cn);
                    ch[c] = (c == 0) ? r.x : (c == 1 ? r.y : r.z);
                    if (c == 1) alb = a;
                }
                rad = f3(ch[0], ch[1], ch[2]);
            } else {
                uint32_t s = init_seed(px, py, f);
                const Ray ray = generate_ray(cam, W, H, px, py, s, 0.0f);
                rad = trace_radiance<kShadowAtParent>(S, ray, s, A.nee_enabled, A.firefly_clamp, alb, g, cn);
            }
            if (bad(rad.x) || bad(rad.y) || bad(rad.z)) rad = f3(0, 0, 0);
            const float l = luma709(rad);
            const float l2 = l * l;
            if (f == 0) {
                acc = make_float4(rad.x, rad.y, rad.z, 1.0f);
                var = l2;
                uint32_t gs = init_seed(px, py, 99991);
                const Ray gr = generate_ray(cam, W, H, px, py, gs, 0.0f);
                cn.closest++;
                const Hit h = trace_closest(S, gr, g);
                float4 gv = make_float4(0.0f, 1.0f, 0.0f, 1e4f);
                if (h.prim >= 0) {
                    cn.hits++;
                    const Surf sf = surface(S, gr, h);
                    const float3 nn = dot(gr.d, sf.normal) < 0.0f ? sf.normal : -sf.normal;
                    gv = make_float4(nn.x, nn.y, nn.z, h.t);
                }
                A.img.gbuf[i] = to_half4(gv.x, gv.y, gv.z, gv.w);
                A.img.galb[i] = to_half4(alb.x, alb.y, alb.z, 1.0f);
            } else {
                acc.x = acc.x + rad.x;
                acc.y = acc.y + rad.y;
                acc.z = acc.z + rad.z;
                acc.w = acc.w + 1.0f;
                var = var + l2;
            }
        }
        A.img.accum[i] = acc;
        A.img.var[i] = var;
    }
    flush_counts(cn, g, A.counters);
}

// photon_trace.comp:146-149
DI float fresnel_schlick(float cos_theta, float ior) {
    float r0 = (1.0f - ior) / (1.0f + ior);
    r0 *= r0;
    return r0 + (1.0f - r0) * pow5(gclamp(1.0f - cos_theta, 0.0f, 1.0f));
}

// photon_trace.comp:168-252: one thread per photon; stored photons are
// appended with a warp-aggregated 32-bit atomicAdd on the counter and linked
// into their cell with a 32-bit atomicExch on the cell head.
template <bool kAtParent>
__global__ void __launch_bounds__(128) photon_trace_kernel(PhotonArgs A) {
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    const DeviceScene& S = A.scene;
    Guard g = {0u, 0u, 0u};
    uint32_t rays = 0, hits = 0;
    bool store = false;
    float3 spos = f3(0, 0, 0), spow = f3(0, 0, 0), sdir = f3(0, 0, 0);
    if (gid < A.photon_count && S.light_count != 0) {
        uint32_t seed = photon_seed((uint32_t)gid, A.seed);
        const float u = rnd(seed);
        int sel = S.light_count - 1;
        for (int i = 0; i < S.light_count; ++i)
            if (u < __ldg(S.light_cdf + i)) {
                sel = i;
                break;
            }
        const float4* L = S.lights + 5 * sel;
        const float4 l0 = __ldg(L + 0), l1 = __ldg(L + 1), l2 = __ldg(L + 2), l3 = __ldg(L + 3), l4 = __ldg(L + 4);
        float r1 = rnd(seed);
        float r2 = rnd(seed);
        if (r1 + r2 > 1.0f) {
            r1 = 1.0f - r1;
            r2 = 1.0f - r2;
        }
        const float3 lv0 = xyz(l0);
        const float3 sp = lv0 + r1 * (xyz(l1) - lv0) + r2 * (xyz(l2) - lv0);
        const float3 en = normalize(xyz(l4));
        const float e1 = rnd(seed);
        const float e2 = rnd(seed);
        float3 rd = cosine_hemisphere(e1, e2, en);
        const float3 em = xyz(l3);
        const float lum = dot(em, f3(0.299f, 0.587f, 0.114f));
        const float per = S.total_light_power / (float)A.photon_count;
        float3 power = (lum > 1e-6f) ? (em / lum) * per : f3(per, per, per);
        Ray ray = make_ray(sp + en * 1e-3f, rd);
        bool spec = false;
        for (int b = 0; b < 8; ++b) {
            ++rays;
            const Hit hit = trace_unordered<kAtParent>(S, ray, g);
            if (hit.prim < 0) break;
            ++hits;
            const Surf sf = surface(S, ray, hit);
            const Mat m = load_mat(S, sf.mat);
            rd = ray.d;
            const float3 n = dot(rd, sf.normal) < 0.0f ? sf.normal : -sf.normal;
            if (m.transmission > 0.5f) {
                const bool entering = dot(rd, sf.normal) < 0.0f;
                const float eta = entering ? (1.0f / m.ior) : m.ior;
                const float cosI = fabs_(dot(rd, n));
                const float F = fresnel_schlick(cosI, m.ior);
                float3 nd;
                if (rnd(seed) < F) {
                    nd = reflect(rd, n);
                } else {
                    float3 refr = refract(rd, n, eta);
                    if (dot(refr, refr) < 0.001f) refr = reflect(rd, n);
                    nd = normalize(refr);
                }
                ray = make_ray(sf.pos + nd * 2e-3f, nd);
                spec = true;
                continue;
            }
            if (m.metallic > 0.5f) {
                power = power * m.albedo;
                const float3 nd = reflect(rd, n);
                ray = make_ray(sf.pos + n * 2e-3f, nd);
                spec = true;
                continue;
            }
            if (spec) {
                store = true;
                spos = sf.pos;
                spow = power;
                sdir = rd;
            }
            break;
        }
    }
    // warp-aggregated counter increment: one atomicAdd per warp
    const unsigned int mask = __ballot_sync(0xffffffffu, store);
    const int lane = threadIdx.x & 31;
    unsigned int base = 0;
    if (mask != 0u) {
        const int leader = __ffs(mask) - 1;
        if (lane == leader) base = atomicAdd(A.counter, (unsigned int)__popc(mask));
        base = __shfl_sync(0xffffffffu, base, leader);
    }
    if (store) {
        const unsigned int idx = base + __popc(mask & ((1u << lane) - 1u));
        if (idx < (unsigned int)A.photon_count) {
            const int cx = (int)floorf(spos.x / A.radius);
            const int cy = (int)floorf(spos.y / A.radius);
            const int cz = (int)floorf(spos.z / A.radius);
            const int h = cell_hash(cx, cy, cz, A.hash_size);
            const int old = atomicExch(A.heads + h, (int)idx);
            A.next[idx] = old;
            A.photons[3 * idx + 0] = make_float4(spos.x, spos.y, spos.z, 0.0f);
            A.photons[3 * idx + 1] = make_float4(spow.x, spow.y, spow.z, 0.0f);
            A.photons[3 * idx + 2] = make_float4(sdir.x, sdir.y, sdir.z, 0.0f);
        }
    }
    const unsigned int rsum = __reduce_add_sync(0xffffffffu, rays);
    if (lane == 0 && rsum) atomicAdd(&A.counters->photon_rays, (unsigned long long)rsum);
    flush_work(g, 0u, 0u, A.counters, true);
}

// photon_gather.comp:128-222: pinhole ray to the first diffuse surface,
// 3x3x3 hash-cell query, Epanechnikov kernel, added into the accumulation.
template <bool kAtParent>
__global__ void __launch_bounds__(128) photon_gather_kernel(GatherArgs A) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int px = blockIdx.x * 16 + (warp & 1) * 8 + (lane & 7);
    const int py = blockIdx.y * 8 + (warp >> 1) * 4 + (lane >> 3);
    const int W = A.img.width, H = A.img.height;
    Guard g = {0u, 0u, 0u};
    uint32_t rays = 0, hits = 0;
    if (px < W && py < H) {
        const DeviceScene& S = A.scene;
        const CamParams& cam = A.cam;
        const float aspect = (float)W / (float)H;
        const float nx = ((float)px + 0.5f) / (float)W * 2.0f - 1.0f;
        const float ny = ((float)py + 0.5f) / (float)H * 2.0f - 1.0f;
        const float3 F = f3(cam.fwd[0], cam.fwd[1], cam.fwd[2]);
        const float3 R = f3(cam.right[0], cam.right[1], cam.right[2]);
        const float3 U = f3(cam.up[0], cam.up[1], cam.up[2]);
        Ray ray = make_ray(f3(cam.pos[0], cam.pos[1], cam.pos[2]),
                           normalize(F + R * (nx * aspect * cam.tan_half) + U * (ny * cam.tan_half)));
        bool found = false;
        float3 hp = f3(0, 0, 0);
        int hm = 0;
        for (int s = 0; s <= 6; ++s) {
            ++rays;
            const Hit hit = trace_unordered<kAtParent>(S, ray, g);
            if (hit.prim < 0) break;
            ++hits;
            const Surf sf = surface(S, ray, hit);
            const Mat m = load_mat(S, sf.mat);
            if (m.metallic <= 0.5f && m.transmission <= 0.5f) {
                found = true;
                hp = sf.pos;
                hm = sf.mat;
                break;
            }
            const float3 cur = ray.d;
            const float3 n = dot(cur, sf.normal) < 0.0f ? sf.normal : -sf.normal;
            float3 nd;
            if (m.transmission > 0.5f) {
                const bool entering = dot(cur, sf.normal) < 0.0f;
                const float eta = entering ? (1.0f / m.ior) : m.ior;
                float3 refr = refract(cur, n, eta);
                if (dot(refr, refr) < 0.001f) refr = reflect(cur, n);
                nd = normalize(refr);
            } else {
                nd = reflect(cur, n);
            }
            ray = make_ray(sf.pos + nd * 2e-3f, nd);
        }
        if (found) {
            const float r = A.radius, r2 = r * r;
            const int ccx = (int)floorf(hp.x / r), ccy = (int)floorf(hp.y / r), ccz = (int)floorf(hp.z / r);
            float3 caustic = f3(0, 0, 0);
            for (int dz = -1; dz <= 1; ++dz)
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dx = -1; dx <= 1; ++dx) {
                        const int h = cell_hash(ccx + dx, ccy + dy, ccz + dz, A.hash_size);
                        int idx = __ldg(A.heads + h);
                        int safety = 0;
                        while (idx >= 0 && safety < 512) {
                            const float4 pp = __ldg(A.photons + 3 * idx);
                            const float3 d = hp - xyz(pp);
                            const float d2 = dot(d, d);
                            if (d2 <= r2) {
                                const float w = 1.0f - d2 / r2;
                                caustic = caustic + xyz(__ldg(A.photons + 3 * idx + 1)) * w;
                            }
                            idx = __ldg(A.next + idx);
                            safety++;
                        }
                    }
            const float PI_G = 3.14159265358979f;
            const float4 ma = __ldg(S.materials + 4 * hm);
            float3 L = (xyz(ma) * caustic) / (PI_G * r2);
            if (bad(L.x) || bad(L.y) || bad(L.z)) L = f3(0, 0, 0);
            if (A.weight != 1.0f) L = L * A.weight;
            float4* a = A.img.accum + (long)py * W + px;
            float4 v = *a;
            v.x = v.x + L.x;
            v.y = v.y + L.y;
            v.z = v.z + L.z;
            v.w = v.w + 0.0f;
            *a = v;
        }
    }
    const unsigned int rsum = __reduce_add_sync(0xffffffffu, rays);
    if (lane == 0 && rsum) atomicAdd(&A.counters->gather_rays, (unsigned long long)rsum);
    flush_work(g, 0u, 0u, A.counters, true);
}

// ---------------------------------------------------------------------------
// denoiser
// ---------------------------------------------------------------------------
DI float3 half3(ushort4 h) {
    return f3(__half2float(__ushort_as_half(h.x)), __half2float(__ushort_as_half(h.y)),
              __half2float(__ushort_as_half(h.z)));
}
DI float halfw(ushort4 h) { return __half2float(__ushort_as_half(h.w)); }
DI int wrap_repeat(int i, int n) {
    int m = i % n;
    return m < 0 ? m + n : m;
}
DI int wrap_clamp(int i, int n) { return i < 0 ? 0 : (i >= n ? n - 1 : i); }

// Colour at a pixel: the p00 normalisation (accum.rgb / N * exposure) when
// reading the raw accumulation, else the previous pass's RGBA32F output.
DI float3 color_at(const AtrousArgs& A, long i) {
    const float4 c = __ldg(A.color + i);
    if (A.normalize) {
        const float n = (float)A.sample_count;
        return f3(c.x / n * A.exposure, c.y / n * A.exposure, c.z / n * A.exposure);
    }
    return xyz(c);
}

// post/atrous_denoise.frag:50-122, one thread per pixel.  Colour taps use
// the framebuffer textures' CLAMP_TO_EDGE addressing; G-buffer, albedo and
// variance taps use the renderer textures' default REPEAT addressing.
__global__ void __launch_bounds__(128) atrous_kernel(AtrousArgs A) {
    const int x = blockIdx.x * 32 + (threadIdx.x & 31);
    const int y = blockIdx.y * 4 + (threadIdx.x >> 5);
    const int W = A.width, H = A.height;
    if (x >= W || y >= H) return;
    const long ci = (long)y * W + x;
    const ushort4 cg = __ldg(A.gbuf + ci);
    const float3 c_norm = half3(cg);
    const float c_depth = halfw(cg);
    const float3 c_col = color_at(A, ci);
    if (c_depth > 9000.0f) {
        A.out[ci] = make_float4(c_col.x, c_col.y, c_col.z, 1.0f);
        return;
    }
    const float3 c_alb = half3(__ldg(A.galb + ci));
    const bool has_alb = luma709(c_alb) > 0.02f;
    const float3 c_irr = has_alb ? c_col / vmax(c_alb, f3(0.01f, 0.01f, 0.01f)) : c_col;
    const float N = (float)A.sample_count;
    const float sum_l2 = __ldg(A.var + ci);
    const float mean_l = luma709(c_col / gmax(A.exposure, 1e-4f));
    const float variance = gmax(0.0f, sum_l2 / N - mean_l * mean_l);
    const float var_denom = A.sigma_color * A.sigma_color * variance + 1e-6f;
    const float depth_denom = A.sigma_depth * A.sigma_depth + 1e-6f;
    const float c_logl = logf_(luma709(c_irr) + 1e-3f);
    const float hk[5] = {1.0f / 16.0f, 1.0f / 4.0f, 3.0f / 8.0f, 1.0f / 4.0f, 1.0f / 16.0f};
    float3 irr_sum = f3(0, 0, 0);
    float w_sum = 0.0f;
#pragma unroll
    for (int j = -2; j <= 2; ++j) {
#pragma unroll
        for (int i = -2; i <= 2; ++i) {
            const int tx = x + i * A.step, ty = y + j * A.step;
            const long ri = (long)wrap_repeat(ty, H) * W + wrap_repeat(tx, W);
            const long ki = (long)wrap_clamp(ty, H) * W + wrap_clamp(tx, W);
            const ushort4 g2 = __ldg(A.gbuf + ri);
            const float3 n2 = half3(g2);
            const float dep2 = halfw(g2);
            const float3 col2 = color_at(A, ki);
            const float3 alb2 = half3(__ldg(A.galb + ri));
            const float3 irr2 = (luma709(alb2) > 0.02f) ? col2 / vmax(alb2, f3(0.01f, 0.01f, 0.01f)) : col2;
            const float hw = hk[i + 2] * hk[j + 2];
            const float wn = powf_(gmax(0.0f, dot(c_norm, n2)), A.sigma_normal);
            const float dd = (c_depth - dep2) / (c_depth + 0.001f);
            const float wd = expf_(-(dd * dd) / depth_denom);
            const float ld = c_logl - logf_(luma709(irr2) + 1e-3f);
            const float wc = expf_(-(ld * ld) / var_denom);
            const float w = hw * wn * wd * wc;
            irr_sum = irr_sum + irr2 * w;
            w_sum += w;
        }
    }
    const float3 res_irr = (w_sum > 1e-6f) ? irr_sum / w_sum : c_irr;
    const float3 res = has_alb ? res_irr * c_alb : res_irr;
    A.out[ci] = make_float4(res.x, res.y, res.z, 1.0f);
}

// post/p00_normalize.frag:18-24 (used alone when the denoiser is off).
__global__ void normalize_kernel(NormalizeArgs A) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.count) return;
    const float n = (float)(A.total_samples > 1 ? A.total_samples : 1);
    const float4 c = A.accum[i];
    A.out[i] = make_float4(c.x / n * A.exposure, c.y / n * A.exposure, c.z / n * A.exposure, 1.0f);
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
cudaError_t launch_render(const RenderArgs& A, cudaStream_t s) {
    const dim3 grid((A.img.width + 15) / 16, (A.img.height + 7) / 8);
    if (A.scene.depth <= 28)
        render_kernel<true><<<grid, 128, 0, s>>>(A);
    else
        render_kernel<false><<<grid, 128, 0, s>>>(A);
    return cudaGetLastError();
}

cudaError_t launch_photon_trace(const PhotonArgs& A, cudaStream_t s) {
    const int blocks = (A.photon_count + 127) / 128;
    if (blocks == 0) return cudaSuccess;
    if (A.scene.depth <= 60)
        photon_trace_kernel<true><<<blocks, 128, 0, s>>>(A);
    else
        photon_trace_kernel<false><<<blocks, 128, 0, s>>>(A);
    return cudaGetLastError();
}

cudaError_t launch_photon_gather(const GatherArgs& A, cudaStream_t s) {
    const dim3 grid((A.img.width + 15) / 16, (A.img.height + 7) / 8);
    if (A.scene.depth <= 60)
        photon_gather_kernel<true><<<grid, 128, 0, s>>>(A);
    else
        photon_gather_kernel<false><<<grid, 128, 0, s>>>(A);
    return cudaGetLastError();
}

cudaError_t launch_atrous(const AtrousArgs& A, cudaStream_t s) {
    const dim3 grid((A.width + 31) / 32, (A.height + 3) / 4);
    atrous_kernel<<<grid, 128, 0, s>>>(A);
    return cudaGetLastError();
}

cudaError_t launch_normalize(const NormalizeArgs& A, cudaStream_t s) {
    normalize_kernel<<<(A.count + 255) / 256, 256, 0, s>>>(A);
    return cudaGetLastError();
}

}  // namespace RC_NS
}  // namespace rc
