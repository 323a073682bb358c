/*
 * oracle.cpp -- TEST INFRASTRUCTURE: the CPU oracle of the render hot path.
 *
 * A hand-written C++ restatement of the reference's shaders
 * (src/main/resources/shaders/pathtrace.comp, photon_trace.comp,
 * photon_gather.comp, post/atrous_denoise.frag, post/p00_normalize.frag) and,
 * via oracle_host.cpp, of its Java host logic.  It is the checker for the
 * CUDA kernels and the timed CPU baseline; nothing in the product links it.
 * It is pinned against oracle/_ref (the reference's own shader source
 * compiled for the host by build_ref.py) and against tests/golden fixtures.
 *
 * Arithmetic rules (shared with oracle/_ref and the exact CUDA build):
 * IEEE single, no contraction, expressions evaluated left to right as the
 * GLSL text reads; sin/cos/exp/log/pow from include/rc_exact_math.h; GLSL
 * min/max definitions (y<x?y:x, x<y?y:x); normalize(v) = v / length(v).
 *
 * Deterministic photon insertion: photons are traced in parallel and then
 * inserted into the hash in emission-index order, which is the order a
 * single-threaded dispatch of photon_trace.comp produces.
 */
#include <omp.h>
#include <stdint.h>
#include <string.h>

#include <vector>

#include "half_soft.h"
#include "oracle_host.h"
#include "rc_exact_math.h"
#include "retrocam.h"

namespace oracle {

/* ----------------------------------------------------------------------- */
/* small vector type                                                        */
/* ----------------------------------------------------------------------- */
struct V3 { float x, y, z; };
struct V2 { float x, y; };
static inline V3 v3(float a, float b, float c) { return V3{a, b, c}; }
static inline V3 add(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline V3 sub(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline V3 mul(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline V3 mul(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
static inline V3 mul(float s, V3 a) { return v3(s * a.x, s * a.y, s * a.z); }
static inline V3 dv(V3 a, float s) { return v3(a.x / s, a.y / s, a.z / s); }
static inline V3 dv(V3 a, V3 b) { return v3(a.x / b.x, a.y / b.y, a.z / b.z); }
static inline V3 neg(V3 a) { return v3(-a.x, -a.y, -a.z); }
static inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline V3 cross(V3 a, V3 b) {
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline float gmin(float x, float y) { return (y < x) ? y : x; }
static inline float gmax(float x, float y) { return (x < y) ? y : x; }
static inline float gclamp(float x, float a, float b) { return gmin(gmax(x, a), b); }
static inline V3 gmin(V3 a, V3 b) { return v3(gmin(a.x, b.x), gmin(a.y, b.y), gmin(a.z, b.z)); }
static inline V3 gmax(V3 a, V3 b) { return v3(gmax(a.x, b.x), gmax(a.y, b.y), gmax(a.z, b.z)); }
static inline float fabs_(float x) { return rcx_bitsf(rcx_fbits(x) & 0x7fffffffu); }
static inline float sqrt_(float x) { return __builtin_sqrtf(x); }
static inline float floor_(float x) { return __builtin_floorf(x); }
static inline V3 normalize(V3 v) { return dv(v, sqrt_(dot(v, v))); }
/* reflect: I - 2*dot(N,I)*N */
static inline V3 reflect(V3 I, V3 N) { return sub(I, mul(2.0f * dot(N, I), N)); }
static inline V3 refract(V3 I, V3 N, float eta) {
    const float d = dot(N, I);
    const float k = 1.0f - eta * eta * (1.0f - d * d);
    if (k < 0.0f) return v3(0.0f, 0.0f, 0.0f);
    return sub(mul(eta, I), mul(eta * d + sqrt_(k), N));
}
static inline bool bad(float x) { return (rcx_fbits(x) & 0x7f800000u) == 0x7f800000u; }
static inline V3 ld3(const float* p) { return v3(p[0], p[1], p[2]); }

/* ----------------------------------------------------------------------- */
/* RNG -- pathtrace.comp:80-98, photon_trace.comp:60-72                     */
/* ----------------------------------------------------------------------- */
static inline uint32_t pcg(uint32_t& s) {
    s = s * 747796405u + 2891336453u;
    const uint32_t w = ((s >> ((s >> 28u) + 4u)) ^ s) * 277803737u;
    return (w >> 22u) ^ w;
}
static inline float rnd(uint32_t& s) { return (float)pcg(s) / 4294967296.0f; }
static inline uint32_t init_seed(int px, int py, int frame) {
    /* int arithmetic with wrap-around, then reinterpreted as uint */
    uint32_t s = (uint32_t)px + (uint32_t)py * 7919u + (uint32_t)frame * 6271u;
    pcg(s); pcg(s);
    return s;
}
static inline uint32_t photon_seed(uint32_t idx, int seed) {
    uint32_t s = idx * 1664525u + (uint32_t)seed * 1013904223u + 2531011u;
    pcg(s); pcg(s);
    return s;
}
/* photon_trace.comp:140-143 (int wrap-around). */
static inline int cell_hash(int cx, int cy, int cz, int hash_size) {
    const uint32_t h = ((uint32_t)cx * 73856093u) ^ ((uint32_t)cy * 19349663u) ^ ((uint32_t)cz * 83492791u);
    return (int)(h & (uint32_t)(hash_size - 1));
}

/* ----------------------------------------------------------------------- */
/* scene view + statistics                                                  */
/* ----------------------------------------------------------------------- */
struct Scene {
    const rc_triangle* tris;
    const rc_bvh_node* nodes;
    const rc_material* mats;
    const rc_light* lights;
    int light_count;
    float total_power;
};

struct Stats {
    uint64_t camera_paths = 0, closest_rays = 0, shadow_rays = 0, photon_rays = 0, gather_rays = 0;
    uint64_t node_tests = 0, tri_tests = 0, closest_hits = 0, material_fetches = 0, light_fetches = 0;
    void add(const Stats& o) {
        camera_paths += o.camera_paths; closest_rays += o.closest_rays; shadow_rays += o.shadow_rays;
        photon_rays += o.photon_rays; gather_rays += o.gather_rays; node_tests += o.node_tests;
        tri_tests += o.tri_tests; closest_hits += o.closest_hits;
        material_fetches += o.material_fetches; light_fetches += o.light_fetches;
    }
};

/* pathtrace.comp:102-110 */
static inline bool hit_aabb(V3 ro, V3 inv, const rc_bvh_node& n, float& tmin) {
    const V3 t0 = mul(sub(ld3(n.aabb_min), ro), inv);
    const V3 t1 = mul(sub(ld3(n.aabb_max), ro), inv);
    const V3 lo = gmin(t0, t1), hi = gmax(t0, t1);
    tmin = gmax(gmax(lo.x, lo.y), lo.z);
    const float tmax = gmin(gmin(hi.x, hi.y), hi.z);
    return tmax >= gmax(tmin, 0.0f);
}

/* pathtrace.comp:112-130 */
static inline bool hit_triangle(V3 ro, V3 rd, const rc_triangle& tri, float& t, float& bu, float& bv) {
    const V3 v0 = ld3(tri.v0);
    const V3 e1 = sub(ld3(tri.v1), v0);
    const V3 e2 = sub(ld3(tri.v2), v0);
    const V3 h = cross(rd, e2);
    const float a = dot(e1, h);
    if (fabs_(a) < 1e-8f) return false;
    const float f = 1.0f / a;
    const V3 s = sub(ro, v0);
    const float u = f * dot(s, h);
    if (u < 0.0f || u > 1.0f) return false;
    const V3 q = cross(s, e1);
    const float v = f * dot(rd, q);
    if (v < 0.0f || u + v > 1.0f) return false;
    t = f * dot(e2, q);
    if (t < 1e-4f) return false;
    bu = u; bv = v;
    return true;
}

struct Hit { bool valid; float t; V3 pos; V3 normal; int mat; };

static inline void accept_hit(Hit& rec, V3 ro, V3 rd, float t, float bu, float bv, const rc_triangle& tri) {
    rec.t = t;
    rec.pos = add(ro, mul(rd, t));
    const float w = 1.0f - bu - bv;
    rec.normal = normalize(add(add(mul(ld3(tri.n0), w), mul(ld3(tri.n1), bu)), mul(ld3(tri.n2), bv)));
    rec.mat = tri.mat_index;
    rec.valid = true;
}

/* pathtrace.comp:142-203: closest hit with near-child-first ordering. */
static Hit traverse_ordered(const Scene& sc, V3 ro, V3 rd, Stats& st) {
    Hit rec; rec.valid = false; rec.t = 1e30f; rec.mat = 0;
    rec.pos = v3(0, 0, 0); rec.normal = v3(0, 0, 0);
    const V3 inv = dv(v3(1.0f, 1.0f, 1.0f), rd);
    int stack[64]; int top = 0; stack[top++] = 0;
    st.closest_rays++;
    while (top > 0) {
        const int idx = stack[--top];
        const rc_bvh_node& node = sc.nodes[idx];
        float aabbT;
        st.node_tests++;
        if (!hit_aabb(ro, inv, node, aabbT)) continue;
        if (aabbT > rec.t) continue;
        if (node.prim_count > 0) {
            for (int i = node.prim_start; i < node.prim_start + node.prim_count; ++i) {
                float t, bu, bv;
                st.tri_tests++;
                if (hit_triangle(ro, rd, sc.tris[i], t, bu, bv) && t < rec.t)
                    accept_hit(rec, ro, rd, t, bu, bv, sc.tris[i]);
            }
        } else if (top < 62) {
            float tl, tr;
            st.node_tests += 2;
            const bool hl = hit_aabb(ro, inv, sc.nodes[node.left_child], tl);
            const bool hr = hit_aabb(ro, inv, sc.nodes[node.right_child], tr);
            if (hl && hr) {
                if (tl < tr) { stack[top++] = node.right_child; stack[top++] = node.left_child; }
                else { stack[top++] = node.left_child; stack[top++] = node.right_child; }
            } else if (hl) {
                stack[top++] = node.left_child;
            } else if (hr) {
                stack[top++] = node.right_child;
            }
        }
    }
    if (rec.valid) st.closest_hits++;
    return rec;
}

/* photon_trace.comp:102-128 / photon_gather.comp:342-371: closest hit,
 * right child pushed first, no ordering. */
static Hit traverse_unordered(const Scene& sc, V3 ro, V3 rd, Stats& st) {
    Hit rec; rec.valid = false; rec.t = 1e30f; rec.mat = 0;
    rec.pos = v3(0, 0, 0); rec.normal = v3(0, 0, 0);
    const V3 inv = dv(v3(1.0f, 1.0f, 1.0f), rd);
    int stack[64]; int top = 0; stack[top++] = 0;
    while (top > 0) {
        const int idx = stack[--top];
        const rc_bvh_node& node = sc.nodes[idx];
        float aabbT;
        st.node_tests++;
        if (!hit_aabb(ro, inv, node, aabbT)) continue;
        if (aabbT > rec.t) continue;
        if (node.prim_count > 0) {
            for (int i = node.prim_start; i < node.prim_start + node.prim_count; ++i) {
                float t, bu, bv;
                st.tri_tests++;
                if (hit_triangle(ro, rd, sc.tris[i], t, bu, bv) && t < rec.t)
                    accept_hit(rec, ro, rd, t, bu, bv, sc.tris[i]);
            }
        } else if (top < 62) {
            stack[top++] = node.right_child;
            stack[top++] = node.left_child;
        }
    }
    if (rec.valid) st.closest_hits++;
    return rec;
}

/* pathtrace.comp:211-242: any hit closer than max_dist. true = unoccluded. */
static bool shadow_ray(const Scene& sc, V3 ro, V3 rd, float max_dist, Stats& st) {
    const V3 inv = dv(v3(1.0f, 1.0f, 1.0f), rd);
    int stack[32]; int top = 0; stack[top++] = 0;
    st.shadow_rays++;
    while (top > 0) {
        const int idx = stack[--top];
        const rc_bvh_node& node = sc.nodes[idx];
        float aabbT;
        st.node_tests++;
        if (!hit_aabb(ro, inv, node, aabbT)) continue;
        if (aabbT > max_dist) continue;
        if (node.prim_count > 0) {
            for (int i = node.prim_start; i < node.prim_start + node.prim_count; ++i) {
                float t, bu, bv;
                st.tri_tests++;
                if (hit_triangle(ro, rd, sc.tris[i], t, bu, bv) && t < max_dist) return false;
            }
        } else if (top < 30) {
            stack[top++] = node.right_child;
            stack[top++] = node.left_child;
        }
    }
    return true;
}

/* pathtrace.comp:252-276 (Heitz 2017 VNDF, y-up local frame). */
static V3 sample_ggx_vndf(V3 wo, float alpha, float ux, float uy) {
    const V3 v = normalize(v3(wo.x * alpha, wo.y, wo.z * alpha));
    const V3 t1 = (v.y < 0.9999f) ? normalize(cross(v, v3(0.0f, 1.0f, 0.0f))) : v3(1.0f, 0.0f, 0.0f);
    const V3 t2 = cross(t1, v);
    const float a = 1.0f / (1.0f + v.y);
    const float r = sqrt_(ux);
    const float phi = (uy < a) ? (uy / a) * 3.14159265359f
                               : 3.14159265359f + (uy - a) / (1.0f - a) * 3.14159265359f;
    const float p1 = r * rcx_cosf(phi);
    const float p2 = r * rcx_sinf(phi) * ((uy < a) ? 1.0f : v.y);
    const V3 n = add(add(mul(p1, t1), mul(p2, t2)), mul(sqrt_(gmax(0.0f, 1.0f - p1 * p1 - p2 * p2)), v));
    return normalize(v3(alpha * n.x, gmax(0.0f, n.y), alpha * n.z));
}

/* pathtrace.comp:279-292 */
static float smith_g1(float NdotV, float alpha) {
    const float a2 = alpha * alpha;
    const float denom = NdotV + sqrt_(a2 + (1.0f - a2) * NdotV * NdotV);
    return 2.0f * NdotV / gmax(denom, 1e-7f);
}
static float smith_g2(float NdotL, float NdotV, float alpha) {
    const float a2 = alpha * alpha;
    const float dA = NdotV * sqrt_(a2 + (1.0f - a2) * NdotL * NdotL);
    const float dB = NdotL * sqrt_(a2 + (1.0f - a2) * NdotV * NdotV);
    return 2.0f * NdotL * NdotV / gmax(dA + dB, 1e-7f);
}

/* pathtrace.comp:296-306 (= photon_trace.comp:131-137). */
static V3 cosine_hemisphere(float ux, float uy, V3 n) {
    const float r = sqrt_(ux);
    const float phi = 6.28318530718f * uy;
    const V3 local = v3(r * rcx_cosf(phi), r * rcx_sinf(phi), sqrt_(gmax(0.0f, 1.0f - ux)));
    const V3 up = fabs_(n.y) < 0.9999f ? v3(0.0f, 1.0f, 0.0f) : v3(1.0f, 0.0f, 0.0f);
    const V3 t = normalize(cross(up, n));
    const V3 b = cross(n, t);
    return normalize(add(add(mul(t, local.x), mul(b, local.y)), mul(n, local.z)));
}

/* pathtrace.comp:310-321 */
static V2 sample_ngon(uint32_t& seed, float radius, int N) {
    float r1 = rnd(seed);
    float r2 = rnd(seed);
    if (r1 + r2 > 1.0f) { r1 = 1.0f - r1; r2 = 1.0f - r2; }
    const int sector = (int)(rnd(seed) * (float)N);
    const float a0 = 6.28318530718f * (float)sector / (float)N;
    const float a1 = 6.28318530718f * (float)(sector + 1) / (float)N;
    const float c0 = rcx_cosf(a0), s0 = rcx_sinf(a0);
    const float c1 = rcx_cosf(a1), s1 = rcx_sinf(a1);
    return V2{(r1 * c0 + r2 * c1) * radius, (r1 * s0 + r2 * s1) * radius};
}

struct Camera {
    V3 pos, right, up, fwd;
    float focal, lens_radius, tan_half, sa;
    int blades;
    float lca[3];
};

static Camera camera_from(const rc_camera* c) {
    Camera k;
    k.pos = ld3(c->cam_pos); k.right = ld3(c->cam_right); k.up = ld3(c->cam_up); k.fwd = ld3(c->cam_forward);
    k.focal = c->focal_dist; k.lens_radius = c->lens_radius; k.tan_half = c->fov_tan_half;
    k.sa = c->sa_strength; k.blades = c->aperture_blades;
    k.lca[0] = c->lca_delta[0]; k.lca[1] = c->lca_delta[1]; k.lca[2] = c->lca_delta[2];
    return k;
}

/* pathtrace.comp:401-439 */
static void generate_ray(const Camera& cam, int W, int H, int px, int py, uint32_t& seed, float offset,
                         V3& ro, V3& rd) {
    const float aspect = (float)W / (float)H;
    const float jx = rnd(seed) - 0.5f;
    const float jy = rnd(seed) - 0.5f;
    const float nx = ((float)px + 0.5f + jx) / (float)W;
    const float ny = ((float)py + 0.5f + jy) / (float)H;
    const float sx = nx * 2.0f - 1.0f;
    const float sy = ny * 2.0f - 1.0f;
    const V3 pin = normalize(add(add(cam.fwd, mul(cam.right, sx * aspect * cam.tan_half)),
                                 mul(cam.up, sy * cam.tan_half)));
    V2 lens = V2{0.0f, 0.0f};
    if (cam.lens_radius > 0.0f) lens = sample_ngon(seed, cam.lens_radius, cam.blades);
    const float nr2 = (cam.lens_radius > 1e-6f)
        ? gclamp((lens.x * lens.x + lens.y * lens.y) / (cam.lens_radius * cam.lens_radius), 0.0f, 1.0f)
        : 0.0f;
    float eff = cam.focal + offset + cam.sa * nr2;
    eff = gmax(eff, 0.01f);
    const float tf = eff / dot(pin, cam.fwd);
    const V3 focal_pt = add(cam.pos, mul(pin, tf));
    ro = add(add(cam.pos, mul(cam.right, lens.x)), mul(cam.up, lens.y));
    rd = normalize(sub(focal_pt, ro));
}

/* pathtrace.comp:341-395 */
static V3 sample_direct_light(const Scene& sc, V3 hit_pos, V3 n, V3 albedo, float clampk,
                              uint32_t& seed, Stats& st) {
    if (sc.light_count <= 0 || sc.total_power <= 0.0f) return v3(0, 0, 0);
    const float u = rnd(seed);
    int sel = sc.light_count - 1;
    for (int i = 0; i < sc.light_count; ++i)
        if (u < sc.lights[i].cdf_weight) { sel = i; break; }
    const rc_light& L = sc.lights[sel];
    st.light_fetches++;
    const float pick = L.power / sc.total_power;
    if (pick <= 0.0f) return v3(0, 0, 0);
    float r1 = rnd(seed);
    float r2 = rnd(seed);
    if (r1 + r2 > 1.0f) { r1 = 1.0f - r1; r2 = 1.0f - r2; }
    const V3 lv0 = ld3(L.v0);
    const V3 lp = add(add(lv0, mul(r1, sub(ld3(L.v1), lv0))), mul(r2, sub(ld3(L.v2), lv0)));
    const V3 to = sub(lp, hit_pos);
    const float dist2 = dot(to, to);
    const float dist = sqrt_(dist2);
    const V3 sd = dv(to, dist);
    const float cos_hit = dot(n, sd);
    if (cos_hit <= 0.0f) return v3(0, 0, 0);
    const float cos_light = fabs_(dot(ld3(L.normal), sd));
    if (cos_light <= 0.0f) return v3(0, 0, 0);
    const float dist2_safe = gmax(dist2, L.area);
    const V3 so = add(hit_pos, mul(n, 2e-3f));
    if (!shadow_ray(sc, so, sd, dist - 4e-3f, st)) return v3(0, 0, 0);
    const float pdf_sa = dist2_safe / (L.area * cos_light);
    const float pdf = pick * pdf_sa;
    if (pdf <= 0.0f) return v3(0, 0, 0);
    const V3 contrib = dv(mul(mul(dv(albedo, 3.14159265359f), ld3(L.emission)), cos_hit), pdf);
    const float lum = dot(ld3(L.emission), v3(0.299f, 0.587f, 0.114f));
    const float cap = lum * clampk;
    return gmin(contrib, v3(cap, cap, cap));
}

/* pathtrace.comp:454-585 */
static V3 trace_radiance(const Scene& sc, V3 ro, V3 rd, uint32_t& seed, int nee, float clampk,
                         V3& first_albedo, Stats& st) {
    first_albedo = v3(1.0f, 1.0f, 1.0f);
    V3 radiance = v3(0, 0, 0);
    V3 thr = v3(1.0f, 1.0f, 1.0f);
    bool last_diffuse = false;
    st.camera_paths++;
    for (int bounce = 0; bounce < 6; ++bounce) {
        const Hit hit = traverse_ordered(sc, ro, rd, st);
        if (!hit.valid) break;
        const rc_material& m = sc.mats[hit.mat];
        st.material_fetches++;
        const V3 albedo = ld3(m.albedo);
        const V3 n = dot(rd, hit.normal) < 0.0f ? hit.normal : neg(hit.normal);
        if (bounce == 0) first_albedo = (m.transmission > 0.5f) ? v3(1.0f, 1.0f, 1.0f) : albedo;
        if (!last_diffuse) radiance = add(radiance, mul(mul(thr, ld3(m.emission)), m.emission_strength));
        if (bounce >= 2) {
            float survive = gmax(albedo.x, gmax(albedo.y, albedo.z));
            if (m.metallic > 0.5f || m.transmission > 0.5f) survive = 0.95f;
            survive = gclamp(survive, 0.01f, 0.95f);
            if (rnd(seed) > survive) break;
            thr = dv(thr, survive);
        }
        if (m.transmission > 0.5f) {
            const bool entering = dot(rd, hit.normal) < 0.0f;
            const float eta = entering ? (1.0f / m.ior) : m.ior;
            const float cosI = fabs_(dot(rd, n));
            float r0 = (1.0f - m.ior) / (1.0f + m.ior);
            r0 *= r0;
            const float F = r0 + (1.0f - r0) * rcx_powf(gclamp(1.0f - cosI, 0.0f, 1.0f), 5.0f);
            if (rnd(seed) < F) {
                rd = reflect(rd, n);
                ro = add(hit.pos, mul(rd, 2e-3f));
            } else {
                V3 refr = refract(rd, n, eta);
                if (dot(refr, refr) < 0.001f) refr = reflect(rd, n);
                rd = normalize(refr);
                ro = add(hit.pos, mul(rd, 2e-3f));
            }
            thr = mul(thr, albedo);
            last_diffuse = false;
        } else if (m.metallic > 0.5f) {
            const V3 wo = neg(rd);
            const float alpha = gmax(m.roughness, 1e-3f);
            const V3 up3 = fabs_(n.y) < 0.9999f ? v3(0.0f, 1.0f, 0.0f) : v3(1.0f, 0.0f, 0.0f);
            const V3 T = normalize(cross(up3, n));
            const V3 B = cross(n, T);
            const V3 wol = v3(dot(wo, T), dot(wo, n), dot(wo, B));
            const float u1 = rnd(seed);
            const float u2 = rnd(seed);
            const V3 hl = sample_ggx_vndf(wol, alpha, u1, u2);
            const V3 h = normalize(add(add(mul(T, hl.x), mul(n, hl.y)), mul(B, hl.z)));
            rd = reflect(neg(wo), h);
            if (dot(rd, n) <= 0.0f) rd = reflect(neg(wo), n);
            const float NdotL = gmax(dot(n, rd), 1e-4f);
            const float NdotV = gmax(dot(n, wo), 1e-4f);
            const float HdotV = gmax(dot(h, wo), 1e-4f);
            const float p5 = rcx_powf(1.0f - HdotV, 5.0f);
            const V3 F = add(albedo, mul(v3(1.0f - albedo.x, 1.0f - albedo.y, 1.0f - albedo.z), p5));
            const float G1 = smith_g1(NdotV, alpha);
            const float G2 = smith_g2(NdotL, NdotV, alpha);
            thr = mul(thr, mul(F, G2 / gmax(G1, 1e-7f)));
            ro = add(hit.pos, mul(n, 2e-3f));
            last_diffuse = false;
        } else {
            if (nee != 0) radiance = add(radiance, mul(thr, sample_direct_light(sc, hit.pos, n, albedo, clampk, seed, st)));
            const float u1 = rnd(seed);
            const float u2 = rnd(seed);
            rd = cosine_hemisphere(u1, u2, n);
            thr = mul(thr, albedo);
            ro = add(hit.pos, mul(n, 1e-3f));
            last_diffuse = true;
        }
    }
    return radiance;
}

/* pathtrace.comp:590-595 */
static void sample_gbuffer(const Scene& sc, V3 ro, V3 rd, float g[4], Stats& st) {
    const Hit hit = traverse_ordered(sc, ro, rd, st);
    if (!hit.valid) { g[0] = 0.0f; g[1] = 1.0f; g[2] = 0.0f; g[3] = 1e4f; return; }
    const V3 n = dot(rd, hit.normal) < 0.0f ? hit.normal : neg(hit.normal);
    g[0] = n.x; g[1] = n.y; g[2] = n.z; g[3] = hit.t;
}

/* pathtrace.comp:601-655 for one pixel and frames first..first+n-1. */
static void render_pixel(const Scene& sc, const Camera& cam, const rc_settings& set, int W, int H,
                         int px, int py, int first, int nspp, float* acc, uint16_t* gbuf,
                         uint16_t* galb, float* var, Stats& st) {
    const long i = (long)py * W + px;
    const bool lca = (fabs_(cam.lca[0]) + fabs_(cam.lca[2])) > 1e-4f;
    for (int f = first; f < first + nspp; ++f) {
        V3 rad, alb;
        if (lca) {
            float ch[3];
            V3 albs[3];
            for (int c = 0; c < 3; ++c) {
                uint32_t s = init_seed(px, py, f * 3 + c);
                V3 ro, rd;
                generate_ray(cam, W, H, px, py, s, cam.lca[c], ro, rd);
                const V3 r = trace_radiance(sc, ro, rd, s, set.nee_enabled, set.nee_firefly_clamp, albs[c], st);
                ch[c] = (c == 0) ? r.x : (c == 1 ? r.y : r.z);
            }
            rad = v3(ch[0], ch[1], ch[2]);
            alb = albs[1];
        } else {
            uint32_t s = init_seed(px, py, f);
            V3 ro, rd;
            generate_ray(cam, W, H, px, py, s, 0.0f, ro, rd);
            rad = trace_radiance(sc, ro, rd, s, set.nee_enabled, set.nee_firefly_clamp, alb, st);
        }
        if (bad(rad.x) || bad(rad.y) || bad(rad.z)) rad = v3(0, 0, 0);
        const float l = dot(rad, v3(0.2126f, 0.7152f, 0.0722f));
        const float l2 = l * l;
        if (f == 0) {
            acc[4 * i + 0] = rad.x; acc[4 * i + 1] = rad.y; acc[4 * i + 2] = rad.z; acc[4 * i + 3] = 1.0f;
            var[i] = l2;
            uint32_t gs = init_seed(px, py, 99991);
            V3 ro, rd;
            generate_ray(cam, W, H, px, py, gs, 0.0f, ro, rd);
            float g[4];
            sample_gbuffer(sc, ro, rd, g, st);
            for (int k = 0; k < 4; ++k) gbuf[4 * i + k] = float_to_half_rne(g[k]);
            galb[4 * i + 0] = float_to_half_rne(alb.x);
            galb[4 * i + 1] = float_to_half_rne(alb.y);
            galb[4 * i + 2] = float_to_half_rne(alb.z);
            galb[4 * i + 3] = float_to_half_rne(1.0f);
        } else {
            acc[4 * i + 0] = acc[4 * i + 0] + rad.x;
            acc[4 * i + 1] = acc[4 * i + 1] + rad.y;
            acc[4 * i + 2] = acc[4 * i + 2] + rad.z;
            acc[4 * i + 3] = acc[4 * i + 3] + 1.0f;
            var[i] = var[i] + l2;
        }
    }
}

/* photon_trace.comp:146-149 */
static float fresnel_schlick(float cos_theta, float ior) {
    float r0 = (1.0f - ior) / (1.0f + ior);
    r0 *= r0;
    return r0 + (1.0f - r0) * rcx_powf(gclamp(1.0f - cos_theta, 0.0f, 1.0f), 5.0f);
}

struct PhotonOut { bool stored; V3 pos, power, dir; };

/* photon_trace.comp:168-252 for one photon, without the hash insertion. */
static PhotonOut trace_photon(const Scene& sc, uint32_t gid, int N, int seed_u, Stats& st) {
    PhotonOut out; out.stored = false;
    uint32_t seed = photon_seed(gid, seed_u);
    const float u = rnd(seed);
    int sel = sc.light_count - 1;
    for (int i = 0; i < sc.light_count; ++i)
        if (u < sc.lights[i].cdf_weight) { sel = i; break; }
    const rc_light& L = sc.lights[sel];
    float r1 = rnd(seed);
    float r2 = rnd(seed);
    if (r1 + r2 > 1.0f) { r1 = 1.0f - r1; r2 = 1.0f - r2; }
    const V3 lv0 = ld3(L.v0);
    const V3 sp = add(add(lv0, mul(r1, sub(ld3(L.v1), lv0))), mul(r2, sub(ld3(L.v2), lv0)));
    const V3 en = normalize(ld3(L.normal));
    const float e1 = rnd(seed);
    const float e2 = rnd(seed);
    const V3 ed = cosine_hemisphere(e1, e2, en);
    const V3 em = ld3(L.emission);
    const float lum = dot(em, v3(0.299f, 0.587f, 0.114f));
    const float per = sc.total_power / (float)N;
    V3 power = (lum > 1e-6f) ? mul(dv(em, lum), per) : v3(per, per, per);
    V3 ro = add(sp, mul(en, 1e-3f));
    V3 rd = ed;
    bool spec = false;
    for (int b = 0; b < 8; ++b) {
        st.photon_rays++;
        const Hit hit = traverse_unordered(sc, ro, rd, st);
        if (!hit.valid) break;
        const rc_material& m = sc.mats[hit.mat];
        const V3 n = dot(rd, hit.normal) < 0.0f ? hit.normal : neg(hit.normal);
        if (m.transmission > 0.5f) {
            const bool entering = dot(rd, hit.normal) < 0.0f;
            const float eta = entering ? (1.0f / m.ior) : m.ior;
            const float cosI = fabs_(dot(rd, n));
            const float F = fresnel_schlick(cosI, m.ior);
            if (rnd(seed) < F) {
                rd = reflect(rd, n);
            } else {
                V3 refr = refract(rd, n, eta);
                if (dot(refr, refr) < 0.001f) refr = reflect(rd, n);
                rd = normalize(refr);
            }
            ro = add(hit.pos, mul(rd, 2e-3f));
            spec = true;
            continue;
        }
        if (m.metallic > 0.5f) {
            power = mul(power, ld3(m.albedo));
            rd = reflect(rd, n);
            ro = add(hit.pos, mul(n, 2e-3f));
            spec = true;
            continue;
        }
        if (spec) { out.stored = true; out.pos = hit.pos; out.power = power; out.dir = rd; }
        break;
    }
    return out;
}

/* photon_gather.comp:128-222 for one pixel. */
static V3 gather_pixel(const Scene& sc, const Camera& cam, int W, int H, int px, int py, float radius,
                       int hash_size, const rc_photon* ph, const int32_t* heads, const int32_t* next,
                       Stats& st) {
    const float aspect = (float)W / (float)H;
    const float nx = ((float)px + 0.5f) / (float)W * 2.0f - 1.0f;
    const float ny = ((float)py + 0.5f) / (float)H * 2.0f - 1.0f;
    const V3 rd = normalize(add(add(cam.fwd, mul(cam.right, nx * aspect * cam.tan_half)),
                                mul(cam.up, ny * cam.tan_half)));
    V3 ro = cam.pos, cur = rd, hit_pos = v3(0, 0, 0);
    int hit_mat = 0;
    bool found = false;
    for (int s = 0; s <= 6; ++s) {
        st.gather_rays++;
        const Hit hit = traverse_unordered(sc, ro, cur, st);
        if (!hit.valid) break;
        const rc_material& m = sc.mats[hit.mat];
        if (m.metallic <= 0.5f && m.transmission <= 0.5f) {
            found = true; hit_pos = hit.pos; hit_mat = hit.mat;
            break;
        }
        const V3 n = dot(cur, hit.normal) < 0.0f ? hit.normal : neg(hit.normal);
        if (m.transmission > 0.5f) {
            const bool entering = dot(cur, hit.normal) < 0.0f;
            const float eta = entering ? (1.0f / m.ior) : m.ior;
            V3 refr = refract(cur, n, eta);
            if (dot(refr, refr) < 0.001f) refr = reflect(cur, n);
            cur = normalize(refr);
        } else {
            cur = reflect(cur, n);
        }
        ro = add(hit.pos, mul(cur, 2e-3f));
    }
    if (!found) return v3(0, 0, 0);
    const float r = radius, r2 = r * r;
    const int ccx = (int)floor_(hit_pos.x / r), ccy = (int)floor_(hit_pos.y / r), ccz = (int)floor_(hit_pos.z / r);
    V3 caustic = v3(0, 0, 0);
    for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx) {
                const int h = cell_hash(ccx + dx, ccy + dy, ccz + dz, hash_size);
                int idx = heads[h];
                int safety = 0;
                while (idx >= 0 && safety < 512) {
                    const V3 d = sub(hit_pos, ld3(ph[idx].position));
                    const float d2 = dot(d, d);
                    if (d2 <= r2) {
                        const float w = 1.0f - d2 / r2;
                        caustic = add(caustic, mul(ld3(ph[idx].power), w));
                    }
                    idx = next[idx];
                    safety++;
                }
            }
    const float PI = 3.14159265358979f;
    V3 L = dv(mul(ld3(sc.mats[hit_mat].albedo), caustic), PI * r2);
    if (bad(L.x) || bad(L.y) || bad(L.z)) L = v3(0, 0, 0);
    return L;
}

static inline float luma709(V3 c) { return dot(c, v3(0.2126f, 0.7152f, 0.0722f)); }
static inline V3 rgb_at(const float* img, long i) { return v3(img[4 * i], img[4 * i + 1], img[4 * i + 2]); }
static inline V3 half3_at(const uint16_t* img, long i) {
    return v3(half_to_float(img[4 * i]), half_to_float(img[4 * i + 1]), half_to_float(img[4 * i + 2]));
}
static inline int wrap_repeat(int i, int n) { int m = i % n; return m < 0 ? m + n : m; }
static inline int wrap_clamp(int i, int n) { return i < 0 ? 0 : (i >= n ? n - 1 : i); }

/* post/atrous_denoise.frag:50-122 for one pixel. */
static void atrous_pixel(const float* col, const uint16_t* gbuf, const uint16_t* galb, const float* var,
                         int W, int H, int x, int y, int step, float sc_, float sn, float sd, int N_,
                         float exposure, float* out) {
    static const float hk[5] = {1.0f / 16.0f, 1.0f / 4.0f, 3.0f / 8.0f, 1.0f / 4.0f, 1.0f / 16.0f};
    const long ci = (long)y * W + x;
    const V3 c_norm = half3_at(gbuf, ci);
    const float c_depth = half_to_float(gbuf[4 * ci + 3]);
    const V3 c_col = rgb_at(col, ci);
    float* o = out + 4 * ci;
    if (c_depth > 9000.0f) { o[0] = c_col.x; o[1] = c_col.y; o[2] = c_col.z; o[3] = 1.0f; return; }
    const V3 c_alb = half3_at(galb, ci);
    const bool has_alb = luma709(c_alb) > 0.02f;
    const V3 c_irr = has_alb ? dv(c_col, gmax(c_alb, v3(0.01f, 0.01f, 0.01f))) : c_col;
    const float N = (float)(N_ > 1 ? N_ : 1);
    const float sum_l2 = var[ci];
    const float mean_l = luma709(dv(c_col, gmax(exposure, 1e-4f)));
    const float variance = gmax(0.0f, sum_l2 / N - mean_l * mean_l);
    const float var_denom = sc_ * sc_ * variance + 1e-6f;
    V3 irr_sum = v3(0, 0, 0);
    float w_sum = 0.0f;
    const float c_logl = rcx_logf(luma709(c_irr) + 1e-3f);
    for (int j = -2; j <= 2; ++j) {
        for (int i = -2; i <= 2; ++i) {
            const int tx = x + i * step, ty = y + j * step;
            const long ri = (long)wrap_repeat(ty, H) * W + wrap_repeat(tx, W);
            const long ki = (long)wrap_clamp(ty, H) * W + wrap_clamp(tx, W);
            const V3 n2 = half3_at(gbuf, ri);
            const float dep2 = half_to_float(gbuf[4 * ri + 3]);
            const V3 col2 = rgb_at(col, ki);
            const V3 alb2 = half3_at(galb, ri);
            const V3 irr2 = (luma709(alb2) > 0.02f) ? dv(col2, gmax(alb2, v3(0.01f, 0.01f, 0.01f))) : col2;
            const float hw = hk[i + 2] * hk[j + 2];
            const float wn = rcx_powf(gmax(0.0f, dot(c_norm, n2)), sn);
            const float dd = (c_depth - dep2) / (c_depth + 0.001f);
            const float wd = rcx_expf(-(dd * dd) / (sd * sd + 1e-6f));
            const float ld = c_logl - rcx_logf(luma709(irr2) + 1e-3f);
            const float wc = rcx_expf(-(ld * ld) / var_denom);
            const float w = hw * wn * wd * wc;
            irr_sum = add(irr_sum, mul(irr2, w));
            w_sum += w;
        }
    }
    const V3 res_irr = (w_sum > 1e-6f) ? dv(irr_sum, w_sum) : c_irr;
    const V3 res = has_alb ? mul(res_irr, c_alb) : res_irr;
    o[0] = res.x; o[1] = res.y; o[2] = res.z; o[3] = 1.0f;
}

static void set_threads(int n) { omp_set_num_threads(n > 0 ? n : omp_get_num_procs()); }

static void stats_out(const Stats& s, uint64_t* out) {
    if (!out) return;
    out[0] = s.camera_paths; out[1] = s.closest_rays; out[2] = s.shadow_rays; out[3] = s.photon_rays;
    out[4] = s.gather_rays; out[5] = s.node_tests; out[6] = s.tri_tests; out[7] = s.closest_hits;
    out[8] = s.material_fetches; out[9] = s.light_fetches;
}

}  // namespace oracle

using namespace oracle;

extern "C" {

/* ---- known-answer helpers ---- */
uint32_t or_pcg_next(uint32_t* state) { return pcg(*state); }
float or_rand(uint32_t* state) { return rnd(*state); }
uint32_t or_init_seed(int px, int py, int frame) { return init_seed(px, py, frame); }
uint32_t or_photon_seed(uint32_t idx, int seed) { return photon_seed(idx, seed); }
int or_cell_hash(int cx, int cy, int cz, int hash_size) { return cell_hash(cx, cy, cz, hash_size); }
int or_intersect_triangle(const float* ro, const float* rd, const rc_triangle* tri, float* t_uv) {
    float t, u, v;
    const bool h = hit_triangle(ld3(ro), ld3(rd), *tri, t, u, v);
    if (h) { t_uv[0] = t; t_uv[1] = u; t_uv[2] = v; }
    return h ? 1 : 0;
}
int or_intersect_aabb(const float* ro, const float* rd, const rc_bvh_node* node, float* tmin) {
    const V3 inv = dv(v3(1.0f, 1.0f, 1.0f), ld3(rd));
    return hit_aabb(ld3(ro), inv, *node, *tmin) ? 1 : 0;
}
float or_sinf(float x) { return rcx_sinf(x); }
float or_cosf(float x) { return rcx_cosf(x); }
float or_expf(float x) { return rcx_expf(x); }
float or_logf(float x) { return rcx_logf(x); }
float or_powf(float x, float y) { return rcx_powf(x, y); }
uint16_t or_float_to_half(float f) { return float_to_half_rne(f); }
float or_half_to_float(uint16_t h) { return half_to_float(h); }

/* ---- Java host restatements ---- */
int or_tess_box(float cx, float cy, float cz, float hx, float hy, float hz, int mat, float rx, float ry,
                float rz, rc_triangle* out) {
    std::vector<rc_triangle> v;
    tess_box(cx, cy, cz, hx, hy, hz, mat, v);
    if (rx != 0.0f || ry != 0.0f || rz != 0.0f) rotate_about(v, 0, cx, cy, cz, rx, ry, rz);
    memcpy(out, v.data(), v.size() * sizeof(rc_triangle));
    return (int)v.size();
}
int or_tess_sphere(float cx, float cy, float cz, float r, int mat, int stacks, int slices, float rx,
                   float ry, float rz, rc_triangle* out, int cap) {
    std::vector<rc_triangle> v;
    tess_sphere(cx, cy, cz, r, mat, stacks, slices, v);
    if (rx != 0.0f || ry != 0.0f || rz != 0.0f) rotate_about(v, 0, cx, cy, cz, rx, ry, rz);
    if ((int)v.size() > cap) return -1;
    memcpy(out, v.data(), v.size() * sizeof(rc_triangle));
    return (int)v.size();
}
int or_flat_triangles(const float* pos, int n, int mat, rc_triangle* out) {
    for (int i = 0; i < n; ++i) {
        rc_triangle t;
        memset(&t, 0, sizeof(t));
        for (int k = 0; k < 3; ++k) { t.v0[k] = pos[9 * i + k]; t.v1[k] = pos[9 * i + 3 + k]; t.v2[k] = pos[9 * i + 6 + k]; }
        t.mat_index = mat;
        with_flat_normal(t);
        out[i] = t;
    }
    return n;
}
/* Returns node count, or -1 when node_cap is too small. */
int or_build_bvh(const rc_triangle* in, int n, rc_triangle* out_tris, rc_bvh_node* out_nodes, int node_cap) {
    std::vector<rc_triangle> t(in, in + n);
    std::vector<rc_bvh_node> nodes;
    build_bvh(t, nodes);
    if ((int)nodes.size() > node_cap) return -1;
    memcpy(out_tris, t.data(), t.size() * sizeof(rc_triangle));
    memcpy(out_nodes, nodes.data(), nodes.size() * sizeof(rc_bvh_node));
    return (int)nodes.size();
}
int or_build_lights(const rc_triangle* tris, int n, const rc_material* mats, rc_light* out, int cap,
                    float* total_power) {
    std::vector<rc_triangle> t(tris, tris + n);
    std::vector<rc_light> L;
    float tp = 0.0f;
    build_lights(t, mats, L, tp);
    *total_power = tp;
    if ((int)L.size() > cap) return -1;
    if (!L.empty()) memcpy(out, L.data(), L.size() * sizeof(rc_light));
    return (int)L.size();
}
/* ThinLensCamera.java:41-68 */
void or_thin_lens(float focal_mm, float fstop, float* lens_radius, float* tan_half) {
    const float fm = focal_mm / 1000.0f;
    *lens_radius = fm / (2.0f * fstop);
    *tan_half = (float)tan(atan((double)(0.012f / fm)));
}
/* OrbitCamera.java:155-171,274-291 */
void or_orbit_basis(float theta, float phi, float radius, float tx, float ty, float tz, float* o) {
    const float sp = (float)sin((double)phi);
    const float ex = tx + radius * sp * (float)cos((double)theta);
    const float ey = ty + radius * (float)cos((double)phi);
    const float ez = tz + radius * sp * (float)sin((double)theta);
    float fx = tx - ex, fy = ty - ey, fz = tz - ez;
    const float fl = (float)sqrt((double)(fx * fx + fy * fy + fz * fz));
    fx /= fl; fy /= fl; fz /= fl;
    float rx = fy * 0.0f - fz * 1.0f, ry = fz * 0.0f - fx * 0.0f, rz = fx * 1.0f - fy * 0.0f;
    const float rl = (float)sqrt((double)(rx * rx + ry * ry + rz * rz));
    rx /= rl; ry /= rl; rz /= rl;
    o[0] = ex; o[1] = ey; o[2] = ez;
    o[3] = fx; o[4] = fy; o[5] = fz;
    o[6] = rx; o[7] = ry; o[8] = rz;
    o[9] = ry * fz - rz * fy; o[10] = rz * fx - rx * fz; o[11] = rx * fy - ry * fx;
}
/* SPPMManager.java:170-173 */
float or_sppm_next_radius(float r, int it, float alpha) {
    const float num = (float)it + alpha;
    return r * (float)sqrt((double)num / ((double)it + 1.0));
}
/* KeyframeTrack.java:102-178 */
float or_keyframe_eval(const float* tm, const float* val, const int32_t* interp, int n, float time, float def) {
    if (n == 0) return def;
    if (n == 1) return val[0];
    if (time <= tm[0]) return val[0];
    if (time >= tm[n - 1]) return val[n - 1];
    int hi = 1;
    while (hi < n && tm[hi] < time) hi++;
    const int lo = hi - 1;
    const float t = (time - tm[lo]) / (tm[hi] - tm[lo]);
    if (interp[lo] == 0) return val[lo];
    if (interp[lo] == 1) return val[lo] + (val[hi] - val[lo]) * t;
    const float dt = tm[hi] - tm[lo];
    const float m0 = lo > 0 ? (val[hi] - val[lo - 1]) / (tm[hi] - tm[lo - 1]) : (val[hi] - val[lo]) / dt;
    const float m1 = hi < n - 1 ? (val[hi + 1] - val[lo]) / (tm[hi + 1] - tm[lo]) : (val[hi] - val[lo]) / dt;
    const float t2 = t * t, t3 = t2 * t;
    const float h00 = 2.0f * t3 - 3.0f * t2 + 1.0f;
    const float h10 = t3 - 2.0f * t2 + t;
    const float h01 = -2.0f * t3 + 3.0f * t2;
    const float h11 = t3 - t2;
    return h00 * val[lo] + h10 * dt * m0 + h01 * val[hi] + h11 * dt * m1;
}

/* ---- shader restatements ---- */

/* Renderer.render repeated nspp times (frames first..first+nspp-1), over
 * pixel rows [row0, row1) -- a row subset bounds CPU-baseline samples. */
int or_render(const rc_triangle* tris, const rc_bvh_node* nodes, const rc_material* mats,
              const rc_light* lights, int light_count, float total_power, const rc_camera* cam_c,
              const rc_settings* set, int W, int H, int first, int nspp, int row0, int row1,
              float* accum, uint16_t* gbuf, uint16_t* galb, float* var, uint64_t* stats_out10,
              int nthreads) {
    const Scene sc{tris, nodes, mats, lights, light_count, total_power};
    const Camera cam = camera_from(cam_c);
    if (row1 <= 0 || row1 > H) row1 = H;
    if (row0 < 0) row0 = 0;
    Stats total;
    set_threads(nthreads);
#pragma omp parallel
    {
        Stats local;
#pragma omp for schedule(dynamic, 1)
        for (int y = row0; y < row1; ++y)
            for (int x = 0; x < W; ++x)
                render_pixel(sc, cam, *set, W, H, x, y, first, nspp, accum, gbuf, galb, var, local);
#pragma omp critical
        total.add(local);
    }
    stats_out(total, stats_out10);
    return 0;
}

/* SPPMManager.tracePhotons incl. PhotonMap.clear; deterministic insertion. */
int or_photon_trace(const rc_triangle* tris, const rc_bvh_node* nodes, const rc_material* mats,
                    const rc_light* lights, int light_count, float total_power, int N, float radius,
                    int seed, int hash_size, rc_photon* photons, int32_t* heads, int32_t* next,
                    uint32_t* counter, uint64_t* stats_out10, int nthreads) {
    const Scene sc{tris, nodes, mats, lights, light_count, total_power};
    for (int i = 0; i < hash_size; ++i) heads[i] = -1;
    *counter = 0;
    if (light_count == 0 || N <= 0) { stats_out(Stats(), stats_out10); return 0; }
    std::vector<PhotonOut> res((size_t)N);
    Stats total;
    set_threads(nthreads);
#pragma omp parallel
    {
        Stats local;
#pragma omp for schedule(dynamic, 1024)
        for (int g = 0; g < N; ++g) res[g] = trace_photon(sc, (uint32_t)g, N, seed, local);
#pragma omp critical
        total.add(local);
    }
    uint32_t cnt = 0;
    for (int g = 0; g < N; ++g) {
        if (!res[g].stored) continue;
        const uint32_t idx = cnt++;
        if (idx >= (uint32_t)N) continue;
        const V3 p = res[g].pos;
        const int h = cell_hash((int)floor_(p.x / radius), (int)floor_(p.y / radius), (int)floor_(p.z / radius),
                                hash_size);
        const int old = heads[h];
        heads[h] = (int)idx;
        next[idx] = old;
        rc_photon& ph = photons[idx];
        memset(&ph, 0, sizeof(ph));
        ph.position[0] = p.x; ph.position[1] = p.y; ph.position[2] = p.z;
        ph.power[0] = res[g].power.x; ph.power[1] = res[g].power.y; ph.power[2] = res[g].power.z;
        ph.dir[0] = res[g].dir.x; ph.dir[1] = res[g].dir.y; ph.dir[2] = res[g].dir.z;
    }
    *counter = cnt;
    stats_out(total, stats_out10);
    return 0;
}

/* SPPMManager.gatherRadiance; weight scales the added radiance. */
int or_photon_gather(const rc_triangle* tris, const rc_bvh_node* nodes, const rc_material* mats,
                     const rc_camera* cam_c, int W, int H, float radius, int hash_size,
                     const rc_photon* photons, const int32_t* heads, const int32_t* next,
                     float weight, float* accum, uint64_t* stats_out10, int nthreads) {
    const Scene sc{tris, nodes, mats, nullptr, 0, 0.0f};
    const Camera cam = camera_from(cam_c);
    Stats total;
    set_threads(nthreads);
#pragma omp parallel
    {
        Stats local;
#pragma omp for schedule(dynamic, 1)
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x) {
                V3 L = gather_pixel(sc, cam, W, H, x, y, radius, hash_size, photons, heads, next, local);
                if (weight != 1.0f) L = mul(L, weight);
                float* a = accum + 4 * ((long)y * W + x);
                a[0] = a[0] + L.x; a[1] = a[1] + L.y; a[2] = a[2] + L.z; a[3] = a[3] + 0.0f;
            }
#pragma omp critical
        total.add(local);
    }
    stats_out(total, stats_out10);
    return 0;
}

/* p00_normalize.frag:18-24 */
int or_p00(const float* accum, int W, int H, int total, float exposure, float* out, int nthreads) {
    const float n = (float)(total > 1 ? total : 1);
    set_threads(nthreads);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)W * H; ++i) {
        out[4 * i + 0] = accum[4 * i + 0] / n * exposure;
        out[4 * i + 1] = accum[4 * i + 1] / n * exposure;
        out[4 * i + 2] = accum[4 * i + 2] / n * exposure;
        out[4 * i + 3] = 1.0f;
    }
    return 0;
}

/* display.frag:11-41 on the export path (export/RenderPipeline.java:244-259)
 * and the GL_RGBA8 store + FrameExporter read-back (FrameExporter.java:51-80):
 * ACES fit, sRGB encode by the shader's mix/step, each channel stored as
 * round(clamp(v, 0, 1) * 255) (NaN as 0), alpha 255, rows written top first
 * (stbi_flip_vertically_on_write). */
static inline float aces_fit(float x) {
    const float a = 2.51f, b = 0.03f, c = 2.43f, d = 0.59f, e = 0.14f;
    return gclamp((x * (a * x + b)) / (x * (c * x + d) + e), 0.0f, 1.0f);
}
static inline float linear_to_srgb(float c) {
    const float t = c < 0.0031308f ? 0.0f : 1.0f;   /* step(0.0031308, c) */
    const float lo = 12.92f * c;
    const float hi = 1.055f * rcx_powf(c, 1.0f / 2.4f) - 0.055f;
    return lo * (1.0f - t) + hi * t;                /* mix(lo, hi, t) */
}
static inline uint8_t unorm8(float v) {
    if (!(v == v)) v = 0.0f;
    v = v < 0.0f ? 0.0f : (v > 1.0f ? 1.0f : v);
    return (uint8_t)floor_(v * 255.0f + 0.5f);
}

int or_display(const float* color, int W, int H, int total, float exposure, uint8_t* out, int nthreads) {
    const float n = (float)(total > 1 ? total : 1);
    set_threads(nthreads);
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            const float* c = color + 4 * ((long)y * W + x);
            uint8_t* o = out + 4 * ((long)(H - 1 - y) * W + x);
            for (int k = 0; k < 3; ++k) o[k] = unorm8(linear_to_srgb(aces_fit(c[k] / n * exposure)));
            o[3] = 255;
        }
    return 0;
}

/* One à-trous pass. */
int or_atrous_pass(const float* col, const uint16_t* gbuf, const uint16_t* galb, const float* var, int W,
                   int H, int step, float sc_, float sn, float sd, int N, float exposure, float* out,
                   int nthreads) {
    set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1)
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x)
            atrous_pixel(col, gbuf, galb, var, W, H, x, y, step, sc_, sn, sd, N, exposure, out);
    return 0;
}

/* AtrousDenoiser.denoise with PostProcessStack gating (p00 first). */
int or_denoise(const float* accum, const uint16_t* gbuf, const uint16_t* galb, const float* var, int W,
               int H, int total, const rc_atrous_params* p, float* out, int nthreads) {
    std::vector<float> a((size_t)W * H * 4), b((size_t)W * H * 4);
    or_p00(accum, W, H, total, p->exposure, a.data(), nthreads);
    const bool over = p->max_spp > 0 && total > p->max_spp;
    if (p->enabled && !over) {
        int passes = p->iterations < 1 ? 1 : (p->iterations > 5 ? 5 : p->iterations);
        const int n = total > 1 ? total : 1;
        for (int i = 0; i < passes; ++i) {
            or_atrous_pass(a.data(), gbuf, galb, var, W, H, 1 << i, p->sigma_color, p->sigma_normal,
                           p->sigma_depth, n, p->exposure, b.data(), nthreads);
            a.swap(b);
        }
    }
    memcpy(out, a.data(), a.size() * sizeof(float));
    return 0;
}

}  /* extern "C" */
