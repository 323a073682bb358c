// wavefront.cu -- the path tracer as a sequence of short kernels over path
// queues (pathtrace.comp semantics, one kernel per stage instead of one
// invocation per pixel).
//
// Per chunk of paths (all pixels x some samples x 1 or 3 lens channels):
//   wf_generate    camera rays (pathtrace.comp:401-439) -> ray queue 0
//   for bounce 0..5:
//     wf_trace     closest hit for the ray queue AND the visibility test of
//                  the shadow rays the previous shade produced (one launch,
//                  two queues: a warp only ever holds one kind of ray)
//     wf_sort      misses finish their path; hits go to material queues
//                  (diffuse / metal or glass) by warp ballot and block append
//     wf_shade     emission, Russian roulette, BSDF, NEE light sample
//                  (pathtrace.comp:454-585) over the material queues, so a
//                  warp runs one BSDF branch; survivors -> next ray queue,
//                  NEE rays -> shadow queue
//   wf_trace       the last bounce's shadow rays
//   wf_accumulate  per pixel, the samples in frame order, LCA channel
//                  assembly, NaN scrub, variance, G-buffer on frame 0
//                  (pathtrace.comp:601-655)
// Queues are compacted with warp ballots: one shared-memory atomic per warp
// and one global atomicAdd per block (generate, shade) or per warp (trace).
// Path arithmetic is the megakernel's, operation for operation, and the
// accumulation adds samples in frame order, so exact-math results stay
// bit-identical to the oracle.  Kernels are grid-stride loops over device-side
// queue lengths, launched with a grid that fills the GPU once.
#include <mutex>

#include "device_common.cuh"
#include "dyn_trace.cuh"

namespace rc {
namespace RC_NS {

// Block-wide appends to two queues with counters la and lb (lb unused when
// no thread wants it): one shared-memory atomic per warp and one global
// atomicAdd per queue per block.  Appends to one global counter serialise in
// L2 (about 1 ns each), so one per warp bounded the generate and shade
// kernels.  Every thread of the block calls it the same number of times;
// `sh.cnt` starts at zero.  Returns each wanting thread's queue slot; a
// warp's slots are consecutive.
struct BlockAppend {
    unsigned int cnt[2];
    unsigned int base[2];
};

DI void block_append(BlockAppend& sh, bool wa, bool wb, unsigned int* la, unsigned int* lb,
                     unsigned int& slot_a, unsigned int& slot_b) {
    const unsigned int FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const unsigned int ma = __ballot_sync(FULL, wa), mb = __ballot_sync(FULL, wb);
    unsigned int oa = 0u, ob = 0u;
    if (lane == 0) {
        if (ma) oa = atomicAdd(&sh.cnt[0], (unsigned int)__popc(ma));
        if (mb) ob = atomicAdd(&sh.cnt[1], (unsigned int)__popc(mb));
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned int ca = sh.cnt[0], cb = sh.cnt[1];
        sh.base[0] = ca ? atomicAdd(la, ca) : 0u;
        sh.base[1] = cb ? atomicAdd(lb, cb) : 0u;
        sh.cnt[0] = 0u;
        sh.cnt[1] = 0u;
    }
    __syncthreads();
    oa = __shfl_sync(FULL, oa, 0);
    ob = __shfl_sync(FULL, ob, 0);
    const unsigned int below = (1u << lane) - 1u;
    slot_a = sh.base[0] + oa + (unsigned int)__popc(ma & below);
    slot_b = sh.base[1] + ob + (unsigned int)__popc(mb & below);
}

struct PathId {
    int px, py, channel, sample;
    bool valid;
};

// The segment holding chunk path p (binary search over path_base).
DI int seg_index(const WaveArgs& A, int p) {
    if (!A.segs) return 0;
    int lo = 0, hi = A.nsegs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(&A.segs[mid].path_base) <= p)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

DI const FrameSeg& seg_at(const WaveArgs& A, int i) { return A.segs ? A.segs[i] : A.one; }

DI PathId decode(const WaveArgs& A, const FrameSeg& sg, int p) {
    PathId id;
    const int local = p - sg.path_base;
    const int j = local % A.npix;
    const int k = local / A.npix;
    id.channel = k % sg.channels;
    id.sample = k / sg.channels;
    const int tile = j >> 5, lane = j & 31;
    id.px = (tile % A.tiles_x) * 8 + (lane & 7);
    id.py = (tile / A.tiles_x) * 4 + (lane >> 3);
    id.valid = id.px < A.width && id.py < A.height;
    return id;
}

DI bool lca_on(const CamParams& c) { return (fabs_(c.lca[0]) + fabs_(c.lca[2])) > 1e-4f; }

__global__ void __launch_bounds__(256) wf_generate(WaveArgs A) {
    const WaveBuffers& B = A.wb;
    __shared__ BlockAppend sh;
    // aperture corners for the first segment's blade count (segments with
    // another count compute theirs directly)
    __shared__ float2 ngon[kNgonTab];
    const int tab_n = seg_at(A, 0).cam.blades;
    const bool tab_ok = ngon_table_ok(tab_n);
    if (tab_ok) fill_ngon_table(ngon, tab_n);
    if (threadIdx.x == 0) sh.cnt[0] = sh.cnt[1] = 0u;
    __syncthreads();
    uint32_t paths = 0;
    for (int p0 = blockIdx.x * blockDim.x; p0 < A.paths; p0 += gridDim.x * blockDim.x) {
        const int p = p0 + threadIdx.x;
        bool want = false;
        const FrameSeg& sg = seg_at(A, seg_index(A, p < A.paths ? p : A.paths - 1));
        const PathId id = decode(A, sg, p);
        const bool lca = sg.channels == 3;
        if (p < A.paths && id.valid) {
            const int f = sg.first_frame + id.sample;
            uint32_t s = init_seed(id.px, id.py, lca ? f * 3 + id.channel : f);
            const Ray r = generate_ray(sg.cam, A.width, A.height, id.px, id.py, s,
                                       lca ? sg.cam.lca[id.channel] : 0.0f,
                                       tab_ok && sg.cam.blades == tab_n ? ngon : nullptr);
            B.o[p] = make_float4(r.o.x, r.o.y, r.o.z, 0.0f);
            B.d[p] = make_float4(r.d.x, r.d.y, r.d.z, 0.0f);
            // throughput (1, 1, 1) and radiance 0 are implied at bounce 0:
            // wf_shade takes them as constants instead of reading them
            B.seed[p] = s;
            want = true;
            ++paths;
        }
        unsigned int slot, unused;
        block_append(sh, want, false, B.qlen + 0, nullptr, slot, unused);
        if (want) B.rq[0][slot] = p;
    }
    const unsigned int n = __reduce_add_sync(__activemask(), paths);
    if ((threadIdx.x & 31) == 0 && n) atomicAdd(&A.counters->camera_paths, (unsigned long long)n);
}

// Shadow records (3 float4 per queue slot): origin and tmax, direction and
// path index, and (throughput * light term, flags).  The flags hold the
// path's last-bounce bit and, per throughput channel, what throughput * 0
// is (0: +0, 1: -0, 2: NaN), so the occluded case adds what the reference's
// `radiance += throughput * 0` adds.
DI int zero_code(float x) { return bad(x) ? 2 : (__float_as_int(x) < 0 ? 1 : 0); }
DI float zero_of(int code) {
    return code == 2 ? __int_as_float(0x7fffffff) : (code == 1 ? -0.0f : 0.0f);
}

// radiance += throughput * sampleDirectLight(...), the light term 0 when
// occluded (pathtrace.comp:341-395 as traceRadiance adds it); the path's
// final radiance when this was its last bounce.
DI void shadow_add(const WaveBuffers& B, int p, bool vis, const float4 sq) {
    const int fl = __float_as_int(sq.w);
    const float3 add = vis ? xyz(sq) : f3(zero_of((fl >> 1) & 3), zero_of((fl >> 3) & 3), zero_of((fl >> 5) & 3));
    const float3 r = xyz(B.rad[p]) + add;
    B.rad[p] = make_float4(r.x, r.y, r.z, 0.0f);
    if (fl & 1) B.res[p] = make_float4(r.x, r.y, r.z, 0.0f);
}

// Closest-hit traversal of ray queue rq[bounce&1] followed (same index
// space) by the visibility tests of shadow queue sq[(bounce+1)&1].
template <bool kShadowAtParent>
__global__ void __launch_bounds__(256) wf_trace(WaveArgs A) {
    const WaveBuffers& B = A.wb;
    const int cur = A.bounce & 1;
    const int prev = cur ^ 1;
    const unsigned int nr = A.bounce < 6 ? B.qlen[cur] : 0u;
    const unsigned int ns = B.qlen[2 + prev];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        B.qlen[prev] = 0u;      // the ray queue shade(bounce) fills
        B.qlen[2 + cur] = 0u;   // the shadow queue shade(bounce) fills
        B.qlen[5] = 0u;         // the material queues sort(bounce) fills
        B.qlen[6] = 0u;
    }
    Guard g = {0u, 0u, 0u};
    uint32_t closest = 0, shadow = 0;
    const unsigned int total = nr + ns;
    for (unsigned int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        if (i < nr) {
            const int p = B.rq[cur][i];
            const Ray r = make_ray(xyz(B.o[p]), xyz(B.d[p]));
            const Hit h = closest_hit<kShadowAtParent>(A.scene, r, g);
            B.hit[p] = make_float4(h.t, h.u, h.v, __int_as_float(h.prim));
            ++closest;
        } else {
            const int k = (int)(i - nr);
            const float4* rec = B.srec[prev] + 3 * k;
            const float4 so = rec[0], sd = rec[1], sq = rec[2];
            const int p = __float_as_int(sd.w);
            const bool vis = unoccluded<kShadowAtParent>(A.scene, make_ray(xyz(so), xyz(sd)), so.w, g);
            ++shadow;
            shadow_add(B, p, vis, sq);
        }
    }
    const unsigned int active = __activemask();
    const unsigned int c = __reduce_add_sync(active, closest);
    const unsigned int s = __reduce_add_sync(active, shadow);
    const unsigned int n = __reduce_add_sync(active, g.nodes);
    const unsigned int t = __reduce_add_sync(active, g.tris);
    const unsigned int gf = __reduce_or_sync(active, g.flags);
    if ((threadIdx.x & 31) == 0) {
        if (c) atomicAdd(&A.counters->closest_rays, (unsigned long long)c);
        if (s) atomicAdd(&A.counters->shadow_rays, (unsigned long long)s);
        if (n) atomicAdd(&A.counters->node_tests, (unsigned long long)n);
        if (t) atomicAdd(&A.counters->tri_tests, (unsigned long long)t);
        if (gf) atomicOr(&A.counters->error_word, gf);
    }
}

// The bounce-0 albedo image is written by the G channel's path (or the only
// one) of frame 0.
DI bool albedo_path(const WaveArgs& A, int p, PathId& id, ushort4*& galb) {
    const FrameSeg& sg = seg_at(A, seg_index(A, p));
    id = decode(A, sg, p);
    galb = sg.img.galb;
    return sg.first_frame + id.sample == 0 && id.channel == (sg.channels == 3 ? 1 : 0);
}

// A path whose ray missed ends: its radiance so far is final; on bounce 0
// the albedo image gets (1,1,1) (pathtrace.comp:476-479, the first-hit
// albedo preset).
DI void finish_miss(const WaveArgs& A, int p, int b) {
    const WaveBuffers& B = A.wb;
    PathId id;
    ushort4* galb;
    if (b == 0 && albedo_path(A, p, id, galb))
        galb[(long)id.py * A.width + id.px] = to_half4(1.0f, 1.0f, 1.0f, 1.0f);
    B.res[p] = b == 0 ? make_float4(0.0f, 0.0f, 0.0f, 0.0f) : B.rad[p];
}

// Material queues (rc_tuning.material_queues): between trace and shade, a
// path whose ray missed ends here (finish_miss) and a hit joins the
// material queue of its surface -- diffuse from the front of mq, metal or
// glass (pathtrace.comp:504-566) from the back -- so wf_shade's warps each
// run one BSDF branch.  Appends are block-aggregated (block_append).
__global__ void __launch_bounds__(256) wf_sort(WaveArgs A) {
    const WaveBuffers& B = A.wb;
    const DeviceScene& S = A.scene;
    const int cur = A.bounce & 1;
    const int b = A.bounce;
    const unsigned int n = B.qlen[cur];
    __shared__ BlockAppend sh;
    if (threadIdx.x == 0) sh.cnt[0] = sh.cnt[1] = 0u;
    __syncthreads();
    // block-uniform trip count: the appends synchronise the block
    for (unsigned int i0 = blockIdx.x * blockDim.x; i0 < n; i0 += gridDim.x * blockDim.x) {
        const unsigned int i = i0 + threadIdx.x;
        bool diffuse = false, specular = false;
        int p = 0;
        if (i < n) {
            p = B.rq[cur][i];
            const int prim = __float_as_int(B.hit[p].w);
            if (prim < 0) {
                finish_miss(A, p, b);
            } else {
                const int m = __float_as_int(__ldg(S.tri_shade + 3 * prim).w);
                // wf_shade's branch tests: transmission > 0.5 glass, metallic > 0.5 metal
                const float metallic = __ldg(S.materials + 4 * m + 0).w;
                const float transmission = __ldg(S.materials + 4 * m + 2).z;
                specular = metallic > 0.5f || transmission > 0.5f;
                diffuse = !specular;
            }
        }
        unsigned int slot_d, slot_s;
        block_append(sh, diffuse, specular, B.qlen + 5, B.qlen + 6, slot_d, slot_s);
        if (diffuse) B.mq[slot_d] = p;
        if (specular) B.mq[B.capacity - 1 - (int)slot_s] = p;
    }
}

// One bounce of pathtrace.comp's traceRadiance for every path in ray queue
// rq[bounce&1] whose closest hit wf_trace has stored (misses end here), or,
// with material queues (kMQ), for the hits wf_sort queued from it.
// Registers capped: the kernel streams path state and waits on memory, so
// resident warps matter more than registers.  Fast build 64 (no spills
// since the radiance is read lazily; 56 spills): 8 blocks of 128 threads
// per SM, 14.8 ms per export frame vs 15.3 at a 72 cap.  Exact build 72
// (64 spills 40 bytes).
template <bool kMQ>
__global__ void __maxnreg__(RC_EXACT ? 72 : 64) wf_shade(WaveArgs A) {
    const WaveBuffers& B = A.wb;
    const DeviceScene& S = A.scene;
    const int cur = A.bounce & 1;
    const int nxt = cur ^ 1;
    const int b = A.bounce;
    const bool last = b == 5;
    const unsigned int nd = kMQ ? B.qlen[5] : B.qlen[cur];
    const unsigned int n = kMQ ? nd + B.qlen[6] : nd;
    if (blockIdx.x == 0 && threadIdx.x == 0) B.qlen[4] = 0u;  // work counter of the next trace
    __shared__ BlockAppend sh;
    if (threadIdx.x == 0) sh.cnt[0] = sh.cnt[1] = 0u;
    __syncthreads();
    uint32_t hits = 0, lights = 0;
    // block-uniform trip count: the appends at the bottom synchronise the block
    for (unsigned int i0 = blockIdx.x * blockDim.x; i0 < n; i0 += gridDim.x * blockDim.x) {
        const unsigned int i = i0 + threadIdx.x;
        {
            // the next item's path state, fetched into L2 while this one runs
            const unsigned int inext = i + gridDim.x * blockDim.x;
            if (inext < n) {
                const int pn = !kMQ ? B.rq[cur][inext]
                                    : (inext < nd ? B.mq[inext] : B.mq[B.capacity - 1 - (int)(inext - nd)]);
                asm volatile("prefetch.global.L2 [%0];" ::"l"(B.hit + pn));
                asm volatile("prefetch.global.L2 [%0];" ::"l"(B.o + pn));
                asm volatile("prefetch.global.L2 [%0];" ::"l"(B.d + pn));
                asm volatile("prefetch.global.L2 [%0];" ::"l"(B.seed + pn));
                if (b > 0) asm volatile("prefetch.global.L2 [%0];" ::"l"(B.thr + pn));
            }
        }
        bool cont = false, shadow_rec = false;
        float4 rec0, rec1, rec2;
        int p = 0;
        if (i < n) {
            p = !kMQ ? B.rq[cur][i] : (i < nd ? B.mq[i] : B.mq[B.capacity - 1 - (int)(i - nd)]);
            const float4 hv = B.hit[p];
            const int prim = __float_as_int(hv.w);
            // radiance so far: implied 0 on bounce 0, else read when first
            // needed (an add that can change it, or the path's end)
            float3 rad = f3(0.0f, 0.0f, 0.0f);
            bool rad_known = b == 0, rad_dirty = b == 0;
            // frame-0 albedo image: first hit of the G channel (or the only one)
            bool alb_path = false;
            PathId id;
            ushort4* galb = nullptr;
            if (b == 0) alb_path = albedo_path(A, p, id, galb);
            if (!kMQ && prim < 0) {
                finish_miss(A, p, b);
            } else {
                ++hits;
                const Ray ray = make_ray(xyz(B.o[p]), xyz(B.d[p]));
                Hit h;
                h.t = hv.x;
                h.u = hv.y;
                h.v = hv.z;
                h.prim = prim;
                const Surf sf = surface(S, ray, h);
                const Mat m = load_mat(S, sf.mat);
                const float3 rd = ray.d;
                const float3 nrm = dot(rd, sf.normal) < 0.0f ? sf.normal : -sf.normal;
                uint32_t seed = B.seed[p];
                const float4 thr4 = b == 0 ? make_float4(1.0f, 1.0f, 1.0f, 0.0f) : B.thr[p];
                float3 thr = xyz(thr4);
                const bool last_diffuse = thr4.w != 0.0f;
                if (alb_path) {
                    const float3 a = (m.transmission > 0.5f) ? f3(1.0f, 1.0f, 1.0f) : m.albedo;
                    galb[(long)id.py * A.width + id.px] = to_half4(a.x, a.y, a.z, 1.0f);
                }
                if (!last_diffuse) {
                    const float3 e = (thr * m.emission) * m.strength;
                    // rad + (+-0) is rad (rad is never -0); NaN != 0 too
                    if (e.x != 0.0f || e.y != 0.0f || e.z != 0.0f) {
                        if (!rad_known) rad = xyz(B.rad[p]);
                        rad = rad + e;
                        rad_known = rad_dirty = true;
                    }
                }
                bool alive = true;
                if (b >= 2) {
                    float survive = gmax(m.albedo.x, gmax(m.albedo.y, m.albedo.z));
                    if (m.metallic > 0.5f || m.transmission > 0.5f) survive = 0.95f;
                    survive = gclamp(survive, 0.01f, 0.95f);
                    if (rnd(seed) > survive) alive = false;
                    else thr = thr / survive;
                }
                float3 no = f3(0, 0, 0), nd = f3(0, 0, 0);
                bool nd_diffuse = false;
                if (alive) {
                    if (m.transmission > 0.5f) {
                        const bool entering = dot(rd, sf.normal) < 0.0f;
                        const float eta = entering ? (1.0f / m.ior) : m.ior;
                        const float cosI = fabs_(dot(rd, nrm));
                        float r0 = (1.0f - m.ior) / (1.0f + m.ior);
                        r0 *= r0;
                        const float F = r0 + (1.0f - r0) * pow5(gclamp(1.0f - cosI, 0.0f, 1.0f));
                        if (rnd(seed) < F) {
                            nd = reflect(rd, nrm);
                        } else {
                            float3 refr = refract(rd, nrm, eta);
                            if (dot(refr, refr) < 0.001f) refr = reflect(rd, nrm);
                            nd = normalize(refr);
                        }
                        no = sf.pos + nd * 2e-3f;
                        thr = thr * m.albedo;
                    } else if (m.metallic > 0.5f) {
                        const float3 wo = -rd;
                        const float alpha = gmax(m.roughness, 1e-3f);
                        const float3 up3 = fabs_(nrm.y) < 0.9999f ? f3(0.0f, 1.0f, 0.0f) : f3(1.0f, 0.0f, 0.0f);
                        const float3 T = normalize(cross(up3, nrm));
                        const float3 Bv = cross(nrm, T);
                        const float3 wol = f3(dot(wo, T), dot(wo, nrm), dot(wo, Bv));
                        const float u1 = rnd(seed);
                        const float u2 = rnd(seed);
                        const float3 hl = sample_ggx_vndf(wol, alpha, u1, u2);
                        const float3 hh = normalize(T * hl.x + nrm * hl.y + Bv * hl.z);
                        nd = reflect(-wo, hh);
                        if (dot(nd, nrm) <= 0.0f) nd = reflect(-wo, nrm);
                        const float NdotL = gmax(dot(nrm, nd), 1e-4f);
                        const float NdotV = gmax(dot(nrm, wo), 1e-4f);
                        const float HdotV = gmax(dot(hh, wo), 1e-4f);
                        const float p5 = pow5(1.0f - HdotV);
                        const float3 F = m.albedo + f3(1.0f - m.albedo.x, 1.0f - m.albedo.y, 1.0f - m.albedo.z) * p5;
                        const float G1 = smith_g1(NdotV, alpha);
                        const float G2 = smith_g2(NdotL, NdotV, alpha);
                        thr = thr * (F * (G2 / gmax(G1, 1e-7f)));
                        no = sf.pos + nrm * 2e-3f;
                    } else {
                        // NEE (pathtrace.comp:341-395) up to the visibility test;
                        // the test and the add happen in the next wf_trace.
                        if (A.nee_enabled != 0) {
                            bool early = true;
                            if (S.light_count > 0 && S.total_light_power > 0.0f) {
                                const float u = rnd(seed);
                                int sel = S.light_count - 1;
                                for (int q = 0; q < S.light_count; ++q)
                                    if (u < __ldg(S.light_cdf + q)) {
                                        sel = q;
                                        break;
                                    }
                                const float4* Lr = S.lights + 5 * sel;
                                const float4 l0 = __ldg(Lr + 0), l1 = __ldg(Lr + 1), l2 = __ldg(Lr + 2);
                                const float4 l3 = __ldg(Lr + 3), l4 = __ldg(Lr + 4);
                                ++lights;
                                const float pick = l3.w / S.total_light_power;
                                if (pick > 0.0f) {
                                    float r1 = rnd(seed);
                                    float r2 = rnd(seed);
                                    if (r1 + r2 > 1.0f) {
                                        r1 = 1.0f - r1;
                                        r2 = 1.0f - r2;
                                    }
                                    const float3 lv0 = xyz(l0);
                                    const float3 lp = lv0 + r1 * (xyz(l1) - lv0) + r2 * (xyz(l2) - lv0);
                                    const float3 to = lp - sf.pos;
                                    const float dist2 = dot(to, to);
                                    const float dist = sqrtf(dist2);
                                    const float3 sd = to / dist;
                                    const float cos_hit = dot(nrm, sd);
                                    if (cos_hit > 0.0f) {
                                        const float cos_light = fabs_(dot(xyz(l4), sd));
                                        if (cos_light > 0.0f) {
                                            const float area = l0.w;
                                            const float dist2_safe = gmax(dist2, area);
                                            const float pdf = pick * (dist2_safe / (area * cos_light));
                                            float3 contrib = f3(0.0f, 0.0f, 0.0f);
                                            if (pdf > 0.0f) {
                                                const float3 em = xyz(l3);
                                                contrib = (((m.albedo / 3.14159265359f) * em) * cos_hit) / pdf;
                                                const float cap = dot(em, f3(0.299f, 0.587f, 0.114f)) * A.firefly_clamp;
                                                contrib = vmin(contrib, f3(cap, cap, cap));
                                            }
                                            const float3 so = sf.pos + nrm * 2e-3f;
                                            rec0 = make_float4(so.x, so.y, so.z, dist - 4e-3f);
                                            rec1 = make_float4(sd.x, sd.y, sd.z, __int_as_float(p));
                                            // the visible light's term, and what throughput * 0 is
                                            // per channel for the occluded case
                                            const float3 q = thr * contrib;
                                            rec2 = make_float4(q.x, q.y, q.z,
                                                               __int_as_float((last ? 1 : 0) | (zero_code(thr.x) << 1) |
                                                                              (zero_code(thr.y) << 3) |
                                                                              (zero_code(thr.z) << 5)));
                                            shadow_rec = true;
                                            early = false;
                                        }
                                    }
                                }
                            }
                            // rad + throughput * 0 changes rad only where a throughput
                            // channel is not finite (NaN)
                            if (early && (bad(thr.x) || bad(thr.y) || bad(thr.z))) {
                                if (!rad_known) rad = xyz(B.rad[p]);
                                rad = rad + thr * f3(0.0f, 0.0f, 0.0f);
                                rad_known = rad_dirty = true;
                            }
                        }
                        const float u1 = rnd(seed);
                        const float u2 = rnd(seed);
                        nd = cosine_hemisphere(u1, u2, nrm);
                        thr = thr * m.albedo;
                        no = sf.pos + nrm * 1e-3f;
                        nd_diffuse = true;
                    }
                    cont = !last;
                }
                if (rad_dirty) B.rad[p] = make_float4(rad.x, rad.y, rad.z, 0.0f);
                if (cont) {
                    B.o[p] = make_float4(no.x, no.y, no.z, 0.0f);
                    B.d[p] = make_float4(nd.x, nd.y, nd.z, 0.0f);
                    B.thr[p] = make_float4(thr.x, thr.y, thr.z, nd_diffuse ? 1.0f : 0.0f);
                    B.seed[p] = seed;
                } else if (!shadow_rec) {
                    if (!rad_known) rad = xyz(B.rad[p]);
                    B.res[p] = make_float4(rad.x, rad.y, rad.z, 0.0f);
                }
            }
        }
        // continuing paths -> rq[nxt]; shadow records -> srec[cur]
        unsigned int slot_r, slot_s;
        block_append(sh, cont, shadow_rec, B.qlen + nxt, B.qlen + 2 + cur, slot_r, slot_s);
        if (cont) B.rq[nxt][slot_r] = p;
        if (shadow_rec) {
            float4* r = B.srec[cur] + 3 * slot_s;
            r[0] = rec0;
            r[1] = rec1;
            r[2] = rec2;
        }
    }
    const unsigned int active = __activemask();
    const unsigned int hs = __reduce_add_sync(active, hits);
    const unsigned int ls = __reduce_add_sync(active, lights);
    if ((threadIdx.x & 31) == 0) {
        if (hs) atomicAdd(&A.counters->surface_hits, (unsigned long long)hs);
        if (ls) atomicAdd(&A.counters->light_samples, (unsigned long long)ls);
    }
}

// pathtrace.comp:633-654 per pixel for the chunk's samples, in frame order;
// on frame 0 also the G-buffer ray (seed 99991, no lens offset).
__global__ void __launch_bounds__(128) wf_accumulate(WaveArgs A) {
    const int W = A.width, H = A.height;
    Guard g = {0u, 0u, 0u};
    uint32_t closest = 0, ghits = 0;
    const int nsegs = A.segs ? A.nsegs : 1;
    const int items = nsegs * A.npix;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < items; t += gridDim.x * blockDim.x) {
        const int j = t % A.npix;
        const FrameSeg& sg = seg_at(A, t / A.npix);
        const int tile = j >> 5, lane = j & 31;
        const int px = (tile % A.tiles_x) * 8 + (lane & 7);
        const int py = (tile / A.tiles_x) * 4 + (lane >> 3);
        if (px >= W || py >= H) continue;
        const long i = (long)py * W + px;
        const Images& img = sg.img;
        const int C = sg.channels;
        float4 acc = make_float4(0, 0, 0, 0);
        float var = 0.0f;
        if (sg.first_frame > 0) {
            acc = img.accum[i];
            var = img.var[i];
        }
        for (int s = 0; s < sg.n_samples; ++s) {
            const int base = sg.path_base + j + A.npix * (C * s);
            float3 rad;
            if (C == 3) {
                rad = f3(A.wb.res[base].x, A.wb.res[base + A.npix].y, A.wb.res[base + 2 * A.npix].z);
            } else {
                rad = xyz(A.wb.res[base]);
            }
            if (bad(rad.x) || bad(rad.y) || bad(rad.z)) rad = f3(0, 0, 0);
            const float l = luma709(rad);
            const float l2 = l * l;
            if (sg.first_frame + s == 0) {
                acc = make_float4(rad.x, rad.y, rad.z, 1.0f);
                var = l2;
                uint32_t gs = init_seed(px, py, 99991);
                const Ray gr = generate_ray(sg.cam, W, H, px, py, gs, 0.0f);
                ++closest;
                const Hit h = closest_hit<false>(A.scene, gr, g);
                float4 gv = make_float4(0.0f, 1.0f, 0.0f, 1e4f);
                if (h.prim >= 0) {
                    ++ghits;
                    const Surf sf = surface(A.scene, gr, h);
                    const float3 nn = dot(gr.d, sf.normal) < 0.0f ? sf.normal : -sf.normal;
                    gv = make_float4(nn.x, nn.y, nn.z, h.t);
                }
                img.gbuf[i] = to_half4(gv.x, gv.y, gv.z, gv.w);
            } else {
                acc.x = acc.x + rad.x;
                acc.y = acc.y + rad.y;
                acc.z = acc.z + rad.z;
                acc.w = acc.w + 1.0f;
                var = var + l2;
            }
        }
        img.accum[i] = acc;
        img.var[i] = var;
    }
    const unsigned int active = __activemask();
    const unsigned int c = __reduce_add_sync(active, closest);
    const unsigned int n = __reduce_add_sync(active, g.nodes);
    const unsigned int t = __reduce_add_sync(active, g.tris);
    const unsigned int h = __reduce_add_sync(active, ghits);
    const unsigned int gf = __reduce_or_sync(active, g.flags);
    if ((threadIdx.x & 31) == 0) {
        if (c) atomicAdd(&A.counters->closest_rays, (unsigned long long)c);
        if (n) atomicAdd(&A.counters->node_tests, (unsigned long long)n);
        if (t) atomicAdd(&A.counters->tri_tests, (unsigned long long)t);
        if (h) atomicAdd(&A.counters->surface_hits, (unsigned long long)h);
        if (gf) atomicOr(&A.counters->error_word, gf);
    }
}

static int grid_for(const void* fn, int block) {
    int dev = 0, sms = 148, per = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, block, 0);
    return sms * (per > 0 ? per : 1);
}

// Persistent trace with dynamic ray fetch: the refill state machine of
// dyn_trace.cuh over the ray queue followed by the shadow queue (one
// atomicAdd per warp on the work counter per refill).  Same rays and results
// as wf_trace (bit for bit in the exact build); only the schedule differs.
// kWide: interior steps over the 4-wide nodes (scene.nodes4) instead of the
// binary records.
// kPacked: interior steps over S.nodes_packed (one-register child
// references, full entry distances on the stack).
template <bool kWide, bool kPacked>
DI void trace_dyn(const WaveArgs& A) {
    const WaveBuffers& B = A.wb;
    const DeviceScene& S = A.scene;
    const StepScene SP = {kPacked ? S.nodes_packed : S.nodes, S.nodes4, S.tri_isect, S.node_count};
    const int cur = A.bounce & 1;
    const int prev = cur ^ 1;
    const unsigned int nr = A.bounce < 6 ? B.qlen[cur] : 0u;
    const unsigned int ns = B.qlen[2 + prev];
    const unsigned int total = nr + ns;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        B.qlen[prev] = 0u;
        B.qlen[2 + cur] = 0u;
        B.qlen[5] = 0u;
        B.qlen[6] = 0u;
    }
    const unsigned int FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    Guard g = {0u, 0u, 0u};
    uint32_t closest = 0, shadow = 0;
    DynStack stk;
    LaneRay L;
    L.item = -1;
    L.top = 0;
    L.have_node = false;
    L.leaf.cnt = 0;
    L.leaf.ref = 0;
    L.any = false;
    while (true) {
        // ---- refill idle lanes ----
        const unsigned int idle = __ballot_sync(FULL, L.item == -1);
        if (idle) {
            const int leader = __ffs(idle) - 1;
            unsigned int base = 0;
            if (lane == leader) base = atomicAdd(B.qlen + 4, (unsigned int)__popc(idle));
            base = __shfl_sync(FULL, base, leader);
            if (L.item == -1) {
                const unsigned int i = base + __popc(idle & ((1u << lane) - 1u));
                L.item = i < total ? (int)i : -2;
                if (L.item >= 0) {
                    if ((unsigned int)L.item < nr) {
                        const int p = B.rq[cur][L.item];
                        L.r = make_ray(xyz(B.o[p]), xyz(B.d[p]));
                        dyn_start(S, L, 1e30f, false, g);
                        if (kPacked) L.node.ref = S.root_packed;
                        ++closest;
                    } else {
                        const float4* rec = B.srec[prev] + 3 * (L.item - (int)nr);
                        const float4 so = rec[0], sd = rec[1];
                        L.r = make_ray(xyz(so), xyz(sd));
                        dyn_start(S, L, so.w, true, g);
                        if (kPacked) L.node.ref = S.root_packed;
                        ++shadow;
                    }
                }
            }
        }
        if (__all_sync(FULL, L.item == -2)) break;
        while (true) {
            bool busy = L.item >= 0;
            bool leaf_phase;
            if (dyn_schedule<kPacked>(L, busy, __ballot_sync(FULL, busy), A.leaf_quarters, leaf_phase) &&
                dyn_step<kWide, false, false, kPacked>(SP, L, stk, leaf_phase, g, A.interior_steps)) {
                const int item = L.item;
                if ((unsigned int)item < nr) {
                    const int p = B.rq[cur][item];
                    B.hit[p] = make_float4(L.h.t, L.h.u, L.h.v, __int_as_float(L.h.prim));
                } else {
                    const float4* rec = B.srec[prev] + 3 * (item - (int)nr);
                    shadow_add(B, __float_as_int(rec[1].w), L.h.prim < 0, rec[2]);
                }
                L.item = -1;
                busy = false;
            }
            if (__popc(__ballot_sync(FULL, busy)) < A.refill_lanes) break;
        }
    }
    const unsigned int c = __reduce_add_sync(FULL, closest);
    const unsigned int s = __reduce_add_sync(FULL, shadow);
    const unsigned int n = __reduce_add_sync(FULL, g.nodes);
    const unsigned int t = __reduce_add_sync(FULL, g.tris);
    const unsigned int gf = __reduce_or_sync(FULL, g.flags);
    if (lane == 0) {
        if (c) atomicAdd(&A.counters->closest_rays, (unsigned long long)c);
        if (s) atomicAdd(&A.counters->shadow_rays, (unsigned long long)s);
        if (n) atomicAdd(&A.counters->node_tests, (unsigned long long)n);
        if (t) atomicAdd(&A.counters->tri_tests, (unsigned long long)t);
        if (gf) atomicOr(&A.counters->error_word, gf);
    }
}

// Binary walk: registers capped at 56 (62 uncapped, no spills either way),
// so 9 blocks of 128 threads fit an SM instead of 8; the kernel waits on L1
// latency and the extra warps pay (65.0 vs 67.4 ms per export frame).
__global__ void __maxnreg__(56) wf_trace_dyn(WaveArgs A) { trace_dyn<false, false>(A); }
// The same over the packed-reference records (scenes that have them).
__global__ void __maxnreg__(56) wf_trace_dynp(WaveArgs A) { trace_dyn<false, true>(A); }
#if !RC_EXACT
// 4-wide walk: uncapped (77 registers; 56 spills)
__global__ void __launch_bounds__(256) wf_trace_dyn4(WaveArgs A) { trace_dyn<true, false>(A); }
#endif

// Launchers; the chunk sequence (generate, 7 x trace, 6 x shade interleaved,
// accumulate) is driven from api.cu so each launch can be timed.  Grids are
// sized to fill every SM (grid-stride and persistent kernels), once per
// kernel and block size (64, 128 or 256 threads).
struct WfGrids {
    int gen = 0, acc = 0, sort = 0;
    int trace0[3] = {}, trace1[3] = {}, shade[3] = {}, shade_mq[3] = {}, dyn[3] = {}, dynp[3] = {}, dyn4[3] = {};
};
static int block_class(int block) { return block <= 64 ? 0 : (block <= 128 ? 1 : 2); }
static void fill_grids(WfGrids& g) {
    g.gen = grid_for((const void*)wf_generate, 256);
    g.acc = grid_for((const void*)wf_accumulate, 128);
    g.sort = grid_for((const void*)wf_sort, 256);
    for (int c = 0; c < 3; ++c) {
        const int b = 64 << c;
        g.trace0[c] = grid_for((const void*)wf_trace<false>, b);
        g.trace1[c] = grid_for((const void*)wf_trace<true>, b);
        g.shade[c] = grid_for((const void*)wf_shade<false>, b);
        g.shade_mq[c] = grid_for((const void*)wf_shade<true>, b);
        g.dyn[c] = grid_for((const void*)wf_trace_dyn, b);
        g.dynp[c] = grid_for((const void*)wf_trace_dynp, b);
#if !RC_EXACT
        g.dyn4[c] = grid_for((const void*)wf_trace_dyn4, b);
#endif
    }
}

// The grids of the current device (SM counts and occupancy differ between
// devices), filled once per device; a process may drive several devices
// from several threads.
static WfGrids& grids() {
    constexpr int kDevs = 64;
    static WfGrids g[kDevs];
    static std::once_flag once[kDevs];
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= kDevs) {
        thread_local WfGrids t;
        fill_grids(t);
        return t;
    }
    std::call_once(once[dev], [&] { fill_grids(g[dev]); });
    return g[dev];
}

cudaError_t launch_wf_generate(const WaveArgs& A, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(A.wb.qlen, 0, 8 * sizeof(unsigned int), s);
    if (e != cudaSuccess) return e;
    wf_generate<<<grids().gen, 256, 0, s>>>(A);
    return cudaGetLastError();
}

cudaError_t launch_wf_trace(const WaveArgs& A, cudaStream_t s, int block) {
    const int c = block_class(block), b = 64 << c;
    // the fast refill trace packs leaf counts into 16 bits of a stack entry
    // chunks below refill_min_paths hold about one wave of rays per launch,
    // where the refill bookkeeping costs more than it recovers (854x480 at
    // 1 spp: trace 0.264 ms grid-stride vs 0.306 ms refill; they tie at 2 spp)
    // BVHs deeper than 28 levels keep the reference's shadow walk (its
    // 32-entry stack can overflow), which the refill walk does not follow
    if (A.dynamic_fetch && A.paths >= A.refill_min_paths && A.scene.max_leaf < 0x10000 &&
        A.scene.depth <= 28) {
#if !RC_EXACT
        if (A.scene.nodes4) {
            wf_trace_dyn4<<<grids().dyn4[c], b, 0, s>>>(A);
            return cudaGetLastError();
        }
#endif
        if (A.scene.nodes_packed) {
            wf_trace_dynp<<<grids().dynp[c], b, 0, s>>>(A);
            return cudaGetLastError();
        }
        wf_trace_dyn<<<grids().dyn[c], b, 0, s>>>(A);
        return cudaGetLastError();
    }
    if (A.scene.depth <= 28)
        wf_trace<true><<<grids().trace1[c], b, 0, s>>>(A);
    else
        wf_trace<false><<<grids().trace0[c], b, 0, s>>>(A);
    return cudaGetLastError();
}

cudaError_t launch_wf_shade(const WaveArgs& A, cudaStream_t s, int block) {
    const int c = block_class(block);
    if (A.material_queues)
        wf_shade<true><<<grids().shade_mq[c], 64 << c, 0, s>>>(A);
    else
        wf_shade<false><<<grids().shade[c], 64 << c, 0, s>>>(A);
    return cudaGetLastError();
}

cudaError_t launch_wf_sort(const WaveArgs& A, cudaStream_t s) {
    wf_sort<<<grids().sort, 256, 0, s>>>(A);
    return cudaGetLastError();
}

cudaError_t launch_wf_accumulate(const WaveArgs& A, cudaStream_t s) {
    wf_accumulate<<<grids().acc, 128, 0, s>>>(A);
    return cudaGetLastError();
}

}  // namespace RC_NS
}  // namespace rc
