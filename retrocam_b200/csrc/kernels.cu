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
//   photon_emit_full_kernel + photon_bounce_kernel
//                         photon_trace.comp main(), split after the first
//                         segment (fast build with the specular/other
//                         BVH split: photon_emit_dyn or photon_emit_kernel
//                         for the first phase)
//   photon_gather_kernel  photon_gather.comp main()
//   atrous_kernel         post/atrous_denoise.frag (p00_normalize fused
//                         into the first pass)
//   normalize_kernel      post/p00_normalize.frag  (denoiser disabled)
//   display_kernel        display.frag + the export framebuffer's RGBA8 store
//
// Every traversal loop is bounded: a traversal that pops more stack
// entries than the scene has nodes (impossible for a validated tree) sets
// RC_GUARD_TRAVERSAL_CAP in the context's error word and stops.
#include <atomic>

#include "device_common.cuh"
#include "dyn_trace.cuh"

namespace rc {
namespace RC_NS {

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
                const Hit h = closest_hit<kShadowAtParent>(S, gr, g);
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

// photon_trace.comp:168-196: the emitted photon -- light picked by the CDF,
// a uniform point on its triangle, a cosine direction about its normal, an
// equal share of the total power.
struct PhotonState {
    Ray ray;
    float3 power;
    uint32_t seed;
};

DI PhotonState emit_photon(const PhotonArgs& A, const DeviceScene& S, int gid) {
    PhotonState st;
    st.seed = photon_seed((uint32_t)gid, A.seed);
    const float u = rnd(st.seed);
    int sel = S.light_count - 1;
    for (int i = 0; i < S.light_count; ++i)
        if (u < __ldg(S.light_cdf + i)) {
            sel = i;
            break;
        }
    const float4* L = S.lights + 5 * sel;
    const float4 l0 = __ldg(L + 0), l1 = __ldg(L + 1), l2 = __ldg(L + 2), l3 = __ldg(L + 3), l4 = __ldg(L + 4);
    float r1 = rnd(st.seed);
    float r2 = rnd(st.seed);
    if (r1 + r2 > 1.0f) {
        r1 = 1.0f - r1;
        r2 = 1.0f - r2;
    }
    const float3 lv0 = xyz(l0);
    const float3 sp = lv0 + r1 * (xyz(l1) - lv0) + r2 * (xyz(l2) - lv0);
    const float3 en = normalize(xyz(l4));
    const float e1 = rnd(st.seed);
    const float e2 = rnd(st.seed);
    const float3 rd = cosine_hemisphere(e1, e2, en);
    const float3 em = xyz(l3);
    const float lum = dot(em, f3(0.299f, 0.587f, 0.114f));
    const float per = S.total_light_power / (float)A.photon_count;
    st.power = (lum > 1e-6f) ? (em / lum) * per : f3(per, per, per);
    st.ray = make_ray(sp + en * 1e-3f, rd);
    return st;
}

struct PhotonStore {
    bool store;
    float3 pos, power, dir;
};

// One hit of a photon's walk (photon_trace.comp:213-248): glass reflects or
// refracts by Fresnel, metal mirrors (both give the next segment in `ray`
// and return 0), the first diffuse hit after a specular bounce is stored
// (returns 1, `out` filled), any other diffuse hit ends the walk (2).
DI int photon_interact(const DeviceScene& S, const Hit& hit, Ray& ray, float3& power, uint32_t& seed, bool& spec,
                       PhotonStore& out) {
    const Surf sf = surface(S, ray, hit);
    const Mat m = load_mat(S, sf.mat);
    const float3 rd = ray.d;
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
        return 0;
    }
    if (m.metallic > 0.5f) {
        power = power * m.albedo;
        const float3 nd = reflect(rd, n);
        ray = make_ray(sf.pos + n * 2e-3f, nd);
        spec = true;
        return 0;
    }
    if (spec) {
        out.store = true;
        out.pos = sf.pos;
        out.power = power;
        out.dir = rd;
        return 1;
    }
    return 2;
}

// photon_trace.comp:205-251: up to 8 segments (photon_interact per hit).
// With `have_first` the first segment's hit is given (already traced and
// counted by the caller).
template <bool kAtParent>
DI PhotonStore photon_walk(const PhotonArgs& A, const DeviceScene& S, PhotonState st, bool have_first,
                           const Hit& first, Guard& g, uint32_t& rays) {
    PhotonStore out;
    out.store = false;
    bool spec = false;
    for (int b = 0; b < 8; ++b) {
        Hit hit;
        if (b == 0 && have_first) {
            hit = first;
        } else {
            ++rays;
            hit = photon_hit<kAtParent>(S, st.ray, g);
        }
        if (hit.prim < 0) break;
        if (photon_interact(S, hit, st.ray, st.power, st.seed, spec, out) != 0) break;
    }
    return out;
}

// Appends the warp's stored photons: one atomicAdd on the counter per warp;
// each photon's hash cell is recorded and counted for the cell-sorted
// layout (the reference links the photon into its cell here with an
// atomicExchange on the head; the scan/scatter kernels below build that
// layout and heads/next from it).  Every lane of the warp calls this.
DI void append_photons(const PhotonArgs& A, const PhotonStore& s) {
    const unsigned int mask = __ballot_sync(0xffffffffu, s.store);
    const int lane = threadIdx.x & 31;
    unsigned int base = 0;
    if (mask != 0u) {
        const int leader = __ffs(mask) - 1;
        if (lane == leader) base = atomicAdd(A.counter, (unsigned int)__popc(mask));
        base = __shfl_sync(0xffffffffu, base, leader);
    }
    if (s.store) {
        const unsigned int idx = base + __popc(mask & ((1u << lane) - 1u));
        if (idx < (unsigned int)A.photon_count) {
            const int cx = (int)floorf(s.pos.x / A.radius);
            const int cy = (int)floorf(s.pos.y / A.radius);
            const int cz = (int)floorf(s.pos.z / A.radius);
            const int h = cell_hash(cx, cy, cz, A.hash_size);
            A.cell_of[idx] = h;
            atomicAdd(A.cell_count + h, 1u);
            A.photons[3 * idx + 0] = make_float4(s.pos.x, s.pos.y, s.pos.z, 0.0f);
            A.photons[3 * idx + 1] = make_float4(s.power.x, s.power.y, s.power.z, 0.0f);
            A.photons[3 * idx + 2] = make_float4(s.dir.x, s.dir.y, s.dir.z, 0.0f);
        }
    }
}

// Queues, for the walks, the photons of the warp that `want` it: (origin,
// seed), (direction, power.x), (power.y, power.z, t, u), (v, triangle) --
// the ray, generator state and power after emission, and the first hit.
// One atomicAdd on A.queue_len per warp; every lane of the warp calls it.
DI void queue_photon(const PhotonArgs& A, bool want, const Ray& ray, uint32_t seed, float3 power, const Hit& h) {
    const unsigned int mask = __ballot_sync(0xffffffffu, want);
    if (mask == 0u) return;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(mask) - 1;
    unsigned int base = 0;
    if (lane == leader) base = atomicAdd(A.queue_len, (unsigned int)__popc(mask));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (want) {
        float4* q = A.queue + 4 * (size_t)(base + __popc(mask & ((1u << lane) - 1u)));
        q[0] = make_float4(ray.o.x, ray.o.y, ray.o.z, __uint_as_float(seed));
        q[1] = make_float4(ray.d.x, ray.d.y, ray.d.z, power.x);
        q[2] = make_float4(power.y, power.z, h.t, h.u);
        q[3] = make_float4(h.v, __int_as_float(h.prim), 0.0f, 0.0f);
    }
}

// append_photons, then the warp's ray and work counters.
DI void store_photons(const PhotonArgs& A, const PhotonStore& s, uint32_t rays, Guard& g) {
    append_photons(A, s);
    const int lane = threadIdx.x & 31;
    const unsigned int rsum = __reduce_add_sync(0xffffffffu, rays);
    if (lane == 0 && rsum) atomicAdd(&A.counters->photon_rays, (unsigned long long)rsum);
    flush_work(g, 0u, 0u, A.counters, true);
}

#if !RC_EXACT
// First segment against the split scene: the nearest specular triangle,
// then whether any other triangle lies before it.  True (with the hit in
// the full scene's numbering) when the photon's first hit is specular.
DI bool first_specular(const PhotonArgs& A, const Ray& ray, Guard& g, Hit& hit) {
    Hit hs, hd;
    traverse_ww<false>(A.spec, ray, 1e30f, g, hs);
    if (hs.prim < 0 || traverse_ww<true>(A.diff, ray, hs.t, g, hd)) return false;
    hit = hs;
    hit.prim = __ldg(A.spec_orig + hs.prim);
    return true;
}
#endif

#if !RC_EXACT
// Two-phase trace (fast build with the split): every photon's emission and
// first segment, and only the photons whose first hit is specular -- the
// only ones that can be stored -- go on, compacted into a queue, so the
// multi-bounce walks run in full warps instead of holding every warp that
// has one of them.  Queue entry: (origin, seed), (direction, power.x),
// (power.y, power.z, t, u), (v, triangle).
__global__ void __launch_bounds__(256) photon_emit_kernel(PhotonArgs A) {
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    const DeviceScene& S = A.scene;
    Guard g = {0u, 0u, 0u};
    uint32_t rays = 0;
    bool want = false;
    PhotonState st{};
    Hit h{};
    if (gid < A.photon_count && S.light_count != 0) {
        st = emit_photon(A, S, gid);
        ++rays;
        want = first_specular(A, st.ray, g, h);
    }
    queue_photon(A, want, st.ray, st.seed, st.power, h);
    PhotonStore none;
    none.store = false;
    store_photons(A, none, rays, g);
}
#endif

// Two-phase trace over the full scene (exact math, and fast math without
// the split): every photon's emission and first segment; photons whose
// first hit is glass or metal (photon_interact's branches) -- the only
// ones that can be stored -- are queued for photon_bounce_kernel as
// photon_emit_kernel queues them.  Same segments, hits and random numbers
// as one walk of all the segments (photon_trace.comp:168-252), split after
// the first segment.
template <bool kAtParent>
__global__ void __launch_bounds__(256) photon_emit_full_kernel(PhotonArgs A) {
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    const DeviceScene& S = A.scene;
    Guard g = {0u, 0u, 0u};
    uint32_t rays = 0;
    bool want = false;
    PhotonState st{};
    Hit h{};
    if (gid < A.photon_count && S.light_count != 0) {
        st = emit_photon(A, S, gid);
        ++rays;
        h = photon_hit<kAtParent>(S, st.ray, g);
        if (h.prim >= 0) {
            const int m = __float_as_int(__ldg(S.tri_shade + 3 * h.prim).w);
            want = __ldg(S.materials + 4 * m + 2).z > 0.5f || __ldg(S.materials + 4 * m + 0).w > 0.5f;
        }
    }
    queue_photon(A, want, st.ray, st.seed, st.power, h);
    PhotonStore none;
    none.store = false;
    store_photons(A, none, rays, g);
}

#if RC_EXACT
// The first phase as a refill kernel (exact build, trees up to 60 levels):
// a lane emits the next photon (work counter A.work) when its photon is
// done and walks the full scene in trace_unordered's order (dyn_step
// <kUnordered>: left child first, the same culls and stack guard, a
// reached leaf tested before the next pop), so each photon gets
// photon_emit_full_kernel's hit bit for bit; photons whose first hit is
// glass or metal are queued as that kernel queues them.
__global__ void __launch_bounds__(128) photon_emit_full_dyn(PhotonArgs A) {
    const unsigned int FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const DeviceScene& S = A.scene;
    const unsigned int total = S.light_count != 0 ? (unsigned int)A.photon_count : 0u;
    Guard g = {0u, 0u, 0u};
    uint32_t rays = 0;
    DynStack stk;
    LaneRay L;
    L.item = -1;
    L.top = 0;
    L.have_node = false;
    L.leaf.cnt = 0;
    L.any = false;
    uint32_t seed = 0u;
    float3 power = f3(0.0f, 0.0f, 0.0f);
    while (true) {
        const unsigned int idle = __ballot_sync(FULL, L.item == -1);
        if (idle) {
            const int leader = __ffs(idle) - 1;
            unsigned int base = 0;
            if (lane == leader) base = atomicAdd(A.work, (unsigned int)__popc(idle));
            base = __shfl_sync(FULL, base, leader);
            if (L.item == -1) {
                const unsigned int i = base + __popc(idle & ((1u << lane) - 1u));
                L.item = i < total ? (int)i : -2;
                if (L.item >= 0) {
                    const PhotonState st = emit_photon(A, S, L.item);
                    seed = st.seed;
                    power = st.power;
                    L.r = st.ray;
                    ++rays;
                    dyn_start(S, L, 1e30f, false, g);
                }
            }
        }
        if (__all_sync(FULL, L.item == -2)) break;
        while (true) {
            bool busy = L.item >= 0;
            bool push = false;
            bool leaf_phase;
            if (dyn_schedule(L, busy, __ballot_sync(FULL, busy), A.leaf_quarters, leaf_phase) &&
                dyn_step<false, true>(S, L, stk, leaf_phase, g, A.interior_steps)) {
                if (L.h.prim >= 0) {
                    const int m = __float_as_int(__ldg(S.tri_shade + 3 * L.h.prim).w);
                    push = __ldg(S.materials + 4 * m + 2).z > 0.5f || __ldg(S.materials + 4 * m + 0).w > 0.5f;
                }
                L.item = -1;
                busy = false;
            }
            queue_photon(A, push, L.r, seed, power, L.h);
            if (__popc(__ballot_sync(FULL, busy)) < A.refill_lanes) break;
        }
    }
    const unsigned int rsum = __reduce_add_sync(FULL, rays);
    if (lane == 0 && rsum) atomicAdd(&A.counters->photon_rays, (unsigned long long)rsum);
    flush_work(g, 0u, 0u, A.counters, true);
}
#endif

template <bool kAtParent>
__global__ void __launch_bounds__(256) photon_bounce_kernel(PhotonArgs A) {
    const unsigned int n = min(*A.queue_len, (unsigned int)A.photon_count);
    Guard g = {0u, 0u, 0u};
    uint32_t rays = 0;
    const int lane = threadIdx.x & 31;
    // a warp takes the next 32 queued photons (work counter A.work, zero at
    // launch) when its last ones are done: a persistent grid sized to the
    // GPU instead of one thread per emitted photon, most of them idle
    while (true) {
        unsigned int base = 0;
        if (lane == 0) base = atomicAdd(A.work, 32u);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= n) break;
        const unsigned int i = base + lane;
        PhotonStore out;
        out.store = false;
        if (i < n) {
            const float4* q = A.queue + 4 * (size_t)i;
            const float4 q0 = q[0], q1 = q[1], q2 = q[2], q3 = q[3];
            PhotonState st;
            st.ray = make_ray(xyz(q0), xyz(q1));
            st.seed = __float_as_uint(q0.w);
            st.power = f3(q1.w, q2.x, q2.y);
            Hit h;
            h.t = q2.z;
            h.u = q2.w;
            h.v = q3.x;
            h.prim = __float_as_int(q3.y);
            out = photon_walk<kAtParent>(A, A.scene, st, true, h, g, rays);
        }
        append_photons(A, out);
    }
    PhotonStore none;
    none.store = false;
    store_photons(A, none, rays, g);
}

// The queued walks: the work counter cleared, then a grid of every SM times
// the blocks that fit it (at most one thread per queue slot).
template <bool kAtParent>
static cudaError_t launch_bounce(const PhotonArgs& A, cudaStream_t s, int b, int blocks) {
    cudaError_t e = cudaMemsetAsync(A.work, 0, sizeof(unsigned int), s);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 148, per = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, photon_bounce_kernel<kAtParent>, b, 0);
    photon_bounce_kernel<kAtParent><<<std::min(blocks, sms * std::max(per, 1)), b, 0, s>>>(A);
    return cudaGetLastError();
}

#if !RC_EXACT
// The first phase as a refill kernel (dyn_trace.cuh): a lane emits the next
// photon (work counter A.work) when its photon is done, walks the specular
// triangles' tree for the nearest hit, then on a hit the other triangles'
// tree for any hit before it; photons whose first hit is specular are
// queued.  The photons, rays and hits are photon_emit_kernel's; one thread
// per photon ran at 5 of 32 lanes (329 vs 244 us per 2M photons).  The
// queued walks stay one thread per photon (photon_bounce_kernel): as a
// refill kernel they were slower (396 vs 310 us), the surface interactions
// between segments running a few lanes at a time.
__global__ void __launch_bounds__(128) photon_emit_dyn(PhotonArgs A) {
    const unsigned int FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const DeviceScene& S = A.scene;
    const unsigned int total = S.light_count != 0 ? (unsigned int)A.photon_count : 0u;
    Guard g = {0u, 0u, 0u};
    uint32_t rays = 0;
    DynStack stk;
    LaneRay L;
    L.item = -1;
    L.top = 0;
    L.have_node = false;
    L.leaf.cnt = 0;
    L.any = false;
    uint32_t seed = 0u;
    float3 power = f3(0.0f, 0.0f, 0.0f);
    Hit hs;
    hs.t = hs.u = hs.v = 0.0f;
    hs.prim = -1;
    bool second = false;   // walking the other triangles for an occluder
    while (true) {
        const unsigned int idle = __ballot_sync(FULL, L.item == -1);
        if (idle) {
            const int leader = __ffs(idle) - 1;
            unsigned int base = 0;
            if (lane == leader) base = atomicAdd(A.work, (unsigned int)__popc(idle));
            base = __shfl_sync(FULL, base, leader);
            if (L.item == -1) {
                const unsigned int i = base + __popc(idle & ((1u << lane) - 1u));
                L.item = i < total ? (int)i : -2;
                if (L.item >= 0) {
                    const PhotonState st = emit_photon(A, S, L.item);
                    seed = st.seed;
                    power = st.power;
                    L.r = st.ray;
                    second = false;
                    ++rays;
                    dyn_start(A.spec, L, 1e30f, false, g);
                }
            }
        }
        if (__all_sync(FULL, L.item == -2)) break;
        while (true) {
            bool busy = L.item >= 0;
            bool push = false;
            bool leaf_phase;
            if (dyn_schedule(L, busy, __ballot_sync(FULL, busy), A.leaf_quarters, leaf_phase) &&
                dyn_step<false>(step_scene(second, A.spec, A.diff), L, stk, leaf_phase, g, A.interior_steps)) {
                if (!second && L.h.prim >= 0) {
                    hs = L.h;
                    hs.prim = __ldg(A.spec_orig + hs.prim);
                    second = true;
                    dyn_start(A.diff, L, hs.t, true, g);
                } else {
                    push = second && L.h.prim < 0;
                    L.item = -1;
                    busy = false;
                }
            }
            queue_photon(A, push, L.r, seed, power, hs);
            if (__popc(__ballot_sync(FULL, busy)) < A.refill_lanes) break;
        }
    }
    const unsigned int rsum = __reduce_add_sync(FULL, rays);
    if (lane == 0 && rsum) atomicAdd(&A.counters->photon_rays, (unsigned long long)rsum);
    flush_work(g, 0u, 0u, A.counters, true);
}
#endif

// The gathered caustic of one pixel scaled into radiance and added into the
// accumulation (photon_gather.comp:200-222).
DI void add_caustic(const GatherArgs& A, long pix, int hm, float3 caustic, float r2) {
    const float PI_G = 3.14159265358979f;
    const float4 ma = __ldg(A.scene.materials + 4 * hm);
    float3 L = (xyz(ma) * caustic) / (PI_G * r2);
    if (bad(L.x) || bad(L.y) || bad(L.z)) L = f3(0, 0, 0);
    if (A.weight != 1.0f) L = L * A.weight;
    float4* a = A.img.accum + pix;
    float4 v = *a;
    v.x = v.x + L.x;
    v.y = v.y + L.y;
    v.z = v.z + L.z;
    v.w = v.w + 0.0f;
    *a = v;
}

// A pixel whose 27 cells hold more than this many photons (as walked, at
// most 512 a cell) is gathered by photon_gather_heavy, one warp per pixel.
// One thread walking 27 x 512 photons held a whole gather launch (the rest
// of the GPU idle) for about 0.5 ms.
constexpr unsigned int kGatherLight = 64;

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
    bool heavy = false;
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
        const long pix = (long)py * W + px;
        if (A.cache_mode == 2) {
            const float4 c = A.hit_cache[pix];
            hm = __float_as_int(c.w);
            found = hm >= 0;
            hp = xyz(c);
        }
        for (int s = 0; s <= 6 && A.cache_mode != 2; ++s) {
            ++rays;
            const Hit hit = photon_hit<kAtParent>(S, ray, g);
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
        if (A.cache_mode == 1) A.hit_cache[pix] = make_float4(hp.x, hp.y, hp.z, __int_as_float(found ? hm : -1));
        const float r = A.radius, r2 = r * r;
        const int ccx = (int)floorf(hp.x / r), ccy = (int)floorf(hp.y / r), ccz = (int)floorf(hp.z / r);
        if (found && A.heavy && A.cache_mode != 0) {
            unsigned int total = 0;
            for (int dz = -1; dz <= 1; ++dz)
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dx = -1; dx <= 1; ++dx) {
                        const int h = cell_hash(ccx + dx, ccy + dy, ccz + dz, A.hash_size);
                        const unsigned int n = __ldg(A.cell_start + h + 1) - __ldg(A.cell_start + h);
                        total += n < 512u ? n : 512u;
                    }
            heavy = total > kGatherLight;
            found = found && !heavy;
        }
        if (found) {
            float3 caustic = f3(0, 0, 0);
            for (int dz = -1; dz <= 1; ++dz)
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dx = -1; dx <= 1; ++dx) {
                        const int h = cell_hash(ccx + dx, ccy + dy, ccz + dz, A.hash_size);
                        // the chain of cell h, walked as the contiguous slots
                        // [s0, s1) in chain order; `safety < 512` caps it
                        const unsigned int s0 = __ldg(A.cell_start + h);
                        const unsigned int s1 = __ldg(A.cell_start + h + 1);
                        const unsigned int n = (s1 - s0) < 512u ? (s1 - s0) : 512u;
                        // four independent loads in flight, then the four
                        // photons in chain order (the sum order is unchanged)
                        unsigned int k = 0;
                        for (; k + 4 <= n; k += 4) {
                            float4 pw[4];
                            float2 yz[4];
#pragma unroll
                            for (int q = 0; q < 4; ++q) {
                                pw[q] = __ldg(A.seg_posw + s0 + k + q);
                                yz[q] = __ldg(A.seg_powyz + s0 + k + q);
                            }
#pragma unroll
                            for (int q = 0; q < 4; ++q) {
                                const float3 d = hp - xyz(pw[q]);
                                const float d2 = dot(d, d);
                                if (d2 <= r2) {
                                    const float w = 1.0f - d2 / r2;
                                    caustic = caustic + f3(pw[q].w, yz[q].x, yz[q].y) * w;
                                }
                            }
                        }
                        for (; k < n; ++k) {
                            const float4 pw = __ldg(A.seg_posw + s0 + k);
                            const float3 d = hp - xyz(pw);
                            const float d2 = dot(d, d);
                            if (d2 <= r2) {
                                const float w = 1.0f - d2 / r2;
                                const float2 yz = __ldg(A.seg_powyz + s0 + k);
                                caustic = caustic + f3(pw.w, yz.x, yz.y) * w;
                            }
                        }
                    }
            add_caustic(A, pix, hm, caustic, r2);
        }
    }
    if (A.heavy) {
        const unsigned int m = __ballot_sync(0xffffffffu, heavy);
        if (m) {
            const int leader = __ffs(m) - 1;
            unsigned int base = 0;
            if (lane == leader) base = atomicAdd(A.heavy_len, (unsigned int)__popc(m));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (heavy) A.heavy[base + __popc(m & ((1u << lane) - 1u))] = py * W + px;
        }
    }
    const unsigned int rsum = __reduce_add_sync(0xffffffffu, rays);
    if (lane == 0 && rsum) atomicAdd(&A.counters->gather_rays, (unsigned long long)rsum);
    flush_work(g, 0u, 0u, A.counters, true);
}

// The heavy pixels of photon_gather_kernel, one warp per pixel: lanes 0..26
// look up the 27 cells, then the warp walks each cell's photons 32 at a
// time.  The photons summed are the reference's (the first 512 of each
// cell's chain).  Fast build: two loads deep (64 photons a round), lane
// sums combined by a butterfly, so only the order of the float additions
// differs from one thread's walk.  Exact build: each lane forms its
// photon's term, and the terms of the photons inside the radius are added
// in chain order (every lane keeps the same running sum from shuffles), so
// the sum is one thread's walk bit for bit.
__global__ void __launch_bounds__(256) photon_gather_heavy(GatherArgs A) {
    const unsigned int FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const unsigned int n = *A.heavy_len;
    const unsigned int nw = (gridDim.x * blockDim.x) >> 5;
    const float r = A.radius, r2 = r * r;
    for (unsigned int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < n; w += nw) {
        const int pix = A.heavy[w];
        const float4 c = A.hit_cache[pix];
        const float3 hp = xyz(c);
        const int hm = __float_as_int(c.w);
        const int ccx = (int)floorf(hp.x / r), ccy = (int)floorf(hp.y / r), ccz = (int)floorf(hp.z / r);
        unsigned int s0 = 0u, cnt = 0u;
        if (lane < 27) {
            const int dx = lane % 3 - 1, dy = (lane / 3) % 3 - 1, dz = lane / 9 - 1;
            const int h = cell_hash(ccx + dx, ccy + dy, ccz + dz, A.hash_size);
            s0 = __ldg(A.cell_start + h);
            const unsigned int s1 = __ldg(A.cell_start + h + 1);
            cnt = (s1 - s0) < 512u ? (s1 - s0) : 512u;
        }
        float3 caustic = f3(0, 0, 0);
#if RC_EXACT
        for (int k = 0; k < 27; ++k) {
            const unsigned int b = __shfl_sync(FULL, s0, k);
            const unsigned int m = __shfl_sync(FULL, cnt, k);
            for (unsigned int q0 = 0; q0 < m; q0 += 32) {
                const unsigned int q = q0 + lane;
                float3 term = f3(0, 0, 0);
                bool inside = false;
                if (q < m) {
                    const float4 p = __ldg(A.seg_posw + b + q);
                    const float3 d = hp - xyz(p);
                    const float d2 = dot(d, d);
                    if (d2 <= r2) {
                        const float w = 1.0f - d2 / r2;
                        const float2 yz = __ldg(A.seg_powyz + b + q);
                        term = f3(p.w, yz.x, yz.y) * w;
                        inside = true;
                    }
                }
                unsigned int in = __ballot_sync(FULL, inside);
                while (in) {
                    const int j = __ffs(in) - 1;
                    in &= in - 1u;
                    caustic = caustic + f3(__shfl_sync(FULL, term.x, j), __shfl_sync(FULL, term.y, j),
                                           __shfl_sync(FULL, term.z, j));
                }
            }
        }
#else
        for (int k = 0; k < 27; ++k) {
            const unsigned int b = __shfl_sync(FULL, s0, k);
            const unsigned int m = __shfl_sync(FULL, cnt, k);
            for (unsigned int q = lane; q < m; q += 64) {
                const bool two = q + 32 < m;
                const float4 p0 = __ldg(A.seg_posw + b + q);
                const float4 p1 = two ? __ldg(A.seg_posw + b + q + 32) : p0;
                const float3 d0 = hp - xyz(p0), d1 = hp - xyz(p1);
                const float e0 = dot(d0, d0), e1 = dot(d1, d1);
                if (e0 <= r2) {
                    const float2 yz = __ldg(A.seg_powyz + b + q);
                    caustic = caustic + f3(p0.w, yz.x, yz.y) * (1.0f - e0 / r2);
                }
                if (two && e1 <= r2) {
                    const float2 yz = __ldg(A.seg_powyz + b + q + 32);
                    caustic = caustic + f3(p1.w, yz.x, yz.y) * (1.0f - e1 / r2);
                }
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            caustic.x += __shfl_xor_sync(FULL, caustic.x, o);
            caustic.y += __shfl_xor_sync(FULL, caustic.y, o);
            caustic.z += __shfl_xor_sync(FULL, caustic.z, o);
        }
#endif
        if (lane == 0) add_caustic(A, pix, hm, caustic, r2);
    }
}

// ---------------------------------------------------------------------------
// photon map: cell-sorted layout
// ---------------------------------------------------------------------------
// Exclusive scan of the per-cell counts into cell_start[0..hash_size], in
// three passes: 4096 counts per 1024-thread block, a scan of the block sums
// (one block, sequential over chunks of 1024), and the add-back.
DI unsigned int block_exclusive_scan(unsigned int v, unsigned int* warp_sums, unsigned int* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        unsigned int w = (lane < (int)(blockDim.x >> 5)) ? warp_sums[lane] : 0u;
        unsigned int z = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned int y = __shfl_up_sync(0xffffffffu, z, o);
            if (lane >= o) z += y;
        }
        if (lane < (int)(blockDim.x >> 5)) warp_sums[lane] = z - w;
        if (lane == 31) *total = z;
    }
    __syncthreads();
    const unsigned int r = warp_sums[warp] + x - v;
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(1024) cell_scan_blocks(const unsigned int* __restrict__ count,
                                                          unsigned int* __restrict__ start,
                                                          unsigned int* __restrict__ block_sums, int n) {
    __shared__ unsigned int ws[32];
    __shared__ unsigned int tot;
    const int base = blockIdx.x * 4096 + threadIdx.x * 4;
    unsigned int c[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) c[k] = (base + k < n) ? count[base + k] : 0u;
    const unsigned int sum = c[0] + c[1] + c[2] + c[3];
    unsigned int off = block_exclusive_scan(sum, ws, &tot);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (base + k < n) start[base + k] = off;
        off += c[k];
    }
    if (threadIdx.x == 0) block_sums[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(1024) cell_scan_top(unsigned int* __restrict__ block_sums, int nblocks,
                                                       unsigned int* __restrict__ start, int n) {
    __shared__ unsigned int ws[32];
    __shared__ unsigned int tot;
    unsigned int carry = 0;
    for (int b0 = 0; b0 < nblocks; b0 += 1024) {
        const int i = b0 + threadIdx.x;
        const unsigned int v = i < nblocks ? block_sums[i] : 0u;
        const unsigned int x = block_exclusive_scan(v, ws, &tot);
        if (i < nblocks) block_sums[i] = x + carry;
        carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) start[n] = carry;
}

__global__ void __launch_bounds__(1024) cell_scan_add(unsigned int* __restrict__ start,
                                                       const unsigned int* __restrict__ block_sums, int n) {
    const int i = blockIdx.x * 1024 + threadIdx.x;
    if (i < n) start[i] += block_sums[i >> 12];
}

// Each stored photon takes a slot in its cell's segment (cell_count counts
// back down to zero, ready for the next trace) and copies the fields the
// gather reads into 24-byte records.
__global__ void __launch_bounds__(256) photon_scatter(PhotonArgs A, const unsigned int* __restrict__ stored) {
    const unsigned int n = *stored < (unsigned int)A.photon_count ? *stored : (unsigned int)A.photon_count;
    for (unsigned int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int h = A.cell_of[i];
        const unsigned int slot = A.cell_start[h] + atomicSub(A.cell_count + h, 1u) - 1u;
        const float4 pos = A.photons[3 * i], pw = A.photons[3 * i + 1];
        A.seg_posw[slot] = make_float4(pos.x, pos.y, pos.z, pw.x);
        A.seg_powyz[slot] = make_float2(pw.y, pw.z);
        A.seg_photon[slot] = (int)i;
    }
}

// heads/next of the reference's PhotonMap, in the segment order.
__global__ void __launch_bounds__(256) photon_links(PhotonArgs A, const unsigned int* __restrict__ stored) {
    const unsigned int n = *stored < (unsigned int)A.photon_count ? *stored : (unsigned int)A.photon_count;
    for (unsigned int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        const int idx = A.seg_photon[s];
        const int h = A.cell_of[idx];
        const unsigned int end = A.cell_start[h + 1];
        A.next[idx] = (s + 1 < end) ? A.seg_photon[s + 1] : -1;
        if (s == A.cell_start[h]) A.heads[h] = idx;
    }
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

// post/atrous_denoise.frag:50-122 as a shared-memory-tiled stencil.
//
// The 25 taps of pixel p sit at p + step*(i, j): on the lattice of pixels
// congruent to p modulo step.  A block takes a 32 x 8 tile of one of the
// step^2 interleaved sub-images (blockIdx.z = the residue (ox, oy)) and
// stages the (32+4) x (8+4) lattice points its taps read, once each: the
// demodulated irradiance irr = col / max(alb, .01) (when luma(alb) > .02)
// with log(luma(irr) + 1e-3), and the normal and depth.  These depend only on
// the tap position q -- the colour at q clamped into the image
// (CLAMP_TO_EDGE framebuffer texture), the G-buffer and albedo at q wrapped
// around it (the renderer textures' default REPEAT) -- so a staged halo point
// holds exactly what every tap at q computed, and the centre pixel's own
// irradiance and log-luma are its lattice point's.  Each thread then runs
// the 25 weights from shared memory.
//
// Exact build: every expression as the shader orders it (bit-identical to
// the per-tap form).  Fast build: the three edge-stopping factors in one
// exp2, pow(d, sn) * exp(a) * exp(b) = exp2(sn*log2(d) + (a + b)*log2(e)),
// two SFU operations per tap instead of four.
constexpr int kAtW = 32, kAtH = 8, kAtPW = kAtW + 4, kAtPH = kAtH + 4;

__global__ void __launch_bounds__(kAtW * kAtH) atrous_kernel(AtrousArgs A) {
    __shared__ float4 s_irr[kAtPH][kAtPW];   // irradiance xyz, log-luma
    __shared__ float4 s_geo[kAtPH][kAtPW];   // normal xyz, depth
    const int W = A.width, H = A.height, st = A.step;
    const int ox = blockIdx.z % st, oy = blockIdx.z / st;
    const int u0 = blockIdx.x * kAtW, v0 = blockIdx.y * kAtH;
    // tiles past this residue's part of the image (the grid is sized for
    // the largest residue class) have nothing to write
    if (ox + u0 * st >= W || oy + v0 * st >= H) return;
    for (int k = threadIdx.x; k < kAtPW * kAtPH; k += kAtW * kAtH) {
        const int lu = k % kAtPW, lv = k / kAtPW;
        const int qx = ox + (u0 + lu - 2) * st, qy = oy + (v0 + lv - 2) * st;
        const long ri = (long)wrap_repeat(qy, H) * W + wrap_repeat(qx, W);
        const long ki = (long)wrap_clamp(qy, H) * W + wrap_clamp(qx, W);
        const ushort4 g = __ldg(A.gbuf + ri);
        const float3 col = color_at(A, ki);
        const float3 alb = half3(__ldg(A.galb + ri));
        const float3 irr = (luma709(alb) > 0.02f) ? col / vmax(alb, f3(0.01f, 0.01f, 0.01f)) : col;
        const float logl = logf_(luma709(irr) + 1e-3f);
        const float3 n = half3(g);
        s_irr[lv][lu] = make_float4(irr.x, irr.y, irr.z, logl);
        s_geo[lv][lu] = make_float4(n.x, n.y, n.z, halfw(g));
    }
    __syncthreads();
    const int tu = threadIdx.x % kAtW, tv = threadIdx.x / kAtW;
    const int x = ox + (u0 + tu) * st, y = oy + (v0 + tv) * st;
    if (x >= W || y >= H) return;
    const long ci = (long)y * W + x;
    const float4 cgeo = s_geo[tv + 2][tu + 2];
    const float3 c_norm = xyz(cgeo);
    const float c_depth = cgeo.w;
    const float3 c_col = color_at(A, ci);
    if (c_depth > 9000.0f) {
        A.out[ci] = make_float4(c_col.x, c_col.y, c_col.z, 1.0f);
        return;
    }
    const float3 c_alb = half3(__ldg(A.galb + ci));
    const bool has_alb = luma709(c_alb) > 0.02f;
    const float4 cirr = s_irr[tv + 2][tu + 2];
    const float3 c_irr = xyz(cirr);
    const float N = (float)A.sample_count;
    const float sum_l2 = __ldg(A.var + ci);
    const float mean_l = luma709(c_col / gmax(A.exposure, 1e-4f));
    const float variance = gmax(0.0f, sum_l2 / N - mean_l * mean_l);
    const float var_denom = A.sigma_color * A.sigma_color * variance + 1e-6f;
    const float depth_denom = A.sigma_depth * A.sigma_depth + 1e-6f;
    const float c_logl = cirr.w;
    const float hk[5] = {1.0f / 16.0f, 1.0f / 4.0f, 3.0f / 8.0f, 1.0f / 4.0f, 1.0f / 16.0f};
    float3 irr_sum = f3(0, 0, 0);
    float w_sum = 0.0f;
#if !RC_EXACT
    const float kLog2e = 1.4426950408889634f;
    const float inv_dd = kLog2e / depth_denom, inv_vd = kLog2e / var_denom;
    const float c_dinv = 1.0f / (c_depth + 0.001f);
#endif
#pragma unroll
    for (int j = -2; j <= 2; ++j) {
#pragma unroll
        for (int i = -2; i <= 2; ++i) {
            const float4 e = s_irr[tv + 2 + j][tu + 2 + i];
            const float4 g2 = s_geo[tv + 2 + j][tu + 2 + i];
            const float3 irr2 = xyz(e);
            const float hw = hk[i + 2] * hk[j + 2];
#if RC_EXACT
            const float wn = powf_(gmax(0.0f, dot(c_norm, xyz(g2))), A.sigma_normal);
            const float dd = (c_depth - g2.w) / (c_depth + 0.001f);
            const float wd = expf_(-(dd * dd) / depth_denom);
            const float ld = c_logl - e.w;
            const float wc = expf_(-(ld * ld) / var_denom);
            const float w = hw * wn * wd * wc;
#else
            const float d = gmax(0.0f, dot(c_norm, xyz(g2)));
            const float dd = (c_depth - g2.w) * c_dinv;
            const float ld = c_logl - e.w;
            const float ex = -(dd * dd) * inv_dd - (ld * ld) * inv_vd;
            // pow(0, sn) is 0 for sn > 0 and 1 for sn == 0 (powf_ above)
            const float w = d > 0.0f ? hw * exp2f(A.sigma_normal * __log2f(d) + ex)
                                     : (A.sigma_normal == 0.0f ? hw * exp2f(ex) : 0.0f);
#endif
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

// display.frag:11-41 (ACES fit, sRGB encode) and the GL_RGBA8 store of the
// export framebuffer (each channel round(clamp(v, 0, 1) * 255), NaN as 0),
// one thread per pixel, the row written at H-1-y: the order FrameExporter
// writes (stbi_flip_vertically_on_write).  Exact math follows the shader's
// operations in order (mix(x, y, a) = x * (1 - a) + y * a, step(e, x) =
// x < e ? 0 : 1, GLSL clamp = min(max)).
DI float aces_fit(float x) {
    const float a = 2.51f, b = 0.03f, c = 2.43f, d = 0.59f, e = 0.14f;
    return gclamp((x * (a * x + b)) / (x * (c * x + d) + e), 0.0f, 1.0f);
}

DI float linear_to_srgb(float c) {
    const float t = c < 0.0031308f ? 0.0f : 1.0f;
    const float lo = 12.92f * c;
    const float hi = 1.055f * powf_(c, 1.0f / 2.4f) - 0.055f;
    return lo * (1.0f - t) + hi * t;
}

DI unsigned char unorm8(float v) {
    if (!(v == v)) v = 0.0f;
    v = v < 0.0f ? 0.0f : (v > 1.0f ? 1.0f : v);
    return (unsigned char)floorf(v * 255.0f + 0.5f);
}

__global__ void __launch_bounds__(256) display_kernel(DisplayArgs A) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= A.width) return;
    const float n = (float)(A.total_samples > 1 ? A.total_samples : 1);
    const float4 c = __ldg(A.color + (long)y * A.width + x);
    const float r = linear_to_srgb(aces_fit(c.x / n * A.exposure));
    const float g = linear_to_srgb(aces_fit(c.y / n * A.exposure));
    const float b = linear_to_srgb(aces_fit(c.z / n * A.exposure));
    A.out[(long)(A.height - 1 - y) * A.width + x] = make_uchar4(unorm8(r), unorm8(g), unorm8(b), 255);
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

// One persistent grid of the build's refill emission kernel
// (photon_emit_dyn, exact build photon_emit_full_dyn) per device: every SM
// times the blocks that fit it, computed once per device.
#if RC_EXACT
#define RC_EMIT_DYN photon_emit_full_dyn
#else
#define RC_EMIT_DYN photon_emit_dyn
#endif
static int emit_grid() {
    constexpr int kDevs = 64;
    static std::atomic<int> cache[kDevs];
    int dev = 0, sms = 148, pe = 1;
    cudaGetDevice(&dev);
    const bool cached = dev >= 0 && dev < kDevs;
    if (cached) {
        const int g = cache[dev].load(std::memory_order_relaxed);
        if (g > 0) return g;
    }
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&pe, RC_EMIT_DYN, 128, 0);
    const int g = sms * (pe > 0 ? pe : 1);
    if (cached) cache[dev].store(g, std::memory_order_relaxed);
    return g;
}
#undef RC_EMIT_DYN

cudaError_t launch_photon_trace(const PhotonArgs& A, cudaStream_t s, int block) {
    const int b = block <= 64 ? 64 : (block <= 128 ? 128 : 256);
    const int blocks = (A.photon_count + b - 1) / b;
    if (blocks == 0) return cudaSuccess;
    // both phases count in A.queue_len (the queue) and A.work (the refill
    // kernels' and the walks' work counters)
    if (!A.queue || !A.queue_len || !A.work) return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(A.queue_len, 0, sizeof(unsigned int), s);
    if (e != cudaSuccess) return e;
    const bool at_parent = A.scene.depth <= 60;
#if !RC_EXACT
    if (A.split) {
        if (A.scene.max_leaf < 0x10000 && A.spec.max_leaf < 0x10000 && A.diff.max_leaf < 0x10000) {
            // refill emission: one persistent grid (the stack entries pack a
            // leaf's triangle count into 16 bits)
            e = cudaMemsetAsync(A.work, 0, sizeof(unsigned int), s);
            if (e != cudaSuccess) return e;
            photon_emit_dyn<<<emit_grid(), 128, 0, s>>>(A);
        } else {
            photon_emit_kernel<<<blocks, b, 0, s>>>(A);
        }
    } else
#else
    // the refill emission follows the test-at-parent walk (trees up to 60 levels)
    if (at_parent) {
        e = cudaMemsetAsync(A.work, 0, sizeof(unsigned int), s);
        if (e != cudaSuccess) return e;
        photon_emit_full_dyn<<<emit_grid(), 128, 0, s>>>(A);
    } else
#endif
    {
        // without the split (exact math, or scenes too large for the split
        // BVHs): the emission and first segment over the full scene, then
        // the queued walks (photon_trace.comp:168-252 in two launches)
        if (at_parent)
            photon_emit_full_kernel<true><<<blocks, b, 0, s>>>(A);
        else
            photon_emit_full_kernel<false><<<blocks, b, 0, s>>>(A);
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return at_parent ? launch_bounce<true>(A, s, b, blocks) : launch_bounce<false>(A, s, b, blocks);
}

// The cell-sorted layout of the map the trace just stored (4 launches).
cudaError_t launch_photon_layout(const PhotonArgs& A, cudaStream_t s) {
    const int n = A.hash_size;
    const int nb = (n + 4095) / 4096;
    cell_scan_blocks<<<nb, 1024, 0, s>>>(A.cell_count, A.cell_start, A.block_sums, n);
    cell_scan_top<<<1, 1024, 0, s>>>(A.block_sums, nb, A.cell_start, n);
    cell_scan_add<<<(n + 1023) / 1024, 1024, 0, s>>>(A.cell_start, A.block_sums, n);
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    photon_scatter<<<sms * 4, 256, 0, s>>>(A, A.counter);
    photon_links<<<sms * 4, 256, 0, s>>>(A, A.counter);
    return cudaGetLastError();
}

cudaError_t launch_photon_gather(const GatherArgs& A, cudaStream_t s) {
    const dim3 grid((A.img.width + 15) / 16, (A.img.height + 7) / 8);
    if (A.heavy) {
        const cudaError_t e = cudaMemsetAsync(A.heavy_len, 0, sizeof(unsigned int), s);
        if (e != cudaSuccess) return e;
    }
    if (A.scene.depth <= 60)
        photon_gather_kernel<true><<<grid, 128, 0, s>>>(A);
    else
        photon_gather_kernel<false><<<grid, 128, 0, s>>>(A);
    if (A.heavy) {
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        photon_gather_heavy<<<sms * 8, 256, 0, s>>>(A);
    }
    return cudaGetLastError();
}

cudaError_t launch_atrous(const AtrousArgs& A, cudaStream_t s) {
    // residue classes (step^2) x tiles of the largest class's lattice
    const int st = A.step < 1 ? 1 : A.step;
    const int lw = (A.width + st - 1) / st, lh = (A.height + st - 1) / st;
    const dim3 grid((lw + kAtW - 1) / kAtW, (lh + kAtH - 1) / kAtH, st * st);
    atrous_kernel<<<grid, kAtW * kAtH, 0, s>>>(A);
    return cudaGetLastError();
}

cudaError_t launch_normalize(const NormalizeArgs& A, cudaStream_t s) {
    normalize_kernel<<<(A.count + 255) / 256, 256, 0, s>>>(A);
    return cudaGetLastError();
}

cudaError_t launch_display(const DisplayArgs& A, cudaStream_t s) {
    const dim3 grid((A.width + 255) / 256, A.height);
    display_kernel<<<grid, 256, 0, s>>>(A);
    return cudaGetLastError();
}

}  // namespace RC_NS
}  // namespace rc
