// api.cu -- the device half of the C ABI declared in include/retrocam.h.
//
// One rc_ctx = one device, one CUDA stream, the four renderer images, the
// uploaded scene in the kernels' layout (device_scene.h), the SPPM photon map
// and a block of device counters.  Calls are asynchronous on the context's
// stream unless they return data to the host.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <string>
#include <system_error>
#include <thread>
#include <vector>

#include "device_scene.h"
#include "host_checks.h"
#include "retrocam.h"

namespace rc {
namespace exact {
cudaError_t launch_render(const RenderArgs&, cudaStream_t);
cudaError_t launch_photon_trace(const PhotonArgs&, cudaStream_t, int block);
cudaError_t launch_photon_layout(const PhotonArgs&, cudaStream_t);
cudaError_t launch_photon_gather(const GatherArgs&, cudaStream_t);
cudaError_t launch_atrous(const AtrousArgs&, cudaStream_t);
cudaError_t launch_normalize(const NormalizeArgs&, cudaStream_t);
cudaError_t launch_display(const DisplayArgs&, cudaStream_t);
cudaError_t launch_wf_generate(const WaveArgs&, cudaStream_t);
cudaError_t launch_wf_trace(const WaveArgs&, cudaStream_t, int block);
cudaError_t launch_wf_shade(const WaveArgs&, cudaStream_t, int block);
cudaError_t launch_wf_sort(const WaveArgs&, cudaStream_t);
cudaError_t launch_wf_accumulate(const WaveArgs&, cudaStream_t);
}  // namespace exact
namespace fast {
cudaError_t launch_render(const RenderArgs&, cudaStream_t);
cudaError_t launch_photon_trace(const PhotonArgs&, cudaStream_t, int block);
cudaError_t launch_photon_layout(const PhotonArgs&, cudaStream_t);
cudaError_t launch_photon_gather(const GatherArgs&, cudaStream_t);
cudaError_t launch_atrous(const AtrousArgs&, cudaStream_t);
cudaError_t launch_normalize(const NormalizeArgs&, cudaStream_t);
cudaError_t launch_display(const DisplayArgs&, cudaStream_t);
cudaError_t launch_wf_generate(const WaveArgs&, cudaStream_t);
cudaError_t launch_wf_trace(const WaveArgs&, cudaStream_t, int block);
cudaError_t launch_wf_shade(const WaveArgs&, cudaStream_t, int block);
cudaError_t launch_wf_sort(const WaveArgs&, cudaStream_t);
cudaError_t launch_wf_accumulate(const WaveArgs&, cudaStream_t);
}  // namespace fast
namespace vhs {
bool has_pass(int pass);
cudaError_t launch_pass(int pass, const float4* in, float4* out, int w, int h, const rc_vhs_params& p,
                        cudaStream_t s);
}  // namespace vhs
namespace kp {
cudaError_t launch_features(const float4* accum, const ushort4* gbuf, const ushort4* galb, __nv_bfloat16* feat,
                            float4* color, int count, cudaStream_t s);
size_t packed_bytes();
cudaError_t run_inference(const float* params, void* packed, bool repack, const float4* accum, const ushort4* gbuf,
                          const ushort4* galb, void* feat, void* act0, void* act1, float* logits, float4* color,
                          float4* out, int W, int H, unsigned int* err, cudaStream_t s);
}  // namespace kp
}  // namespace rc

using namespace rc;

struct DevBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
};

struct rc_ctx {
    int device = 0;
    int width = 0, height = 0;
    int math_mode = RC_MATH_FAST;
    cudaStream_t stream = nullptr;      // stream the work runs on
    cudaStream_t own_stream = nullptr;  // the context's own stream
    Images img;
    float4* out = nullptr;    // last denoised / normalised frame
    float4* ping = nullptr;   // à-trous ping-pong
    float4* pong = nullptr;
    float4* result = nullptr; // which buffer holds the last output
    int total_samples = 0;
    // scene
    DeviceScene scene;
    bool has_scene = false;
    DevBuf nodes, nodes_packed, nodes4, tri_isect, tri_shade, mats, lights, cdf;
    // SPPM
    DevBuf photons, heads, next, counter, cell_of, cell_count, cell_start, block_sums, seg_photon, seg_posw,
        seg_powyz;
    int photon_cap = 0, hash_cap = 0, last_hash = 0, last_photons = 0;
    float sppm_radius = 0.05f;
    int sppm_iteration = 0;
    // counters
    DevCounters* counters = nullptr;
    unsigned long long launches = 0, h2d = 0, d2h = 0;
    // kernel timing with CUDA events on the launching stream
    bool timing = false;
    struct Timed {
        int kind;
        cudaEvent_t a, b;
    };
    std::vector<Timed> pending;
    double ms[RC_KERNEL_KINDS] = {};
    unsigned long long nlaunch[RC_KERNEL_KINDS] = {};
    // path-tracer engine and wavefront path state
    int engine = RC_ENGINE_WAVEFRONT;
    int chunk_paths = 0;   // 0: default
    int wide_bvh = 0;
    int trace_block = 128, shade_block = 128, photon_block = 128;
    int photon_full_first = 0;
    int refill_lanes = 16, leaf_quarters = 2;
    int refill_min_paths = 1 << 20;
    int material_queues = 0;
    int interior_steps = 6;
    DevBuf wf_o, wf_d, wf_thr, wf_rad, wf_hit, wf_res, wf_seed, wf_rq0, wf_rq1, wf_sq0, wf_sq1, wf_srec0, wf_srec1,
        wf_qlen, wf_mq;
    int wf_capacity = 0;
    // batched frames (rc_render_frames) and their captured graph
    DevBuf frames;
    DevBuf batch_img, batch_segs;   // per-frame images and chunk segments of a batch
    // photon first-segment split: specular / other triangles with own BVHs
    DevBuf sp_nodes, sp_isect, sp_orig, df_nodes, df_isect, ph_queue, ph_queue_len;
    // gather hits per pixel (see GatherArgs::hit_cache); the heavy-pixel
    // list of the fast gather (count, then pixel indices)
    DevBuf gcache, batch_gcache, gheavy;
    DevBuf disp;   // RGBA8 export image of rc_display
    int batch_frames = 0;   // frames of the last rc_render_frames kept in `frames`
    uint64_t gcache_key = 0;
    bool gcache_valid = false;
    unsigned int scene_gen = 0;
    float4* gcache_force = nullptr;   // a batch frame's slice, and its mode
    int gcache_force_mode = 0;
    DeviceScene spec_view, diff_view;
    bool photon_split = false;
    // learned denoiser scratch
    DevBuf kp_feat, kp_act0, kp_act1, kp_logits, kp_color, kp_params, kp_packed;
    std::vector<float> kp_host;   // parameters last uploaded to kp_params
    void* kp_packed_at = nullptr; // kp_packed holds kp_host packed (its address then)
    cudaGraphExec_t graph_exec = nullptr;
    uint64_t graph_key = 0;
    unsigned long long graph_launches = 0;
    int graph_total_samples = 0, graph_iteration = 0;
    float graph_radius = 0.0f;
    std::string err;
};

// Launch one kernel through `fn` (a launcher returning cudaError_t), with
// optional event bracketing for rc_get_kernel_times.
template <class F>
static cudaError_t timed_launch(rc_ctx* ctx, int kind, F fn, int kernels = 1) {
    cudaEvent_t a = nullptr, b = nullptr;
    if (ctx->timing) {
        cudaError_t e = cudaEventCreate(&a);
        if (e == cudaSuccess) e = cudaEventCreate(&b);
        if (e == cudaSuccess) e = cudaEventRecord(a, ctx->stream);
        if (e != cudaSuccess) return e;
    }
    cudaError_t e = fn();
    if (e != cudaSuccess) return e;
    ctx->launches += kernels;
    if (ctx->timing) {
        e = cudaEventRecord(b, ctx->stream);
        if (e != cudaSuccess) return e;
        ctx->pending.push_back({kind, a, b});
    }
    return cudaSuccess;
}

static cudaError_t copy_h2d(rc_ctx* ctx, void* dst, const void* src, size_t n) {
    ctx->h2d += n;
    return cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, ctx->stream);
}

static cudaError_t copy_d2h(rc_ctx* ctx, void* dst, const void* src, size_t n) {
    ctx->d2h += n;
    return cudaMemcpyAsync(dst, src, n, cudaMemcpyDeviceToHost, ctx->stream);
}

static std::mutex g_err_mutex;
static std::string g_create_err;

namespace rc {
// Error text of calls that have no context (read with rc_last_error(NULL)).
__attribute__((visibility("hidden"))) int set_global_error(int code, const char* msg) {
    std::lock_guard<std::mutex> lk(g_err_mutex);
    g_create_err = msg;
    return code;
}
}  // namespace rc

static int fail(rc_ctx* c, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (c) {
        c->err = buf;
    } else {
        std::lock_guard<std::mutex> lk(g_err_mutex);
        g_create_err = buf;
    }
    return code;
}

#define CK(call)                                                                                    \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess)                                                                      \
            return fail(ctx, e_ == cudaErrorMemoryAllocation ? RC_ERR_OUT_OF_MEMORY : RC_ERR_CUDA,  \
                        "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__);       \
    } while (0)

static cudaError_t ensure(DevBuf& b, size_t bytes) {
    if (b.bytes >= bytes && b.ptr) return cudaSuccess;
    if (b.ptr) cudaFree(b.ptr);
    b.ptr = nullptr;
    b.bytes = 0;
    if (bytes == 0) return cudaSuccess;
    cudaError_t e = cudaMalloc(&b.ptr, bytes);
    if (e == cudaSuccess) b.bytes = bytes;
    return e;
}

static void release(DevBuf& b) {
    if (b.ptr) cudaFree(b.ptr);
    b.ptr = nullptr;
    b.bytes = 0;
}

static CamParams cam_params(const rc_camera* c) {
    CamParams k;
    for (int a = 0; a < 3; ++a) {
        k.pos[a] = c->cam_pos[a];
        k.right[a] = c->cam_right[a];
        k.up[a] = c->cam_up[a];
        k.fwd[a] = c->cam_forward[a];
        k.lca[a] = c->lca_delta[a];
    }
    k.focal = c->focal_dist;
    k.lens_radius = c->lens_radius;
    k.tan_half = c->fov_tan_half;
    k.sa = c->sa_strength;
    k.blades = c->aperture_blades;
    return k;
}

extern "C" {

int rc_ctx_create(int width, int height, int device, rc_ctx** out) {
    rc_ctx* ctx = nullptr;
    if (!out || width < 1 || height < 1 || width > 16384 || height > 16384)
        return fail(nullptr, RC_ERR_INVALID_ARG, "rc_ctx_create: bad size %dx%d", width, height);
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || device < 0 || device >= ndev)
        return fail(nullptr, RC_ERR_CUDA, "rc_ctx_create: device %d unavailable (%s)", device,
                    e == cudaSuccess ? "no such device" : cudaGetErrorString(e));
    ctx = new rc_ctx();
    ctx->device = device;
    ctx->width = width;
    ctx->height = height;
    const size_t px = (size_t)width * height;
    auto bail = [&](cudaError_t err, const char* what) {
        fail(nullptr, err == cudaErrorMemoryAllocation ? RC_ERR_OUT_OF_MEMORY : RC_ERR_CUDA, "rc_ctx_create: %s: %s",
             what, cudaGetErrorString(err));
        rc_ctx_destroy(ctx);
        return err == cudaErrorMemoryAllocation ? RC_ERR_OUT_OF_MEMORY : RC_ERR_CUDA;
    };
    if ((e = cudaSetDevice(device)) != cudaSuccess) return bail(e, "cudaSetDevice");
    if ((e = cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking)) != cudaSuccess)
        return bail(e, "cudaStreamCreate");
    ctx->stream = ctx->own_stream;
    if ((e = cudaMalloc(&ctx->img.accum, px * sizeof(float4))) != cudaSuccess) return bail(e, "accum");
    if ((e = cudaMalloc(&ctx->img.gbuf, px * sizeof(ushort4))) != cudaSuccess) return bail(e, "gbuffer");
    if ((e = cudaMalloc(&ctx->img.galb, px * sizeof(ushort4))) != cudaSuccess) return bail(e, "albedo");
    if ((e = cudaMalloc(&ctx->img.var, px * sizeof(float))) != cudaSuccess) return bail(e, "variance");
    if ((e = cudaMalloc(&ctx->out, px * sizeof(float4))) != cudaSuccess) return bail(e, "out");
    if ((e = cudaMalloc(&ctx->ping, px * sizeof(float4))) != cudaSuccess) return bail(e, "ping");
    if ((e = cudaMalloc(&ctx->pong, px * sizeof(float4))) != cudaSuccess) return bail(e, "pong");
    if ((e = cudaMalloc(&ctx->counters, sizeof(DevCounters))) != cudaSuccess) return bail(e, "counters");
    ctx->img.width = width;
    ctx->img.height = height;
    ctx->result = ctx->out;
    if ((e = cudaMemsetAsync(ctx->counters, 0, sizeof(DevCounters), ctx->stream)) != cudaSuccess)
        return bail(e, "memset counters");
    int rcode = rc_reset(ctx);
    if (rcode != RC_OK) {
        fail(nullptr, rcode, "rc_ctx_create: reset failed: %s", ctx->err.c_str());
        rc_ctx_destroy(ctx);
        return rcode;
    }
    *out = ctx;
    return RC_OK;
}

int rc_ctx_destroy(rc_ctx* ctx) {
    if (!ctx) return RC_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (auto& t : ctx->pending) {
        cudaEventDestroy(t.a);
        cudaEventDestroy(t.b);
    }
    for (void* p : {(void*)ctx->img.accum, (void*)ctx->img.gbuf, (void*)ctx->img.galb, (void*)ctx->img.var,
                    (void*)ctx->out, (void*)ctx->ping, (void*)ctx->pong, (void*)ctx->counters})
        if (p) cudaFree(p);
    for (DevBuf* b : {&ctx->nodes, &ctx->nodes_packed, &ctx->nodes4, &ctx->tri_isect, &ctx->tri_shade, &ctx->mats, &ctx->lights, &ctx->cdf,
                      &ctx->photons, &ctx->heads, &ctx->next, &ctx->counter, &ctx->cell_of, &ctx->cell_count,
                      &ctx->cell_start, &ctx->block_sums, &ctx->seg_photon, &ctx->seg_posw, &ctx->seg_powyz,
                      &ctx->wf_o, &ctx->wf_d, &ctx->wf_thr,
                      &ctx->wf_rad, &ctx->wf_hit, &ctx->wf_res, &ctx->wf_seed, &ctx->wf_rq0, &ctx->wf_rq1,
                      &ctx->wf_sq0, &ctx->wf_sq1, &ctx->wf_srec0, &ctx->wf_srec1, &ctx->wf_qlen, &ctx->wf_mq,
                      &ctx->frames,
                      &ctx->kp_feat, &ctx->kp_act0, &ctx->kp_act1, &ctx->kp_logits, &ctx->kp_color,
                      &ctx->kp_params, &ctx->kp_packed, &ctx->batch_img, &ctx->batch_segs, &ctx->sp_nodes,
                      &ctx->sp_isect, &ctx->sp_orig, &ctx->df_nodes, &ctx->df_isect, &ctx->ph_queue,
                      &ctx->ph_queue_len, &ctx->gcache, &ctx->batch_gcache, &ctx->gheavy, &ctx->disp})
        release(*b);
    if (ctx->graph_exec) cudaGraphExecDestroy(ctx->graph_exec);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return RC_OK;
}

int rc_last_error(const rc_ctx* ctx, char* buf, size_t n) {
    if (!buf || n == 0) return RC_ERR_INVALID_ARG;
    std::string s;
    if (ctx) {
        s = ctx->err;
    } else {
        std::lock_guard<std::mutex> lk(g_err_mutex);
        s = g_create_err;
    }
    const size_t k = s.size() < n - 1 ? s.size() : n - 1;
    memcpy(buf, s.data(), k);
    buf[k] = '\0';
    return RC_OK;
}

int rc_set_math_mode(rc_ctx* ctx, int mode) {
    if (!ctx) return RC_ERR_INVALID_ARG;
    if (mode != RC_MATH_FAST && mode != RC_MATH_EXACT) return fail(ctx, RC_ERR_INVALID_ARG, "bad math mode %d", mode);
    ctx->math_mode = mode;
    return RC_OK;
}

int rc_synchronize(rc_ctx* ctx) {
    if (!ctx) return RC_ERR_INVALID_ARG;
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->stream));
    unsigned int word = 0;
    CK(cudaMemcpy(&word, &ctx->counters->error_word, sizeof(word), cudaMemcpyDeviceToHost));
    if (word) return fail(ctx, RC_ERR_DEVICE_GUARD, "kernel guard raised (error word 0x%x)", word);
    return RC_OK;
}

}  // extern "C"

// The kernels' record of interior node n: both children's boxes and refs.
static void node_record(const rc_bvh_node* nodes, const rc_bvh_node& n, NodeRec& r) {
    const rc_bvh_node& L = nodes[n.left_child];
    const rc_bvh_node& R = nodes[n.right_child];
    // x and y bounds of each box side by side (one register pair each for
    // the paired FMA of the fast build's slab test), the z bounds together
    r.a = make_float4(L.aabb_min[0], L.aabb_min[1], L.aabb_max[0], L.aabb_max[1]);
    r.b = make_float4(R.aabb_min[0], R.aabb_min[1], R.aabb_max[0], R.aabb_max[1]);
    r.c = make_float4(L.aabb_min[2], L.aabb_max[2], R.aabb_min[2], R.aabb_max[2]);
    r.d = make_int4(L.prim_count > 0 ? L.prim_start : n.left_child, L.prim_count,
                    R.prim_count > 0 ? R.prim_start : n.right_child, R.prim_count);
}

static void isect_record(const rc_triangle& t, float4* out3) {
    // e1, e2 with the same float subtraction the reference does per test;
    // the w components hold n = e1 x e2 for the fast build's test (the
    // exact build reads only xyz)
    const float e1[3] = {t.v1[0] - t.v0[0], t.v1[1] - t.v0[1], t.v1[2] - t.v0[2]};
    const float e2[3] = {t.v2[0] - t.v0[0], t.v2[1] - t.v0[1], t.v2[2] - t.v0[2]};
    const float nx = e1[1] * e2[2] - e1[2] * e2[1];
    const float ny = e1[2] * e2[0] - e1[0] * e2[2];
    const float nz = e1[0] * e2[1] - e1[1] * e2[0];
    out3[0] = make_float4(t.v0[0], t.v0[1], t.v0[2], nx);
    out3[1] = make_float4(e1[0], e1[1], e1[2], ny);
    out3[2] = make_float4(e2[0], e2[1], e2[2], nz);
}

// A BVH over a subset of the scene's triangles, in the kernels' layout,
// with each subset triangle's index in the full scene.  Only the fast
// build's photon trace walks these, and any BVH gives its walks the same
// hits (ties aside), so they come from a binned SAH builder of their own --
// the reference's builder took about 10 ms for the export scene's 7,936
// specular triangles, most of an upload's host time.
struct SubsetBvh {
    std::vector<NodeRec> recs;
    std::vector<float4> isect;
    std::vector<int> orig;
    rc_bvh_node root;
    int node_count = 0;
    int max_leaf = 0;   // most triangles in one leaf
};

// Binned SAH: 16 bins over the centroid extent of each axis, split where
// (left area x count + right area x count) is least, a leaf of at
// most 4 triangles when no split beats the leaf's cost (and always at 2 or
// fewer); an all-in-one-bin node is split at the median index.  Nodes in
// pre-order from the root at 0, each interior node's children adjacent.
struct BinnedBuilder {
    struct Box {
        float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        // plain compares (a NaN coordinate is skipped), which compile to
        // min/max instructions where fminf/fmaxf are library calls
        void grow(const Box& b) {
            for (int a = 0; a < 3; ++a) {
                lo[a] = b.lo[a] < lo[a] ? b.lo[a] : lo[a];
                hi[a] = b.hi[a] > hi[a] ? b.hi[a] : hi[a];
            }
        }
        void grow(const float* p) {
            for (int a = 0; a < 3; ++a) {
                lo[a] = p[a] < lo[a] ? p[a] : lo[a];
                hi[a] = p[a] > hi[a] ? p[a] : hi[a];
            }
        }
        float area() const {
            if (!(hi[0] >= lo[0])) return 0.0f;
            const float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
            return dx * dy + dy * dz + dz * dx;
        }
    };
    const std::vector<Box>& tb;   // triangle boxes
    const std::vector<float>& cen;  // centroids, 3 per triangle
    std::vector<int>& idx;        // triangle order; a builder owns a range of it
    std::vector<rc_bvh_node> nodes;

    BinnedBuilder(const std::vector<Box>& t, const std::vector<float>& c, std::vector<int>& i)
        : tb(t), cen(c), idx(i) {}

    void set_node(int ni, const Box& b) {
        for (int a = 0; a < 3; ++a) {
            nodes[ni].aabb_min[a] = b.lo[a];
            nodes[ni].aabb_max[a] = b.hi[a];
        }
    }

    // `spawn` levels below this one build their right subtree on a thread
    // of its own (into its own node array, appended afterwards).
    void build(int ni, int begin, int end, int spawn) {
        Box nb, cb;
        for (int i = begin; i < end; ++i) {
            nb.grow(tb[idx[i]]);
            cb.grow(&cen[3 * (size_t)idx[i]]);
        }
        set_node(ni, nb);
        const int n = end - begin;
        auto leaf = [&] {
            nodes[ni].left_child = nodes[ni].right_child = -1;
            nodes[ni].prim_start = begin;
            nodes[ni].prim_count = n;
        };
        if (n <= 2) return leaf();
        int axis = 0;
        float ext = cb.hi[0] - cb.lo[0];
        for (int a = 1; a < 3; ++a)
            if (cb.hi[a] - cb.lo[a] > ext) {
                ext = cb.hi[a] - cb.lo[a];
                axis = a;
            }
        int mid = begin + n / 2;
        if (ext > 0.0f) {
            constexpr int kBins = 16;
            int best = -1;
            float best_cost = INFINITY, scale = 0.0f;
            // one pass bins every axis
            Box bb[3][kBins];
            int bc[3][kBins] = {};
            float sa[3];
            for (int a = 0; a < 3; ++a) {
                const float ea = cb.hi[a] - cb.lo[a];
                sa[a] = ea > 0.0f ? kBins / ea : 0.0f;
            }
            for (int i = begin; i < end; ++i) {
                const int t = idx[i];
                const float* c = &cen[3 * (size_t)t];
                for (int a = 0; a < 3; ++a) {
                    int b = (int)((c[a] - cb.lo[a]) * sa[a]);
                    b = b < 0 ? 0 : (b >= kBins ? kBins - 1 : b);
                    bb[a][b].grow(tb[t]);
                    ++bc[a][b];
                }
            }
            for (int a = 0; a < 3; ++a) {
                if (!(sa[a] > 0.0f)) continue;
                float right_area[kBins];
                int right_count[kBins];
                Box acc;
                int cnt = 0;
                for (int b = kBins - 1; b > 0; --b) {
                    acc.grow(bb[a][b]);
                    cnt += bc[a][b];
                    right_area[b] = acc.area();
                    right_count[b] = cnt;
                }
                Box left;
                int lc = 0;
                for (int b = 1; b < kBins; ++b) {
                    left.grow(bb[a][b - 1]);
                    lc += bc[a][b - 1];
                    if (lc == 0 || right_count[b] == 0) continue;
                    const float cost = left.area() * lc + right_area[b] * right_count[b];
                    if (cost < best_cost) {
                        best_cost = cost;
                        best = b;
                        axis = a;
                        scale = sa[a];
                    }
                }
            }
            auto bin_of = [&](int t) {
                const int b = (int)((cen[3 * (size_t)t + axis] - cb.lo[axis]) * scale);
                return b < 0 ? 0 : (b >= kBins ? kBins - 1 : b);
            };
            // traversal cost ~ one triangle test: split when it beats testing all
            if (best < 0 || (n <= 4 && best_cost >= nb.area() * (n - 1))) {
                if (n <= 4) return leaf();
            } else {
                int* p = std::partition(idx.data() + begin, idx.data() + end, [&](int t) { return bin_of(t) < best; });
                mid = (int)(p - idx.data());
            }
        } else if (n <= 4) {
            return leaf();
        }
        if (mid <= begin || mid >= end) mid = begin + n / 2;
        const int l = (int)nodes.size();
        nodes.emplace_back();
        nodes.emplace_back();
        nodes[ni].left_child = l;
        nodes[ni].right_child = l + 1;
        nodes[ni].prim_start = 0;
        nodes[ni].prim_count = 0;
        if (spawn <= 0 || n < 4096) {
            build(l, begin, mid, 0);
            build(l + 1, mid, end, 0);
            return;
        }
        BinnedBuilder right(tb, cen, idx);
        right.nodes.reserve(2 * (size_t)(end - mid));
        right.nodes.emplace_back();
        // no exception may leave the C ABI: without a thread to be had, the
        // right subtree is built here after the left one (disjoint ranges)
        std::thread job;
        try {
            job = std::thread([&] { right.build(0, mid, end, spawn - 1); });
        } catch (const std::system_error&) {
        }
        build(l, begin, mid, spawn - 1);
        if (job.joinable())
            job.join();
        else
            right.build(0, mid, end, spawn - 1);
        // the right subtree's root takes slot l + 1, its other nodes follow
        const int base = (int)nodes.size() - 1;
        auto place = [&](int j) { return j == 0 ? l + 1 : base + j; };
        for (size_t j = 0; j < right.nodes.size(); ++j) {
            rc_bvh_node m = right.nodes[j];
            if (m.prim_count <= 0) {
                m.left_child = place(m.left_child);
                m.right_child = place(m.right_child);
            }
            if (j == 0) nodes[l + 1] = m;
            else nodes.push_back(m);
        }
    }
};

static bool build_subset(const std::vector<rc_triangle>& in, int scene_tris, SubsetBvh& out) {
    const int n = (int)in.size();
    if (n == 0) return false;
    std::vector<BinnedBuilder::Box> tb(n);
    std::vector<float> cen(3 * (size_t)n);
    std::vector<int> idx(n);
    for (int i = 0; i < n; ++i) {
        tb[i].grow(in[i].v0);
        tb[i].grow(in[i].v1);
        tb[i].grow(in[i].v2);
        for (int a = 0; a < 3; ++a) cen[3 * (size_t)i + a] = (in[i].v0[a] + in[i].v1[a] + in[i].v2[a]) * (1.0f / 3.0f);
        idx[i] = i;
    }
    BinnedBuilder B(tb, cen, idx);
    B.nodes.reserve(2 * (size_t)n);
    B.nodes.emplace_back();
    B.build(0, 0, n, 2);   // up to four subtrees at once
    std::vector<rc_triangle> tris(n);
    for (int i = 0; i < n; ++i) tris[i] = in[idx[i]];
    const std::vector<rc_bvh_node>& nodes = B.nodes;
    const int nn = (int)nodes.size();
    out.recs.assign(nn, NodeRec{});
    out.max_leaf = 0;
    for (int i = 0; i < nn; ++i) {
        if (nodes[i].prim_count <= 0) node_record(nodes.data(), nodes[i], out.recs[i]);
        if (nodes[i].prim_count > out.max_leaf) out.max_leaf = nodes[i].prim_count;
    }
    out.isect.resize(3 * (size_t)n);
    out.orig.resize(n);
    for (int i = 0; i < n; ++i) {
        isect_record(tris[i], &out.isect[3 * (size_t)i]);
        int o;
        memcpy(&o, &tris[i].pad6, sizeof(int));   // the full-scene index rides in a pad field
        if (o < 0 || o >= scene_tris) return false;
        out.orig[i] = o;
    }
    out.root = nodes[0];
    out.node_count = nn;
    return true;
}

static DeviceScene subset_view(const SubsetBvh& b, const DevBuf& nodes, const DevBuf& isect) {
    DeviceScene S;
    S.nodes = (const NodeRec*)nodes.ptr;
    S.tri_isect = (const float4*)isect.ptr;
    S.node_count = b.node_count;
    S.tri_count = (int)b.orig.size();
    for (int a = 0; a < 3; ++a) {
        S.root_min[a] = b.root.aabb_min[a];
        S.root_max[a] = b.root.aabb_max[a];
    }
    S.root_ref = b.root.prim_count > 0 ? b.root.prim_start : 0;
    S.root_count = b.root.prim_count;
    S.max_leaf = b.max_leaf;
    return S;
}

// Collapses the binary BVH below interior node `bin` into 4-wide nodes,
// pre-order, returning the index of the node made for `bin`.  A node takes
// its two children and keeps opening the interior child of largest surface
// area until it holds four.
static float node_area(const rc_bvh_node& n) {
    const float dx = n.aabb_max[0] - n.aabb_min[0], dy = n.aabb_max[1] - n.aabb_min[1];
    const float dz = n.aabb_max[2] - n.aabb_min[2];
    return dx * dy + dy * dz + dz * dx;
}

static int collapse4(const rc_bvh_node* nodes, int bin, std::vector<Node4>& out) {
    int kids[4] = {nodes[bin].left_child, nodes[bin].right_child, -1, -1};
    int n = 2;
    while (n < 4) {
        int best = -1;
        float best_area = -1.0f;
        for (int k = 0; k < n; ++k) {
            const rc_bvh_node& c = nodes[kids[k]];
            if (c.prim_count <= 0 && node_area(c) > best_area) {
                best_area = node_area(c);
                best = k;
            }
        }
        if (best < 0) break;
        const rc_bvh_node& c = nodes[kids[best]];
        kids[best] = c.left_child;
        kids[n++] = c.right_child;
    }
    const int self = (int)out.size();
    out.push_back(Node4());
    float lo[3][4], hi[3][4];
    int ref[4], cnt[4];
    for (int k = 0; k < 4; ++k) {
        if (k < n) {
            const rc_bvh_node& c = nodes[kids[k]];
            for (int a = 0; a < 3; ++a) {
                lo[a][k] = c.aabb_min[a];
                hi[a][k] = c.aabb_max[a];
            }
            if (c.prim_count > 0) {
                ref[k] = c.prim_start;
                cnt[k] = c.prim_count;
            } else {
                ref[k] = collapse4(nodes, kids[k], out);
                cnt[k] = 0;
            }
        } else {
            for (int a = 0; a < 3; ++a) {
                lo[a][k] = 0.0f;
                hi[a][k] = 0.0f;
            }
            ref[k] = 0;
            cnt[k] = -1;
        }
    }
    Node4& w = out[self];
    w.lox = make_float4(lo[0][0], lo[0][1], lo[0][2], lo[0][3]);
    w.hix = make_float4(hi[0][0], hi[0][1], hi[0][2], hi[0][3]);
    w.loy = make_float4(lo[1][0], lo[1][1], lo[1][2], lo[1][3]);
    w.hiy = make_float4(hi[1][0], hi[1][1], hi[1][2], hi[1][3]);
    w.loz = make_float4(lo[2][0], lo[2][1], lo[2][2], lo[2][3]);
    w.hiz = make_float4(hi[2][0], hi[2][1], hi[2][2], hi[2][3]);
    w.ref = make_int4(ref[0], ref[1], ref[2], ref[3]);
    w.cnt = make_int4(cnt[0], cnt[1], cnt[2], cnt[3]);
    return self;
}

extern "C" {

int rc_ctx_set_stream(rc_ctx* ctx, void* cuda_stream) {
    if (!ctx) return RC_ERR_INVALID_ARG;
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->stream = cuda_stream ? (cudaStream_t)cuda_stream : ctx->own_stream;
    return RC_OK;
}

int rc_set_kernel_timing(rc_ctx* ctx, int enable) {
    if (!ctx) return RC_ERR_INVALID_ARG;
    ctx->timing = enable != 0;
    return RC_OK;
}

int rc_get_kernel_times(rc_ctx* ctx, double* ms_out, uint64_t* launches_out) {
    if (!ctx) return RC_ERR_INVALID_ARG;
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->stream));
    for (auto& t : ctx->pending) {
        float ms = 0.0f;
        CK(cudaEventElapsedTime(&ms, t.a, t.b));
        ctx->ms[t.kind] += ms;
        ctx->nlaunch[t.kind]++;
        cudaEventDestroy(t.a);
        cudaEventDestroy(t.b);
    }
    ctx->pending.clear();
    for (int k = 0; k < RC_KERNEL_KINDS; ++k) {
        if (ms_out) ms_out[k] = ctx->ms[k];
        if (launches_out) launches_out[k] = ctx->nlaunch[k];
        ctx->ms[k] = 0.0;
        ctx->nlaunch[k] = 0;
    }
    return RC_OK;
}

// Scenes up to this size also get the photon first-segment split (two more
// host SAH builds at upload).
static const int kSplitMaxTris = 1 << 18;

// The photon trace's first-segment split (fast build): BVHs over the
// specular (metal or glass) triangles and over the others, each triangle's
// scene index kept.  Host work only, on the caller's arrays.
static bool build_split(const rc_triangle* tris, int tri_count, const rc_material* mats, SubsetBvh& sb,
                        SubsetBvh& db) {
    std::vector<char> is_spec(tri_count);
    int n_spec = 0;
    for (int i = 0; i < tri_count; ++i) {
        const rc_material& m = mats[tris[i].mat_index];
        is_spec[i] = m.metallic > 0.5f || m.transmission > 0.5f;
        n_spec += is_spec[i];
    }
    if (n_spec == 0 || n_spec == tri_count) return false;
    auto make = [&](bool spec, int count, SubsetBvh& out) {
        std::vector<rc_triangle> sub;
        sub.reserve(count);
        for (int i = 0; i < tri_count; ++i) {
            if ((is_spec[i] != 0) != spec) continue;
            rc_triangle t = tris[i];
            memcpy(&t.pad6, &i, sizeof(int));
            sub.push_back(t);
        }
        return build_subset(sub, tri_count, out);
    };
    return make(true, n_spec, sb) && make(false, tri_count - n_spec, db);
}

// Joins a helper thread on every way out of the scope.
struct JoinOnExit {
    std::thread t;
    ~JoinOnExit() {
        if (t.joinable()) t.join();
    }
};

int rc_scene_upload(rc_ctx* ctx, const rc_triangle* tris, int tri_count, const rc_bvh_node* nodes,
                    int node_count, const rc_material* mats, int material_count, const rc_light* lights,
                    int light_count, float total_light_power) {
    if (!ctx) return RC_ERR_INVALID_ARG;
    if (tri_count < 0 || node_count < 1 || material_count < 1 || light_count < 0 || !nodes || !mats ||
        (tri_count > 0 && !tris) || (light_count > 0 && !lights))
        return fail(ctx, RC_ERR_INVALID_ARG, "rc_scene_upload: bad arguments");
    // ---- validate: a tree rooted at node 0 over [0, tri_count) ----
    std::vector<int> seen(node_count, 0), depth(node_count, 0);
    std::vector<int> todo;
    todo.push_back(0);
    seen[0] = 1;
    int max_depth = 0, max_leaf = 0;
    while (!todo.empty()) {
        const int i = todo.back();
        todo.pop_back();
        const rc_bvh_node& n = nodes[i];
        if (n.prim_count > 0) {
            if (n.prim_start < 0 || (long)n.prim_start + n.prim_count > tri_count)
                return fail(ctx, RC_ERR_BAD_SCENE, "node %d: primitives [%d,+%d) outside %d triangles", i,
                            n.prim_start, n.prim_count, tri_count);
            if (depth[i] > max_depth) max_depth = depth[i];
            if (n.prim_count > max_leaf) max_leaf = n.prim_count;
            continue;
        }
        if (tri_count == 0 && i == 0) break;
        for (int ch : {n.left_child, n.right_child}) {
            if (ch < 0 || ch >= node_count)
                return fail(ctx, RC_ERR_BAD_SCENE, "node %d: child index %d out of range [0,%d)", i, ch, node_count);
            if (seen[ch]) return fail(ctx, RC_ERR_BAD_SCENE, "node %d: child %d referenced twice", i, ch);
            seen[ch] = 1;
            depth[ch] = depth[i] + 1;
            todo.push_back(ch);
        }
    }
    for (int i = 0; i < tri_count; ++i)
        if (tris[i].mat_index < 0 || tris[i].mat_index >= material_count)
            return fail(ctx, RC_ERR_BAD_SCENE, "triangle %d: material %d out of range", i, tris[i].mat_index);
    // the photon-split BVHs build on a helper thread while the rest of the
    // upload converts and copies
    const bool want_split = tri_count > 0 && tri_count <= kSplitMaxTris && light_count > 0;
    SubsetBvh sb, db;
    bool built = false;
    JoinOnExit split_job;
    bool split_inline = false;  // no helper thread could be started: build at the join
    if (want_split) {
        try {
            split_job.t = std::thread([&] { built = build_split(tris, tri_count, mats, sb, db); });
        } catch (const std::system_error&) {
            split_inline = true;
        }
    }
    // ---- convert to the kernels' layout ----
    std::vector<NodeRec> recs(node_count);
    memset(recs.data(), 0, recs.size() * sizeof(NodeRec));
    for (int i = 0; i < node_count; ++i) {
        const rc_bvh_node& n = nodes[i];
        if (n.prim_count > 0 || !seen[i] || (tri_count == 0)) continue;
        node_record(nodes, n, recs[i]);
    }
    // packed-reference copy for the refill trace (DeviceScene::nodes_packed)
    const bool packable = tri_count > 0 && max_leaf <= 31 && tri_count < (1 << 26);
    auto packed_ref = [&](int c) {
        return nodes[c].prim_count > 0
                   ? (int)(0x80000000u | ((unsigned int)nodes[c].prim_start << 5) | (unsigned int)nodes[c].prim_count)
                   : c;
    };
    std::vector<NodeRec> precs;
    if (packable) {
        precs = recs;
        for (int i = 0; i < node_count; ++i) {
            const rc_bvh_node& n = nodes[i];
            if (n.prim_count > 0 || !seen[i]) continue;
            precs[i].d = make_int4(packed_ref(n.left_child), packed_ref(n.right_child), 0, 0);
        }
    }
    // 4-wide copy for the fast build's traversal; a tree deeper than any SAH
    // build makes keeps the binary traversal (the collapse recurses per level).
    std::vector<Node4> wide;
    if (tri_count > 0 && nodes[0].prim_count <= 0 && max_depth <= 256) collapse4(nodes, 0, wide);
    std::vector<float4> isect(3 * (size_t)tri_count), shade(3 * (size_t)tri_count);
    for (int i = 0; i < tri_count; ++i) {
        const rc_triangle& t = tris[i];
        isect_record(t, &isect[3 * (size_t)i]);
        float mbits;
        memcpy(&mbits, &t.mat_index, 4);
        shade[3 * i + 0] = make_float4(t.n0[0], t.n0[1], t.n0[2], mbits);
        shade[3 * i + 1] = make_float4(t.n1[0], t.n1[1], t.n1[2], 0.0f);
        shade[3 * i + 2] = make_float4(t.n2[0], t.n2[1], t.n2[2], 0.0f);
    }
    std::vector<float> cdf(light_count > 0 ? light_count : 1, 1.0f);
    for (int i = 0; i < light_count; ++i) cdf[i] = lights[i].cdf_weight;
    rc_light stub;
    memset(&stub, 0, sizeof(stub));
    CK(cudaSetDevice(ctx->device));
    CK(cudaStreamSynchronize(ctx->stream));  // buffers may be in use by queued work
    CK(ensure(ctx->nodes, recs.size() * sizeof(NodeRec)));
    CK(ensure(ctx->nodes4, std::max<size_t>(sizeof(Node4), wide.size() * sizeof(Node4))));
    if (!wide.empty()) CK(copy_h2d(ctx, ctx->nodes4.ptr, wide.data(), wide.size() * sizeof(Node4)));
    CK(ensure(ctx->tri_isect, std::max<size_t>(16, isect.size() * sizeof(float4))));
    CK(ensure(ctx->tri_shade, std::max<size_t>(16, shade.size() * sizeof(float4))));
    CK(ensure(ctx->mats, (size_t)material_count * sizeof(rc_material)));
    CK(ensure(ctx->lights, (size_t)(light_count > 0 ? light_count : 1) * sizeof(rc_light)));
    CK(ensure(ctx->cdf, cdf.size() * sizeof(float)));
    CK(copy_h2d(ctx, ctx->nodes.ptr, recs.data(), recs.size() * sizeof(NodeRec)));
    if (packable) {
        CK(ensure(ctx->nodes_packed, precs.size() * sizeof(NodeRec)));
        CK(copy_h2d(ctx, ctx->nodes_packed.ptr, precs.data(), precs.size() * sizeof(NodeRec)));
    }
    if (tri_count > 0) {
        CK(copy_h2d(ctx, ctx->tri_isect.ptr, isect.data(), isect.size() * sizeof(float4)));
        CK(copy_h2d(ctx, ctx->tri_shade.ptr, shade.data(), shade.size() * sizeof(float4)));
    }
    CK(copy_h2d(ctx, ctx->mats.ptr, mats, (size_t)material_count * sizeof(rc_material)));
    CK(copy_h2d(ctx, ctx->lights.ptr, light_count > 0 ? (const void*)lights : (const void*)&stub,
                (size_t)(light_count > 0 ? light_count : 1) * sizeof(rc_light)));
    CK(copy_h2d(ctx, ctx->cdf.ptr, cdf.data(), cdf.size() * sizeof(float)));
    CK(cudaStreamSynchronize(ctx->stream));  // host staging vectors go out of scope
    DeviceScene& S = ctx->scene;
    S.nodes = (const NodeRec*)ctx->nodes.ptr;
    S.nodes_packed = packable ? (const NodeRec*)ctx->nodes_packed.ptr : nullptr;
    S.root_packed = packable ? packed_ref(0) : 0;
    S.nodes4 = wide.empty() ? nullptr : (const Node4*)ctx->nodes4.ptr;
    S.tri_isect = (const float4*)ctx->tri_isect.ptr;
    S.tri_shade = (const float4*)ctx->tri_shade.ptr;
    S.materials = (const float4*)ctx->mats.ptr;
    S.lights = (const float4*)ctx->lights.ptr;
    S.light_cdf = (const float*)ctx->cdf.ptr;
    S.node_count = node_count;
    S.tri_count = tri_count;
    S.material_count = material_count;
    S.light_count = light_count;
    S.total_light_power = total_light_power;
    for (int a = 0; a < 3; ++a) {
        S.root_min[a] = nodes[0].aabb_min[a];
        S.root_max[a] = nodes[0].aabb_max[a];
    }
    if (tri_count == 0) {
        // no geometry: an inverted root box that no ray can enter
        for (int a = 0; a < 3; ++a) {
            S.root_min[a] = 1e30f;
            S.root_max[a] = -1e30f;
        }
    }
    S.root_ref = nodes[0].prim_count > 0 ? nodes[0].prim_start : 0;
    S.root_count = nodes[0].prim_count;
    S.depth = max_depth;
    S.max_leaf = max_leaf;
    // ---- first-segment split of the photon trace (fast build): BVHs over
    //      the specular (metal or glass) triangles and over the others ----
    ctx->photon_split = false;
    if (want_split) {
        if (split_inline)
            built = build_split(tris, tri_count, mats, sb, db);
        else
            split_job.t.join();
        if (built) {
            CK(ensure(ctx->sp_nodes, sb.recs.size() * sizeof(NodeRec)));
            CK(ensure(ctx->sp_isect, sb.isect.size() * sizeof(float4)));
            CK(ensure(ctx->sp_orig, sb.orig.size() * sizeof(int)));
            CK(ensure(ctx->df_nodes, db.recs.size() * sizeof(NodeRec)));
            CK(ensure(ctx->df_isect, db.isect.size() * sizeof(float4)));
            CK(copy_h2d(ctx, ctx->sp_nodes.ptr, sb.recs.data(), sb.recs.size() * sizeof(NodeRec)));
            CK(copy_h2d(ctx, ctx->sp_isect.ptr, sb.isect.data(), sb.isect.size() * sizeof(float4)));
            CK(copy_h2d(ctx, ctx->sp_orig.ptr, sb.orig.data(), sb.orig.size() * sizeof(int)));
            CK(copy_h2d(ctx, ctx->df_nodes.ptr, db.recs.data(), db.recs.size() * sizeof(NodeRec)));
            CK(copy_h2d(ctx, ctx->df_isect.ptr, db.isect.data(), db.isect.size() * sizeof(float4)));
            CK(cudaStreamSynchronize(ctx->stream));
            ctx->spec_view = subset_view(sb, ctx->sp_nodes, ctx->sp_isect);
            ctx->diff_view = subset_view(db, ctx->df_nodes, ctx->df_isect);
            ctx->photon_split = true;
        }
    }
    ctx->scene_gen++;
    ctx->has_scene = true;
    return RC_OK;
}

static int launch_err(rc_ctx* ctx, cudaError_t e, const char* what) {
    if (e == cudaSuccess) return RC_OK;
    return fail(ctx, RC_ERR_CUDA, "%s launch failed: %s", what, cudaGetErrorString(e));
}

int rc_set_engine(rc_ctx* ctx, int engine, int chunk_paths) {
    if (!ctx) return RC_ERR_INVALID_ARG;
    if ((engine != RC_ENGINE_MEGAKERNEL && engine != RC_ENGINE_WAVEFRONT && engine != RC_ENGINE_WAVEFRONT_STATIC) ||
        chunk_paths < 0)
        return fail(ctx, RC_ERR_INVALID_ARG, "rc_set_engine: bad engine %d or chunk %d", engine, chunk_paths);
    ctx->engine = engine;
    ctx->chunk_paths = chunk_paths;
    return RC_OK;
}

static bool valid_block(int b) { return b == 0 || b == 64 || b == 128 || b == 256; }

int rc_set_tuning(rc_ctx* ctx, const rc_tuning* t) {
    if (!ctx) return RC_ERR_INVALID_ARG;
    if (!t) return fail(ctx, RC_ERR_INVALID_ARG, "rc_set_tuning: null tuning");
    if ((t->engine != RC_ENGINE_MEGAKERNEL && t->engine != RC_ENGINE_WAVEFRONT &&
         t->engine != RC_ENGINE_WAVEFRONT_STATIC) ||
        t->chunk_paths < 0 || (t->wide_bvh & ~(RC_WIDE_PATHS | RC_WIDE_PHOTONS)) || !valid_block(t->trace_block) ||
        !valid_block(t->shade_block) || !valid_block(t->photon_block) ||
        (t->photon_full_first != 0 && t->photon_full_first != 1) || t->refill_lanes < 0 || t->refill_lanes > 32 ||
        t->leaf_quarters < 0 || t->leaf_quarters > 4 || t->refill_min_paths < 0 ||
        (t->material_queues != 0 && t->material_queues != 1) || t->interior_steps < 0 || t->interior_steps > 8)
        return fail(ctx, RC_ERR_INVALID_ARG,
                    "rc_set_tuning: engine %d chunk %d wide %d blocks %d/%d/%d first %d refill %d leaf %d "
                    "refill_min %d material_queues %d interior_steps %d",
                    t->engine, t->chunk_paths, t->wide_bvh, t->trace_block, t->shade_block, t->photon_block,
                    t->photon_full_first, t->refill_lanes, t->leaf_quarters, t->refill_min_paths,
                    t->material_queues, t->interior_steps);
    ctx->engine = t->engine;
    ctx->chunk_paths = t->chunk_paths;
    ctx->wide_bvh = t->wide_bvh;
    ctx->trace_block = t->trace_block ? t->trace_block : 128;
    ctx->shade_block = t->shade_block ? t->shade_block : 128;
    ctx->photon_block = t->photon_block ? t->photon_block : 128;
    ctx->photon_full_first = t->photon_full_first;
    ctx->refill_lanes = t->refill_lanes ? t->refill_lanes : 16;
    ctx->leaf_quarters = t->leaf_quarters ? t->leaf_quarters : 2;
    ctx->refill_min_paths = t->refill_min_paths ? t->refill_min_paths : (1 << 20);
    ctx->material_queues = t->material_queues;
    ctx->interior_steps = t->interior_steps ? t->interior_steps : 6;
    return RC_OK;
}

int rc_get_tuning(rc_ctx* ctx, rc_tuning* out) {
    if (!ctx) return RC_ERR_INVALID_ARG;
    if (!out) return fail(ctx, RC_ERR_INVALID_ARG, "rc_get_tuning: null output");
    out->engine = ctx->engine;
    out->chunk_paths = ctx->chunk_paths;
    out->wide_bvh = ctx->wide_bvh;
    out->trace_block = ctx->trace_block;
    out->shade_block = ctx->shade_block;
    out->photon_block = ctx->photon_block;
    out->photon_full_first = ctx->photon_full_first;
    out->refill_lanes = ctx->refill_lanes;
    out->leaf_quarters = ctx->leaf_quarters;
    out->refill_min_paths = ctx->refill_min_paths;
    out->material_queues = ctx->material_queues;
    out->interior_steps = ctx->interior_steps;
    return RC_OK;
}

// The scene as one class of rays sees it: without the 4-wide nodes unless the
// context's wide_bvh bit for that class is set.
static DeviceScene scene_for(const rc_ctx* ctx, int wide_bit) {
    DeviceScene S = ctx->scene;
    if (!(ctx->wide_bvh & wide_bit)) S.nodes4 = nullptr;
    return S;
}

// Default wavefront chunk: every sample of the call, up to 16M paths.
static const int kDefaultChunkPaths = 16 << 20;

// Paths in flight for a call of n_spp samples with or without lens channels.
static long wavefront_capacity(const rc_ctx* ctx, int n_spp, bool lca, int* samples_per_chunk) {
    const int tiles_x = (ctx->width + 7) / 8, tiles_y = (ctx->height + 3) / 4;
    const long per_sample = (long)tiles_x * tiles_y * 32 * (lca ? 3 : 1);
    const long cap_paths = ctx->chunk_paths > 0 ? ctx->chunk_paths : kDefaultChunkPaths;
    const int ns = (int)std::max<long>(1, std::min<long>(n_spp, cap_paths / per_sample));
    if (samples_per_chunk) *samples_per_chunk = ns;
    return per_sample * ns;
}

static bool lca_active(const CamParams& c) {
    // the device decides LCA with the same float expression
    return (fabsf(c.lca[0]) + fabsf(c.lca[2])) > 1e-4f;
}

static int wavefront_reserve(rc_ctx* ctx, long cap) {
    if (cap > ctx->wf_capacity) {
        CK(cudaStreamSynchronize(ctx->stream));
        const size_t n = (size_t)cap;
        CK(ensure(ctx->wf_o, n * 16));
        CK(ensure(ctx->wf_d, n * 16));
        CK(ensure(ctx->wf_thr, n * 16));
        CK(ensure(ctx->wf_rad, n * 16));
        CK(ensure(ctx->wf_hit, n * 16));
        CK(ensure(ctx->wf_res, n * 16));
        CK(ensure(ctx->wf_seed, n * 4));
        CK(ensure(ctx->wf_rq0, n * 4));
        CK(ensure(ctx->wf_rq1, n * 4));
        CK(ensure(ctx->wf_sq0, n * 4));
        CK(ensure(ctx->wf_sq1, n * 4));
        CK(ensure(ctx->wf_srec0, n * 48));
        CK(ensure(ctx->wf_srec1, n * 48));
        CK(ensure(ctx->wf_mq, n * 4));
        CK(ensure(ctx->wf_qlen, 8 * sizeof(unsigned int)));
        ctx->wf_capacity = (int)cap;
    }
    return RC_OK;
}

// Path state of the wavefront engine and the chunk-invariant launch fields.
static WaveArgs wave_args(rc_ctx* ctx, const DeviceScene& scene, int nee_enabled, float firefly_clamp) {
    const int W = ctx->width, H = ctx->height;
    const int tiles_x = (W + 7) / 8, tiles_y = (H + 3) / 4;
    WaveArgs A;
    A.scene = scene;
    A.segs = nullptr;
    A.nsegs = 1;
    A.width = W;
    A.height = H;
    WaveBuffers& B = A.wb;
    B.o = (float4*)ctx->wf_o.ptr;
    B.d = (float4*)ctx->wf_d.ptr;
    B.thr = (float4*)ctx->wf_thr.ptr;
    B.rad = (float4*)ctx->wf_rad.ptr;
    B.hit = (float4*)ctx->wf_hit.ptr;
    B.res = (float4*)ctx->wf_res.ptr;
    B.seed = (uint32_t*)ctx->wf_seed.ptr;
    B.rq[0] = (int*)ctx->wf_rq0.ptr;
    B.rq[1] = (int*)ctx->wf_rq1.ptr;
    B.sq[0] = (int*)ctx->wf_sq0.ptr;
    B.sq[1] = (int*)ctx->wf_sq1.ptr;
    B.srec[0] = (float4*)ctx->wf_srec0.ptr;
    B.srec[1] = (float4*)ctx->wf_srec1.ptr;
    B.qlen = (unsigned int*)ctx->wf_qlen.ptr;
    B.mq = (int*)ctx->wf_mq.ptr;
    B.capacity = ctx->wf_capacity;
    A.nee_enabled = nee_enabled;
    A.firefly_clamp = firefly_clamp;
    A.tiles_x = tiles_x;
    A.npix = tiles_x * tiles_y * 32;
    A.counters = ctx->counters;
    A.dynamic_fetch = ctx->engine == RC_ENGINE_WAVEFRONT ? 1 : 0;
    A.refill_min_paths = ctx->refill_min_paths;
    A.refill_lanes = ctx->refill_lanes;
    A.leaf_quarters = ctx->leaf_quarters;
    A.material_queues = ctx->material_queues;
    A.interior_steps = ctx->interior_steps;
    A.bounce = 0;
    return A;
}

// One chunk: generate, 7 traces and 6 shades interleaved, accumulate.
static int wavefront_chunk(rc_ctx* ctx, WaveArgs& A) {
    const bool ex = ctx->math_mode == RC_MATH_EXACT;
    A.bounce = 0;
    cudaError_t e = timed_launch(ctx, RC_KERNEL_WF_GENERATE, [&] {
        return ex ? exact::launch_wf_generate(A, ctx->stream) : fast::launch_wf_generate(A, ctx->stream);
    });
    if (e != cudaSuccess) return launch_err(ctx, e, "wavefront generate");
    for (int b = 0; b <= 6; ++b) {
        A.bounce = b;
        e = timed_launch(ctx, RC_KERNEL_WF_TRACE, [&] {
            return ex ? exact::launch_wf_trace(A, ctx->stream, ctx->trace_block)
                      : fast::launch_wf_trace(A, ctx->stream, ctx->trace_block);
        });
        if (e != cudaSuccess) return launch_err(ctx, e, "wavefront trace");
        if (b == 6) break;
        if (A.material_queues) {
            e = timed_launch(ctx, RC_KERNEL_WF_SORT, [&] {
                return ex ? exact::launch_wf_sort(A, ctx->stream) : fast::launch_wf_sort(A, ctx->stream);
            });
            if (e != cudaSuccess) return launch_err(ctx, e, "wavefront sort");
        }
        e = timed_launch(ctx, RC_KERNEL_WF_SHADE, [&] {
            return ex ? exact::launch_wf_shade(A, ctx->stream, ctx->shade_block)
                      : fast::launch_wf_shade(A, ctx->stream, ctx->shade_block);
        });
        if (e != cudaSuccess) return launch_err(ctx, e, "wavefront shade");
    }
    e = timed_launch(ctx, RC_KERNEL_WF_ACCUMULATE, [&] {
        return ex ? exact::launch_wf_accumulate(A, ctx->stream) : fast::launch_wf_accumulate(A, ctx->stream);
    });
    if (e != cudaSuccess) return launch_err(ctx, e, "wavefront accumulate");
    return RC_OK;
}

static int wavefront_render(rc_ctx* ctx, const RenderArgs& R) {
    const bool lca = lca_active(R.cam);
    const int C = lca ? 3 : 1;
    int ns = 1;
    const long cap = wavefront_capacity(ctx, R.n_spp, lca, &ns);
    const int rr = wavefront_reserve(ctx, cap);
    if (rr != RC_OK) return rr;
    WaveArgs A = wave_args(ctx, R.scene, R.nee_enabled, R.firefly_clamp);
    A.one.img = R.img;
    A.one.cam = R.cam;
    A.one.channels = C;
    A.one.path_base = 0;
    for (int s0 = 0; s0 < R.n_spp; s0 += ns) {
        A.one.first_frame = R.first_frame + s0;
        A.one.n_samples = std::min(ns, R.n_spp - s0);
        A.paths = (int)((long)A.npix * C * A.one.n_samples);
        const int r = wavefront_chunk(ctx, A);
        if (r != RC_OK) return r;
    }
    return RC_OK;
}

int rc_render(rc_ctx* ctx, const rc_camera* cam, const rc_settings* settings, int first_frame, int n_spp) {
    if (!ctx) return RC_ERR_INVALID_ARG;
    if (!cam || !settings || first_frame < 0 || n_spp < 0)
        return fail(ctx, RC_ERR_INVALID_ARG, "rc_render: bad arguments");
    if (!ctx->has_scene) return fail(ctx, RC_ERR_NO_SCENE, "rc_render: no scene uploaded");
    if (n_spp == 0) return RC_OK;
    CK(cudaSetDevice(ctx->device));
    RenderArgs A;
    A.scene = scene_for(ctx, RC_WIDE_PATHS);
    A.img = ctx->img;
    A.cam = cam_params(cam);
    A.nee_enabled = settings->nee_enabled;
    A.firefly_clamp = settings->nee_firefly_clamp;
    A.first_frame = first_frame;
    A.n_spp = n_spp;
    A.counters = ctx->counters;
    if (ctx->engine == RC_ENGINE_WAVEFRONT || ctx->engine == RC_ENGINE_WAVEFRONT_STATIC) {
        const int r = wavefront_render(ctx, A);
        if (r != RC_OK) return r;
    } else {
        const bool ex = ctx->math_mode == RC_MATH_EXACT;
        const cudaError_t e = timed_launch(ctx, RC_KERNEL_RENDER, [&] {
            return ex ? exact::launch_render(A, ctx->stream) : fast::launch_render(A, ctx->stream);
        });
        if (e != cudaSuccess) return launch_err(ctx, e, "render");
    }
    // Renderer.getTotalSamples(): frames 0 .. first_frame + n_spp - 1 done
    ctx->total_samples = first_frame + n_spp;
    return RC_OK;
}

int rc_reset(rc_ctx* ctx) {
    if (!ctx) return RC_ERR_INVALID_ARG;
    const size_t px = (size_t)ctx->width * ctx->height;
    CK(cudaSetDevice(ctx->device));
    CK(cudaMemsetAsync(ctx->img.accum, 0, px * sizeof(float4), ctx->stream));
    CK(cudaMemsetAsync(ctx->img.gbuf, 0, px * sizeof(ushort4), ctx->stream));
    CK(cudaMemsetAsync(ctx->img.galb, 0, px * sizeof(ushort4), ctx->stream));
    CK(cudaMemsetAsync(ctx->img.var, 0, px * sizeof(float), ctx->stream));
    ctx->total_samples = 0;
    return RC_OK;
}

int rc_total_samples(const rc_ctx* ctx) { return ctx ? ctx->total_samples : RC_ERR_INVALID_ARG; }

int rc_sppm_reset(rc_ctx* ctx, float initial_radius) {
    if (!ctx) return RC_ERR_INVALID_ARG;
    if (!(initial_radius > 0.0f)) return fail(ctx, RC_ERR_INVALID_ARG, "rc_sppm_reset: radius must be > 0");
    ctx->sppm_radius = initial_radius;
    ctx->sppm_iteration = 0;
    // a new SPPM sequence (a new export frame) traces its gather rays again:
    // the per-pixel gather hits are reused only within one sequence
    ctx->gcache_valid = false;
    return RC_OK;
}

int rc_sppm_update_radius(rc_ctx* ctx, float alpha) {
    if (!ctx) return RC_ERR_INVALID_ARG;
    ctx->sppm_radius = rc_sppm_next_radius(ctx->sppm_radius, ctx->sppm_iteration, alpha);
    ctx->sppm_iteration++;
    return RC_OK;
}

int rc_sppm_state(const rc_ctx* ctx, float* radius, int* iteration) {
    if (!ctx) return RC_ERR_INVALID_ARG;
    if (radius) *radius = ctx->sppm_radius;
    if (iteration) *iteration = ctx->sppm_iteration;
    return RC_OK;
}

static int check_sppm(rc_ctx* ctx, const rc_sppm_params* p) {
    if (!p || p->photon_count < 0 || p->hash_size < 1 || (p->hash_size & (p->hash_size - 1)) != 0)
        return fail(ctx, RC_ERR_INVALID_ARG, "sppm: photon_count must be >= 0 and hash_size a power of two");
    return RC_OK;
}

// Sizes the photon map for `photons` photons and a hash of `hash_size` cells.
static int photon_reserve(rc_ctx* ctx, const rc_sppm_params* p) {
    const int cap = p->photon_count > 0 ? p->photon_count : 1;
    if (cap > ctx->photon_cap || p->hash_size > ctx->hash_cap) CK(cudaStreamSynchronize(ctx->stream));
    if (cap > ctx->photon_cap) {
        CK(ensure(ctx->photons, (size_t)cap * 3 * sizeof(float4)));
        CK(ensure(ctx->next, (size_t)cap * sizeof(int)));
        CK(ensure(ctx->cell_of, (size_t)cap * sizeof(int)));
        CK(ensure(ctx->seg_photon, (size_t)cap * sizeof(int)));
        CK(ensure(ctx->seg_posw, (size_t)cap * sizeof(float4)));
        CK(ensure(ctx->seg_powyz, (size_t)cap * sizeof(float2)));
        CK(ensure(ctx->ph_queue, (size_t)cap * 4 * sizeof(float4)));
        ctx->photon_cap = cap;
    }
    if (p->hash_size > ctx->hash_cap) {
        CK(ensure(ctx->heads, (size_t)p->hash_size * sizeof(int)));
        CK(ensure(ctx->cell_count, (size_t)p->hash_size * sizeof(unsigned int)));
        CK(ensure(ctx->cell_start, ((size_t)p->hash_size + 1) * sizeof(unsigned int)));
        CK(ensure(ctx->block_sums, (((size_t)p->hash_size + 4095) / 4096) * sizeof(unsigned int)));
        ctx->hash_cap = p->hash_size;
    }
    CK(ensure(ctx->counter, sizeof(unsigned int)));
    CK(ensure(ctx->ph_queue_len, 2 * sizeof(unsigned int)));   // queue length, emission work counter
    return RC_OK;
}

int rc_sppm_trace(rc_ctx* ctx, const rc_sppm_params* p) {
    if (!ctx) return RC_ERR_INVALID_ARG;
    int r = check_sppm(ctx, p);
    if (r != RC_OK) return r;
    if (!ctx->has_scene) return fail(ctx, RC_ERR_NO_SCENE, "rc_sppm_trace: no scene uploaded");
    CK(cudaSetDevice(ctx->device));
    if ((r = photon_reserve(ctx, p)) != RC_OK) return r;
    // PhotonMap.clear(): heads = -1, counter = 0
    CK(cudaMemsetAsync(ctx->heads.ptr, 0xff, (size_t)p->hash_size * sizeof(int), ctx->stream));
    CK(cudaMemsetAsync(ctx->counter.ptr, 0, sizeof(unsigned int), ctx->stream));
    CK(cudaMemsetAsync(ctx->cell_count.ptr, 0, (size_t)p->hash_size * sizeof(unsigned int), ctx->stream));
    CK(cudaMemsetAsync(ctx->cell_start.ptr, 0, ((size_t)p->hash_size + 1) * sizeof(unsigned int), ctx->stream));
    ctx->last_hash = p->hash_size;
    ctx->last_photons = p->photon_count;
    if (p->photon_count == 0 || ctx->scene.light_count == 0) return RC_OK;
    PhotonArgs A;
    A.scene = scene_for(ctx, RC_WIDE_PHOTONS);
    A.photons = (float4*)ctx->photons.ptr;
    A.heads = (int*)ctx->heads.ptr;
    A.next = (int*)ctx->next.ptr;
    A.counter = (unsigned int*)ctx->counter.ptr;
    A.cell_of = (int*)ctx->cell_of.ptr;
    A.cell_count = (unsigned int*)ctx->cell_count.ptr;
    A.cell_start = (unsigned int*)ctx->cell_start.ptr;
    A.block_sums = (unsigned int*)ctx->block_sums.ptr;
    A.seg_photon = (int*)ctx->seg_photon.ptr;
    A.seg_posw = (float4*)ctx->seg_posw.ptr;
    A.seg_powyz = (float2*)ctx->seg_powyz.ptr;
    A.photon_count = p->photon_count;
    A.hash_size = p->hash_size;
    A.radius = ctx->sppm_radius;
    A.seed = ctx->sppm_iteration * 7919 + 6271;
    // the split walks other BVHs; past 60 levels the photon walk keeps the
    // reference's own order over its BVH (its 64-entry stack can overflow)
    A.split = (ctx->math_mode == RC_MATH_FAST && ctx->photon_split && !ctx->photon_full_first &&
               ctx->scene.depth <= 60) ? 1 : 0;
    A.spec = ctx->spec_view;
    A.diff = ctx->diff_view;
    A.spec_orig = (const int*)ctx->sp_orig.ptr;
    A.queue = (float4*)ctx->ph_queue.ptr;
    A.queue_len = (unsigned int*)ctx->ph_queue_len.ptr;
    A.work = (unsigned int*)ctx->ph_queue_len.ptr + 1;
    A.refill_lanes = ctx->refill_lanes;
    A.leaf_quarters = ctx->leaf_quarters;
    A.interior_steps = ctx->interior_steps;
    A.counters = ctx->counters;
    const bool ex = ctx->math_mode == RC_MATH_EXACT;
    cudaError_t e = timed_launch(
        ctx, RC_KERNEL_PHOTON_TRACE,
        [&] {
            return ex ? exact::launch_photon_trace(A, ctx->stream, ctx->photon_block)
                      : fast::launch_photon_trace(A, ctx->stream, ctx->photon_block);
        },
        2);   // emission and first segments, then the queued walks
    if (e != cudaSuccess) return launch_err(ctx, e, "photon trace");
    e = timed_launch(ctx, RC_KERNEL_PHOTON_LAYOUT, [&] {
        return ex ? exact::launch_photon_layout(A, ctx->stream) : fast::launch_photon_layout(A, ctx->stream);
    }, 5);
    return launch_err(ctx, e, "photon trace");
}

static uint64_t fnv1a(uint64_t h, const void* p, size_t n);

int rc_sppm_gather(rc_ctx* ctx, const rc_camera* cam, const rc_sppm_params* p, float weight) {
    if (!ctx) return RC_ERR_INVALID_ARG;
    int r = check_sppm(ctx, p);
    if (r != RC_OK) return r;
    if (!cam) return fail(ctx, RC_ERR_INVALID_ARG, "rc_sppm_gather: null camera");
    if (!ctx->has_scene) return fail(ctx, RC_ERR_NO_SCENE, "rc_sppm_gather: no scene uploaded");
    if (!ctx->heads.ptr || p->hash_size != ctx->last_hash)
        return fail(ctx, RC_ERR_INVALID_ARG, "rc_sppm_gather: no photon map traced with hash_size %d", p->hash_size);
    CK(cudaSetDevice(ctx->device));
    GatherArgs A;
    A.scene = scene_for(ctx, RC_WIDE_PHOTONS);
    A.img = ctx->img;
    A.cam = cam_params(cam);
    A.cell_start = (const unsigned int*)ctx->cell_start.ptr;
    A.seg_posw = (const float4*)ctx->seg_posw.ptr;
    A.seg_powyz = (const float2*)ctx->seg_powyz.ptr;
    A.hash_size = p->hash_size;
    A.radius = ctx->sppm_radius;
    A.weight = weight;
    A.counters = ctx->counters;
    // per-pixel gather hits: reused while the camera, scene, math mode and
    // traversal stay the same (a batch passes each frame's own slice)
    if (ctx->gcache_force) {
        A.hit_cache = ctx->gcache_force;
        A.cache_mode = ctx->gcache_force_mode;
    } else {
        uint64_t key = fnv1a(1469598103934665603ull, &A.cam, sizeof(A.cam));
        const int salt[4] = {(int)ctx->scene_gen, ctx->math_mode, ctx->wide_bvh, ctx->width * 65536 + ctx->height};
        key = fnv1a(key, salt, sizeof(salt));
        CK(ensure(ctx->gcache, (size_t)ctx->width * ctx->height * sizeof(float4)));
        A.hit_cache = (float4*)ctx->gcache.ptr;
        A.cache_mode = (ctx->gcache_valid && ctx->gcache_key == key) ? 2 : 1;
        ctx->gcache_key = key;
        ctx->gcache_valid = true;
    }
    const bool ex = ctx->math_mode == RC_MATH_EXACT;
    // the dense pixels' list (a batch allocated it before its capture)
    if (!ctx->gcache_force) CK(ensure(ctx->gheavy, ((size_t)ctx->width * ctx->height + 1) * sizeof(int)));
    A.heavy_len = (unsigned int*)ctx->gheavy.ptr;
    A.heavy = (int*)ctx->gheavy.ptr + 1;
    const cudaError_t e = timed_launch(ctx, RC_KERNEL_PHOTON_GATHER, [&] {
        return ex ? exact::launch_photon_gather(A, ctx->stream) : fast::launch_photon_gather(A, ctx->stream);
    }, 2);
    return launch_err(ctx, e, "photon gather");
}

int rc_denoise_atrous(rc_ctx* ctx, const rc_atrous_params* p, float* out_rgba) {
    if (!ctx) return RC_ERR_INVALID_ARG;
    if (!p) return fail(ctx, RC_ERR_INVALID_ARG, "rc_denoise_atrous: null params");
    CK(cudaSetDevice(ctx->device));
    const int N = ctx->total_samples;
    const int W = ctx->width, H = ctx->height;
    const bool over = p->max_spp > 0 && N > p->max_spp;
    const bool ex = ctx->math_mode == RC_MATH_EXACT;
    if (p->enabled && !over) {
        const int passes = p->iterations < 1 ? 1 : (p->iterations > 5 ? 5 : p->iterations);
        const float4* src = ctx->img.accum;
        float4* bufs[2] = {ctx->ping, ctx->pong};
        for (int i = 0; i < passes; ++i) {
            float4* dst = (i == passes - 1) ? ctx->out : bufs[i & 1];
            AtrousArgs A;
            A.color = src;
            A.gbuf = ctx->img.gbuf;
            A.galb = ctx->img.galb;
            A.var = ctx->img.var;
            A.out = dst;
            A.width = W;
            A.height = H;
            A.step = 1 << i;
            A.sigma_color = p->sigma_color;
            A.sigma_normal = p->sigma_normal;
            A.sigma_depth = p->sigma_depth;
            A.sample_count = N > 1 ? N : 1;
            A.exposure = p->exposure;
            A.normalize = (i == 0) ? 1 : 0;
            A.inv_n_unused = 0.0f;
            const cudaError_t e = timed_launch(ctx, RC_KERNEL_ATROUS, [&] {
                return ex ? exact::launch_atrous(A, ctx->stream) : fast::launch_atrous(A, ctx->stream);
            });
            if (e != cudaSuccess) return launch_err(ctx, e, "atrous");
            src = dst;
        }
    } else {
        NormalizeArgs A;
        A.accum = ctx->img.accum;
        A.out = ctx->out;
        A.count = W * H;
        A.total_samples = N;
        A.exposure = p->exposure;
        const cudaError_t e = timed_launch(ctx, RC_KERNEL_NORMALIZE, [&] {
            return ex ? exact::launch_normalize(A, ctx->stream) : fast::launch_normalize(A, ctx->stream);
        });
        if (e != cudaSuccess) return launch_err(ctx, e, "normalize");
    }
    ctx->result = ctx->out;
    if (out_rgba) return rc_read_output(ctx, out_rgba);
    return RC_OK;
}

int rc_kp_features(rc_ctx* ctx, void* feat, void* color) {
    if (!ctx) return RC_ERR_INVALID_ARG;
    if (!feat || !color) return fail(ctx, RC_ERR_INVALID_ARG, "rc_kp_features: null buffer");
    if (!rc::aligned_to(feat, 16) || !rc::aligned_to(color, 16))
        return fail(ctx, RC_ERR_INVALID_ARG, "rc_kp_features: buffers must be 16-byte aligned");
    CK(cudaSetDevice(ctx->device));
    const cudaError_t e = timed_launch(ctx, RC_KERNEL_KPCNN, [&] {
        return kp::launch_features(ctx->img.accum, ctx->img.gbuf, ctx->img.galb, static_cast<__nv_bfloat16*>(feat),
                                   static_cast<float4*>(color), ctx->width * ctx->height, ctx->stream);
    });
    if (e != cudaSuccess) return launch_err(ctx, e, "kpcnn features");
    return RC_OK;
}

int rc_denoise_learned(rc_ctx* ctx, const rc_kpcnn* weights, float* out_rgba) {
    if (!ctx) return RC_ERR_INVALID_ARG;
    if (!weights || !weights->params || weights->param_count != RC_KPCNN_PARAMS)
        return fail(ctx, RC_ERR_INVALID_ARG, "rc_denoise_learned: need %d parameters", RC_KPCNN_PARAMS);
    CK(cudaSetDevice(ctx->device));
    const size_t px = (size_t)ctx->width * ctx->height;
    if (ctx->kp_params.bytes < RC_KPCNN_PARAMS * sizeof(float) || ctx->kp_logits.bytes < px * 128)
        CK(cudaStreamSynchronize(ctx->stream));
    CK(ensure(ctx->kp_feat, px * 32));
    CK(ensure(ctx->kp_act0, px * 64));
    CK(ensure(ctx->kp_act1, px * 64));
    CK(ensure(ctx->kp_logits, px * 128));
    CK(ensure(ctx->kp_color, px * 16));
    CK(ensure(ctx->kp_params, RC_KPCNN_PARAMS * sizeof(float)));
    CK(ensure(ctx->kp_packed, kp::packed_bytes()));
    // upload (and repack) only when the parameters changed since the last call
    const bool same = ctx->kp_host.size() == (size_t)RC_KPCNN_PARAMS &&
                      memcmp(ctx->kp_host.data(), weights->params, RC_KPCNN_PARAMS * sizeof(float)) == 0;
    if (!same) {
        ctx->kp_packed_at = nullptr;
        ctx->kp_host.assign(weights->params, weights->params + RC_KPCNN_PARAMS);
        const cudaError_t ce = copy_h2d(ctx, ctx->kp_params.ptr, ctx->kp_host.data(), RC_KPCNN_PARAMS * sizeof(float));
        if (ce != cudaSuccess) {
            ctx->kp_host.clear();
            return launch_err(ctx, ce, "kpcnn parameter upload");
        }
    }
    // the packed bf16 weights are redone only when the parameters changed
    const bool repack = ctx->kp_packed_at != ctx->kp_packed.ptr;
    const cudaError_t e = timed_launch(
        ctx, RC_KERNEL_KPCNN,
        [&] {
            return kp::run_inference((const float*)ctx->kp_params.ptr, ctx->kp_packed.ptr, repack, ctx->img.accum,
                                     ctx->img.gbuf, ctx->img.galb, ctx->kp_feat.ptr, ctx->kp_act0.ptr,
                                     ctx->kp_act1.ptr, (float*)ctx->kp_logits.ptr, (float4*)ctx->kp_color.ptr,
                                     ctx->out, ctx->width, ctx->height, &ctx->counters->error_word, ctx->stream);
        },
        repack ? 6 : 5);
    if (e != cudaSuccess) {
        ctx->kp_packed_at = nullptr;
        return launch_err(ctx, e, "kpcnn");
    }
    ctx->kp_packed_at = ctx->kp_packed.ptr;
    ctx->result = ctx->out;
    if (out_rgba) return rc_read_output(ctx, out_rgba);
    return RC_OK;
}

int rc_render_frame(rc_ctx* ctx, const rc_camera* cam, const rc_settings* settings, int spp,
                    const rc_sppm_params* sppm, float sppm_initial_radius, int sppm_iterations,
                    const rc_atrous_params* atrous, float* out_rgba) {
    if (!ctx) return RC_ERR_INVALID_ARG;
    if (!cam || !settings || !atrous || spp < 1 || sppm_iterations < 0 || sppm_iterations > spp ||
        (sppm_iterations > 0 && !sppm))
        return fail(ctx, RC_ERR_INVALID_ARG, "rc_render_frame: bad arguments");
    if (!ctx->has_scene) return fail(ctx, RC_ERR_NO_SCENE, "rc_render_frame: no scene uploaded");
    int r = rc_reset(ctx);
    if (r != RC_OK) return r;
    const bool use_sppm = sppm_iterations > 0 && ctx->scene.light_count > 0;
    if (use_sppm) {
        if ((r = rc_sppm_reset(ctx, sppm_initial_radius)) != RC_OK) return r;
        for (int k = 0; k < sppm_iterations; ++k) {
            const int s0 = (int)((long)k * spp / sppm_iterations);
            const int s1 = (int)((long)(k + 1) * spp / sppm_iterations);
            if ((r = rc_sppm_trace(ctx, sppm)) != RC_OK) return r;
            if ((r = rc_render(ctx, cam, settings, s0, s1 - s0)) != RC_OK) return r;
            if ((r = rc_sppm_gather(ctx, cam, sppm, (float)(s1 - s0))) != RC_OK) return r;
            if ((r = rc_sppm_update_radius(ctx, sppm->alpha)) != RC_OK) return r;
        }
    } else {
        if ((r = rc_render(ctx, cam, settings, 0, spp)) != RC_OK) return r;
    }
    return rc_denoise_atrous(ctx, atrous, out_rgba);
}

int rc_frame_part_range(int spp, int sppm_iterations, int part, int parts, int* k0, int* k1, int* s0,
                        int* s1) {
    if (spp < 1 || sppm_iterations < 0 || sppm_iterations > spp || parts < 1 || part < 0 || part >= parts ||
        !k0 || !k1 || !s0 || !s1)
        return RC_ERR_INVALID_ARG;
    if (sppm_iterations > 0) {
        // whole SPPM iterations, each with rc_render_frame's sample block
        *k0 = (int)((long)part * sppm_iterations / parts);
        *k1 = (int)((long)(part + 1) * sppm_iterations / parts);
        *s0 = (int)((long)*k0 * spp / sppm_iterations);
        *s1 = (int)((long)*k1 * spp / sppm_iterations);
    } else {
        *k0 = *k1 = 0;
        *s0 = (int)((long)part * spp / parts);
        *s1 = (int)((long)(part + 1) * spp / parts);
    }
    return RC_OK;
}

int rc_render_frame_part(rc_ctx* ctx, const rc_camera* cam, const rc_settings* settings, int spp,
                         const rc_sppm_params* sppm, float sppm_initial_radius, int sppm_iterations, int part,
                         int parts) {
    if (!ctx) return RC_ERR_INVALID_ARG;
    int k0, k1, s0, s1;
    if (!cam || !settings || (sppm_iterations > 0 && !sppm) ||
        rc_frame_part_range(spp, sppm_iterations, part, parts, &k0, &k1, &s0, &s1) != RC_OK)
        return fail(ctx, RC_ERR_INVALID_ARG, "rc_render_frame_part: bad arguments");
    if (!ctx->has_scene) return fail(ctx, RC_ERR_NO_SCENE, "rc_render_frame_part: no scene uploaded");
    int r = rc_reset(ctx);
    if (r != RC_OK) return r;
    if (sppm_iterations > 0 && ctx->scene.light_count > 0) {
        // the radius and iteration count iteration k0 starts from, as
        // updateRadius leaves them after k0 iterations
        if ((r = rc_sppm_reset(ctx, sppm_initial_radius)) != RC_OK) return r;
        for (int k = 0; k < k0; ++k)
            if ((r = rc_sppm_update_radius(ctx, sppm->alpha)) != RC_OK) return r;
        for (int k = k0; k < k1; ++k) {
            const int b0 = (int)((long)k * spp / sppm_iterations);
            const int b1 = (int)((long)(k + 1) * spp / sppm_iterations);
            if ((r = rc_sppm_trace(ctx, sppm)) != RC_OK) return r;
            if ((r = rc_render(ctx, cam, settings, b0, b1 - b0)) != RC_OK) return r;
            if ((r = rc_sppm_gather(ctx, cam, sppm, (float)(b1 - b0))) != RC_OK) return r;
            if ((r = rc_sppm_update_radius(ctx, sppm->alpha)) != RC_OK) return r;
        }
    } else if (s1 > s0) {
        if ((r = rc_render(ctx, cam, settings, s0, s1 - s0)) != RC_OK) return r;
    }
    // this part's samples only; rc_set_total_samples after the merge
    ctx->total_samples = s1 - s0;
    return RC_OK;
}

int rc_set_total_samples(rc_ctx* ctx, int total_samples) {
    if (!ctx) return RC_ERR_INVALID_ARG;
    if (total_samples < 0) return fail(ctx, RC_ERR_INVALID_ARG, "rc_set_total_samples: negative count");
    ctx->total_samples = total_samples;
    return RC_OK;
}

int rc_get_images(rc_ctx* ctx, void** accum, void** gbuf, void** galb, void** var, void** stream) {
    if (!ctx) return RC_ERR_INVALID_ARG;
    if (accum) *accum = ctx->img.accum;
    if (gbuf) *gbuf = ctx->img.gbuf;
    if (galb) *galb = ctx->img.galb;
    if (var) *var = ctx->img.var;
    if (stream) *stream = ctx->stream;
    return RC_OK;
}

int rc_read_buffers(rc_ctx* ctx, float* accum, uint16_t* gbuf, uint16_t* galb, float* var) {
    if (!ctx) return RC_ERR_INVALID_ARG;
    const size_t px = (size_t)ctx->width * ctx->height;
    CK(cudaSetDevice(ctx->device));
    if (accum) CK(copy_d2h(ctx, accum, ctx->img.accum, px * sizeof(float4)));
    if (gbuf) CK(copy_d2h(ctx, gbuf, ctx->img.gbuf, px * sizeof(ushort4)));
    if (galb) CK(copy_d2h(ctx, galb, ctx->img.galb, px * sizeof(ushort4)));
    if (var) CK(copy_d2h(ctx, var, ctx->img.var, px * sizeof(float)));
    return rc_synchronize(ctx);
}

int rc_read_output(rc_ctx* ctx, float* out_rgba) {
    if (!ctx || !out_rgba) return RC_ERR_INVALID_ARG;
    const size_t px = (size_t)ctx->width * ctx->height;
    CK(cudaSetDevice(ctx->device));
    CK(copy_d2h(ctx, out_rgba, ctx->result, px * sizeof(float4)));
    return rc_synchronize(ctx);
}

int rc_post_vhs(rc_ctx* ctx, const rc_vhs_params* p) {
    if (!ctx || !p) return RC_ERR_INVALID_ARG;
    CK(cudaSetDevice(ctx->device));
    // PingPongBuffer: each pass reads the previous result and writes the other image
    const float4* src = ctx->result;
    for (int k = 1; k <= 16; ++k) {
        if (!(p->enabled & RC_VHS_PASS(k)) || !vhs::has_pass(k)) continue;
        float4* dst = (src == ctx->ping) ? ctx->pong : ctx->ping;
        const cudaError_t e = timed_launch(ctx, RC_KERNEL_VHS, [&] {
            return vhs::launch_pass(k, src, dst, ctx->width, ctx->height, *p, ctx->stream);
        });
        if (e != cudaSuccess) return launch_err(ctx, e, "vhs pass");
        src = dst;
    }
    ctx->result = const_cast<float4*>(src);
    return RC_OK;
}

static int display_from(rc_ctx* ctx, const float4* color, int total_samples, float exposure, uint8_t* out_rgba8) {
    const size_t px = (size_t)ctx->width * ctx->height;
    CK(cudaSetDevice(ctx->device));
    CK(ensure(ctx->disp, px * sizeof(uchar4)));
    DisplayArgs A;
    A.color = color;
    A.out = (uchar4*)ctx->disp.ptr;
    A.width = ctx->width;
    A.height = ctx->height;
    A.total_samples = total_samples;
    A.exposure = exposure;
    const bool ex = ctx->math_mode == RC_MATH_EXACT;
    const cudaError_t e = timed_launch(ctx, RC_KERNEL_DISPLAY, [&] {
        return ex ? exact::launch_display(A, ctx->stream) : fast::launch_display(A, ctx->stream);
    });
    if (e != cudaSuccess) return launch_err(ctx, e, "display");
    if (!out_rgba8) return RC_OK;
    CK(copy_d2h(ctx, out_rgba8, ctx->disp.ptr, px * sizeof(uchar4)));
    return rc_synchronize(ctx);
}

int rc_display(rc_ctx* ctx, int total_samples, float exposure, uint8_t* out_rgba8) {
    if (!ctx) return RC_ERR_INVALID_ARG;
    return display_from(ctx, ctx->result, total_samples, exposure, out_rgba8);
}

int rc_display_frame(rc_ctx* ctx, int frame, int total_samples, float exposure, uint8_t* out_rgba8) {
    if (!ctx) return RC_ERR_INVALID_ARG;
    if (frame < 0 || frame >= ctx->batch_frames)
        return fail(ctx, RC_ERR_INVALID_ARG, "rc_display_frame: frame %d of a batch of %d", frame, ctx->batch_frames);
    const size_t px = (size_t)ctx->width * ctx->height;
    return display_from(ctx, (const float4*)ctx->frames.ptr + (size_t)frame * px, total_samples, exposure, out_rgba8);
}

int rc_read_photon_map(rc_ctx* ctx, rc_photon* photons, int photon_capacity, int32_t* heads, int hash_size,
                       int32_t* next, uint32_t* counter) {
    if (!ctx) return RC_ERR_INVALID_ARG;
    if (!ctx->heads.ptr) return fail(ctx, RC_ERR_INVALID_ARG, "rc_read_photon_map: no photon map");
    if (heads && hash_size != ctx->last_hash)
        return fail(ctx, RC_ERR_INVALID_ARG, "rc_read_photon_map: hash_size %d != traced %d", hash_size,
                    ctx->last_hash);
    const int n = photon_capacity < ctx->photon_cap ? photon_capacity : ctx->photon_cap;
    CK(cudaSetDevice(ctx->device));
    if (photons && n > 0)
        CK(cudaMemcpyAsync(photons, ctx->photons.ptr, (size_t)n * sizeof(rc_photon), cudaMemcpyDeviceToHost,
                           ctx->stream));
    if (heads)
        CK(cudaMemcpyAsync(heads, ctx->heads.ptr, (size_t)hash_size * sizeof(int), cudaMemcpyDeviceToHost,
                           ctx->stream));
    if (next && n > 0)
        CK(cudaMemcpyAsync(next, ctx->next.ptr, (size_t)n * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    if (counter) CK(cudaMemcpyAsync(counter, ctx->counter.ptr, sizeof(unsigned int), cudaMemcpyDeviceToHost, ctx->stream));
    return rc_synchronize(ctx);
}

int rc_get_counters(rc_ctx* ctx, rc_counters* out) {
    if (!ctx || !out) return RC_ERR_INVALID_ARG;
    DevCounters d;
    CK(cudaSetDevice(ctx->device));
    CK(cudaMemcpyAsync(&d, ctx->counters, sizeof(d), cudaMemcpyDeviceToHost, ctx->stream));
    unsigned int stored = 0;
    if (ctx->counter.ptr)
        CK(cudaMemcpyAsync(&stored, ctx->counter.ptr, sizeof(stored), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    out->camera_paths = d.camera_paths;
    out->closest_rays = d.closest_rays;
    out->shadow_rays = d.shadow_rays;
    out->photon_rays = d.photon_rays;
    out->gather_rays = d.gather_rays;
    out->photons_stored = stored < (unsigned)ctx->last_photons ? stored : (unsigned)ctx->last_photons;
    out->node_tests = d.node_tests;
    out->tri_tests = d.tri_tests;
    out->surface_hits = d.surface_hits;
    out->light_samples = d.light_samples;
    out->photon_node_tests = d.photon_node_tests;
    out->photon_tri_tests = d.photon_tri_tests;
    out->kernel_launches = ctx->launches;
    out->h2d_bytes = ctx->h2d;
    out->d2h_bytes = ctx->d2h;
    out->error_word = d.error_word;
    out->bvh_depth = ctx->has_scene ? (uint32_t)ctx->scene.depth : 0u;
    return RC_OK;
}

int rc_reset_counters(rc_ctx* ctx) {
    if (!ctx) return RC_ERR_INVALID_ARG;
    CK(cudaSetDevice(ctx->device));
    CK(cudaMemsetAsync(ctx->counters, 0, sizeof(DevCounters), ctx->stream));
    ctx->launches = ctx->h2d = ctx->d2h = 0;
    return RC_OK;
}

// ---------------------------------------------------------------------------
// Batched export frames (keyframed animations)
// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// Batched frames: every frame's SPPM iteration k uses the same photon map
// (the map depends on the scene, the iteration seed k*7919+6271 and the
// radius r_k only), so iteration k traces it once and then renders slice k
// of EVERY frame -- packed into shared wavefront chunks as segments -- and
// gathers it into each frame.  Per frame, the samples and gathers are added
// in the order rc_render_frame adds them.
// ---------------------------------------------------------------------------
struct BatchChunk {
    int iteration;
    int seg_begin, seg_count;
    long paths;
};

struct BatchPlan {
    std::vector<FrameSeg> segs;
    std::vector<BatchChunk> chunks;
    int iterations = 0;
    long capacity = 0;
};

static int slices_of(const rc_frame_desc& d) { return d.sppm_iterations > 0 ? d.sppm_iterations : 1; }

static void slice_range(const rc_frame_desc& d, int k, int& s0, int& s1) {
    const int it = slices_of(d);
    s0 = (int)((long)k * d.spp / it);
    s1 = (int)((long)(k + 1) * d.spp / it);
}

static Images frame_images(rc_ctx* ctx, int f) {
    const size_t px = (size_t)ctx->width * ctx->height;
    char* base = (char*)ctx->batch_img.ptr;
    Images im;
    im.width = ctx->width;
    im.height = ctx->height;
    im.accum = (float4*)base + (size_t)f * px;
    char* after_accum = base + ctx->batch_img.bytes / 36 * 16;
    im.gbuf = (ushort4*)after_accum + (size_t)f * px;
    char* after_gbuf = after_accum + ctx->batch_img.bytes / 36 * 8;
    im.galb = (ushort4*)after_gbuf + (size_t)f * px;
    char* after_galb = after_gbuf + ctx->batch_img.bytes / 36 * 8;
    im.var = (float*)after_galb + (size_t)f * px;
    return im;
}

// Plans the chunks: per iteration, slices of all frames in frame order,
// split at sample boundaries so no chunk exceeds the wavefront capacity.
static BatchPlan plan_batch(rc_ctx* ctx, const rc_frame_desc* frames, int n) {
    BatchPlan P;
    const int tiles_x = (ctx->width + 7) / 8, tiles_y = (ctx->height + 3) / 4;
    const long npix = (long)tiles_x * tiles_y * 32;
    const long cap = ctx->chunk_paths > 0 ? ctx->chunk_paths : kDefaultChunkPaths;
    for (int f = 0; f < n; ++f) P.iterations = std::max(P.iterations, slices_of(frames[f]));
    for (int k = 0; k < P.iterations; ++k) {
        BatchChunk cur{k, (int)P.segs.size(), 0, 0};
        for (int f = 0; f < n; ++f) {
            const rc_frame_desc& d = frames[f];
            if (k >= slices_of(d)) continue;
            int s0, s1;
            slice_range(d, k, s0, s1);
            const CamParams cam = cam_params(&d.camera);
            const int C = lca_active(cam) ? 3 : 1;
            const long per_sample = npix * C;
            while (s0 < s1) {
                long room = (cap - cur.paths) / per_sample;
                if (room < 1 && cur.seg_count > 0) {   // close the chunk
                    P.chunks.push_back(cur);
                    P.capacity = std::max(P.capacity, cur.paths);
                    cur = BatchChunk{k, (int)P.segs.size(), 0, 0};
                    room = cap / per_sample;
                }
                const int take = (int)std::max<long>(1, std::min<long>(room, s1 - s0));
                FrameSeg sg;
                sg.cam = cam;
                sg.img = frame_images(ctx, f);
                sg.first_frame = s0;
                sg.n_samples = take;
                sg.channels = C;
                sg.path_base = (int)cur.paths;
                P.segs.push_back(sg);
                cur.seg_count++;
                cur.paths += per_sample * take;
                s0 += take;
            }
        }
        if (cur.seg_count > 0) {
            P.chunks.push_back(cur);
            P.capacity = std::max(P.capacity, cur.paths);
        }
    }
    return P;
}

static int batched_sequence(rc_ctx* ctx, const rc_frame_desc* frames, int n, const rc_settings* settings,
                            const rc_sppm_params* sppm, float r0, const rc_atrous_params* atrous,
                            const BatchPlan& P) {
    const size_t px = (size_t)ctx->width * ctx->height;
    const Images saved_img = ctx->img;
    float4* const saved_out = ctx->out;
    const bool sppm_on = sppm && ctx->scene.light_count > 0;
    int r = RC_OK;
    if (sppm_on && (r = rc_sppm_reset(ctx, r0)) != RC_OK) return r;
    const FrameSeg* segs_dev = (const FrameSeg*)ctx->batch_segs.ptr;
    size_t ci = 0;
    for (int k = 0; k < P.iterations && r == RC_OK; ++k) {
        bool gather_k = false;
        for (int f = 0; f < n; ++f) gather_k = gather_k || (frames[f].sppm_iterations > k);
        gather_k = gather_k && sppm_on;
        if (gather_k && (r = rc_sppm_trace(ctx, sppm)) != RC_OK) break;
        for (; ci < P.chunks.size() && P.chunks[ci].iteration == k; ++ci) {
            const BatchChunk& c = P.chunks[ci];
            WaveArgs A = wave_args(ctx, scene_for(ctx, RC_WIDE_PATHS), settings->nee_enabled,
                                   settings->nee_firefly_clamp);
            A.segs = segs_dev + c.seg_begin;
            A.nsegs = c.seg_count;
            A.one = P.segs[c.seg_begin];
            A.paths = (int)c.paths;
            if ((r = wavefront_chunk(ctx, A)) != RC_OK) break;
        }
        if (r != RC_OK) break;
        if (gather_k) {
            for (int f = 0; f < n && r == RC_OK; ++f) {
                if (frames[f].sppm_iterations <= k) continue;
                int s0, s1;
                slice_range(frames[f], k, s0, s1);
                ctx->img = frame_images(ctx, f);
                ctx->gcache_force = (float4*)ctx->batch_gcache.ptr + (size_t)f * px;
                ctx->gcache_force_mode = k == 0 ? 1 : 2;
                r = rc_sppm_gather(ctx, &frames[f].camera, sppm, (float)(s1 - s0));
                ctx->gcache_force = nullptr;
            }
            if (r == RC_OK) r = rc_sppm_update_radius(ctx, sppm->alpha);
        }
    }
    for (int f = 0; f < n && r == RC_OK; ++f) {
        ctx->img = frame_images(ctx, f);
        ctx->total_samples = frames[f].spp;
        ctx->out = (float4*)ctx->frames.ptr + (size_t)f * px;
        r = rc_denoise_atrous(ctx, atrous, nullptr);
    }
    ctx->img = saved_img;
    ctx->out = saved_out;
    ctx->result = (float4*)ctx->frames.ptr + (size_t)(n - 1) * px;
    return r;
}

static uint64_t fnv1a(uint64_t h, const void* p, size_t n) {
    const unsigned char* c = (const unsigned char*)p;
    for (size_t i = 0; i < n; ++i) {
        h ^= c[i];
        h *= 1099511628211ull;
    }
    return h;
}

int rc_render_frames(rc_ctx* ctx, const rc_frame_desc* frames, int n_frames, const rc_settings* settings,
                     const rc_sppm_params* sppm, float sppm_initial_radius, const rc_atrous_params* atrous,
                     float* out_frames, int use_graph) {
    if (!ctx) return RC_ERR_INVALID_ARG;
    if (!frames || n_frames < 1 || !settings || !atrous)
        return fail(ctx, RC_ERR_INVALID_ARG, "rc_render_frames: bad arguments");
    if (!ctx->has_scene) return fail(ctx, RC_ERR_NO_SCENE, "rc_render_frames: no scene uploaded");
    for (int f = 0; f < n_frames; ++f) {
        const rc_frame_desc& d = frames[f];
        if (d.spp < 1 || d.sppm_iterations < 0 || d.sppm_iterations > d.spp || (d.sppm_iterations > 0 && !sppm))
            return fail(ctx, RC_ERR_INVALID_ARG, "rc_render_frames: frame %d: bad spp/iterations", f);
    }
    CK(cudaSetDevice(ctx->device));
    const size_t px = (size_t)ctx->width * ctx->height;
    // ---- reserve every buffer the sequence touches (no allocation may
    //      happen while the stream is being captured) ----
    const bool batched = ctx->engine != RC_ENGINE_MEGAKERNEL;
    long cap = 0;
    bool any_sppm = false;
    for (int f = 0; f < n_frames; ++f) {
        const rc_frame_desc& d = frames[f];
        const int it = d.sppm_iterations;
        const int block = it > 0 ? (d.spp + it - 1) / it : d.spp;
        cap = std::max(cap, wavefront_capacity(ctx, block, lca_active(cam_params(&d.camera)), nullptr));
        any_sppm = any_sppm || (it > 0);
    }
    CK(cudaStreamSynchronize(ctx->stream));
    BatchPlan plan;
    if (batched) {
        // per-frame images: accum | gbuf | galb | var regions of n_frames x px
        CK(ensure(ctx->batch_img, (size_t)n_frames * px * 36));
        if (any_sppm) CK(ensure(ctx->batch_gcache, (size_t)n_frames * px * sizeof(float4)));
        plan = plan_batch(ctx, frames, n_frames);
        cap = std::max(cap, plan.capacity);
        CK(ensure(ctx->batch_segs, plan.segs.size() * sizeof(FrameSeg)));
        CK(cudaMemcpy(ctx->batch_segs.ptr, plan.segs.data(), plan.segs.size() * sizeof(FrameSeg),
                      cudaMemcpyHostToDevice));
        ctx->h2d += plan.segs.size() * sizeof(FrameSeg);
    }
    if (ctx->engine != RC_ENGINE_MEGAKERNEL) {
        const int r = wavefront_reserve(ctx, cap);
        if (r != RC_OK) return r;
    }
    if (any_sppm) {
        int r = check_sppm(ctx, sppm);
        if (r == RC_OK) r = photon_reserve(ctx, sppm);
        if (r != RC_OK) return r;
    }
    CK(ensure(ctx->frames, (size_t)n_frames * px * sizeof(float4)));
    ctx->batch_frames = n_frames;   // rc_display_frame's range (valid once this call succeeds)
    CK(cudaStreamSynchronize(ctx->stream));
    // ---- the sequence ----
    if (any_sppm) CK(ensure(ctx->gcache, px * sizeof(float4)));
    if (any_sppm) CK(ensure(ctx->gheavy, (px + 1) * sizeof(int)));
    auto sequence = [&]() -> int {
        ctx->gcache_valid = false;   // each replay traces its frames' gather hits afresh
        if (batched)
            return batched_sequence(ctx, frames, n_frames, settings, sppm, sppm_initial_radius, atrous, plan);
        for (int f = 0; f < n_frames; ++f) {
            const rc_frame_desc& d = frames[f];
            int r = rc_render_frame(ctx, &d.camera, settings, d.spp, sppm, sppm_initial_radius, d.sppm_iterations,
                                    atrous, nullptr);
            if (r != RC_OK) return r;
            cudaError_t e = cudaMemcpyAsync((float4*)ctx->frames.ptr + (size_t)f * px, ctx->result,
                                            px * sizeof(float4), cudaMemcpyDeviceToDevice, ctx->stream);
            if (e != cudaSuccess) return fail(ctx, RC_ERR_CUDA, "frame copy: %s", cudaGetErrorString(e));
        }
        return RC_OK;
    };
    if (!use_graph) {
        const int r = sequence();
        if (r != RC_OK) return r;
    } else {
        uint64_t key = 1469598103934665603ull;
        key = fnv1a(key, frames, sizeof(rc_frame_desc) * (size_t)n_frames);
        key = fnv1a(key, settings, sizeof(*settings));
        if (sppm) key = fnv1a(key, sppm, sizeof(*sppm));
        key = fnv1a(key, &sppm_initial_radius, sizeof(float));
        key = fnv1a(key, atrous, sizeof(*atrous));
        key = fnv1a(key, &ctx->engine, sizeof(int));
        key = fnv1a(key, &ctx->math_mode, sizeof(int));
        key = fnv1a(key, &ctx->stream, sizeof(void*));
        key = fnv1a(key, &ctx->frames.ptr, sizeof(void*));
        key = fnv1a(key, &ctx->batch_img.ptr, sizeof(void*));
        key = fnv1a(key, &ctx->batch_segs.ptr, sizeof(void*));
        key = fnv1a(key, &ctx->wf_o.ptr, sizeof(void*));
        for (const DevBuf* b : {&ctx->photons, &ctx->heads, &ctx->next, &ctx->cell_of, &ctx->cell_count,
                                &ctx->cell_start, &ctx->block_sums, &ctx->seg_photon, &ctx->seg_posw,
                                &ctx->seg_powyz, &ctx->ph_queue, &ctx->ph_queue_len, &ctx->gcache,
                                &ctx->batch_gcache, &ctx->gheavy})
            key = fnv1a(key, &b->ptr, sizeof(void*));
        const int shape[12] = {ctx->chunk_paths,  ctx->wide_bvh,       ctx->trace_block,
                               ctx->shade_block,  ctx->photon_block,   ctx->width,
                               ctx->photon_full_first, ctx->refill_lanes, ctx->leaf_quarters,
                               ctx->refill_min_paths, ctx->material_queues, ctx->interior_steps};
        key = fnv1a(key, shape, sizeof(shape));
        if (!ctx->graph_exec || ctx->graph_key != key) {
            if (ctx->graph_exec) {
                cudaGraphExecDestroy(ctx->graph_exec);
                ctx->graph_exec = nullptr;
            }
            const bool timing = ctx->timing;
            ctx->timing = false;  // event pairs are not recorded into the graph
            const unsigned long long launches0 = ctx->launches;
            CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
            const int r = sequence();
            cudaGraph_t graph = nullptr;
            const cudaError_t ec = cudaStreamEndCapture(ctx->stream, &graph);
            ctx->timing = timing;
            if (r != RC_OK) {
                if (graph) cudaGraphDestroy(graph);
                return r;
            }
            if (ec != cudaSuccess) return fail(ctx, RC_ERR_CUDA, "graph capture: %s", cudaGetErrorString(ec));
            const cudaError_t ei = cudaGraphInstantiate(&ctx->graph_exec, graph, 0);
            cudaGraphDestroy(graph);
            if (ei != cudaSuccess) {
                ctx->graph_exec = nullptr;
                return fail(ctx, RC_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(ei));
            }
            ctx->graph_key = key;
            ctx->graph_launches = ctx->launches - launches0;
            ctx->launches = launches0;
            ctx->graph_total_samples = ctx->total_samples;
            ctx->graph_radius = ctx->sppm_radius;
            ctx->graph_iteration = ctx->sppm_iteration;
        }
        CK(cudaGraphLaunch(ctx->graph_exec, ctx->stream));
        ctx->launches += ctx->graph_launches;
        ctx->total_samples = ctx->graph_total_samples;
        ctx->sppm_radius = ctx->graph_radius;
        ctx->sppm_iteration = ctx->graph_iteration;
    }
    if (out_frames) {
        CK(copy_d2h(ctx, out_frames, ctx->frames.ptr, (size_t)n_frames * px * sizeof(float4)));
        return rc_synchronize(ctx);
    }
    return RC_OK;
}

}  // extern "C"
