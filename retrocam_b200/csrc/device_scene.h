// device_scene.h -- device-side layout of a scene and of the per-context
// images, shared by the C-ABI layer (api.cu) and the kernels.
//
// HBM layout (all arrays 16-byte aligned, read with 128-bit loads):
//   node records   64 B per BVH node: the AABBs of BOTH children plus their
//                  (ref, count) pairs, so an interior visit is one 64-byte
//                  line and the child tests need no further loads.
//                    a = (L.min.x, L.min.y, L.max.x, L.max.y)
//                    b = (R.min.x, R.min.y, R.max.x, R.max.y)
//                    c = (L.min.z, L.max.z, R.min.z, R.max.z)
//                    d = (L.ref, L.count, R.ref, R.count)
//                  ref is a node index when count == 0, else prim_start.
//                  Records of leaf nodes are never read.  A second copy with
//                  packed child references (DeviceScene::nodes_packed) serves
//                  the refill trace.
//   tri_isect      48 B per triangle: v0, e1 = v1 - v0, e2 = v2 - v0 (the
//                  differences the reference computes per test, computed once
//                  on the host with the same float subtraction); the w
//                  components hold n = e1 x e2 for the fast build's test.
//   tri_shade      48 B per triangle: n0 (+ material index bits in .w), n1, n2;
//                  read only for the accepted closest hit.
//   materials      64 B per material (the std430 record).
//   lights         80 B per light (the std430 record) + a separate float CDF
//                  array so the linear CDF scan touches 4 B per light.
// Triangles and nodes keep the reference's BVH order, so indices match the
// reference buffers one to one.
#ifndef RC_DEVICE_SCENE_H
#define RC_DEVICE_SCENE_H

#include <cuda_runtime.h>
#include <stdint.h>

namespace rc {

struct NodeRec {
    float4 a;   // left child:  min x, min y, max x, max y
    float4 b;   // right child: min x, min y, max x, max y
    float4 c;   // left min z, left max z, right min z, right max z
    int4 d;     // left (ref, count), right (ref, count)
};

// 4-wide node of the fast build's traversal (128 B, two cache lines): the
// boxes of up to four children as SoA lanes, and per child (ref, count) with
// ref a Node4 index when count == 0 and a primitive start otherwise.  Unused
// slots have count -1 (and a zero box) and are never tested.
// Built on the host by collapsing the reference's binary BVH; the triangles
// and their order are unchanged.
struct Node4 {
    float4 lox, hix, loy, hiy, loz, hiz;
    int4 ref, cnt;
};

struct DeviceScene {
    const NodeRec* nodes = nullptr;
    // The refill trace's copy of the interior records (both builds): as
    // `nodes` with d = (left, right, 0, 0) packed child references -- a
    // child node's index, or for a leaf INT_MIN | prim_start << 5 | count --
    // built when every leaf holds 1..31 triangles and the scene fewer than
    // 2^26; null otherwise.  root_packed: the root as such a reference.
    const NodeRec* nodes_packed = nullptr;
    int root_packed = 0;
    const Node4* nodes4 = nullptr;       // root at index 0 unless the root is a leaf
    const float4* tri_isect = nullptr;   // 3 per triangle
    const float4* tri_shade = nullptr;   // 3 per triangle
    const float4* materials = nullptr;   // 4 per material
    const float4* lights = nullptr;      // 5 per light
    const float* light_cdf = nullptr;
    int node_count = 0;
    int tri_count = 0;
    int material_count = 0;
    int light_count = 0;
    float total_light_power = 0.0f;
    // root node as the reference stores it
    float root_min[3] = {0, 0, 0};
    float root_max[3] = {0, 0, 0};
    int root_ref = 0;     // prim_start when the root is a leaf, else 0
    int root_count = 0;   // > 0 when the root is a leaf
    int depth = 0;        // max leaf depth (root = 0)
    int max_leaf = 0;     // most triangles in one leaf
};

// Per-context images (core/Renderer.java:152-193).
struct Images {
    float4* accum = nullptr;      // RGBA32F running sum, alpha = samples
    ushort4* gbuf = nullptr;      // RGBA16F (facing normal, hit t)
    ushort4* galb = nullptr;      // RGBA16F first-hit albedo
    float* var = nullptr;         // R32F sum of luma^2
    int width = 0, height = 0;
};

// Camera uniforms of pathtrace.comp:11-24.
struct CamParams {
    float pos[3], right[3], up[3], fwd[3];
    float focal, lens_radius, tan_half, sa;
    int blades;
    float lca[3];
};

// Device counters; one block of these per context.
struct DevCounters {
    unsigned long long camera_paths;
    unsigned long long closest_rays;
    unsigned long long shadow_rays;
    unsigned long long photon_rays;
    unsigned long long gather_rays;
    unsigned long long photons_stored;
    unsigned long long node_tests;
    unsigned long long tri_tests;
    unsigned long long surface_hits;
    unsigned long long light_samples;
    unsigned long long photon_node_tests;   // photon trace + gather traversals
    unsigned long long photon_tri_tests;
    unsigned int error_word;
    unsigned int pad;
};

struct RenderArgs {
    DeviceScene scene;
    Images img;
    CamParams cam;
    int nee_enabled;
    float firefly_clamp;
    int first_frame;
    int n_spp;
    DevCounters* counters;
};

// The photon map (scene/PhotonMap.java) plus its cell-sorted copy.  The trace
// appends records and counts photons per hash cell; a scan of the counts and a
// scatter lay each cell's photons out contiguously (cell_start, seg_*), and
// the reference's heads/next chains are rebuilt from that order, so both
// views list the same photons in the same order.
struct PhotonArgs {
    DeviceScene scene;
    // First segment split (fast build): a photon's first segment leaves the
    // light and only matters when its nearest hit is specular (a diffuse
    // first hit ends it unstored).  `spec` holds the specular triangles,
    // `diff` the others, each with its own BVH; spec_orig maps a `spec`
    // triangle to its index in `scene`.  split == 0 traces the full scene.
    DeviceScene spec;
    DeviceScene diff;
    const int* spec_orig;
    int split;
    // photons whose first hit is specular, for the second phase of the
    // split trace (4 float4 each), and their count
    float4* queue;
    unsigned int* queue_len;
    // work counter of the refill emission kernel (zero before the trace;
    // null: one thread per photon) and its schedule (see WaveArgs)
    unsigned int* work;
    int refill_lanes;
    int leaf_quarters;
    int interior_steps;   // tree moves per lane per scheduling round of the refill emission
    float4* photons;        // 3 float4 per photon (std430 record)
    int* heads;
    int* next;
    unsigned int* counter;
    int* cell_of;           // hash cell of each stored photon
    unsigned int* cell_count;   // hash_size counters, zero before the trace
    unsigned int* cell_start;   // hash_size + 1 exclusive prefix sums
    unsigned int* block_sums;   // scan scratch
    int* seg_photon;        // photon index at each cell-sorted slot
    float4* seg_posw;       // (position.xyz, power.x) per slot
    float2* seg_powyz;      // (power.y, power.z) per slot
    int photon_count;
    int hash_size;
    float radius;
    int seed;
    DevCounters* counters;
};

struct GatherArgs {
    DeviceScene scene;
    Images img;
    CamParams cam;
    const unsigned int* cell_start;
    const float4* seg_posw;
    const float2* seg_powyz;
    int hash_size;
    float radius;
    float weight;
    DevCounters* counters;
    // The gather ray of a pixel (pixel centre, no lens) and its specular walk
    // are the same in every SPPM iteration of one camera: cache_mode 1 traces
    // them and stores the first diffuse hit (position, material; -1 = none)
    // per pixel in hit_cache, 2 reads it back, 0 traces without the cache.
    float4* hit_cache;
    int cache_mode;
    // Fast build with a hit cache: pixels whose 27 cells hold many photons
    // are listed here (heavy_len of them, pixel index y * W + x) and
    // gathered one warp per pixel by a second kernel; null: one pass.
    int* heavy;
    unsigned int* heavy_len;
};

struct AtrousArgs {
    const float4* color;      // RGBA32F input (or accum when normalize != 0)
    const ushort4* gbuf;
    const ushort4* galb;
    const float* var;
    float4* out;
    int width, height;
    int step;
    float sigma_color, sigma_normal, sigma_depth;
    int sample_count;         // max(N, 1)
    float exposure;
    int normalize;            // 1: color is the raw accumulation (p00 fused)
    float inv_n_unused;
};

struct NormalizeArgs {
    const float4* accum;
    float4* out;
    int count;
    int total_samples;
    float exposure;
};

// display.frag on the export path (rc_display): RGBA32F in, RGBA8 out with
// the rows in file order (top first).
struct DisplayArgs {
    const float4* color;
    uchar4* out;
    int width, height;
    int total_samples;
    float exposure;
};

// Wavefront path state, structure of arrays over the paths of one chunk
// (path p = tiled pixel j + NPIX * (channel + C * sample)).  Queues hold
// path indices; counters: qlen[0..1] ray queues, qlen[2..3] shadow queues.
struct WaveBuffers {
    float4* o;        // ray origin
    float4* d;        // ray direction
    float4* thr;      // throughput
    float4* rad;      // radiance so far
    float4* hit;      // t, u, v, primitive (int bits; -1 = miss)
    float4* res;      // final radiance of the path
    uint32_t* seed;   // PCG state
    int* rq[2];       // ray queues (ping-pong by bounce)
    int* sq[2];       // shadow queues
    float4* srec[2];  // shadow records, 3 float4 per queue slot (wavefront.cu)
    int* mq;          // material queues of the bounce's hits: diffuse paths
                      // from the front (count qlen[5]), metal and glass
                      // paths from the back (count qlen[6])
    unsigned int* qlen;
    int capacity;     // paths per chunk
};

// One frame's share of a wavefront chunk: samples [first_frame,
// first_frame + n_samples) of the frame with camera `cam` and images `img`,
// occupying paths [path_base, path_base + npix * channels * n_samples) of
// the chunk (path = path_base + tiled pixel + npix * (channel + channels *
// sample)).  A chunk of a single render call has one segment; a batch of
// frames packs slices of many frames into one chunk.
struct FrameSeg {
    CamParams cam;
    Images img;
    int first_frame;
    int n_samples;
    int channels;      // 3 with per-channel lens offsets, else 1
    int path_base;
};

struct WaveArgs {
    DeviceScene scene;
    WaveBuffers wb;
    FrameSeg one;            // the segment when segs == nullptr
    const FrameSeg* segs;    // nsegs segments sorted by path_base, or null
    int nsegs;
    int width, height;       // image size of every segment
    int nee_enabled;
    float firefly_clamp;
    int tiles_x;       // 8x4-pixel tiles across
    int npix;          // tiles * 32
    int paths;         // paths of the chunk (all segments)
    int bounce;
    int dynamic_fetch; // fast build: persistent trace kernel with ray refill
    int refill_min_paths;  // ... for chunks of at least this many paths
    int refill_lanes;  // refill when fewer lanes than this are busy (1..32)
    int leaf_quarters; // leaf phase once this many quarters of the busy lanes are blocked (1..4)
    int material_queues; // wf_sort ran: wf_shade walks the material queues (hits only)
    int interior_steps;  // refill trace: tree moves per lane per scheduling round (1..8)
    DevCounters* counters;
};

}  // namespace rc

#endif
