// noalloc.cu -- an à-trous entry point that allocates no device memory.
//
// Some hosts cannot let a library call cudaMalloc: engines that own every
// byte of device memory through their own pool and budget it per frame, or
// loops that cannot afford the device-wide synchronisation an allocation may
// cause in the middle of a frame.  rc_denoise_atrous_noalloc serves them:
// the caller passes the four renderer images and the output image as device
// pointers, and the one intermediate image the pass chain needs lives in the
// file-scope array below, which every GPU that loads this library holds for
// the life of the process (RC_NOALLOC_MAX_PIXELS * 16 bytes = 16 MiB).
//
// The passes alternate between that array and the caller's output so that
// the last pass always lands in the output; one intermediate buffer is
// enough.  Every call on a device shares the array and leaves its last
// contents there; nothing in it needs to start at zero because each pass
// overwrites every pixel it later reads.  Two calls whose work overlaps on
// the GPU (different streams, or different host threads) race on the array.
#include <cuda_runtime.h>

#include <cstdint>

#include "device_scene.h"
#include "host_checks.h"
#include "retrocam.h"

namespace rc {
namespace exact {
cudaError_t launch_atrous(const AtrousArgs&, cudaStream_t);
cudaError_t launch_normalize(const NormalizeArgs&, cudaStream_t);
}  // namespace exact
namespace fast {
cudaError_t launch_atrous(const AtrousArgs&, cudaStream_t);
cudaError_t launch_normalize(const NormalizeArgs&, cudaStream_t);
}  // namespace fast
}  // namespace rc

static __device__ __align__(256) float4 g_atrous_scratch[RC_NOALLOC_MAX_PIXELS];

namespace {

// The address of g_atrous_scratch in the current CUDA context.  Host code
// cannot use the symbol's name as a pointer (it is a host-side stand-in), so
// every call asks the runtime for the real address, with the caller's device
// current.  The address belongs to the context that loaded this module: a
// cached copy would outlive a cudaDeviceReset or point into another context
// on the same device, so it is looked up again each time (cheap once the
// module is loaded; the first call on a device loads it).
cudaError_t scratch_for_current_device(float4** out) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_atrous_scratch);
    if (e != cudaSuccess) return e;
    *out = (float4*)p;
    return cudaSuccess;
}

// [a, a+na) and [b, b+nb) share a byte.
bool overlaps(const void* a, size_t na, const void* b, size_t nb) {
    const uintptr_t x = (uintptr_t)a, y = (uintptr_t)b;
    return x < y + nb && y < x + na;
}

}  // namespace

namespace rc {
// api.cu: stores text for rc_last_error(NULL, ...) and returns code.
int set_global_error(int code, const char* msg);
}  // namespace rc

static int rc_noalloc_fail(int code, const char* msg) { return rc::set_global_error(code, msg); }

extern "C" int rc_denoise_atrous_noalloc(const float* accum, const uint16_t* gbuffer, const uint16_t* albedo,
                                         const float* variance, float* out, int width, int height,
                                         int total_samples, const rc_atrous_params* p, int math_mode,
                                         void* cuda_stream) {
    using namespace rc;
    if (!accum || !gbuffer || !albedo || !variance || !out || !p || width < 1 || height < 1 ||
        (math_mode != RC_MATH_FAST && math_mode != RC_MATH_EXACT))
        return rc_noalloc_fail(RC_ERR_INVALID_ARG, "rc_denoise_atrous_noalloc: bad arguments");
    if (!aligned_to(accum, 16) || !aligned_to(out, 16) || !aligned_to(gbuffer, 8) || !aligned_to(albedo, 8) ||
        !aligned_to(variance, 4))
        return rc_noalloc_fail(RC_ERR_INVALID_ARG, "rc_denoise_atrous_noalloc: misaligned buffer");
    if ((long long)width * height > RC_NOALLOC_MAX_PIXELS)
        return rc_noalloc_fail(RC_ERR_CAPACITY,
                               "rc_denoise_atrous_noalloc: width*height exceeds RC_NOALLOC_MAX_PIXELS "
                               "(1048576); use rc_denoise_atrous");
    // every pass reads its neighbours' pixels from the inputs while others
    // write the output, so the output may share no byte with any input
    const size_t npx = (size_t)width * height;
    if (overlaps(out, npx * 16, accum, npx * 16) || overlaps(out, npx * 16, gbuffer, npx * 8) ||
        overlaps(out, npx * 16, albedo, npx * 8) || overlaps(out, npx * 16, variance, npx * 4))
        return rc_noalloc_fail(RC_ERR_INVALID_ARG, "rc_denoise_atrous_noalloc: out overlaps an input image");
    float4* scratch = nullptr;
    cudaError_t e = scratch_for_current_device(&scratch);
    if (e != cudaSuccess)
        return rc_noalloc_fail(RC_ERR_CUDA, "rc_denoise_atrous_noalloc: cannot resolve the scratch array");
    cudaStream_t s = (cudaStream_t)cuda_stream;
    const bool ex = math_mode == RC_MATH_EXACT;
    const int N = total_samples;
    const bool over = p->max_spp > 0 && N > p->max_spp;
    if (p->enabled && !over) {
        const int passes = p->iterations < 1 ? 1 : (p->iterations > 5 ? 5 : p->iterations);
        const float4* src = (const float4*)accum;
        for (int i = 0; i < passes; ++i) {
            // the last pass writes the output; earlier ones alternate so that
            // no pass reads the buffer it writes
            float4* dst = ((passes - 1 - i) % 2 == 0) ? (float4*)out : scratch;
            AtrousArgs A;
            A.color = src;
            A.gbuf = (const ushort4*)gbuffer;
            A.galb = (const ushort4*)albedo;
            A.var = variance;
            A.out = dst;
            A.width = width;
            A.height = height;
            A.step = 1 << i;
            A.sigma_color = p->sigma_color;
            A.sigma_normal = p->sigma_normal;
            A.sigma_depth = p->sigma_depth;
            A.sample_count = N > 1 ? N : 1;
            A.exposure = p->exposure;
            A.normalize = (i == 0) ? 1 : 0;
            A.inv_n_unused = 0.0f;
            e = ex ? exact::launch_atrous(A, s) : fast::launch_atrous(A, s);
            if (e != cudaSuccess) return rc_noalloc_fail(RC_ERR_CUDA, "rc_denoise_atrous_noalloc: launch failed");
            src = dst;
        }
    } else {
        NormalizeArgs A;
        A.accum = (const float4*)accum;
        A.out = (float4*)out;
        A.count = width * height;
        A.total_samples = N;
        A.exposure = p->exposure;
        e = ex ? exact::launch_normalize(A, s) : fast::launch_normalize(A, s);
        if (e != cudaSuccess) return rc_noalloc_fail(RC_ERR_CUDA, "rc_denoise_atrous_noalloc: launch failed");
    }
    return RC_OK;
}
