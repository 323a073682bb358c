/*
 * glsl_compat.h -- TEST INFRASTRUCTURE (oracle). Never linked into the product.
 *
 * A small GLSL 4.30 subset in C++ so that the reference's own compute and
 * fragment shaders (pathtrace.comp, photon_trace.comp, photon_gather.comp,
 * post/atrous_denoise.frag, post/p00_normalize.frag) compile unchanged in
 * meaning on the host after the mechanical text transforms in build_ref.py.
 * The result (oracle/_ref/libretrocam_ref.so) is the reference itself, run
 * on the CPU, and pins the hand-written oracle in oracle/oracle.cpp.
 *
 * Semantics chosen where GLSL leaves room (the same choices are made by the
 * oracle and by the exact build of the CUDA kernels):
 *   - float arithmetic is IEEE single, no contraction (-ffp-contract=off);
 *   - sin/cos/exp/log/pow come from include/rc_exact_math.h;
 *   - min(x,y) = y < x ? y : x and max(x,y) = x < y ? y : x, the GLSL 4.30
 *     section 8.3 definitions; clamp(x,a,b) = min(max(x,a),b);
 *   - dot, cross, length, normalize (v / length(v)), reflect and refract
 *     use the formulas of GLSL 4.30 section 8.5, evaluated left to right;
 *   - images: rgba32f/r32f stored as float, rgba16f rounded to half (RNE);
 *   - texture(): NEAREST or LINEAR with 8-bit filter weights, REPEAT or
 *     CLAMP_TO_EDGE, as the reference configures each texture
 *     (core/Renderer.java:152-193, gl/Framebuffer.java:72-77).
 * Everything lives in namespace glsl so that unqualified calls from the
 * shader text resolve here before any libc overload.
 */
#ifndef RC_GLSL_COMPAT_H
#define RC_GLSL_COMPAT_H

#include <stdint.h>
#include "rc_exact_math.h"
#include "half_soft.h"

namespace glsl {

typedef unsigned int uint;

struct bvec2 { bool x, y; };
struct bvec3 { bool x, y, z; };
struct uvec2;
struct ivec2;
struct uvec3 {
    uint x, y, z;
    uvec2 xy() const;
};
struct ivec2 {
    int x, y;
    ivec2() : x(0), y(0) {}
    ivec2(int a, int b) : x(a), y(b) {}
    explicit ivec2(const uvec2& u);
    explicit ivec2(const struct vec2& v);
};
struct uvec2 {
    uint x, y;
    uvec2() : x(0), y(0) {}
    uvec2(uint a, uint b) : x(a), y(b) {}
};
inline uvec2 uvec3::xy() const { return uvec2(x, y); }
inline ivec2::ivec2(const uvec2& u) : x((int)u.x), y((int)u.y) {}

struct vec2 {
    float x, y;
    vec2() : x(0), y(0) {}
    explicit vec2(float s) : x(s), y(s) {}
    template <class A, class B> vec2(A a, B b) : x((float)a), y((float)b) {}
    explicit vec2(const ivec2& v) : x((float)v.x), y((float)v.y) {}
};
inline ivec2::ivec2(const vec2& v) : x((int)v.x), y((int)v.y) {}
struct vec3 {
    float x, y, z;
    vec3() : x(0), y(0), z(0) {}
    explicit vec3(float s) : x(s), y(s), z(s) {}
    template <class A, class B, class C> vec3(A a, B b, C c) : x((float)a), y((float)b), z((float)c) {}
    vec3(float a, const vec2& b) : x(a), y(b.x), z(b.y) {}
    vec2 xy() const { return vec2(x, y); }
    vec2 yz() const { return vec2(y, z); }
    void set_yz(const vec2& v) { y = v.x; z = v.y; }   /* the .yz = ... swizzle write */
    vec3 xyz() const { return *this; }
};
struct vec4 {
    float x, y, z, w;
    vec4() : x(0), y(0), z(0), w(0) {}
    explicit vec4(float s) : x(s), y(s), z(s), w(s) {}
    vec4(const vec3& v, float s) : x(v.x), y(v.y), z(v.z), w(s) {}
    template <class A, class B, class C, class D>
    vec4(A a, B b, C c, D d) : x((float)a), y((float)b), z((float)c), w((float)d) {}
    vec3 xyz() const { return vec3(x, y, z); }
};
struct ivec3 {
    int x, y, z;
    ivec3() : x(0), y(0), z(0) {}
    ivec3(int a, int b, int c) : x(a), y(b), z(c) {}
    explicit ivec3(const vec3& v) : x((int)v.x), y((int)v.y), z((int)v.z) {}
};
struct mat3 {
    vec3 c0, c1, c2;
    mat3(const vec3& a, const vec3& b, const vec3& c) : c0(a), c1(b), c2(c) {}
};

/* ---- vector arithmetic, component-wise ---- */
#define RCG_BIN(OP)                                                                     \
    inline vec2 operator OP(const vec2& a, const vec2& b) { return vec2(a.x OP b.x, a.y OP b.y); } \
    inline vec2 operator OP(const vec2& a, float s) { return vec2(a.x OP s, a.y OP s); }           \
    inline vec2 operator OP(float s, const vec2& a) { return vec2(s OP a.x, s OP a.y); }           \
    inline vec3 operator OP(const vec3& a, const vec3& b) { return vec3(a.x OP b.x, a.y OP b.y, a.z OP b.z); } \
    inline vec3 operator OP(const vec3& a, float s) { return vec3(a.x OP s, a.y OP s, a.z OP s); }  \
    inline vec3 operator OP(float s, const vec3& a) { return vec3(s OP a.x, s OP a.y, s OP a.z); }  \
    inline vec4 operator OP(const vec4& a, const vec4& b) { return vec4(a.x OP b.x, a.y OP b.y, a.z OP b.z, a.w OP b.w); } \
    inline vec4 operator OP(const vec4& a, float s) { return vec4(a.x OP s, a.y OP s, a.z OP s, a.w OP s); }
RCG_BIN(+)
RCG_BIN(-)
RCG_BIN(*)
RCG_BIN(/)
#undef RCG_BIN
inline vec2& operator+=(vec2& a, const vec2& b) { a = a + b; return a; }
inline vec3& operator+=(vec3& a, const vec3& b) { a = a + b; return a; }
inline vec2& operator*=(vec2& a, float s) { a = a * s; return a; }
inline vec2& operator/=(vec2& a, float s) { a = a / s; return a; }
inline vec3& operator*=(vec3& a, const vec3& b) { a = a * b; return a; }
inline vec3& operator*=(vec3& a, float s) { a = a * s; return a; }
inline vec3& operator/=(vec3& a, float s) { a = a / s; return a; }
inline vec4& operator+=(vec4& a, const vec4& b) { a = a + b; return a; }
inline vec3 operator-(const vec3& a) { return vec3(-a.x, -a.y, -a.z); }
inline vec2 operator-(const vec2& a) { return vec2(-a.x, -a.y); }
inline ivec3 operator+(const ivec3& a, const ivec3& b) { return ivec3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline vec3 operator*(const mat3& m, const vec3& v) { return m.c0 * v.x + m.c1 * v.y + m.c2 * v.z; }

/* ---- scalar built-ins ---- */
inline float abs(float x) { return rcx_bitsf(rcx_fbits(x) & 0x7fffffffu); }
inline float sqrt(float x) { return __builtin_sqrtf(x); }
inline float floor(float x) { return __builtin_floorf(x); }
#ifdef RC_REF_HOST_LIBM
/* timing variant of the compiled reference (oracle/_ref/libretrocam_ref_libm.so):
 * the host C library's single-precision functions, as a GL driver's compiler
 * would use its own fast ones; not used for parity */
inline float sin(float x) { return __builtin_sinf(x); }
inline float cos(float x) { return __builtin_cosf(x); }
inline float exp(float x) { return __builtin_expf(x); }
inline float log(float x) { return __builtin_logf(x); }
inline float pow(float x, float y) { return __builtin_powf(x, y); }
#else
inline float sin(float x) { return rcx_sinf(x); }
inline float cos(float x) { return rcx_cosf(x); }
inline float exp(float x) { return rcx_expf(x); }
inline float log(float x) { return rcx_logf(x); }
inline float pow(float x, float y) { return rcx_powf(x, y); }
#endif
inline float min(float x, float y) { return (y < x) ? y : x; }
inline float max(float x, float y) { return (x < y) ? y : x; }
inline int min(int x, int y) { return (y < x) ? y : x; }
inline int max(int x, int y) { return (x < y) ? y : x; }
inline float clamp(float x, float a, float b) { return min(max(x, a), b); }
inline int clamp(int x, int a, int b) { return min(max(x, a), b); }
/* GLSL 4.30 section 8.3; round() ties away from zero (the spec leaves the
 * direction to the implementation) */
inline float fract(float x) { return x - floor(x); }
inline float round(float x) { return __builtin_roundf(x); }
inline float sign(float x) { return x > 0.0f ? 1.0f : (x < 0.0f ? -1.0f : 0.0f); }
inline float radians(float d) { return d * 0.017453292519943295f; }
inline float step(float e, float x) { return x < e ? 0.0f : 1.0f; }
inline float mix(float x, float y, float a) { return x * (1.0f - a) + y * a; }
inline float smoothstep(float e0, float e1, float x) {
    const float t = clamp((x - e0) / (e1 - e0), 0.0f, 1.0f);
    return t * t * (3.0f - 2.0f * t);
}
inline bool isnan_s(float x) { return (rcx_fbits(x) & 0x7fffffffu) > 0x7f800000u; }
inline bool isinf_s(float x) { return (rcx_fbits(x) & 0x7fffffffu) == 0x7f800000u; }

/* ---- vector built-ins ---- */
inline vec3 floor(const vec3& v) { return vec3(floor(v.x), floor(v.y), floor(v.z)); }
inline vec3 min(const vec3& a, const vec3& b) { return vec3(min(a.x, b.x), min(a.y, b.y), min(a.z, b.z)); }
inline vec3 max(const vec3& a, const vec3& b) { return vec3(max(a.x, b.x), max(a.y, b.y), max(a.z, b.z)); }
inline vec3 clamp(const vec3& v, float a, float b) { return vec3(clamp(v.x, a, b), clamp(v.y, a, b), clamp(v.z, a, b)); }
inline vec3 pow(const vec3& x, const vec3& y) { return vec3(pow(x.x, y.x), pow(x.y, y.y), pow(x.z, y.z)); }
/* GLSL 4.30 section 8.3: step(edge, x) = x < edge ? 0 : 1; mix(x, y, a) = x * (1 - a) + y * a */
inline vec3 step(float e, const vec3& x) {
    return vec3(x.x < e ? 0.0f : 1.0f, x.y < e ? 0.0f : 1.0f, x.z < e ? 0.0f : 1.0f);
}
inline vec3 mix(const vec3& x, const vec3& y, const vec3& a) { return x * (vec3(1.0f) - a) + y * a; }
inline vec3 mix(const vec3& x, const vec3& y, float a) { return x * (1.0f - a) + y * a; }
inline vec2 clamp(const vec2& v, const vec2& a, const vec2& b) { return vec2(clamp(v.x, a.x, b.x), clamp(v.y, a.y, b.y)); }
inline float dot(const vec2& a, const vec2& b) { return a.x * b.x + a.y * b.y; }
inline float dot(const vec3& a, const vec3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline vec3 cross(const vec3& a, const vec3& b) {
    return vec3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
inline float length(const vec3& v) { return sqrt(dot(v, v)); }
inline vec3 normalize(const vec3& v) { return v / length(v); }
inline vec3 reflect(const vec3& I, const vec3& N) { return I - 2.0f * dot(N, I) * N; }
inline vec3 refract(const vec3& I, const vec3& N, float eta) {
    const float d = dot(N, I);
    const float k = 1.0f - eta * eta * (1.0f - d * d);
    if (k < 0.0f) return vec3(0.0f);
    return eta * I - (eta * d + sqrt(k)) * N;
}
inline bvec3 isnan(const vec3& v) { return bvec3{isnan_s(v.x), isnan_s(v.y), isnan_s(v.z)}; }
inline bvec3 isinf(const vec3& v) { return bvec3{isinf_s(v.x), isinf_s(v.y), isinf_s(v.z)}; }
inline bool any(const bvec3& b) { return b.x || b.y || b.z; }
inline bool any(const bvec2& b) { return b.x || b.y; }
inline bvec2 greaterThanEqual(const ivec2& a, const ivec2& b) { return bvec2{a.x >= b.x, a.y >= b.y}; }

/* ---- atomics on SSBO words ---- */
inline uint atomicAdd(uint& mem, uint v) { return __atomic_fetch_add(&mem, v, __ATOMIC_SEQ_CST); }
inline int atomicExchange(int& mem, int v) { return __atomic_exchange_n(&mem, v, __ATOMIC_SEQ_CST); }

/* ---- images (imageLoad / imageStore) ---- */
enum ImgFormat { FMT_RGBA32F = 0, FMT_RGBA16F = 1, FMT_R32F = 2 };
struct image2D {
    void* data = nullptr;
    int w = 0, h = 0;
    int fmt = FMT_RGBA32F;
};
inline vec4 imageLoad(const image2D& im, const ivec2& p) {
    const long i = (long)p.y * im.w + p.x;
    if (im.fmt == FMT_RGBA32F) {
        const float* f = (const float*)im.data + 4 * i;
        return vec4(f[0], f[1], f[2], f[3]);
    }
    if (im.fmt == FMT_R32F) return vec4(((const float*)im.data)[i], 0.0f, 0.0f, 1.0f);
    const uint16_t* hh = (const uint16_t*)im.data + 4 * i;
    return vec4(half_to_float(hh[0]), half_to_float(hh[1]), half_to_float(hh[2]), half_to_float(hh[3]));
}
inline void imageStore(image2D& im, const ivec2& p, const vec4& v) {
    const long i = (long)p.y * im.w + p.x;
    if (im.fmt == FMT_RGBA32F) {
        float* f = (float*)im.data + 4 * i;
        f[0] = v.x; f[1] = v.y; f[2] = v.z; f[3] = v.w;
    } else if (im.fmt == FMT_R32F) {
        ((float*)im.data)[i] = v.x;
    } else {
        uint16_t* hh = (uint16_t*)im.data + 4 * i;
        hh[0] = float_to_half_rne(v.x); hh[1] = float_to_half_rne(v.y);
        hh[2] = float_to_half_rne(v.z); hh[3] = float_to_half_rne(v.w);
    }
}

/* ---- textures (texture()) ---- */
enum TexFilter { FILTER_NEAREST = 0, FILTER_LINEAR = 1 };
enum TexWrap { WRAP_REPEAT = 0, WRAP_CLAMP = 1 };
struct sampler2D {
    image2D img;
    int filter = FILTER_NEAREST;
    int wrap = WRAP_REPEAT;
};
inline int wrap_index(int i, int n, int wrap) {
    if (wrap == WRAP_CLAMP) return i < 0 ? 0 : (i >= n ? n - 1 : i);
    int m = i % n;
    return m < 0 ? m + n : m;
}
inline ivec2 textureSize(const sampler2D& s, int) { return ivec2(s.img.w, s.img.h); }
inline vec4 texel(const sampler2D& s, int ix, int iy) {
    return imageLoad(s.img, ivec2(wrap_index(ix, s.img.w, s.wrap), wrap_index(iy, s.img.h, s.wrap)));
}
/* Filter weights are quantised to 1/256 as texture units do. */
inline float quant_weight(float a) { return floor(a * 256.0f + 0.5f) * (1.0f / 256.0f); }
inline vec4 texture(const sampler2D& s, const vec2& uv) {
    const float fx = uv.x * (float)s.img.w;
    const float fy = uv.y * (float)s.img.h;
    if (s.filter == FILTER_NEAREST) return texel(s, (int)floor(fx), (int)floor(fy));
    const float gx = fx - 0.5f, gy = fy - 0.5f;
    const float x0 = floor(gx), y0 = floor(gy);
    const float ax = quant_weight(gx - x0), ay = quant_weight(gy - y0);
    const int ix = (int)x0, iy = (int)y0;
    const int sx = (ax >= 1.0f) ? 1 : 0, sy = (ay >= 1.0f) ? 1 : 0;
    const bool exact_x = (ax == 0.0f) || (ax >= 1.0f);
    const bool exact_y = (ay == 0.0f) || (ay >= 1.0f);
    if (exact_x && exact_y) return texel(s, ix + sx, iy + sy);
    /* General bilinear blend (never reached at the integer texel offsets
     * the reference uses, kept for completeness). */
    const vec4 t00 = texel(s, ix, iy), t10 = texel(s, ix + 1, iy);
    const vec4 t01 = texel(s, ix, iy + 1), t11 = texel(s, ix + 1, iy + 1);
    const vec4 a = t00 * (1.0f - ax) + t10 * ax;
    const vec4 b = t01 * (1.0f - ax) + t11 * ax;
    return a * (1.0f - ay) + b * ay;
}

} /* namespace glsl */

#endif
