// post_vhs.cu -- the VHS chain: post/PostProcessStack.java:149-277 with the
// fragment shaders post/p01_downsample.frag .. post/p16_interlace.frag, one
// kernel launch per enabled pass over RGBA32F images (one thread per pixel,
// the pixel centre as v_uv, gl_FragCoord = pixel + 0.5).
//
// Built with the exact-math flags only (-fmad=false, IEEE divide and
// square root, no flush to zero) and the transcendentals of
// include/rc_exact_math.h: each pass follows its shader's operations in
// order, and texture() is the LINEAR / CLAMP_TO_EDGE lookup of the
// ping-pong textures (gl/Framebuffer.java:74-77) with filter weights
// quantised to 1/256, so results are bit-identical to the shaders compiled
// for the host.  The passes are a few microseconds each; both math modes
// use these kernels.  GLSL built-ins as GLSL 4.30 section 8 defines them;
// round() ties away from zero (the direction the spec leaves open).
#include <cuda_runtime.h>
#include <stdint.h>

#include "host_checks.h"
#include "rc_exact_math.h"
#include "retrocam.h"

namespace rc {
namespace vhs {

#define DI __device__ __forceinline__

struct V2 {
    float x, y;
};
struct V3 {
    float x, y, z;
};
DI V3 v3(float a, float b, float c) { return V3{a, b, c}; }
DI V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
DI V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
DI V3 operator*(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
DI V3 operator/(V3 a, float s) { return v3(a.x / s, a.y / s, a.z / s); }

DI float gmin(float x, float y) { return (y < x) ? y : x; }
DI float gmax(float x, float y) { return (x < y) ? y : x; }
DI int imin(int x, int y) { return (y < x) ? y : x; }
DI int imax(int x, int y) { return (x < y) ? y : x; }
DI float gclamp(float x, float a, float b) { return gmin(gmax(x, a), b); }
DI V3 gclamp3(V3 v, float a, float b) { return v3(gclamp(v.x, a, b), gclamp(v.y, a, b), gclamp(v.z, a, b)); }
DI float gabs(float x) { return rcx_bitsf(rcx_fbits(x) & 0x7fffffffu); }
DI float fract_(float x) { return x - floorf(x); }
DI float sign_(float x) { return x > 0.0f ? 1.0f : (x < 0.0f ? -1.0f : 0.0f); }
DI float step_(float e, float x) { return x < e ? 0.0f : 1.0f; }
DI float mix_(float x, float y, float a) { return x * (1.0f - a) + y * a; }
DI V3 mix3(V3 x, V3 y, float a) { return x * (1.0f - a) + y * a; }
DI float smoothstep_(float e0, float e1, float x) {
    const float t = gclamp((x - e0) / (e1 - e0), 0.0f, 1.0f);
    return t * t * (3.0f - 2.0f * t);
}
DI float dot3(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
DI float gauss(float x, float sigma) { return rcx_expf(-(x * x) / (2.0f * sigma * sigma)); }

// texture(u_tex, uv).rgb of an RGBA32F texture, LINEAR with 8-bit weights,
// CLAMP_TO_EDGE (the integer-offset lookups land on one texel exactly).
struct Tex {
    const float4* img;
    int w, h;
};
DI float4 texel(const Tex& t, int ix, int iy) {
    ix = ix < 0 ? 0 : (ix >= t.w ? t.w - 1 : ix);
    iy = iy < 0 ? 0 : (iy >= t.h ? t.h - 1 : iy);
    return __ldg(t.img + (size_t)iy * t.w + ix);
}
DI float quant_weight(float a) { return floorf(a * 256.0f + 0.5f) * (1.0f / 256.0f); }
DI V3 tex(const Tex& t, float u, float v) {
    const float fx = u * (float)t.w, fy = v * (float)t.h;
    const float gx = fx - 0.5f, gy = fy - 0.5f;
    const float x0 = floorf(gx), y0 = floorf(gy);
    const float ax = quant_weight(gx - x0), ay = quant_weight(gy - y0);
    const int ix = (int)x0, iy = (int)y0;
    const int sx = (ax >= 1.0f) ? 1 : 0, sy = (ay >= 1.0f) ? 1 : 0;
    const bool exact_x = (ax == 0.0f) || (ax >= 1.0f);
    const bool exact_y = (ay == 0.0f) || (ay >= 1.0f);
    if (exact_x && exact_y) {
        const float4 c = texel(t, ix + sx, iy + sy);
        return v3(c.x, c.y, c.z);
    }
    const float4 t00 = texel(t, ix, iy), t10 = texel(t, ix + 1, iy);
    const float4 t01 = texel(t, ix, iy + 1), t11 = texel(t, ix + 1, iy + 1);
    const V3 a = v3(t00.x, t00.y, t00.z) * (1.0f - ax) + v3(t10.x, t10.y, t10.z) * ax;
    const V3 b = v3(t01.x, t01.y, t01.z) * (1.0f - ax) + v3(t11.x, t11.y, t11.z) * ax;
    return a * (1.0f - ay) + b * ay;
}

// The two YCbCr matrices of the passes: five decimals (p02, p07, p09, p13,
// p14, p15) and three (p03, p04).
DI V3 ycc5(V3 c) {
    return v3(0.29900f * c.x + 0.58700f * c.y + 0.11400f * c.z,
              -0.16874f * c.x - 0.33126f * c.y + 0.50000f * c.z + 0.5f,
              0.50000f * c.x - 0.41869f * c.y - 0.08131f * c.z + 0.5f);
}
DI V3 rgb5(V3 ycc) {
    const float y = ycc.x, cb = ycc.y - 0.5f, cr = ycc.z - 0.5f;
    return v3(y + 1.40200f * cr, y - 0.34414f * cb - 0.71414f * cr, y + 1.77200f * cb);
}
DI V3 ycc3(V3 c) {
    return v3(0.299f * c.x + 0.587f * c.y + 0.114f * c.z, -0.169f * c.x - 0.331f * c.y + 0.500f * c.z + 0.5f,
              0.500f * c.x - 0.419f * c.y - 0.081f * c.z + 0.5f);
}
DI V3 rgb3(V3 ycc) {
    const float Y = ycc.x, Cb = ycc.y - 0.5f, Cr = ycc.z - 0.5f;
    return v3(Y + 1.402f * Cr, Y - 0.344f * Cb - 0.714f * Cr, Y + 1.772f * Cb);
}
DI V2 rotate_cbcr(V2 cbcr, float theta) {
    const float c = rcx_cosf(theta), s = rcx_sinf(theta);
    return V2{cbcr.x * c - cbcr.y * s, cbcr.x * s + cbcr.y * c};
}
DI float hash_to_float(uint32_t h) { return (float)h / 4294967295.0f; }
// p12's hash; p13 and p14 use the two-round one
DI uint32_t uhash12(uint32_t x) {
    x ^= x >> 16u;
    x *= 0x45d9f3bu;
    x ^= x >> 16u;
    return x;
}
DI uint32_t uhash2(uint32_t x) {
    x = ((x >> 16u) ^ x) * 0x45d9f3bu;
    x = ((x >> 16u) ^ x) * 0x45d9f3bu;
    x = (x >> 16u) ^ x;
    return x;
}
DI float fhash12(uint32_t a, uint32_t b) { return (float)uhash12(a ^ uhash12(b) * 2654435761u) / 4294967295.0f; }
DI float fhash2(uint32_t a, uint32_t b) { return (float)uhash2(a ^ uhash2(b) * 2654435761u) / 4294967295.0f; }

struct Frag {
    float u, v;      // v_uv
    float fx, fy;    // gl_FragCoord.xy
};

// ---------------------------------------------------------------------------
// the passes: each returns fragColor.rgb (alpha is 1 for every pass)
// ---------------------------------------------------------------------------
// Tap weights that depend only on the tap and the uniforms (the Gaussians
// of p01/p02, the 0.70^i decay of p08): one block computes each once, by
// the shader's own expression, into shared memory.
constexpr int kWeightTaps = 151;
DI int p02_radius(const rc_vhs_params& P) {
    const float sigma = gmax(P.chroma_res_sigma, 0.5f);
    return imin(imax((int)(sigma * 2.5f + 0.5f), 1), 32);
}
DI void fill_weights(int pass, const rc_vhs_params& P, float* wtab) {
    for (int j = threadIdx.x; j < kWeightTaps; j += blockDim.x) {
        if (pass == 1 && j < 9) {
            wtab[j] = gauss((float)(j - 4), gmax(P.luma_blur_sigma, 0.01f));
        } else if (pass == 2) {
            const int r = p02_radius(P);
            if (j <= 2 * r) wtab[j] = gauss((float)(j - r), gmax(P.chroma_res_sigma, 0.5f));
        } else if (pass == 8 && j >= 1) {
            wtab[j] = rcx_powf(0.70f, (float)j);
        }
    }
}

// p01_downsample.frag: 9-tap horizontal Gaussian
DI V3 p01(const Tex& t, const Frag& f, const rc_vhs_params& P, const float* wtab) {
    const float tsx = 1.0f / (float)t.w;
    V3 sum = v3(0.0f, 0.0f, 0.0f);
    float wt = 0.0f;
    for (int i = -4; i <= 4; i++) {
        const float w = wtab[i + 4];
        sum = sum + tex(t, f.u + (float)i * tsx, f.v + 0.0f) * w;
        wt += w;
    }
    return sum / wt;
}

// p02_chroma_res.frag: Gaussian blur of Cb/Cr only
DI V3 p02(const Tex& t, const Frag& f, const rc_vhs_params& P, const float* wtab) {
    const float tsx = 1.0f / (float)t.w;
    const int radius = p02_radius(P);
    const float lumaY = ycc5(tex(t, f.u, f.v)).x;
    float cb = 0.0f, cr = 0.0f, wt = 0.0f;
    for (int i = -radius; i <= radius; i++) {
        const float w = wtab[i + radius];
        const V3 c = ycc5(tex(t, f.u + (float)i * tsx, f.v + 0.0f));
        cb = cb + c.y * w;
        cr = cr + c.z * w;
        wt += w;
    }
    cb = cb / wt;
    cr = cr / wt;
    return rgb5(v3(lumaY, cb, cr));
}

// p03_color_matrix.frag: saturation, hue rotation, temperature and drift
DI V3 p03(const Tex& t, const Frag& f, const rc_vhs_params& P) {
    V3 ycc = ycc3(tex(t, f.u, f.v));
    V2 ch = V2{ycc.y - 0.5f, ycc.z - 0.5f};
    ch = V2{ch.x * P.color_saturation, ch.y * P.color_saturation};
    const float rad = P.color_hue_rot * 0.017453292519943295f;
    const float cosH = rcx_cosf(rad), sinH = rcx_sinf(rad);
    ch = V2{cosH * ch.x - sinH * ch.y, sinH * ch.x + cosH * ch.y};
    const float drift = rcx_sinf(P.time_s * P.color_drift_speed) * 0.015f;
    const float temp = P.color_temp_bias * 0.05f + drift;
    ch.y += temp;
    ch.x -= temp * 0.75f;
    ycc.y = ch.x + 0.5f;
    ycc.z = ch.y + 0.5f;
    return gclamp3(rgb3(ycc), 0.0f, 1.0f);
}

// p04_dynamic_range.frag: shadow crush, black lift, highlight knee on luma
DI float shadow_crush(float x, float c) {
    if (x >= c) return x;
    const float t = x / gmax(c, 0.0001f);
    const float u = t * t * (3.0f - 2.0f * t);
    return u * c;
}
DI float knee_(float x, float knee, float clip) {
    if (x <= knee) return x;
    const float t = (x - knee) / gmax(1.0f - knee, 0.0001f);
    const float rolled = knee + (clip - knee) * (1.0f - rcx_expf(-3.5f * t));
    return gmin(rolled, clip);
}
DI V3 p04(const Tex& t, const Frag& f, const rc_vhs_params& P) {
    V3 ycc = ycc3(tex(t, f.u, f.v));
    const float Yin = ycc.x;
    float Y = Yin;
    Y = shadow_crush(Y, P.dr_shadow_crush);
    Y = P.dr_black_lift + (1.0f - P.dr_black_lift) * Y;
    Y = knee_(Y, P.dr_highlight_knee, P.dr_highlight_clip);
    const float ls = (Yin > 0.001f) ? (Y / Yin) : 1.0f;
    ycc.x = Y;
    ycc.y = (ycc.y - 0.5f) * ls + 0.5f;
    ycc.z = (ycc.z - 0.5f) * ls + 0.5f;
    return gclamp3(rgb3(ycc), 0.0f, 1.0f);
}

// p07_ccd_noise.frag: luminance-dependent PCG noise, AGC-scaled, row bands
DI uint32_t pcg_hash(uint32_t v) {
    v = v * 747796405u + 2891336453u;
    const uint32_t w = ((v >> ((v >> 28u) + 4u)) ^ v) * 277803737u;
    return (w >> 22u) ^ w;
}
DI float rand7(int px, int py, int seed) {
    const uint32_t h = pcg_hash((uint32_t)px ^ ((uint32_t)py * 1619u) ^ ((uint32_t)seed * 2654435761u));
    return hash_to_float(h) * 2.0f - 1.0f;
}
DI V3 p07(const Tex& t, const Frag& f, const rc_vhs_params& P) {
    const int px = (int)(f.u * (float)t.w), py = (int)(f.v * (float)t.h);
    V3 ycc = ycc5(tex(t, f.u, f.v));
    const float lum = gclamp(ycc.x, 0.0f, 1.0f);
    const float lumaAmp = (P.ccd_noise_luma_base + 0.04f * (1.0f - lum)) * P.agc_gain;
    const float chromaAmp = lumaAmp * P.ccd_noise_chroma_scale;
    const float nY = rand7(px, py, P.frame_index) * lumaAmp;
    const float nCb = rand7(px, py, P.frame_index + 137) * chromaAmp;
    const float nCr = rand7(px, py, P.frame_index + 271) * chromaAmp;
    const int rowSeed = py * 7 + (P.frame_index / 8);
    const float band = rand7(0, rowSeed, 0) * 0.005f * P.agc_gain;
    ycc.x += nY + band;
    ycc.y += nCb;
    ycc.z += nCr;
    return rgb5(ycc);
}

// p08_ccd_smear.frag: vertical overflow streaks above and below bright pixels
DI float luma601(V3 c) { return 0.299f * c.x + 0.587f * c.y + 0.114f * c.z; }
DI V3 p08(const Tex& t, const Frag& f, const rc_vhs_params& P, const float* wtab) {
    const V3 base = tex(t, f.u, f.v);
    const float tsy = 1.0f / (float)t.h;
    float pa = 0.0f;
    int pt = 0;
    for (int i = 1; i <= 150; i++) {
        if (i > P.ccd_smear_length) break;
        const float sy = f.v + (float)i * tsy;
        if (sy > 1.0f) break;
        pa += gmax(0.0f, luma601(tex(t, f.u + 0.0f, sy)) - P.ccd_smear_threshold);
        pt++;
    }
    const float pc = (pt > 0) ? (pa / (float)pt) * P.ccd_smear_intensity : 0.0f;
    const int sl = imax(1, (int)((float)P.ccd_smear_length * 0.30f));
    float sa = 0.0f;
    int st = 0;
    for (int i = 1; i <= 150; i++) {
        if (i > sl) break;
        const float sy = f.v - (float)i * tsy;
        if (sy < 0.0f) break;
        sa += gmax(0.0f, luma601(tex(t, f.u - 0.0f, sy)) - P.ccd_smear_threshold) * wtab[i];
        st++;
    }
    const float sc = (st > 0) ? (sa / (float)st) * P.ccd_smear_intensity * 0.25f : 0.0f;
    const float total = pc + sc;
    return gclamp3(base + v3(total, total, total), 0.0f, 1.0f);
}

// p09_chroma_bleed.frag: rightward exponential chroma smear
DI V3 p09(const Tex& t, const Frag& f, const rc_vhs_params& P) {
    const float tsx = 1.0f / (float)t.w;
    const float k = gclamp(P.chroma_bleed_factor, 0.0f, 0.98f);
    const float lumaY = ycc5(tex(t, f.u, f.v)).x;
    float cb = 0.0f, cr = 0.0f, wt = 0.0f, kpow = 1.0f;
    const float scale = 1.0f - k;
    for (int i = 0; i < 24; i++) {
        const V3 c = ycc5(tex(t, f.u - (float)i * tsx, f.v));
        const float w = scale * kpow;
        cb = cb + c.y * w;
        cr = cr + c.z * w;
        wt += w;
        kpow *= k;
    }
    cb = cb / wt;
    cr = cr / wt;
    return rgb5(v3(lumaY, cb, cr));
}

// p10_timebase.frag: per-scanline horizontal jitter (sine + value noise)
DI float hash10(float x) { return fract_(rcx_sinf(x * 127.1f + 311.7f) * 43758.5453f); }
DI float noise10(float x) {
    const float i = floorf(x), fr = fract_(x);
    const float u = fr * fr * (3.0f - 2.0f * fr);
    return mix_(hash10(i), hash10(i + 1.0f), u);
}
DI V3 p10(const Tex& t, const Frag& f, const rc_vhs_params& P) {
    const float sx = (float)t.w, sy = (float)t.h;
    const float scan = f.v * sy;
    const float bucket = (float)(P.frame_index / 4) * 0.137f;
    const float sinPart = rcx_sinf(scan * P.timebase_freq + P.time_s * P.timebase_speed);
    const float noisePart = noise10(scan * 0.05f + bucket) * 2.0f - 1.0f;
    const float offsetPx = P.timebase_amplitude_px * (sinPart * 0.5f + noisePart * 0.5f);
    const float uvOffset = offsetPx / sx;
    return tex(t, gclamp(f.u + uvOffset, 0.0f, 1.0f), f.v);
}

// p11_dot_crawl.frag: subcarrier crosstalk on luma edges
DI float luma709(V3 c) { return dot3(c, v3(0.2126f, 0.7152f, 0.0722f)); }
DI V3 p11(const Tex& t, const Frag& f, const rc_vhs_params& P) {
    const float rx = (float)t.w, ry = (float)t.h;
    const V3 col = tex(t, f.u, f.v);
    const float pixX = f.u * rx;
    const float lineY = floorf(f.v * ry);
    const float pxW = 1.0f / rx;
    const float lumC = luma709(col);
    const float lumL = luma709(tex(t, f.u - pxW, f.v));
    const float lumR = luma709(tex(t, f.u + pxW, f.v));
    const float grad = gmax(gabs(lumC - lumL), gabs(lumR - lumC));
    const float gate = smoothstep_(P.dot_crawl_edge_thresh, P.dot_crawl_edge_thresh * 3.0f, grad);
    const float linePhase = lineY * 3.14159265f;
    const float framePhase = (float)P.frame_index * (3.14159265f * 0.5f);
    const float hPhase = pixX * P.dot_crawl_subcarrier * 2.0f * 3.14159265f;
    const float sub = rcx_sinf(hPhase + linePhase + framePhase);
    const float I = sub * P.dot_crawl_intensity * gate;
    const float Q = rcx_cosf(hPhase + linePhase + framePhase) * P.dot_crawl_intensity * gate * 0.5f;
    const V3 cont = v3(1.0000f * I + 0.9562f * Q, -0.2721f * I - 0.6474f * Q, -1.1069f * I + 1.7046f * Q);
    return gclamp3(col + cont, 0.0f, 1.0f);
}

// p12_dropout.frag: tape dropouts (horizontal streaks replaced by displaced
// picture), in bursts per one-second window
DI float burst_activity(uint32_t vf, const rc_vhs_params& P) {
    const uint32_t window = vf / 30u, prevWin = window - 1u;
    const float thr = 1.0f - P.dropout_burst_rate;
    const float thisActive = step_(thr, fhash12(window, 0xDEADBEEFu));
    const float prevActive = step_(thr, fhash12(prevWin, 0xDEADBEEFu));
    const float windowPos = (float)(vf % 30u) / (float)30u;
    const float bleed = prevActive * smoothstep_(0.7f, 1.0f, 1.0f - windowPos);
    return gmax(thisActive, bleed);
}
DI V3 p12(const Tex& t, const Frag& f, const rc_vhs_params& P) {
    const float rx = (float)t.w, ry = (float)t.h;
    const V3 col = tex(t, f.u, f.v);
    const float fragX = f.u * rx, fragY = floorf(f.v * ry);
    const uint32_t vf = (uint32_t)(P.frame_index / 2);
    const float activity = burst_activity(vf, P);
    if (activity < 0.001f) return col;
    const float ageFactor = 0.05f + P.tape_age * 0.95f;
    const int nEvents = 1 + (int)roundf(activity * ageFactor * (float)(14 - 1));
    float bestWeight = 0.0f, bestBurst = 0.0f;
    float bu = f.u, bv = f.v;
    for (int i = 0; i < nEvents; i++) {
        const uint32_t si = (uint32_t)i;
        const float evY = floorf(fhash12(vf * 31u + si, si * 13u + 1u) * ry);
        const int evH = (fhash12(vf + si * 3u, si + 77u) > 0.88f) ? 2 : 1;
        if (fragY < evY || fragY >= evY + (float)evH) continue;
        const float wr = fhash12(vf * 7u + si, si * 7u + 2u);
        float evWidth;
        if (fhash12(vf * 2u + si, si + 55u) > 0.88f)
            evWidth = 80.0f + wr * 140.0f;
        else
            evWidth = 8.0f + wr * wr * 32.0f;
        const float maxStart = gmax(0.0f, rx - evWidth);
        const float evX = fhash12(vf * 5u + si, si * 7u + 3u) * maxStart;
        if (fragX < evX || fragX >= evX + evWidth) continue;
        const float dLeft = fragX - evX;
        const float dRight = (evX + evWidth) - fragX;
        const float weight = smoothstep_(0.0f, 1.5f, dLeft) * smoothstep_(0.0f, 5.0f, dRight);
        const float dxNorm = fhash12(vf * 11u + si, si * 7u + 4u) * 2.0f - 1.0f;
        const float dx = dxNorm * (4.0f + P.tape_age * 16.0f);
        const float dyRnd = fhash12(vf * 13u + si, si * 7u + 5u);
        const float dy = (dyRnd > 0.6f) ? (dyRnd > 0.8f ? -1.0f : 1.0f) : 0.0f;
        const float stretchR = fhash12(vf * 17u + si, si * 7u + 6u);
        const float stretch = (stretchR > 0.7f) ? (1.0f + stretchR * P.tape_age * 0.5f) : 1.0f;
        const float centreX = evX + evWidth * 0.5f;
        const float stretchedX = centreX + (fragX - centreX) * stretch + dx;
        const float du = gclamp(stretchedX / rx, 0.0f, 1.0f), dv = gclamp((fragY + dy) / ry, 0.0f, 1.0f);
        const float burstFade = smoothstep_(3.0f, 0.0f, dLeft) * P.dropout_bright;
        if (weight > bestWeight) {
            bestWeight = weight;
            bu = du;
            bv = dv;
            bestBurst = burstFade;
        }
        break;
    }
    if (bestWeight < 0.001f) return col;
    V3 rep = tex(t, bu, bv);
    rep = rep * (1.0f + bestBurst * 0.3f);
    const float lumR = dot3(rep, v3(0.2126f, 0.7152f, 0.0722f));
    rep = mix3(rep, v3(lumR, lumR, lumR), bestBurst * 0.4f);
    return mix3(col, rep, bestWeight);
}

// p13_headswitch.frag: jitter, luma ripple and chroma rotation on the
// bottom scanlines
DI float noise13(float x, uint32_t seed) {
    const float i = floorf(x), fr = fract_(x);
    const float u = fr * fr * (3.0f - 2.0f * fr);
    const float a = fhash2((uint32_t)i, seed), b = fhash2((uint32_t)i + 1u, seed);
    return mix_(a, b, u) * 2.0f - 1.0f;
}
DI V3 p13(const Tex& t, const Frag& f, const rc_vhs_params& P) {
    const float sx = (float)t.w, sy = (float)t.h;
    const float dist = floorf(f.v * sy);
    const float zone = (float)P.head_switch_lines;
    if (dist >= zone) return tex(t, f.u, f.v);
    const float prox = 1.0f - (dist / zone);
    const float settle = prox * prox;
    const uint32_t seed = (uint32_t)P.frame_index;
    const float scanNoise = noise13(dist * 0.8f, seed);
    const float fastNoise = noise13(dist * 3.0f, seed + 7u);
    const float jitterPx = P.head_switch_jitter * settle * (scanNoise * 0.7f + fastNoise * 0.3f);
    const float uvOffset = jitterPx / sx;
    const float su = gclamp(f.u + uvOffset, 0.0f, 1.0f);
    const float phaseRand = fhash2(seed, 0xCAFEBABEu) * 6.283185f;
    const float rippleSin = rcx_sinf(dist * 1.570796f + phaseRand);
    const float ripple = P.head_switch_ripple * settle * rippleSin;
    const float chromaSign = (fhash2(seed, 0xBEEFu) > 0.5f) ? 1.0f : -1.0f;
    const float chromaAngle = P.head_switch_chroma * settle * chromaSign;
    V3 ycc = ycc5(tex(t, su, f.v));
    ycc.x += ripple;
    const V2 cbcr = rotate_cbcr(V2{ycc.y - 0.5f, ycc.z - 0.5f}, chromaAngle);
    ycc.y = cbcr.x + 0.5f;
    ycc.z = cbcr.y + 0.5f;
    return rgb5(ycc);
}

// p14_tracking.frag: tracking-error bands (displacement, fringe colour,
// guard-band noise) from up to two events per one-second epoch
DI float noise14(float x, uint32_t seed) {
    const float i = floorf(x), fr = fract_(x);
    const float u2 = fr * fr * (3.0f - 2.0f * fr);
    return mix_(fhash2((uint32_t)i, seed), fhash2((uint32_t)i + 1u, seed), u2);
}
DI V3 p14(const Tex& t, const Frag& f, const rc_vhs_params& P) {
    const float sx = (float)t.w, sy = (float)t.h;
    const float fragY = floorf(f.v * sy);
    const V3 col = tex(t, f.u, f.v);
    if (P.tracking_severity < 0.001f) return col;
    const uint32_t curEpoch = (uint32_t)P.frame_index / 30u;
    float disp = 0.0f, fringe = 0.0f, noise = 0.0f, hue = 0.0f, weight = 0.0f;
    for (int e = 0; e < 2; e++) {
        const uint32_t ei = (uint32_t)e;
        for (int ep = 0; ep < 3; ep++) {
            const uint32_t epoch = curEpoch - (uint32_t)ep;
            const float spawnChance = 0.08f + 0.62f * P.tracking_severity;
            const float spawnRnd = fhash2(epoch * 7919u + ei * 3u, 0xDEADBEEFu);
            if (spawnRnd > spawnChance) continue;
            const float durRnd = fhash2(epoch * 1009u + ei, 0xCAFEu);
            const uint32_t evDuration = (uint32_t)(15.0f + durRnd * 105.0f);
            const float startRnd = fhash2(epoch * 503u + ei, 0xBEEFu);
            const uint32_t evStart = epoch * 30u + (uint32_t)(startRnd * (float)30);
            const uint32_t evEnd = evStart + evDuration;
            const uint32_t frame = (uint32_t)P.frame_index;
            if (frame < evStart || frame >= evEnd) continue;
            const float yRnd = fhash2(epoch * 2017u + ei, 0x1111u);
            const float hRnd = fhash2(epoch * 3001u + ei, 0x2222u);
            const float evHeight = 20.0f + hRnd * 60.0f * P.tracking_severity;
            const float evY0 = yRnd * (sy - evHeight);
            const float evY1 = evY0 + evHeight;
            if (fragY < evY0 || fragY >= evY1) continue;
            const float bandT = (fragY - evY0) / gmax(evHeight - 1.0f, 1.0f);
            const float dirSign = (fhash2(epoch * 4003u + ei, 0x3333u) > 0.5f) ? 1.0f : -1.0f;
            const float baseDisp = dirSign * P.tracking_max_displace_px * P.tracking_severity * (bandT - 0.5f) * 2.0f;
            const float framePhase = (float)frame * 0.37f + (float)ei * 1.57f;
            const float wobble =
                rcx_sinf(bandT * 6.28318f + framePhase) * P.tracking_max_displace_px * 0.20f * P.tracking_severity;
            const float micro = (noise14(fragY * 0.25f, frame + ei * 17u) * 2.0f - 1.0f) * 2.5f * P.tracking_severity;
            const float totalPx = baseDisp + wobble + micro;
            const float distTop = fragY - evY0, distBottom = evY1 - fragY;
            const float edgeWeight = smoothstep_(0.0f, 1.5f, distTop) * smoothstep_(0.0f, 4.0f, distBottom);
            const float edgeDist = gmin(distTop, distBottom);
            const float fringeAmt = (1.0f - smoothstep_(0.0f, P.tracking_fringe_width_px, edgeDist)) * edgeWeight;
            const float noiseAmt = fringeAmt * 0.7f;
            const float hueAngle = dirSign * 0.436f * P.tracking_severity * (1.0f - fringeAmt);
            if (edgeWeight > weight) {
                weight = edgeWeight;
                disp = totalPx;
                fringe = fringeAmt;
                noise = noiseAmt;
                hue = hueAngle;
            }
        }
    }
    if (weight < 0.001f) return col;
    const float uvShift = (disp / sx) * weight;
    V3 ycc = ycc5(tex(t, gclamp(f.u + uvShift, 0.0f, 1.0f), f.v));
    if (gabs(hue) > 0.001f) {
        const V2 cbcr = rotate_cbcr(V2{ycc.y - 0.5f, ycc.z - 0.5f}, hue);
        ycc.y = cbcr.x + 0.5f;
        ycc.z = cbcr.y + 0.5f;
    }
    if (fringe > 0.001f) {
        const float fringePhase = (float)P.frame_index * 0.12f + f.v * 8.0f;
        const float fringeAngle = rcx_sinf(fringePhase) * 0.9f;
        V2 fc = rotate_cbcr(V2{ycc.y - 0.5f, ycc.z - 0.5f}, fringeAngle);
        const float s = 1.0f + fringe * 1.2f;
        fc = V2{fc.x * s, fc.y * s};
        ycc.y = mix_(ycc.y, fc.x + 0.5f, fringe);
        ycc.z = mix_(ycc.z, fc.y + 0.5f, fringe);
        const uint32_t nSeed = uhash2((uint32_t)fragY * 1619u ^ (uint32_t)P.frame_index * 2654435761u);
        const float buzz = ((float)uhash2(nSeed ^ (uint32_t)(f.fx * 37.0f)) / 4294967295.0f) * 2.0f - 1.0f;
        ycc.x += buzz * 0.15f * noise;
    }
    return mix3(col, rgb5(ycc), weight);
}

// p15_edge_enhance.frag: cored unsharp mask on luma (5x5 binomial blur)
DI V3 p15(const Tex& t, const Frag& f, const rc_vhs_params& P) {
    const float px = 1.0f / (float)t.w, py = 1.0f / (float)t.h;
    V3 ycc = ycc5(tex(t, f.u, f.v));
    const float Y = ycc.x;
    const float w[5] = {0.0625f, 0.25f, 0.375f, 0.25f, 0.0625f};
    float blur = 0.0f;
    for (int dy = -2; dy <= 2; dy++)
        for (int dx = -2; dx <= 2; dx++) {
            const float sY = ycc5(tex(t, f.u + (float)dx * px, f.v + (float)dy * py)).x;
            blur += sY * w[dx + 2] * w[dy + 2];
        }
    float detail = Y - blur;
    const float core = smoothstep_(P.edge_enhance_core_threshold * 0.5f, P.edge_enhance_core_threshold, gabs(detail));
    detail *= core;
    ycc.x = Y + P.edge_enhance_amount * detail;
    return rgb5(ycc);
}

// p16_interlace.frag: field offset, combing on vertical edges, line weighting
DI V3 p16(const Tex& t, const Frag& f, const rc_vhs_params& P) {
    const float px = 1.0f / (float)t.w, py = 1.0f / (float)t.h;
    const int fragY = (int)floorf(f.v * (float)t.h);
    const bool even = (fragY & 1) == 0;
    const float vertShift = even ? (+P.interlace_field_offset_px * 0.5f * py) : (-P.interlace_field_offset_px * 0.5f * py);
    const V3 cHere = tex(t, f.u, f.v);
    const V3 cAbove = tex(t, f.u, f.v - py);
    const V3 cBelow = tex(t, f.u, f.v + py);
    const V3 cLeft = tex(t, f.u - px, f.v);
    const V3 LUM = v3(0.299f, 0.587f, 0.114f);
    const float yHere = dot3(cHere, LUM), yAbove = dot3(cAbove, LUM), yBelow = dot3(cBelow, LUM);
    const float yLeft = dot3(cLeft, LUM);
    const float vertGrad = gabs(yAbove - yBelow);
    const float hDir = sign_(yHere - yLeft);
    float comb = 0.0f;
    if (even) {
        const float ew = smoothstep_(P.interlace_comb_edge_thresh, P.interlace_comb_edge_thresh * 3.0f, vertGrad);
        comb = hDir * ew * P.interlace_comb_strength;
    }
    const float su = gclamp(f.u + comb * px, 0.0f, 1.0f), sv = gclamp(f.v + vertShift, 0.0f, 1.0f);
    const V3 col = tex(t, su, sv);
    return col * (even ? (1.0f - P.interlace_line_weighting) : (1.0f + P.interlace_line_weighting * 0.5f));
}

// ---------------------------------------------------------------------------
// kernel and launch
// ---------------------------------------------------------------------------
struct VhsArgs {
    const float4* in;
    float4* out;
    int w, h;
    int pass;
    rc_vhs_params p;
};

// One instantiation per pass, so each pass gets the registers it needs
// (the multi-tap passes bound the occupancy of a single switch kernel).
template <int K>
__global__ void __launch_bounds__(128) vhs_pass_kernel(VhsArgs A) {
    __shared__ float wtab[kWeightTaps];
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (K == 1 || K == 2 || K == 8) {
        fill_weights(K, A.p, wtab);
        __syncthreads();
    }
    if (x >= A.w) return;
    const Tex t{A.in, A.w, A.h};
    const Frag f{((float)x + 0.5f) / (float)A.w, ((float)y + 0.5f) / (float)A.h, (float)x + 0.5f, (float)y + 0.5f};
    V3 c;
    if (K == 1) c = p01(t, f, A.p, wtab);
    else if (K == 2) c = p02(t, f, A.p, wtab);
    else if (K == 3) c = p03(t, f, A.p);
    else if (K == 4) c = p04(t, f, A.p);
    else if (K == 7) c = p07(t, f, A.p);
    else if (K == 8) c = p08(t, f, A.p, wtab);
    else if (K == 9) c = p09(t, f, A.p);
    else if (K == 10) c = p10(t, f, A.p);
    else if (K == 11) c = p11(t, f, A.p);
    else if (K == 12) c = p12(t, f, A.p);
    else if (K == 13) c = p13(t, f, A.p);
    else if (K == 14) c = p14(t, f, A.p);
    else if (K == 15) c = p15(t, f, A.p);
    else c = p16(t, f, A.p);
    A.out[(size_t)y * A.w + x] = make_float4(c.x, c.y, c.z, 1.0f);
}

bool has_pass(int pass) { return pass >= 1 && pass <= 16 && pass != 5 && pass != 6; }

cudaError_t launch_pass(int pass, const float4* in, float4* out, int w, int h, const rc_vhs_params& p,
                        cudaStream_t s) {
    VhsArgs A{in, out, w, h, pass, p};
    const dim3 grid((w + 127) / 128, h);
    switch (pass) {
        case 1: vhs_pass_kernel<1><<<grid, 128, 0, s>>>(A); break;
        case 2: vhs_pass_kernel<2><<<grid, 128, 0, s>>>(A); break;
        case 3: vhs_pass_kernel<3><<<grid, 128, 0, s>>>(A); break;
        case 4: vhs_pass_kernel<4><<<grid, 128, 0, s>>>(A); break;
        case 7: vhs_pass_kernel<7><<<grid, 128, 0, s>>>(A); break;
        case 8: vhs_pass_kernel<8><<<grid, 128, 0, s>>>(A); break;
        case 9: vhs_pass_kernel<9><<<grid, 128, 0, s>>>(A); break;
        case 10: vhs_pass_kernel<10><<<grid, 128, 0, s>>>(A); break;
        case 11: vhs_pass_kernel<11><<<grid, 128, 0, s>>>(A); break;
        case 12: vhs_pass_kernel<12><<<grid, 128, 0, s>>>(A); break;
        case 13: vhs_pass_kernel<13><<<grid, 128, 0, s>>>(A); break;
        case 14: vhs_pass_kernel<14><<<grid, 128, 0, s>>>(A); break;
        case 15: vhs_pass_kernel<15><<<grid, 128, 0, s>>>(A); break;
        case 16: vhs_pass_kernel<16><<<grid, 128, 0, s>>>(A); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace vhs
}  // namespace rc

extern "C" {

void rc_vhs_defaults(rc_vhs_params* p) {
    if (!p) return;
    rc_vhs_params d{};
    d.enabled = 0;
    d.frame_index = 0;
    d.time_s = 0.0f;
    d.agc_gain = 1.0f;
    d.luma_blur_sigma = 1.5f;
    d.chroma_res_sigma = 7.0f;
    d.color_temp_bias = 0.0f;
    d.color_hue_rot = 0.0f;
    d.color_saturation = 0.95f;
    d.color_drift_speed = 0.05f;
    d.dr_black_lift = 0.01f;
    d.dr_shadow_crush = 0.03f;
    d.dr_highlight_knee = 0.78f;
    d.dr_highlight_clip = 0.95f;
    d.ccd_noise_luma_base = 0.015f;
    d.ccd_noise_chroma_scale = 1.6f;
    d.ccd_smear_threshold = 0.85f;
    d.ccd_smear_intensity = 0.009f;
    d.ccd_smear_length = 20;
    d.chroma_bleed_factor = 0.35f;
    d.timebase_amplitude_px = 1.5f;
    d.timebase_freq = 0.02f;
    d.timebase_speed = 0.70f;
    d.dot_crawl_intensity = 0.25f;
    d.dot_crawl_subcarrier = 0.14f;
    d.dot_crawl_edge_thresh = 0.04f;
    d.tape_age = 0.3f;
    d.dropout_bright = 0.92f;
    d.dropout_burst_rate = 0.45f;
    d.head_switch_lines = 12;
    d.head_switch_jitter = 4.0f;
    d.head_switch_ripple = 0.10f;
    d.head_switch_chroma = 0.35f;
    d.tracking_severity = 0.1f;
    d.tracking_max_displace_px = 28.0f;
    d.tracking_fringe_width_px = 4.0f;
    d.edge_enhance_amount = 1.5f;
    d.edge_enhance_core_threshold = 0.025f;
    d.interlace_field_offset_px = 0.5f;
    d.interlace_comb_strength = 1.5f;
    d.interlace_comb_edge_thresh = 0.04f;
    d.interlace_line_weighting = 0.05f;
    *p = d;
}

int rc_vhs_pass(int pass, const void* in_rgba, void* out_rgba, int w, int h, const rc_vhs_params* p, void* stream) {
    if (!rc::vhs::has_pass(pass) || !in_rgba || !out_rgba || !p || w <= 0 || h <= 0 || w > 16384 || h > 16384 ||
        in_rgba == out_rgba || !rc::aligned_to(in_rgba, 16) || !rc::aligned_to(out_rgba, 16))
        return RC_ERR_INVALID_ARG;
    return rc::vhs::launch_pass(pass, static_cast<const float4*>(in_rgba), static_cast<float4*>(out_rgba), w, h, *p,
                                static_cast<cudaStream_t>(stream)) == cudaSuccess
               ? RC_OK
               : RC_ERR_CUDA;
}

}  // extern "C"
