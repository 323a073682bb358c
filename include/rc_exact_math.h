/*
 * rc_exact_math.h -- deterministic transcendental functions shared by the
 * CPU oracle and the "exact" build of the CUDA kernels.
 *
 * The GLSL 4.30 specification leaves the precision of sin, cos, exp, log and
 * pow to the implementation, so the reference shaders have no single
 * bit-level answer for them.  This header fixes one: every function takes a
 * float, evaluates in IEEE double with a fixed sequence of +,-,*,/ (no fused
 * multiply-add, which both compilers are told to avoid), and rounds once to
 * float.  Because IEEE double arithmetic is reproducible, the host build and
 * the sm_100a build return identical bits, and the result is the correctly
 * rounded float in all but vanishingly rare double-rounding cases.
 *
 * Methods (published, restated here from the mathematics):
 *   - sin/cos: Cody & Waite (1980) additive range reduction by pi/2 with a
 *     three-part split of pi/2 (each part holds 33 significant bits, so
 *     k * part is exact for |k| < 2^20), then the Taylor series of sin and
 *     cos on |r| <= pi/4 evaluated by Horner's rule.
 *   - exp: reduction x = k*ln2 + r with a three-part split of ln2, Taylor
 *     series of e^r on |r| <= ln2/2, scaling by an exactly built 2^k.
 *   - log: x = m * 2^e with m in [sqrt(1/2), sqrt(2)), log m = 2 atanh(s),
 *     s = (m-1)/(m+1), by its odd power series.
 *   - pow(x, y) = exp(y * log x) with both halves kept in double.
 * The split constants were derived from 200-digit expansions of pi and ln 2
 * by rounding to 33 significant bits, taking the remainder, and repeating.
 */
#ifndef RC_EXACT_MATH_H
#define RC_EXACT_MATH_H

#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define RCX_FN __host__ __device__ __forceinline__
#else
#define RCX_FN static inline
#endif

/* Bit casts that work on both sides. */
RCX_FN uint64_t rcx_dbits(double d) {
#if defined(__CUDA_ARCH__)
    return (uint64_t)__double_as_longlong(d);
#else
    uint64_t u; memcpy(&u, &d, 8); return u;
#endif
}
RCX_FN double rcx_bitsd(uint64_t u) {
#if defined(__CUDA_ARCH__)
    return __longlong_as_double((long long)u);
#else
    double d; memcpy(&d, &u, 8); return d;
#endif
}
RCX_FN uint32_t rcx_fbits(float f) {
#if defined(__CUDA_ARCH__)
    return (uint32_t)__float_as_uint(f);
#else
    uint32_t u; memcpy(&u, &f, 4); return u;
#endif
}
RCX_FN float rcx_bitsf(uint32_t u) {
#if defined(__CUDA_ARCH__)
    return __uint_as_float(u);
#else
    float f; memcpy(&f, &u, 4); return f;
#endif
}

/* floor(x + 0.5) in double: rounds half up; deterministic on both sides. */
RCX_FN double rcx_round_half_up(double x) {
#if defined(__CUDA_ARCH__)
    return floor(x + 0.5);
#else
    return __builtin_floor(x + 0.5);
#endif
}

/* 2^k as a double for -1022 <= k <= 1023, built from its bits. */
RCX_FN double rcx_pow2i(int k) {
    return rcx_bitsd((uint64_t)(k + 1023) << 52);
}

/* pi/2 = RCX_PIO2_A + RCX_PIO2_B + RCX_PIO2_C (33 + 33 + 53 bits). */
#define RCX_PIO2_A 0x1.921fb54400000p+0
#define RCX_PIO2_B 0x1.0b4611a600000p-34
#define RCX_PIO2_C 0x1.3198a2e037073p-69
#define RCX_TWO_OVER_PI 0x1.45f306dc9c883p-1
/* ln 2 = RCX_LN2_A + RCX_LN2_B + RCX_LN2_C. */
#define RCX_LN2_A 0x1.62e42ff000000p-1
#define RCX_LN2_B (-0x1.718432a200000p-35)
#define RCX_LN2_C 0x1.3c7673007e5edp-69
#define RCX_LOG2E 0x1.71547652b82fep+0
#define RCX_LN2 0x1.62e42fefa39efp-1

/* Taylor series of sin(r) and cos(r), |r| <= pi/4, terms through r^21/r^22
 * (the first omitted term is below 1e-22 relative). Coefficients are
 * (-1)^k / (2k+1)! and (-1)^k / (2k)! as doubles. */
RCX_FN double rcx_sin_poly(double r) {
    const double r2 = r * r;
    double p = -1.0 / 51090942171709440000.0;          /* -1/21! */
    p = p * r2 + 1.0 / 121645100408832000.0;           /* 1/19! */
    p = p * r2 - 1.0 / 355687428096000.0;              /* 1/17! */
    p = p * r2 + 1.0 / 1307674368000.0;                /* 1/15! */
    p = p * r2 - 1.0 / 6227020800.0;                   /* 1/13! */
    p = p * r2 + 1.0 / 39916800.0;                     /* 1/11! */
    p = p * r2 - 1.0 / 362880.0;                       /* 1/9!  */
    p = p * r2 + 1.0 / 5040.0;                         /* 1/7!  */
    p = p * r2 - 1.0 / 120.0;                          /* 1/5!  */
    p = p * r2 + 1.0 / 6.0;                            /* 1/3!  */
    /* sin r = r - r^3 p' ... written as r - r*r2*(1/6 - ...) */
    return r - (r * r2) * p;
}
RCX_FN double rcx_cos_poly(double r) {
    const double r2 = r * r;
    double p = 1.0 / 1124000727777607680000.0;         /* 1/22! */
    p = p * r2 - 1.0 / 2432902008176640000.0;          /* 1/20! */
    p = p * r2 + 1.0 / 6402373705728000.0;             /* 1/18! */
    p = p * r2 - 1.0 / 20922789888000.0;               /* 1/16! */
    p = p * r2 + 1.0 / 87178291200.0;                  /* 1/14! */
    p = p * r2 - 1.0 / 479001600.0;                    /* 1/12! */
    p = p * r2 + 1.0 / 3628800.0;                      /* 1/10! */
    p = p * r2 - 1.0 / 40320.0;                        /* 1/8!  */
    p = p * r2 + 1.0 / 720.0;                          /* 1/6!  */
    p = p * r2 - 1.0 / 24.0;                           /* 1/4!  */
    p = p * r2 + 0.5;                                  /* 1/2!  */
    return 1.0 - r2 * p;
}

/* Reduce x by k*(pi/2); returns r and the quadrant k mod 4. */
RCX_FN double rcx_reduce_pio2(double x, int* quadrant) {
    const double k = rcx_round_half_up(x * RCX_TWO_OVER_PI);
    double r = x - k * RCX_PIO2_A;
    r = r - k * RCX_PIO2_B;
    r = r - k * RCX_PIO2_C;
    const long long ki = (long long)k;
    *quadrant = (int)(ki & 3);
    return r;
}

RCX_FN float rcx_sinf(float xf) {
    if (xf != xf) return xf;
    if (rcx_fbits(xf) << 1 == 0xff000000u) return rcx_bitsf(0x7fc00000u); /* +-inf */
    int q;
    const double r = rcx_reduce_pio2((double)xf, &q);
    double v;
    switch (q) {
        case 0: v = rcx_sin_poly(r); break;
        case 1: v = rcx_cos_poly(r); break;
        case 2: v = -rcx_sin_poly(r); break;
        default: v = -rcx_cos_poly(r); break;
    }
    return (float)v;
}

RCX_FN float rcx_cosf(float xf) {
    if (xf != xf) return xf;
    if (rcx_fbits(xf) << 1 == 0xff000000u) return rcx_bitsf(0x7fc00000u);
    int q;
    const double r = rcx_reduce_pio2((double)xf, &q);
    double v;
    switch (q) {
        case 0: v = rcx_cos_poly(r); break;
        case 1: v = -rcx_sin_poly(r); break;
        case 2: v = -rcx_cos_poly(r); break;
        default: v = rcx_sin_poly(r); break;
    }
    return (float)v;
}

/* e^x in double for finite x; overflow -> +inf, deep underflow -> 0. */
RCX_FN double rcx_exp_d(double x) {
    if (x != x) return x;
    if (x > 709.0) return rcx_bitsd(0x7ff0000000000000ull);
    if (x < -745.0) return 0.0;
    const double k = rcx_round_half_up(x * RCX_LOG2E);
    double r = x - k * RCX_LN2_A;
    r = r - k * RCX_LN2_B;
    r = r - k * RCX_LN2_C;
    /* Taylor series of e^r, |r| <= 0.3466, through r^14/14!. */
    double p = 1.0 / 87178291200.0;                    /* 1/14! */
    p = p * r + 1.0 / 6227020800.0;                    /* 1/13! */
    p = p * r + 1.0 / 479001600.0;                     /* 1/12! */
    p = p * r + 1.0 / 39916800.0;                      /* 1/11! */
    p = p * r + 1.0 / 3628800.0;                       /* 1/10! */
    p = p * r + 1.0 / 362880.0;                        /* 1/9!  */
    p = p * r + 1.0 / 40320.0;                         /* 1/8!  */
    p = p * r + 1.0 / 5040.0;                          /* 1/7!  */
    p = p * r + 1.0 / 720.0;                           /* 1/6!  */
    p = p * r + 1.0 / 120.0;                           /* 1/5!  */
    p = p * r + 1.0 / 24.0;                            /* 1/4!  */
    p = p * r + 1.0 / 6.0;                             /* 1/3!  */
    p = p * r + 0.5;                                   /* 1/2!  */
    p = p * r + 1.0;
    p = p * r + 1.0;
    int ki = (int)k;
    /* Split 2^k in two factors so that both stay normal doubles. */
    const int k1 = ki / 2;
    const int k2 = ki - k1;
    return (p * rcx_pow2i(k1)) * rcx_pow2i(k2);
}

/* Natural log of a positive finite float, evaluated in double. */
RCX_FN double rcx_log_d(float xf) {
    uint32_t u = rcx_fbits(xf);
    if (xf != xf) return (double)xf;
    if (u == 0u || u == 0x80000000u) return -rcx_bitsd(0x7ff0000000000000ull); /* log(+-0) = -inf */
    if (u & 0x80000000u) return rcx_bitsd(0x7ff8000000000000ull);            /* x < 0 -> NaN */
    if (u == 0x7f800000u) return rcx_bitsd(0x7ff0000000000000ull);           /* log(inf) = inf */
    int e;
    double m;
    if ((u >> 23) == 0) {
        /* Subnormal float: exact in double; normalise by hand. */
        double d = (double)xf * 0x1p52;                /* exact scaling */
        uint64_t b = rcx_dbits(d);
        e = (int)((b >> 52) & 0x7ff) - 1023 - 52;
        m = rcx_bitsd((b & 0x000fffffffffffffull) | 0x3ff0000000000000ull);
    } else {
        e = (int)(u >> 23) - 127;
        m = (double)rcx_bitsf((u & 0x007fffffu) | 0x3f800000u);
    }
    if (m > 1.4142135623730951) { m = m * 0.5; e = e + 1; }
    const double s = (m - 1.0) / (m + 1.0);
    const double s2 = s * s;
    /* 2 atanh(s) = 2 (s + s^3/3 + ... + s^23/23); |s| <= 0.1716. */
    double p = 1.0 / 23.0;
    p = p * s2 + 1.0 / 21.0;
    p = p * s2 + 1.0 / 19.0;
    p = p * s2 + 1.0 / 17.0;
    p = p * s2 + 1.0 / 15.0;
    p = p * s2 + 1.0 / 13.0;
    p = p * s2 + 1.0 / 11.0;
    p = p * s2 + 1.0 / 9.0;
    p = p * s2 + 1.0 / 7.0;
    p = p * s2 + 1.0 / 5.0;
    p = p * s2 + 1.0 / 3.0;
    const double logm = 2.0 * s + (2.0 * s) * (s2 * p);
    const double ed = (double)e;
    return (ed * RCX_LN2_A + logm) + ed * (RCX_LN2_B + RCX_LN2_C);
}

RCX_FN float rcx_expf(float x) { return (float)rcx_exp_d((double)x); }

RCX_FN float rcx_logf(float x) { return (float)rcx_log_d(x); }

/* GLSL pow(x, y): results for x < 0 are undefined in GLSL; here NaN.
 * y == 0 gives 1; x == 0 gives 0 for y > 0 and +inf for y < 0. */
RCX_FN float rcx_powf(float x, float y) {
    if (y == 0.0f) return 1.0f;
    if (x == 1.0f) return 1.0f;
    if (x != x || y != y) return x + y;
    if (x == 0.0f) return (y > 0.0f) ? 0.0f : rcx_bitsf(0x7f800000u);
    if (x < 0.0f) return rcx_bitsf(0x7fc00000u);
    const double t = (double)y * rcx_log_d(x);
    return (float)rcx_exp_d(t);
}

#endif /* RC_EXACT_MATH_H */
