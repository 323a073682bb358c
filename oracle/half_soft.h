/*
 * half_soft.h -- TEST INFRASTRUCTURE (oracle). IEEE 754 binary16 conversion in
 * portable integer code, used where the reference stores rgba16f images
 * (core/Renderer.java:163-183: G-buffer and albedo textures).
 * float -> half rounds to nearest, ties to even, with subnormals, overflow to
 * infinity and NaN preserved; half -> float is exact.
 */
#ifndef RC_HALF_SOFT_H
#define RC_HALF_SOFT_H

#include <stdint.h>
#include <string.h>

static inline uint16_t float_to_half_rne(float f) {
    uint32_t x;
    memcpy(&x, &f, 4);
    const uint32_t sign = (x >> 16) & 0x8000u;
    const uint32_t absx = x & 0x7fffffffu;
    if (absx >= 0x7f800000u) {                       /* inf or NaN */
        return (uint16_t)(sign | 0x7c00u | (absx > 0x7f800000u ? 0x200u | ((absx >> 13) & 0x3ffu) : 0u));
    }
    if (absx >= 0x477ff000u) return (uint16_t)(sign | 0x7c00u); /* rounds past 65504 */
    if (absx >= 0x38800000u) {                       /* normal half range */
        uint32_t mant = absx & 0x7fffffu;
        uint32_t exp = (absx >> 23) - 127 + 15;
        uint32_t h = (exp << 10) | (mant >> 13);
        const uint32_t rem = mant & 0x1fffu;
        if (rem > 0x1000u || (rem == 0x1000u && (h & 1u))) h += 1u; /* carry may bump exponent: correct */
        return (uint16_t)(sign | h);
    }
    if (absx < 0x33000000u) return (uint16_t)sign;   /* below half of the smallest subnormal */
    /* Subnormal half: value = mant * 2^-24. */
    const uint32_t e = absx >> 23;                   /* biased float exponent, 102..112 */
    const uint32_t mant = (absx & 0x7fffffu) | 0x800000u;
    const uint32_t shift = 126u - e;                 /* 14..24 */
    uint32_t h = mant >> shift;
    const uint32_t rem = mant & ((1u << shift) - 1u);
    const uint32_t halfway = 1u << (shift - 1u);
    if (rem > halfway || (rem == halfway && (h & 1u))) h += 1u;
    return (uint16_t)(sign | h);
}

static inline float half_to_float(uint16_t h) {
    const uint32_t sign = ((uint32_t)h & 0x8000u) << 16;
    const uint32_t exp = ((uint32_t)h >> 10) & 0x1fu;
    uint32_t mant = (uint32_t)h & 0x3ffu;
    uint32_t x;
    if (exp == 0x1fu) {
        x = sign | 0x7f800000u | (mant << 13);
    } else if (exp != 0) {
        x = sign | ((exp - 15 + 127) << 23) | (mant << 13);
    } else if (mant == 0) {
        x = sign;
    } else {
        int e = -14;
        while ((mant & 0x400u) == 0) { mant <<= 1; e -= 1; }
        mant &= 0x3ffu;
        x = sign | ((uint32_t)(e + 127) << 23) | (mant << 13);
    }
    float f;
    memcpy(&f, &x, 4);
    return f;
}

#endif
