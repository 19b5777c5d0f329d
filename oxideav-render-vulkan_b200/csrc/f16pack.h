// f32 -> f16 bits for the RGBA16F atlas (f32_to_f16, src/scene.rs:242-272):
// round to nearest even, overflow to infinity, subnormals, NaN kept quiet.
// Integer arithmetic only, shared by the host preparation and the device
// atlas builder so both write the same halfs.
#pragma once

#include "fmath.h"

FM_FN uint16_t fm_f32_to_f16(float v) {
    uint32_t bits = fm_bits(v);
    uint16_t sign = (uint16_t)((bits >> 16) & 0x8000u);
    int32_t exp = (int32_t)((bits >> 23) & 0xffu);
    uint32_t mant = bits & 0x007fffffu;
    if (exp == 0xff) return (uint16_t)(sign | 0x7c00u | (mant ? 0x200u : 0u));
    int32_t e = exp - 127 + 15;
    if (e >= 0x1f) return (uint16_t)(sign | 0x7c00u);
    if (e <= 0) {
        if (e < -10) return sign;
        uint32_t m = mant | 0x00800000u;
        uint32_t shift = (uint32_t)(14 - e);
        uint32_t half = m >> shift;
        uint32_t rem = m & ((1u << shift) - 1u);
        uint32_t mid = 1u << (shift - 1u);
        int round = rem > mid || (rem == mid && (half & 1u));
        return (uint16_t)(sign | (half + (round ? 1u : 0u)));
    }
    uint32_t half = ((uint32_t)e << 10) | (mant >> 13);
    uint32_t rem = mant & 0x1fffu;
    int round = rem > 0x1000u || (rem == 0x1000u && (half & 1u));
    return (uint16_t)(sign | (half + (round ? 1u : 0u)));
}

// sRGB-encoded channel to linear (the decode the texture crate applies to
// sRGB slots before building mips), with the portable pow so host and
// device agree to the bit.
FM_FN float fm_srgb_decode(float c) {
    if (c <= 0.04045f) return c / 12.92f;
    return fm_pow((c + 0.055f) / 1.055f, 2.4f);
}
