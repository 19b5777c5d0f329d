// Portable single-precision transcendentals for the path tracer.
//
// The estimator (pathtrace.wgsl: sample_vndf :951-969, cosine_hemisphere
// :1029-1047, d_charlie :984-991, triangle_solid_angle :1486-1497,
// sample_spherical_triangle :1510-1556, env_texel :1594-1603, env_sample
// :1627-1654, the medium term :1778 and :2014, cone_lod :473; resolve.wgsl
// srgb_to_linear / linear_to_srgb :38-50) calls sin, cos, acos, atan2, exp,
// log, log2 and pow. Every platform rounds those differently, so the CUDA
// tracer and the CPU oracle both evaluate them here, with nothing but IEEE
// +, -, *, /, sqrt and integer bit manipulation (build both sides without
// FMA contraction). The results are then bit-identical on host and device.
//
// Methods (all classical, coefficients are exact Taylor terms or exact
// splits of the constants):
//   * sin/cos: Cody & Waite (1980) argument reduction by pi/2 with a
//     three-part split of pi/2, Taylor polynomials on [-pi/4, pi/4].
//   * atan: reduction to |t| <= tan(pi/12) with the pi/6 addition formula
//     (Hart et al., "Computer Approximations", 1968), odd Taylor series.
//   * atan2: quadrant logic of C99 Annex F on top of atan.
//   * acos: acos(x) = 2 atan(sqrt((1 - x) / (1 + x))).
//   * exp / exp2: Cody & Waite reduction by ln 2 (two-part split), Taylor
//     polynomial, exponent scaling by exact powers of two.
//   * log / log2: mantissa in [sqrt(1/2), sqrt(2)), s = (m-1)/(m+1),
//     atanh series log(m) = 2 (s + s^3/3 + ...).
//   * pow: exp2(y * log2(x)) with the C99 special cases the tracer can meet.
// Accuracy is a few ulp (checked against float64 in the CPU test suite).
#pragma once

#include <stdint.h>
#include <string.h>
#include <math.h>

// Device code compiled with OXPT_FAST (the tolerance plan's second build
// of the shading kernels, with -use_fast_math) calls the CUDA library's
// functions instead: not bit-identical to the host, checked by image PSNR.
#if defined(__CUDA_ARCH__) && defined(OXPT_FAST)
#define FM_FAST 1
#endif

#if defined(__CUDACC__)
#define FM_FN static __host__ __device__ __forceinline__
#else
#define FM_FN static inline
#endif

FM_FN uint32_t fm_bits(float x) {
#if defined(__CUDA_ARCH__)
    return __float_as_uint(x);
#else
    uint32_t u;
    memcpy(&u, &x, 4);
    return u;
#endif
}

FM_FN float fm_float(uint32_t u) {
#if defined(__CUDA_ARCH__)
    return __uint_as_float(u);
#else
    float x;
    memcpy(&x, &u, 4);
    return x;
#endif
}

FM_FN int fm_isnan(float x) { return (fm_bits(x) & 0x7fffffffu) > 0x7f800000u; }
FM_FN int fm_isinf(float x) { return (fm_bits(x) & 0x7fffffffu) == 0x7f800000u; }
FM_FN int fm_finite(float x) { return (fm_bits(x) & 0x7f800000u) != 0x7f800000u; }
FM_FN float fm_abs(float x) { return fm_float(fm_bits(x) & 0x7fffffffu); }
FM_FN float fm_copysign(float m, float s) {
    return fm_float((fm_bits(m) & 0x7fffffffu) | (fm_bits(s) & 0x80000000u));
}
FM_FN float fm_nan(void) { return fm_float(0x7fc00000u); }

// 2^k for k in [-126, 127] (normal range only).
FM_FN float fm_pow2i(int k) { return fm_float((uint32_t)(k + 127) << 23); }

// x * 2^k with two exact steps so that results in the subnormal range
// round once, deterministically.
FM_FN float fm_ldexp(float x, int k) {
    if (k > 127) {
        x = x * fm_pow2i(127);
        k -= 127;
        if (k > 127) k = 127;
    } else if (k < -126) {
        x = x * fm_pow2i(-126);
        k += 126;
        if (k < -126) k = -126;
    }
    return x * fm_pow2i(k);
}

// Round to the nearest integer, halves away from zero (deterministic and
// independent of the rounding mode).
FM_FN float fm_round(float x) {
    float a = floorf(fm_abs(x) + 0.5f);
    return fm_copysign(a, x);
}

// ---------------------------------------------------------------------
// sin / cos.
// ---------------------------------------------------------------------

#define FM_PIO2_1 1.5703125f
#define FM_PIO2_2 4.837512969970703125e-4f
#define FM_PIO2_3 7.549790126404332e-08f
#define FM_2OPI 0.636619746685028076171875f

// sin(r), cos(r) for |r| <= pi/4.
FM_FN float fm_sin_poly(float r) {
    float z = r * r;
    float p = -1.0f / 5040.0f + z * (1.0f / 362880.0f);
    p = 1.0f / 120.0f + z * p;
    p = -1.0f / 6.0f + z * p;
    return r + (r * z) * p;
}

FM_FN float fm_cos_poly(float r) {
    float z = r * r;
    float p = 1.0f / 40320.0f + z * (-1.0f / 3628800.0f);
    p = -1.0f / 720.0f + z * p;
    p = 1.0f / 24.0f + z * p;
    p = -0.5f + z * p;
    return 1.0f + z * p;
}

// Reduce x to r in [-pi/4, pi/4] and the quadrant q = k mod 4.
FM_FN float fm_reduce_pio2(float x, int* q) {
    float k = fm_round(x * FM_2OPI);
    float r = ((x - k * FM_PIO2_1) - k * FM_PIO2_2) - k * FM_PIO2_3;
    // k mod 4 without a float -> int conversion of a possibly huge k.
    float m4 = k - 4.0f * floorf(k * 0.25f);
    *q = (int)m4;
    return r;
}

FM_FN float fm_sin(float x) {
#ifdef FM_FAST
    return sinf(x);
#endif
    if (!fm_finite(x)) return fm_nan();
    if (fm_abs(x) < 1.0e-4f) return x;  // sin x = x to float precision
    int q;
    float r = fm_reduce_pio2(x, &q);
    float s = fm_sin_poly(r), c = fm_cos_poly(r);
    switch (q) {
        case 0: return s;
        case 1: return c;
        case 2: return -s;
        default: return -c;
    }
}

FM_FN float fm_cos(float x) {
#ifdef FM_FAST
    return cosf(x);
#endif
    if (!fm_finite(x)) return fm_nan();
    int q;
    float r = fm_reduce_pio2(x, &q);
    float s = fm_sin_poly(r), c = fm_cos_poly(r);
    switch (q) {
        case 0: return c;
        case 1: return -s;
        case 2: return -c;
        default: return s;
    }
}

// ---------------------------------------------------------------------
// atan / atan2 / acos.
// ---------------------------------------------------------------------

#define FM_PI 3.1415927410125732f
#define FM_PIO2 1.5707963705062866f
#define FM_PIO6 0.5235987901687622f
#define FM_SQRT3 1.7320507764816284f
#define FM_TAN_PIO12 0.2679491937160492f

// atan on [0, +inf].
FM_FN float fm_atan_pos(float a) {
    if (fm_isinf(a)) return FM_PIO2;
    int inv = 0;
    if (a > 1.0f) {
        a = 1.0f / a;
        inv = 1;
    }
    float off = 0.0f;
    if (a > FM_TAN_PIO12) {
        a = (a * FM_SQRT3 - 1.0f) / (FM_SQRT3 + a);
        off = FM_PIO6;
    }
    float z = a * a;
    float p = -1.0f / 11.0f + z * (1.0f / 13.0f);
    p = 1.0f / 9.0f + z * p;
    p = -1.0f / 7.0f + z * p;
    p = 1.0f / 5.0f + z * p;
    p = -1.0f / 3.0f + z * p;
    float r = off + (a + (a * z) * p);
    if (inv) r = FM_PIO2 - r;
    return r;
}

FM_FN float fm_atan(float x) {
    if (fm_isnan(x)) return x;
    return fm_copysign(fm_atan_pos(fm_abs(x)), x);
}

FM_FN float fm_atan2(float y, float x) {
#ifdef FM_FAST
    return atan2f(y, x);
#endif
    if (fm_isnan(x) || fm_isnan(y)) return fm_nan();
    int xneg = (fm_bits(x) & 0x80000000u) != 0;
    if (y == 0.0f) {
        if (!xneg) return y;             // +-0
        return fm_copysign(FM_PI, y);    // x < 0 or x == -0
    }
    if (x == 0.0f) return fm_copysign(FM_PIO2, y);
    float t;
    if (fm_isinf(x) && fm_isinf(y)) {
        t = 0.7853981852531433f;  // pi/4
    } else if (fm_isinf(x)) {
        t = 0.0f;
    } else if (fm_isinf(y)) {
        t = FM_PIO2;
    } else {
        t = fm_atan_pos(fm_abs(y) / fm_abs(x));
    }
    if (xneg) t = FM_PI - t;
    return fm_copysign(t, y);
}

FM_FN float fm_acos(float x) {
#ifdef FM_FAST
    return acosf(x);
#endif
    if (fm_isnan(x) || x > 1.0f || x < -1.0f) return fm_nan();
    if (x == -1.0f) return FM_PI;
    return 2.0f * fm_atan_pos(sqrtf((1.0f - x) / (1.0f + x)));
}

// ---------------------------------------------------------------------
// exp / exp2 / log / log2 / pow.
// ---------------------------------------------------------------------

#define FM_LN2_1 0.693115234375f
#define FM_LN2_2 3.194618329871446e-05f
#define FM_LN2 0.6931471824645996f
#define FM_LOG2E 1.4426950216293335f

// e^r for |r| <= ln(2)/2.
FM_FN float fm_exp_poly(float r) {
    float p = 1.0f / 5040.0f + r * (1.0f / 40320.0f);
    p = 1.0f / 720.0f + r * p;
    p = 1.0f / 120.0f + r * p;
    p = 1.0f / 24.0f + r * p;
    p = 1.0f / 6.0f + r * p;
    p = 0.5f + r * p;
    p = 1.0f + r * p;
    return 1.0f + r * p;
}

FM_FN float fm_exp(float x) {
#ifdef FM_FAST
    return expf(x);
#endif
    if (fm_isnan(x)) return x;
    if (x > 88.72283935546875f) return fm_float(0x7f800000u);
    if (x < -103.97208404541016f) return 0.0f;
    float k = fm_round(x * FM_LOG2E);
    float r = (x - k * FM_LN2_1) - k * FM_LN2_2;
    return fm_ldexp(fm_exp_poly(r), (int)k);
}

FM_FN float fm_exp2(float t) {
#ifdef FM_FAST
    return exp2f(t);
#endif
    if (fm_isnan(t)) return t;
    if (t >= 128.0f) return fm_float(0x7f800000u);
    if (t < -150.0f) return 0.0f;
    float k = fm_round(t);
    float f = t - k;  // exact: |t| < 2^23
    return fm_ldexp(fm_exp_poly(f * FM_LN2), (int)k);
}

// Split a positive finite x into m * 2^e, m in [sqrt(1/2), sqrt(2)).
FM_FN float fm_frexp_centered(float x, int* e) {
    uint32_t u = fm_bits(x);
    int adj = 0;
    if ((u & 0x7f800000u) == 0) {  // subnormal
        x = x * 8388608.0f;        // 2^23
        u = fm_bits(x);
        adj = -23;
    }
    int ex = (int)((u >> 23) & 0xffu) - 127;
    float m = fm_float((u & 0x007fffffu) | 0x3f800000u);
    if (m > 1.4142135381698608f) {
        m = m * 0.5f;
        ex += 1;
    }
    *e = ex + adj;
    return m;
}

// log(m) for m in [sqrt(1/2), sqrt(2)).
FM_FN float fm_log_m(float m) {
    float s = (m - 1.0f) / (m + 1.0f);
    float z = s * s;
    float p = 1.0f / 11.0f + z * (1.0f / 13.0f);
    p = 1.0f / 9.0f + z * p;
    p = 1.0f / 7.0f + z * p;
    p = 1.0f / 5.0f + z * p;
    p = 1.0f / 3.0f + z * p;
    return 2.0f * s + (2.0f * s * z) * p;
}

FM_FN float fm_log(float x) {
#ifdef FM_FAST
    return logf(x);
#endif
    if (fm_isnan(x) || x < 0.0f) return fm_nan();
    if (x == 0.0f) return fm_float(0xff800000u);
    if (fm_isinf(x)) return x;
    int e;
    float m = fm_frexp_centered(x, &e);
    float lm = fm_log_m(m);
    float fe = (float)e;
    return fe * FM_LN2_1 + (lm + fe * FM_LN2_2);
}

FM_FN float fm_log2(float x) {
#ifdef FM_FAST
    return log2f(x);
#endif
    if (fm_isnan(x) || x < 0.0f) return fm_nan();
    if (x == 0.0f) return fm_float(0xff800000u);
    if (fm_isinf(x)) return x;
    int e;
    float m = fm_frexp_centered(x, &e);
    return (float)e + fm_log_m(m) * FM_LOG2E;
}

FM_FN float fm_pow(float x, float y) {
#ifdef FM_FAST
    return powf(x, y);
#endif
    if (y == 0.0f || x == 1.0f) return 1.0f;
    if (fm_isnan(x) || fm_isnan(y)) return fm_nan();
    if (x < 0.0f) return fm_nan();  // the tracer never raises negatives
    if (x == 0.0f) return y > 0.0f ? 0.0f : fm_float(0x7f800000u);
    if (fm_isinf(x)) return y > 0.0f ? x : 0.0f;
    return fm_exp2(y * fm_log2(x));
}
