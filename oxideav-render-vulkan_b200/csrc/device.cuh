// Device-side path-tracer building blocks for sm_100a.
//
// The per-path arithmetic follows the reference estimator
// (src/shaders/pathtrace.wgsl) operation for operation so that a sample
// here equals the same sample of the CPU estimator bit for bit; this file
// is compiled without FMA contraction (--fmad=false) for that reason, and
// all transcendentals come from fmath.h. What differs from the reference is
// the execution structure (see trace.cu): persistent path slots with
// regeneration, child-pair node fetches, read-only cached loads, guarded
// table and atlas reads, and an ordered per-pixel reduction.
#pragma once

#include <cuda_fp16.h>
#include <stdint.h>

#include "../../include/oxpt.h"
#include "fmath.h"

// Large shading functions (texture filtering, material, BSDF evaluation and
// sampling, light sampling) are kept out of line when OXPT_OUTLINE_SHADING
// is defined: a smaller hot loop against call overhead, chosen by
// measurement.
#if defined(OXPT_OUTLINE_SHADING)
#define OXD_HEAVY __noinline__
#else
#define OXD_HEAVY
#endif

namespace oxd {

constexpr float PI = 3.14159265358979f;
constexpr float INF = 3.0e38f;
constexpr uint32_t NONE = 0xffffffffu;
constexpr float MIN_ALPHA = 1.0e-3f;
constexpr float MIN_SPHERICAL_SOLID_ANGLE = 1.0e-4f;
constexpr uint32_t SHEEN_COS = 32u;
constexpr uint32_t SHEEN_ROUGH = 16u;
constexpr uint32_t F_NORMALS = 1u, F_TANGENTS = 2u, F_COLORS = 4u, F_UV0 = 8u, F_UV1 = 16u;
constexpr uint32_t MAT_STRIDE = 136u, M_FLAGS = 7u, M_SLOTS = 32u;
constexpr uint32_t S_BASE = 0, S_MR = 1, S_NORMAL = 2, S_EMISSIVE = 3, S_SPEC = 4, S_SPEC_COLOR = 5,
                   S_TRANSMISSION = 6, S_THICKNESS = 7, S_CC = 8, S_CC_ROUGH = 9, S_CC_NORMAL = 10,
                   S_SHEEN_COLOR = 11, S_SHEEN_ROUGH = 12;
constexpr int STACK = 64;

// ---------------------------------------------------------------------
// Small vector type with explicit, contraction-free operators.
// ---------------------------------------------------------------------
struct f3 {
    float x, y, z;
    __device__ __forceinline__ float operator[](uint32_t i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
__device__ __forceinline__ f3 mk(float a, float b, float c) { return {a, b, c}; }
__device__ __forceinline__ f3 sp(float a) { return {a, a, a}; }
__device__ __forceinline__ f3 operator+(f3 a, f3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ f3 operator-(f3 a, f3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ f3 operator*(f3 a, f3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
__device__ __forceinline__ f3 operator*(f3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ f3 operator*(float s, f3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ f3 operator/(f3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ f3 operator-(f3 a) { return {-a.x, -a.y, -a.z}; }
__device__ __forceinline__ float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ f3 cross(f3 a, f3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ f3 vmin(f3 a, f3 b) { return {fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)}; }
__device__ __forceinline__ f3 vmax(f3 a, f3 b) { return {fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)}; }
__device__ __forceinline__ float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }
__device__ __forceinline__ f3 xyz(float4 v) { return {v.x, v.y, v.z}; }
__device__ __forceinline__ float4 add4(float4 a, float4 b) { return {a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }
__device__ __forceinline__ float4 mul4(float4 a, float4 b) { return {a.x * b.x, a.y * b.y, a.z * b.z, a.w * b.w}; }
__device__ __forceinline__ float4 scale4(float4 a, float s) { return {a.x * s, a.y * s, a.z * s, a.w * s}; }
__device__ __forceinline__ float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }
__device__ __forceinline__ float4 mix4(float4 a, float4 b, float t) {
    return {mixf(a.x, b.x, t), mixf(a.y, b.y, t), mixf(a.z, b.z, t), mixf(a.w, b.w, t)};
}
__device__ __forceinline__ bool finite(float x) { return (__float_as_uint(x) & 0x7f800000u) != 0x7f800000u; }
__device__ __forceinline__ bool finite3(f3 v) { return finite(v.x) && finite(v.y) && finite(v.z); }
__device__ __forceinline__ bool is_black(f3 a) { return !(a.x > 0.0f || a.y > 0.0f || a.z > 0.0f); }
__device__ __forceinline__ float max3(f3 a) { return fmaxf(fmaxf(a.x, a.y), a.z); }
__device__ __forceinline__ float mean3(f3 a) { return (a.x + a.y + a.z) * (1.0f / 3.0f); }
__device__ __forceinline__ f3 nrm(f3 v) {
    float len = sqrtf(dot(v, v));
    if (len < 1.1920929e-7f) return sp(0.0f);
    return v / len;
}
__device__ __forceinline__ f3 nrm_any(f3 v) {
    float l = sqrtf(dot(v, v));
    if (l > 0.0f) return v / l;
    return sp(0.0f);
}
__device__ __forceinline__ float sign_of(float x) { return (__float_as_uint(x) & 0x80000000u) ? -1.0f : 1.0f; }
// Saturating conversions (WGSL semantics).
__device__ __forceinline__ int32_t to_i32(float x) { return __float2int_rz(x); }
__device__ __forceinline__ uint32_t to_u32(float x) { return __float2uint_rz(x); }
__device__ __forceinline__ int32_t wadd(int32_t a, int32_t b) { return (int32_t)((uint32_t)a + (uint32_t)b); }

// ---------------------------------------------------------------------
// Scene view passed to every kernel by value (lives in the parameter
// constant bank).
// ---------------------------------------------------------------------
struct Scene {
    const float4* geom;
    uint64_t geom_vec4;
    const float4* attrs;
    uint64_t slot_count;
    const uint32_t* tables;
    uint64_t table_words;
    const uint2* atlas;  // RGBA16F texels
    uint32_t side, layers;
    oxpt_params P;
    // Four-wide tree for any-hit queries (8 float4 per node), or null;
    // bvh4_ok: 1 when it answers this scene's any-hit queries exactly.
    const float4* bvh4 = nullptr;
    uint32_t bvh4_root = 0xffffffffu, bvh4_nodes = 0u, bvh4_ok = 0u, pad_ = 0u;
};

__device__ __forceinline__ uint32_t tw(const Scene& s, uint32_t i) {
    return (uint64_t)i < s.table_words ? __ldg(s.tables + i) : 0u;
}
__device__ __forceinline__ float tf(const Scene& s, uint32_t i) { return __uint_as_float(tw(s, i)); }
__device__ __forceinline__ f3 tv3(const Scene& s, uint32_t i) { return {tf(s, i), tf(s, i + 1), tf(s, i + 2)}; }
__device__ __forceinline__ float4 tv4(const Scene& s, uint32_t i) {
    return {tf(s, i), tf(s, i + 1), tf(s, i + 2), tf(s, i + 3)};
}
__device__ __forceinline__ float4 geomv(const Scene& s, uint64_t i) {
    return i < s.geom_vec4 ? __ldg(s.geom + i) : make_float4(0.f, 0.f, 0.f, 0.f);
}
__device__ __forceinline__ float4 attr(const Scene& s, uint32_t slot, uint32_t k) {
    return (uint64_t)slot < s.slot_count ? __ldg(s.attrs + (uint64_t)slot * 12u + k) : make_float4(0.f, 0.f, 0.f, 0.f);
}

// ---------------------------------------------------------------------
// §2 random numbers (pathtrace.wgsl:158-228). Sobol' directions live in
// shared memory, one copy per block.
// ---------------------------------------------------------------------
__device__ __forceinline__ uint32_t pcg_hash(uint32_t x) {
    uint32_t state = x * 747796405u + 2891336453u;
    uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
    return (word >> 22u) ^ word;
}
__device__ __forceinline__ uint32_t hash_mix(uint32_t a, uint32_t b) { return pcg_hash(a ^ pcg_hash(b)); }
__device__ __forceinline__ uint32_t sobol(const uint32_t* dirs, uint32_t index, uint32_t dim) {
    uint32_t r = 0u;
    const uint32_t* v = dirs + dim * 32u;
    // Visit only the set bits of the index.
    while (index) {
        uint32_t k = __ffs(index) - 1u;
        r ^= v[k];
        index &= index - 1u;
    }
    return r;
}
__device__ __forceinline__ uint32_t laine_karras(uint32_t x, uint32_t seed) {
    x += seed;
    x ^= x * 0x6c50b47cu;
    x ^= x * 0xb82f1e52u;
    x ^= x * 0xc7afe638u;
    x ^= x * 0x8d22f6e6u;
    return x;
}
__device__ __forceinline__ uint32_t nus(uint32_t x, uint32_t seed) { return __brev(laine_karras(__brev(x), seed)); }
__device__ __forceinline__ float to_unit(uint32_t v) { return (float)(v >> 8u) * (1.0f / 16777216.0f); }

struct Sampler {
    uint32_t pixel_seed, index, path_seed;
};
__device__ __forceinline__ Sampler make_sampler(uint32_t seed, uint32_t x, uint32_t y, uint32_t index) {
    uint32_t ps = hash_mix(hash_mix(seed, y), x);
    return {ps, index, hash_mix(ps, index)};
}
__device__ __forceinline__ void pattern_u(const uint32_t* dirs, const Sampler& s, uint32_t p, uint32_t out[4]) {
    uint32_t seed = hash_mix(s.pixel_seed, p);
    uint32_t i = nus(s.index, seed);
#pragma unroll
    for (uint32_t d = 0; d < 4; d++) out[d] = nus(sobol(dirs, i, d), hash_mix(seed, d));
}
__device__ __forceinline__ float4 pattern(const uint32_t* dirs, const Sampler& s, uint32_t p) {
    uint32_t u[4];
    pattern_u(dirs, s, p, u);
    return {to_unit(u[0]), to_unit(u[1]), to_unit(u[2]), to_unit(u[3])};
}
__device__ __forceinline__ float coin(const Sampler& s, uint32_t ray, uint32_t tri) {
    return to_unit(hash_mix(hash_mix(s.path_seed, ray), tri));
}

// ---------------------------------------------------------------------
// Geometry and material access (pathtrace.wgsl:234-304).
// ---------------------------------------------------------------------
__device__ __forceinline__ uint64_t tri_base(const Scene& s, uint32_t slot) {
    return (uint64_t)s.P.offs2[2] + 3ull * slot;
}
__device__ __forceinline__ f3 tri_pos(const Scene& s, uint32_t slot, uint32_t v) { return xyz(geomv(s, tri_base(s, slot) + v)); }
__device__ __forceinline__ uint32_t tri_word(const Scene& s, uint32_t slot, uint32_t v) {
    return __float_as_uint(geomv(s, tri_base(s, slot) + v).w);
}
__device__ __forceinline__ uint32_t attr_flags(const Scene& s, uint32_t slot) { return __float_as_uint(attr(s, slot, 0).w); }
__device__ __forceinline__ f3 interp3a(const Scene& s, uint32_t slot, uint32_t k, f3 b) {
    return xyz(attr(s, slot, k)) * b.x + xyz(attr(s, slot, k + 1u)) * b.y + xyz(attr(s, slot, k + 2u)) * b.z;
}
__device__ __forceinline__ float4 interp4a(const Scene& s, uint32_t slot, uint32_t k, f3 b) {
    return add4(add4(scale4(attr(s, slot, k), b.x), scale4(attr(s, slot, k + 1u), b.y)),
                scale4(attr(s, slot, k + 2u), b.z));
}
__device__ __forceinline__ float2 vertex_uv(const Scene& s, uint32_t slot, uint32_t uvset, uint32_t v) {
    float4 a = attr(s, slot, 6u + v);
    return uvset == 0u ? make_float2(a.x, a.y) : make_float2(a.z, a.w);
}
__device__ __forceinline__ bool has_uv(const Scene& s, uint32_t slot, uint32_t uvset) {
    uint32_t f = attr_flags(s, slot);
    if (uvset == 0u) return (f & F_UV0) != 0u;
    if (uvset == 1u) return (f & F_UV1) != 0u;
    return false;
}
__device__ __forceinline__ uint32_t mat_off(const Scene& s, uint32_t m) { return s.P.offs0[2] + m * MAT_STRIDE; }
__device__ __forceinline__ uint32_t mat_flags(const Scene& s, uint32_t m) { return tw(s, mat_off(s, m) + M_FLAGS); }

// ---------------------------------------------------------------------
// Textures: manual taps on the RGBA16F atlas (pathtrace.wgsl:306-507).
// ---------------------------------------------------------------------
struct Level {
    int32_t layer, x, y, w, h;
};
__device__ __forceinline__ Level tex_level(const Scene& s, uint32_t desc, uint32_t level) {
    uint32_t skip = tw(s, desc + 4u), kept = tw(s, desc + 5u);
    int32_t li = (int32_t)level - (int32_t)skip;
    uint32_t l = (uint32_t)(li > 0 ? li : 0);
    uint32_t km = kept - 1u;
    l = l < km ? l : km;
    uint32_t o = desc + 8u + 4u * l;
    uint32_t wh = tw(s, o + 3u);
    return {(int32_t)tw(s, o), (int32_t)tw(s, o + 1u), (int32_t)tw(s, o + 2u), (int32_t)(wh & 0xffffu),
            (int32_t)(wh >> 16u)};
}
__device__ __forceinline__ int32_t wrap_index(int32_t i, int32_t n, uint32_t mode) {
    if (mode == 0u) {
        int32_t m = i > 0 ? i : 0;
        return m < n - 1 ? m : n - 1;
    }
    if (mode == 1u) {
        int32_t m = ((i % (2 * n)) + 2 * n) % (2 * n);
        return m >= n ? 2 * n - 1 - m : m;
    }
    return ((i % n) + n) % n;
}
__device__ __forceinline__ float4 fetch(const Scene& s, const Level& lv, int32_t x, int32_t y, uint32_t ws, uint32_t wt) {
    int32_t xi = wrap_index(x, lv.w, ws), yi = wrap_index(y, lv.h, wt);
    int64_t px = (int64_t)lv.x + xi, py = (int64_t)lv.y + yi;
    if (px < 0 || py < 0 || px >= s.side || py >= s.side || lv.layer < 0 || (uint32_t)lv.layer >= s.layers)
        return make_float4(0.f, 0.f, 0.f, 0.f);
    uint2 t = __ldg(s.atlas + ((uint64_t)lv.layer * s.side + (uint64_t)py) * s.side + (uint64_t)px);
    __half2 lo = *reinterpret_cast<__half2*>(&t.x), hi = *reinterpret_cast<__half2*>(&t.y);
    float2 a = __half22float2(lo), b = __half22float2(hi);
    return {a.x, a.y, b.x, b.y};
}
static __device__ float4 filter_level(const Scene& s, const Level& lv, float2 uv, bool linear, uint32_t ws, uint32_t wt) {
    float u = uv.x, v = uv.y;
    if (!finite(u)) u = 0.0f;
    if (!finite(v)) v = 0.0f;
    u = clampf(u, -1.0e6f, 1.0e6f);
    v = clampf(v, -1.0e6f, 1.0e6f);
    float x = u * (float)lv.w, y = v * (float)lv.h;
    if (!linear) return fetch(s, lv, to_i32(floorf(x)), to_i32(floorf(y)), ws, wt);
    float xf = x - 0.5f, yf = y - 0.5f;
    float x0f = floorf(xf), y0f = floorf(yf);
    float fx = xf - x0f, fy = yf - y0f;
    int32_t x0 = to_i32(x0f), y0 = to_i32(y0f);
    float4 t0 = fetch(s, lv, x0, y0, ws, wt);
    float4 t1 = fetch(s, lv, wadd(x0, 1), y0, ws, wt);
    float4 t2 = fetch(s, lv, x0, wadd(y0, 1), ws, wt);
    float4 t3 = fetch(s, lv, wadd(x0, 1), wadd(y0, 1), ws, wt);
    return mix4(mix4(t0, t1, fx), mix4(t2, t3, fx), fy);
}
static __device__ OXD_HEAVY float4 sample_lod(const Scene& s, uint32_t desc, float2 uv, float lod) {
    uint32_t levels = tw(s, desc), flags = tw(s, desc + 1u);
    uint32_t ws = flags & 3u, wt = (flags >> 2u) & 3u, minf = (flags >> 5u) & 7u;
    bool lin = minf == 1u || minf == 3u || minf == 5u;
    float max_level = (float)(levels - 1u);
    uint32_t l0 = 0u, l1 = 0u;
    float f = 0.0f;
    if (!finite(lod) || lod <= 0.0f) {
        lin = (flags & 16u) != 0u;
    } else if (minf <= 1u) {
        l0 = 0u;
    } else if (minf <= 3u) {
        l0 = to_u32(clampf(floorf(lod + 0.5f), 0.0f, max_level));
    } else {
        float l = clampf(lod, 0.0f, max_level);
        l0 = to_u32(floorf(l));
        l1 = l0 + 1u < levels - 1u ? l0 + 1u : levels - 1u;
        f = l - (float)l0;
    }
    float4 r0 = filter_level(s, tex_level(s, desc, l0), uv, lin, ws, wt);
    if (!(f > 0.0f && l0 != l1)) return r0;
    float4 r1 = filter_level(s, tex_level(s, desc, l1), uv, lin, ws, wt);
    return mix4(r0, r1, f);
}
__device__ __forceinline__ uint32_t slot_word(const Scene& s, uint32_t m, uint32_t k) { return mat_off(s, m) + M_SLOTS + 8u * k; }
__device__ __forceinline__ bool slot_present(const Scene& s, uint32_t m, uint32_t k, uint32_t slot) {
    uint32_t o = slot_word(s, m, k);
    return tw(s, o) != NONE && has_uv(s, slot, tw(s, o + 1u));
}
__device__ __forceinline__ float2 slot_xform(const Scene& s, uint32_t o, float2 uv) {
    return make_float2(tf(s, o + 2u) * uv.x + tf(s, o + 3u) * uv.y + tf(s, o + 4u),
                       tf(s, o + 5u) * uv.x + tf(s, o + 6u) * uv.y + tf(s, o + 7u));
}
struct Lod {
    float width;
    f3 dir;
};
static __device__ float cone_lod(const Scene& s, uint32_t o, uint32_t slot, const Lod& lod) {
    uint32_t desc = tw(s, o), uvset = tw(s, o + 1u);
    float2 uv0 = slot_xform(s, o, vertex_uv(s, slot, uvset, 0u));
    float2 uv1 = slot_xform(s, o, vertex_uv(s, slot, uvset, 1u));
    float2 uv2 = slot_xform(s, o, vertex_uv(s, slot, uvset, 2u));
    float ta = (float)tw(s, desc + 2u) * (float)tw(s, desc + 3u) *
               fabsf((uv1.x - uv0.x) * (uv2.y - uv0.y) - (uv2.x - uv0.x) * (uv1.y - uv0.y));
    f3 p0 = tri_pos(s, slot, 0u);
    f3 cr = cross(tri_pos(s, slot, 1u) - p0, tri_pos(s, slot, 2u) - p0);
    float pa = sqrtf(dot(cr, cr));
    if (!(ta > 0.0f && pa > 0.0f && lod.width > 0.0f)) return 0.0f;
    f3 n = cr / pa;
    float c = fmaxf(fabsf(dot(n, lod.dir)), 1.0e-3f);
    float l = 0.5f * fm_log2(ta / pa) + fm_log2(lod.width / c);
    return finite(l) ? l : 0.0f;
}
static __device__ OXD_HEAVY float4 slot_sample(const Scene& s, uint32_t m, uint32_t k, uint32_t slot, f3 b, const Lod& lod) {
    uint32_t o = slot_word(s, m, k);
    uint32_t uvset = tw(s, o + 1u);
    float2 a0 = vertex_uv(s, slot, uvset, 0u), a1 = vertex_uv(s, slot, uvset, 1u), a2 = vertex_uv(s, slot, uvset, 2u);
    float2 uv = make_float2(a0.x * b.x + a1.x * b.y + a2.x * b.z, a0.y * b.x + a1.y * b.y + a2.y * b.z);
    float l = 0.0f;
    if (lod.width >= 0.0f) l = cone_lod(s, o, slot, lod);
    return sample_lod(s, tw(s, o), slot_xform(s, o, uv), l);
}
__device__ __forceinline__ Lod base_lod() { return {-1.0f, sp(0.0f)}; }
static __device__ float hit_alpha(const Scene& s, uint32_t slot, uint32_t m, f3 b) {
    float a = tf(s, mat_off(s, m) + 3u);
    if (slot_present(s, m, S_BASE, slot)) a *= slot_sample(s, m, S_BASE, slot, b, base_lod()).w;
    if ((attr_flags(s, slot) & F_COLORS) != 0u) a *= interp4a(s, slot, 9u, b).w;
    return a;
}

// ---------------------------------------------------------------------
// Rays (pathtrace.wgsl:513-568).
// ---------------------------------------------------------------------
struct Ray {
    f3 o, d, inv, shear;
    uint32_t kx, ky, kz;
    bool valid;
};
__device__ __forceinline__ Ray make_ray(f3 o, f3 d) {
    Ray r;
    r.inv.x = fabsf(d.x) < 1.0e-30f ? sign_of(d.x) * 1.0e30f : 1.0f / d.x;
    r.inv.y = fabsf(d.y) < 1.0e-30f ? sign_of(d.y) * 1.0e30f : 1.0f / d.y;
    r.inv.z = fabsf(d.z) < 1.0e-30f ? sign_of(d.z) * 1.0e30f : 1.0f / d.z;
    float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
    uint32_t kz = 2u;
    if (ax >= ay && ax >= az) kz = 0u;
    else if (ay >= az) kz = 1u;
    uint32_t kx = kz == 2u ? 0u : kz + 1u;
    uint32_t ky = kx == 2u ? 0u : kx + 1u;
    float dz = d[kz];
    if (dz < 0.0f) {
        uint32_t t = kx;
        kx = ky;
        ky = t;
    }
    r.shear = sp(0.0f);
    if (dz != 0.0f) r.shear = mk(d[kx] / dz, d[ky] / dz, 1.0f / dz);
    r.o = o;
    r.d = d;
    r.kx = kx;
    r.ky = ky;
    r.kz = kz;
    r.valid = finite3(o) && finite3(d) && (d.x != 0.0f || d.y != 0.0f || d.z != 0.0f);
    return r;
}
// Robust slab test (Williams et al. 2005, Ize 2013 far scaling).
// Returns the entry distance, or -1 when the box is missed.
__device__ __forceinline__ float slab6(const Ray& r, float lox, float loy, float loz, float hix, float hiy, float hiz,
                                       float t_max) {
    float t0x = (lox - r.o.x) * r.inv.x, t1x = (hix - r.o.x) * r.inv.x;
    float t0y = (loy - r.o.y) * r.inv.y, t1y = (hiy - r.o.y) * r.inv.y;
    float t0z = (loz - r.o.z) * r.inv.z, t1z = (hiz - r.o.z) * r.inv.z;
    float tnx = fminf(t0x, t1x), tny = fminf(t0y, t1y), tnz = fminf(t0z, t1z);
    float tfx = fmaxf(t0x, t1x), tfy = fmaxf(t0y, t1y), tfz = fmaxf(t0z, t1z);
    float t0 = fmaxf(fmaxf(0.0f, tnx), fmaxf(tny, tnz));
    float t1 = fminf(t_max, fminf(tfx, fminf(tfy, tfz)) * 1.0000004f);
    return t0 <= t1 ? t0 : -1.0f;
}
__device__ __forceinline__ float slab(const Ray& r, float4 lo, float4 hi, float t_max) {
    return slab6(r, lo.x, lo.y, lo.z, hi.x, hi.y, hi.z, t_max);
}

struct Hit {
    uint32_t slot;
    float t;
    f3 b;
    bool front;
};

// Woop-Benthin-Wald watertight test (pathtrace.wgsl:577-619) on the three
// vertex records of a slot, already loaded.
__device__ __forceinline__ bool intersect(const Ray& r, float4 q0, float4 q1, float4 q2, float t_max, Hit* h) {
    f3 p0 = xyz(q0), p1 = xyz(q1), p2 = xyz(q2);
    f3 a = p0 - r.o, b = p1 - r.o, c = p2 - r.o;
    float akz = a[r.kz], bkz = b[r.kz], ckz = c[r.kz];
    float ax = a[r.kx] - r.shear.x * akz;
    float ay = a[r.ky] - r.shear.y * akz;
    float bx = b[r.kx] - r.shear.x * bkz;
    float by = b[r.ky] - r.shear.y * bkz;
    float cx = c[r.kx] - r.shear.x * ckz;
    float cy = c[r.ky] - r.shear.y * ckz;
    float uu = cx * by - cy * bx;
    float vv = ax * cy - ay * cx;
    float ww = bx * ay - by * ax;
    if ((uu < 0.0f || vv < 0.0f || ww < 0.0f) && (uu > 0.0f || vv > 0.0f || ww > 0.0f)) return false;
    float det = uu + vv + ww;
    if (det == 0.0f || !finite(det)) return false;
    float az = r.shear.z * akz, bz = r.shear.z * bkz, cz = r.shear.z * ckz;
    float rcp = 1.0f / det;
    float t = (uu * az + vv * bz + ww * cz) * rcp;
    if (!(t >= 0.0f && t <= t_max)) return false;
    float u = vv * rcp, v = ww * rcp;
    h->t = t;
    h->b = mk(1.0f - u - v, u, v);
    h->front = dot(r.d, cross(p1 - p0, p2 - p0)) < 0.0f;
    return true;
}

// Wächter & Binder 2019 origin offset (pathtrace.wgsl:737-759).
__device__ __forceinline__ float offset1(float p, float n) {
    int32_t of_i = to_i32(256.0f * n);
    uint32_t bits = __float_as_uint(p);
    uint32_t moved = p < 0.0f ? bits - (uint32_t)of_i : bits + (uint32_t)of_i;
    float p_i = __uint_as_float(moved);
    if (fabsf(p) < 1.0f / 32.0f) return p + (1.0f / 65536.0f) * n;
    if (finite(p_i)) return p_i;
    return p;
}
__device__ __forceinline__ f3 offset_ray_origin(f3 p, f3 n) {
    return mk(offset1(p.x, n.x), offset1(p.y, n.y), offset1(p.z, n.z));
}
__device__ __forceinline__ f3 spawn(f3 p, f3 ng, f3 dir) {
    return dot(dir, ng) >= 0.0f ? offset_ray_origin(p, ng) : offset_ray_origin(p, -ng);
}

}  // namespace oxd
