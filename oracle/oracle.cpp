// CPU oracle — TEST INFRASTRUCTURE ONLY (see oracle.h for scope and
// pinning). A line-by-line restatement of pathtrace.wgsl and
// fs_resolve_pt; every function names the WGSL lines it follows. Build
// with -ffp-contract=off so that no multiply-add is fused.
#include "oracle.h"

#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

#include "../oxideav-render-vulkan_b200/csrc/fmath.h"

namespace {

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

struct Params {
    float eye[4], forward[4], side[4], up[4];
    uint32_t dims[4], cfg[4], env[4], offs0[4], offs1[4], offs2[4];
    float fparams[4];
};
static_assert(sizeof(Params) == 176, "Params layout");

struct v2 {
    float x, y;
};
struct v3 {
    float x, y, z;
    float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
struct v4 {
    float x, y, z, w;
    float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
    v3 xyz() const { return {x, y, z}; }
};

inline v3 V3(float a, float b, float c) { return {a, b, c}; }
inline v3 S3(float a) { return {a, a, a}; }
inline v3 operator+(v3 a, v3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline v3 operator-(v3 a, v3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline v3 operator*(v3 a, v3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
inline v3 operator*(v3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline v3 operator*(float s, v3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline v3 operator/(v3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
inline v3 operator/(v3 a, v3 b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
inline v3 operator-(v3 a) { return {-a.x, -a.y, -a.z}; }
inline v4 operator+(v4 a, v4 b) { return {a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }
inline v4 operator*(v4 a, v4 b) { return {a.x * b.x, a.y * b.y, a.z * b.z, a.w * b.w}; }
inline v4 operator*(v4 a, float s) { return {a.x * s, a.y * s, a.z * s, a.w * s}; }
inline v2 operator+(v2 a, v2 b) { return {a.x + b.x, a.y + b.y}; }
inline v2 operator*(v2 a, float s) { return {a.x * s, a.y * s}; }
inline float dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline v3 cross(v3 a, v3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
// WGSL min/max/clamp on floats.
inline float fmn(float a, float b) { return std::fmin(a, b); }
inline float fmx(float a, float b) { return std::fmax(a, b); }
inline float clampf(float x, float lo, float hi) { return fmn(fmx(x, lo), hi); }
inline v3 vmin(v3 a, v3 b) { return {fmn(a.x, b.x), fmn(a.y, b.y), fmn(a.z, b.z)}; }
inline v3 vmax(v3 a, v3 b) { return {fmx(a.x, b.x), fmx(a.y, b.y), fmx(a.z, b.z)}; }
inline v3 vabs(v3 a) { return {std::fabs(a.x), std::fabs(a.y), std::fabs(a.z)}; }
inline v3 vclamp(v3 a, v3 lo, v3 hi) { return vmin(vmax(a, lo), hi); }
inline float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }
inline v4 mix4(v4 a, v4 b, float t) {
    return {mixf(a.x, b.x, t), mixf(a.y, b.y, t), mixf(a.z, b.z, t), mixf(a.w, b.w, t)};
}

inline uint32_t fbits(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}
inline float ffrom(uint32_t u) {
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}
inline uint32_t reverse_bits(uint32_t x) {
    uint32_t r = 0;
    for (int i = 0; i < 32; i++) {
        r = (r << 1) | (x & 1u);
        x >>= 1;
    }
    return r;
}
// WGSL f32 -> i32 / u32 conversions saturate.
inline int32_t to_i32(float x) {
    if (x != x) return 0;
    if (x >= 2147483648.0f) return 2147483647;
    if (x <= -2147483648.0f) return (int32_t)0x80000000u;
    return (int32_t)x;
}
inline uint32_t to_u32(float x) {
    if (x != x || x <= 0.0f) return 0u;
    if (x >= 4294967296.0f) return 0xffffffffu;
    return (uint32_t)x;
}
// WGSL i32 arithmetic wraps.
inline int32_t wadd(int32_t a, int32_t b) { return (int32_t)((uint32_t)a + (uint32_t)b); }

float half_to_float(uint16_t h) {
    uint32_t s = (uint32_t)(h & 0x8000u) << 16, e = (h >> 10) & 0x1fu, m = h & 0x3ffu;
    if (e == 0) {
        if (m == 0) return ffrom(s);
        float v = (float)m * (1.0f / 16777216.0f);  // m * 2^-24
        return s ? -v : v;
    }
    if (e == 31) return ffrom(s | 0x7f800000u | (m << 13));
    return ffrom(s | ((e + 112u) << 23) | (m << 13));
}

struct Counters {
    uint64_t c[8] = {0, 0, 0, 0, 0, 0, 0, 0};
};

struct Ctx {
    const uint32_t* geom;
    size_t geom_words;
    const float* attrs;
    const uint32_t* tables;
    size_t table_words;
    const uint16_t* atlas;
    uint32_t side, layers;
    Params P;
    bool libm;
    uint32_t wg_sobol[128];
    float wg_sheen[512];
    Counters* cnt;

    // ---- transcendentals
    float SIN(float x) const { return libm ? std::sin(x) : fm_sin(x); }
    float COS(float x) const { return libm ? std::cos(x) : fm_cos(x); }
    float ACOS(float x) const { return libm ? std::acos(x) : fm_acos(x); }
    float ATAN2(float y, float x) const { return libm ? std::atan2(y, x) : fm_atan2(y, x); }
    float EXP(float x) const { return libm ? std::exp(x) : fm_exp(x); }
    float LOG(float x) const { return libm ? std::log(x) : fm_log(x); }
    float LOG2(float x) const { return libm ? std::log2(x) : fm_log2(x); }
    float POW(float x, float y) const { return libm ? std::pow(x, y) : fm_pow(x, y); }

    // ---- small helpers (pathtrace.wgsl:106-152)
    uint32_t tw(uint32_t i) const { return i < table_words ? tables[i] : 0u; }
    float tf(uint32_t i) const { return ffrom(tw(i)); }
    v3 tv3(uint32_t i) const { return {tf(i), tf(i + 1), tf(i + 2)}; }
    v4 tv4(uint32_t i) const { return {tf(i), tf(i + 1), tf(i + 2), tf(i + 3)}; }
    v4 geomv(uint32_t i) const {
        if ((size_t)i * 4 + 3 >= geom_words) return {0, 0, 0, 0};
        const uint32_t* g = geom + (size_t)i * 4;
        return {ffrom(g[0]), ffrom(g[1]), ffrom(g[2]), ffrom(g[3])};
    }
    v4 attr(uint32_t slot, uint32_t k) const {
        const float* a = attrs + ((size_t)slot * 12 + k) * 4;
        return {a[0], a[1], a[2], a[3]};
    }
};

inline bool finite(float x) { return (fbits(x) & 0x7f800000u) != 0x7f800000u; }
inline bool finite3(v3 v) { return finite(v.x) && finite(v.y) && finite(v.z); }
inline bool is_black(v3 a) { return !(a.x > 0.0f || a.y > 0.0f || a.z > 0.0f); }
inline float max3(v3 a) { return fmx(fmx(a.x, a.y), a.z); }
inline float mean3(v3 a) { return (a.x + a.y + a.z) * (1.0f / 3.0f); }
inline v3 nrm(v3 v) {
    float len = std::sqrt(dot(v, v));
    if (len < 1.1920929e-7f) return S3(0.0f);
    return v / len;
}
inline float sign_of(float x) { return (fbits(x) & 0x80000000u) ? -1.0f : 1.0f; }

// ---- §2 random numbers (pathtrace.wgsl:158-228)
inline uint32_t pcg_hash(uint32_t x) {
    uint32_t state = x * 747796405u + 2891336453u;
    uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
    return (word >> 22u) ^ word;
}
inline uint32_t hash_mix(uint32_t a, uint32_t b) { return pcg_hash(a ^ pcg_hash(b)); }

uint32_t sobol(const uint32_t* dirs, uint32_t index, uint32_t dim) {
    uint32_t r = 0, i = index, k = 0;
    while (i != 0u) {
        if ((i & 1u) == 1u) r ^= dirs[dim * 32u + k];
        i >>= 1u;
        k += 1u;
    }
    return r;
}
inline uint32_t laine_karras(uint32_t x0, uint32_t seed) {
    uint32_t x = x0 + seed;
    x ^= x * 0x6c50b47cu;
    x ^= x * 0xb82f1e52u;
    x ^= x * 0xc7afe638u;
    x ^= x * 0x8d22f6e6u;
    return x;
}
inline uint32_t nested_uniform_scramble(uint32_t x, uint32_t seed) {
    return reverse_bits(laine_karras(reverse_bits(x), seed));
}
inline float to_unit(uint32_t v) { return (float)(v >> 8u) * (1.0f / 16777216.0f); }

void sobol_owen_4d_u(const uint32_t* dirs, uint32_t index, uint32_t pattern_seed, uint32_t out[4]) {
    uint32_t i = nested_uniform_scramble(index, pattern_seed);
    for (uint32_t d = 0; d < 4; d++)
        out[d] = nested_uniform_scramble(sobol(dirs, i, d), hash_mix(pattern_seed, d));
}

struct Sampler {
    uint32_t pixel_seed, index, path_seed;
};
inline Sampler make_sampler(uint32_t seed, uint32_t x, uint32_t y, uint32_t index) {
    uint32_t pixel_seed = hash_mix(hash_mix(seed, y), x);
    return {pixel_seed, index, hash_mix(pixel_seed, index)};
}
v4 pattern(const Ctx& c, const Sampler& s, uint32_t p) {
    uint32_t u[4];
    sobol_owen_4d_u(c.wg_sobol, s.index, hash_mix(s.pixel_seed, p), u);
    return {to_unit(u[0]), to_unit(u[1]), to_unit(u[2]), to_unit(u[3])};
}
inline float coin(const Sampler& s, uint32_t ray, uint32_t tri) {
    return to_unit(hash_mix(hash_mix(s.path_seed, ray), tri));
}

// ---- geometry access (pathtrace.wgsl:234-304)
inline uint32_t tri_base(const Ctx& c, uint32_t slot) { return c.P.offs2[2] + 3u * slot; }
inline v3 tri_pos(const Ctx& c, uint32_t slot, uint32_t v) { return c.geomv(tri_base(c, slot) + v).xyz(); }
inline uint32_t tri_global(const Ctx& c, uint32_t slot) { return fbits(c.geomv(tri_base(c, slot)).w); }
inline uint32_t tri_light(const Ctx& c, uint32_t slot) { return fbits(c.geomv(tri_base(c, slot) + 1u).w); }
inline uint32_t tri_material(const Ctx& c, uint32_t slot) { return fbits(c.geomv(tri_base(c, slot) + 2u).w); }
inline uint32_t attr_flags(const Ctx& c, uint32_t slot) { return fbits(c.attr(slot, 0).w); }
inline v3 interp3a(const Ctx& c, uint32_t slot, uint32_t k, v3 b) {
    return c.attr(slot, k).xyz() * b.x + c.attr(slot, k + 1u).xyz() * b.y + c.attr(slot, k + 2u).xyz() * b.z;
}
inline v4 interp4a(const Ctx& c, uint32_t slot, uint32_t k, v3 b) {
    return c.attr(slot, k) * b.x + c.attr(slot, k + 1u) * b.y + c.attr(slot, k + 2u) * b.z;
}
inline v2 vertex_uv(const Ctx& c, uint32_t slot, uint32_t uvset, uint32_t v) {
    v4 a = c.attr(slot, 6u + v);
    if (uvset == 0u) return {a.x, a.y};
    return {a.z, a.w};
}
inline bool has_uv(const Ctx& c, uint32_t slot, uint32_t uvset) {
    uint32_t f = attr_flags(c, slot);
    if (uvset == 0u) return (f & F_UV0) != 0u;
    if (uvset == 1u) return (f & F_UV1) != 0u;
    return false;
}
inline uint32_t mat_off(const Ctx& c, uint32_t m) { return c.P.offs0[2] + m * MAT_STRIDE; }
inline uint32_t mat_flags(const Ctx& c, uint32_t m) { return c.tw(mat_off(c, m) + M_FLAGS); }
inline bool mat_double_sided(const Ctx& c, uint32_t m) { return (mat_flags(c, m) & 4u) != 0u; }

// ---- textures (pathtrace.wgsl:306-507)
struct Level {
    int32_t layer, x, y, w, h;
};
Level tex_level(const Ctx& c, uint32_t desc, uint32_t level) {
    uint32_t skip = c.tw(desc + 4u);
    uint32_t kept = c.tw(desc + 5u);
    int32_t li = (int32_t)level - (int32_t)skip;
    uint32_t l = (uint32_t)(li > 0 ? li : 0);
    if (l > kept - 1u) l = kept - 1u;
    uint32_t o = desc + 8u + 4u * l;
    uint32_t wh = c.tw(o + 3u);
    return {(int32_t)c.tw(o), (int32_t)c.tw(o + 1u), (int32_t)c.tw(o + 2u), (int32_t)(wh & 0xffffu),
            (int32_t)(wh >> 16u)};
}
int32_t wrap_index(int32_t i, int32_t n, uint32_t mode) {
    if (mode == 0u) {
        int32_t m = i > 0 ? i : 0;  // clamp(i, 0, n - 1) = min(max(i, 0), n - 1)
        return m < n - 1 ? m : n - 1;
    }
    if (mode == 1u) {
        int32_t m = ((i % (2 * n)) + 2 * n) % (2 * n);
        if (m >= n) return 2 * n - 1 - m;
        return m;
    }
    return ((i % n) + n) % n;
}
v4 fetch(const Ctx& c, const Level& lv, int32_t x, int32_t y, uint32_t ws, uint32_t wt) {
    int32_t xi = wrap_index(x, lv.w, ws);
    int32_t yi = wrap_index(y, lv.h, wt);
    int64_t px = (int64_t)lv.x + xi, py = (int64_t)lv.y + yi;
    if (px < 0 || py < 0 || px >= c.side || py >= c.side || lv.layer < 0 || (uint32_t)lv.layer >= c.layers)
        return {0, 0, 0, 0};
    const uint16_t* t = c.atlas + (((size_t)lv.layer * c.side + (size_t)py) * c.side + (size_t)px) * 4;
    return {half_to_float(t[0]), half_to_float(t[1]), half_to_float(t[2]), half_to_float(t[3])};
}
v4 filter_level(const Ctx& c, const Level& lv, v2 uv, bool linear, uint32_t ws, uint32_t wt) {
    float u = uv.x, v = uv.y;
    if (!finite(u)) u = 0.0f;
    if (!finite(v)) v = 0.0f;
    u = clampf(u, -1.0e6f, 1.0e6f);
    v = clampf(v, -1.0e6f, 1.0e6f);
    float x = u * (float)lv.w;
    float y = v * (float)lv.h;
    if (!linear) return fetch(c, lv, to_i32(std::floor(x)), to_i32(std::floor(y)), ws, wt);
    float xf = x - 0.5f, yf = y - 0.5f;
    float x0f = std::floor(xf), y0f = std::floor(yf);
    float fx = xf - x0f, fy = yf - y0f;
    int32_t x0 = to_i32(x0f), y0 = to_i32(y0f);
    v4 taps[4];
    for (int32_t t = 0; t < 4; t++) taps[t] = fetch(c, lv, wadd(x0, t & 1), wadd(y0, t >> 1), ws, wt);
    return mix4(mix4(taps[0], taps[1], fx), mix4(taps[2], taps[3], fx), fy);
}
v4 sample_lod(const Ctx& c, uint32_t desc, v2 uv, float lod) {
    uint32_t levels = c.tw(desc);
    uint32_t flags = c.tw(desc + 1u);
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
        l0 = to_u32(clampf(std::floor(lod + 0.5f), 0.0f, max_level));
    } else {
        float l = clampf(lod, 0.0f, max_level);
        l0 = to_u32(std::floor(l));
        l1 = l0 + 1u < levels - 1u ? l0 + 1u : levels - 1u;
        f = l - (float)l0;
    }
    uint32_t n = 1u;
    if (f > 0.0f && l0 != l1) n = 2u;
    v4 r[2];
    for (uint32_t i = 0; i < n; i++) {
        uint32_t level = i == 1u ? l1 : l0;
        r[i] = filter_level(c, tex_level(c, desc, level), uv, lin, ws, wt);
    }
    if (n == 1u) return r[0];
    return mix4(r[0], r[1], f);
}
inline uint32_t slot_word(const Ctx& c, uint32_t m, uint32_t s) { return mat_off(c, m) + M_SLOTS + 8u * s; }
inline bool slot_present(const Ctx& c, uint32_t m, uint32_t s, uint32_t slot) {
    uint32_t o = slot_word(c, m, s);
    return c.tw(o) != NONE && has_uv(c, slot, c.tw(o + 1u));
}
inline v2 slot_xform(const Ctx& c, uint32_t m, uint32_t s, v2 uv) {
    uint32_t o = slot_word(c, m, s);
    return {c.tf(o + 2u) * uv.x + c.tf(o + 3u) * uv.y + c.tf(o + 4u),
            c.tf(o + 5u) * uv.x + c.tf(o + 6u) * uv.y + c.tf(o + 7u)};
}
struct Lod {
    float width;
    v3 dir;
};
float cone_lod(const Ctx& c, uint32_t m, uint32_t s, uint32_t slot, const Lod& lod) {
    uint32_t o = slot_word(c, m, s);
    uint32_t desc = c.tw(o), uvset = c.tw(o + 1u);
    v2 uv0 = slot_xform(c, m, s, vertex_uv(c, slot, uvset, 0u));
    v2 uv1 = slot_xform(c, m, s, vertex_uv(c, slot, uvset, 1u));
    v2 uv2 = slot_xform(c, m, s, vertex_uv(c, slot, uvset, 2u));
    float ta = (float)c.tw(desc + 2u) * (float)c.tw(desc + 3u) *
               std::fabs((uv1.x - uv0.x) * (uv2.y - uv0.y) - (uv2.x - uv0.x) * (uv1.y - uv0.y));
    v3 p0 = tri_pos(c, slot, 0u);
    v3 cr = cross(tri_pos(c, slot, 1u) - p0, tri_pos(c, slot, 2u) - p0);
    float pa = std::sqrt(dot(cr, cr));
    if (!(ta > 0.0f && pa > 0.0f && lod.width > 0.0f)) return 0.0f;
    v3 n = cr / pa;
    float cc = fmx(std::fabs(dot(n, lod.dir)), 1.0e-3f);
    float l = 0.5f * c.LOG2(ta / pa) + c.LOG2(lod.width / cc);
    if (finite(l)) return l;
    return 0.0f;
}
v4 slot_sample(const Ctx& c, uint32_t m, uint32_t s, uint32_t slot, v3 b, const Lod& lod) {
    uint32_t o = slot_word(c, m, s);
    uint32_t uvset = c.tw(o + 1u);
    v2 uv = vertex_uv(c, slot, uvset, 0u) * b.x + vertex_uv(c, slot, uvset, 1u) * b.y +
            vertex_uv(c, slot, uvset, 2u) * b.z;
    float l = 0.0f;
    if (lod.width >= 0.0f) l = cone_lod(c, m, s, slot, lod);
    return sample_lod(c, c.tw(o), slot_xform(c, m, s, uv), l);
}
inline Lod base_lod() { return {-1.0f, S3(0.0f)}; }
float hit_alpha(const Ctx& c, uint32_t slot, v3 b) {
    uint32_t m = tri_material(c, slot);
    float a = c.tf(mat_off(c, m) + 3u);
    if (slot_present(c, m, S_BASE, slot)) a *= slot_sample(c, m, S_BASE, slot, b, base_lod()).w;
    if ((attr_flags(c, slot) & F_COLORS) != 0u) a *= interp4a(c, slot, 9u, b).w;
    return a;
}

// ---- rays and traversal (pathtrace.wgsl:513-735)
struct Ray {
    v3 o, d, inv;
    uint32_t kx, ky, kz;
    v3 shear;
    bool valid;
};
Ray make_ray(v3 o, v3 d) {
    Ray r;
    float inv[3];
    for (int k = 0; k < 3; k++) {
        if (std::fabs(d[k]) < 1.0e-30f) inv[k] = sign_of(d[k]) * 1.0e30f;
        else inv[k] = 1.0f / d[k];
    }
    r.inv = {inv[0], inv[1], inv[2]};
    v3 ad = vabs(d);
    uint32_t kz = 2u;
    if (ad.x >= ad.y && ad.x >= ad.z) kz = 0u;
    else if (ad.y >= ad.z) kz = 1u;
    uint32_t kx = (kz + 1u) % 3u, ky = (kx + 1u) % 3u;
    if (d[kz] < 0.0f) {
        uint32_t t = kx;
        kx = ky;
        ky = t;
    }
    v3 shear = S3(0.0f);
    if (d[kz] != 0.0f) shear = {d[kx] / d[kz], d[ky] / d[kz], 1.0f / d[kz]};
    r.o = o;
    r.d = d;
    r.kx = kx;
    r.ky = ky;
    r.kz = kz;
    r.shear = shear;
    r.valid = finite3(o) && finite3(d) && (d.x != 0.0f || d.y != 0.0f || d.z != 0.0f);
    return r;
}
float slab(const Ray& r, v3 bmin, v3 bmax, float t_max) {
    v3 t0s = (bmin - r.o) * r.inv;
    v3 t1s = (bmax - r.o) * r.inv;
    v3 tn = vmin(t0s, t1s);
    v3 tf_ = vmax(t0s, t1s);
    float t0 = fmx(fmx(0.0f, tn.x), fmx(tn.y, tn.z));
    float t1 = fmn(t_max, fmn(tf_.x, fmn(tf_.y, tf_.z)) * 1.0000004f);
    if (t0 <= t1) return t0;
    return -1.0f;
}
struct Hit {
    uint32_t slot;
    float t;
    v3 b;
    bool front;
};
Hit intersect(const Ctx& c, const Ray& r, uint32_t slot, float t_max) {
    Hit h;
    h.slot = NONE;
    h.t = 0;
    h.b = S3(0);
    h.front = false;
    v3 p0 = tri_pos(c, slot, 0u), p1 = tri_pos(c, slot, 1u), p2 = tri_pos(c, slot, 2u);
    v3 a = p0 - r.o, b = p1 - r.o, cc = p2 - r.o;
    float ax = a[r.kx] - r.shear.x * a[r.kz];
    float ay = a[r.ky] - r.shear.y * a[r.kz];
    float bx = b[r.kx] - r.shear.x * b[r.kz];
    float by = b[r.ky] - r.shear.y * b[r.kz];
    float cx = cc[r.kx] - r.shear.x * cc[r.kz];
    float cy = cc[r.ky] - r.shear.y * cc[r.kz];
    float uu = cx * by - cy * bx;
    float vv = ax * cy - ay * cx;
    float ww = bx * ay - by * ax;
    if ((uu < 0.0f || vv < 0.0f || ww < 0.0f) && (uu > 0.0f || vv > 0.0f || ww > 0.0f)) return h;
    float det = uu + vv + ww;
    if (det == 0.0f || !finite(det)) return h;
    float az = r.shear.z * a[r.kz], bz = r.shear.z * b[r.kz], cz = r.shear.z * cc[r.kz];
    float rcp = 1.0f / det;
    float t = (uu * az + vv * bz + ww * cz) * rcp;
    if (!(t >= 0.0f && t <= t_max)) return h;
    float u = vv * rcp, v = ww * rcp;
    h.slot = slot;
    h.t = t;
    h.b = {1.0f - u - v, u, v};
    h.front = dot(r.d, cross(p1 - p0, p2 - p0)) < 0.0f;
    return h;
}
bool accept(const Ctx& c, const Hit& h, const Sampler& s, uint32_t ray_id, bool primary) {
    uint32_t m = tri_material(c, h.slot);
    uint32_t fl = mat_flags(c, m);
    if (primary && !h.front && (fl & 4u) == 0u) return false;
    uint32_t mode = fl & 3u;
    if (mode == 0u) return true;
    if (mode == 1u) return hit_alpha(c, h.slot, h.b) >= c.tf(mat_off(c, m) + 11u);
    return coin(s, ray_id, tri_global(c, h.slot)) < hit_alpha(c, h.slot, h.b);
}
inline v4 node_lo(const Ctx& c, uint32_t i) { return c.geomv(2u * i); }
inline v4 node_hi(const Ctx& c, uint32_t i) { return c.geomv(2u * i + 1u); }

Hit traverse(const Ctx& c, const Ray& r, float t_max_in, const Sampler& s, uint32_t ray_id, bool primary,
             bool any, uint32_t skip) {
    Hit best;
    best.slot = NONE;
    best.t = 0;
    best.b = S3(0);
    best.front = false;
    if (c.P.env[3] == 0u || !r.valid) return best;
    float t_max = t_max_in;
    c.cnt->c[3] += 1;
    if (slab(r, node_lo(c, 0u).xyz(), node_hi(c, 0u).xyz(), t_max) < 0.0f) return best;
    uint32_t stack[64];
    float stack_t[64];
    uint32_t sp = 0u, idx = 0u;
    for (;;) {
        v4 lo = node_lo(c, idx), hi = node_hi(c, idx);
        uint32_t count = fbits(hi.w), first = fbits(lo.w);
        bool descended = false;
        if (count > 0u) {
            c.cnt->c[4] += 1;
            bool done = false;
            for (uint32_t slot = first; slot < first + count; slot++) {
                c.cnt->c[5] += 1;
                Hit h = intersect(c, r, slot, t_max);
                if (h.slot != NONE && tri_global(c, slot) != skip && accept(c, h, s, ray_id, primary)) {
                    best = h;
                    if (any) {
                        done = true;
                        break;
                    }
                    t_max = h.t;
                }
            }
            if (done) break;
        } else {
            c.cnt->c[3] += 2;
            uint32_t l = first;
            float tl = slab(r, node_lo(c, l).xyz(), node_hi(c, l).xyz(), t_max);
            float tr = slab(r, node_lo(c, l + 1u).xyz(), node_hi(c, l + 1u).xyz(), t_max);
            if (tl >= 0.0f && tr >= 0.0f) {
                uint32_t near = l, far = l + 1u;
                float t_far = tr;
                if (tl > tr) {
                    near = l + 1u;
                    far = l;
                    t_far = tl;
                }
                if (sp < 64u) {
                    stack[sp] = far;
                    stack_t[sp] = t_far;
                    sp += 1u;
                }
                idx = near;
                descended = true;
            } else if (tl >= 0.0f) {
                idx = l;
                descended = true;
            } else if (tr >= 0.0f) {
                idx = l + 1u;
                descended = true;
            }
        }
        if (descended) continue;
        bool found = false;
        while (sp != 0u) {
            sp -= 1u;
            c.cnt->c[7] += 1;
            if (stack_t[sp] <= t_max) {
                idx = stack[sp];
                found = true;
                break;
            }
        }
        if (!found) break;
    }
    return best;
}

v3 offset_ray_origin(v3 p, v3 n) {
    float out[3];
    for (int k = 0; k < 3; k++) {
        int32_t of_i = to_i32(256.0f * n[k]);
        int32_t bits = (int32_t)fbits(p[k]);
        int32_t moved = p[k] < 0.0f ? (int32_t)((uint32_t)bits - (uint32_t)of_i)
                                    : (int32_t)((uint32_t)bits + (uint32_t)of_i);
        float p_i = ffrom((uint32_t)moved);
        if (std::fabs(p[k]) < 1.0f / 32.0f) out[k] = p[k] + (1.0f / 65536.0f) * n[k];
        else if (finite(p_i)) out[k] = p_i;
        else out[k] = p[k];
    }
    return {out[0], out[1], out[2]};
}

// ---- surface + material (pathtrace.wgsl:765-916)
struct Surface {
    v3 position, ng, sn;
};
Surface surface(const Ctx& c, const Hit& h) {
    v3 p0 = tri_pos(c, h.slot, 0u), p1 = tri_pos(c, h.slot, 1u), p2 = tri_pos(c, h.slot, 2u);
    v3 b = h.b;
    Surface s;
    s.position = p0 * b.x + p1 * b.y + p2 * b.z;
    v3 cr = cross(p1 - p0, p2 - p0);
    float len = std::sqrt(dot(cr, cr));
    if (len > 0.0f) s.ng = cr / len;
    else s.ng = V3(0.0f, 0.0f, 1.0f);
    s.sn = s.ng;
    if ((attr_flags(c, h.slot) & F_NORMALS) != 0u) {
        v3 n = nrm(interp3a(c, h.slot, 0u, b));
        if (dot(n, n) > 0.5f) s.sn = n;
    }
    return s;
}
struct Mat {
    v4 base;
    float metallic, roughness;
    v3 normal;
    bool unlit;
    v3 emission;
    float ior, specular;
    v3 specular_color;
    float transmission, thickness;
    v3 atten_color;
    float atten_dist, clearcoat, cc_rough;
    v3 cc_normal, sheen;
    float sheen_rough;
};
v3 perturb(const Ctx& c, uint32_t slot, v3 b, v3 n, v4 t, float scale) {
    if ((attr_flags(c, slot) & F_TANGENTS) == 0u) return n;
    v4 tg = interp4a(c, slot, 3u, b);
    float w = 1.0f;
    if (c.attr(slot, 3u).w < 0.0f) w = -1.0f;
    v3 t3 = tg.xyz();
    float d = dot(n, t3);
    v3 tt = nrm(t3 - n * d);
    if (dot(tt, tt) < 0.5f) return n;
    v3 bt = cross(n, tt) * w;
    v3 ts = {(t.x * 2.0f - 1.0f) * scale, (t.y * 2.0f - 1.0f) * scale, t.z * 2.0f - 1.0f};
    v3 nn = nrm(tt * ts.x + bt * ts.y + n * ts.z);
    if (dot(nn, nn) > 0.5f) return nn;
    return n;
}
Mat material(const Ctx& c, const Hit& h, const Surface& surf, const Lod& lod, bool flip) {
    v3 sn = surf.sn;
    if (flip) sn = -sn;
    uint32_t m = tri_material(c, h.slot);
    uint32_t o = mat_off(c, m);
    uint32_t slot = h.slot;
    v3 b = h.b;
    v4 tex[13];
    uint32_t present = 0u;
    for (uint32_t si = 0; si < 13u; si++) {
        tex[si] = {1.0f, 1.0f, 1.0f, 1.0f};
        if (slot_present(c, m, si, slot)) {
            present |= 1u << si;
            Lod l = lod;
            if (si == S_EMISSIVE) l = base_lod();
            tex[si] = slot_sample(c, m, si, slot, b, l);
        }
    }
    Mat r;
    v4 col = c.tv4(o) * tex[S_BASE];
    if ((attr_flags(c, slot) & F_COLORS) != 0u) col = col * interp4a(c, slot, 9u, b);
    r.base = col;
    r.metallic = clampf(c.tf(o + 8u) * tex[S_MR].z, 0.0f, 1.0f);
    r.roughness = clampf(c.tf(o + 9u) * tex[S_MR].y, 0.0f, 1.0f);
    r.normal = sn;
    if ((present & (1u << S_NORMAL)) != 0u) r.normal = perturb(c, slot, b, sn, tex[S_NORMAL], c.tf(o + 10u));
    r.unlit = (c.tw(o + M_FLAGS) & 8u) != 0u;
    r.emission = S3(0.0f);
    v3 e = c.tv3(o + 4u);
    if (!r.unlit && !is_black(e)) r.emission = e * tex[S_EMISSIVE].xyz();
    r.ior = c.tf(o + 12u);
    r.specular = c.tf(o + 13u) * tex[S_SPEC].w;
    r.specular_color = c.tv3(o + 14u) * tex[S_SPEC_COLOR].xyz();
    r.transmission = c.tf(o + 17u) * tex[S_TRANSMISSION].x;
    r.thickness = c.tf(o + 18u) * tex[S_THICKNESS].y;
    r.atten_color = c.tv3(o + 19u);
    r.atten_dist = c.tf(o + 22u);
    r.clearcoat = c.tf(o + 23u) * tex[S_CC].x;
    r.cc_rough = c.tf(o + 24u) * tex[S_CC_ROUGH].y;
    r.cc_normal = sn;
    if ((present & (1u << S_CC_NORMAL)) != 0u)
        r.cc_normal = perturb(c, slot, b, sn, tex[S_CC_NORMAL], c.tf(o + 25u));
    r.sheen = c.tv3(o + 26u) * tex[S_SHEEN_COLOR].xyz();
    r.sheen_rough = c.tf(o + 29u) * tex[S_SHEEN_ROUGH].w;
    return r;
}
v3 emission(const Ctx& c, const Hit& h) {
    uint32_t m = tri_material(c, h.slot);
    uint32_t o = mat_off(c, m);
    v3 e = c.tv3(o + 4u);
    if ((c.tw(o + M_FLAGS) & 8u) != 0u || is_black(e)) return S3(0.0f);
    if (slot_present(c, m, S_EMISSIVE, h.slot))
        return e * slot_sample(c, m, S_EMISSIVE, h.slot, h.b, base_lod()).xyz();
    return e;
}

// ---- §4 BSDF (pathtrace.wgsl:918-1380)
float d_ggx(float n_dot_h, float a) {
    if (n_dot_h <= 0.0f) return 0.0f;
    float a2 = a * a;
    float d = n_dot_h * n_dot_h * (a2 - 1.0f) + 1.0f;
    return a2 / (PI * d * d);
}
float lambda(float c_in, float a) {
    float cc = fmx(std::fabs(c_in), 1.0e-7f);
    float a2 = a * a;
    return (std::sqrt(a2 + (1.0f - a2) * cc * cc) / cc - 1.0f) * 0.5f;
}
inline float g1(float cc, float a) { return 1.0f / (1.0f + lambda(cc, a)); }
inline float g2(float cv, float cl, float a) { return 1.0f / (1.0f + lambda(cv, a) + lambda(cl, a)); }
v3 schlick(v3 f0, float cc) {
    float x = 1.0f - clampf(cc, 0.0f, 1.0f);
    float k = x * x * x * x * x;
    return f0 + (S3(1.0f) - f0) * k;
}
v3 sample_vndf(const Ctx& c, v3 v, float a, float u0, float u1) {
    v3 vh = nrm(V3(a * v.x, a * v.y, v.z));
    float lensq = vh.x * vh.x + vh.y * vh.y;
    v3 t1 = V3(1.0f, 0.0f, 0.0f);
    if (lensq > 0.0f) {
        float il = 1.0f / std::sqrt(lensq);
        t1 = V3(-vh.y * il, vh.x * il, 0.0f);
    }
    v3 t2 = cross(vh, t1);
    float r = std::sqrt(u0);
    float phi = 2.0f * PI * u1;
    float p1 = r * c.COS(phi);
    float p2 = r * c.SIN(phi);
    float s = 0.5f * (1.0f + vh.z);
    p2 = (1.0f - s) * std::sqrt(fmx(1.0f - p1 * p1, 0.0f)) + s * p2;
    float pz = std::sqrt(fmx(1.0f - p1 * p1 - p2 * p2, 0.0f));
    v3 nh = t1 * p1 + t2 * p2 + vh * pz;
    return nrm(V3(a * nh.x, a * nh.y, fmx(nh.z, 1.0e-6f)));
}
float vndf_reflect_pdf(v3 n, v3 v, v3 h, float a) {
    float nv = dot(n, v), nh = dot(n, h);
    if (nv <= 0.0f || nh <= 0.0f || dot(v, h) <= 0.0f) return 0.0f;
    return g1(nv, a) * d_ggx(nh, a) / (4.0f * nv);
}
inline v3 reflect_h(v3 v, v3 h) { return 2.0f * dot(v, h) * h - v; }
float d_charlie(const Ctx& c, float n_dot_h, float a) {
    float inv = 1.0f / fmx(a, 1.0e-3f);
    float sin2 = fmx(1.0f - n_dot_h * n_dot_h, 0.0f);
    if (sin2 <= 0.0f) return 0.0f;
    return (2.0f + inv) * c.POW(sin2, inv * 0.5f) / (2.0f * PI);
}
inline float v_neubelt(float nl, float nv) { return 1.0f / fmx(4.0f * (nl + nv - nl * nv), 1.0e-6f); }
float sheen_albedo(const Ctx& c, float cc, float rough) {
    float x = clampf(clampf(cc, 0.0f, 1.0f) * (float)SHEEN_COS - 0.5f, 0.0f, (float)(SHEEN_COS - 1u));
    float y = clampf(clampf(rough, 0.0f, 1.0f) * (float)(SHEEN_ROUGH - 1u), 0.0f, (float)(SHEEN_ROUGH - 1u));
    uint32_t x0 = to_u32(std::floor(x)), y0 = to_u32(std::floor(y));
    uint32_t x1 = x0 + 1u < SHEEN_COS - 1u ? x0 + 1u : SHEEN_COS - 1u;
    uint32_t y1 = y0 + 1u < SHEEN_ROUGH - 1u ? y0 + 1u : SHEEN_ROUGH - 1u;
    float fx = x - (float)x0, fy = y - (float)y0;
    float a00 = c.wg_sheen[y0 * SHEEN_COS + x0];
    float a10 = c.wg_sheen[y0 * SHEEN_COS + x1];
    float a01 = c.wg_sheen[y1 * SHEEN_COS + x0];
    float a11 = c.wg_sheen[y1 * SHEEN_COS + x1];
    float a = a00 + (a10 - a00) * fx;
    float bb = a01 + (a11 - a01) * fx;
    return a + (bb - a) * fy;
}
v3 basis_t(v3 n) {
    float sign = sign_of(n.z);
    float a = -1.0f / (sign + n.z);
    float b = n.x * n.y * a;
    return V3(1.0f + sign * n.x * n.x * a, sign * b, -sign * n.x);
}
v3 basis_b(v3 n) {
    float sign = sign_of(n.z);
    float a = -1.0f / (sign + n.z);
    float b = n.x * n.y * a;
    return V3(b, sign + n.y * n.y * a, -n.y);
}
v3 cosine_hemisphere(const Ctx& c, float u0, float u1) {
    float a = 2.0f * u0 - 1.0f, b = 2.0f * u1 - 1.0f;
    float r = 0.0f, phi = 0.0f;
    if (a == 0.0f && b == 0.0f) {
        r = 0.0f;
        phi = 0.0f;
    } else if (std::fabs(a) > std::fabs(b)) {
        r = a;
        phi = (PI / 4.0f) * (b / a);
    } else {
        r = b;
        phi = PI / 2.0f - (PI / 4.0f) * (a / b);
    }
    float x = r * c.COS(phi), y = r * c.SIN(phi);
    return V3(x, y, std::sqrt(fmx(1.0f - x * x - y * y, 0.0f)));
}
struct Bsdf {
    v3 v, n, ng, ncc, base;
    float metallic, alpha, specular;
    v3 f0d;
    float transmission;
    bool thin;
    float eta_i, eta_t, clearcoat, cc_alpha;
    v3 sheen;
    float sheen_rough, sheen_alpha, w_cc;
    v4 p;
    float p4;
};
v3 fresnel_d(const Bsdf& bs, float cc) {
    if (bs.eta_i > bs.eta_t) {
        float eta = bs.eta_i / bs.eta_t;
        float s2 = eta * eta * fmx(1.0f - cc * cc, 0.0f);
        if (s2 >= 1.0f) return S3(1.0f);
        return schlick(bs.f0d, std::sqrt(1.0f - s2));
    }
    return schlick(bs.f0d, cc);
}
Bsdf make_bsdf(const Ctx& c, const Mat& m, v3 v, v3 ng_in, bool front) {
    float fl = front ? 1.0f : -1.0f;
    v3 ng = ng_in * fl;
    v3 n = m.normal * fl;
    if (dot(n, v) <= 1.0e-4f) n = ng;
    v3 ncc = m.cc_normal * fl;
    if (dot(ncc, v) <= 1.0e-4f) ncc = n;
    bool thin = m.thickness <= 0.0f;
    float ior = 1.5f;
    if (finite(m.ior) && m.ior >= 1.0f) ior = m.ior;
    float eta_i = ior, eta_t = 1.0f;
    if (thin || front) {
        eta_i = 1.0f;
        eta_t = ior;
    }
    bool inside = !thin && !front;
    float q = (ior - 1.0f) / (ior + 1.0f);
    float r0 = q * q;
    Bsdf b;
    b.v = v;
    b.n = n;
    b.ng = ng;
    b.ncc = ncc;
    b.base = m.base.xyz();
    b.metallic = m.metallic;
    b.alpha = fmx(m.roughness * m.roughness, MIN_ALPHA);
    b.specular = clampf(m.specular, 0.0f, 1.0f);
    b.f0d = vmin(r0 * m.specular_color, S3(1.0f));
    b.transmission = m.transmission;
    b.thin = thin;
    b.eta_i = eta_i;
    b.eta_t = eta_t;
    b.clearcoat = m.clearcoat;
    b.sheen = m.sheen;
    if (inside) {
        b.clearcoat = 0.0f;
        b.sheen = S3(0.0f);
    }
    b.cc_alpha = fmx(m.cc_rough * m.cc_rough, MIN_ALPHA);
    b.sheen_rough = m.sheen_rough;
    b.sheen_alpha = fmx(m.sheen_rough * m.sheen_rough, 1.0e-3f);
    float cv = fmx(dot(n, v), 1.0e-4f);
    b.w_cc = 0.0f;
    if (b.clearcoat > 0.0f) b.w_cc = b.clearcoat * schlick(S3(0.04f), dot(ncc, v)).x;
    float sheen_max = max3(b.sheen);
    float e_v = 0.0f;
    if (sheen_max > 0.0f) e_v = sheen_albedo(c, cv, b.sheen_rough);
    float s_scale = (1.0f - b.w_cc) * (1.0f - sheen_max * e_v);
    float fd = b.specular * max3(fresnel_d(b, cv));
    float fm = mean3(schlick(b.base, cv));
    float mm = b.metallic;
    float base_mean = fmx(mean3(b.base), 0.0f);
    v4 p = {s_scale * (1.0f - mm) * (1.0f - b.transmission) * (1.0f - fd) * base_mean,
            s_scale * ((1.0f - mm) * fd + mm * fm),
            s_scale * (1.0f - mm) * b.transmission * (1.0f - fd) * base_mean, b.w_cc};
    float p4 = (1.0f - b.w_cc) * sheen_max * e_v;
    float sum = p.x + p.y + p.z + p.w + p4;
    if (sum > 0.0f && finite(sum)) {
        p = {p.x / sum, p.y / sum, p.z / sum, p.w / sum};
        p4 = p4 / sum;
    } else {
        p = {0, 0, 0, 0};
        p4 = 0.0f;
    }
    b.p = p;
    b.p4 = p4;
    return b;
}
inline bool bsdf_black(const Bsdf& b) {
    return b.p.x <= 0.0f && b.p.y <= 0.0f && b.p.z <= 0.0f && b.p.w <= 0.0f && b.p4 <= 0.0f;
}
inline float lobe_p(const Bsdf& b, uint32_t i) { return i == 4u ? b.p4 : b.p[(int)i]; }
struct Eval {
    v3 f;
    float pdf;
};
Eval bsdf_eval(const Ctx& c, const Bsdf& b, v3 l) {
    v3 v = b.v, n = b.n;
    float nv = fmx(dot(n, v), 1.0e-4f);
    if (dot(b.ng, l) > 0.0f) {
        float nl = dot(n, l);
        v3 h = nrm(v + l);
        float vh = fmx(dot(v, h), 0.0f);
        float nh = dot(n, h);
        v3 f = S3(0.0f);
        float pdf = 0.0f;
        if (nl > 0.0f) {
            v3 fd = fresnel_d(b, vh);
            v3 fm = schlick(b.base, vh);
            float spec_c = d_ggx(nh, b.alpha) * g2(nv, nl, b.alpha) / (4.0f * nv * nl);
            float m = b.metallic;
            float diff_k = (1.0f - m) * (1.0f - b.transmission) * (1.0f - b.specular * max3(fd)) / PI;
            v3 layer = spec_c * ((1.0f - m) * b.specular * fd + m * fm) + diff_k * b.base;
            float smax = max3(b.sheen);
            if (smax > 0.0f) {
                float scale = fmn(1.0f - smax * sheen_albedo(c, nv, b.sheen_rough),
                                  1.0f - smax * sheen_albedo(c, nl, b.sheen_rough));
                float sh = d_charlie(c, nh, b.sheen_alpha) * v_neubelt(nl, nv);
                layer = layer * scale + b.sheen * sh;
            }
            f = layer * (1.0f - b.w_cc);
            pdf += (b.p.x + b.p4) * nl / PI;
            pdf += b.p.y * vndf_reflect_pdf(n, v, h, b.alpha);
        }
        if (b.clearcoat > 0.0f) {
            float cnv = fmx(dot(b.ncc, v), 1.0e-4f);
            float cnl = dot(b.ncc, l);
            if (cnl > 0.0f) {
                float cnh = dot(b.ncc, h);
                float cc = b.w_cc * d_ggx(cnh, b.cc_alpha) * g2(cnv, cnl, b.cc_alpha) / (4.0f * cnv * cnl);
                f = f + S3(cc);
                pdf += b.p.w * vndf_reflect_pdf(b.ncc, v, h, b.cc_alpha);
            }
        }
        return {f * fmx(nl, 0.0f), pdf};
    }
    if (b.transmission <= 0.0f || b.metallic >= 1.0f) return {S3(0.0f), 0.0f};
    float nl = -dot(n, l);
    if (nl <= 0.0f) return {S3(0.0f), 0.0f};
    float smax = max3(b.sheen);
    float sheen_scale = 1.0f;
    if (smax > 0.0f) sheen_scale = 1.0f - smax * sheen_albedo(c, nv, b.sheen_rough);
    float w = (1.0f - b.metallic) * b.transmission * (1.0f - b.w_cc) * sheen_scale;
    float val = 0.0f, pdf_t = 0.0f;
    if (b.thin) {
        v3 lm = l + n * (2.0f * nl);
        v3 h = nrm(v + lm);
        float vh = dot(v, h), nh = dot(n, h);
        if (vh <= 0.0f || nh <= 0.0f) return {S3(0.0f), 0.0f};
        float fd = b.specular * max3(fresnel_d(b, vh));
        val = d_ggx(nh, b.alpha) * g2(nv, nl, b.alpha) / (4.0f * nv * nl) * (1.0f - fd);
        pdf_t = vndf_reflect_pdf(n, v, h, b.alpha);
    } else {
        float ei = b.eta_i, et = b.eta_t;
        v3 h = nrm(-(ei * v + et * l));
        if (dot(h, n) < 0.0f) h = -h;
        float vh = dot(v, h), lh = dot(l, h), nh = dot(n, h);
        if (vh <= 0.0f || lh >= 0.0f || nh <= 0.0f) return {S3(0.0f), 0.0f};
        float denom = ei * vh + et * lh;
        if (std::fabs(denom) < 1.0e-6f) return {S3(0.0f), 0.0f};
        float d = d_ggx(nh, b.alpha);
        float fd = b.specular * max3(fresnel_d(b, vh));
        float jac = et * et * std::fabs(lh) / (denom * denom);
        val = vh * std::fabs(lh) * d * g2(nv, nl, b.alpha) * et * et * (1.0f - fd) / (nv * nl * denom * denom);
        pdf_t = g1(nv, b.alpha) * vh * d / nv * jac;
    }
    return {b.base * (w * val * nl), b.p.z * pdf_t};
}
struct BSample {
    bool ok;
    v3 l, f;
    float pdf;
};
bool refract_h(v3 v, v3 h, float eta, v3* out) {
    float ci = dot(v, h);
    float s2 = eta * eta * fmx(1.0f - ci * ci, 0.0f);
    if (s2 >= 1.0f) return false;
    float ct = std::sqrt(1.0f - s2);
    float k = eta * ci - ct;
    *out = nrm(-eta * v + k * h);
    return true;
}
BSample bsdf_sample(const Ctx& c, const Bsdf& b, v3 u) {
    BSample res;
    res.ok = false;
    res.l = res.f = S3(0);
    res.pdf = 0;
    float acc = 0.0f;
    uint32_t lobe = NONE;
    for (uint32_t i = 0; i < 5u; i++) {
        float p = lobe_p(b, i);
        acc += p;
        if (p > 0.0f && u.z < acc) {
            lobe = i;
            break;
        }
    }
    if (lobe == NONE) {
        for (uint32_t i = 0; i < 5u; i++)
            if (lobe_p(b, i) > 0.0f) lobe = i;
        if (lobe == NONE) return res;
    }
    v3 v = b.v;
    v3 l;
    if (lobe == 0u || lobe == 4u) {
        v3 t = basis_t(b.n), bb = basis_b(b.n);
        v3 cc = cosine_hemisphere(c, u.x, u.y);
        l = t * cc.x + bb * cc.y + b.n * cc.z;
    } else {
        v3 nn = b.n;
        float a = b.alpha;
        if (lobe == 3u) {
            nn = b.ncc;
            a = b.cc_alpha;
        }
        v3 t = basis_t(nn), bb = basis_b(nn);
        v3 vl = V3(dot(v, t), dot(v, bb), dot(v, nn));
        if (vl.z <= 0.0f) return res;
        v3 hl = sample_vndf(c, vl, a, u.x, u.y);
        v3 h = t * hl.x + bb * hl.y + nn * hl.z;
        if (lobe != 2u) {
            l = reflect_h(v, h);
        } else if (b.thin) {
            v3 r = reflect_h(v, h);
            float d = dot(r, b.n);
            l = r + b.n * (-2.0f * d);
        } else {
            v3 rl;
            if (!refract_h(v, h, b.eta_i / b.eta_t, &rl)) return res;
            l = rl;
        }
    }
    if (!finite3(l) || dot(l, l) < 0.5f) return res;
    bool reflection = dot(b.ng, l) > 0.0f;
    if (reflection == (lobe == 2u)) return res;
    Eval e = bsdf_eval(c, b, l);
    if (e.pdf <= 0.0f || !finite(e.pdf) || is_black(e.f) || !finite3(e.f)) return res;
    res.ok = true;
    res.l = l;
    res.f = e.f;
    res.pdf = e.pdf;
    return res;
}

// ---- lights (pathtrace.wgsl:1382-1654)
struct LightSample {
    bool ok;
    v3 l;
    float distance;
    v3 radiance;
};
LightSample punctual_sample(const Ctx& c, uint32_t j, v3 p) {
    uint32_t o = c.P.offs0[3] + 16u * j;
    LightSample r;
    r.ok = false;
    r.l = r.radiance = S3(0);
    r.distance = 0;
    uint32_t kind = c.tw(o + 3u);
    v3 base = c.tv3(o + 8u), dir = c.tv3(o + 4u);
    if (kind == 0u) {
        r.ok = true;
        r.l = -dir;
        r.distance = -1.0f;
        r.radiance = base;
        return r;
    }
    v3 to = c.tv3(o) - p;
    float d2 = dot(to, to);
    if (!(d2 > 1.0e-12f)) return r;
    float d = std::sqrt(d2);
    v3 l = to / d;
    float att = 1.0f / d2;
    float range = c.tf(o + 7u);
    if (range > 0.0f) {
        float x = d / range;
        att *= clampf(1.0f - x * x * x * x, 0.0f, 1.0f);
    }
    if (kind == 2u) {
        float cd = dot(dir, -l);
        float a = clampf(cd * c.tf(o + 12u) + c.tf(o + 13u), 0.0f, 1.0f);
        att *= a * a;
    }
    if (att <= 0.0f) return r;
    r.ok = true;
    r.l = l;
    r.distance = d;
    r.radiance = base * att;
    return r;
}
uint32_t partition_point(const Ctx& c, uint32_t o, uint32_t n, float u) {
    uint32_t lo = 0u, hi = n;
    while (lo < hi) {
        uint32_t mid = (lo + hi) / 2u;
        if (c.tf(o + mid) <= u) lo = mid + 1u;
        else hi = mid;
    }
    return lo;
}
inline float elight_pmf(const Ctx& c, uint32_t li) { return c.tf(c.P.offs1[0] + 4u * li + 1u); }
inline uint32_t elight_slot(const Ctx& c, uint32_t li) { return c.tw(c.P.offs1[0] + 4u * li + 3u); }
uint32_t pick_elight(const Ctx& c, float u) {
    uint32_t n = c.P.cfg[3];
    uint32_t lo = 0u, hi = n;
    while (lo < hi) {
        uint32_t mid = (lo + hi) / 2u;
        if (c.tf(c.P.offs1[0] + 4u * mid) <= u) lo = mid + 1u;
        else hi = mid;
    }
    return lo < n - 1u ? lo : n - 1u;
}
inline v3 nrm_any(v3 v) {
    float l = std::sqrt(dot(v, v));
    if (l > 0.0f) return v / l;
    return S3(0.0f);
}
float triangle_solid_angle(const Ctx& c, v3 p, v3 a0, v3 b0, v3 c0) {
    v3 a = nrm_any(a0 - p), b = nrm_any(b0 - p), cc = nrm_any(c0 - p);
    float num = std::fabs(dot(a, cross(b, cc)));
    float den = 1.0f + dot(a, b) + dot(b, cc) + dot(cc, a);
    float o = 2.0f * c.ATAN2(num, den);
    if (finite(o)) return fmx(o, 0.0f);
    return 0.0f;
}
v3 sample_spherical_triangle(const Ctx& c, v3 p, v3 a0, v3 b0, v3 c0, float u0, float u1) {
    v3 zero = S3(0.0f);
    v3 a = nrm_any(a0 - p), b = nrm_any(b0 - p), cc = nrm_any(c0 - p);
    v3 nab = nrm_any(cross(a, b)), nbc = nrm_any(cross(b, cc)), nca = nrm_any(cross(cc, a));
    if (dot(a, a) == 0.0f || dot(b, b) == 0.0f || dot(cc, cc) == 0.0f || dot(nab, nab) == 0.0f ||
        dot(nbc, nbc) == 0.0f || dot(nca, nca) == 0.0f)
        return zero;
    float alpha = c.ACOS(clampf(-dot(nab, nca), -1.0f, 1.0f));
    float beta = c.ACOS(clampf(-dot(nbc, nab), -1.0f, 1.0f));
    float gamma = c.ACOS(clampf(-dot(nca, nbc), -1.0f, 1.0f));
    float area = alpha + beta + gamma - PI;
    if (!(area > 0.0f)) return zero;
    float ap = u0 * area;
    float s = c.SIN(ap - alpha), t = c.COS(ap - alpha);
    float sa = c.SIN(alpha), ca = c.COS(alpha);
    float cos_c = dot(a, b);
    float uu = t - ca;
    float vv = s + sa * cos_c;
    float den = (vv * s + uu * t) * sa;
    if (std::fabs(den) < 1.0e-30f) return zero;
    float q = clampf(((vv * t - uu * s) * ca - vv) / den, -1.0f, 1.0f);
    v3 ca_perp = nrm_any(cc - dot(cc, a) * a);
    if (dot(ca_perp, ca_perp) == 0.0f) return zero;
    float r = std::sqrt(fmx(1.0f - q * q, 0.0f));
    v3 cp = q * a + r * ca_perp;
    float z = 1.0f - u1 * (1.0f - dot(cp, b));
    v3 cb_perp = nrm_any(cp - dot(cp, b) * b);
    float w = std::sqrt(fmx(1.0f - z * z, 0.0f));
    v3 d = b;
    if (dot(cb_perp, cb_perp) > 0.0f) d = z * b + w * cb_perp;
    return nrm_any(d);
}
inline float p_env(const Ctx& c) { return c.P.fparams[2]; }
float tri_pdf(const Ctx& c, uint32_t li, uint32_t slot, v3 p, v3 q) {
    v3 a = tri_pos(c, slot, 0u), b = tri_pos(c, slot, 1u), cc = tri_pos(c, slot, 2u);
    float sel = (1.0f - p_env(c)) * elight_pmf(c, li);
    float omega = triangle_solid_angle(c, p, a, b, cc);
    if (omega >= MIN_SPHERICAL_SOLID_ANGLE) return sel / omega;
    v3 cr = cross(b - a, cc - a);
    float len = std::sqrt(dot(cr, cr));
    v3 to = q - p;
    float d2 = dot(to, to);
    if (len <= 0.0f || d2 <= 0.0f) return 0.0f;
    float cs = std::fabs(dot(cr, to) / (len * std::sqrt(d2)));
    if (cs <= 0.0f) return 0.0f;
    return sel * d2 / (0.5f * len * cs);
}
struct Texel {
    uint32_t x, y;
    float st;
};
Texel env_texel(const Ctx& c, v3 d) {
    uint32_t w = c.P.env[0], h = c.P.env[1];
    float u = 0.5f + c.ATAN2(d.x, -d.z) / (2.0f * PI);
    float th = c.ACOS(clampf(d.y, -1.0f, 1.0f));
    float v = th / PI;
    uint32_t x = to_u32(fmx(u * (float)w, 0.0f));
    if (x > w - 1u) x = w - 1u;
    uint32_t y = to_u32(fmx(v * (float)h, 0.0f));
    if (y > h - 1u) y = h - 1u;
    return {x, y, c.SIN(th)};
}
v3 env_radiance(const Ctx& c, v3 d) {
    Texel t = env_texel(c, d);
    return c.tv3(c.P.offs2[1] + 3u * (t.y * c.P.env[0] + t.x));
}
float env_pdf(const Ctx& c, v3 d) {
    Texel t = env_texel(c, d);
    if (t.st <= 1.0e-6f) return 0.0f;
    uint32_t w = c.P.env[0], h = c.P.env[1];
    return c.tf(c.P.offs2[0] + t.y * w + t.x) * (float)(w * h) / (2.0f * PI * PI * t.st);
}
struct EnvSample {
    bool ok;
    v3 d, le;
    float pdf;
};
EnvSample env_sample(const Ctx& c, float u0, float u1) {
    EnvSample r;
    r.ok = false;
    r.d = r.le = S3(0);
    r.pdf = 0;
    uint32_t w = c.P.env[0], h = c.P.env[1];
    uint32_t marg = c.P.offs1[2];
    uint32_t pp = partition_point(c, marg, h + 1u, u0);
    uint32_t y = (pp < 1u ? 1u : (pp > h ? h : pp)) - 1u;
    uint32_t row = c.P.offs1[3] + y * (w + 1u);
    uint32_t px = partition_point(c, row, w + 1u, u1);
    uint32_t x = (px < 1u ? 1u : (px > w ? w : px)) - 1u;
    float my = (u0 - c.tf(marg + y)) / fmx(c.tf(marg + y + 1u) - c.tf(marg + y), 1.0e-12f);
    float mx = (u1 - c.tf(row + x)) / fmx(c.tf(row + x + 1u) - c.tf(row + x), 1.0e-12f);
    float u = ((float)x + clampf(mx, 0.0f, 0.99999f)) / (float)w;
    float v = ((float)y + clampf(my, 0.0f, 0.99999f)) / (float)h;
    float phi = 2.0f * PI * (u - 0.5f);
    float th = PI * v;
    float st = c.SIN(th), ct = c.COS(th);
    v3 d = V3(st * c.SIN(phi), ct, -st * c.COS(phi));
    float pdf = env_pdf(c, d);
    if (pdf <= 0.0f || !finite(pdf)) return r;
    r.ok = true;
    r.d = d;
    r.le = env_radiance(c, d);
    r.pdf = pdf;
    return r;
}

// ---- §3 integrator (pathtrace.wgsl:1660-2045)
float power_heuristic(float a, float b) {
    float a2 = a * a, b2 = b * b;
    if (a2 + b2 > 0.0f && finite(a2 + b2)) return a2 / (a2 + b2);
    if (!finite(a) && a > 0.0f) return 1.0f;
    return 0.0f;
}
v3 clamp_c(const Ctx& c, v3 col) {
    float m = max3(col);
    float cl = c.P.fparams[1];
    if (cl > 0.0f && m > cl) return col * (cl / m);
    return col;
}
inline v3 spawn(v3 p, v3 ng, v3 dir) {
    if (dot(dir, ng) >= 0.0f) return offset_ray_origin(p, ng);
    return offset_ray_origin(p, -ng);
}
float light_pdf(const Ctx& c, const Hit& h, v3 p, v3 q) {
    uint32_t li = tri_light(c, h.slot);
    if (li == NONE) return 0.0f;
    return tri_pdf(c, li, h.slot, p, q);
}
struct PathResult {
    bool covered;
    v3 radiance;
};

PathResult trace_sample(const Ctx& c, uint32_t x, uint32_t y, uint32_t index) {
    const Params& P = c.P;
    Sampler s = make_sampler(P.dims[2], x, y, index);
    v4 p0 = pattern(c, s, 0u);
    float width = (float)P.dims[0], height = (float)P.dims[1];
    float ndc_x = (((float)x + p0.x) / fmx(width, 1.0f)) * 2.0f - 1.0f;
    float ndc_y = 1.0f - (((float)y + p0.y) / fmx(height, 1.0f)) * 2.0f;
    bool orthographic = P.eye[3] > 0.5f;
    float half_w = P.forward[3], half_h = P.side[3];
    v3 eye = V3(P.eye[0], P.eye[1], P.eye[2]);
    v3 fwd = V3(P.forward[0], P.forward[1], P.forward[2]);
    v3 side = V3(P.side[0], P.side[1], P.side[2]);
    v3 up = V3(P.up[0], P.up[1], P.up[2]);
    v3 o, d;
    if (orthographic) {
        o = eye + (side * (ndc_x * half_w) + up * (ndc_y * half_h));
        d = fwd;
    } else {
        o = eye;
        d = nrm(side * (ndc_x * half_w) + up * (ndc_y * half_h) + fwd);
    }
    v3 beta = S3(1.0f), radiance = S3(0.0f);
    float prev_pdf = 0.0f;
    v3 prev_pos = S3(0.0f);
    bool in_medium = false;
    v3 sigma = S3(0.0f);
    uint32_t strategy = P.cfg[1];
    bool has_env = P.env[2] != 0u;
    uint32_t n_elights = P.cfg[3], n_punct = P.cfg[2];
    uint32_t k = 0u;
    bool shadow = false;
    v3 r_o = o, r_d = d;
    float r_tmax = INF;
    uint32_t r_id = 0u, r_skip = NONE;
    v3 pending = S3(0.0f);
    Bsdf bsdf{};
    v3 p = S3(0.0f), ng = S3(0.0f);
    float thickness = 0.0f, transmission = 0.0f;
    v3 atten_color = S3(1.0f);
    float atten_dist = -1.0f;
    bool front = true;
    v4 pl_u = {0, 0, 0, 0};
    uint32_t job = 0u;
    for (;;) {
        c.cnt->c[shadow ? 2 : 1] += 1;
        Hit hit = traverse(c, make_ray(r_o, r_d), r_tmax, s, r_id, !shadow && k == 0u, shadow, r_skip);
        if (shadow) {
            if (hit.slot == NONE) radiance = radiance + pending;
            job += 1u;
        } else {
            if (in_medium) {
                if (hit.slot == NONE) break;
                v3 ex = -sigma * hit.t;
                beta = beta * V3(c.EXP(ex.x), c.EXP(ex.y), c.EXP(ex.z));
            }
            if (hit.slot == NONE) {
                if (k == 0u) return {false, S3(0.0f)};
                v3 le = S3(P.fparams[0]);
                float w = 1.0f;
                if (has_env) {
                    le = env_radiance(c, d);
                    if (strategy == 0u) w = power_heuristic(prev_pdf, p_env(c) * env_pdf(c, d));
                    else if (strategy == 1u) w = 0.0f;
                }
                if (w > 0.0f) radiance = radiance + clamp_c(c, beta * le * w);
                break;
            }
            c.cnt->c[6] += 1;
            Surface surf = surface(c, hit);
            uint32_t mflags = mat_flags(c, tri_material(c, hit.slot));
            bool double_sided = (mflags & 4u) != 0u;
            Lod lod = base_lod();
            if (k == 0u) {
                float cw = P.up[3];
                if (!orthographic) cw = P.up[3] * hit.t;
                lod = {cw, d};
            }
            bool flip = !hit.front && double_sided;
            Mat mat = material(c, hit, surf, lod, flip);
            if (flip) {
                mat.normal = -mat.normal;
                mat.cc_normal = -mat.cc_normal;
            }
            if ((hit.front || double_sided) && !is_black(mat.emission)) {
                v3 le = mat.emission;
                if (k == 0u) {
                    radiance = radiance + beta * le;
                } else {
                    float pl = light_pdf(c, hit, prev_pos, surf.position);
                    float w = 1.0f;
                    if (pl > 0.0f) {
                        if (strategy == 0u) w = power_heuristic(prev_pdf, pl);
                        else if (strategy == 1u) w = 0.0f;
                    }
                    if (w > 0.0f) radiance = radiance + clamp_c(c, beta * le * w);
                }
            }
            if (mat.unlit) {
                v3 contrib = beta * mat.base.xyz();
                if (k == 0u) radiance = radiance + contrib;
                else radiance = radiance + clamp_c(c, contrib);
                break;
            }
            if (k >= P.dims[3]) break;
            bsdf = make_bsdf(c, mat, -d, surf.ng, hit.front);
            if (bsdf_black(bsdf)) break;
            p = surf.position;
            ng = bsdf.ng;
            thickness = mat.thickness;
            transmission = mat.transmission;
            atten_color = mat.atten_color;
            atten_dist = mat.atten_dist;
            front = hit.front;
            pl_u = pattern(c, s, 2u + 2u * k);
            job = 0u;
        }
        // Next NEE shadow ray.
        bool armed = false;
        uint32_t ray_id = k << 16u;
        while (job <= n_punct) {
            bool ok = false;
            v3 l = S3(0.0f);
            float tmax = INF;
            uint32_t rid = ray_id | 0xffffu;
            uint32_t skip = NONE;
            v3 le = S3(0.0f);
            float pl = -1.0f;
            if (job < n_punct) {
                LightSample ls = punctual_sample(c, job, p);
                if (ls.ok) {
                    ok = true;
                    l = ls.l;
                    if (ls.distance >= 0.0f) tmax = ls.distance * (1.0f - 1.0e-4f);
                    rid = ray_id | 0x8000u | (job & 0x7fffu);
                    le = ls.radiance;
                }
            } else if (strategy != 2u && (has_env || n_elights > 0u)) {
                float pe = p_env(c);
                if (pl_u.z < pe) {
                    if (has_env) {
                        EnvSample es = env_sample(c, pl_u.x, pl_u.y);
                        if (es.ok && pe * es.pdf > 0.0f) {
                            ok = true;
                            l = es.d;
                            le = es.le;
                            pl = pe * es.pdf;
                        }
                    }
                } else if (n_elights > 0u) {
                    float us = pl_u.z;
                    if (pe > 0.0f) us = clampf((pl_u.z - pe) / (1.0f - pe), 0.0f, 0.999999f);
                    uint32_t li = pick_elight(c, us);
                    uint32_t lslot = elight_slot(c, li);
                    v3 a = tri_pos(c, lslot, 0u), b = tri_pos(c, lslot, 1u), cc = tri_pos(c, lslot, 2u);
                    bool has_target = false;
                    v3 q = S3(0.0f);
                    if (triangle_solid_angle(c, p, a, b, cc) >= MIN_SPHERICAL_SOLID_ANGLE) {
                        v3 sl = sample_spherical_triangle(c, p, a, b, cc, pl_u.x, pl_u.y);
                        if (dot(sl, sl) > 0.0f) {
                            v3 n = cross(b - a, cc - a);
                            float dn = dot(sl, n);
                            if (dn != 0.0f) {
                                float t = dot(a - p, n) / dn;
                                if (t > 0.0f && finite(t)) {
                                    q = p + sl * t;
                                    has_target = true;
                                }
                            }
                        }
                    } else {
                        float su = std::sqrt(pl_u.x);
                        v3 w3 = V3(1.0f - su, su * (1.0f - pl_u.y), su * pl_u.y);
                        q = a * w3.x + b * w3.y + cc * w3.z;
                        has_target = true;
                    }
                    if (has_target) {
                        v3 e1 = b - a, e2 = cc - a, rr = q - a;
                        float d11 = dot(e1, e1), d12 = dot(e1, e2), d22 = dot(e2, e2);
                        float r1 = dot(rr, e1), r2 = dot(rr, e2);
                        float det = d11 * d22 - d12 * d12;
                        v3 to = q - p;
                        float dist2 = dot(to, to);
                        if (finite(det) && std::fabs(det) > 1.17549435e-38f && dist2 > 1.0e-12f) {
                            float bu = (d22 * r1 - d12 * r2) / det;
                            float bv = (d11 * r2 - d12 * r1) / det;
                            Hit lh;
                            lh.slot = lslot;
                            lh.t = std::sqrt(dist2);
                            lh.b = vclamp(V3(1.0f - bu - bv, bu, bv), S3(0.0f), S3(1.0f));
                            lh.front = true;
                            v3 lng = surface(c, lh).ng;
                            bool lds = mat_double_sided(c, tri_material(c, lslot));
                            float dist = std::sqrt(dist2);
                            v3 ld = to / dist;
                            float cos_l = -dot(lng, ld);
                            float tp = tri_pdf(c, li, lslot, p, q);
                            if ((cos_l > 0.0f || (lds && cos_l < 0.0f)) && tp > 0.0f && finite(tp)) {
                                ok = true;
                                l = ld;
                                le = emission(c, lh);
                                pl = tp;
                                tmax = fmx(dist * (1.0f - 1.0e-4f), 0.0f);
                                skip = tri_global(c, lslot);
                            }
                        }
                    }
                }
            }
            if (ok) {
                Eval e = bsdf_eval(c, bsdf, l);
                if (!is_black(e.f) && !is_black(le)) {
                    if (pl < 0.0f) {
                        pending = clamp_c(c, beta * e.f * le);
                    } else {
                        float w = 1.0f;
                        if (strategy == 0u) w = power_heuristic(pl, e.pdf);
                        pending = clamp_c(c, beta * e.f * le * (w / pl));
                    }
                    r_o = spawn(p, ng, l);
                    r_d = l;
                    r_tmax = tmax;
                    r_id = rid;
                    r_skip = skip;
                    armed = true;
                    break;
                }
            }
            job += 1u;
        }
        if (armed) {
            shadow = true;
            continue;
        }
        // BSDF sampling -> next path ray.
        v4 pb_u = pattern(c, s, 1u + 2u * k);
        BSample bs = bsdf_sample(c, bsdf, pb_u.xyz());
        if (!bs.ok) break;
        beta = beta * (bs.f * (1.0f / bs.pdf));
        if (!finite3(beta)) break;
        prev_pdf = bs.pdf;
        prev_pos = p;
        if (dot(bs.l, ng) < 0.0f && thickness > 0.0f && transmission > 0.0f) {
            if (front) {
                if (atten_dist >= 0.0f) {
                    v3 la = vmax(atten_color, S3(1.0e-6f));
                    sigma = -V3(c.LOG(la.x), c.LOG(la.y), c.LOG(la.z)) / atten_dist;
                    in_medium = true;
                } else {
                    in_medium = false;
                }
            } else {
                in_medium = false;
            }
        }
        if (k + 1u >= P.cfg[0]) {
            float q = clampf(max3(beta), 0.05f, 1.0f);
            if (q < 1.0f) {
                if (pb_u.w >= q) break;
                beta = beta * (1.0f / q);
            }
        }
        k += 1u;
        d = bs.l;
        shadow = false;
        r_o = spawn(p, ng, bs.l);
        r_d = d;
        r_tmax = INF;
        r_id = k << 16u;
        r_skip = NONE;
    }
    if (finite3(radiance)) return {true, radiance};
    return {true, S3(0.0f)};
}

void load_ctx(Ctx& c, const oxo_scene* sc, const void* params, int libm) {
    c.geom = sc->geom;
    c.geom_words = sc->geom_words;
    c.attrs = sc->attrs;
    c.tables = sc->tables;
    c.table_words = sc->table_words;
    c.atlas = sc->atlas;
    c.side = sc->atlas_side;
    c.layers = sc->atlas_layers;
    std::memcpy(&c.P, params, sizeof(Params));
    c.libm = libm != 0;
    for (uint32_t i = 0; i < 128u; i++) c.wg_sobol[i] = c.tw(c.P.offs0[0] + i);
    for (uint32_t i = 0; i < 512u; i++) c.wg_sheen[i] = c.tf(c.P.offs0[1] + i);
    c.cnt = nullptr;
}

// ---- resolve.wgsl:38-75, 138-188
float srgb_to_linear(float c, bool libm) {
    if (c <= 0.04045f) return c / 12.92f;
    return libm ? std::pow((c + 0.055f) / 1.055f, 2.4f) : fm_pow((c + 0.055f) / 1.055f, 2.4f);
}
float linear_to_srgb(float c, bool libm) {
    float x = clampf(c, 0.0f, 1.0f);
    if (x <= 0.0031308f) return 12.92f * x;
    return 1.055f * (libm ? std::pow(x, 1.0f / 2.4f) : fm_pow(x, 1.0f / 2.4f)) - 0.055f;
}
float aces(float x) {
    float y = x * 0.6f;
    return clampf((y * (2.51f * y + 0.03f)) / (y * (2.43f * y + 0.59f) + 0.14f), 0.0f, 1.0f);
}
v3 tone_map(v3 rgb_in, uint32_t op) {
    v3 rgb = vmax(rgb_in, S3(0.0f));
    if (op == 1u) {
        float l = dot(rgb, V3(0.2126f, 0.7152f, 0.0722f));
        if (l <= 0.0f) return S3(0.0f);
        return vmin(rgb / (1.0f + l), S3(1.0f));
    }
    if (op == 2u) return V3(aces(rgb.x), aces(rgb.y), aces(rgb.z));
    return vmin(rgb, S3(1.0f));
}
inline uint8_t unorm8(float v) {
    float x = clampf(v, 0.0f, 1.0f);
    return (uint8_t)(x * 255.0f + 0.5f);
}

template <class F>
void parallel_rows(uint32_t rows, int threads, F&& f) {
    if (threads <= 1 || rows < 2) {
        f(0u, rows, 0);
        return;
    }
    uint32_t nt = (uint32_t)threads < rows ? (uint32_t)threads : rows;
    std::vector<std::thread> pool;
    for (uint32_t t = 0; t < nt; t++) {
        uint32_t a = rows * t / nt, b = rows * (t + 1) / nt;
        pool.emplace_back([&, a, b, t] { f(a, b, (int)t); });
    }
    for (auto& th : pool) th.join();
}

}  // namespace

extern "C" {

int oxo_dispatch(const oxo_scene* scene, const void* params, const uint32_t frame[4], float* accum,
                 int threads, int libm, uint64_t* counters) {
    Ctx base;
    load_ctx(base, scene, params, libm);
    uint32_t w = base.P.dims[0], h = base.P.dims[1];
    uint32_t first = frame[0], count = frame[1], y0 = frame[2], rows = frame[3];
    if (threads <= 0) threads = (int)std::thread::hardware_concurrency();
    std::vector<Counters> cnts((size_t)std::max(threads, 1));
    parallel_rows(rows, threads, [&](uint32_t a, uint32_t b, int tid) {
        Ctx c = base;
        c.cnt = &cnts[(size_t)tid];
        for (uint32_t gy = a; gy < b; gy++) {
            uint32_t y = y0 + gy;
            if (y >= h) continue;
            for (uint32_t x = 0; x < w; x++) {
                size_t idx = (size_t)y * w + x;
                v4 acc = {accum[idx * 4], accum[idx * 4 + 1], accum[idx * 4 + 2], accum[idx * 4 + 3]};
                for (uint32_t i = 0; i < count; i++) {
                    c.cnt->c[0] += 1;
                    PathResult r = trace_sample(c, x, y, first + i);
                    if (r.covered) acc = acc + v4{r.radiance.x, r.radiance.y, r.radiance.z, 1.0f};
                }
                accum[idx * 4] = acc.x;
                accum[idx * 4 + 1] = acc.y;
                accum[idx * 4 + 2] = acc.z;
                accum[idx * 4 + 3] = acc.w;
            }
        }
    });
    if (counters)
        for (int k = 0; k < 8; k++) {
            counters[k] = 0;
            for (auto& cc : cnts) counters[k] += cc.c[k];
        }
    return 0;
}

void oxo_resolve(const float* accum, uint32_t w, uint32_t h, const void* rparams, int hdr_i, int libm_i,
                 void* out) {
    struct RP {
        uint32_t cfg[4];
        float exposure[4];
        float background[4];
    } p;
    std::memcpy(&p, rparams, sizeof(p));
    bool libm = libm_i != 0;
    bool hdr = hdr_i != 0;
    v3 bg_lin = V3(srgb_to_linear(p.background[0], libm), srgb_to_linear(p.background[1], libm),
                   srgb_to_linear(p.background[2], libm));
    float ba = p.background[3];
    float n = p.exposure[1];
    for (uint32_t y = 0; y < h; y++)
        for (uint32_t x = 0; x < w; x++) {
            size_t idx = (size_t)y * w + x;
            v4 a = {accum[idx * 4], accum[idx * 4 + 1], accum[idx * 4 + 2], accum[idx * 4 + 3]};
            v4 o;
            if (a.w <= 0.0f || n <= 0.0f) {
                o = {bg_lin.x, bg_lin.y, bg_lin.z, ba};
            } else {
                v3 m = a.xyz() / a.w;
                float f = clampf(a.w / n, 0.0f, 1.0f);
                v3 cc = m;
                if (!hdr) cc = tone_map(m * p.exposure[0], p.cfg[2]);
                if (f >= 1.0f) {
                    o = {cc.x, cc.y, cc.z, 1.0f};
                } else {
                    float a_sum = f + (1.0f - f) * ba;
                    if (a_sum > 0.0f) {
                        v3 r = (f * cc + (1.0f - f) * bg_lin * ba) / a_sum;
                        o = {r.x, r.y, r.z, a_sum};
                    } else {
                        v3 r = f * cc + (1.0f - f) * bg_lin;
                        o = {r.x, r.y, r.z, 0.0f};
                    }
                }
            }
            if (hdr) {
                float* of = (float*)out + idx * 4;
                of[0] = o.x;
                of[1] = o.y;
                of[2] = o.z;
                of[3] = o.w;
            } else {
                uint8_t* ob = (uint8_t*)out + idx * 4;
                ob[0] = unorm8(linear_to_srgb(o.x, libm));
                ob[1] = unorm8(linear_to_srgb(o.y, libm));
                ob[2] = unorm8(linear_to_srgb(o.z, libm));
                ob[3] = unorm8(o.w);
            }
        }
}

void oxo_sobol(const uint32_t* dirs, uint32_t seed, size_t n, const uint32_t* x, const uint32_t* y,
               const uint32_t* index, const uint32_t* pattern_id, uint32_t* out) {
    for (size_t i = 0; i < n; i++) {
        Sampler s = make_sampler(seed, x[i], y[i], index[i]);
        sobol_owen_4d_u(dirs, s.index, hash_mix(s.pixel_seed, pattern_id[i]), out + 4 * i);
    }
}

void oxo_trace_rays(const oxo_scene* scene, const void* params, size_t n, const float* rays, uint32_t flags,
                    uint32_t* slot, uint32_t* global_id, float* t, float* bary, int threads,
                    uint64_t* counters) {
    Ctx base;
    load_ctx(base, scene, params, 0);
    if (threads <= 0) threads = (int)std::thread::hardware_concurrency();
    std::vector<Counters> cnts((size_t)std::max(threads, 1));
    uint32_t chunks = (uint32_t)std::min<size_t>(n, 4096);
    parallel_rows(chunks, threads, [&](uint32_t a, uint32_t b, int tid) {
        Ctx c = base;
        c.cnt = &cnts[(size_t)tid];
        Sampler s = {0u, 0u, 0u};
        for (size_t i = n * a / chunks; i < n * b / chunks; i++) {
            const float* r = rays + i * 8;
            uint32_t skip;
            std::memcpy(&skip, &r[7], 4);
            Hit h = traverse(c, make_ray(V3(r[0], r[1], r[2]), V3(r[4], r[5], r[6])), r[3], s, 0u,
                             (flags & 2u) != 0u, (flags & 1u) != 0u, skip);
            if (slot) slot[i] = h.slot;
            if (global_id) global_id[i] = h.slot == NONE ? NONE : tri_global(c, h.slot);
            if (t) t[i] = h.slot == NONE ? 0.0f : h.t;
            if (bary) {
                bary[i * 3] = h.slot == NONE ? 0.0f : h.b.x;
                bary[i * 3 + 1] = h.slot == NONE ? 0.0f : h.b.y;
                bary[i * 3 + 2] = h.slot == NONE ? 0.0f : h.b.z;
            }
        }
    });
    if (counters)
        for (int k = 0; k < 8; k++) {
            counters[k] = 0;
            for (auto& cc : cnts) counters[k] += cc.c[k];
        }
}

uint16_t oxo_f32_to_f16(float v) {
    // src/scene.rs:242-272.
    uint32_t bits = fbits(v);
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
        bool round = rem > mid || (rem == mid && (half & 1u) == 1u);
        return (uint16_t)(sign | (uint16_t)(half + (round ? 1u : 0u)));
    }
    uint32_t half = ((uint32_t)e << 10) | (mant >> 13);
    uint32_t rem = mant & 0x1fffu;
    bool round = rem > 0x1000u || (rem == 0x1000u && (half & 1u) == 1u);
    return (uint16_t)(sign | (uint16_t)(half + (round ? 1u : 0u)));
}

void oxo_math(int op, size_t n, const float* a, const float* b, float* out, int libm) {
    Ctx c;
    c.libm = libm != 0;
    for (size_t i = 0; i < n; i++) {
        float x = a[i], y = b ? b[i] : 0.0f, r = 0.0f;
        switch (op) {
            case 0: r = c.SIN(x); break;
            case 1: r = c.COS(x); break;
            case 2: r = c.ACOS(x); break;
            case 3: r = c.ATAN2(x, y); break;
            case 4: r = c.EXP(x); break;
            case 5: r = c.LOG(x); break;
            case 6: r = c.LOG2(x); break;
            case 7: r = c.POW(x, y); break;
            default: r = 0.0f;
        }
        out[i] = r;
    }
}

}  // extern "C"
