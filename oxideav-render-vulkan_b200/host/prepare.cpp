// Scene preparation into the reference's flat buffers.
//
// Mirrors GpuPathTracer::upload / ensure_binding and their helpers
// (src/pathtrace.rs:847-1461, 1463-1627; src/scene.rs:242-272): BVH nodes
// then triangles in leaf-slot order in `geom`, 12 vec4 of attributes per
// slot, one flat `tables` word array (Sobol' directions, sheen LUT,
// texture descriptors, materials, punctual lights, emissive CDF, then the
// environment CDFs), and the shelf-packed RGBA16F atlas. Inputs the
// reference takes from its external crates (Sobol' matrices, sheen LUT,
// emissive pmf, environment CDFs, camera framing) are built here by this
// project's own rules, stated at each function; FP64 is used only for the
// emissive and environment CDFs.
#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <thread>

#include "../csrc/f16pack.h"
#include "model.hpp"

namespace oxpt {

namespace {

inline uint32_t fbits(float v) {
    uint32_t u;
    std::memcpy(&u, &v, 4);
    return u;
}

inline float fin(float v, float d) { return std::isfinite(v) ? v : d; }
inline float clamp01(float v) { return std::fmin(std::fmax(v, 0.0f), 1.0f); }

// Colour space per material texture slot (src/pathtrace.rs:1042-1096):
// base colour, emissive, specular colour and sheen colour are sRGB.
bool slot_srgb(int s) {
    return s == OXPT_SLOT_BASE || s == OXPT_SLOT_EMISSIVE || s == OXPT_SLOT_SPEC_COLOR ||
           s == OXPT_SLOT_SHEEN_COLOR;
}

// sampler_flags (src/pathtrace.rs:1317-1333).
uint32_t sampler_flags(const oxpt_sampler& s) {
    return (s.wrap_s & 3u) | (s.wrap_t & 3u) << 2 | (s.mag_linear ? 1u : 0u) << 4 |
           (s.min_filter & 7u) << 5;
}

// material_words (src/pathtrace.rs:1338-1423): the scalar part of a
// MAT_STRIDE-word record.
std::vector<uint32_t> material_words(const oxpt_material& m) {
    std::vector<uint32_t> w(MAT_STRIDE, 0);
    auto put = [&](int i, float v) { w[i] = fbits(v); };
    for (int k = 0; k < 4; k++) put(k, m.base_color[k]);
    for (int k = 0; k < 3; k++) put(4 + k, m.emissive[k]);
    uint32_t mode = m.alpha_mode == OXPT_ALPHA_MASK ? 1u : (m.alpha_mode == OXPT_ALPHA_BLEND ? 2u : 0u);
    float cutoff = m.alpha_mode == OXPT_ALPHA_MASK ? m.alpha_cutoff : 0.0f;
    put(8, m.metallic);
    put(9, m.roughness);
    put(10, m.normal_scale);
    put(11, cutoff);
    put(12, m.ior);
    float specular = 1.0f, sc[3] = {1, 1, 1};
    if (m.has_specular) {
        specular = clamp01(fin(m.specular, 1.0f));
        for (int k = 0; k < 3; k++) sc[k] = std::fmax(fin(m.specular_color[k], 1.0f), 0.0f);
    }
    put(13, specular);
    for (int k = 0; k < 3; k++) put(14 + k, sc[k]);
    put(17, m.has_transmission ? clamp01(fin(m.transmission, 0.0f)) : 0.0f);
    float thickness = 0.0f, ac[3] = {1, 1, 1}, ad = -1.0f;
    if (m.has_volume) {
        thickness = std::fmax(fin(m.thickness, 0.0f), 0.0f);
        for (int k = 0; k < 3; k++) ac[k] = clamp01(fin(m.attenuation_color[k], 1.0f));
        float d = m.attenuation_distance;
        if (std::isfinite(d) && d > 0.0f) ad = d;
    }
    put(18, thickness);
    for (int k = 0; k < 3; k++) put(19 + k, ac[k]);
    put(22, ad);
    float cc = 0.0f, ccr = 0.0f, ccs = 1.0f;
    if (m.has_clearcoat) {
        cc = clamp01(fin(m.clearcoat, 0.0f));
        ccr = clamp01(fin(m.clearcoat_roughness, 0.0f));
        ccs = fin(m.clearcoat_normal_scale, 1.0f);
    }
    put(23, cc);
    put(24, ccr);
    put(25, ccs);
    float shc[3] = {0, 0, 0}, sr = 0.0f;
    if (m.has_sheen) {
        for (int k = 0; k < 3; k++) shc[k] = clamp01(fin(m.sheen_color[k], 0.0f));
        sr = clamp01(fin(m.sheen_roughness, 0.0f));
    }
    for (int k = 0; k < 3; k++) put(26 + k, shc[k]);
    put(29, sr);
    bool emissive_lit = m.emissive[0] > 0 || m.emissive[1] > 0 || m.emissive[2] > 0;
    w[7] = mode | (m.double_sided ? 1u : 0u) << 2 | (m.unlit ? 1u : 0u) << 3 |
           (emissive_lit ? 1u : 0u) << 4;
    return w;
}

struct Rect {
    uint32_t layer, x, y, w, h;
};
struct Placed {
    uint32_t skip = 0;
    std::vector<Rect> rects;
};

}  // namespace

// ---------------------------------------------------------------------
// f32 -> f16 (src/scene.rs:242-272): round to nearest even, overflow to
// infinity, subnormals, NaN kept quiet.
// ---------------------------------------------------------------------
uint16_t f32_to_f16(float v) { return fm_f32_to_f16(v); }

// ---------------------------------------------------------------------
// Sobol' direction numbers for 4 dimensions x 32 bits, MSB-first (the
// table the reference takes from sobol_direction_numbers(), consumed by
// pathtrace.wgsl:168-183). Dimension 0 is van der Corput; dimensions 1-3
// follow Joe & Kuo's construction ("Constructing Sobol sequences with
// better two-dimensional projections", 2008) with their first three
// primitive polynomials and initial numbers: (s=1, a=0, m=1),
// (s=2, a=1, m=1,3), (s=3, a=1, m=1,3,1).
// ---------------------------------------------------------------------
void sobol_directions(uint32_t out[128]) {
    for (int k = 0; k < 32; k++) out[k] = 1u << (31 - k);
    struct Poly {
        int s;
        uint32_t a;
        uint32_t m[3];
    };
    const Poly polys[3] = {{1, 0, {1, 0, 0}}, {2, 1, {1, 3, 0}}, {3, 1, {1, 3, 1}}};
    for (int d = 0; d < 3; d++) {
        const Poly& p = polys[d];
        uint32_t v[32];
        for (int k = 0; k < 32; k++) {
            if (k < p.s) {
                v[k] = p.m[k] << (31 - k);
            } else {
                uint32_t x = v[k - p.s] ^ (v[k - p.s] >> p.s);
                for (int i = 1; i < p.s; i++)
                    if ((p.a >> (p.s - 1 - i)) & 1u) x ^= v[k - i];
                v[k] = x;
            }
        }
        for (int k = 0; k < 32; k++) out[(d + 1) * 32 + k] = v[k];
    }
}

// ---------------------------------------------------------------------
// Charlie sheen directional albedo (the reference's sheen_albedo_table(),
// consumed by pathtrace.wgsl:997-1013): entry [r][c] = integral over the
// hemisphere of D_charlie(n.h, alpha) V_neubelt(n.l, n.v) (n.l) dl with
// n.v = (c + 0.5) / 32 and alpha = max(rough^2, 1e-3), rough = r / 15.
// Midpoint quadrature in (cos theta_l, phi), float64, clamped to [0, 1].
// ---------------------------------------------------------------------
const float* sheen_albedo_lut() {
    static float lut[512];
    static std::once_flag once;
    std::call_once(once, [] {
        const double pi = 3.14159265358979323846;
        const int NU = 256, NP = 128;
        for (uint32_t r = 0; r < SHEEN_ROUGH; r++) {
            double rough = (double)r / (SHEEN_ROUGH - 1);
            double a = std::max(rough * rough, 1e-3);
            double inv = 1.0 / std::max(a, 1e-3);
            for (uint32_t c = 0; c < SHEEN_COS; c++) {
                double nv = (c + 0.5) / SHEEN_COS;
                double sv = std::sqrt(std::max(0.0, 1.0 - nv * nv));
                double sum = 0.0;
                for (int iu = 0; iu < NU; iu++) {
                    double nl = (iu + 0.5) / NU;
                    double sl = std::sqrt(std::max(0.0, 1.0 - nl * nl));
                    double vis = 1.0 / std::max(4.0 * (nl + nv - nl * nv), 1e-6);
                    double row = 0.0;
                    for (int ip = 0; ip < NP; ip++) {
                        double phi = (ip + 0.5) / NP * pi;  // symmetric: x2 below
                        // v = (sv, 0, nv), l = (sl cos phi, sl sin phi, nl)
                        double hx = sv + sl * std::cos(phi), hy = sl * std::sin(phi), hz = nv + nl;
                        double hl = std::sqrt(hx * hx + hy * hy + hz * hz);
                        double nh = hz / hl;
                        double sin2 = std::max(1.0 - nh * nh, 0.0);
                        double d = sin2 > 0 ? (2.0 + inv) * std::pow(sin2, inv * 0.5) / (2.0 * pi) : 0.0;
                        row += d;
                    }
                    sum += row * vis * nl;
                }
                double e = sum * (1.0 / NU) * (2.0 * pi / NP);
                lut[r * SHEEN_COS + c] = (float)std::min(std::max(e, 0.0), 1.0);
            }
        }
    });
    return lut;
}

// ---------------------------------------------------------------------
// Environment words (env_words, src/pathtrace.rs:1428-1461): marginal CDF
// (h + 1), conditional CDFs (h rows of w + 1), texel mass (w h), radiance
// (3 w h). The CDFs are built in float64 from luminance x sin(theta) of
// the scaled radiance; the texel mass is the pmf of a texel, so that
// env_pdf = mass w h / (2 pi^2 sin theta) (pathtrace.wgsl:1610-1618).
// ---------------------------------------------------------------------
EnvWords env_words(const Env& env) {
    EnvWords out;
    uint32_t w = std::max(env.w, 1u), h = std::max(env.h, 1u);
    out.w = w;
    out.h = h;
    const double pi = 3.14159265358979323846;
    float k = env.intensity;
    std::vector<float> rad((size_t)w * h * 3, 0.0f);
    for (size_t i = 0; i < (size_t)w * h; i++) {
        if (i * 4 + 3 > env.rgba.size()) break;
        const float* p = &env.rgba[i * 4];
        if (!(std::isfinite(p[0]) && std::isfinite(p[1]) && std::isfinite(p[2]))) continue;
        for (int c = 0; c < 3; c++) rad[i * 3 + c] = std::fmax(p[c], 0.0f) * k;
    }
    std::vector<double> wt((size_t)w * h), row(h, 0.0);
    double total = 0.0;
    for (uint32_t y = 0; y < h; y++) {
        double st = std::sin(pi * (y + 0.5) / h);
        for (uint32_t x = 0; x < w; x++) {
            const float* c = &rad[((size_t)y * w + x) * 3];
            double lum = 0.2126 * c[0] + 0.7152 * c[1] + 0.0722 * c[2];
            double v = lum * st;
            if (!(v > 0.0) || !std::isfinite(v)) v = 0.0;
            wt[(size_t)y * w + x] = v;
            row[y] += v;
        }
        total += row[y];
    }
    if (!(total > 0.0)) {
        // Black map: sample by solid angle.
        total = 0.0;
        for (uint32_t y = 0; y < h; y++) {
            double st = std::sin(pi * (y + 0.5) / h);
            row[y] = 0.0;
            for (uint32_t x = 0; x < w; x++) {
                wt[(size_t)y * w + x] = st;
                row[y] += st;
            }
            total += row[y];
        }
    }
    auto& words = out.words;
    out.marg = 0;
    double acc = 0.0;
    words.push_back(fbits(0.0f));
    for (uint32_t y = 0; y < h; y++) {
        acc += row[y];
        words.push_back(fbits(y + 1 == h ? 1.0f : (float)(acc / total)));
    }
    out.cond = (uint32_t)words.size();
    for (uint32_t y = 0; y < h; y++) {
        words.push_back(fbits(0.0f));
        double ra = 0.0;
        for (uint32_t x = 0; x < w; x++) {
            ra += wt[(size_t)y * w + x];
            float v;
            if (x + 1 == w) v = 1.0f;
            else if (row[y] > 0.0) v = (float)(ra / row[y]);
            else v = (float)((x + 1.0) / w);
            words.push_back(fbits(v));
        }
    }
    out.mass = (uint32_t)words.size();
    for (size_t i = 0; i < (size_t)w * h; i++) words.push_back(fbits((float)(wt[i] / total)));
    out.rad = (uint32_t)words.size();
    for (size_t i = 0; i < rad.size(); i++) words.push_back(fbits(rad[i]));
    return out;
}

// ---------------------------------------------------------------------
// Camera::resolve stand-in: the scene camera when asked for, otherwise a
// 45-degree pinhole on +z framing the scene bounds.
// ---------------------------------------------------------------------
// Bounds of every vertex for camera framing. A coordinate replaces the
// running bound only when strictly beyond it (NaN never does), so the
// result is the first extreme value in vertex order; pieces of the vertex
// list are bounded on several threads and combined in order by the same
// rule, which gives the same bits as one sequential pass.
Framing framing_of(const oxpt_scene& s) {
    Framing f;
    f.cameras = s.cameras;
    struct Piece {
        const float* p;
        size_t n;  // vertices
        float lo[3], hi[3];
    };
    const size_t PIECE = 1u << 18;
    std::vector<Piece> pieces;
    for (auto& m : s.meshes) {
        size_t nv = m.pos.size() / 3;
        for (size_t v = 0; v < nv; v += PIECE)
            pieces.push_back({m.pos.data() + v * 3, std::min(PIECE, nv - v), {}, {}});
    }
    if (pieces.empty()) return f;
    auto bound = [](Piece& pc) {
        float lo[3] = {1e30f, 1e30f, 1e30f}, hi[3] = {-1e30f, -1e30f, -1e30f};
        for (size_t i = 0; i < pc.n; i++)
            for (int k = 0; k < 3; k++) {
                float x = pc.p[i * 3 + k];
                lo[k] = x < lo[k] ? x : lo[k];
                hi[k] = x > hi[k] ? x : hi[k];
            }
        for (int k = 0; k < 3; k++) {
            pc.lo[k] = lo[k];
            pc.hi[k] = hi[k];
        }
    };
    unsigned threads = std::max(1u, std::min<unsigned>(8u, std::thread::hardware_concurrency()));
    threads = (unsigned)std::min<size_t>(threads, pieces.size());
    if (threads <= 1) {
        for (auto& pc : pieces) bound(pc);
    } else {
        std::vector<std::thread> pool;
        for (unsigned t = 0; t < threads; t++)
            pool.emplace_back([&, t] {
                for (size_t i = t; i < pieces.size(); i += threads) bound(pieces[i]);
            });
        for (auto& th : pool) th.join();
    }
    float lo[3] = {1e30f, 1e30f, 1e30f}, hi[3] = {-1e30f, -1e30f, -1e30f};
    for (auto& pc : pieces)
        for (int k = 0; k < 3; k++) {
            lo[k] = pc.lo[k] < lo[k] ? pc.lo[k] : lo[k];
            hi[k] = pc.hi[k] > hi[k] ? pc.hi[k] : hi[k];
        }
    f.lo = V3{lo[0], lo[1], lo[2]};
    f.hi = V3{hi[0], hi[1], hi[2]};
    return f;
}

ResolvedCamera resolve_camera(const Framing& fr, const oxpt_render_options& o, uint32_t w, uint32_t h) {
    ResolvedCamera rc;
    float aspect = (float)w / (float)std::max(h, 1u);
    oxpt_camera cam{};
    if (o.scene_camera >= 0 && (size_t)o.scene_camera < fr.cameras.size()) {
        cam = fr.cameras[o.scene_camera];
    } else {
        V3 c = (fr.lo + fr.hi) * 0.5f;
        float r = std::fmax(length(fr.hi - fr.lo) * 0.5f, 1e-3f);
        cam.yfov = 0.7853982f;
        float d = r / std::sin(cam.yfov * 0.5f);
        cam.eye[0] = c.x;
        cam.eye[1] = c.y;
        cam.eye[2] = c.z + d;
        cam.target[0] = c.x;
        cam.target[1] = c.y;
        cam.target[2] = c.z;
        cam.up[1] = 1.0f;
    }
    V3 eye{cam.eye[0], cam.eye[1], cam.eye[2]};
    V3 fwd = normalize(V3{cam.target[0], cam.target[1], cam.target[2]} - eye);
    V3 up0{cam.up[0], cam.up[1], cam.up[2]};
    if (length(up0) == 0.0f) up0 = V3{0, 1, 0};
    V3 side = normalize(cross(fwd, up0));
    if (length(side) == 0.0f) side = normalize(cross(fwd, V3{1, 0, 0}));
    V3 up = cross(side, fwd);
    rc.eye = eye;
    rc.forward = fwd;
    rc.side = side;
    rc.up = up;
    rc.ortho = cam.orthographic != 0;
    rc.half_h = rc.ortho ? cam.ymag : std::tan(cam.yfov * 0.5f);
    rc.half_w = rc.half_h * aspect;
    return rc;
}

// ---------------------------------------------------------------------
// upload (src/pathtrace.rs:970-1239).
// ---------------------------------------------------------------------
namespace {

// Level sizes of a mip chain: each level halves (at least 1) down to 1 x 1,
// as Texture::mips builds them.
std::vector<std::pair<uint32_t, uint32_t>> chain_dims(uint32_t w, uint32_t h) {
    std::vector<std::pair<uint32_t, uint32_t>> d{{w, h}};
    while (w > 1 || h > 1) {
        w = std::max(1u, w / 2);
        h = std::max(1u, h / 2);
        d.push_back({w, h});
    }
    return d;
}

}  // namespace

std::unique_ptr<SceneBuffers> upload_scene(const oxpt_scene& s, float headlight, DeviceFlatten device,
                                           void* device_arg, oxpt_status* status) {
    if (status) *status = OXPT_OK;
    auto sb = std::make_unique<SceneBuffers>();
    // Materials: meshes without one use a trailing glTF default.
    std::vector<oxpt_material> materials = s.materials;
    int32_t default_mat = -1;
    for (auto& m : s.meshes)
        if (m.material < 0 || (size_t)m.material >= s.materials.size()) {
            oxpt_material d;
            oxpt_material_default(&d);
            default_mat = (int32_t)materials.size();
            materials.push_back(d);
            break;
        }
    auto mesh_mat = [&](const Mesh& m) {
        return (m.material < 0 || (size_t)m.material >= s.materials.size()) ? (uint32_t)default_mat
                                                                            : (uint32_t)m.material;
    };
    size_t ntri = 0;
    for (auto& m : s.meshes) ntri += m.ntri;
    if (ntri == 0) device = nullptr;  // nothing to build on the device
    // Emissive lights: non-unlit triangles with a positive emissive factor
    // and area; pmf proportional to area x mean emissive factor (float64).
    // Global ids run through the meshes in order.
    std::vector<uint32_t> light_tris;
    std::vector<double> power;
    {
        uint32_t g = 0;
        for (auto& mesh : s.meshes) {
            const oxpt_material& m = materials[mesh_mat(mesh)];
            if (m.unlit || !(m.emissive[0] > 0 || m.emissive[1] > 0 || m.emissive[2] > 0)) {
                g += mesh.ntri;
                continue;
            }
            double le = (std::fmax(m.emissive[0], 0.0f) + std::fmax(m.emissive[1], 0.0f) +
                         std::fmax(m.emissive[2], 0.0f)) / 3.0;
            for (uint32_t t = 0; t < mesh.ntri; t++, g++) {
                const float* p = &mesh.pos[(size_t)t * 9];
                double e1[3], e2[3];
                for (int k = 0; k < 3; k++) {
                    e1[k] = (double)p[3 + k] - p[k];
                    e2[k] = (double)p[6 + k] - p[k];
                }
                double cx = e1[1] * e2[2] - e1[2] * e2[1], cy = e1[2] * e2[0] - e1[0] * e2[2],
                       cz = e1[0] * e2[1] - e1[1] * e2[0];
                double area = 0.5 * std::sqrt(cx * cx + cy * cy + cz * cz);
                if (!(area > 0.0) || !(le > 0.0)) continue;
                light_tris.push_back(g);
                power.push_back(area * le);
            }
        }
    }
    double total_power = 0.0;
    for (double p : power) total_power += p;

    // Atlas placement: shelf-pack every kept level, tallest first
    // (AtlasBuilder::pack, src/pathtrace.rs:1512-1592). Only level sizes
    // are needed here; texels are written below (host) or on the device.
    std::map<std::pair<int32_t, bool>, uint32_t> descs;  // texture descriptors keyed by (texture, sRGB)
    for (auto& m : materials)
        for (int sl = 0; sl < OXPT_SLOT_COUNT; sl++) {
            int32_t ti = m.tex[sl].texture;
            if (ti >= 0 && (size_t)ti < s.textures.size()) descs[{ti, slot_srgb(sl)}] = 0;
        }
    std::vector<std::pair<int32_t, bool>> chains;
    for (auto& kv : descs) chains.push_back(kv.first);
    uint32_t biggest = 1;
    for (auto& c : chains) {
        const Texture& tx = s.textures[c.first];
        biggest = std::max(biggest, std::max(tx.w, tx.h));
    }
    uint32_t side = 1;
    while (side < biggest) side <<= 1;
    side = std::min(std::max(side, 1u), MAX_LAYER);
    struct Item {
        uint32_t ci, li, w, h;
    };
    std::vector<Item> items;
    std::vector<Placed> placed(chains.size());
    std::vector<uint32_t> chain_levels(chains.size());
    for (uint32_t ci = 0; ci < chains.size(); ci++) {
        const Texture& tx = s.textures[chains[ci].first];
        auto dims = chain_dims(tx.w, tx.h);
        chain_levels[ci] = (uint32_t)dims.size();
        uint32_t skip = 0;
        while (skip < dims.size() && (dims[skip].first > side || dims[skip].second > side)) skip++;
        placed[ci].skip = skip;
        for (uint32_t li = skip; li < dims.size(); li++) items.push_back({ci, li, dims[li].first, dims[li].second});
    }
    std::stable_sort(items.begin(), items.end(), [](const Item& a, const Item& b) {
        if (a.h != b.h) return a.h > b.h;
        return a.w > b.w;
    });
    uint32_t layer = 0, x = 0, y = 0, shelf = 0;
    struct Placement {
        uint32_t ci, li;
        Rect r;
    };
    std::vector<Placement> rects;
    for (auto& it : items) {
        if (x + it.w > side) {
            x = 0;
            y += shelf;
            shelf = 0;
        }
        if (y + it.h > side) {
            layer++;
            x = 0;
            y = 0;
            shelf = 0;
        }
        rects.push_back({it.ci, it.li, Rect{layer, x, y, it.w, it.h}});
        x += it.w;
        shelf = std::max(shelf, it.h);
    }
    uint32_t layers = layer + 1;
    std::stable_sort(rects.begin(), rects.end(), [](const Placement& a, const Placement& b) {
        if (a.ci != b.ci) return a.ci < b.ci;
        return a.li < b.li;
    });
    for (auto& pl : rects) placed[pl.ci].rects.push_back(pl.r);
    sb->atlas_side = side;
    sb->atlas_layers = layers;

    std::vector<uint32_t> light_slot(light_tris.size(), NONE);
    if (device) {
        // BVH, slot flattening and atlas texels on the device.
        std::vector<oxpt_mesh_src> msrc;
        msrc.reserve(s.meshes.size());
        for (auto& m : s.meshes) {
            oxpt_mesh_src d{};
            d.ntri = m.ntri;
            d.material = mesh_mat(m);
            d.pos = m.pos.data();
            d.nrm = m.nrm.empty() ? nullptr : m.nrm.data();
            d.tan = m.tan.empty() ? nullptr : m.tan.data();
            d.uv0 = m.uv0.empty() ? nullptr : m.uv0.data();
            d.uv1 = m.uv1.empty() ? nullptr : m.uv1.data();
            d.col = m.col.empty() ? nullptr : m.col.data();
            msrc.push_back(d);
        }
        std::vector<std::vector<uint32_t>> rect_words(chains.size());
        std::vector<oxpt_chain_src> csrc(chains.size());
        for (uint32_t ci = 0; ci < chains.size(); ci++) {
            const Texture& tx = s.textures[chains[ci].first];
            for (auto& r : placed[ci].rects) rect_words[ci].insert(rect_words[ci].end(), {r.layer, r.x, r.y, r.w | (r.h << 16)});
            oxpt_chain_src& c = csrc[ci];
            c.width = tx.w;
            c.height = tx.h;
            c.rgba = tx.rgba.data();
            c.srgb_decode = (chains[ci].second && tx.srgb_encoded) ? 1u : 0u;
            c.skip = placed[ci].skip;
            c.n_rects = (uint32_t)placed[ci].rects.size();
            c.rects = rect_words[ci].data();
        }
        oxpt_scene_src src{};
        src.meshes = msrc.data();
        src.n_meshes = (uint32_t)msrc.size();
        src.light_tris = light_tris.data();
        src.n_lights = (uint32_t)light_tris.size();
        src.chains = csrc.data();
        src.n_chains = (uint32_t)csrc.size();
        src.atlas_side = side;
        src.atlas_layers = layers;
        uint32_t out[3] = {0, 0, 0};
        oxpt_status st = device(src, light_slot.data(), out, device_arg);
        if (st) {
            if (status) *status = st;
            return nullptr;
        }
        sb->on_device = true;
        sb->node_count = out[0];
        sb->slot_count = out[1];
        sb->bvh_depth = out[2];
        sb->tri_base = sb->node_count * 2;
    } else {
        // Triangle soup in global-id order.
        std::vector<float> pos;
        pos.reserve(ntri * 9);
        struct Ref {
            uint32_t mesh, tri;
        };
        std::vector<Ref> refs;
        refs.reserve(ntri);
        for (uint32_t mi = 0; mi < s.meshes.size(); mi++) {
            auto& m = s.meshes[mi];
            pos.insert(pos.end(), m.pos.begin(), m.pos.begin() + (size_t)m.ntri * 9);
            for (uint32_t t = 0; t < m.ntri; t++) refs.push_back({mi, t});
        }
        std::vector<uint32_t> lookup(ntri, NONE);
        for (uint32_t li = 0; li < light_tris.size(); li++) lookup[light_tris[li]] = li;
        // BVH.
        BvhBuild bvh = build_bvh(pos);
        sb->bvh_depth = bvh.depth;
        sb->node_count = (uint32_t)(bvh.node_words.size() / 8);
        sb->tri_base = sb->node_count * 2;
        sb->slot_count = (uint32_t)bvh.slots.size();
        for (uint32_t sl = 0; sl < bvh.slots.size(); sl++) {
            uint32_t g = bvh.slots[sl];
            if (lookup[g] != NONE) light_slot[lookup[g]] = sl;
        }
        auto& geom = sb->geom;
        geom = std::move(bvh.node_words);
        geom.reserve(geom.size() + (size_t)sb->slot_count * 12);
        auto& attrs = sb->attrs;
        attrs.reserve((size_t)sb->slot_count * 48);
        for (uint32_t g : bvh.slots) {
            const float* p = &pos[(size_t)g * 9];
            const Mesh& m = s.meshes[refs[g].mesh];
            uint32_t ws[3] = {g, lookup[g], mesh_mat(m)};
            for (int v = 0; v < 3; v++) {
                geom.push_back(fbits(p[v * 3]));
                geom.push_back(fbits(p[v * 3 + 1]));
                geom.push_back(fbits(p[v * 3 + 2]));
                geom.push_back(ws[v]);
            }
            // push_attrs (src/pathtrace.rs:1274-1315).
            uint32_t t = refs[g].tri;
            bool normals = !m.nrm.empty(), tangents = !m.tan.empty(), colors = !m.col.empty();
            bool uv0 = !m.uv0.empty(), uv1 = !m.uv1.empty();
            uint32_t flags = (normals ? 1u : 0u) | (tangents ? 1u : 0u) << 1 | (colors ? 1u : 0u) << 2 |
                             (uv0 ? 1u : 0u) << 3 | (uv1 ? 1u : 0u) << 4;
            float flagf;
            std::memcpy(&flagf, &flags, 4);
            for (int v = 0; v < 3; v++) {
                for (int k = 0; k < 3; k++) attrs.push_back(normals ? m.nrm[(size_t)t * 9 + v * 3 + k] : 0.0f);
                attrs.push_back(v == 0 ? flagf : 0.0f);
            }
            for (int v = 0; v < 3; v++)
                for (int k = 0; k < 4; k++) attrs.push_back(tangents ? m.tan[(size_t)t * 12 + v * 4 + k] : 0.0f);
            for (int v = 0; v < 3; v++) {
                attrs.push_back(uv0 ? m.uv0[(size_t)t * 6 + v * 2] : 0.0f);
                attrs.push_back(uv0 ? m.uv0[(size_t)t * 6 + v * 2 + 1] : 0.0f);
                attrs.push_back(uv1 ? m.uv1[(size_t)t * 6 + v * 2] : 0.0f);
                attrs.push_back(uv1 ? m.uv1[(size_t)t * 6 + v * 2 + 1] : 0.0f);
            }
            for (int v = 0; v < 3; v++)
                for (int k = 0; k < 4; k++) attrs.push_back(colors ? m.col[(size_t)t * 12 + v * 4 + k] : 1.0f);
        }
        if (geom.empty()) geom.resize(8, 0);
        if (attrs.empty()) attrs.resize(48, 0.0f);
        // Atlas texels.
        sb->atlas.assign((size_t)side * side * 4 * layers, 0);
        for (auto& pl : rects) {
            const auto& mips = s.textures[chains[pl.ci].first].mips(chains[pl.ci].second);
            const Mip& m = mips[pl.li];
            uint16_t* dst = &sb->atlas[(size_t)pl.r.layer * side * side * 4];
            for (uint32_t row = 0; row < pl.r.h; row++)
                for (uint32_t col = 0; col < pl.r.w; col++) {
                    const float* tx = &m.texels[((size_t)row * pl.r.w + col) * 4];
                    size_t at = (((size_t)(pl.r.y + row)) * side + pl.r.x + col) * 4;
                    for (int c = 0; c < 4; c++) dst[at + c] = f32_to_f16(tx[c]);
                }
        }
    }

    // ---- Tables.
    auto& t = sb->tables;
    sb->off_sobol = (uint32_t)t.size();
    uint32_t dirs[128];
    sobol_directions(dirs);
    t.insert(t.end(), dirs, dirs + 128);
    sb->off_sheen = (uint32_t)t.size();
    const float* lut = sheen_albedo_lut();
    for (int i = 0; i < 512; i++) t.push_back(fbits(lut[i]));
    // Texture descriptors, in key order.
    for (uint32_t ci = 0; ci < chains.size(); ci++) {
        const Texture& tx = s.textures[chains[ci].first];
        descs[chains[ci]] = (uint32_t)t.size();
        t.insert(t.end(), {chain_levels[ci], sampler_flags(tx.sampler), tx.w, tx.h,
                           placed[ci].skip, (uint32_t)placed[ci].rects.size(), 0u, 0u});
        for (auto& r : placed[ci].rects) t.insert(t.end(), {r.layer, r.x, r.y, r.w | (r.h << 16)});
    }
    // Materials.
    sb->off_mat = (uint32_t)t.size();
    for (auto& m : materials) {
        std::vector<uint32_t> w = material_words(m);
        for (int sl = 0; sl < OXPT_SLOT_COUNT; sl++) {
            uint32_t at = MAT_SLOTS + 8 * sl;
            int32_t ti = m.tex[sl].texture;
            auto it = (ti >= 0 && (size_t)ti < s.textures.size()) ? descs.find({ti, slot_srgb(sl)})
                                                                   : descs.end();
            if (it == descs.end()) {
                w[at] = NONE;
                continue;
            }
            w[at] = it->second;
            w[at + 1] = m.tex[sl].uv_set;
            for (int k = 0; k < 6; k++) w[at + 2 + k] = fbits(m.tex[sl].transform[k]);
        }
        t.insert(t.end(), w.begin(), w.end());
    }
    // Punctual lights (16 words each).
    sb->off_plights = (uint32_t)t.size();
    std::vector<oxpt_light> lights = s.lights;
    if (headlight > 0.0f) {
        oxpt_light l{};
        l.kind = OXPT_LIGHT_DIRECTIONAL;
        V3 d = normalize(V3{-0.3f, -1.0f, -0.6f});
        l.direction[0] = d.x;
        l.direction[1] = d.y;
        l.direction[2] = d.z;
        l.color[0] = l.color[1] = l.color[2] = 1.0f;
        l.intensity = headlight;
        lights.push_back(l);
    }
    for (auto& l : lights) {
        float base[3] = {l.color[0] * l.intensity, l.color[1] * l.intensity, l.color[2] * l.intensity};
        float cos_outer = std::cos(l.outer_cone), cos_inner = std::cos(l.inner_cone);
        float scale = 1.0f / std::fmax(cos_inner - cos_outer, 0.001f);
        float offset = -cos_outer * scale;
        t.insert(t.end(), {fbits(l.position[0]), fbits(l.position[1]), fbits(l.position[2]), l.kind,
                           fbits(l.direction[0]), fbits(l.direction[1]), fbits(l.direction[2]),
                           fbits(l.range), fbits(base[0]), fbits(base[1]), fbits(base[2]), 0u,
                           fbits(scale), fbits(offset), 0u, 0u});
    }
    sb->n_punctual = (uint32_t)lights.size();
    // Emissive triangles: {cdf, pmf, global id, slot}.
    sb->off_elights = (uint32_t)t.size();
    double acc = 0.0;
    for (uint32_t li = 0; li < light_tris.size(); li++) {
        acc += power[li];
        float cdf = li + 1 == light_tris.size() ? 1.0f : (float)(acc / total_power);
        float pmf = (float)(power[li] / total_power);
        t.insert(t.end(), {fbits(cdf), fbits(pmf), light_tris[li], light_slot[li]});
    }
    sb->n_emissive = (uint32_t)light_tris.size();
    return sb;
}

// ---------------------------------------------------------------------
// ensure_binding (src/pathtrace.rs:847-926): final tables and Params.
// ---------------------------------------------------------------------
void bind_params(const SceneBuffers& sb, const EnvWords* env, const ResolvedCamera& cam,
                 const oxpt_render_options& o, uint32_t w, uint32_t h, std::vector<uint32_t>* tables,
                 oxpt_params* P) {
    *tables = sb.tables;
    uint32_t env_base = (uint32_t)tables->size();
    if (env) tables->insert(tables->end(), env->words.begin(), env->words.end());
    if (tables->empty()) tables->push_back(0);
    bool has_env = env != nullptr;
    float p_env = has_env ? (sb.n_emissive > 0 ? 0.5f : 1.0f) : 0.0f;
    uint32_t strategy = o.strategy == OXPT_STRATEGY_LIGHT ? 1u : (o.strategy == OXPT_STRATEGY_BSDF ? 2u : 0u);
    std::memset(P, 0, sizeof(*P));
    P->eye[0] = cam.eye.x;
    P->eye[1] = cam.eye.y;
    P->eye[2] = cam.eye.z;
    P->eye[3] = cam.ortho ? 1.0f : 0.0f;
    P->forward[0] = cam.forward.x;
    P->forward[1] = cam.forward.y;
    P->forward[2] = cam.forward.z;
    P->forward[3] = cam.half_w;
    P->side[0] = cam.side.x;
    P->side[1] = cam.side.y;
    P->side[2] = cam.side.z;
    P->side[3] = cam.half_h;
    P->up[0] = cam.up.x;
    P->up[1] = cam.up.y;
    P->up[2] = cam.up.z;
    P->up[3] = 2.0f * cam.half_h / (float)h;
    P->dims[0] = w;
    P->dims[1] = h;
    P->dims[2] = o.seed;
    P->dims[3] = o.max_bounces;
    P->cfg[0] = o.rr_start;
    P->cfg[1] = strategy;
    P->cfg[2] = sb.n_punctual;
    P->cfg[3] = sb.n_emissive;
    P->env[0] = has_env ? env->w : 0;
    P->env[1] = has_env ? env->h : 0;
    P->env[2] = has_env ? 1u : 0u;
    P->env[3] = sb.node_count;
    P->offs0[0] = sb.off_sobol;
    P->offs0[1] = sb.off_sheen;
    P->offs0[2] = sb.off_mat;
    P->offs0[3] = sb.off_plights;
    P->offs1[0] = sb.off_elights;
    P->offs1[1] = 0;
    P->offs1[2] = has_env ? env_base + env->marg : 0;
    P->offs1[3] = has_env ? env_base + env->cond : 0;
    P->offs2[0] = has_env ? env_base + env->mass : 0;
    P->offs2[1] = has_env ? env_base + env->rad : 0;
    P->offs2[2] = sb.tri_base;
    P->offs2[3] = 0;
    P->fparams[0] = std::isfinite(o.ambient) ? std::fmax(o.ambient, 0.0f) : 0.0f;
    P->fparams[1] = o.clamp;
    P->fparams[2] = p_env;
    P->fparams[3] = 0.0f;
}

}  // namespace oxpt

// ---------------------------------------------------------------------
// C API: stand-alone preparation and exported helpers.
// ---------------------------------------------------------------------
extern "C" {

oxpt_prepared* oxpt_prepare(const oxpt_scene* scene, const oxpt_render_options* opts,
                            const oxpt_env* env) {
    auto* p = new oxpt_prepared();
    p->sb = oxpt::upload_scene(*scene, opts->light_intensity);
    uint32_t w = std::max(opts->width, 1u), h = std::max(opts->height, 1u);
    oxpt::ResolvedCamera cam = oxpt::resolve_camera(oxpt::framing_of(*scene), *opts, w, h);
    oxpt::EnvWords ew;
    if (env) ew = oxpt::env_words(env->env);
    oxpt::bind_params(*p->sb, env ? &ew : nullptr, cam, *opts, w, h, &p->tables, &p->params);
    return p;
}

void oxpt_prepared_view_of(const oxpt_prepared* p, oxpt_prepared_view* v) {
    std::memset(v, 0, sizeof(*v));
    v->geom = p->sb->geom.data();
    v->geom_words = p->sb->geom.size();
    v->attrs = p->sb->attrs.data();
    v->attr_floats = p->sb->attrs.size();
    v->tables = p->tables.data();
    v->table_words = p->tables.size();
    v->atlas = p->sb->atlas.data();
    v->atlas_side = p->sb->atlas_side;
    v->atlas_layers = p->sb->atlas_layers;
    v->node_count = p->sb->node_count;
    v->slot_count = p->sb->slot_count;
    v->params = p->params;
    v->bvh_depth = p->sb->bvh_depth;
}

void oxpt_prepared_free(oxpt_prepared* p) { delete p; }

uint16_t oxpt_f32_to_f16(float v) { return oxpt::f32_to_f16(v); }
void oxpt_sobol_directions(uint32_t out[128]) { oxpt::sobol_directions(out); }
void oxpt_sheen_albedo_table(float out[512]) {
    std::memcpy(out, oxpt::sheen_albedo_lut(), 512 * sizeof(float));
}

}  // extern "C"
