// Scene model, procedural scenes and environment maps.
//
// The reference takes scenes as oxideav_mesh3d::Scene3D and prepares them
// with oxideav-render (external crates, not vendored). This file is the
// stand-in scene model: triangle soups with glTF materials, decoded float
// textures, punctual lights and cameras, plus the seeded procedural scenes
// the benchmarks and tests use.
#include <algorithm>
#include <cstring>
#include <unordered_map>

#include "../csrc/f16pack.h"
#include "model.hpp"

using namespace oxpt;

namespace {

float srgb_decode(float c) { return fm_srgb_decode(c); }

// splitmix64: seeded, platform-independent random numbers for the
// procedural scenes.
struct Rng {
    uint64_t s;
    explicit Rng(uint64_t seed) : s(seed) {}
    uint64_t next() {
        uint64_t z = (s += 0x9e3779b97f4a7c15ull);
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
        return z ^ (z >> 31);
    }
    float uniform() { return (float)((next() >> 40) * (1.0 / 16777216.0)); }
    float uniform(float a, float b) { return a + (b - a) * uniform(); }
};

uint32_t hash32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

// 3-D value noise in [-1, 1]: hashed lattice values, smoothstep-weighted
// trilinear interpolation.
float value_noise(float x, float y, float z, uint32_t seed) {
    float fx = std::floor(x), fy = std::floor(y), fz = std::floor(z);
    int ix = (int)fx, iy = (int)fy, iz = (int)fz;
    float tx = x - fx, ty = y - fy, tz = z - fz;
    auto sm = [](float t) { return t * t * (3.0f - 2.0f * t); };
    tx = sm(tx);
    ty = sm(ty);
    tz = sm(tz);
    auto lat = [&](int a, int b, int c) {
        uint32_t h = hash32((uint32_t)a * 73856093u ^ (uint32_t)b * 19349663u ^
                            (uint32_t)c * 83492791u ^ seed * 2654435761u);
        return (float)(h >> 8) * (2.0f / 16777216.0f) - 1.0f;
    };
    float v[8];
    for (int i = 0; i < 8; i++) v[i] = lat(ix + (i & 1), iy + ((i >> 1) & 1), iz + (i >> 2));
    float x00 = v[0] + (v[1] - v[0]) * tx, x10 = v[2] + (v[3] - v[2]) * tx;
    float x01 = v[4] + (v[5] - v[4]) * tx, x11 = v[6] + (v[7] - v[6]) * tx;
    float y0 = x00 + (x10 - x00) * ty, y1 = x01 + (x11 - x01) * ty;
    return y0 + (y1 - y0) * tz;
}

float fbm(V3 p, int octaves, uint32_t seed) {
    float sum = 0, amp = 0.5f, norm = 0, f = 1;
    for (int o = 0; o < octaves; o++) {
        sum += amp * value_noise(p.x * f, p.y * f, p.z * f, seed + o);
        norm += amp;
        amp *= 0.5f;
        f *= 2.0f;
    }
    return sum / norm;
}

void push3(std::vector<float>& v, V3 a) {
    v.push_back(a.x);
    v.push_back(a.y);
    v.push_back(a.z);
}

// Append a quad (two triangles a-b-c, a-c-d) with flat normals implied.
void quad(std::vector<float>& pos, V3 a, V3 b, V3 c, V3 d) {
    push3(pos, a);
    push3(pos, b);
    push3(pos, c);
    push3(pos, a);
    push3(pos, c);
    push3(pos, d);
}

// Box of size (sx, sy, sz) on the floor at (cx, cz) rotated by `angle`
// about +y; outward winding (front faces face out).
void box(std::vector<float>& pos, float cx, float cz, float sx, float sy, float sz, float angle,
         float y0 = 0.0f) {
    float c = std::cos(angle), s = std::sin(angle);
    auto P = [&](float x, float y, float z) {
        float lx = (x - 0.5f) * sx, lz = (z - 0.5f) * sz;
        return V3{cx + c * lx + s * lz, y0 + y * sy, cz - s * lx + c * lz};
    };
    V3 v[8];
    for (int i = 0; i < 8; i++) v[i] = P((float)(i & 1), (float)((i >> 1) & 1), (float)(i >> 2));
    // Faces wound so that cross(p1 - p0, p2 - p0) points outwards.
    quad(pos, v[0], v[2], v[3], v[1]);  // z = 0 (-z side)
    quad(pos, v[4], v[5], v[7], v[6]);  // z = 1
    quad(pos, v[0], v[1], v[5], v[4]);  // y = 0
    quad(pos, v[2], v[6], v[7], v[3]);  // y = 1
    quad(pos, v[0], v[4], v[6], v[2]);  // x = 0
    quad(pos, v[1], v[3], v[7], v[5]);  // x = 1
}

oxpt_material lambert(float r, float g, float b) {
    oxpt_material m;
    oxpt_material_default(&m);
    m.base_color[0] = r;
    m.base_color[1] = g;
    m.base_color[2] = b;
    m.metallic = 0.0f;
    m.roughness = 1.0f;
    m.has_specular = 1;
    m.specular = 0.0f;
    return m;
}

// Procedural RGBA float texture: checkers (even index) or value noise
// (odd), 2 colours derived from the index.
void procedural_texture(oxpt_scene* s, uint32_t index, uint32_t size, uint64_t seed) {
    Rng rng(seed * 7919u + index);
    float c0[3], c1[3];
    for (int k = 0; k < 3; k++) {
        c0[k] = rng.uniform(0.15f, 1.0f);
        c1[k] = rng.uniform(0.05f, 0.6f);
    }
    std::vector<float> px((size_t)size * size * 4);
    uint32_t cells = 8u << (index % 3);
    for (uint32_t y = 0; y < size; y++) {
        for (uint32_t x = 0; x < size; x++) {
            float t;
            if ((index & 1) == 0) {
                uint32_t cx = x * cells / size, cy = y * cells / size;
                t = ((cx + cy) & 1) ? 1.0f : 0.0f;
            } else {
                float u = (float)x / size * 16.0f, v = (float)y / size * 16.0f;
                t = 0.5f + 0.5f * fbm(V3{u, v, 0.37f * index}, 4, (uint32_t)(seed + index));
            }
            float* p = &px[((size_t)y * size + x) * 4];
            for (int k = 0; k < 3; k++) p[k] = c0[k] * t + c1[k] * (1.0f - t);
            p[3] = 1.0f;
        }
    }
    oxpt_sampler smp{OXPT_WRAP_REPEAT, OXPT_WRAP_REPEAT, 1, OXPT_MIN_LINEAR_MIP_LINEAR};
    oxpt_scene_add_texture(s, size, size, px.data(), 0, &smp);
}

void random_material(oxpt_material* m, Rng& rng, uint32_t mix, uint32_t idx) {
    oxpt_material_default(m);
    m->metallic = rng.uniform() < 0.3f ? 1.0f : 0.0f;
    m->roughness = rng.uniform(0.05f, 1.0f);
    for (int k = 0; k < 3; k++) m->base_color[k] = rng.uniform(0.1f, 0.9f);
    if (!mix) return;
    float u = (float)((hash32(idx * 2654435761u + 17u) >> 8) * (1.0 / 16777216.0));
    if (u < 0.2f) {
        m->metallic = 0.0f;
        m->has_transmission = 1;
        m->transmission = 1.0f;
        m->has_volume = 1;
        m->thickness = 1.0f;
        m->ior = rng.uniform(1.3f, 1.7f);
        m->attenuation_distance = rng.uniform(0.1f, 2.0f);
        for (int k = 0; k < 3; k++) m->attenuation_color[k] = rng.uniform(0.4f, 1.0f);
        m->roughness = rng.uniform(0.0f, 0.3f);
    } else if (u < 0.4f) {
        m->has_clearcoat = 1;
        m->clearcoat = rng.uniform(0.0f, 1.0f);
        m->clearcoat_roughness = rng.uniform(0.0f, 0.3f);
    } else if (u < 0.5f) {
        m->has_sheen = 1;
        for (int k = 0; k < 3; k++) m->sheen_color[k] = rng.uniform(0.2f, 1.0f);
        m->sheen_roughness = rng.uniform(0.1f, 1.0f);
        m->metallic = 0.0f;
    }
}

}  // namespace

// ---------------------------------------------------------------------
// Texture mip chains (TextureData::mips, per colour space).
// ---------------------------------------------------------------------

const std::vector<Mip>& Texture::mips(bool srgb) const {
    int k = srgb ? 1 : 0;
    if (built[k]) return chains[k];
    Mip l0;
    l0.w = w;
    l0.h = h;
    l0.texels = rgba;
    if (srgb && srgb_encoded) {
        for (size_t i = 0; i < l0.texels.size(); i += 4)
            for (int c = 0; c < 3; c++) l0.texels[i + c] = srgb_decode(l0.texels[i + c]);
    }
    chains[k].push_back(std::move(l0));
    while (chains[k].back().w > 1 || chains[k].back().h > 1) {
        const Mip& a = chains[k].back();
        Mip b;
        b.w = std::max(1u, a.w / 2);
        b.h = std::max(1u, a.h / 2);
        b.texels.resize((size_t)b.w * b.h * 4);
        for (uint32_t y = 0; y < b.h; y++) {
            for (uint32_t x = 0; x < b.w; x++) {
                uint32_t x0 = std::min(2 * x, a.w - 1), x1 = std::min(2 * x + 1, a.w - 1);
                uint32_t y0 = std::min(2 * y, a.h - 1), y1 = std::min(2 * y + 1, a.h - 1);
                for (int c = 0; c < 4; c++) {
                    float s = a.texels[((size_t)y0 * a.w + x0) * 4 + c] +
                              a.texels[((size_t)y0 * a.w + x1) * 4 + c] +
                              a.texels[((size_t)y1 * a.w + x0) * 4 + c] +
                              a.texels[((size_t)y1 * a.w + x1) * 4 + c];
                    b.texels[((size_t)y * b.w + x) * 4 + c] = s * 0.25f;
                }
            }
        }
        chains[k].push_back(std::move(b));
    }
    built[k] = true;
    return chains[k];
}

// ---------------------------------------------------------------------
// C API: scene building.
// ---------------------------------------------------------------------

extern "C" {

void oxpt_material_default(oxpt_material* m) {
    std::memset(m, 0, sizeof(*m));
    for (int k = 0; k < 4; k++) m->base_color[k] = 1.0f;
    m->metallic = 1.0f;
    m->roughness = 1.0f;
    m->normal_scale = 1.0f;
    m->alpha_cutoff = 0.5f;
    m->ior = 1.5f;
    m->specular = 1.0f;
    for (int k = 0; k < 3; k++) {
        m->specular_color[k] = 1.0f;
        m->attenuation_color[k] = 1.0f;
    }
    m->attenuation_distance = INFINITY;
    m->clearcoat_normal_scale = 1.0f;
    for (int s = 0; s < OXPT_SLOT_COUNT; s++) {
        m->tex[s].texture = -1;
        m->tex[s].transform[0] = 1.0f;
        m->tex[s].transform[4] = 1.0f;
    }
}

oxpt_scene* oxpt_scene_new(void) { return new oxpt_scene(); }
void oxpt_scene_free(oxpt_scene* s) { delete s; }

int32_t oxpt_scene_add_material(oxpt_scene* s, const oxpt_material* m) {
    s->materials.push_back(*m);
    return (int32_t)s->materials.size() - 1;
}

int32_t oxpt_scene_add_texture(oxpt_scene* s, uint32_t w, uint32_t h, const float* rgba,
                               uint32_t srgb_encoded, const oxpt_sampler* sampler) {
    if (!w || !h || !rgba) return -1;
    Texture t;
    t.w = w;
    t.h = h;
    t.rgba.assign(rgba, rgba + (size_t)w * h * 4);
    t.srgb_encoded = srgb_encoded != 0;
    t.sampler = sampler ? *sampler : oxpt_sampler{OXPT_WRAP_REPEAT, OXPT_WRAP_REPEAT, 1,
                                                  OXPT_MIN_LINEAR_MIP_LINEAR};
    s->textures.push_back(std::move(t));
    return (int32_t)s->textures.size() - 1;
}

int32_t oxpt_scene_add_mesh(oxpt_scene* s, uint32_t ntri, const float* positions,
                            const float* normals, const float* tangents, const float* uv0,
                            const float* uv1, const float* colors, int32_t material) {
    if (!positions) return -1;
    Mesh m;
    m.ntri = ntri;
    m.pos.assign(positions, positions + (size_t)ntri * 9);
    if (normals) m.nrm.assign(normals, normals + (size_t)ntri * 9);
    if (tangents) m.tan.assign(tangents, tangents + (size_t)ntri * 12);
    if (uv0) m.uv0.assign(uv0, uv0 + (size_t)ntri * 6);
    if (uv1) m.uv1.assign(uv1, uv1 + (size_t)ntri * 6);
    if (colors) m.col.assign(colors, colors + (size_t)ntri * 12);
    m.material = material;
    s->meshes.push_back(std::move(m));
    return (int32_t)s->meshes.size() - 1;
}

int32_t oxpt_scene_add_light(oxpt_scene* s, const oxpt_light* l) {
    s->lights.push_back(*l);
    return (int32_t)s->lights.size() - 1;
}

int32_t oxpt_scene_add_camera(oxpt_scene* s, const oxpt_camera* c) {
    s->cameras.push_back(*c);
    return (int32_t)s->cameras.size() - 1;
}

uint64_t oxpt_scene_triangle_count(const oxpt_scene* s) {
    uint64_t n = 0;
    for (auto& m : s->meshes) n += m.ntri;
    return n;
}

// ---------------------------------------------------------------------
// Procedural scenes.
// ---------------------------------------------------------------------

oxpt_scene* oxpt_scene_cornell(void) {
    auto* s = new oxpt_scene();
    oxpt_material white = lambert(0.73f, 0.73f, 0.73f);
    oxpt_material red = lambert(0.63f, 0.065f, 0.05f);
    oxpt_material green = lambert(0.14f, 0.45f, 0.09f);
    oxpt_material light = lambert(0.0f, 0.0f, 0.0f);
    light.emissive[0] = 17.0f;
    light.emissive[1] = 12.0f;
    light.emissive[2] = 4.0f;
    int mw = oxpt_scene_add_material(s, &white);
    int mr = oxpt_scene_add_material(s, &red);
    int mg = oxpt_scene_add_material(s, &green);
    int ml = oxpt_scene_add_material(s, &light);
    // Unit room [0,1]^3, open towards +z; walls wound to face inwards.
    std::vector<float> p;
    quad(p, {0, 0, 0}, {0, 0, 1}, {1, 0, 1}, {1, 0, 0});  // floor, normal +y
    quad(p, {0, 1, 0}, {1, 1, 0}, {1, 1, 1}, {0, 1, 1});  // ceiling, normal -y
    quad(p, {0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0});  // back wall, normal +z
    oxpt_scene_add_mesh(s, 6, p.data(), nullptr, nullptr, nullptr, nullptr, nullptr, mw);
    p.clear();
    quad(p, {0, 0, 0}, {0, 1, 0}, {0, 1, 1}, {0, 0, 1});  // left wall x=0, normal +x
    oxpt_scene_add_mesh(s, 2, p.data(), nullptr, nullptr, nullptr, nullptr, nullptr, mr);
    p.clear();
    quad(p, {1, 0, 0}, {1, 0, 1}, {1, 1, 1}, {1, 1, 0});  // right wall x=1, normal -x
    oxpt_scene_add_mesh(s, 2, p.data(), nullptr, nullptr, nullptr, nullptr, nullptr, mg);
    p.clear();
    const float pi = 3.14159265358979f;
    box(p, 0.66f, 0.62f, 0.3f, 0.3f, 0.3f, -18.0f * pi / 180.0f);  // short box
    box(p, 0.34f, 0.36f, 0.3f, 0.6f, 0.3f, 18.0f * pi / 180.0f);   // tall box
    oxpt_scene_add_mesh(s, 24, p.data(), nullptr, nullptr, nullptr, nullptr, nullptr, mw);
    p.clear();
    float y = 0.999f, a = 0.375f, b = 0.625f;
    quad(p, {a, y, a}, {b, y, a}, {b, y, b}, {a, y, b});  // emitter, normal -y
    oxpt_scene_add_mesh(s, 2, p.data(), nullptr, nullptr, nullptr, nullptr, nullptr, ml);
    oxpt_camera cam{};
    float d = 0.5f / std::tan(20.0f * pi / 180.0f);
    cam.eye[0] = 0.5f;
    cam.eye[1] = 0.5f;
    cam.eye[2] = 1.0f + d;
    cam.target[0] = 0.5f;
    cam.target[1] = 0.5f;
    cam.target[2] = 0.0f;
    cam.up[1] = 1.0f;
    cam.yfov = 40.0f * pi / 180.0f;
    oxpt_scene_add_camera(s, &cam);
    return s;
}

oxpt_scene* oxpt_scene_furnace(float rho, float le) {
    auto* s = new oxpt_scene();
    oxpt_material m = lambert(rho, rho, rho);
    m.emissive[0] = m.emissive[1] = m.emissive[2] = le;
    m.double_sided = 1;
    int mi = oxpt_scene_add_material(s, &m);
    std::vector<float> p;
    box(p, 0.0f, 0.0f, 2.0f, 2.0f, 2.0f, 0.0f, -1.0f);
    oxpt_scene_add_mesh(s, 12, p.data(), nullptr, nullptr, nullptr, nullptr, nullptr, mi);
    oxpt_camera cam{};
    cam.eye[0] = 0.2f;
    cam.eye[1] = 0.1f;
    cam.eye[2] = 0.4f;
    cam.target[0] = 0.0f;
    cam.target[1] = -0.3f;
    cam.target[2] = -1.0f;
    cam.up[1] = 1.0f;
    cam.yfov = 1.2f;
    oxpt_scene_add_camera(s, &cam);
    return s;
}

oxpt_scene* oxpt_scene_icosphere(uint32_t freq, uint64_t seed, uint32_t n_materials,
                                 uint32_t n_textures, uint32_t tex_size, uint32_t n_punctual,
                                 uint32_t n_emissive, uint32_t material_mix) {
    auto* s = new oxpt_scene();
    if (freq == 0) freq = 1;
    Rng rng(seed);
    // Icosahedron.
    const float t = (1.0f + std::sqrt(5.0f)) * 0.5f;
    V3 ico[12] = {{-1, t, 0}, {1, t, 0}, {-1, -t, 0}, {1, -t, 0}, {0, -1, t}, {0, 1, t},
                  {0, -1, -t}, {0, 1, -t}, {t, 0, -1}, {t, 0, 1}, {-t, 0, -1}, {-t, 0, 1}};
    const int faces[20][3] = {{0, 11, 5}, {0, 5, 1},  {0, 1, 7},   {0, 7, 10}, {0, 10, 11},
                              {1, 5, 9},  {5, 11, 4}, {11, 10, 2}, {10, 7, 6}, {7, 1, 8},
                              {3, 9, 4},  {3, 4, 2},  {3, 2, 6},   {3, 6, 8},  {3, 8, 9},
                              {4, 9, 5},  {2, 4, 11}, {6, 2, 10},  {8, 6, 7},  {9, 8, 1}};
    for (auto& v : ico) v = normalize(v);
    // Vertices keyed canonically by their (icosahedron vertex, weight)
    // decomposition so that edge vertices shared by two faces are computed
    // by the same expression (no cracks).
    std::unordered_map<uint64_t, uint32_t> index;
    std::vector<V3> verts, dirs;
    auto vertex = [&](int fi, uint32_t i, uint32_t j) {
        uint32_t w[3] = {freq - i - j, i, j};
        int id[3] = {faces[fi][0], faces[fi][1], faces[fi][2]};
        std::pair<int, uint32_t> c[3] = {{id[0], w[0]}, {id[1], w[1]}, {id[2], w[2]}};
        std::sort(c, c + 3);
        // Zero weights are left out: the third corner of a shared edge
        // differs between the two faces.
        uint64_t key = 0;
        for (auto& e : c)
            if (e.second) key = key * 65536u + (uint64_t)e.first * 4096u + e.second;
        auto it = index.find(key);
        if (it != index.end()) return it->second;
        V3 p{0, 0, 0};
        for (auto& e : c) {
            if (!e.second) continue;
            p = p + ico[e.first] * ((float)e.second / (float)freq);
        }
        V3 d = normalize(p);
        float r = 1.0f + 0.1f * fbm(d * 3.0f, 4, (uint32_t)seed);
        uint32_t n = (uint32_t)verts.size();
        verts.push_back(d * r);
        dirs.push_back(d);
        index.emplace(key, n);
        return n;
    };
    std::vector<uint32_t> tris;
    tris.reserve((size_t)20 * freq * freq * 3);
    for (int f = 0; f < 20; f++) {
        for (uint32_t i = 0; i < freq; i++) {
            for (uint32_t j = 0; j + i < freq; j++) {
                uint32_t a = vertex(f, i, j), b = vertex(f, i + 1, j), c = vertex(f, i, j + 1);
                tris.insert(tris.end(), {a, b, c});
                if (i + j + 1 < freq) {
                    uint32_t d = vertex(f, i + 1, j + 1);
                    tris.insert(tris.end(), {b, d, c});
                }
            }
        }
    }
    size_t ntri = tris.size() / 3;
    // Area-weighted smooth normals.
    std::vector<V3> vn(verts.size(), V3{0, 0, 0});
    for (size_t k = 0; k < ntri; k++) {
        V3 a = verts[tris[3 * k]], b = verts[tris[3 * k + 1]], c = verts[tris[3 * k + 2]];
        V3 n = cross(b - a, c - a);
        for (int e = 0; e < 3; e++) vn[tris[3 * k + e]] = vn[tris[3 * k + e]] + n;
    }
    for (auto& n : vn) n = normalize(n);
    // Textures and materials.
    for (uint32_t ti = 0; ti < n_textures; ti++) procedural_texture(s, ti, tex_size, seed);
    for (uint32_t mi = 0; mi < n_materials; mi++) {
        oxpt_material m;
        random_material(&m, rng, material_mix, mi);
        if (n_textures) {
            m.tex[OXPT_SLOT_BASE].texture = (int32_t)(mi % n_textures);
            if (mi & 1) m.tex[OXPT_SLOT_MR].texture = (int32_t)((mi / 2 + 3) % n_textures);
        }
        oxpt_scene_add_material(s, &m);
    }
    const uint32_t n_emit_mats = 4;
    int32_t emit_base = (int32_t)s->materials.size();
    for (uint32_t e = 0; e < n_emit_mats; e++) {
        oxpt_material m = lambert(0, 0, 0);
        m.emissive[0] = rng.uniform(4.0f, 12.0f);
        m.emissive[1] = rng.uniform(3.0f, 10.0f);
        m.emissive[2] = rng.uniform(2.0f, 8.0f);
        oxpt_scene_add_material(s, &m);
    }
    // Per-triangle material by hash; `n_emissive` triangles emit.
    std::vector<int32_t> tri_mat(ntri);
    for (size_t k = 0; k < ntri; k++)
        tri_mat[k] = n_materials ? (int32_t)(hash32((uint32_t)k ^ (uint32_t)seed) % n_materials) : -1;
    if (n_emissive && ntri) {
        uint32_t stride = (uint32_t)std::max<size_t>(1, ntri / n_emissive);
        for (uint32_t e = 0; e < n_emissive && (size_t)e * stride < ntri; e++) {
            size_t k = (size_t)e * stride + (hash32(e + 99u) % stride);
            if (k >= ntri) k = ntri - 1;
            tri_mat[k] = emit_base + (int32_t)(e % n_emit_mats);
        }
    }
    // Group triangles by material into meshes (soup per material).
    int32_t nm = (int32_t)s->materials.size();
    std::vector<std::vector<size_t>> by(nm + 1);
    for (size_t k = 0; k < ntri; k++) by[tri_mat[k] < 0 ? nm : tri_mat[k]].push_back(k);
    const float pi = 3.14159265358979f;
    for (int32_t mi = 0; mi <= nm; mi++) {
        auto& list = by[mi];
        if (list.empty()) continue;
        std::vector<float> pos, nrm, uv;
        pos.reserve(list.size() * 9);
        nrm.reserve(list.size() * 9);
        uv.reserve(list.size() * 6);
        for (size_t k : list) {
            float us[3], vs[3];
            for (int e = 0; e < 3; e++) {
                uint32_t v = tris[3 * k + e];
                push3(pos, verts[v]);
                push3(nrm, vn[v]);
                V3 d = dirs[v];
                us[e] = 0.5f + std::atan2(d.z, d.x) / (2.0f * pi);
                vs[e] = std::acos(std::fmax(-1.0f, std::fmin(1.0f, d.y))) / pi;
            }
            float umax = std::max(us[0], std::max(us[1], us[2]));
            for (int e = 0; e < 3; e++) {
                if (umax - us[e] > 0.5f) us[e] += 1.0f;  // seam
                uv.push_back(us[e] * 4.0f);
                uv.push_back(vs[e] * 2.0f);
            }
        }
        oxpt_scene_add_mesh(s, (uint32_t)list.size(), pos.data(), nrm.data(), nullptr, uv.data(),
                            nullptr, nullptr, mi == nm ? -1 : mi);
    }
    // Punctual lights on a shell around the sphere.
    for (uint32_t li = 0; li < n_punctual; li++) {
        oxpt_light l{};
        float z = rng.uniform(-1.0f, 1.0f), ph = rng.uniform(0.0f, 2.0f * pi);
        float rr = std::sqrt(std::fmax(0.0f, 1.0f - z * z)), dist = rng.uniform(2.2f, 4.0f);
        V3 p{rr * std::cos(ph) * dist, z * dist, rr * std::sin(ph) * dist};
        l.kind = (li % 4 == 3) ? OXPT_LIGHT_SPOT : OXPT_LIGHT_POINT;
        l.position[0] = p.x;
        l.position[1] = p.y;
        l.position[2] = p.z;
        V3 dir = normalize(-p);
        l.direction[0] = dir.x;
        l.direction[1] = dir.y;
        l.direction[2] = dir.z;
        for (int k = 0; k < 3; k++) l.color[k] = rng.uniform(0.6f, 1.0f);
        l.intensity = rng.uniform(2.0f, 10.0f);
        l.range = 0.0f;
        l.inner_cone = 0.3f;
        l.outer_cone = 0.6f;
        oxpt_scene_add_light(s, &l);
    }
    oxpt_camera cam{};
    cam.eye[0] = 0.0f;
    cam.eye[1] = 0.35f;
    cam.eye[2] = 3.1f;
    cam.up[1] = 1.0f;
    cam.yfov = 40.0f * pi / 180.0f;
    oxpt_scene_add_camera(s, &cam);
    return s;
}

oxpt_scene* oxpt_scene_box_field(uint32_t n, uint64_t seed, uint32_t material_mix) {
    auto* s = new oxpt_scene();
    Rng rng(seed);
    const uint32_t nmat = 16;
    for (uint32_t mi = 0; mi < nmat; mi++) {
        oxpt_material m;
        random_material(&m, rng, material_mix, mi + (uint32_t)seed * 131u);
        oxpt_scene_add_material(s, &m);
    }
    oxpt_material ground = lambert(0.6f, 0.6f, 0.6f);
    int mg = oxpt_scene_add_material(s, &ground);
    oxpt_material em = lambert(0, 0, 0);
    em.emissive[0] = 10.0f;
    em.emissive[1] = 9.0f;
    em.emissive[2] = 8.0f;
    int me = oxpt_scene_add_material(s, &em);
    float extent = 1.0f + 0.25f * std::sqrt((float)n);
    std::vector<float> p;
    quad(p, {-extent, 0, -extent}, {-extent, 0, extent}, {extent, 0, extent}, {extent, 0, -extent});
    oxpt_scene_add_mesh(s, 2, p.data(), nullptr, nullptr, nullptr, nullptr, nullptr, mg);
    std::vector<std::vector<float>> per(nmat);
    const float pi = 3.14159265358979f;
    for (uint32_t i = 0; i < n; i++) {
        float sx = rng.uniform(0.05f, 0.3f), sy = rng.uniform(0.05f, 0.6f), sz = rng.uniform(0.05f, 0.3f);
        float cx = rng.uniform(-extent, extent) * 0.9f, cz = rng.uniform(-extent, extent) * 0.9f;
        float ang = rng.uniform(0.0f, pi);
        box(per[i % nmat], cx, cz, sx, sy, sz, ang, rng.uniform(0.0f, 0.2f));
    }
    for (uint32_t mi = 0; mi < nmat; mi++)
        if (!per[mi].empty())
            oxpt_scene_add_mesh(s, (uint32_t)(per[mi].size() / 9), per[mi].data(), nullptr, nullptr,
                                nullptr, nullptr, nullptr, (int32_t)mi);
    p.clear();
    float hy = 3.0f, a = 0.6f;
    quad(p, {-a, hy, -a}, {a, hy, -a}, {a, hy, a}, {-a, hy, a});
    oxpt_scene_add_mesh(s, 2, p.data(), nullptr, nullptr, nullptr, nullptr, nullptr, me);
    oxpt_light l{};
    l.kind = OXPT_LIGHT_POINT;
    l.position[0] = extent * 0.5f;
    l.position[1] = 2.5f;
    l.position[2] = extent * 0.3f;
    l.color[0] = l.color[1] = l.color[2] = 1.0f;
    l.intensity = 6.0f + extent;
    oxpt_scene_add_light(s, &l);
    oxpt_camera cam{};
    cam.eye[0] = 0.0f;
    cam.eye[1] = extent * 0.9f;
    cam.eye[2] = extent * 1.6f;
    cam.up[1] = 1.0f;
    cam.yfov = 45.0f * pi / 180.0f;
    oxpt_scene_add_camera(s, &cam);
    return s;
}

// ---------------------------------------------------------------------
// Environment maps.
// ---------------------------------------------------------------------

oxpt_env* oxpt_env_new(uint32_t w, uint32_t h, const float* rgba, float intensity) {
    if (!w || !h || !rgba) return nullptr;
    auto* e = new oxpt_env();
    e->env.w = w;
    e->env.h = h;
    e->env.rgba.assign(rgba, rgba + (size_t)w * h * 4);
    e->env.intensity = intensity;
    return e;
}

oxpt_env* oxpt_env_sky(uint32_t w, uint32_t h, const float sun_dir[3], float sun_radiance) {
    std::vector<float> px((size_t)w * h * 4);
    const float pi = 3.14159265358979f;
    V3 sun = normalize(V3{sun_dir[0], sun_dir[1], sun_dir[2]});
    const float cos_sun = std::cos(1.5f * pi / 180.0f);
    for (uint32_t y = 0; y < h; y++) {
        for (uint32_t x = 0; x < w; x++) {
            float u = (x + 0.5f) / w, v = (y + 0.5f) / h;
            float th = pi * v, ph = 2.0f * pi * (u - 0.5f);
            V3 d{std::sin(th) * std::sin(ph), std::cos(th), -std::sin(th) * std::cos(ph)};
            float r, g, b;
            if (d.y >= 0.0f) {
                float t = std::pow(1.0f - d.y, 3.0f);
                r = 0.25f + 0.6f * t;
                g = 0.45f + 0.45f * t;
                b = 0.95f + 0.05f * t;
            } else {
                float t = std::fmin(1.0f, -d.y * 4.0f);
                r = 0.3f * (1 - t) + 0.12f * t;
                g = 0.28f * (1 - t) + 0.1f * t;
                b = 0.25f * (1 - t) + 0.08f * t;
            }
            if (dot(d, sun) > cos_sun) {
                r = sun_radiance;
                g = sun_radiance * 0.92f;
                b = sun_radiance * 0.8f;
            }
            float* p = &px[((size_t)y * w + x) * 4];
            p[0] = r;
            p[1] = g;
            p[2] = b;
            p[3] = 1.0f;
        }
    }
    return oxpt_env_new(w, h, px.data(), 1.0f);
}

void oxpt_env_free(oxpt_env* e) { delete e; }

void oxpt_render_options_default(oxpt_render_options* o) {
    std::memset(o, 0, sizeof(*o));
    o->width = 256;
    o->height = 256;
    o->scene_camera = 0;
    o->background[0] = 0;
    o->background[1] = 0;
    o->background[2] = 0;
    o->background[3] = 255;
    o->exposure = 1.0f;
    o->tone_map = OXPT_TONEMAP_CLAMP;
    o->ambient = 0.0f;
    o->light_intensity = 0.0f;
    o->samples_per_pixel = 16;
    o->max_bounces = 8;
    o->rr_start = 3;
    o->seed = 0;
    o->strategy = OXPT_STRATEGY_MIS;
    o->clamp = 0.0f;
}

}  // extern "C"
