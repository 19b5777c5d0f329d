// Internal host model: scene, textures, environment, prepared buffers.
#pragma once

#include <cmath>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "../../include/oxpt_host.h"

namespace oxpt {

constexpr uint32_t NONE = 0xffffffffu;
constexpr uint32_t MAT_STRIDE = 136;   // pathtrace.wgsl:82
constexpr uint32_t MAT_SLOTS = 32;     // pathtrace.wgsl:84
constexpr uint32_t MAX_LAYER = 4096;   // src/pathtrace.rs:86
constexpr uint32_t SHEEN_COS = 32;     // pathtrace.wgsl:71
constexpr uint32_t SHEEN_ROUGH = 16;   // pathtrace.wgsl:72

struct V3 {
    float x = 0, y = 0, z = 0;
    V3() = default;
    V3(float a, float b, float c) : x(a), y(b), z(c) {}
    float& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
    float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline float length(V3 a) { return std::sqrt(dot(a, a)); }
inline V3 normalize(V3 a) {
    float l = length(a);
    return l > 0 ? V3{a.x / l, a.y / l, a.z / l} : V3{0, 0, 0};
}
inline V3 vmin(V3 a, V3 b) { return {std::fmin(a.x, b.x), std::fmin(a.y, b.y), std::fmin(a.z, b.z)}; }
inline V3 vmax(V3 a, V3 b) { return {std::fmax(a.x, b.x), std::fmax(a.y, b.y), std::fmax(a.z, b.z)}; }

struct Mip {
    uint32_t w = 0, h = 0;
    std::vector<float> texels;  // rgba
};

struct Texture {
    uint32_t w = 0, h = 0;
    std::vector<float> rgba;
    bool srgb_encoded = false;
    oxpt_sampler sampler{};
    // Mip chains per colour space (0 linear, 1 sRGB), built on demand.
    mutable std::vector<Mip> chains[2];
    mutable bool built[2] = {false, false};
    const std::vector<Mip>& mips(bool srgb) const;
};

struct Mesh {
    uint32_t ntri = 0;
    std::vector<float> pos, nrm, tan, uv0, uv1, col;  // per vertex, 3 per triangle
    int32_t material = -1;
};

struct Env {
    uint32_t w = 1, h = 1;
    std::vector<float> rgba;
    float intensity = 1.0f;
};

}  // namespace oxpt

struct oxpt_scene {
    std::vector<oxpt_material> materials;
    std::vector<oxpt::Texture> textures;
    std::vector<oxpt::Mesh> meshes;
    std::vector<oxpt_light> lights;
    std::vector<oxpt_camera> cameras;
};

struct oxpt_env {
    oxpt::Env env;
};

namespace oxpt {

struct BvhBuild {
    std::vector<uint32_t> node_words;  // 8 words per node
    std::vector<uint32_t> slots;       // leaf slot -> global triangle id
    uint32_t depth = 0;
};

// Binned-SAH BVH over triangle boxes (the TraceScene BVH the reference
// consumes through Bvh::node_words / Bvh::triangles, src/pathtrace.rs:
// 974-977): node = {lo.xyz, first | hi.xyz, count}; inner nodes keep their
// two children adjacent at `first`, `first + 1`; the root is node 0.
BvhBuild build_bvh(const std::vector<float>& tri_pos /* 9 per tri */);

struct EnvWords {
    std::vector<uint32_t> words;
    uint32_t w = 0, h = 0, marg = 0, cond = 0, mass = 0, rad = 0;
};
EnvWords env_words(const Env& env);

struct ResolvedCamera {
    V3 eye, forward, side, up;
    float half_w = 1, half_h = 1;
    bool ortho = false;
};
// What camera resolution needs from a prepared scene: its cameras and
// bounds (the reference keeps a light copy of the PreparedScene for this,
// src/pathtrace.rs:1212-1222).
struct Framing {
    std::vector<oxpt_camera> cameras;
    V3 lo{-1, -1, -1}, hi{1, 1, 1};
};
Framing framing_of(const oxpt_scene& s);
ResolvedCamera resolve_camera(const Framing& f, const oxpt_render_options& o, uint32_t w, uint32_t h);

// Scene part of upload(): everything independent of the options except the
// headlight.
struct SceneBuffers {
    std::vector<uint32_t> geom;
    std::vector<float> attrs;
    std::vector<uint32_t> tables;
    std::vector<uint16_t> atlas;
    uint32_t atlas_side = 1, atlas_layers = 1;
    uint32_t node_count = 0, slot_count = 0, tri_base = 0;
    uint32_t n_punctual = 0, n_emissive = 0;
    uint32_t off_sobol = 0, off_sheen = 0, off_mat = 0, off_plights = 0, off_elights = 0;
    uint32_t bvh_depth = 0;
    bool on_device = false;  // geom / attrs / atlas were built on the device
};
// Builds geom / attrs / atlas on a device instead of the host
// (oxpt_build_scene): gets the scene's sources, writes the leaf slot of
// each light triangle and {node_count, slot_count, depth}.
using DeviceFlatten = oxpt_status (*)(const oxpt_scene_src& src, uint32_t* light_slots, uint32_t out[3], void* arg);
// With `device`, the BVH, slot flattening and atlas texels are built there
// (SceneBuffers::on_device; geom / attrs / atlas stay empty on the host);
// on its failure this returns null with *status set. Scenes without
// triangles are always prepared on the host.
std::unique_ptr<SceneBuffers> upload_scene(const oxpt_scene& s, float headlight, DeviceFlatten device = nullptr,
                                           void* device_arg = nullptr, oxpt_status* status = nullptr);

// ensure_binding(): final tables (scene + env) and Params.
void bind_params(const SceneBuffers& sb, const EnvWords* env, const ResolvedCamera& cam,
                 const oxpt_render_options& o, uint32_t w, uint32_t h, std::vector<uint32_t>* tables,
                 oxpt_params* params);

void sobol_directions(uint32_t out[128]);
const float* sheen_albedo_lut();  // 512 floats
uint16_t f32_to_f16(float v);

}  // namespace oxpt

struct oxpt_prepared {
    std::unique_ptr<oxpt::SceneBuffers> sb;
    std::vector<uint32_t> tables;
    oxpt_params params{};
};
