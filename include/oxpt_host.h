/*
 * oxpt_host.h — host side of the B200 path tracer, above the oxpt.h ABI.
 *
 * The reference crate's host driver is Rust (src/pathtrace.rs) on top of
 * two external crates (oxideav-render, oxideav-mesh3d) that prepare scenes:
 * posing, materials, the binned-SAH BVH, emissive-light and environment
 * CDFs, Sobol' tables, the sheen LUT. No Rust toolchain exists on this
 * build's machines, so this C++ layer stands in for both: a scene model
 * and its preparation into the reference's flat buffers, and a
 * GpuPathTracer with the reference's progressive API and reset rules.
 * A Rust build keeps the external crates for preparation and binds only
 * oxpt.h; this header is what the tests and benches here drive.
 */
#ifndef OXPT_HOST_H
#define OXPT_HOST_H

#include <stddef.h>
#include <stdint.h>

#include "oxpt.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oxpt_scene oxpt_scene;
typedef struct oxpt_env oxpt_env;
typedef struct oxpt_tracer oxpt_tracer;
typedef struct oxpt_prepared oxpt_prepared;

/* ---- scene model (oxideav_mesh3d::Scene3D, reduced to what the path
 * tracer consumes) */

typedef enum { OXPT_WRAP_CLAMP = 0, OXPT_WRAP_MIRROR = 1, OXPT_WRAP_REPEAT = 2 } oxpt_wrap;
typedef enum {
    OXPT_MIN_NEAREST = 0,
    OXPT_MIN_LINEAR = 1,
    OXPT_MIN_NEAREST_MIP_NEAREST = 2,
    OXPT_MIN_LINEAR_MIP_NEAREST = 3,
    OXPT_MIN_NEAREST_MIP_LINEAR = 4,
    OXPT_MIN_LINEAR_MIP_LINEAR = 5
} oxpt_min_filter;

typedef struct oxpt_sampler {
    uint32_t wrap_s, wrap_t; /* oxpt_wrap */
    uint32_t mag_linear;     /* 1 linear, 0 nearest */
    uint32_t min_filter;     /* oxpt_min_filter */
} oxpt_sampler;

/* Texture slot order of a material record (pathtrace.wgsl:85-97). */
enum {
    OXPT_SLOT_BASE = 0,
    OXPT_SLOT_MR = 1,
    OXPT_SLOT_NORMAL = 2,
    OXPT_SLOT_EMISSIVE = 3,
    OXPT_SLOT_SPEC = 4,
    OXPT_SLOT_SPEC_COLOR = 5,
    OXPT_SLOT_TRANSMISSION = 6,
    OXPT_SLOT_THICKNESS = 7,
    OXPT_SLOT_CC = 8,
    OXPT_SLOT_CC_ROUGH = 9,
    OXPT_SLOT_CC_NORMAL = 10,
    OXPT_SLOT_SHEEN_COLOR = 11,
    OXPT_SLOT_SHEEN_ROUGH = 12,
    OXPT_SLOT_COUNT = 13
};

typedef struct oxpt_texref {
    int32_t texture;     /* -1 = none */
    uint32_t uv_set;     /* 0 or 1 */
    float transform[6];  /* KHR_texture_transform rows: u' = m0 u + m1 v + m2,
                            v' = m3 u + m4 v + m5 */
} oxpt_texref;

typedef enum { OXPT_ALPHA_OPAQUE = 0, OXPT_ALPHA_MASK = 1, OXPT_ALPHA_BLEND = 2 } oxpt_alpha_mode;

/* glTF metallic-roughness material with the KHR extensions the tracer
 * shades (specular, transmission, volume, clearcoat, sheen). `has_*` = 0
 * means the extension is absent (material_words defaults,
 * src/pathtrace.rs:1338-1423). */
typedef struct oxpt_material {
    float base_color[4];
    float emissive[3];
    float metallic, roughness, normal_scale;
    uint32_t alpha_mode;
    float alpha_cutoff;
    uint32_t double_sided, unlit;
    float ior;
    uint32_t has_specular;
    float specular, specular_color[3];
    uint32_t has_transmission;
    float transmission;
    uint32_t has_volume;
    float thickness, attenuation_color[3], attenuation_distance; /* <= 0 or inf: none */
    uint32_t has_clearcoat;
    float clearcoat, clearcoat_roughness, clearcoat_normal_scale;
    uint32_t has_sheen;
    float sheen_color[3], sheen_roughness;
    oxpt_texref tex[OXPT_SLOT_COUNT];
} oxpt_material;

typedef enum { OXPT_LIGHT_DIRECTIONAL = 0, OXPT_LIGHT_POINT = 1, OXPT_LIGHT_SPOT = 2 } oxpt_light_kind;

typedef struct oxpt_light {
    uint32_t kind;
    float position[3];
    float direction[3]; /* unit, the direction light travels */
    float color[3];
    float intensity;
    float range;        /* 0 = unlimited */
    float inner_cone, outer_cone;
} oxpt_light;

typedef struct oxpt_camera {
    float eye[3], target[3], up[3];
    float yfov;         /* radians (perspective) */
    uint32_t orthographic;
    float ymag;         /* half height (orthographic) */
} oxpt_camera;

/* Default material: glTF defaults (white, metallic 1, roughness 1). */
void oxpt_material_default(oxpt_material* m);

oxpt_scene* oxpt_scene_new(void);
void oxpt_scene_free(oxpt_scene* s);
int32_t oxpt_scene_add_material(oxpt_scene* s, const oxpt_material* m);
/* RGBA float texels, w*h*4, row-major. `srgb_encoded` = 1 when the colour
 * channels are sRGB-encoded (decoded to linear for sRGB slots). */
int32_t oxpt_scene_add_texture(oxpt_scene* s, uint32_t w, uint32_t h, const float* rgba,
                               uint32_t srgb_encoded, const oxpt_sampler* sampler);
/* Triangle soup: `ntri` triangles, 3 vertices each. positions 9/tri;
 * optional (NULL) normals 9/tri, tangents 12/tri, uv0 and uv1 6/tri,
 * colours 12/tri. */
int32_t oxpt_scene_add_mesh(oxpt_scene* s, uint32_t ntri, const float* positions,
                            const float* normals, const float* tangents, const float* uv0,
                            const float* uv1, const float* colors, int32_t material);
int32_t oxpt_scene_add_light(oxpt_scene* s, const oxpt_light* l);
int32_t oxpt_scene_add_camera(oxpt_scene* s, const oxpt_camera* c);
uint64_t oxpt_scene_triangle_count(const oxpt_scene* s);

/* Procedural scenes (seeded, deterministic). */
/* Cornell box: 5 walls, two rotated boxes (0.3 / 0.6 tall), emissive
 * 0.25 x 0.25 ceiling quad of radiance (17, 12, 4), pinhole 40 deg. */
oxpt_scene* oxpt_scene_cornell(void);
/* Displaced geodesic icosphere of frequency `freq` (20 freq^2 tris) with
 * `n_materials` materials hashed per triangle, `n_textures` procedural
 * size^2 textures with full mips, `n_punctual` lights and `n_emissive`
 * emissive triangles; `material_mix` 0 = metallic-roughness only, 1 = the
 * layered mix (20% transmission+volume, 20% clearcoat, 10% sheen). */
oxpt_scene* oxpt_scene_icosphere(uint32_t freq, uint64_t seed, uint32_t n_materials,
                                 uint32_t n_textures, uint32_t tex_size, uint32_t n_punctual,
                                 uint32_t n_emissive, uint32_t material_mix);
/* Field of `n` instanced, randomly rotated boxes (12 tris each). */
oxpt_scene* oxpt_scene_box_field(uint32_t n, uint64_t seed, uint32_t material_mix);
/* The white furnace: closed double-sided emissive Lambert cube [-1,1]^3
 * of albedo rho and emission le, camera inside. */
oxpt_scene* oxpt_scene_furnace(float rho, float le);

/* ---- environment (oxideav_render::pathtrace::EnvironmentMap) */
oxpt_env* oxpt_env_new(uint32_t w, uint32_t h, const float* rgba, float intensity);
/* Analytic sky: gradient plus a sun disk of the given direction. */
oxpt_env* oxpt_env_sky(uint32_t w, uint32_t h, const float sun_dir[3], float sun_radiance);
void oxpt_env_free(oxpt_env* e);

/* ---- render options (oxideav_render::RenderOptions) */
typedef enum { OXPT_TONEMAP_CLAMP = 0, OXPT_TONEMAP_REINHARD = 1, OXPT_TONEMAP_ACES = 2 } oxpt_tonemap;
typedef enum { OXPT_STRATEGY_MIS = 0, OXPT_STRATEGY_LIGHT = 1, OXPT_STRATEGY_BSDF = 2 } oxpt_strategy;

typedef struct oxpt_render_options {
    uint32_t width, height;
    int32_t scene_camera;      /* -1 = frame the scene bounds */
    uint8_t background[4];     /* sRGB bytes */
    float exposure;
    uint32_t tone_map;
    float ambient;
    float light_intensity;     /* headlight (directional along the view); 0 = none */
    /* path_trace */
    uint32_t samples_per_pixel;
    uint32_t max_bounces;
    uint32_t rr_start;
    uint32_t seed;
    uint32_t strategy;
    float clamp;               /* 0 = off */
} oxpt_render_options;

void oxpt_render_options_default(oxpt_render_options* o);

/* ---- prepared scene (TraceScene + upload's flat buffers) */
typedef struct oxpt_prepared_view {
    const uint32_t* geom;
    size_t geom_words;
    const float* attrs;
    size_t attr_floats;
    const uint32_t* tables;     /* scene tables + environment words */
    size_t table_words;
    const uint16_t* atlas;
    uint32_t atlas_side, atlas_layers;
    uint32_t node_count, slot_count;
    oxpt_params params;
    uint32_t bvh_depth;
} oxpt_prepared_view;

/* ---- GpuPathTracer (src/pathtrace.rs:186-1264) */
oxpt_status oxpt_tracer_new(int device, oxpt_tracer** out);
void oxpt_tracer_free(oxpt_tracer* t);
const char* oxpt_tracer_last_error(const oxpt_tracer* t);
oxpt_ctx* oxpt_tracer_ctx(oxpt_tracer* t);
void oxpt_tracer_set_environment(oxpt_tracer* t, const oxpt_env* env);
void oxpt_tracer_invalidate_scene(oxpt_tracer* t);
void oxpt_tracer_set_texture_resolver(oxpt_tracer* t);
oxpt_status oxpt_tracer_reset(oxpt_tracer* t);
uint32_t oxpt_tracer_samples(const oxpt_tracer* t);
int oxpt_tracer_is_converged(const oxpt_tracer* t);
void oxpt_tracer_size(const oxpt_tracer* t, uint32_t* w, uint32_t* h);
/* sync: *did_reset = 1 when the accumulation was reset. */
oxpt_status oxpt_tracer_sync(oxpt_tracer* t, const oxpt_scene* scene,
                             const oxpt_render_options* opts, int* did_reset);
oxpt_status oxpt_tracer_refine(oxpt_tracer* t, uint32_t samples);
/* Prepare the scene on the tracer's GPU (oxpt_build_scene: the BVH, the
 * leaf-slot flattening and the atlas texels; the same buffers as the host
 * preparation, word for word). On by default; 0 selects the host
 * preparation. Sources beyond the device build's limits (more than 2^30
 * triangles, textures wider than 65535) are prepared by the host instead.
 * Changing it makes the next sync prepare again. */
void oxpt_tracer_set_gpu_prepare(oxpt_tracer* t, int on);
/* refine() restricted to rows [y0, y0 + rows): the per-GPU share of a
 * frame split by row tiles across GPUs (sample indices and the samples()
 * count advance exactly as for refine). */
oxpt_status oxpt_tracer_refine_rows(oxpt_tracer* t, uint32_t samples, uint32_t y0, uint32_t rows);
/* refine() of several tracers at once: tracer k gets samples[k] more
 * samples over all its rows, traced as one wavefront by `exec`
 * (oxpt_refine_batch; NULL = the first tracer's context). Each tracer's
 * accumulation ends bit-identical to its own refine(samples[k]). On error
 * no tracer's sample count advances; the message is the executor's
 * oxpt_last_error. */
oxpt_status oxpt_tracers_refine_batch(oxpt_tracer* const* tracers, uint32_t count, const uint32_t* samples,
                                      oxpt_ctx* exec);
oxpt_status oxpt_tracer_finish(oxpt_tracer* t);
/* w*h*4 bytes (RGBA8, sRGB-encoded). */
oxpt_status oxpt_tracer_image(oxpt_tracer* t, uint8_t* out);
/* w*h*4 floats, scene-linear. */
oxpt_status oxpt_tracer_hdr(oxpt_tracer* t, float* out);
/* image() without waiting: the RGBA8 bytes land in `out` (keep it valid,
 * preferably pinned) while later work proceeds; oxpt_tracer_present_wait
 * returns once they have. (oxpt_resolve_async.) */
oxpt_status oxpt_tracer_image_async(oxpt_tracer* t, uint8_t* out);
oxpt_status oxpt_tracer_present_wait(oxpt_tracer* t);
oxpt_status oxpt_tracer_draw_texture(oxpt_tracer* t, oxpt_devimage* out);
oxpt_status oxpt_tracer_read_accum(oxpt_tracer* t, float* out);
/* The flat buffers and Params of the current binding (valid until the next
 * sync / set_environment). */
oxpt_status oxpt_tracer_prepared(oxpt_tracer* t, oxpt_prepared_view* out);
oxpt_status oxpt_tracer_resolve_params(oxpt_tracer* t, int hdr, oxpt_resolve_params* out);

/* Stand-alone preparation (no device): scene + options + env -> flat
 * buffers and Params, exactly as the tracer would upload them. */
oxpt_prepared* oxpt_prepare(const oxpt_scene* scene, const oxpt_render_options* opts,
                            const oxpt_env* env);
void oxpt_prepared_view_of(const oxpt_prepared* p, oxpt_prepared_view* out);
void oxpt_prepared_free(oxpt_prepared* p);

/* Host helpers restated from the reference, exported for tests. */
uint16_t oxpt_f32_to_f16(float v);                     /* src/scene.rs:242-272 */
void oxpt_sobol_directions(uint32_t out[128]);         /* 4 dims x 32 words */
void oxpt_sheen_albedo_table(float out[512]);          /* 16 rough x 32 cos */

#ifdef __cplusplus
}
#endif
#endif /* OXPT_HOST_H */
