// GpuPathTracer: the reference's progressive host driver
// (src/pathtrace.rs:186-1264) on top of the oxpt.h C ABI. Same reset rules:
// re-prepare when the scene was invalidated or a preparation input
// changed, reset the accumulation when anything affecting radiance
// changed, never for display-only options (background, tone map, exposure,
// sample target). Sample indices continue from samples(), so
// refine(a); refine(b) takes exactly the samples of refine(a + b).
#include <algorithm>
#include <cstring>
#include <optional>
#include <string>

#include "../../include/oxpt_batch.h"
#include "../../include/oxpt_serve.h"
#include "../../include/oxpt_nrc.h"
#include "model.hpp"

namespace {

// radiance_key: every option that changes the converged image. The
// reference takes it from oxideav-render (src/pathtrace.rs:529); the
// display-only options are left out, as its reset test requires
// (tests/pathtrace.rs:451-496).
struct RadianceKey {
    uint32_t width, height;
    int32_t scene_camera;
    float ambient, light_intensity, clamp;
    uint32_t max_bounces, rr_start, seed, strategy;
    bool operator==(const RadianceKey& o) const { return std::memcmp(this, &o, sizeof(*this)) == 0; }
};
RadianceKey radiance_key(const oxpt_render_options& o) {
    RadianceKey k;
    std::memset(&k, 0, sizeof(k));
    k.width = o.width;
    k.height = o.height;
    k.scene_camera = o.scene_camera;
    k.ambient = o.ambient;
    k.light_intensity = o.light_intensity;
    k.clamp = o.clamp;
    k.max_bounces = o.max_bounces;
    k.rr_start = o.rr_start;
    k.seed = o.seed;
    k.strategy = o.strategy;
    return k;
}

uint32_t tone_map_code(uint32_t t) { return t == OXPT_TONEMAP_REINHARD ? 1u : (t == OXPT_TONEMAP_ACES ? 2u : 0u); }

constexpr uint32_t MAX_DIM = 32768;

}  // namespace

struct oxpt_tracer {
    oxpt_ctx* ctx = nullptr;
    std::string err;
    oxpt_render_options opts{};
    std::optional<float> prep;  // PrepareOptions: the headlight intensity
    bool dirty = true;
    std::shared_ptr<oxpt::SceneBuffers> scene;
    // A view shares `owner`'s prepared scene and device buffers and never
    // prepares itself (serving sessions); `cam` overrides the camera.
    const oxpt_tracer* owner = nullptr;
    std::optional<oxpt_camera> cam;
    bool gpu_prepare = true;  // BVH, slot flattening and atlas built on the context's GPU
    oxpt::Framing framing;
    std::optional<oxpt::Env> env;
    std::optional<oxpt::EnvWords> env_words;
    std::optional<oxpt::ResolvedCamera> camera;
    uint32_t w = 1, h = 1;
    bool has_accum = false;
    bool binding = false;
    std::vector<uint32_t> tables;
    oxpt_params params{};
    uint32_t samples = 0;

    oxpt_status check(oxpt_status s) {
        if (s != OXPT_OK) err = oxpt_last_error(ctx);
        return s;
    }
    oxpt_status fail(oxpt_status s, const std::string& m) {
        err = m;
        return s;
    }

    oxpt_status reset() {
        samples = 0;
        if (has_accum) return check(oxpt_reset(ctx));
        return OXPT_OK;
    }

    static oxpt_status device_flatten(const oxpt_scene_src& src, uint32_t* light_slots, uint32_t out[3], void* arg) {
        auto* t = static_cast<oxpt_tracer*>(arg);
        return t->check(oxpt_build_scene(t->ctx, &src, light_slots, out));
    }

    oxpt_status upload(const oxpt_scene& s, float headlight) {
        std::unique_ptr<oxpt::SceneBuffers> sb;
        if (gpu_prepare) {
            oxpt_status st = OXPT_OK;
            sb = oxpt::upload_scene(s, headlight, &device_flatten, this, &st);
            if (sb && sb->on_device) {
                framing = oxpt::framing_of(s);
                scene = std::move(sb);
                return OXPT_OK;
            }
            // A scene without triangles comes back prepared on the host and
            // is uploaded below; sources beyond the device build's limits
            // (OXPT_E_LIMIT) are prepared by the host; any other failure is
            // the device's and is reported.
            if (!sb && st != OXPT_E_LIMIT) return st;
        }
        if (!sb) sb = oxpt::upload_scene(s, headlight);
        oxpt_scene_desc d;
        d.geom = sb->geom.data();
        d.geom_words = sb->geom.size();
        d.attrs = sb->attrs.data();
        d.attr_floats = sb->attrs.size();
        d.atlas = sb->atlas.data();
        d.atlas_side = sb->atlas_side;
        d.atlas_layers = sb->atlas_layers;
        d.node_count = sb->node_count;
        d.slot_count = sb->slot_count;
        oxpt_status st = check(oxpt_upload_scene(ctx, &d));
        if (st) return st;
        framing = oxpt::framing_of(s);
        // The flat buffers stay on the host only for oxpt_tracer_prepared.
        scene = std::move(sb);
        return OXPT_OK;
    }

    // s may be null for a view (which never prepares).
    oxpt_status sync(const oxpt_scene* s, const oxpt_render_options& o, bool* did_reset) {
        *did_reset = false;
        float p = o.light_intensity;
        bool need_prepare = dirty || !scene || !prep || *prep != p;
        if ((owner || !s) && need_prepare)
            return fail(OXPT_E_INVALID, "a view cannot prepare: its owner's scene and light intensity are fixed");
        bool changed = need_prepare || !(radiance_key(o) == radiance_key(opts));
        opts = o;
        if (!changed) return OXPT_OK;
        uint32_t width = std::max(o.width, 1u), height = std::max(o.height, 1u);
        if (width > MAX_DIM || height > MAX_DIM)
            return fail(OXPT_E_INVALID, std::to_string(width) + "x" + std::to_string(height) +
                                            " exceeds the tracer's " + std::to_string(MAX_DIM) + " maximum side");
        if (need_prepare) {
            oxpt_status st = upload(*s, p);
            if (st) return st;
            prep = p;
            dirty = false;
        }
        camera = resolve(o, width, height);
        if (w != width || h != height || !has_accum) {
            w = width;
            h = height;
            oxpt_status st = check(oxpt_resize(ctx, w, h));
            if (st) return st;
            has_accum = true;
        }
        binding = false;
        oxpt_status st = reset();
        if (st) return st;
        *did_reset = true;
        return OXPT_OK;
    }

    oxpt::ResolvedCamera resolve(const oxpt_render_options& o, uint32_t width, uint32_t height) const {
        if (!cam) return oxpt::resolve_camera(framing, o, width, height);
        oxpt::Framing f = framing;
        f.cameras = {*cam};
        oxpt_render_options oc = o;
        oc.scene_camera = 0;
        return oxpt::resolve_camera(f, oc, width, height);
    }

    oxpt_status ensure_binding() {
        if (binding) return OXPT_OK;
        if (env && !env_words) env_words = oxpt::env_words(*env);
        oxpt::bind_params(*scene, env ? &*env_words : nullptr, *camera, opts, w, h, &tables, &params);
        oxpt_status st;
        if (owner && owner->binding && owner->tables == tables) {
            st = check(oxpt_share_tables(ctx, owner->ctx));  // the owner's resident tables
        } else {
            st = check(oxpt_set_tables(ctx, tables.data(), tables.size()));
        }
        if (st) return st;
        st = check(oxpt_set_params(ctx, &params));
        if (st) return st;
        binding = true;
        return OXPT_OK;
    }

    oxpt_status refine(uint32_t n) { return refine_rows(n, 0, h); }

    oxpt_status refine_rows(uint32_t n, uint32_t y0, uint32_t rows) {
        if (!scene || n == 0) return OXPT_OK;
        if (y0 > h || rows > h - y0) return fail(OXPT_E_INVALID, "row range outside the image");
        n = std::min(n, 0xffffffffu - samples);
        oxpt_status st = ensure_binding();
        if (st) return st;
        if (rows > 0) {
            oxpt_frame f{samples, n, y0, rows};
            st = check(oxpt_dispatch(ctx, &f));
            if (st) return st;
        }
        samples += n;
        return OXPT_OK;
    }

    oxpt_resolve_params resolve_params(bool hdr) const {
        oxpt_resolve_params rp;
        rp.cfg[0] = 1;
        rp.cfg[1] = 3;
        rp.cfg[2] = tone_map_code(opts.tone_map);
        rp.cfg[3] = hdr ? 1u : 0u;
        rp.exposure[0] = std::fmax(opts.exposure, 0.0f);
        rp.exposure[1] = (float)samples;
        rp.exposure[2] = (float)w;
        rp.exposure[3] = 0.0f;
        for (int k = 0; k < 4; k++) rp.background[k] = (float)opts.background[k] / 255.0f;
        return rp;
    }

    oxpt_status resolve(bool hdr, void* host, oxpt_devimage* dev) {
        if (!has_accum) {
            // Never synced: an all-background frame of the current size.
            oxpt_status st = check(oxpt_resize(ctx, w, h));
            if (st) return st;
            has_accum = true;
        }
        oxpt_resolve_params rp = resolve_params(hdr);
        return check(oxpt_resolve(ctx, &rp, hdr ? 1 : 0, host, dev));
    }
};

extern "C" {

oxpt_status oxpt_tracer_new(int device, oxpt_tracer** out) {
    if (!out) return OXPT_E_INVALID;
    *out = nullptr;
    oxpt_ctx* c = nullptr;
    oxpt_status s = oxpt_create(device, &c);
    if (s) return s;
    auto* t = new oxpt_tracer();
    t->ctx = c;
    *out = t;
    return OXPT_OK;
}

void oxpt_tracer_free(oxpt_tracer* t) {
    if (!t) return;
    oxpt_destroy(t->ctx);
    delete t;
}

const char* oxpt_tracer_last_error(const oxpt_tracer* t) { return t ? t->err.c_str() : "null tracer"; }
oxpt_ctx* oxpt_tracer_ctx(oxpt_tracer* t) { return t ? t->ctx : nullptr; }

void oxpt_tracer_set_environment(oxpt_tracer* t, const oxpt_env* env) {
    if (env) t->env = env->env;
    else t->env.reset();
    t->env_words.reset();
    t->binding = false;
    t->reset();
}

void oxpt_tracer_invalidate_scene(oxpt_tracer* t) { t->dirty = true; }
void oxpt_tracer_set_texture_resolver(oxpt_tracer* t) { t->dirty = true; }
oxpt_status oxpt_tracer_reset(oxpt_tracer* t) { return t->reset(); }
uint32_t oxpt_tracer_samples(const oxpt_tracer* t) { return t->samples; }
int oxpt_tracer_is_converged(const oxpt_tracer* t) { return t->samples >= t->opts.samples_per_pixel; }
void oxpt_tracer_size(const oxpt_tracer* t, uint32_t* w, uint32_t* h) {
    if (w) *w = t->w;
    if (h) *h = t->h;
}

oxpt_status oxpt_tracer_sync(oxpt_tracer* t, const oxpt_scene* scene, const oxpt_render_options* opts, int* did_reset) {
    if (!t || !scene || !opts) return OXPT_E_INVALID;
    bool r = false;
    oxpt_status s = t->sync(scene, *opts, &r);
    if (did_reset) *did_reset = r ? 1 : 0;
    return s;
}

oxpt_status oxpt_tracer_refine(oxpt_tracer* t, uint32_t n) { return t->refine(n); }
oxpt_status oxpt_tracer_refine_rows(oxpt_tracer* t, uint32_t n, uint32_t y0, uint32_t rows) {
    return t->refine_rows(n, y0, rows);
}
oxpt_status oxpt_tracers_refine_batch(oxpt_tracer* const* ts, uint32_t count, const uint32_t* samples,
                                      oxpt_ctx* exec) {
    if (count == 0) return OXPT_OK;
    if (!ts || !samples) return OXPT_E_INVALID;
    std::vector<oxpt_batch_frame> frames;
    std::vector<uint32_t> adds(count, 0);
    for (uint32_t k = 0; k < count; k++) {
        oxpt_tracer* t = ts[k];
        if (!t) return OXPT_E_INVALID;
        if (!t->scene || samples[k] == 0) continue;
        uint32_t n = std::min(samples[k], 0xffffffffu - t->samples);
        oxpt_status st = t->ensure_binding();
        if (st) return st;
        frames.push_back({t->ctx, t->samples, n, 0u, t->h});
        adds[k] = n;
    }
    if (frames.empty()) return OXPT_OK;
    oxpt_ctx* e = exec ? exec : frames[0].ctx;
    oxpt_status st = oxpt_refine_batch(e, frames.data(), (uint32_t)frames.size());
    if (st) {
        for (uint32_t k = 0; k < count; k++)
            if (adds[k]) ts[k]->err = oxpt_last_error(e);
        return st;
    }
    for (uint32_t k = 0; k < count; k++) ts[k]->samples += adds[k];
    return OXPT_OK;
}

oxpt_status oxpt_tracer_refine_nrc(oxpt_tracer* t, oxpt_nrc* nrc, uint32_t frames, const oxpt_nrc_config* cfg,
                                   float* loss) {
    if (!t || !nrc || !cfg) return OXPT_E_INVALID;
    if (!t->scene || frames == 0) return OXPT_OK;
    frames = std::min(frames, 0xffffffffu - t->samples);
    oxpt_status st = t->ensure_binding();
    if (st) return st;
    st = t->check(oxpt_nrc_refine(nrc, t->ctx, t->samples, frames, cfg, loss));
    if (st) return st;
    t->samples += frames;
    return OXPT_OK;
}

void oxpt_tracer_set_gpu_prepare(oxpt_tracer* t, int on) {
    if (!t) return;
    if ((on != 0) != t->gpu_prepare) t->dirty = true;  // the next sync prepares again
    t->gpu_prepare = on != 0;
}

oxpt_status oxpt_tracer_new_view(const oxpt_tracer* owner, oxpt_tracer** out) {
    if (!owner || !out) return OXPT_E_INVALID;
    *out = nullptr;
    if (!owner->scene || owner->owner) return OXPT_E_INVALID;
    oxpt_tracer* t = nullptr;
    oxpt_status s = oxpt_tracer_new(oxpt_ctx_device(owner->ctx), &t);
    if (s) return s;
    s = oxpt_share_scene(t->ctx, owner->ctx);
    if (s) {
        oxpt_tracer_free(t);
        return s;
    }
    t->owner = owner;
    t->scene = owner->scene;
    t->framing = owner->framing;
    t->env = owner->env;
    t->env_words = owner->env_words;
    t->prep = owner->prep;
    t->dirty = false;
    *out = t;
    return OXPT_OK;
}

oxpt_status oxpt_tracer_view_sync(oxpt_tracer* t, const oxpt_render_options* opts, int* did_reset) {
    if (!t || !opts || !t->owner) return OXPT_E_INVALID;
    bool r = false;
    oxpt_status s = t->sync(nullptr, *opts, &r);
    if (did_reset) *did_reset = r ? 1 : 0;
    return s;
}

oxpt_status oxpt_tracer_set_camera(oxpt_tracer* t, const oxpt_camera* cam) {
    if (!t) return OXPT_E_INVALID;
    if (cam) t->cam = *cam;
    else t->cam.reset();
    if (!t->scene) return OXPT_OK;
    uint32_t width = std::max(t->opts.width, 1u), height = std::max(t->opts.height, 1u);
    t->camera = t->resolve(t->opts, width, height);
    t->binding = false;
    return t->reset();  // a camera move resets the accumulation, as sync does
}

oxpt_status oxpt_tracer_finish(oxpt_tracer* t) { return t->check(oxpt_finish(t->ctx)); }
oxpt_status oxpt_tracer_image(oxpt_tracer* t, uint8_t* out) { return t->resolve(false, out, nullptr); }
oxpt_status oxpt_tracer_hdr(oxpt_tracer* t, float* out) { return t->resolve(true, out, nullptr); }
oxpt_status oxpt_tracer_image_async(oxpt_tracer* t, uint8_t* out) {
    if (!t || !out) return OXPT_E_INVALID;
    if (!t->has_accum) return t->resolve(false, out, nullptr);  // never synced: background, synchronously
    oxpt_resolve_params rp = t->resolve_params(false);
    return t->check(oxpt_resolve_async(t->ctx, &rp, 0, out));
}
oxpt_status oxpt_tracer_present_wait(oxpt_tracer* t) { return t ? t->check(oxpt_resolve_wait(t->ctx)) : OXPT_E_INVALID; }
oxpt_status oxpt_tracer_draw_texture(oxpt_tracer* t, oxpt_devimage* out) { return t->resolve(false, nullptr, out); }

oxpt_status oxpt_tracer_read_accum(oxpt_tracer* t, float* out) {
    if (!t->has_accum) return t->fail(OXPT_E_INVALID, "no accumulator before the first sync");
    return t->check(oxpt_read_accum(t->ctx, out));
}

oxpt_status oxpt_tracer_prepared(oxpt_tracer* t, oxpt_prepared_view* v) {
    if (!t || !v) return OXPT_E_INVALID;
    if (!t->scene) return t->fail(OXPT_E_INVALID, "no scene: sync first");
    oxpt_status s = t->ensure_binding();
    if (s) return s;
    if (t->scene->on_device && t->scene->geom.empty()) {
        // Built on the device: read the buffers back once.
        auto& sb = *t->scene;
        sb.geom.resize((size_t)sb.node_count * 8 + (size_t)sb.slot_count * 12);
        sb.attrs.resize((size_t)sb.slot_count * 48);
        sb.atlas.resize((size_t)sb.atlas_side * sb.atlas_side * sb.atlas_layers * 4);
        s = t->check(oxpt_read_scene(t->ctx, sb.geom.data(), sb.attrs.data(), sb.atlas.data()));
        if (s) {
            sb.geom.clear();
            return s;
        }
    }
    std::memset(v, 0, sizeof(*v));
    v->geom = t->scene->geom.data();
    v->geom_words = t->scene->geom.size();
    v->attrs = t->scene->attrs.data();
    v->attr_floats = t->scene->attrs.size();
    v->tables = t->tables.data();
    v->table_words = t->tables.size();
    v->atlas = t->scene->atlas.data();
    v->atlas_side = t->scene->atlas_side;
    v->atlas_layers = t->scene->atlas_layers;
    v->node_count = t->scene->node_count;
    v->slot_count = t->scene->slot_count;
    v->params = t->params;
    v->bvh_depth = t->scene->bvh_depth;
    return OXPT_OK;
}

oxpt_status oxpt_tracer_resolve_params(oxpt_tracer* t, int hdr, oxpt_resolve_params* out) {
    if (!t || !out) return OXPT_E_INVALID;
    *out = t->resolve_params(hdr != 0);
    return OXPT_OK;
}

}  // extern "C"
