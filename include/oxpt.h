/*
 * oxpt.h — C ABI of the B200 path tracer (the `-sys` layer).
 *
 * This is the surface a Rust `oxideav-render-cuda-sys` crate binds with
 * `extern "C"` declarations. Everything the wgpu path tracer of
 * OxideAV/oxideav-render-vulkan hands to wgpu (buffers, uniforms,
 * dispatches, resolve passes and readbacks) crosses here as plain pointers
 * and sizes. No C++ or torch types appear in any signature.
 *
 * Threading: an oxpt_ctx is used by one thread at a time (the reference's
 * `&mut self` on every GpuPathTracer method). Distinct contexts may be used
 * from distinct threads. All launches go to the context's CUDA stream and
 * return without waiting, except the calls documented as blocking.
 *
 * Errors: every entry point returns an oxpt_status. A non-zero status
 * leaves a message readable with oxpt_last_error(ctx). The Rust side maps
 * OXPT_E_INVALID to Error::InvalidOptions and every other code to
 * Error::Backend (the reference's error split, src/pathtrace.rs:252-273,
 * 536-541, 567-576).
 */
#ifndef OXPT_H
#define OXPT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OXPT_ABI_VERSION 2u

typedef enum oxpt_status {
    OXPT_OK = 0,
    OXPT_E_NODEV = 1,   /* no CUDA device / wrong architecture */
    OXPT_E_NOMEM = 2,   /* device allocation failed */
    OXPT_E_LIMIT = 3,   /* a size exceeds a device or library limit */
    OXPT_E_INVALID = 4, /* bad argument (null pointer, inconsistent sizes) */
    OXPT_E_TIMEOUT = 5, /* a bounded device-side wait gave up */
    OXPT_E_CUDA = 6     /* any other CUDA runtime error */
} oxpt_status;

typedef struct oxpt_ctx oxpt_ctx;

/*
 * Per-launch uniforms. Byte-for-byte the reference's `Params`
 * (src/pathtrace.rs:100-114, pathtrace.wgsl:17-41): 11 x 16 bytes.
 *   eye      xyz eye, w = 1 for orthographic
 *   forward  xyz forward, w = half_w
 *   side     xyz side, w = half_h
 *   up       xyz up, w = pixel spread (cone width per unit distance)
 *   dims     width, height, seed, max_bounces
 *   cfg      rr_start, strategy (0 MIS, 1 light only, 2 BSDF only),
 *            punctual light count, emissive triangle count
 *   env      env width, env height, has env, BVH node count
 *   offs0    table word offsets: sobol, sheen, materials, punctual lights
 *   offs1    emissive lights, unused, env marginal, env conditional
 *   offs2    env mass, env radiance, first triangle vec4 in geom, unused
 *   fparams  ambient, clamp, P_env, unused
 */
typedef struct oxpt_params {
    float eye[4];
    float forward[4];
    float side[4];
    float up[4];
    uint32_t dims[4];
    uint32_t cfg[4];
    uint32_t env[4];
    uint32_t offs0[4];
    uint32_t offs1[4];
    uint32_t offs2[4];
    float fparams[4];
} oxpt_params;

/* One dispatch: samples [first, first + count) of rows [y0, y0 + rows).
 * The reference's `FrameParams` (src/pathtrace.rs:116-123). */
typedef struct oxpt_frame {
    uint32_t first;
    uint32_t count;
    uint32_t y0;
    uint32_t rows;
} oxpt_frame;

/* Resolve uniforms: the reference's `ResolveParams` (src/pathtrace.rs:
 * 125-131, 781-791; resolve.wgsl:18-26).
 *   cfg        x = aa (1), y = class (3), z = tone map (0 clamp,
 *              1 Reinhard, 2 ACES fitted), w = 1 for HDR output
 *   exposure   x = exposure, y = samples taken, z = width
 *   background sRGB-encoded background bytes / 255 */
typedef struct oxpt_resolve_params {
    uint32_t cfg[4];
    float exposure[4];
    float background[4];
} oxpt_resolve_params;

/*
 * Flat scene buffers, in the layouts the reference's `upload` writes
 * (src/pathtrace.rs:970-1239):
 *   geom   BVH nodes (8 words each: lo.xyz, first, hi.xyz, count) followed
 *          by the triangles in leaf-slot order (12 words each: p0.xyz,
 *          global id, p1.xyz, emissive light index or 0xffffffff, p2.xyz,
 *          material index). Float words are IEEE bit patterns.
 *   attrs  48 floats per leaf slot (normals, tangents, uv0|uv1, colours;
 *          w of the first normal = attribute flags bits).
 *   atlas  RGBA16F texels, `atlas_layers` square layers of `atlas_side`^2,
 *          layer-major then row-major, 4 halves per texel.
 * The library copies everything; the caller may free its buffers when the
 * call returns.
 */
typedef struct oxpt_scene_desc {
    const uint32_t* geom;
    size_t geom_words;
    const float* attrs;
    size_t attr_floats;
    const uint16_t* atlas;
    uint32_t atlas_side;
    uint32_t atlas_layers;
    uint32_t node_count;
    uint32_t slot_count;
} oxpt_scene_desc;

/* A headless device image (the `draw_texture` result): device pointer,
 * size and format. Valid until the next resize or destroy. */
typedef enum oxpt_format { OXPT_FORMAT_RGBA8 = 0, OXPT_FORMAT_RGBA32F = 1 } oxpt_format;
typedef struct oxpt_devimage {
    void* data;
    uint32_t width;
    uint32_t height;
    uint32_t pitch_bytes;
    uint32_t format;
} oxpt_devimage;

/* ---- context (GpuPathTracer::new / from_device, src/pathtrace.rs:309-455) */
uint32_t oxpt_abi_version(void);
oxpt_status oxpt_create(int device, oxpt_ctx** out);
oxpt_status oxpt_destroy(oxpt_ctx* ctx);
const char* oxpt_last_error(const oxpt_ctx* ctx);
/* Run on a caller's stream (a cudaStream_t passed as void*); NULL restores
 * the context's own stream. */
oxpt_status oxpt_set_stream(oxpt_ctx* ctx, void* stream);
void* oxpt_get_stream(const oxpt_ctx* ctx);
/* "<name> (sm_XX, N SMs, M MiB)" — adapter_summary (src/pathtrace.rs:464). */
oxpt_status oxpt_device_summary(const oxpt_ctx* ctx, char* buf, size_t len);

/* ---- scene + uniforms (upload, src/pathtrace.rs:970-1239; ensure_binding,
 * :847-966). `oxpt_set_tables` takes the final word array: the scene
 * tables with the environment words appended. */
oxpt_status oxpt_upload_scene(oxpt_ctx* ctx, const oxpt_scene_desc* scene);
oxpt_status oxpt_set_tables(oxpt_ctx* ctx, const uint32_t* words, size_t count);

/*
 * The next scene and its tables (oxpt_upload_scene + oxpt_set_tables in one
 * call) uploaded while work already queued on the context keeps tracing the
 * current scene: the reference's upload (src/pathtrace.rs:970-1239) waits
 * for the device, this does not. The context keeps a second set of scene
 * buffers; the copies and the upload's tree passes run on a stream of
 * their own, after the last work that traced that set. The call returns
 * once the host buffers have been read (pinned host memory makes the copies
 * asynchronous DMA); the next oxpt_refine / oxpt_dispatch on the context
 * waits for the upload on the device and traces the new scene. Params for
 * the new scene may be set before that call. oxpt_upload_scene,
 * oxpt_set_tables and oxpt_build_scene first make a staged scene current.
 * Not for contexts that lend their scene to others (oxpt_share_scene) or
 * borrow one, nor for contexts traced by another context's batches
 * (oxpt_refine_batch with a different executor): those must use
 * oxpt_upload_scene. No reference counterpart.
 */
oxpt_status oxpt_stage_scene(oxpt_ctx* ctx, const oxpt_scene_desc* scene, const uint32_t* tables,
                             size_t table_words);

/*
 * Scene preparation on the device: the buffers of oxpt_upload_scene built
 * by the GPU from the scene's sources instead of by the host. Replaces the
 * host passes of upload (src/pathtrace.rs:970-1239): the BVH the external
 * TraceScene builds (binned SAH; the tree of the host builder, node for
 * node), the leaf-slot flattening of triangles and push_attrs
 * (:1274-1315), and the texel work of AtlasBuilder (:1482-1627: the mip
 * chains, sRGB decode, f32_to_f16 into the shelf rectangles). The caller
 * keeps the cheap host parts: materials, the emissive triangle list, and
 * the atlas placement (rectangles per packed level). The device buffers
 * equal, word for word, those oxpt_upload_scene takes from the host
 * preparation of the same scene. Pointers are read during the call only.
 */
typedef struct oxpt_mesh_src {
    uint32_t ntri;
    uint32_t material;   /* material word of its triangles */
    const float* pos;    /* 9 per triangle */
    const float* nrm;    /* optional (NULL): 9 per triangle */
    const float* tan;    /* optional: 12 per triangle */
    const float* uv0;    /* optional: 6 per triangle */
    const float* uv1;    /* optional: 6 per triangle */
    const float* col;    /* optional: 12 per triangle (absent: 1.0) */
} oxpt_mesh_src;

typedef struct oxpt_chain_src {
    uint32_t width, height;  /* level 0; each next level max(1, side / 2) down to 1 x 1 */
    const float* rgba;       /* level-0 texels, RGBA, row-major */
    uint32_t srgb_decode;    /* 1: decode RGB from sRGB before building the chain */
    uint32_t skip;           /* leading levels left out of the atlas */
    uint32_t n_rects;        /* packed levels: skip .. skip + n_rects - 1 */
    const uint32_t* rects;   /* 4 words per packed level: layer, x, y, w | h << 16 */
} oxpt_chain_src;

typedef struct oxpt_scene_src {
    const oxpt_mesh_src* meshes;
    uint32_t n_meshes;        /* global triangle ids run through the meshes in order */
    const uint32_t* light_tris;
    uint32_t n_lights;        /* emissive triangles by global id; light index = position */
    const oxpt_chain_src* chains;
    uint32_t n_chains;
    uint32_t atlas_side, atlas_layers;
} oxpt_scene_src;

/* light_slots (n_lights entries, may be NULL when n_lights is 0) receives
 * the leaf slot of each light triangle (for the emissive records);
 * out = {node_count, slot_count, bvh depth}. At least one triangle. */
oxpt_status oxpt_build_scene(oxpt_ctx* ctx, const oxpt_scene_src* src, uint32_t* light_slots, uint32_t out[3]);
/* Copies the context's device scene back in the layouts of
 * oxpt_scene_desc: the whole geom buffer (node_count * 8 + slot_count * 12
 * words for a device-built scene; the uploaded words otherwise), attrs
 * (slot_count * 48 floats) and the atlas (side^2 * layers * 4 halfs). */
oxpt_status oxpt_read_scene(oxpt_ctx* ctx, uint32_t* geom, float* attrs, uint16_t* atlas);
/*
 * Borrow another context's device scene (geometry, attributes, atlas,
 * four-wide tree) or tables instead of uploading copies: contexts that
 * render the same scene from different cameras, resolutions or sample
 * counts (serving sessions) keep one resident copy. The lending context
 * must outlive the borrower; a later upload / set_tables on the borrower
 * replaces the borrowed buffers with its own. No reference counterpart.
 */
oxpt_status oxpt_share_scene(oxpt_ctx* ctx, const oxpt_ctx* owner);
oxpt_status oxpt_share_tables(oxpt_ctx* ctx, const oxpt_ctx* owner);
oxpt_status oxpt_set_params(oxpt_ctx* ctx, const oxpt_params* params);

/* ---- accumulation (sync's accumulator, :551-564; reset, :495-502) */
oxpt_status oxpt_resize(oxpt_ctx* ctx, uint32_t width, uint32_t height);
oxpt_status oxpt_reset(oxpt_ctx* ctx);

/* ---- tracing (refine, :584-671; trace_main, pathtrace.wgsl:2047-2073).
 * oxpt_dispatch runs one frame exactly. oxpt_refine takes samples
 * [first, first + count) of every row, scheduling launches itself.
 * Both are asynchronous. */
oxpt_status oxpt_dispatch(oxpt_ctx* ctx, const oxpt_frame* frame);
oxpt_status oxpt_refine(oxpt_ctx* ctx, uint32_t first_sample, uint32_t count);
/* Block until all queued work finished (finish, :674-679). */
oxpt_status oxpt_finish(oxpt_ctx* ctx);

/* ---- resolve (encode_resolve + image/hdr/draw_texture, :687-844;
 * fs_resolve_pt, resolve.wgsl:151-188). Writes the device image; when
 * `host_out` is non-null also copies it there (w*h*4 bytes for RGBA8,
 * w*h*16 for RGBA32F) and blocks. `dev_out` (optional) receives the device
 * image handle. */
oxpt_status oxpt_resolve(oxpt_ctx* ctx, const oxpt_resolve_params* params, int hdr,
                         void* host_out, oxpt_devimage* dev_out);

/* Raw accumulator (w*h*4 floats: sum rgb over covered samples, covered
 * count). Blocking. */
/*
 * Present path (§ image() / draw_texture(), src/pathtrace.rs:687-725, as an
 * asynchronous readback): resolves on the context's stream into a device
 * image, then copies it to `host_out` on a separate copy stream, so the
 * copy overlaps whatever is enqueued next on the context (the next refine
 * does not wait for it). `host_out` must stay valid until
 * oxpt_resolve_wait returns; pinned memory (oxpt_host_alloc) makes the copy
 * truly asynchronous. A later oxpt_resolve_async waits on the device for
 * the previous copy before reusing the image.
 */
oxpt_status oxpt_resolve_async(oxpt_ctx* ctx, const oxpt_resolve_params* params, int hdr, void* host_out);
oxpt_status oxpt_resolve_wait(oxpt_ctx* ctx);
/* Page-locked host memory for present buffers (NULL on failure). */
void* oxpt_host_alloc(size_t bytes);
void oxpt_host_free(void* p);
oxpt_status oxpt_read_accum(oxpt_ctx* ctx, float* host_out);

/* The accumulator itself as a device image (RGBA32F, read-write), for
 * gathering the row tiles of a frame split across GPUs with a collective
 * that writes into it. No counterpart in the reference (single device). */
oxpt_status oxpt_accum_view(oxpt_ctx* ctx, oxpt_devimage* out);

/*
 * Allocation-free dispatch. This entry point has no counterpart in the
 * reference.
 *
 * For callers that may not let a library allocate or free device memory:
 * an application that owns all device memory through its own allocator and
 * hands each component the buffers it may use, or one that cannot afford
 * the device synchronisation that cudaMalloc / cudaFree can cause in the
 * middle of a frame. Everything here is the caller's: the scene buffers
 * (device pointers, in the layouts of oxpt_scene_desc / oxpt_set_tables),
 * the Params, and the accumulator (device pointer, w*h*4 floats, updated in
 * place exactly as oxpt_dispatch updates the context's accumulator, so the
 * results are bit-identical). No context is needed and nothing is
 * allocated: the per-path scratch of the dispatch lives in a fixed array
 * of OXPT_NOALLOC_MAX_PATHS x 16 bytes (4 MiB) that every GPU loading the
 * library holds until the process exits; larger frames run as several
 * launches over it. An image row wider than OXPT_NOALLOC_MAX_PATHS pixels
 * is rejected with OXPT_E_LIMIT.
 *
 * The first call on a device looks up the array's device address with
 * that device current (so make that first call before any stream capture).
 * Launches go to `stream` (a cudaStream_t; NULL = the legacy default
 * stream) and the call returns without waiting. All calls share the one
 * array, which keeps the previous call's contents: calls whose work
 * overlaps on the GPU (different streams, or different host threads on the
 * same device) race on it and must be ordered by the caller. A malformed
 * BVH is cut short on the device and not reported (the call has no place to
 * return the device's error word without a readback): pass scenes that this
 * library prepared (oxpt_build_scene, the host preparation) or that the
 * caller has checked. After a device reset (cudaDeviceReset, or a reset of
 * the primary context) the next call looks the array's address up again.
 */
#define OXPT_NOALLOC_MAX_PATHS (1u << 18)
typedef struct oxpt_device_scene {
    const void* geom;    /* device: node + triangle words */
    size_t geom_words;
    const void* attrs;   /* device: 48 floats per slot */
    size_t attr_floats;
    const void* tables;  /* device: scene tables + environment words */
    size_t table_words;
    const void* atlas;   /* device: RGBA16F layers */
    uint32_t atlas_side;
    uint32_t atlas_layers;
} oxpt_device_scene;
oxpt_status oxpt_dispatch_noalloc(const oxpt_device_scene* scene, const oxpt_params* params,
                                  const oxpt_frame* frame, float* accum, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* OXPT_H */
