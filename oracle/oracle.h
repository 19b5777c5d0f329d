/*
 * CPU oracle for the B200 path tracer — TEST INFRASTRUCTURE ONLY.
 *
 * A scalar C++ restatement of the reference's GPU estimator
 * (src/shaders/pathtrace.wgsl:1-2073) and its resolve
 * (src/shaders/resolve.wgsl:38-75, 138-188), reading the same flat
 * buffers (geom, attrs, tables, atlas, Params, FrameParams) the reference
 * kernel binds. It is the checker the parity tests, smoke() and the
 * bench's CPU-baseline leg compare against; the product never calls it.
 *
 * Parity pinning: the reference's own CPU tracer (oxideav_render::
 * PathTracer) lives in an external crate that is not in the reference tree
 * and there is no Rust toolchain, so this oracle is pinned only by the
 * reference's known-answer tests that do not need that crate: the f16
 * conversion vectors (src/scene.rs:496-510), the white-furnace analytic
 * value (tests/pathtrace.rs:295-317) and the bit-exact behavioural
 * invariants (tests/pathtrace.rs:420-565). Everything the external crate
 * would supply (Sobol' matrices, sheen LUT, BVH, CDFs) is this project's
 * own; beyond those tests parity is unpinned.
 *
 * Transcendentals: `libm` = 0 evaluates sin/cos/acos/atan2/exp/log/log2/
 * pow with the project's portable float routines (the ones the CUDA
 * kernel uses), so results are comparable bit for bit; `libm` = 1 uses the
 * C library's float functions, as a Rust CPU tracer would.
 */
#ifndef OXO_ORACLE_H
#define OXO_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oxo_scene {
    const uint32_t* geom;
    size_t geom_words;
    const float* attrs;
    size_t attr_floats;
    const uint32_t* tables;
    size_t table_words;
    const uint16_t* atlas;
    uint32_t atlas_side;
    uint32_t atlas_layers;
} oxo_scene;

/* One trace_main dispatch over frame {first, count, y0, rows}; `params`
 * is the 176-byte Params block. accum: w*h*4 floats, updated in place.
 * counters (optional, 8 x u64): paths, path rays, shadow rays, AABBs
 * slab-tested, leaves visited, triangle tests, shaded hits, stack pops. */
int oxo_dispatch(const oxo_scene* scene, const void* params, const uint32_t frame[4],
                 float* accum, int threads, int libm, uint64_t* counters);

/* fs_resolve_pt over the whole accumulator; `rparams` = 48-byte
 * ResolveParams. out: w*h*4 bytes (hdr = 0) or w*h*4 floats (hdr = 1). */
void oxo_resolve(const float* accum, uint32_t w, uint32_t h, const void* rparams, int hdr,
                 int libm, void* out);

/* pattern(make_sampler(seed, x, y, index), pattern_id) before to_unit. */
void oxo_sobol(const uint32_t* dirs, uint32_t seed, size_t n, const uint32_t* x,
               const uint32_t* y, const uint32_t* index, const uint32_t* pattern_id,
               uint32_t* out);

/* traverse() for n rays (o.xyz, t_max, d.xyz, skip bits); flags bit 0
 * any-hit, bit 1 primary. Outputs may be NULL. */
void oxo_trace_rays(const oxo_scene* scene, const void* params, size_t n, const float* rays,
                    uint32_t flags, uint32_t* slot, uint32_t* global_id, float* t, float* bary,
                    int threads, uint64_t* counters);

uint16_t oxo_f32_to_f16(float v);
void oxo_math(int op, size_t n, const float* a, const float* b, float* out, int libm);

#ifdef __cplusplus
}
#endif
#endif
