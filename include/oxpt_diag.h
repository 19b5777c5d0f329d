/*
 * oxpt_diag.h — diagnostic entry points of the B200 path tracer.
 *
 * These have no counterpart in the reference's FFI. They expose single
 * stages of the device path (Sobol' generation, BVH ray queries, the
 * portable transcendentals, traversal counters) so that the parity tests
 * can compare each stage with the CPU oracle on its own. They run on the
 * context's stream and block until their results are on the host.
 */
#ifndef OXPT_DIAG_H
#define OXPT_DIAG_H

#include "oxpt.h"

#ifdef __cplusplus
extern "C" {
#endif

/*
 * Owen-scrambled Sobol' points, pathtrace.wgsl:158-228 (make_sampler +
 * pattern). For each i: sampler = make_sampler(seed, x[i], y[i], index[i]);
 * out[4i..4i+3] = the four 32-bit scrambled values of pattern(sampler,
 * pattern_id[i]) before `to_unit` (so both the integers and the floats
 * `(v >> 8) * 2^-24` can be compared). `sobol_dirs` = 128 direction words.
 */
oxpt_status oxpt_diag_sobol(oxpt_ctx* ctx, const uint32_t* sobol_dirs, uint32_t seed, size_t n,
                            const uint32_t* x, const uint32_t* y, const uint32_t* index,
                            const uint32_t* pattern_id, uint32_t* out);

/*
 * BVH ray queries on the uploaded scene and tables (traverse,
 * pathtrace.wgsl:646-735). rays[8i..8i+7] = o.xyz, t_max, d.xyz, skip
 * (global triangle id bits, 0xffffffff = none). flags bit 0 = any-hit,
 * bit 1 = primary (back-face culling of single-sided materials), bit 2 =
 * any-hit rays walk the four-wide tree (OXPT_E_INVALID when none was
 * built; which occluder is reported may differ, occlusion may not), bit 3
 * = closest-hit rays walk the four-wide tree (the tolerance plan's walk:
 * the hit may differ only between candidates at nearly equal distance).
 * Outputs per ray: slot (0xffffffff = miss), global id, t, barycentrics
 * (3 floats). Any output pointer may be NULL.
 */
oxpt_status oxpt_diag_trace_rays(oxpt_ctx* ctx, size_t n, const float* rays, uint32_t flags,
                                 uint32_t* slot, uint32_t* global_id, float* t, float* bary);

/* Portable transcendental `op` (0 sin, 1 cos, 2 acos, 3 atan2(a, b),
 * 4 exp, 5 log, 6 log2, 7 pow(a, b)) evaluated on the device. */
oxpt_status oxpt_diag_math(oxpt_ctx* ctx, int op, size_t n, const float* a, const float* b,
                           float* out);

/*
 * Run samples [first, first + count) of every row with the counting build
 * of the trace kernel and return its totals: out[0] paths, out[1] path
 * rays, out[2] shadow rays, out[3] AABBs slab-tested (the root, then two
 * per inner node visited), out[4] leaves visited, out[5] triangle tests,
 * out[6] shaded hits, out[7] stack pops. The accumulator is updated
 * exactly as by oxpt_refine.
 */
oxpt_status oxpt_diag_refine_counted(oxpt_ctx* ctx, uint32_t first_sample, uint32_t count,
                                     uint64_t out[8]);

/*
 * Kernel timing. While enabled, every trace and reduce launch is bracketed
 * by CUDA events on the context's stream. oxpt_diag_timing synchronises the
 * stream and returns (then clears) the summed device milliseconds and the
 * number of launches of each kind since the last call.
 */
oxpt_status oxpt_diag_set_timing(oxpt_ctx* ctx, int enabled);
oxpt_status oxpt_diag_timing(oxpt_ctx* ctx, double* trace_ms, uint64_t* trace_launches,
                             double* reduce_ms, uint64_t* reduce_launches);
/* The per-kind figures of the last oxpt_diag_timing call: kind 0 the trace
 * phase of each launch (the megakernel, or a whole wavefront run), 1 the
 * ordered reduce, 2 wavefront logic, 3 wavefront extension traversal, 4
 * wavefront shadow traversal, 5 split-wavefront shading, 6 split-wavefront
 * NEE, 7 radiance-cache inference, 8 cache training forward, 9 cache
 * backward, 10 continuation-ray reordering; 11 unused. */
oxpt_status oxpt_diag_timing_kinds(const oxpt_ctx* ctx, double ms[12], uint64_t n[12]);
/* The last oxpt_diag_refine_counted totals split by ray kind: out[0..7] for
 * continuation rays and shading (wavefront logic + extension), out[8..15]
 * for shadow rays (wavefront shadow kernel); the megakernel reports all in
 * the first half. */
oxpt_status oxpt_diag_counters_split(const oxpt_ctx* ctx, uint64_t out[16]);

/* Launch-shape override for tuning: threads per block and resident blocks
 * per SM of the megakernel (0 = library default), and the largest number
 * of paths one launch may take (both execution modes). */
oxpt_status oxpt_diag_set_launch(oxpt_ctx* ctx, uint32_t threads, uint32_t blocks_per_sm,
                                 uint64_t max_paths_per_launch);

/* Traversal kernels of trace_variant 3-5: walk-stack entries per lane kept
 * in shared memory (at most 16; deeper entries live in local memory) and
 * the number of top nodes of the binary tree each CTA stages in shared
 * memory (within what the variant's occupancy leaves a block). Both only
 * move data between memories (results are unchanged); shared memory is
 * taken from L1, so the defaults are measured choices. 0 entries puts the
 * whole stack in local memory, which lets tests exercise that path. */
oxpt_status oxpt_diag_set_walk(oxpt_ctx* ctx, uint32_t stack_entries, uint32_t staged_nodes);
oxpt_status oxpt_diag_get_walk(const oxpt_ctx* ctx, uint32_t out[2]);
/* Split plan with at most 32 NEE jobs per vertex: 1 (default) = the shadow
 * kernels set a per-slot visibility bit and only queued jobs' contributions
 * are stored, 0 = a pending record per job with a visibility word. The
 * logic kernel adds the same contributions in the same order either way. */
oxpt_status oxpt_diag_set_nee_mask(oxpt_ctx* ctx, int on);
/* Four-wide shadow walks of trace_variant 3-5: 1 = lanes park the leaves
 * they reach and keep walking inner nodes, and the warp tests parked
 * leaves together once no lane has node work left (speculative traversal);
 * 0 (default) = each lane tests a leaf when it reaches it. Occlusion does
 * not depend on the order, so results are the same. */
oxpt_status oxpt_diag_set_shadow_postpone(oxpt_ctx* ctx, int on);
/* Wavefront plans, bit 0: before the closest-hit walk the continuation
 * rays are reordered (counting sort on direction octant and a 16^3 Morton
 * cell of the origin in the scene's root box) so that a warp walks similar
 * rays; bit 1 (trace_variant 3-5): the shadow rays are walked in the order
 * of their light and origin cell; 0 (default) = queue order. Each ray is
 * walked alone by one lane, so results are the same either way. The
 * reordering launches time as kind 10. */
oxpt_status oxpt_diag_set_ray_order(oxpt_ctx* ctx, int mode);
/* on = 1: the short-stack traversal kernels (trace_variant 3-5) of launches
 * over one scene mark the tree nodes they read (the binary nodes for
 * closest hits, the four-wide tree for shadow rays) as persisting L2 lines
 * through an access-policy window, half of the L2 set-aside each; the
 * process's persisting set-aside is raised to the device maximum, a limit
 * of this process's CUDA context. *granted (optional) = the set-aside in
 * bytes. A performance hint only: results are the same bits. 0 = off. */
oxpt_status oxpt_diag_set_l2_window(oxpt_ctx* ctx, int on, uint64_t* granted);

/*
 * Execution plan of a context, chosen by the autotuner (tuner.py) or left
 * at the defaults. Every plan produces bit-identical accumulators; only
 * speed differs.
 *   mode           OXPT_MODE_MEGAKERNEL: one persistent kernel runs whole
 *                  paths; OXPT_MODE_WAVEFRONT: path state in HBM, one
 *                  shading launch and two traversal launches per bounce.
 *   threads, blocks_per_sm, max_paths   megakernel launch shape.
 *   wave_slots     paths in flight (wavefront); wave_items its paths per
 *                  launch round (0 = 2^27: a 1080p frame of 64 spp in one
 *                  round; the result buffer holds 16 bytes per path of a
 *                  round); check_every its bounces between completion
 *                  checks.
 *   shade_variant  wavefront logic kernel compiled for 2 / 3 / 4 resident
 *                  blocks per SM (0 / 1 / 2): registers against occupancy.
 *   trace_variant  wavefront traversal kernels: 0-2 with local-memory walk
 *                  stacks for 6 / 8 / 10 blocks per SM; 3-5 with short
 *                  stacks in shared memory, alpha tests out of line and
 *                  optional staged top nodes (oxpt_diag_set_walk), for
 *                  6 / 8 / 10 blocks. Default 4.
 *   nee_variant    split wavefront NEE kernel: job-major (0, 1, 2) or
 *                  vertex-major (3, 4, 5) for 4 / 5 / 6 blocks.
 *   OXPT_MODE_WAVEFRONT_SPLIT: the wavefront with the shading of a bounce
 *                  in three kernels (path logic, surface shading, one thread
 *                  per NEE job); shade_variant then applies to the shading
 *                  kernel.
 *   stack          traversal stack entries: 32 or 64; 0 = 32 when the BVH
 *                  is at most 32 levels deep, else 64 (exact either way).
 *   shadow_walk    wavefront shadow rays: 0 = the four-wide tree built on
 *                  upload when the scene allows it (same occlusion), 1 =
 *                  the binary ordered walk.
 *   graphs         batched refinement (oxpt_batch.h) as one CUDA graph per
 *                  refine step: each round's wavefront loop is a device-side
 *                  while node (no host round trips), reused while the step's
 *                  shape is unchanged; 0 = host-driven loop.
 *   refill         wavefront traversal: a warp gives its idle lanes new rays
 *                  once this many of its 32 lanes are idle (1 = as soon as
 *                  one is; 32 = when all are); 0 = library default (8).
 *   closest_walk   0 = continuation rays take the reference's ordered
 *                  binary walk (every plan above is then bit-identical);
 *                  1 = the four-wide tree, nearest child first with entry
 *                  distances on the stack (trace_variant 3-5 only; scenes
 *                  without an exact four-wide tree keep the binary walk).
 *                  The tolerance plan: a closest hit can differ from the
 *                  binary walk's only between candidates within rounding of
 *                  the same distance, so accumulators match the oracle to
 *                  image tolerance (>= 60 dB PSNR), not bit for bit.
 *   fast_shading   0 = the split wavefront's shading kernels as built for
 *                  bit equality; 1 = their second build with FMA
 *                  contraction, approximate division and square root and
 *                  the CUDA library's transcendentals (mode 2 only). With
 *                  closest_walk 1 this is the tolerance plan: images within
 *                  >= 60 dB PSNR of the oracle, traversal unchanged.
 */
enum { OXPT_MODE_MEGAKERNEL = 0, OXPT_MODE_WAVEFRONT = 1, OXPT_MODE_WAVEFRONT_SPLIT = 2 };
typedef struct oxpt_tuning {
    uint32_t mode;
    uint32_t threads;
    uint32_t blocks_per_sm;
    uint32_t wave_slots;
    uint64_t max_paths;
    uint64_t wave_items;
    uint32_t check_every;
    uint32_t shade_variant;
    uint32_t trace_variant;
    uint32_t stack;
    uint32_t nee_variant;
    uint32_t shadow_walk;
    uint32_t graphs;
    uint32_t refill;
    uint32_t closest_walk;
    uint32_t fast_shading;
} oxpt_tuning;
oxpt_status oxpt_set_tuning(oxpt_ctx* ctx, const oxpt_tuning* t);
oxpt_status oxpt_get_tuning(const oxpt_ctx* ctx, oxpt_tuning* t);
/* The four-wide any-hit tree of the uploaded scene: out[0] 1 when built
 * (0: the scene keeps the binary walk for every ray), out[1] its nodes,
 * out[2] its root reference, out[3] the stack entries its walk needs. */
oxpt_status oxpt_diag_bvh4(const oxpt_ctx* ctx, uint32_t out[4]);
/* Timing of the context's last oxpt_build_scene, in milliseconds: device
 * time (CUDA events) of [0] the source upload, [1] the BVH build, [2] the
 * slot flattening, [3] the atlas (texel upload and mip chains, on a stream
 * of its own that overlaps [0]-[2]); host wall time of [4] the whole call
 * and [5] the upload of its four-wide tree (collapsed on the host while the
 * atlas builds); [6] the number of
 * kernels it launched; [7] unused (0). */
oxpt_status oxpt_diag_scene_build(const oxpt_ctx* ctx, float ms[8]);
/* Host-side collapse of binary node words (node i at words 8i..8i+7) into
 * the four-wide layout: 32 words per node, written to `out` when it has
 * room for them (`cap` words); *words = the words needed, *root = the root
 * reference, *stack_need as above. OXPT_E_INVALID when the tree cannot be
 * collapsed exactly (malformed, a child box outside its parent's, a leaf of
 * more than 16 triangles). Needs no GPU. */
oxpt_status oxpt_diag_bvh4_build(const uint32_t* geom, uint32_t node_count, uint32_t* out, size_t cap,
                                 size_t* words, uint32_t* root, uint32_t* stack_need);
/* The same collapse on `device` (the path scene uploads take), plus the
 * binary tree's depth counted on the device (*depth) and by the host walk
 * (*host_depth; both 65 when deeper than 64 levels or malformed). Equal
 * outputs to oxpt_diag_bvh4_build; OXPT_E_INVALID when it refuses the
 * tree, OXPT_E_LIMIT when the device pass leaves it to the host. */
oxpt_status oxpt_diag_bvh4_build_device(int device, const uint32_t* geom, uint32_t node_count, uint32_t* out,
                                        size_t cap, size_t* words, uint32_t* root, uint32_t* stack_need,
                                        uint32_t* depth, uint32_t* host_depth);
/* BVH of n triangles (tri_pos: 9 floats each) by the host builder
 * (on_gpu = 0) or the GPU builder on `device` (on_gpu = 1): node words
 * (8 per node, at most 2n nodes), leaf slot -> triangle, node count and
 * depth. Both give the same words. */
oxpt_status oxpt_diag_bvh_build(int device, const float* tri_pos, uint32_t n, int on_gpu, uint32_t* words,
                                uint32_t* slots, uint32_t* node_count, uint32_t* depth);
/* Wavefront bounces (logic + extend + shadow launches) run so far (waits
 * for the context's stream when graph-resident loops have run). */
oxpt_status oxpt_diag_wave_iterations(const oxpt_ctx* ctx, uint64_t* out);
/* CUDA graphs instantiated for batched refinement so far. */
oxpt_status oxpt_diag_graph_builds(const oxpt_ctx* ctx, uint64_t* out);

/* Number of kernels launched by this context (waits for the context's
 * stream when graph-resident loops have run, whose launches the device
 * counts). */
oxpt_status oxpt_diag_launch_count(const oxpt_ctx* ctx, uint64_t* out);

#ifdef __cplusplus
}
#endif
#endif /* OXPT_DIAG_H */
