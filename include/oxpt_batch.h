/*
 * oxpt_batch.h — batched refinement: the frames of several scenes traced
 * as one wavefront.
 *
 * The reference renders one scene per GpuPathTracer and one dispatch per
 * row tile (src/pathtrace.rs:584-671); a server holding many scenes would
 * run them one after another, and each frame's wavefront ends with a tail
 * in which few paths are left. Here one executor context traces the frames
 * of any number of contexts (each with its own scene, tables, params and
 * accumulator) as a single wavefront: its slots take paths from every
 * frame, so the tail of one frame overlaps the others, and every launch of
 * the wavefront serves all of them. This has no counterpart in the
 * reference.
 *
 * Results: every path keeps its scene, pixel and sample index, and each
 * pixel's samples are added in sample order, so every context's
 * accumulator ends bit-identical to what oxpt_refine / oxpt_dispatch on
 * that context alone gives.
 */
#ifndef OXPT_BATCH_H
#define OXPT_BATCH_H

#include "oxpt.h"

#ifdef __cplusplus
extern "C" {
#endif

/* One frame of a batch: samples [first, first + count) over rows
 * [y0, y0 + rows) of `ctx`'s image. */
typedef struct oxpt_batch_frame {
    oxpt_ctx* ctx;
    uint32_t first, count, y0, rows;
} oxpt_batch_frame;

/*
 * Traces the frames on `exec`'s stream with `exec`'s execution plan
 * (oxpt_set_tuning; a megakernel plan runs as the split wavefront) and its
 * path-state buffers; `exec` may be one of the frames' contexts. Every
 * context must be ready (scene, tables, params, accumulator) and on
 * `exec`'s device, and every scene's Sobol' and sheen tables must hold the
 * same words (they are fixed tables). Each frame context's stream is
 * synchronised before the batch starts and made to wait for its end, so
 * later calls on those contexts see the results. Frames wider than the
 * plan's items per launch are cut into row bands and rounds.
 * OXPT_E_INVALID names the offending frame.
 */
oxpt_status oxpt_refine_batch(oxpt_ctx* exec, const oxpt_batch_frame* frames, uint32_t count);

/*
 * The round plan of a batch, without a GPU (for tests): frames[5k..5k+4] =
 * width, first, count, y0, rows; cap = items per round. Writes up to
 * `capacity` pieces as out[7p..7p+6] = round, frame, first, count, y0,
 * rows, base; *pieces = the number of pieces of the plan.
 */
oxpt_status oxpt_diag_batch_plan(const uint32_t* frames, uint32_t count, uint64_t cap, uint64_t* out,
                                 size_t capacity, size_t* pieces);

#ifdef __cplusplus
}
#endif
#endif /* OXPT_BATCH_H */
