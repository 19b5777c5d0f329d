/*
 * oxpt_nrc.h — neural radiance cache: a small MLP trained online on the
 * tracer's own path samples, which ends paths after a few bounces with its
 * prediction of the radiance still to come. No counterpart in the
 * reference (its tracer is the unbiased plain form, which stays the
 * fallback here and the image the cache's error is measured against).
 *
 * Network: inputs = position (normalised to the scene bounds), outgoing
 * direction, shading normal (each component mapped to [0, 1]) and
 * roughness, 12 sine / cosine frequencies each (plus the raw values and a
 * constant), 5 layers 256 -> 64 -> 64 -> 64 -> 64 -> 3 with ReLU, BF16
 * weights and activations, FP32 accumulation on the tensor cores; loss =
 * relative L2; Adam (lr 1e-2 by default).
 */
#ifndef OXPT_NRC_H
#define OXPT_NRC_H

#include "oxpt.h"
#include "oxpt_host.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oxpt_nrc oxpt_nrc;

#define OXPT_NRC_PARAMS 29696u /* FP32 weights: 64x256, 3 x 64x64, 16x64 (rows 3..15 unused), row-major */
#define OXPT_NRC_INPUTS 12u    /* floats per sample: pos.xyz, roughness, dir.xyz, 0, normal.xyz, 0 */

/* A cache on `ctx`'s device, weights initialised from `seed` (uniform He
 * initialisation), Adam state zero. It has its own stream for the calls
 * below that take host buffers; cache frames (oxpt_nrc_refine) run on the
 * rendering context's stream. It may outlive `ctx`. */
oxpt_status oxpt_nrc_create(oxpt_ctx* ctx, uint64_t seed, oxpt_nrc** out);
void oxpt_nrc_destroy(oxpt_nrc* nrc);
const char* oxpt_nrc_last_error(const oxpt_nrc* nrc);

oxpt_status oxpt_nrc_get_weights(oxpt_nrc* nrc, float* out);
/* Replaces the weights and clears the Adam moments and step count. */
oxpt_status oxpt_nrc_set_weights(oxpt_nrc* nrc, const float* weights);
oxpt_status oxpt_nrc_set_adam(oxpt_nrc* nrc, float lr, float beta1, float beta2, float eps);

/* Predictions for n samples (inputs n x 12 floats, out n x 4: rgb, 0),
 * host buffers. */
oxpt_status oxpt_nrc_infer(oxpt_nrc* nrc, const float* inputs, uint32_t n, float* out);
/* One training step on n samples (targets n x 4: rgb, unused): forward,
 * backward, and an Adam update when `apply` is non-zero. *loss = the mean
 * relative L2 loss before the update; `grad` (optional) receives the
 * gradient of that loss (OXPT_NRC_PARAMS floats). Host buffers. */
oxpt_status oxpt_nrc_train(oxpt_nrc* nrc, const float* inputs, const float* targets, uint32_t n, int apply,
                           float* loss, float* grad);

/*
 * Rendering with the cache: each frame traces one sample per pixel of
 * `ctx`'s image with the split wavefront. A path that is not a training
 * path stops at the vertex hit by ray `query_bounce` (2: after two bounces;
 * it keeps that vertex's emission) and the cache's prediction times its
 * throughput there is added instead of the rest of the path. One path in
 * `train_one_in` (by its path seed) is traced to the end as the plain
 * tracer would and becomes a training sample: the vertex's inputs and the
 * radiance it gathered from there on per unit throughput. After a frame's
 * results are reduced into the accumulator, the cache takes one Adam step
 * on that frame's samples (at most `max_train`) when `train` is set.
 * With `train_suffix` > 0 a training path ends into the cache that many
 * bounces after the query vertex and its target adds the cache's
 * prediction there (self-training, which keeps every path short). All of
 * a frame's paths are in flight at once (one wavefront slot per pixel);
 * with `frames_per_wave` > 1 consecutive frames share one wavefront, and
 * the training step follows each wave rather than each frame.
 * `enabled` = 0 renders plain frames (the ablation). The frame must fit
 * one launch of the context's plan (width x height <= its items per
 * launch).
 */
typedef struct oxpt_nrc_config {
    uint32_t enabled;
    uint32_t query_bounce;
    uint32_t train_one_in;  /* a power of two */
    uint32_t max_train;
    uint32_t train;
    uint32_t train_suffix;  /* training paths end into the cache this many bounces after the
                               query vertex (self-training); 0 = they run to the end */
    float spread;           /* path-spread heuristic (Mueller et al. 2021): a path ends into the
                               cache at the first vertex at or after query_bounce where
                               (sum over its bounces of sqrt(t^2 / (pdf |cos|)))^2 exceeds
                               spread x the primary vertex's t^2 / (4 pi |cos|); 0 = exactly
                               at query_bounce */
    uint32_t frames_per_wave; /* frames traced as one wavefront (0 or 1: one), at most 64: the
                               next frame's paths take the slots the previous frame's paths free,
                               so frame tails overlap; the wave's queries are answered and one
                               training step (on at most max_train samples) is taken after it */
} oxpt_nrc_config;
void oxpt_nrc_config_default(oxpt_nrc_config* cfg); /* 1, 2, 16, 65536, 1, 4, 0.01, 1 */

/* `count` cache frames with sample indices first_sample.. on `ctx`'s
 * accumulator; *loss (optional, waits for the GPU) = the last training
 * step's mean loss before its update. */
oxpt_status oxpt_nrc_refine(oxpt_nrc* nrc, oxpt_ctx* ctx, uint32_t first_sample, uint32_t count,
                            const oxpt_nrc_config* cfg, float* loss);
/* refine() of a tracer with cache frames: `frames` samples per pixel, one
 * per frame, on the tracer's bound scene and options; its sample count
 * advances as with oxpt_tracer_refine. */
oxpt_status oxpt_tracer_refine_nrc(oxpt_tracer* t, oxpt_nrc* nrc, uint32_t frames, const oxpt_nrc_config* cfg,
                                   float* loss);
/* Training samples and cache queries of the last frame (waits). */
oxpt_status oxpt_nrc_frame_counts(oxpt_nrc* nrc, uint32_t* queries, uint32_t* samples);

#ifdef __cplusplus
}
#endif
#endif /* OXPT_NRC_H */
