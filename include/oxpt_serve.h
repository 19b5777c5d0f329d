/*
 * oxpt_serve.h — what a serving loop needs beyond a single tracer: views
 * (sessions) that share one resident prepared scene, camera moves, and
 * device-memory accounting for admission. No reference counterpart: the
 * reference renders one scene per GpuPathTracer.
 */
#ifndef OXPT_SERVE_H
#define OXPT_SERVE_H

#include "oxpt_host.h"

#ifdef __cplusplus
extern "C" {
#endif

/* CUDA device of a context. */
int oxpt_ctx_device(const oxpt_ctx* ctx);

/* Stream marks: oxpt_mark records the current position of the context's
 * stream; oxpt_wait_mark blocks until the stream has passed it (the last
 * 64 marks are kept; an older one waits for the newest). A scheduler that
 * queues the next batch before the previous one is done uses them to learn
 * when each finished. */
oxpt_status oxpt_mark(oxpt_ctx* ctx, uint64_t* mark);
oxpt_status oxpt_wait_mark(oxpt_ctx* ctx, uint64_t mark);

/* Device bytes a context holds: out[0] its own scene buffers (geometry,
 * attributes, atlas, four-wide tree; 0 when borrowed), out[1] its own
 * tables, out[2] accumulator and output images, out[3] working buffers
 * (per-path results, wavefront state, batch records). */
oxpt_status oxpt_ctx_memory(const oxpt_ctx* ctx, uint64_t out[4]);

/*
 * A view of `owner` (a tracer synced to a scene): a tracer with its own
 * context, camera, resolution, options and accumulator that borrows the
 * owner's prepared scene and its device buffers (and its device tables
 * when they are the same words). The owner must outlive the view.
 */
oxpt_status oxpt_tracer_new_view(const oxpt_tracer* owner, oxpt_tracer** out);
/* sync() of a view: options only (its scene is the owner's; the light
 * intensity, a preparation input, must be the owner's). Same reset rules. */
oxpt_status oxpt_tracer_view_sync(oxpt_tracer* view, const oxpt_render_options* opts, int* did_reset);
/* Camera override of a tracer or view (NULL: back to the options' camera).
 * Like a camera change seen by sync, it resets the accumulation. */
oxpt_status oxpt_tracer_set_camera(oxpt_tracer* t, const oxpt_camera* camera);

#ifdef __cplusplus
}
#endif
#endif /* OXPT_SERVE_H */
