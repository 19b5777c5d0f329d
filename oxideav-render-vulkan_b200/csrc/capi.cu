// C ABI of the path tracer (include/oxpt.h, include/oxpt_diag.h).
//
// One oxpt_ctx owns a CUDA stream and the device buffers that the
// reference's GpuPathTracer owns through wgpu (src/pathtrace.rs:145-237):
// geometry, attributes, tables, the texture atlas, the accumulator and the
// output images. The launch schedule of oxpt_refine replaces the
// reference's row tiles / sample runs of at most 2^20 paths
// (src/pathtrace.rs:584-671): a B200 has no display watchdog, so a launch
// takes up to `max_paths` paths, sized so that its per-path result buffer
// stays L2-resident, and the persistent grid fills every SM.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/oxpt.h"
#include "../../include/oxpt_batch.h"
#include "../../include/oxpt_diag.h"
#include "../../include/oxpt_serve.h"
#include "kernels.cuh"
#include "wavefront.cuh"
#include "../../include/oxpt_nrc.h"
#include "nrc.cuh"
#include "nrc_state.hpp"
#include "../host/batch.hpp"
#include "../host/bvh4.hpp"
#include "scene_prep.cuh"

// A scene's device buffers and what the context knows of them. The
// context traces its current set (the oxpt_ctx fields of the same names);
// oxpt_stage_scene fills a second set while queued work still traces the
// current one, and the next trace call swaps them.
struct SceneSet {
    float4* geom = nullptr;
    size_t geom_vec4 = 0, geom_cap = 0;
    float4* attrs = nullptr;
    size_t slot_count = 0, attrs_cap = 0;
    uint2* atlas = nullptr;
    uint32_t side = 1, layers = 1;
    size_t atlas_cap = 0;
    uint32_t node_count = 0, bvh_depth = 0;
    float4* bvh4 = nullptr;
    size_t bvh4_cap = 0;
    bool bvh4_built = false;
    uint32_t bvh4_nodes = 0, bvh4_root = 0xffffffffu, bvh4_need = 0;
    uint32_t* tables = nullptr;
    size_t table_words = 0, tables_cap = 0;
    std::vector<uint32_t> table_head;
};

struct oxpt_ctx {
    int device = 0;
    cudaStream_t own = nullptr;
    cudaStream_t stream = nullptr;
    std::string err;
    int sms = 0;
    // scene
    float4* geom = nullptr;
    size_t geom_vec4 = 0;
    float4* attrs = nullptr;
    size_t slot_count = 0;
    uint2* atlas = nullptr;
    uint32_t side = 1, layers = 1;
    uint32_t node_count = 0;
    uint32_t* tables = nullptr;
    size_t table_words = 0;
    // scene buffers / tables borrowed from another context (oxpt_share_*)
    bool borrowed_scene = false, borrowed_tables = false;
    std::vector<uint32_t> table_head;  // host copy of the first table words (fixed tables)
    // present path (oxpt_resolve_async): image buffer, copy stream, events
    void* present = nullptr;
    size_t present_bytes = 0;
    cudaStream_t copy = nullptr;
    cudaEvent_t resolved = nullptr, copied = nullptr;
    cudaEvent_t ready = nullptr;       // this context's stream position, for batches
    // stream marks (oxpt_mark): a ring of events
    std::vector<cudaEvent_t> marks;
    uint64_t next_mark = 0;
    oxpt_params params{};
    bool has_scene = false, has_tables = false, has_params = false;
    // accumulation + outputs
    float4* accum = nullptr;
    uint32_t w = 0, h = 0;
    void* img8 = nullptr;
    void* img32 = nullptr;
    // per-launch path results
    float4* out = nullptr;
    uint64_t out_cap = 0;
    // device words: error flags, counters
    uint32_t* dev_err = nullptr;
    unsigned long long* dev_counters = nullptr;
    // launch shape
    uint32_t threads = oxd::TRACE_THREADS;
    uint32_t blocks_per_sm = 0;
    uint64_t max_paths = 1ull << 22;
    uint64_t launches = 0;
    // optional per-launch event timing: {start, end, kind (0 trace, 1 reduce)}
    bool timing = false;
    struct Timed {
        cudaEvent_t a, b;
        int kind;
    };
    std::vector<Timed> timed;
    double kind_ms[12] = {0}, last_ms[12] = {0};
    uint64_t kind_n[12] = {0}, last_n[12] = {0};
    uint64_t split_counts[2 * oxd::C_N] = {0};
    // execution mode: megakernel or wavefront, and the wavefront's buffers
    uint32_t mode = OXPT_MODE_WAVEFRONT;
    uint32_t wave_slots = 1u << 20;
    uint64_t wave_items = oxd::DEFAULT_WAVE_ITEMS;
    uint32_t check_every = 4;
    uint32_t shade_variant = 1, trace_variant = 4, nee_variant = 3, stack = 0;
    uint32_t bvh_depth = 0;
    // four-wide any-hit tree (host/bvh4.cpp), built on upload when exact
    float4* bvh4 = nullptr;
    bool bvh4_built = false;
    uint32_t bvh4_nodes = 0, bvh4_root = 0xffffffffu, bvh4_need = 0;
    uint32_t shadow_walk = 0;
    uint32_t closest_walk = 0;  // 1: continuation rays on the four-wide tree (tolerance plan)
    uint32_t fast_shading = 0;  // 1: the split kernels' fast-math build (tolerance plan)
    // split plan: per-slot visibility masks instead of a pending record per
    // NEE job (oxpt_diag_set_nee_mask; results are the same either way)
    bool nee_mask = true;
    uint32_t shadow_post = 0;  // four-wide shadow walks with postponed leaves (oxpt_diag_set_shadow_postpone)
    uint32_t ray_order = 0;    // continuation queue reordered before the walk (oxpt_diag_set_ray_order)
    // tree nodes of the walks as persisting L2 lines (oxpt_diag_set_l2_window):
    // the set-aside granted and the largest window the device takes
    uint64_t l2_setaside = 0, l2_max_window = 0;
    uint32_t refill = 8;  // traversal lanes idle in a warp before it fetches rays
    // traversal variants 3-5: stack entries per lane kept in shared memory,
    // top nodes of the binary tree staged per CTA (oxpt_diag_set_walk)
    uint32_t walk_lim = oxd::WaveArgs{}.walk_lim, walk_stage = oxd::WaveArgs{}.walk_stage;
    void* wave_mem = nullptr;
    size_t wave_bytes = 0;
    uint32_t wave_cap_slots = 0, wave_cap_jobs = 0;
    uint32_t* wave_host = nullptr;  // pinned: [0..2] counters snapshot
    uint64_t wave_iterations = 0;
    // batched refinement as an executor: frame records of every round
    oxd::BatchFrame* batch_dev = nullptr;
    size_t batch_cap = 0;
    cudaEvent_t batch_done = nullptr;
    oxd::BatchFrame* batch_host = nullptr;  // pinned staging of the records
    cudaEvent_t batch_copied = nullptr;     // the staging buffer's last upload
    std::vector<oxpt_ctx*> batch_ctx;  // frame contexts of the current batch
    // CUDA-graph batches: the instantiated graph of the last step shape
    uint32_t graphs = 0;
    cudaStream_t capture = nullptr;  // stream the loop bodies are captured on
    cudaGraphExec_t bgraph = nullptr;
    std::vector<uint64_t> bgraph_key;
    // the step shape before it: a context that re-stages its scene every
    // step alternates between its two scene buffer sets, one graph each
    cudaGraphExec_t bgraph_alt = nullptr;
    std::vector<uint64_t> bgraph_alt_key;
    uint64_t graph_builds = 0;
    unsigned long long* dev_tally = nullptr;  // graph loops: kernels launched, iterations
    float build_ms[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // last oxpt_build_scene: phases, wall, tree, launches
    size_t geom_cap = 0, attrs_cap = 0, atlas_cap = 0;  // bytes of the owned scene buffers
    size_t bvh4_cap = 0, tables_cap = 0;
    // oxpt_stage_scene: the second buffer set, its upload stream and events
    SceneSet back;
    bool staged = false;          // `back` holds a scene not yet traced
    bool back_free_valid = false;  // back_free marks the back set's last use
    cudaStream_t upload = nullptr;
    cudaEvent_t staged_ready = nullptr, back_free = nullptr;
};

namespace {

oxpt_status fail(oxpt_ctx* c, oxpt_status s, const std::string& msg) {
    if (c) c->err = msg;
    return s;
}

oxpt_status cuda_fail(oxpt_ctx* c, cudaError_t e, const char* what) {
    (void)cudaGetLastError();
    std::string m = std::string("cuda: ") + what + ": " + cudaGetErrorString(e);
    return fail(c, e == cudaErrorMemoryAllocation ? OXPT_E_NOMEM : OXPT_E_CUDA, m);
}

#define CK(c, expr, what)                                  \
    do {                                                   \
        cudaError_t e_ = (expr);                           \
        if (e_ != cudaSuccess) return cuda_fail(c, e_, what); \
    } while (0)

template <class T>
oxpt_status realloc_dev(oxpt_ctx* c, T** p, size_t bytes, const char* what) {
    if (*p) {
        cudaFree(*p);
        *p = nullptr;
    }
    if (bytes == 0) return OXPT_OK;
    cudaError_t e = cudaMalloc((void**)p, bytes);
    if (e != cudaSuccess) {
        *p = nullptr;
        return cuda_fail(c, e, what);
    }
    return OXPT_OK;
}

// The four-wide tree answers any-hit queries exactly when it was built from
// the whole tree the params name and the binary walk it replaces never
// overflows its 64-entry stack (at most 64 levels).
bool bvh4_usable(const oxpt_ctx* c) {
    return c->bvh4_built && c->params.env[3] == c->node_count && c->bvh_depth <= 64 && c->bvh4_need <= 64;
}

// Keeps an owned scene buffer that already holds `bytes` (and is at most
// twice that) instead of freeing and allocating it again: a re-upload of the
// same scene then costs only its copies.
template <class T>
oxpt_status reserve_dev(oxpt_ctx* c, T** p, size_t* cap, size_t bytes, const char* what) {
    if (*p && bytes > 0 && *cap >= bytes && *cap / 2 <= bytes) return OXPT_OK;
    oxpt_status s = realloc_dev(c, p, bytes, what);
    *cap = s ? 0 : bytes;
    return s;
}

// A borrowed scene is not freed here: the lending context owns it.
void drop_borrowed_scene(oxpt_ctx* c) {
    if (!c->borrowed_scene) return;
    c->geom_cap = c->attrs_cap = c->atlas_cap = 0;
    c->bvh4_cap = 0;
    c->geom = nullptr;
    c->attrs = nullptr;
    c->atlas = nullptr;
    c->bvh4 = nullptr;
    c->borrowed_scene = false;
    c->bvh4_built = false;
}

oxd::Scene scene_view(const oxpt_ctx* c) {
    oxd::Scene s;
    s.geom = c->geom;
    s.geom_vec4 = c->geom_vec4;
    s.attrs = c->attrs;
    s.slot_count = c->slot_count;
    s.tables = c->tables;
    s.table_words = c->table_words;
    s.atlas = c->atlas;
    s.side = c->side;
    s.layers = c->layers;
    s.P = c->params;
    if (bvh4_usable(c)) {
        s.bvh4 = c->bvh4;
        s.bvh4_root = c->bvh4_root;
        s.bvh4_nodes = c->bvh4_nodes;
        s.bvh4_ok = 1u;
    }
    return s;
}

oxpt_status set_device(oxpt_ctx* c) {
    CK(c, cudaSetDevice(c->device), "cudaSetDevice");
    return OXPT_OK;
}

void swap_scene(oxpt_ctx* c) {
    SceneSet& b = c->back;
    std::swap(c->geom, b.geom);
    std::swap(c->geom_vec4, b.geom_vec4);
    std::swap(c->geom_cap, b.geom_cap);
    std::swap(c->attrs, b.attrs);
    std::swap(c->slot_count, b.slot_count);
    std::swap(c->attrs_cap, b.attrs_cap);
    std::swap(c->atlas, b.atlas);
    std::swap(c->side, b.side);
    std::swap(c->layers, b.layers);
    std::swap(c->atlas_cap, b.atlas_cap);
    std::swap(c->node_count, b.node_count);
    std::swap(c->bvh_depth, b.bvh_depth);
    std::swap(c->bvh4, b.bvh4);
    std::swap(c->bvh4_cap, b.bvh4_cap);
    std::swap(c->bvh4_built, b.bvh4_built);
    std::swap(c->bvh4_nodes, b.bvh4_nodes);
    std::swap(c->bvh4_root, b.bvh4_root);
    std::swap(c->bvh4_need, b.bvh4_need);
    std::swap(c->tables, b.tables);
    std::swap(c->table_words, b.table_words);
    std::swap(c->tables_cap, b.tables_cap);
    std::swap(c->table_head, b.table_head);
}

// Makes a staged scene current: work enqueued from here on waits for its
// upload on the device and traces it; everything enqueued before traced
// the previous set, whose last use the back_free event marks.
oxpt_status activate_staged(oxpt_ctx* c) {
    if (!c->staged) return OXPT_OK;
    CK(c, cudaSetDevice(c->device), "cudaSetDevice");
    CK(c, cudaStreamWaitEvent(c->stream, c->staged_ready, 0), "staged scene order");
    swap_scene(c);
    c->staged = false;
    c->has_scene = true;
    c->has_tables = true;
    if (c->stack == 32 && c->bvh_depth > 32) c->stack = 0;
    CK(c, cudaEventRecord(c->back_free, c->stream), "staged scene order");
    c->back_free_valid = true;
    return OXPT_OK;
}

oxpt_status ready(oxpt_ctx* c) {
    oxpt_status s = activate_staged(c);
    if (s) return s;
    if (!c->has_scene || !c->has_tables || !c->has_params) return fail(c, OXPT_E_INVALID, "scene, tables and params must be set first");
    if (!c->accum) return fail(c, OXPT_E_INVALID, "no accumulator: call oxpt_resize first");
    if (c->params.dims[0] != c->w || c->params.dims[1] != c->h)
        return fail(c, OXPT_E_INVALID, "params dims do not match the accumulator size");
    return OXPT_OK;
}

oxpt_status ensure_out(oxpt_ctx* c, uint64_t paths) {
    if (paths <= c->out_cap) return OXPT_OK;
    oxpt_status s = realloc_dev(c, &c->out, paths * sizeof(float4), "path result buffer");
    if (s != OXPT_OK) {
        c->out_cap = 0;
        return s;
    }
    c->out_cap = paths;
    return OXPT_OK;
}

uint32_t trace_grid(oxpt_ctx* c, uint64_t total, bool count) {
    uint32_t bpsm = c->blocks_per_sm;
    if (bpsm == 0) bpsm = (uint32_t)std::max(1, oxd::trace_blocks_per_sm(c->threads, count));
    uint64_t blocks = (uint64_t)c->sms * bpsm;
    uint64_t need = (total + c->threads - 1) / c->threads;
    return (uint32_t)std::max<uint64_t>(1, std::min(blocks, need));
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Levels of the BVH (root = 1), walking the node words on the host; a
// malformed tree (child index out of range or a cycle) reports 65 so that
// the reference's 64-entry stack is used.
uint32_t bvh_depth_of(const uint32_t* geom, uint32_t nodes) {
    if (nodes == 0) return 0;
    std::vector<std::pair<uint32_t, uint32_t>> st;
    st.push_back({0u, 1u});
    uint32_t depth = 0;
    uint64_t visits = 0;
    while (!st.empty()) {
        auto [n, d] = st.back();
        st.pop_back();
        if (++visits > (uint64_t)nodes || d > 64) return 65;
        depth = std::max(depth, d);
        uint32_t first = geom[(size_t)n * 8 + 3], count = geom[(size_t)n * 8 + 7];
        if (count == 0) {
            if ((uint64_t)first + 1 >= nodes) return 65;
            st.push_back({first, d + 1});
            st.push_back({first + 1, d + 1});
        }
    }
    return depth;
}

// Carve the wavefront's path state and queues out of one allocation.
oxpt_status ensure_wave(oxpt_ctx* c, uint32_t slots, uint32_t jobs, oxd::WaveState* st, oxd::WaveQueues* q,
                        uint32_t** ctr, unsigned long long** work) {
    size_t P = slots, PJ = (size_t)slots * jobs;
    bool split = c->mode == OXPT_MODE_WAVEFRONT_SPLIT;
    size_t sizes[] = {P * 8, P * 16, P * 16, P * 16, P * 16, P * 16, P * 16, P * 16, P * 16, P * 4, P * 4,
                      PJ * 16, P * 4, PJ * 16, PJ * 16, PJ * 16, 64,
                      split ? P * 4 : 0, split ? P * 4 : 0, split ? 13 * P * 16 : 0, P * 4,
                      (split && jobs <= 32) ? P * 4 : 0, P * 4, PJ * 4, PJ * 4, (size_t)(1u << 17) * 4, PJ * 4};
    constexpr int NB = 27;
    size_t total = 0;
    for (size_t s : sizes) total += align256(s);
    if (slots > c->wave_cap_slots || jobs > c->wave_cap_jobs || total > c->wave_bytes) {
        if (c->wave_mem) cudaFree(c->wave_mem);
        c->wave_mem = nullptr;
        c->wave_bytes = 0;
        cudaError_t e = cudaMalloc(&c->wave_mem, total);
        if (e != cudaSuccess) {
            c->wave_mem = nullptr;
            c->wave_cap_slots = c->wave_cap_jobs = 0;
            return cuda_fail(c, e, "wavefront path state");
        }
        c->wave_bytes = total;
        c->wave_cap_slots = slots;
        c->wave_cap_jobs = jobs;
    }
    char* p = (char*)c->wave_mem;
    void* ptr[NB];
    for (int k = 0; k < NB; k++) {
        ptr[k] = p;
        p += align256(sizes[k]);
    }
    q->shade = split ? (uint32_t*)ptr[17] : nullptr;
    q->vslot = split ? (uint32_t*)ptr[18] : nullptr;
    q->vrec = split ? (float4*)ptr[19] : nullptr;
    st->item = (unsigned long long*)ptr[0];
    st->seed = (uint4*)ptr[1];
    st->beta = (float4*)ptr[2];
    st->rad = (float4*)ptr[3];
    st->dir = (float4*)ptr[4];
    st->org = (float4*)ptr[5];
    st->prev = (float4*)ptr[6];
    st->sigma = (float4*)ptr[7];
    st->hit = (uint4*)ptr[8];
    st->hmeta = (uint32_t*)ptr[9];
    st->nee_n = (uint32_t*)ptr[10];
    st->pend = (float4*)ptr[11];
    st->frame = (uint32_t*)ptr[20];
    st->vis = (split && jobs <= 32 && c->nee_mask) ? (uint32_t*)ptr[21] : nullptr;
    q->ext_sorted = (uint32_t*)ptr[22];
    q->ord_key = (uint32_t*)ptr[23];
    q->ord_rank = (uint32_t*)ptr[24];
    q->ord_hist = (uint32_t*)ptr[25];
    q->sh_perm = (uint32_t*)ptr[26];
    q->ext = (uint32_t*)ptr[12];
    q->sh_o = (float4*)ptr[13];
    q->sh_d = (float4*)ptr[14];
    q->sh_m = (uint4*)ptr[15];
    *ctr = (uint32_t*)ptr[16];
    *work = (unsigned long long*)((char*)ptr[16] + 32);
    if (!c->wave_host) {
        cudaError_t e = cudaMallocHost((void**)&c->wave_host, 64);
        if (e != cudaSuccess) {
            c->wave_host = nullptr;
            return cuda_fail(c, e, "pinned counters");
        }
    }
    return OXPT_OK;
}

// One sub-frame through the wavefront: iterate logic / extend / shadow
// until every slot is empty, then reduce in sample order.
oxpt_status wave_loop(oxpt_ctx* c, const oxd::WaveArgs& wa, bool count, bool four, int sd, int sd4,
                      uint32_t max_bounces);

oxpt_status run_wave(oxpt_ctx* c, const oxd::TraceArgs& ta, bool count, const oxd::NrcWave* nrc = nullptr) {
    uint32_t J = c->params.cfg[2] + 1u;
    uint64_t total = ta.total;
    uint32_t P = (uint32_t)std::min<uint64_t>(total, c->wave_slots);
    oxd::WaveArgs wa;
    oxpt_status s = ensure_wave(c, P, J, &wa.st, &wa.q, &wa.ctr, &wa.work);
    if (s) return s;
    wa.s = ta.s;
    wa.slots = P;
    wa.vcap = P;
    wa.jobs = J;
    wa.refill = c->refill;
    wa.first = ta.first;
    wa.y0 = ta.y0;
    wa.npix = ta.npix;
    wa.total = total;
    wa.out = ta.out;
    wa.counters = ta.counters;
    wa.err = ta.err;
    wa.frames = nullptr;
    wa.nframes = 0;
    wa.nrc = nrc ? *nrc : oxd::NrcWave{};
    wa.walk_lim = c->walk_lim;
    wa.walk_stage = c->walk_stage;
    wa.shadow_post = c->shadow_post;
    wa.ray_order = c->ray_order;
    wa.l2_share = c->l2_setaside / 2;  // two trees: binary for closest hits, four-wide for shadows
    wa.l2_max_window = c->l2_max_window;
    wa.closest4 = (c->closest_walk && c->trace_variant >= 3 && bvh4_usable(c)) ? 1u : 0u;
    // Stack depth: 32 entries are exact when the BVH has at most 32 levels.
    int sd = c->stack ? (int)c->stack : (c->bvh_depth <= 32 ? 32 : 64);
    bool four = c->shadow_walk == 0 && bvh4_usable(c);
    int sd4 = c->bvh4_need <= 32 ? 32 : 64;
    return wave_loop(c, wa, count, four, sd, sd4, c->params.dims[3]);
}

// The iteration bound of a wavefront run: four times the bounces of every
// path a slot can take, plus slack. A run that has not drained by then is
// an error, not a hang.
uint64_t wave_cap(const oxd::WaveArgs& wa, uint32_t max_bounces) {
    uint64_t per_slot = wa.total / wa.slots + 1;
    uint64_t bounces = std::min<uint64_t>(max_bounces, 1u << 20);
    return 4 * (bounces + 2) * per_slot + 1024;
}

cudaError_t wave_init(const oxd::WaveArgs& wa, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(wa.st.rad, 0, (size_t)wa.slots * 16, st);
    if (!e) e = cudaMemsetAsync(wa.st.nee_n, 0, (size_t)wa.slots * 4, st);
    if (!e) e = cudaMemsetAsync(wa.ctr, 0, 64, st);
    return e;
}

// Kernels of one wavefront iteration on `st`: queue reset, shading
// (one logic kernel, or logic + surface shading + NEE jobs in the split
// plan), extension and shadow traversal. `wrap(kind, launch)` runs each
// launch (timing hooks); returns the kernels enqueued, or -1 on error.
template <class Wrap>
int enqueue_iteration(oxpt_ctx* c, const oxd::WaveArgs& wa, const oxd::WaveArgs& wsh, bool count, bool four, int sd,
                      int sd4, cudaStream_t st, Wrap&& wrap, cudaError_t* err) {
    int n = 0;
    auto run = [&](int kind, auto&& launch) {
        if (*err) return;
        *err = wrap(kind, launch);
        n++;
    };
    *err = cudaMemsetAsync(wa.ctr, 0, 32, st);
    if (c->mode == OXPT_MODE_WAVEFRONT_SPLIT && c->fast_shading) {
        run(2, [&] { return oxd::fast::launch_split_logic(wa, count, st); });
        run(5, [&] { return oxd::fast::launch_split_shade(wa, count, (int)c->shade_variant, c->sms, st); });
        run(6, [&] { return oxd::fast::launch_split_nee(wa, count, (int)c->nee_variant, c->sms, st); });
    } else if (c->mode == OXPT_MODE_WAVEFRONT_SPLIT) {
        run(2, [&] { return oxd::launch_split_logic(wa, count, st); });
        run(5, [&] { return oxd::launch_split_shade(wa, count, (int)c->shade_variant, c->sms, st); });
        run(6, [&] { return oxd::launch_split_nee(wa, count, (int)c->nee_variant, c->sms, st); });
    } else {
        run(2, [&] { return oxd::launch_wave_logic(wa, count, (int)c->shade_variant, st); });
    }
    if (wa.ray_order & 1u) {
        run(10, [&] { return oxd::launch_order_ext(wa, c->sms, st); });
        oxd::WaveArgs wo = wa;
        wo.q.ext = wa.q.ext_sorted;
        run(3, [&] { return oxd::launch_wave_extend(wo, count, (int)c->trace_variant, wa.closest4 ? sd4 : sd, c->sms, st); });
    } else {
        run(3, [&] { return oxd::launch_wave_extend(wa, count, (int)c->trace_variant, wa.closest4 ? sd4 : sd, c->sms, st); });
    }
    if ((wa.ray_order & 2u) && c->trace_variant >= 3)
        run(10, [&] { return oxd::launch_order_shadow(wa, c->sms, st); });
    run(4, [&] {
        return oxd::launch_wave_shadow(wsh, count, four, (int)c->trace_variant, four ? sd4 : sd, c->sms, st);
    });
    return *err ? -1 : n;
}

// Iterates the wavefront's kernels over `wa` until every slot is empty,
// checking the active-slot count on the host every check_every iterations.
oxpt_status wave_loop(oxpt_ctx* c, const oxd::WaveArgs& wa, bool count, bool four, int sd, int sd4,
                      uint32_t max_bounces) {
    CK(c, wave_init(wa, c->stream), "wave init");
    const uint64_t cap = wave_cap(wa, max_bounces);
    oxd::WaveArgs wsh = wa;  // shadow rays count into the second counter half
    if (wsh.counters) wsh.counters += oxd::C_N;
    auto timed = [&](int kind, auto&& launch) -> cudaError_t {
        oxpt_ctx::Timed t{nullptr, nullptr, kind};
        if (c->timing) {
            cudaEventCreate(&t.a);
            cudaEventCreate(&t.b);
            cudaEventRecord(t.a, c->stream);
        }
        cudaError_t e = launch();
        if (c->timing) {
            cudaEventRecord(t.b, c->stream);
            c->timed.push_back(t);
        }
        return e;
    };
    for (uint64_t it = 0;; it++) {
        if (it > cap) return fail(c, OXPT_E_TIMEOUT, "wavefront did not drain within its iteration bound");
        cudaError_t e = cudaSuccess;
        int n = enqueue_iteration(c, wa, wsh, count, four, sd, sd4, c->stream, timed, &e);
        if (n < 0) return cuda_fail(c, e, "wavefront iteration");
        c->launches += (uint64_t)n;
        c->wave_iterations++;
        if ((it + 1) % c->check_every == 0) {
            CK(c, cudaMemcpyAsync(c->wave_host, wa.ctr, 16, cudaMemcpyDeviceToHost, c->stream), "queue readback");
            CK(c, cudaStreamSynchronize(c->stream), "queue readback");
            if (c->wave_host[2] == 0) break;
        }
    }
    return OXPT_OK;
}

// One dispatch = frame {first, count, y0, rows}, split into launches of at
// most max_paths paths (megakernel) or wave_items (wavefront); each launch
// traces into `out` and reduces in sample order.
oxpt_status run_frame(oxpt_ctx* c, const oxpt_frame& f, bool count) {
    if (f.count == 0 || f.rows == 0) return OXPT_OK;
    if (f.y0 >= c->h || f.rows > c->h - f.y0) return fail(c, OXPT_E_INVALID, "frame rows outside the image");
    if (c->graphs && !count && c->mode != OXPT_MODE_MEGAKERNEL) {
        // Graph plan: the frame as a batch of one, one CUDA graph per step.
        oxpt_batch_frame bf{c, f.first, f.count, f.y0, f.rows};
        return oxpt_refine_batch(c, &bf, 1);
    }
    bool wave = c->mode != OXPT_MODE_MEGAKERNEL;
    uint64_t cap = std::max<uint64_t>(wave ? c->wave_items : c->max_paths, c->w);
    uint32_t rows_per = f.rows, per = f.count;
    uint64_t row_paths = (uint64_t)c->w * f.rows;
    if (row_paths > cap) {
        rows_per = (uint32_t)std::max<uint64_t>(1, cap / c->w);
        per = 1;
    } else {
        per = (uint32_t)std::min<uint64_t>(f.count, cap / row_paths);
    }
    oxpt_status st = ensure_out(c, (uint64_t)c->w * rows_per * per);
    if (st != OXPT_OK) return st;
    oxd::TraceArgs ta;
    ta.s = scene_view(c);
    ta.out = c->out;
    ta.counters = c->dev_counters;
    ta.err = c->dev_err;
    for (uint32_t s0 = 0; s0 < f.count; s0 += per) {
        uint32_t n = std::min(per, f.count - s0);
        for (uint32_t r0 = 0; r0 < f.rows; r0 += rows_per) {
            uint32_t rows = std::min(rows_per, f.rows - r0);
            ta.first = f.first + s0;
            ta.count = n;
            ta.y0 = f.y0 + r0;
            ta.rows = rows;
            ta.npix = c->w * rows;
            ta.total = (uint64_t)ta.npix * n;
            oxpt_ctx::Timed tt{nullptr, nullptr, 0}, tr{nullptr, nullptr, 1};
            if (c->timing) {
                CK(c, cudaEventCreate(&tt.a), "event");
                CK(c, cudaEventCreate(&tt.b), "event");
                CK(c, cudaEventCreate(&tr.a), "event");
                CK(c, cudaEventCreate(&tr.b), "event");
                CK(c, cudaEventRecord(tt.a, c->stream), "event record");
            }
            if (wave) {
                oxpt_status ws = run_wave(c, ta, count);
                if (ws) return ws;
            } else {
                CK(c, oxd::launch_trace(ta, count, trace_grid(c, ta.total, count), c->threads, c->stream),
                   "trace launch");
                c->launches += 1;
            }
            if (c->timing) {
                CK(c, cudaEventRecord(tt.b, c->stream), "event record");
                CK(c, cudaEventRecord(tr.a, c->stream), "event record");
            }
            oxd::ReduceArgs ra{c->accum, c->out, c->w, ta.y0, ta.npix, n};
            CK(c, oxd::launch_reduce(ra, c->stream), "reduce launch");
            if (c->timing) {
                CK(c, cudaEventRecord(tr.b, c->stream), "event record");
                c->timed.push_back(tt);
                c->timed.push_back(tr);
            }
            c->launches += 1;
        }
    }
    return OXPT_OK;
}

}  // namespace

extern "C" {

uint32_t oxpt_abi_version(void) { return OXPT_ABI_VERSION; }

oxpt_status oxpt_create(int device, oxpt_ctx** out) {
    if (!out) return OXPT_E_INVALID;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        (void)cudaGetLastError();
        return OXPT_E_NODEV;
    }
    if (device < 0 || device >= n) return OXPT_E_NODEV;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return OXPT_E_NODEV;
    if (prop.major < 10) return OXPT_E_NODEV;  // built for sm_100a only
    auto* c = new oxpt_ctx();
    c->device = device;
    c->sms = prop.multiProcessorCount;
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc((void**)&c->dev_err, sizeof(uint32_t)) != cudaSuccess ||
        cudaMalloc((void**)&c->dev_counters, sizeof(unsigned long long) * 2 * oxd::C_N) != cudaSuccess ||
        cudaMemset(c->dev_err, 0, sizeof(uint32_t)) != cudaSuccess) {
        (void)cudaGetLastError();
        oxpt_destroy(c);
        return OXPT_E_CUDA;
    }
    c->stream = c->own;
    *out = c;
    return OXPT_OK;
}

oxpt_status oxpt_destroy(oxpt_ctx* c) {
    if (!c) return OXPT_OK;
    cudaSetDevice(c->device);
    if (c->own) cudaStreamSynchronize(c->own);
    if (c->stream && c->stream != c->own) cudaStreamSynchronize(c->stream);
    for (auto& t : c->timed) {
        cudaEventDestroy(t.a);
        cudaEventDestroy(t.b);
    }
    drop_borrowed_scene(c);
    if (c->borrowed_tables) c->tables = nullptr;
    if (c->upload) cudaStreamSynchronize(c->upload);
    void* ptrs[] = {c->geom, c->attrs, c->atlas, c->tables, c->accum, c->img8, c->img32, c->out, c->dev_err,
                    c->dev_counters, c->wave_mem, c->bvh4, c->batch_dev, c->back.geom, c->back.attrs,
                    c->back.atlas, c->back.bvh4, c->back.tables};
    if (c->upload) cudaStreamDestroy(c->upload);
    if (c->staged_ready) cudaEventDestroy(c->staged_ready);
    if (c->back_free) cudaEventDestroy(c->back_free);
    if (c->batch_done) cudaEventDestroy(c->batch_done);
    if (c->copy) cudaStreamSynchronize(c->copy);
    if (c->present) cudaFree(c->present);
    if (c->resolved) cudaEventDestroy(c->resolved);
    if (c->copied) cudaEventDestroy(c->copied);
    if (c->copy) cudaStreamDestroy(c->copy);
    if (c->batch_copied) cudaEventDestroy(c->batch_copied);
    if (c->batch_host) cudaFreeHost(c->batch_host);
    if (c->ready) cudaEventDestroy(c->ready);
    for (cudaEvent_t ev : c->marks) cudaEventDestroy(ev);
    if (c->bgraph) cudaGraphExecDestroy(c->bgraph);
    if (c->bgraph_alt) cudaGraphExecDestroy(c->bgraph_alt);
    if (c->dev_tally) cudaFree(c->dev_tally);
    if (c->capture) cudaStreamDestroy(c->capture);
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (c->wave_host) cudaFreeHost(c->wave_host);
    if (c->own) cudaStreamDestroy(c->own);
    (void)cudaGetLastError();
    delete c;
    return OXPT_OK;
}

const char* oxpt_last_error(const oxpt_ctx* c) { return c ? c->err.c_str() : "null context"; }

oxpt_status oxpt_set_stream(oxpt_ctx* c, void* stream) {
    if (!c) return OXPT_E_INVALID;
    c->stream = stream ? (cudaStream_t)stream : c->own;
    return OXPT_OK;
}

void* oxpt_get_stream(const oxpt_ctx* c) { return c ? (void*)c->stream : nullptr; }

oxpt_status oxpt_device_summary(const oxpt_ctx* c, char* buf, size_t len) {
    if (!c || !buf || !len) return OXPT_E_INVALID;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, c->device) != cudaSuccess) return OXPT_E_CUDA;
    std::snprintf(buf, len, "%s (sm_%d%d, %d SMs, %zu MiB)", prop.name, prop.major, prop.minor,
                  prop.multiProcessorCount, (size_t)(prop.totalGlobalMem >> 20));
    return OXPT_OK;
}

// Collapse the uploaded binary tree into the four-wide any-hit tree; a
// tree that does not collapse exactly keeps the binary walk.
static oxpt_status install_bvh4(oxpt_ctx* c, bool ok, const std::vector<uint32_t>& words, uint32_t root) {
    c->bvh4_built = false;
    if (!ok) return OXPT_OK;  // the binary walk serves every ray
    oxpt_status s = reserve_dev(c, &c->bvh4, &c->bvh4_cap, words.size() * 4, "four-wide tree");
    if (s) return s;
    if (!words.empty()) {
        CK(c, cudaMemcpyAsync(c->bvh4, words.data(), words.size() * 4, cudaMemcpyHostToDevice, c->stream),
           "four-wide tree upload");
        CK(c, cudaStreamSynchronize(c->stream), "four-wide tree upload");
    }
    c->bvh4_nodes = (uint32_t)(words.size() / oxpt::BVH4_NODE_WORDS);
    c->bvh4_root = root;
    c->bvh4_need = oxpt::bvh4_stack_need(words, root);
    c->bvh4_built = true;
    return OXPT_OK;
}

static oxpt_status upload_bvh4(oxpt_ctx* c, const uint32_t* node_words, uint32_t node_count) {
    std::vector<uint32_t> words;
    uint32_t root = 0xffffffffu;
    bool ok = oxpt::build_bvh4(node_words, node_count, &words, &root);
    return install_bvh4(c, ok, words, root);
}

// The four-wide tree of the scene now in c->geom, collapsed on the device
// (the host collapse's words); a tree too wide or deep for the device pass
// is read back and collapsed on the host.
static oxpt_status device_bvh4(oxpt_ctx* c) {
    c->bvh4_built = false;
    uint32_t* out = reinterpret_cast<uint32_t*>(c->bvh4);  // reused when large enough
    uint32_t n4 = 0, root = 0xffffffffu, need = 1;
    std::string e;
    const uint32_t* words = reinterpret_cast<const uint32_t*>(c->geom);
    oxd::Collapse r = oxd::collapse4_device(words, c->node_count, c->stream, &out, &c->bvh4_cap, &n4, &root, &need, &e);
    c->bvh4 = reinterpret_cast<float4*>(out);
    if (r == oxd::Collapse::FAILED) return fail(c, OXPT_E_CUDA, e);
    if (r == oxd::Collapse::REFUSED) return OXPT_OK;  // the binary walk serves every ray
    if (r == oxd::Collapse::UNSUPPORTED) {
        std::vector<uint32_t> host((size_t)c->node_count * 8);
        CK(c, cudaMemcpy(host.data(), c->geom, host.size() * 4, cudaMemcpyDeviceToHost), "node readback");
        return upload_bvh4(c, host.data(), c->node_count);
    }
    c->bvh4_nodes = n4;
    c->bvh4_root = root;
    c->bvh4_need = need;
    c->bvh4_built = true;
    return OXPT_OK;
}

oxpt_status oxpt_upload_scene(oxpt_ctx* c, const oxpt_scene_desc* d) {
    if (!c || !d) return fail(c, OXPT_E_INVALID, "null argument");
    if (oxpt_status sa = activate_staged(c)) return sa;
    if (!d->geom || d->geom_words < 8 || d->geom_words % 4 != 0) return fail(c, OXPT_E_INVALID, "geom must hold at least one node (8 words), a multiple of 4 words");
    if (!d->attrs || d->attr_floats < 48 || d->attr_floats % 48 != 0) return fail(c, OXPT_E_INVALID, "attrs must be 48 floats per slot");
    if ((size_t)d->node_count * 8 + (size_t)d->slot_count * 12 > d->geom_words) return fail(c, OXPT_E_INVALID, "geom smaller than nodes + triangles");
    if ((size_t)d->slot_count * 48 > d->attr_floats) return fail(c, OXPT_E_INVALID, "attrs smaller than the slot count");
    if (!d->atlas || d->atlas_side == 0 || d->atlas_layers == 0) return fail(c, OXPT_E_INVALID, "atlas must have at least one layer");
    if (d->atlas_side > 16384) return fail(c, OXPT_E_LIMIT, "atlas layer side above 16384");
    oxpt_status s = set_device(c);
    if (s) return s;
    CK(c, cudaStreamSynchronize(c->stream), "sync before upload");
    c->has_scene = false;
    drop_borrowed_scene(c);
    size_t gbytes = d->geom_words * 4, abytes = d->attr_floats * 4;
    size_t tbytes = (size_t)d->atlas_side * d->atlas_side * d->atlas_layers * 8;
    if ((s = reserve_dev(c, &c->geom, &c->geom_cap, gbytes, "geom buffer"))) return s;
    if ((s = reserve_dev(c, &c->attrs, &c->attrs_cap, abytes, "attribute buffer"))) return s;
    if ((s = reserve_dev(c, &c->atlas, &c->atlas_cap, tbytes, "texture atlas"))) return s;
    CK(c, cudaMemcpyAsync(c->geom, d->geom, gbytes, cudaMemcpyHostToDevice, c->stream), "geom upload");
    CK(c, cudaMemcpyAsync(c->attrs, d->attrs, abytes, cudaMemcpyHostToDevice, c->stream), "attr upload");
    CK(c, cudaMemcpyAsync(c->atlas, d->atlas, tbytes, cudaMemcpyHostToDevice, c->stream), "atlas upload");
    CK(c, cudaStreamSynchronize(c->stream), "upload");
    c->geom_vec4 = d->geom_words / 4;
    c->slot_count = d->attr_floats / 48;
    c->side = d->atlas_side;
    c->layers = d->atlas_layers;
    c->node_count = d->node_count;
    {
        // Depth and four-wide tree from the uploaded words, on the device.
        std::string e;
        uint32_t depth = 0;
        if (!oxd::binary_depth_device(reinterpret_cast<const uint32_t*>(c->geom), d->node_count, c->stream, &depth,
                                      &e))
            return fail(c, OXPT_E_CUDA, e);
        c->bvh_depth = depth;
    }
    if (c->stack == 32 && c->bvh_depth > 32) c->stack = 0;
    if ((s = device_bvh4(c))) return s;
    c->has_scene = true;
    return OXPT_OK;
}

// The staged upload: the scene's buffers and tables go into the context's
// second buffer set on its upload stream, after the work that last traced
// that set; the tree passes of an upload (depth, four-wide collapse) run
// there too. The host waits for those, not for the context's stream, so
// the copies overlap whatever is already queued there.
oxpt_status oxpt_stage_scene(oxpt_ctx* c, const oxpt_scene_desc* d, const uint32_t* tables, size_t table_words) {
    if (!c || !d) return fail(c, OXPT_E_INVALID, "null argument");
    if (!tables || table_words == 0) return fail(c, OXPT_E_INVALID, "empty tables");
    if (!d->geom || d->geom_words < 8 || d->geom_words % 4 != 0) return fail(c, OXPT_E_INVALID, "geom must hold at least one node (8 words), a multiple of 4 words");
    if (!d->attrs || d->attr_floats < 48 || d->attr_floats % 48 != 0) return fail(c, OXPT_E_INVALID, "attrs must be 48 floats per slot");
    if ((size_t)d->node_count * 8 + (size_t)d->slot_count * 12 > d->geom_words) return fail(c, OXPT_E_INVALID, "geom smaller than nodes + triangles");
    if ((size_t)d->slot_count * 48 > d->attr_floats) return fail(c, OXPT_E_INVALID, "attrs smaller than the slot count");
    if (!d->atlas || d->atlas_side == 0 || d->atlas_layers == 0) return fail(c, OXPT_E_INVALID, "atlas must have at least one layer");
    if (d->atlas_side > 16384) return fail(c, OXPT_E_LIMIT, "atlas layer side above 16384");
    if (c->borrowed_scene || c->borrowed_tables)
        return fail(c, OXPT_E_INVALID, "a context borrowing a scene or tables cannot stage one");
    oxpt_status s = set_device(c);
    if (s) return s;
    if (!c->upload) CK(c, cudaStreamCreateWithFlags(&c->upload, cudaStreamNonBlocking), "upload stream");
    if (!c->staged_ready) CK(c, cudaEventCreateWithFlags(&c->staged_ready, cudaEventDisableTiming), "upload event");
    if (!c->back_free) CK(c, cudaEventCreateWithFlags(&c->back_free, cudaEventDisableTiming), "upload event");
    SceneSet& b = c->back;
    c->staged = false;
    // The back set was last traced by work enqueued before the last swap.
    if (c->back_free_valid) CK(c, cudaStreamWaitEvent(c->upload, c->back_free, 0), "upload order");
    size_t gbytes = d->geom_words * 4, abytes = d->attr_floats * 4;
    size_t tbytes = (size_t)d->atlas_side * d->atlas_side * d->atlas_layers * 8;
    if (b.geom_cap < gbytes || b.attrs_cap < abytes || b.atlas_cap < tbytes || b.tables_cap < table_words * 4)
        CK(c, cudaStreamSynchronize(c->upload), "upload order");  // the buffers may be freed
    if ((s = reserve_dev(c, &b.geom, &b.geom_cap, gbytes, "geom buffer"))) return s;
    if ((s = reserve_dev(c, &b.attrs, &b.attrs_cap, abytes, "attribute buffer"))) return s;
    if ((s = reserve_dev(c, &b.atlas, &b.atlas_cap, tbytes, "texture atlas"))) return s;
    if ((s = reserve_dev(c, &b.tables, &b.tables_cap, table_words * 4, "tables"))) return s;
    CK(c, cudaMemcpyAsync(b.geom, d->geom, gbytes, cudaMemcpyHostToDevice, c->upload), "geom upload");
    CK(c, cudaMemcpyAsync(b.attrs, d->attrs, abytes, cudaMemcpyHostToDevice, c->upload), "attr upload");
    CK(c, cudaMemcpyAsync(b.atlas, d->atlas, tbytes, cudaMemcpyHostToDevice, c->upload), "atlas upload");
    CK(c, cudaMemcpyAsync(b.tables, tables, table_words * 4, cudaMemcpyHostToDevice, c->upload), "tables upload");
    b.geom_vec4 = d->geom_words / 4;
    b.slot_count = d->attr_floats / 48;
    b.side = d->atlas_side;
    b.layers = d->atlas_layers;
    b.node_count = d->node_count;
    b.table_words = table_words;
    b.table_head.assign(tables, tables + std::min<size_t>(table_words, 4096));
    std::string e;
    uint32_t depth = 0;
    const uint32_t* words = reinterpret_cast<const uint32_t*>(b.geom);
    if (!oxd::binary_depth_device(words, d->node_count, c->upload, &depth, &e)) return fail(c, OXPT_E_CUDA, e);
    b.bvh_depth = depth;
    b.bvh4_built = false;
    uint32_t* out = reinterpret_cast<uint32_t*>(b.bvh4);
    uint32_t n4 = 0, root = 0xffffffffu, need = 1;
    oxd::Collapse r = oxd::collapse4_device(words, d->node_count, c->upload, &out, &b.bvh4_cap, &n4, &root, &need, &e);
    b.bvh4 = reinterpret_cast<float4*>(out);
    if (r == oxd::Collapse::FAILED) return fail(c, OXPT_E_CUDA, e);
    if (r == oxd::Collapse::BUILT) {
        b.bvh4_nodes = n4;
        b.bvh4_root = root;
        b.bvh4_need = need;
        b.bvh4_built = true;
    }
    // REFUSED / UNSUPPORTED: the binary walk serves every ray of this scene.
    CK(c, cudaEventRecord(c->staged_ready, c->upload), "upload event");
    CK(c, cudaStreamSynchronize(c->upload), "staged upload");  // host buffers consumed
    c->staged = true;
    return OXPT_OK;
}

oxpt_status oxpt_build_scene(oxpt_ctx* c, const oxpt_scene_src* src, uint32_t* light_slots, uint32_t out[3]) {
    if (!c || !src || !out) return fail(c, OXPT_E_INVALID, "null argument");
    if (oxpt_status sa = activate_staged(c)) return sa;
    oxpt_status s = set_device(c);
    if (s) return s;
    CK(c, cudaStreamSynchronize(c->stream), "sync before scene build");
    c->has_scene = false;
    drop_borrowed_scene(c);
    // The old scene's buffers go first: the build needs the room.
    realloc_dev(c, &c->geom, 0, "geom buffer");
    realloc_dev(c, &c->attrs, 0, "attribute buffer");
    realloc_dev(c, &c->atlas, 0, "texture atlas");
    c->geom_cap = c->attrs_cap = c->atlas_cap = 0;
    realloc_dev(c, &c->bvh4, 0, "four-wide tree");
    c->bvh4_cap = 0;
    c->bvh4_built = false;
    auto t0 = std::chrono::steady_clock::now();
    oxd::prep::DeviceScene ds;
    std::string e;
    if ((s = oxd::prep::build_scene(*src, c->stream, &ds, light_slots, &e))) return fail(c, s, e);
    auto t1 = std::chrono::steady_clock::now();
    c->geom = ds.geom;
    c->geom_vec4 = ds.geom_vec4;
    c->geom_cap = ds.geom_vec4 * 16;
    c->attrs_cap = ds.slot_count * 192;
    c->atlas_cap = (size_t)src->atlas_side * src->atlas_side * src->atlas_layers * 8;
    c->attrs = ds.attrs;
    c->slot_count = ds.slot_count;
    c->atlas = ds.atlas;
    c->side = src->atlas_side;
    c->layers = src->atlas_layers;
    c->node_count = ds.node_count;
    c->bvh_depth = std::min(ds.depth, 65u);  // bvh_depth_of's cap
    if (c->stack == 32 && c->bvh_depth > 32) c->stack = 0;
    if ((s = device_bvh4(c))) return s;
    auto t2 = std::chrono::steady_clock::now();
    for (int k = 0; k < 4; k++) c->build_ms[k] = ds.phase_ms[k];
    c->build_ms[4] = std::chrono::duration<float, std::milli>(t2 - t0).count();
    c->build_ms[5] = std::chrono::duration<float, std::milli>(t2 - t1).count();
    c->build_ms[6] = (float)ds.launches;
    c->has_scene = true;
    out[0] = ds.node_count;
    out[1] = (uint32_t)ds.slot_count;
    out[2] = ds.depth;
    return OXPT_OK;
}

oxpt_status oxpt_read_scene(oxpt_ctx* c, uint32_t* geom, float* attrs, uint16_t* atlas) {
    if (!c || !geom || !attrs || !atlas) return fail(c, OXPT_E_INVALID, "null argument");
    if (oxpt_status sa = activate_staged(c)) return sa;
    if (!c->has_scene) return fail(c, OXPT_E_INVALID, "no scene");
    oxpt_status s = set_device(c);
    if (s) return s;
    CK(c, cudaStreamSynchronize(c->stream), "sync before scene readback");
    CK(c, cudaMemcpy(geom, c->geom, c->geom_vec4 * 16, cudaMemcpyDeviceToHost), "geom readback");
    CK(c, cudaMemcpy(attrs, c->attrs, c->slot_count * 48 * 4, cudaMemcpyDeviceToHost), "attribute readback");
    CK(c, cudaMemcpy(atlas, c->atlas, (size_t)c->side * c->side * c->layers * 8, cudaMemcpyDeviceToHost),
       "atlas readback");
    return OXPT_OK;
}

oxpt_status oxpt_set_tables(oxpt_ctx* c, const uint32_t* words, size_t count) {
    if (!c || !words || count == 0) return fail(c, OXPT_E_INVALID, "empty tables");
    if (oxpt_status sa = activate_staged(c)) return sa;
    oxpt_status s = set_device(c);
    if (s) return s;
    CK(c, cudaStreamSynchronize(c->stream), "sync before tables");
    c->has_tables = false;
    if (c->borrowed_tables) {
        c->tables = nullptr;
        c->tables_cap = 0;
        c->borrowed_tables = false;
    }
    if ((s = reserve_dev(c, &c->tables, &c->tables_cap, count * 4, "tables"))) return s;
    CK(c, cudaMemcpyAsync(c->tables, words, count * 4, cudaMemcpyHostToDevice, c->stream), "tables upload");
    c->table_head.assign(words, words + std::min<size_t>(count, 4096));
    CK(c, cudaStreamSynchronize(c->stream), "tables upload");
    c->table_words = count;
    c->has_tables = true;
    return OXPT_OK;
}

oxpt_status oxpt_share_scene(oxpt_ctx* c, const oxpt_ctx* owner) {
    if (!c || !owner || c == owner) return fail(c, OXPT_E_INVALID, "sharing needs two contexts");
    if (!owner->has_scene) return fail(c, OXPT_E_INVALID, "the lending context has no scene");
    if (owner->staged || owner->back_free_valid || c->staged)
        return fail(c, OXPT_E_INVALID, "contexts that stage scenes (oxpt_stage_scene) do not share them");
    if (owner->device != c->device) return fail(c, OXPT_E_INVALID, "the lending context is on another device");
    oxpt_status s = set_device(c);
    if (s) return s;
    CK(c, cudaStreamSynchronize(c->stream), "sync before sharing");
    CK(c, cudaStreamSynchronize(owner->stream), "sync before sharing");
    drop_borrowed_scene(c);
    void* own[] = {c->geom, c->attrs, c->atlas, c->bvh4};
    for (void* p : own)
        if (p) cudaFree(p);
    c->geom_cap = c->attrs_cap = c->atlas_cap = 0;
    c->bvh4_cap = 0;
    c->geom = owner->geom;
    c->geom_vec4 = owner->geom_vec4;
    c->attrs = owner->attrs;
    c->slot_count = owner->slot_count;
    c->atlas = owner->atlas;
    c->side = owner->side;
    c->layers = owner->layers;
    c->node_count = owner->node_count;
    c->bvh_depth = owner->bvh_depth;
    c->bvh4 = owner->bvh4;
    c->bvh4_built = owner->bvh4_built;
    c->bvh4_nodes = owner->bvh4_nodes;
    c->bvh4_root = owner->bvh4_root;
    c->bvh4_need = owner->bvh4_need;
    c->borrowed_scene = true;
    c->has_scene = true;
    if (c->stack == 32 && c->bvh_depth > 32) c->stack = 0;
    return OXPT_OK;
}

oxpt_status oxpt_share_tables(oxpt_ctx* c, const oxpt_ctx* owner) {
    if (!c || !owner || c == owner) return fail(c, OXPT_E_INVALID, "sharing needs two contexts");
    if (!owner->has_tables) return fail(c, OXPT_E_INVALID, "the lending context has no tables");
    if (owner->device != c->device) return fail(c, OXPT_E_INVALID, "the lending context is on another device");
    oxpt_status s = set_device(c);
    if (s) return s;
    CK(c, cudaStreamSynchronize(c->stream), "sync before sharing");
    CK(c, cudaStreamSynchronize(owner->stream), "sync before sharing");
    if (c->borrowed_tables) c->tables = nullptr;
    else if (c->tables) cudaFree(c->tables);
    c->tables_cap = 0;
    c->tables = owner->tables;
    c->table_words = owner->table_words;
    c->table_head = owner->table_head;
    c->borrowed_tables = true;
    c->has_tables = true;
    return OXPT_OK;
}

oxpt_status oxpt_set_params(oxpt_ctx* c, const oxpt_params* p) {
    if (!c || !p) return fail(c, OXPT_E_INVALID, "null params");
    const bool scene = c->has_scene || c->staged;
    const uint32_t nodes = c->staged ? c->back.node_count : c->node_count;
    if (scene && p->env[3] > nodes) return fail(c, OXPT_E_INVALID, "node count above the uploaded nodes");
    if (p->env[2] && (p->env[0] == 0 || p->env[1] == 0)) return fail(c, OXPT_E_INVALID, "environment of zero size");
    c->params = *p;
    c->has_params = true;
    return OXPT_OK;
}

oxpt_status oxpt_resize(oxpt_ctx* c, uint32_t w, uint32_t h) {
    if (!c) return OXPT_E_INVALID;
    if (w == 0 || h == 0) return fail(c, OXPT_E_INVALID, "zero-sized image");
    if (w > 65536 || h > 65536) return fail(c, OXPT_E_LIMIT, "image side above 65536");
    oxpt_status s = set_device(c);
    if (s) return s;
    if (c->accum && c->w == w && c->h == h) return OXPT_OK;
    CK(c, cudaStreamSynchronize(c->stream), "sync before resize");
    size_t px = (size_t)w * h;
    if ((s = realloc_dev(c, &c->accum, px * 16, "accumulator"))) return s;
    if ((s = realloc_dev(c, &c->img8, px * 4, "RGBA8 output"))) return s;
    if ((s = realloc_dev(c, &c->img32, px * 16, "RGBA32F output"))) return s;
    c->w = w;
    c->h = h;
    CK(c, cudaMemsetAsync(c->accum, 0, px * 16, c->stream), "accumulator clear");
    return OXPT_OK;
}

oxpt_status oxpt_reset(oxpt_ctx* c) {
    if (!c) return OXPT_E_INVALID;
    if (!c->accum) return OXPT_OK;
    oxpt_status s = set_device(c);
    if (s) return s;
    CK(c, cudaMemsetAsync(c->accum, 0, (size_t)c->w * c->h * 16, c->stream), "accumulator clear");
    return OXPT_OK;
}

oxpt_status oxpt_dispatch(oxpt_ctx* c, const oxpt_frame* f) {
    if (!c || !f) return fail(c, OXPT_E_INVALID, "null frame");
    oxpt_status s = ready(c);
    if (s) return s;
    if ((s = set_device(c))) return s;
    return run_frame(c, *f, false);
}

oxpt_status oxpt_refine(oxpt_ctx* c, uint32_t first, uint32_t count) {
    if (!c) return OXPT_E_INVALID;
    oxpt_status s = ready(c);
    if (s) return s;
    if ((s = set_device(c))) return s;
    if (count > 0xffffffffu - first) return fail(c, OXPT_E_INVALID, "sample index overflow");
    oxpt_frame f{first, count, 0, c->h};
    return run_frame(c, f, false);
}

oxpt_status oxpt_finish(oxpt_ctx* c) {
    if (!c) return OXPT_E_INVALID;
    oxpt_status s = set_device(c);
    if (s) return s;
    CK(c, cudaStreamSynchronize(c->stream), "finish");
    uint32_t e = 0;
    CK(c, cudaMemcpy(&e, c->dev_err, 4, cudaMemcpyDeviceToHost), "error word");
    if (e) {
        cudaMemset(c->dev_err, 0, 4);
        if (e & 8u) return fail(c, OXPT_E_TIMEOUT, "wavefront did not drain within its iteration bound");
        return fail(c, OXPT_E_LIMIT, "traversal exceeded the node count: malformed BVH");
    }
    return OXPT_OK;
}

oxpt_status oxpt_resolve(oxpt_ctx* c, const oxpt_resolve_params* p, int hdr, void* host_out, oxpt_devimage* dev_out) {
    if (!c || !p) return fail(c, OXPT_E_INVALID, "null resolve params");
    if (!c->accum) return fail(c, OXPT_E_INVALID, "no accumulator: call oxpt_resize first");
    oxpt_status s = set_device(c);
    if (s) return s;
    oxd::ResolveArgs ra;
    ra.accum = c->accum;
    ra.w = c->w;
    ra.h = c->h;
    ra.p = *p;
    ra.hdr = hdr ? 1 : 0;
    ra.out = hdr ? c->img32 : c->img8;
    CK(c, oxd::launch_resolve(ra, c->stream), "resolve launch");
    c->launches += 1;
    size_t bytes = (size_t)c->w * c->h * (hdr ? 16 : 4);
    if (dev_out) {
        dev_out->data = ra.out;
        dev_out->width = c->w;
        dev_out->height = c->h;
        dev_out->pitch_bytes = c->w * (hdr ? 16u : 4u);
        dev_out->format = hdr ? OXPT_FORMAT_RGBA32F : OXPT_FORMAT_RGBA8;
    }
    if (host_out) {
        CK(c, cudaMemcpyAsync(host_out, ra.out, bytes, cudaMemcpyDeviceToHost, c->stream), "readback");
        CK(c, cudaStreamSynchronize(c->stream), "readback");
    }
    return OXPT_OK;
}

oxpt_status oxpt_resolve_async(oxpt_ctx* c, const oxpt_resolve_params* p, int hdr, void* host_out) {
    if (!c || !p || !host_out) return fail(c, OXPT_E_INVALID, "null argument");
    if (!c->accum) return fail(c, OXPT_E_INVALID, "no accumulator: call oxpt_resize first");
    oxpt_status s = set_device(c);
    if (s) return s;
    size_t bytes = (size_t)c->w * c->h * (hdr ? 16 : 4);
    if (!c->copy) CK(c, cudaStreamCreateWithFlags(&c->copy, cudaStreamNonBlocking), "copy stream");
    if (!c->resolved) CK(c, cudaEventCreateWithFlags(&c->resolved, cudaEventDisableTiming), "present event");
    if (!c->copied) CK(c, cudaEventCreateWithFlags(&c->copied, cudaEventDisableTiming), "present event");
    if (bytes > c->present_bytes) {
        CK(c, cudaStreamSynchronize(c->copy), "present buffer");
        if ((s = realloc_dev(c, &c->present, bytes, "present buffer"))) {
            c->present_bytes = 0;
            return s;
        }
        c->present_bytes = bytes;
    }
    // The previous copy out of the buffer finishes before it is rewritten.
    CK(c, cudaStreamWaitEvent(c->stream, c->copied, 0), "present order");
    oxd::ResolveArgs ra;
    ra.accum = c->accum;
    ra.w = c->w;
    ra.h = c->h;
    ra.p = *p;
    ra.hdr = hdr ? 1 : 0;
    ra.out = c->present;
    CK(c, oxd::launch_resolve(ra, c->stream), "resolve launch");
    c->launches += 1;
    CK(c, cudaEventRecord(c->resolved, c->stream), "present event");
    CK(c, cudaStreamWaitEvent(c->copy, c->resolved, 0), "present order");
    CK(c, cudaMemcpyAsync(host_out, c->present, bytes, cudaMemcpyDeviceToHost, c->copy), "present copy");
    CK(c, cudaEventRecord(c->copied, c->copy), "present event");
    return OXPT_OK;
}

oxpt_status oxpt_resolve_wait(oxpt_ctx* c) {
    if (!c) return OXPT_E_INVALID;
    if (!c->copied) return OXPT_OK;
    oxpt_status s = set_device(c);
    if (s) return s;
    CK(c, cudaEventSynchronize(c->copied), "present wait");
    return OXPT_OK;
}

void* oxpt_host_alloc(size_t bytes) {
    void* p = nullptr;
    if (cudaMallocHost(&p, bytes ? bytes : 1) != cudaSuccess) {
        (void)cudaGetLastError();
        return nullptr;
    }
    return p;
}

void oxpt_host_free(void* p) {
    if (p) cudaFreeHost(p);
}

oxpt_status oxpt_read_accum(oxpt_ctx* c, float* out) {
    if (!c || !out) return fail(c, OXPT_E_INVALID, "null output");
    if (!c->accum) return fail(c, OXPT_E_INVALID, "no accumulator");
    oxpt_status s = set_device(c);
    if (s) return s;
    CK(c, cudaMemcpyAsync(out, c->accum, (size_t)c->w * c->h * 16, cudaMemcpyDeviceToHost, c->stream), "accum readback");
    CK(c, cudaStreamSynchronize(c->stream), "accum readback");
    return OXPT_OK;
}

oxpt_status oxpt_accum_view(oxpt_ctx* c, oxpt_devimage* out) {
    if (!c || !out) return fail(c, OXPT_E_INVALID, "null output");
    if (!c->accum) return fail(c, OXPT_E_INVALID, "no accumulator");
    out->data = c->accum;
    out->width = c->w;
    out->height = c->h;
    out->pitch_bytes = c->w * 16u;
    out->format = OXPT_FORMAT_RGBA32F;
    return OXPT_OK;
}

// ---------------------------------------------------------------------
// Diagnostics (oxpt_diag.h).
// ---------------------------------------------------------------------

oxpt_status oxpt_diag_sobol(oxpt_ctx* c, const uint32_t* dirs, uint32_t seed, size_t n, const uint32_t* x,
                            const uint32_t* y, const uint32_t* index, const uint32_t* pattern_id, uint32_t* out) {
    if (!c || !dirs || (n && (!x || !y || !index || !pattern_id || !out))) return fail(c, OXPT_E_INVALID, "null argument");
    if (n == 0) return OXPT_OK;
    oxpt_status s = set_device(c);
    if (s) return s;
    uint32_t* buf = nullptr;
    size_t words = 128 + n * 4 + n * 4;
    CK(c, cudaMalloc((void**)&buf, words * 4), "sobol buffers");
    uint32_t *dd = buf, *dx = buf + 128, *dy = dx + n, *di = dy + n, *dp = di + n, *dout = dp + n;
    cudaError_t e = cudaMemcpyAsync(dd, dirs, 512, cudaMemcpyHostToDevice, c->stream);
    if (!e) e = cudaMemcpyAsync(dx, x, n * 4, cudaMemcpyHostToDevice, c->stream);
    if (!e) e = cudaMemcpyAsync(dy, y, n * 4, cudaMemcpyHostToDevice, c->stream);
    if (!e) e = cudaMemcpyAsync(di, index, n * 4, cudaMemcpyHostToDevice, c->stream);
    if (!e) e = cudaMemcpyAsync(dp, pattern_id, n * 4, cudaMemcpyHostToDevice, c->stream);
    if (!e) e = oxd::launch_sobol(dd, seed, n, dx, dy, di, dp, dout, c->stream);
    if (!e) e = cudaMemcpyAsync(out, dout, n * 16, cudaMemcpyDeviceToHost, c->stream);
    if (!e) e = cudaStreamSynchronize(c->stream);
    cudaFree(buf);
    if (e) return cuda_fail(c, e, "sobol");
    return OXPT_OK;
}

oxpt_status oxpt_diag_trace_rays(oxpt_ctx* c, size_t n, const float* rays, uint32_t flags, uint32_t* slot,
                                 uint32_t* gid, float* t, float* bary) {
    if (!c || (n && !rays)) return fail(c, OXPT_E_INVALID, "null argument");
    if (oxpt_status sa = activate_staged(c)) return sa;
    if (!c->has_scene || !c->has_tables || !c->has_params) return fail(c, OXPT_E_INVALID, "scene, tables and params must be set first");
    if ((flags & 12u) && !bvh4_usable(c)) return fail(c, OXPT_E_INVALID, "no four-wide tree for this scene");
    if (n == 0) return OXPT_OK;
    oxpt_status s = set_device(c);
    if (s) return s;
    char* buf = nullptr;
    size_t bytes = n * (32 + 4 + 4 + 4 + 12);
    CK(c, cudaMalloc((void**)&buf, bytes), "ray buffers");
    float* dr = (float*)buf;
    uint32_t* ds = (uint32_t*)(buf + n * 32);
    uint32_t* dg = ds + n;
    float* dt = (float*)(dg + n);
    float* db = dt + n;
    oxd::RayArgs ra;
    ra.s = scene_view(c);
    ra.n = n;
    ra.rays = dr;
    ra.flags = flags;
    ra.slot = ds;
    ra.gid = dg;
    ra.t = dt;
    ra.bary = db;
    ra.counters = nullptr;
    ra.err = c->dev_err;
    cudaError_t e = cudaMemcpyAsync(dr, rays, n * 32, cudaMemcpyHostToDevice, c->stream);
    if (!e) e = oxd::launch_rays(ra, c->stream);
    if (!e && slot) e = cudaMemcpyAsync(slot, ds, n * 4, cudaMemcpyDeviceToHost, c->stream);
    if (!e && gid) e = cudaMemcpyAsync(gid, dg, n * 4, cudaMemcpyDeviceToHost, c->stream);
    if (!e && t) e = cudaMemcpyAsync(t, dt, n * 4, cudaMemcpyDeviceToHost, c->stream);
    if (!e && bary) e = cudaMemcpyAsync(bary, db, n * 12, cudaMemcpyDeviceToHost, c->stream);
    if (!e) e = cudaStreamSynchronize(c->stream);
    cudaFree(buf);
    if (e) return cuda_fail(c, e, "trace rays");
    return OXPT_OK;
}

oxpt_status oxpt_diag_math(oxpt_ctx* c, int op, size_t n, const float* a, const float* b, float* out) {
    if (!c || (n && (!a || !out))) return fail(c, OXPT_E_INVALID, "null argument");
    if (n == 0) return OXPT_OK;
    oxpt_status s = set_device(c);
    if (s) return s;
    float* buf = nullptr;
    CK(c, cudaMalloc((void**)&buf, n * 12), "math buffers");
    float *da = buf, *db = buf + n, *dout = buf + 2 * n;
    cudaError_t e = cudaMemcpyAsync(da, a, n * 4, cudaMemcpyHostToDevice, c->stream);
    if (!e && b) e = cudaMemcpyAsync(db, b, n * 4, cudaMemcpyHostToDevice, c->stream);
    if (!e) e = oxd::launch_math(op, n, da, b ? db : nullptr, dout, c->stream);
    if (!e) e = cudaMemcpyAsync(out, dout, n * 4, cudaMemcpyDeviceToHost, c->stream);
    if (!e) e = cudaStreamSynchronize(c->stream);
    cudaFree(buf);
    if (e) return cuda_fail(c, e, "math");
    return OXPT_OK;
}

oxpt_status oxpt_diag_refine_counted(oxpt_ctx* c, uint32_t first, uint32_t count, uint64_t out[8]) {
    if (!c || !out) return fail(c, OXPT_E_INVALID, "null argument");
    oxpt_status s = ready(c);
    if (s) return s;
    if ((s = set_device(c))) return s;
    CK(c, cudaMemsetAsync(c->dev_counters, 0, sizeof(unsigned long long) * 2 * oxd::C_N, c->stream), "counter clear");
    oxpt_frame f{first, count, 0, c->h};
    if ((s = run_frame(c, f, true))) return s;
    unsigned long long host[2 * oxd::C_N];
    CK(c, cudaMemcpyAsync(host, c->dev_counters, sizeof(host), cudaMemcpyDeviceToHost, c->stream), "counters");
    CK(c, cudaStreamSynchronize(c->stream), "counters");
    for (int k = 0; k < 2 * oxd::C_N; k++) c->split_counts[k] = host[k];
    for (int k = 0; k < 8; k++) out[k] = k < oxd::C_N ? host[k] + host[oxd::C_N + k] : 0;
    return oxpt_finish(c);
}

oxpt_status oxpt_diag_counters_split(const oxpt_ctx* c, uint64_t out[16]) {
    if (!c || !out) return OXPT_E_INVALID;
    for (int k = 0; k < 16; k++) out[k] = k < 2 * oxd::C_N ? c->split_counts[k] : 0;
    return OXPT_OK;
}

oxpt_status oxpt_diag_set_walk(oxpt_ctx* c, uint32_t stack_entries, uint32_t staged_nodes) {
    if (!c) return OXPT_E_INVALID;
    c->walk_lim = stack_entries;
    c->walk_stage = staged_nodes;
    return OXPT_OK;
}

oxpt_status oxpt_diag_set_ray_order(oxpt_ctx* c, int mode) {
    if (!c || mode < 0 || mode > 3) return fail(c, OXPT_E_INVALID, "ray order is 0 to 3");
    c->ray_order = (uint32_t)mode;
    return OXPT_OK;
}

oxpt_status oxpt_diag_set_l2_window(oxpt_ctx* c, int on, uint64_t* granted) {
    if (!c || on < 0 || on > 1) return fail(c, OXPT_E_INVALID, "l2 window is 0 or 1");
    oxpt_status s = set_device(c);
    if (s) return s;
    if (!on) {
        c->l2_setaside = 0;
        if (granted) *granted = 0;
        return OXPT_OK;
    }
    int maxp = 0, maxw = 0;
    CK(c, cudaDeviceGetAttribute(&maxp, cudaDevAttrMaxPersistingL2CacheSize, c->device), "l2 attribute");
    CK(c, cudaDeviceGetAttribute(&maxw, cudaDevAttrMaxAccessPolicyWindowSize, c->device), "l2 attribute");
    if (maxp <= 0 || maxw <= 0) return fail(c, OXPT_E_LIMIT, "the device has no persisting L2 set-aside");
    // A limit of this process's context (it ends with the process).
    size_t cur = 0;
    CK(c, cudaDeviceGetLimit(&cur, cudaLimitPersistingL2CacheSize), "l2 limit");
    if (cur < (size_t)maxp) CK(c, cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, (size_t)maxp), "l2 limit");
    CK(c, cudaDeviceGetLimit(&cur, cudaLimitPersistingL2CacheSize), "l2 limit");
    c->l2_setaside = cur;
    c->l2_max_window = (uint64_t)maxw;
    if (granted) *granted = cur;
    return OXPT_OK;
}

oxpt_status oxpt_diag_set_shadow_postpone(oxpt_ctx* c, int on) {
    if (!c) return OXPT_E_INVALID;
    c->shadow_post = on ? 1u : 0u;
    return OXPT_OK;
}

oxpt_status oxpt_diag_set_nee_mask(oxpt_ctx* c, int on) {
    if (!c) return OXPT_E_INVALID;
    c->nee_mask = on != 0;
    return OXPT_OK;
}

oxpt_status oxpt_diag_get_walk(const oxpt_ctx* c, uint32_t out[2]) {
    if (!c || !out) return OXPT_E_INVALID;
    out[0] = c->walk_lim;
    out[1] = c->walk_stage;
    return OXPT_OK;
}

oxpt_status oxpt_diag_set_launch(oxpt_ctx* c, uint32_t threads, uint32_t blocks_per_sm, uint64_t max_paths) {
    if (!c) return OXPT_E_INVALID;
    if (threads && (threads % 32 != 0 || threads > oxd::TRACE_THREADS))
        return fail(c, OXPT_E_INVALID, "threads must be a multiple of 32 and at most the kernel's block bound");
    c->threads = threads ? threads : oxd::TRACE_THREADS;
    c->blocks_per_sm = blocks_per_sm;
    c->max_paths = max_paths ? max_paths : (1ull << 22);
    c->wave_items = max_paths ? max_paths : oxd::DEFAULT_WAVE_ITEMS;
    return OXPT_OK;
}

oxpt_status oxpt_set_tuning(oxpt_ctx* c, const oxpt_tuning* t) {
    if (!c || !t) return OXPT_E_INVALID;
    if (t->mode > OXPT_MODE_WAVEFRONT_SPLIT) return fail(c, OXPT_E_INVALID, "unknown execution mode");
    if (t->threads && (t->threads % 32 != 0 || t->threads > oxd::TRACE_THREADS))
        return fail(c, OXPT_E_INVALID, "threads must be a multiple of 32 and at most the kernel's block bound");
    if (t->wave_slots > (1u << 26)) return fail(c, OXPT_E_LIMIT, "at most 2^26 wavefront slots");
    c->mode = t->mode;
    c->threads = t->threads ? t->threads : oxd::TRACE_THREADS;
    c->blocks_per_sm = t->blocks_per_sm;
    c->wave_slots = t->wave_slots ? t->wave_slots : (1u << 20);
    c->max_paths = t->max_paths ? t->max_paths : (1ull << 22);
    c->wave_items = t->wave_items ? t->wave_items : oxd::DEFAULT_WAVE_ITEMS;
    c->check_every = t->check_every ? t->check_every : 4u;
    if (t->shade_variant > 2 || t->trace_variant > 5 || t->nee_variant > 5)
        return fail(c, OXPT_E_INVALID, "shade variants are 0, 1 or 2; trace and NEE variants 0 to 5");
    if (t->stack && t->stack != 32 && t->stack != 64) return fail(c, OXPT_E_INVALID, "stack is 0, 32 or 64");
    if (t->stack == 32 && c->bvh_depth > 32) return fail(c, OXPT_E_INVALID, "the BVH is deeper than 32 levels");
    if (t->shadow_walk > 1) return fail(c, OXPT_E_INVALID, "shadow_walk is 0 or 1");
    if (t->graphs > 1) return fail(c, OXPT_E_INVALID, "graphs is 0 or 1");
    if (t->refill > 32) return fail(c, OXPT_E_INVALID, "refill is 0 (default) to 32");
    if (t->closest_walk > 1) return fail(c, OXPT_E_INVALID, "closest_walk is 0 or 1");
    if (t->closest_walk && t->trace_variant < 3)
        return fail(c, OXPT_E_INVALID, "closest_walk 1 needs the short-stack traversal kernels (trace_variant 3-5)");
    c->closest_walk = t->closest_walk;
    if (t->fast_shading > 1) return fail(c, OXPT_E_INVALID, "fast_shading is 0 or 1");
    if (t->fast_shading && t->mode != OXPT_MODE_WAVEFRONT_SPLIT)
        return fail(c, OXPT_E_INVALID, "fast_shading 1 needs the split wavefront (mode 2)");
    c->fast_shading = t->fast_shading;
    c->refill = t->refill ? t->refill : 8u;
    c->shadow_walk = t->shadow_walk;
    c->graphs = t->graphs;
    c->shade_variant = t->shade_variant;
    c->trace_variant = t->trace_variant;
    c->nee_variant = t->nee_variant;
    c->stack = t->stack;
    return OXPT_OK;
}

oxpt_status oxpt_get_tuning(const oxpt_ctx* c, oxpt_tuning* t) {
    if (!c || !t) return OXPT_E_INVALID;
    std::memset(t, 0, sizeof(*t));
    t->mode = c->mode;
    t->threads = c->threads;
    t->blocks_per_sm = c->blocks_per_sm;
    t->wave_slots = c->wave_slots;
    t->max_paths = c->max_paths;
    t->wave_items = c->wave_items;
    t->check_every = c->check_every;
    t->shade_variant = c->shade_variant;
    t->trace_variant = c->trace_variant;
    t->nee_variant = c->nee_variant;
    t->stack = c->stack;
    t->shadow_walk = c->shadow_walk;
    t->graphs = c->graphs;
    t->refill = c->refill;
    t->closest_walk = c->closest_walk;
    t->fast_shading = c->fast_shading;
    return OXPT_OK;
}

// Device-side tally of graph-resident loops: {kernels, iterations}.
static void read_tally(const oxpt_ctx* c, uint64_t out[2]) {
    out[0] = out[1] = 0;
    if (!c->dev_tally) return;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    unsigned long long v[2] = {0, 0};
    if (cudaMemcpy(v, c->dev_tally, 16, cudaMemcpyDeviceToHost) == cudaSuccess) {
        out[0] = v[0];
        out[1] = v[1];
    }
}

int oxpt_ctx_device(const oxpt_ctx* c) { return c ? c->device : -1; }

constexpr size_t MARK_RING = 64;

oxpt_status oxpt_mark(oxpt_ctx* c, uint64_t* mark) {
    if (!c || !mark) return OXPT_E_INVALID;
    oxpt_status s = set_device(c);
    if (s) return s;
    if (c->marks.empty()) {
        c->marks.resize(MARK_RING, nullptr);
        for (auto& ev : c->marks) CK(c, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "mark event");
    }
    uint64_t m = c->next_mark++;
    CK(c, cudaEventRecord(c->marks[m % MARK_RING], c->stream), "mark");
    *mark = m;
    return OXPT_OK;
}

oxpt_status oxpt_wait_mark(oxpt_ctx* c, uint64_t mark) {
    if (!c) return OXPT_E_INVALID;
    if (mark >= c->next_mark) return fail(c, OXPT_E_INVALID, "mark not recorded yet");
    oxpt_status s = set_device(c);
    if (s) return s;
    if (c->next_mark - mark > MARK_RING) {  // overwritten: everything up to the newest mark
        CK(c, cudaEventSynchronize(c->marks[(c->next_mark - 1) % MARK_RING]), "mark wait");
        return OXPT_OK;
    }
    CK(c, cudaEventSynchronize(c->marks[mark % MARK_RING]), "mark wait");
    return OXPT_OK;
}

oxpt_status oxpt_ctx_memory(const oxpt_ctx* c, uint64_t out[4]) {
    if (!c || !out) return OXPT_E_INVALID;
    uint64_t scene = 0;
    if (!c->borrowed_scene && c->has_scene) {
        scene = (uint64_t)c->geom_vec4 * 16 + (uint64_t)c->slot_count * 192 +
                (uint64_t)c->side * c->side * c->layers * 8 + (uint64_t)c->bvh4_nodes * 128;
    }
    scene += c->back.geom_cap + c->back.attrs_cap + c->back.atlas_cap + c->back.bvh4_cap;
    out[0] = scene;
    out[1] = (c->borrowed_tables ? 0 : (uint64_t)c->table_words * 4) + c->back.tables_cap;
    uint64_t px = (uint64_t)c->w * c->h;
    out[2] = c->accum ? px * 16 + (c->img8 ? px * 4 : 0) + (c->img32 ? px * 16 : 0) : 0;
    out[3] = c->out_cap * 16 + c->wave_bytes + c->batch_cap * sizeof(oxd::BatchFrame);
    return OXPT_OK;
}

oxpt_status oxpt_diag_graph_builds(const oxpt_ctx* c, uint64_t* out) {
    if (!c || !out) return OXPT_E_INVALID;
    *out = c->graph_builds;
    return OXPT_OK;
}

oxpt_status oxpt_diag_scene_build(const oxpt_ctx* c, float ms[8]) {
    if (!c || !ms) return OXPT_E_INVALID;
    for (int k = 0; k < 8; k++) ms[k] = c->build_ms[k];
    return OXPT_OK;
}

oxpt_status oxpt_diag_bvh4(const oxpt_ctx* c, uint32_t out[4]) {
    if (!c || !out) return OXPT_E_INVALID;
    out[0] = bvh4_usable(c) ? 1u : 0u;
    out[1] = c->bvh4_nodes;
    out[2] = c->bvh4_root;
    out[3] = c->bvh4_need;
    return OXPT_OK;
}

oxpt_status oxpt_diag_bvh4_build(const uint32_t* geom, uint32_t node_count, uint32_t* out, size_t cap, size_t* words,
                                 uint32_t* root, uint32_t* stack_need) {
    if ((node_count && !geom) || !words || !root || !stack_need) return OXPT_E_INVALID;
    std::vector<uint32_t> w;
    uint32_t r = 0xffffffffu;
    if (!oxpt::build_bvh4(geom, node_count, &w, &r)) return OXPT_E_INVALID;
    *words = w.size();
    *root = r;
    *stack_need = oxpt::bvh4_stack_need(w, r);
    if (out && cap >= w.size()) std::memcpy(out, w.data(), w.size() * 4);
    return OXPT_OK;
}

oxpt_status oxpt_diag_bvh4_build_device(int device, const uint32_t* geom, uint32_t node_count, uint32_t* out,
                                        size_t cap, size_t* words, uint32_t* root, uint32_t* stack_need,
                                        uint32_t* depth, uint32_t* host_depth) {
    if ((node_count && !geom) || !words || !root || !stack_need || !depth || !host_depth) return OXPT_E_INVALID;
    *host_depth = bvh_depth_of(geom, node_count);
    if (cudaSetDevice(device) != cudaSuccess) return OXPT_E_NODEV;
    cudaStream_t st = nullptr;
    uint32_t *d = nullptr, *o = nullptr;
    uint32_t n4 = 0, r = 0xffffffffu, need = 1;
    size_t ocap = 0;
    oxpt_status res = OXPT_OK;
    std::string e;
    oxd::Collapse c4 = oxd::Collapse::FAILED;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return OXPT_E_CUDA;
    if (cudaMalloc((void**)&d, std::max<size_t>((size_t)node_count * 32, 32)) != cudaSuccess ||
        cudaMemcpy(d, geom, (size_t)node_count * 32, cudaMemcpyHostToDevice) != cudaSuccess) {
        res = OXPT_E_CUDA;
        goto done;
    }
    if (!oxd::binary_depth_device(d, node_count, st, depth, &e)) {
        res = OXPT_E_CUDA;
        goto done;
    }
    c4 = oxd::collapse4_device(d, node_count, st, &o, &ocap, &n4, &r, &need, &e);
    if (c4 == oxd::Collapse::FAILED) res = OXPT_E_CUDA;
    else if (c4 == oxd::Collapse::REFUSED) res = OXPT_E_INVALID;
    else if (c4 == oxd::Collapse::UNSUPPORTED) res = OXPT_E_LIMIT;
    else {
        *words = (size_t)n4 * 32;
        *root = r;
        *stack_need = need;
        if (out && cap >= *words && n4 && cudaMemcpy(out, o, *words * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
            res = OXPT_E_CUDA;
    }
done:
    if (o) cudaFree(o);
    if (d) cudaFree(d);
    cudaStreamDestroy(st);
    return res;
}

oxpt_status oxpt_diag_wave_iterations(const oxpt_ctx* c, uint64_t* out) {
    if (!c || !out) return OXPT_E_INVALID;
    uint64_t t[2];
    read_tally(c, t);
    *out = c->wave_iterations + t[1];
    return OXPT_OK;
}

oxpt_status oxpt_diag_set_timing(oxpt_ctx* c, int enabled) {
    if (!c) return OXPT_E_INVALID;
    c->timing = enabled != 0;
    return OXPT_OK;
}

oxpt_status oxpt_diag_timing(oxpt_ctx* c, double* trace_ms, uint64_t* trace_n, double* reduce_ms, uint64_t* reduce_n) {
    if (!c) return OXPT_E_INVALID;
    oxpt_status s = set_device(c);
    if (s) return s;
    CK(c, cudaStreamSynchronize(c->stream), "timing sync");
    for (auto& t : c->timed) {
        float e = 0.0f;
        cudaEventElapsedTime(&e, t.a, t.b);
        c->kind_ms[t.kind] += e;
        c->kind_n[t.kind] += 1;
        cudaEventDestroy(t.a);
        cudaEventDestroy(t.b);
    }
    c->timed.clear();
    if (trace_ms) *trace_ms = c->kind_ms[0];
    if (trace_n) *trace_n = c->kind_n[0];
    if (reduce_ms) *reduce_ms = c->kind_ms[1];
    if (reduce_n) *reduce_n = c->kind_n[1];
    std::memcpy(c->last_ms, c->kind_ms, sizeof(c->last_ms));
    std::memcpy(c->last_n, c->kind_n, sizeof(c->last_n));
    for (int k = 0; k < 12; k++) {
        c->kind_ms[k] = 0.0;
        c->kind_n[k] = 0;
    }
    return OXPT_OK;
}

oxpt_status oxpt_diag_timing_kinds(const oxpt_ctx* c, double ms[12], uint64_t n[12]) {
    if (!c || !ms || !n) return OXPT_E_INVALID;
    for (int k = 0; k < 12; k++) {
        ms[k] = c->last_ms[k];
        n[k] = c->last_n[k];
    }
    return OXPT_OK;
}

oxpt_status oxpt_diag_launch_count(const oxpt_ctx* c, uint64_t* out) {
    if (!c || !out) return OXPT_E_INVALID;
    uint64_t t[2];
    read_tally(c, t);
    *out = c->launches + t[0];
    return OXPT_OK;
}

// ---------------------------------------------------------------------
// Batched refinement as one CUDA graph per refine step.
// ---------------------------------------------------------------------

}  // extern "C"

namespace {

// Key of a batch graph: everything baked into its nodes (plan, buffers,
// launch shapes, per-round sizes, reduce targets). Frame records (sample
// indices, scene views) live in device memory and are re-uploaded before
// every launch, so a refine step with the same shape reuses the graph.
template <class Reduces>
oxpt_status batch_graph_run(oxpt_ctx* e, const std::vector<oxd::WaveArgs>& args,
                            const std::vector<std::vector<oxpt::BatchPiece>>& rounds, int sd, bool four,
                            uint32_t max_bounces, size_t pieces, Reduces&& enqueue_reduces) {
    if (!e->dev_tally) {
        CK(e, cudaMalloc((void**)&e->dev_tally, 16), "graph tally");
        CK(e, cudaMemset(e->dev_tally, 0, 16), "graph tally");
    }
    if (!e->capture) CK(e, cudaStreamCreateWithFlags(&e->capture, cudaStreamNonBlocking), "capture stream");
    std::vector<uint64_t> key = {e->mode, e->fast_shading, e->shade_variant, e->trace_variant, e->nee_variant, (uint64_t)sd,
                                 four ? 1ull : 0ull, (uint64_t)e->sms, (uint64_t)(uintptr_t)e->wave_mem,
                                 (uint64_t)(uintptr_t)e->out, (uint64_t)(uintptr_t)e->dev_err,
                                 (uint64_t)(uintptr_t)e->stream, args.empty() ? 0 : args[0].vcap,
                                 args.empty() ? 0 : args[0].jobs};
    if (!args.empty()) {
        // Launch parameters the captured kernels keep: the staged scene's
        // node words (one-scene batches), the walk's storage split and tree.
        const oxd::WaveArgs& a0 = args[0];
        key.insert(key.end(), {(uint64_t)(uintptr_t)a0.s.geom, a0.s.geom_vec4, a0.s.P.env[3], a0.one_scene,
                               a0.closest4, a0.walk_lim, a0.walk_stage, (uint64_t)(uintptr_t)a0.st.vis,
                               a0.shadow_post, a0.ray_order, a0.l2_share, a0.l2_max_window});
    }
    for (size_t k = 0; k < rounds.size(); k++) {
        const oxd::WaveArgs& wa = args[k];
        key.insert(key.end(), {wa.slots, wa.total, (uint64_t)(uintptr_t)wa.frames, wa.nframes,
                               wave_cap(wa, max_bounces)});
        for (const oxpt::BatchPiece& pc : rounds[k]) {
            const oxpt_ctx* c = e->batch_ctx[pc.frame];
            key.insert(key.end(), {(uint64_t)(uintptr_t)c->accum, c->w, pc.base, pc.y0, pc.rows, pc.count});
        }
    }
    if ((key != e->bgraph_key || !e->bgraph) && e->bgraph_alt && key == e->bgraph_alt_key) {
        std::swap(e->bgraph, e->bgraph_alt);
        std::swap(e->bgraph_key, e->bgraph_alt_key);
    }
    if (key != e->bgraph_key || !e->bgraph) {
        if (e->bgraph_alt) cudaGraphExecDestroy(e->bgraph_alt);
        e->bgraph_alt = e->bgraph;
        e->bgraph_alt_key = std::move(e->bgraph_key);
        e->bgraph = nullptr;
        e->bgraph_key.clear();
        cudaGraph_t g = nullptr;
        cudaError_t ce = cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal);
        if (ce) return cuda_fail(e, ce, "graph capture");
        auto abort_capture = [&](cudaError_t why, const char* what) {
            cudaGraph_t dead = nullptr;
            cudaStreamEndCapture(e->stream, &dead);
            if (dead) cudaGraphDestroy(dead);
            return cuda_fail(e, why, what);
        };
        for (size_t k = 0; k < rounds.size(); k++) {
            const oxd::WaveArgs& wa = args[k];
            if ((ce = wave_init(wa, e->stream))) return abort_capture(ce, "graph wave init");
            cudaStreamCaptureStatus cs;
            cudaGraph_t cg = nullptr;
            const cudaGraphNode_t* deps = nullptr;
            size_t nd = 0;
            if ((ce = cudaStreamGetCaptureInfo(e->stream, &cs, nullptr, &cg, &deps, &nd)))
                return abort_capture(ce, "graph capture info");
            cudaGraphConditionalHandle h;
            if ((ce = cudaGraphConditionalHandleCreate(&h, cg, 1, cudaGraphCondAssignDefault)))
                return abort_capture(ce, "graph condition");
            cudaGraphNodeParams np{};
            np.type = cudaGraphNodeTypeConditional;
            np.conditional.handle = h;
            np.conditional.type = cudaGraphCondTypeWhile;
            np.conditional.size = 1;
            cudaGraphNode_t loop;
            if ((ce = cudaGraphAddNode(&loop, cg, deps, nd, &np))) return abort_capture(ce, "graph loop node");
            if ((ce = cudaStreamUpdateCaptureDependencies(e->stream, &loop, 1, cudaStreamSetCaptureDependencies)))
                return abort_capture(ce, "graph loop dependency");
            cudaGraph_t body = np.conditional.phGraph_out[0];
            if ((ce = cudaStreamBeginCaptureToGraph(e->capture, body, nullptr, nullptr, 0,
                                                    cudaStreamCaptureModeThreadLocal)))
                return abort_capture(ce, "graph body capture");
            cudaError_t ie = cudaSuccess;
            int kernels = enqueue_iteration(e, wa, wa, false, four, sd, sd, e->capture,
                                            [](int, auto&& launch) { return launch(); }, &ie);
            if (kernels >= 0) {
                uint64_t cap = std::min<uint64_t>(wave_cap(wa, max_bounces), 0xffffffffull);
                ie = oxd::launch_wave_continue(h, wa.ctr, (uint32_t)cap, e->dev_err, e->dev_tally,
                                               (uint32_t)kernels + 1u, e->capture);
            }
            cudaGraph_t body_out = nullptr;
            cudaError_t ee = cudaStreamEndCapture(e->capture, &body_out);
            if (ie) return abort_capture(ie, "graph body");
            if (ee) return abort_capture(ee, "graph body capture end");
            if ((ce = enqueue_reduces(k, e->stream))) return abort_capture(ce, "graph reduce");
        }
        if ((ce = cudaStreamEndCapture(e->stream, &g))) return cuda_fail(e, ce, "graph capture end");
        ce = cudaGraphInstantiate(&e->bgraph, g, 0);
        cudaGraphDestroy(g);
        if (ce) {
            e->bgraph = nullptr;
            return cuda_fail(e, ce, "graph instantiate");
        }
        e->bgraph_key = key;
        e->graph_builds++;
    }
    oxpt_ctx::Timed tt{nullptr, nullptr, 0};
    if (e->timing) {
        cudaEventCreate(&tt.a);
        cudaEventCreate(&tt.b);
        cudaEventRecord(tt.a, e->stream);
    }
    CK(e, cudaGraphLaunch(e->bgraph, e->stream), "graph launch");
    if (e->timing) {
        cudaEventRecord(tt.b, e->stream);
        e->timed.push_back(tt);
    }
    e->launches += pieces;  // reduces; the wavefront kernels are tallied on the device
    return OXPT_OK;
}

}  // namespace

extern "C" {

// ---------------------------------------------------------------------
// Batched refinement (oxpt_batch.h).
// ---------------------------------------------------------------------

oxpt_status oxpt_diag_batch_plan(const uint32_t* frames, uint32_t count, uint64_t cap, uint64_t* out,
                                 size_t capacity, size_t* pieces) {
    if ((count && !frames) || !pieces || cap == 0) return OXPT_E_INVALID;
    std::vector<oxpt::BatchInput> in(count);
    for (uint32_t k = 0; k < count; k++) {
        const uint32_t* f = frames + 5 * (size_t)k;
        if (f[0] > cap) return OXPT_E_INVALID;
        in[k] = {f[0], f[1], f[2], f[3], f[4]};
    }
    auto rounds = oxpt::plan_batch(in, cap);
    size_t n = 0;
    for (size_t r = 0; r < rounds.size(); r++)
        for (const oxpt::BatchPiece& pc : rounds[r]) {
            if (out && n < capacity) {
                uint64_t* o = out + 7 * n;
                o[0] = r;
                o[1] = pc.frame;
                o[2] = pc.first;
                o[3] = pc.count;
                o[4] = pc.y0;
                o[5] = pc.rows;
                o[6] = pc.base;
            }
            n++;
        }
    *pieces = n;
    return OXPT_OK;
}

oxpt_status oxpt_refine_batch(oxpt_ctx* e, const oxpt_batch_frame* fr, uint32_t n) {
    if (!e || (n && !fr)) return fail(e, OXPT_E_INVALID, "null argument");
    oxpt_status s = set_device(e);
    if (s) return s;
    // Validate every frame; the fixed tables must match the first frame's.
    std::vector<uint32_t> ref_tables, tab(640);
    std::vector<oxpt::BatchInput> in(n);
    for (uint32_t k = 0; k < n; k++) {
        oxpt_ctx* c = fr[k].ctx;
        std::string at = "batch frame " + std::to_string(k) + ": ";
        if (!c) return fail(e, OXPT_E_INVALID, at + "null context");
        in[k] = {c->w, fr[k].first, fr[k].count, fr[k].y0, fr[k].rows};
        if (fr[k].count == 0 || fr[k].rows == 0) continue;
        if (c->device != e->device) return fail(e, OXPT_E_INVALID, at + "context on another device");
        if (c != e && (c->staged || c->back_free_valid))
            return fail(e, OXPT_E_INVALID, at + "a context that stages scenes is traced by its own refine");
        if ((s = ready(c))) return fail(e, s, at + c->err);
        if (fr[k].y0 >= c->h || fr[k].rows > c->h - fr[k].y0) return fail(e, OXPT_E_INVALID, at + "rows outside the image");
        uint64_t o0 = c->params.offs0[0], o1 = c->params.offs0[1];
        if (o0 + 128 > c->table_words || o1 + 512 > c->table_words)
            return fail(e, OXPT_E_INVALID, at + "tables too short for the Sobol' and sheen words");
        if (c->stream != e->stream) {
            // The batch starts after the frame context's queued work (no host wait).
            if (!c->ready) CK(e, cudaEventCreateWithFlags(&c->ready, cudaEventDisableTiming), "frame event");
            CK(e, cudaEventRecord(c->ready, c->stream), "frame event");
            CK(e, cudaStreamWaitEvent(e->stream, c->ready, 0), "frame event");
        }
        if (n == 1) continue;  // a single frame stages its own tables
        if (o0 + 128 <= c->table_head.size() && o1 + 512 <= c->table_head.size()) {
            std::copy(c->table_head.begin() + o0, c->table_head.begin() + o0 + 128, tab.begin());
            std::copy(c->table_head.begin() + o1, c->table_head.begin() + o1 + 512, tab.begin() + 128);
        } else {
            CK(e, cudaStreamSynchronize(c->stream), "frame context sync");
            CK(e, cudaMemcpy(tab.data(), c->tables + o0, 128 * 4, cudaMemcpyDeviceToHost), "table check");
            CK(e, cudaMemcpy(tab.data() + 128, c->tables + o1, 512 * 4, cudaMemcpyDeviceToHost), "table check");
        }
        if (ref_tables.empty()) ref_tables = tab;
        else if (tab != ref_tables) return fail(e, OXPT_E_INVALID, at + "Sobol' or sheen table differs from the first frame's");
    }
    uint64_t cap = e->wave_items;
    for (uint32_t k = 0; k < n; k++)
        if (fr[k].count && fr[k].rows) cap = std::max<uint64_t>(cap, fr[k].ctx->w);
    e->batch_ctx.assign(n, nullptr);
    for (uint32_t k = 0; k < n; k++) e->batch_ctx[k] = fr[k].ctx;
    auto rounds = oxpt::plan_batch(in, cap);
    if (rounds.empty()) return OXPT_OK;
    // Frame records of every round, uploaded at once.
    std::vector<oxd::BatchFrame> recs;
    uint32_t J = 1, max_bounces = 0;
    int sd = e->stack == 64 ? 64 : 32;
    for (auto& r : rounds)
        for (const oxpt::BatchPiece& pc : r) {
            oxpt_ctx* c = fr[pc.frame].ctx;
            oxd::BatchFrame b{};
            b.s = scene_view(c);
            b.npix = c->w * pc.rows;
            b.base = pc.base;
            b.total = (uint64_t)b.npix * pc.count;
            b.first = pc.first;
            b.y0 = pc.y0;
            recs.push_back(b);
            J = std::max(J, c->params.cfg[2] + 1u);
            max_bounces = std::max(max_bounces, c->params.dims[3]);
            if (c->bvh_depth > 32) sd = 64;
            if ((e->shadow_walk == 0 || e->closest_walk) && bvh4_usable(c) && c->bvh4_need > 32) sd = 64;
        }
    // Records go through pinned staging: the host waits only until the
    // previous batch's records were copied, not for that batch to finish.
    if (e->batch_copied) CK(e, cudaEventSynchronize(e->batch_copied), "batch records staging");
    if (recs.size() > e->batch_cap) {
        if (e->batch_host) cudaFreeHost(e->batch_host);
        e->batch_host = nullptr;
        e->batch_cap = 0;
        if ((s = realloc_dev(e, &e->batch_dev, recs.size() * sizeof(oxd::BatchFrame), "batch frame records")))
            return s;
        CK(e, cudaMallocHost((void**)&e->batch_host, recs.size() * sizeof(oxd::BatchFrame)), "batch records staging");
        e->batch_cap = recs.size();
    }
    std::memcpy((void*)e->batch_host, (const void*)recs.data(), recs.size() * sizeof(oxd::BatchFrame));
    CK(e, cudaMemcpyAsync(e->batch_dev, e->batch_host, recs.size() * sizeof(oxd::BatchFrame), cudaMemcpyHostToDevice,
                          e->stream), "batch frame records");
    if (!e->batch_copied) CK(e, cudaEventCreateWithFlags(&e->batch_copied, cudaEventDisableTiming), "batch event");
    CK(e, cudaEventRecord(e->batch_copied, e->stream), "batch event");
    if ((s = ensure_out(e, cap))) return s;
    uint32_t saved_mode = e->mode;
    if (e->mode == OXPT_MODE_MEGAKERNEL) e->mode = OXPT_MODE_WAVEFRONT_SPLIT;
    // Path state for the largest round, allocated before any launch (and
    // before a graph capture, which allows no allocation).
    std::vector<oxd::WaveArgs> args;
    uint32_t pmax = 1;
    for (auto& r : rounds) {
        uint64_t total = 0;
        for (const oxpt::BatchPiece& pc : r) total += (uint64_t)fr[pc.frame].ctx->w * pc.rows * pc.count;
        pmax = std::max(pmax, (uint32_t)std::min<uint64_t>(total, e->wave_slots));
        oxd::WaveArgs wa{};
        wa.total = total;
        args.push_back(wa);
    }
    bool closest4 = e->closest_walk && e->trace_variant >= 3;
    for (uint32_t k = 0; k < n; k++)
        if (fr[k].count && fr[k].rows && !bvh4_usable(fr[k].ctx)) closest4 = false;
    oxd::WaveArgs base{};
    {
        // One scene for every frame (a single tracer's refine, or views of
        // one resident scene): the traversal kernels may stage its nodes.
        const oxpt_ctx* s0 = nullptr;
        bool one = true;
        for (uint32_t k = 0; k < n && one; k++) {
            const oxpt_ctx* c = fr[k].ctx;
            if (!fr[k].count || !fr[k].rows) continue;
            if (!s0) s0 = c;
            else one = c->geom == s0->geom && c->geom_vec4 == s0->geom_vec4 &&
                       c->params.env[3] == s0->params.env[3];
        }
        if (s0 && one) {
            base.s = scene_view(s0);
            base.one_scene = 1u;
        }
    }
    if ((s = ensure_wave(e, pmax, J, &base.st, &base.q, &base.ctr, &base.work))) {
        e->mode = saved_mode;
        return s;
    }
    size_t off = 0;
    for (size_t k = 0; k < rounds.size(); k++) {
        oxd::WaveArgs& wa = args[k];
        uint64_t total = wa.total;
        wa = base;
        wa.slots = (uint32_t)std::min<uint64_t>(total, e->wave_slots);
        wa.vcap = pmax;
        wa.jobs = J;
        wa.refill = e->refill;
        wa.walk_lim = e->walk_lim;
        wa.walk_stage = e->walk_stage;
        wa.shadow_post = e->shadow_post;
        wa.ray_order = e->ray_order;
        wa.l2_share = e->l2_setaside / 2;
        wa.l2_max_window = e->l2_max_window;
        wa.closest4 = closest4 ? 1u : 0u;
        wa.total = total;
        wa.out = e->out;
        wa.counters = nullptr;
        wa.err = e->dev_err;
        wa.frames = e->batch_dev + off;
        wa.nframes = (uint32_t)rounds[k].size();
        off += rounds[k].size();
    }
    bool four = e->shadow_walk == 0;
    for (uint32_t k = 0; k < n; k++)
        if (fr[k].count && fr[k].rows && !bvh4_usable(fr[k].ctx)) four = false;
    auto enqueue_reduces = [&](size_t k, cudaStream_t st) -> cudaError_t {
        for (const oxpt::BatchPiece& pc : rounds[k]) {
            oxpt_ctx* c = fr[pc.frame].ctx;
            oxd::ReduceArgs ra{c->accum, e->out + pc.base, c->w, pc.y0, c->w * pc.rows, pc.count};
            cudaError_t ce = oxd::launch_reduce(ra, st);
            if (ce != cudaSuccess) return ce;
        }
        return cudaSuccess;
    };
    size_t pieces = off;
    if (e->graphs) {
        s = batch_graph_run(e, args, rounds, sd, four, max_bounces, pieces, enqueue_reduces);
    } else {
        for (size_t k = 0; k < rounds.size() && !s; k++) {
            oxpt_ctx::Timed tt{nullptr, nullptr, 0};
            if (e->timing) {
                cudaEventCreate(&tt.a);
                cudaEventCreate(&tt.b);
                cudaEventRecord(tt.a, e->stream);
            }
            if ((s = wave_loop(e, args[k], false, four, sd, sd, max_bounces))) break;
            if (e->timing) {
                cudaEventRecord(tt.b, e->stream);
                e->timed.push_back(tt);
            }
            cudaError_t ce = enqueue_reduces(k, e->stream);
            if (ce != cudaSuccess) s = cuda_fail(e, ce, "batch reduce");
            e->launches += rounds[k].size();
        }
    }
    e->mode = saved_mode;
    if (s) return s;
    // Later work on the frame contexts' own streams waits for the batch.
    if (!e->batch_done) CK(e, cudaEventCreateWithFlags(&e->batch_done, cudaEventDisableTiming), "batch event");
    CK(e, cudaEventRecord(e->batch_done, e->stream), "batch event");
    for (uint32_t k = 0; k < n; k++) {
        oxpt_ctx* c = fr[k].ctx;
        if (c && c->stream != e->stream) CK(e, cudaStreamWaitEvent(c->stream, e->batch_done, 0), "batch event");
    }
    return OXPT_OK;
}

// ---------------------------------------------------------------------
// Radiance-cache frames (oxpt_nrc.h).
// ---------------------------------------------------------------------

void oxpt_nrc_config_default(oxpt_nrc_config* cfg) {
    if (!cfg) return;
    std::memset(cfg, 0, sizeof(*cfg));
    cfg->enabled = 1;
    cfg->query_bounce = 2;
    cfg->train_one_in = 16;
    cfg->max_train = 65536;
    cfg->train = 1;
    cfg->train_suffix = 4;
    cfg->spread = 0.01f;
    cfg->frames_per_wave = 1;
}

}  // extern "C"

namespace {

template <class T>
oxpt_status grow(oxpt_ctx* c, T** p, size_t* cap, size_t need, size_t elems_per, const char* what) {
    if (need <= *cap && *p) return OXPT_OK;
    if (*p) cudaFree(*p);
    *p = nullptr;
    *cap = 0;
    CK(c, cudaMalloc((void**)p, need * elems_per * sizeof(T)), what);
    *cap = need;
    return OXPT_OK;
}

oxpt_status nrc_buffers(oxpt_ctx* c, oxpt_nrc* r, size_t q, size_t t, size_t slots) {
    oxpt_status s;
    size_t dummy = 0;
    if (!r->counts && (s = grow(c, &r->counts, &dummy, 2, 1, "cache counters"))) return s;
    if (q > r->q_cap) {
        size_t c1 = 0, c2 = 0, c3 = 0, c4 = 0;
        if ((s = grow(c, &r->q_in, &c1, q, 3, "cache queries"))) return s;
        if ((s = grow(c, &r->q_beta, &c2, q, 1, "cache queries"))) return s;
        if ((s = grow(c, &r->q_item, &c3, q, 1, "cache queries"))) return s;
        if ((s = grow(c, &r->q_pred, &c4, q, 1, "cache queries"))) return s;
        r->q_cap = q;
    }
    if (t > r->t_cap) {
        size_t c1 = 0, c2 = 0, c3 = 0;
        if ((s = grow(c, &r->t_in, &c1, t, 3, "cache training samples"))) return s;
        if ((s = grow(c, &r->t_target, &c2, t, 1, "cache training samples"))) return s;
        if ((s = grow(c, &r->t_tail, &c3, t, 1, "cache training samples"))) return s;
        r->t_cap = t;
    }
    if (slots > r->s_cap) {
        size_t c1 = 0, c2 = 0, c3 = 0, c4 = 0, c5 = 0;
        if ((s = grow(c, &r->s_pre, &c1, slots, 1, "cache slot state"))) return s;
        if ((s = grow(c, &r->s_beta, &c2, slots, 1, "cache slot state"))) return s;
        if ((s = grow(c, &r->s_tidx, &c3, slots, 1, "cache slot state"))) return s;
        if ((s = grow(c, &r->s_spread, &c4, slots, 1, "cache slot state"))) return s;
        if ((s = grow(c, &r->s_tail, &c5, slots, 1, "cache slot state"))) return s;
        r->s_cap = slots;
    }
    return OXPT_OK;
}

}  // namespace

extern "C" {

}  // extern "C"

// Per-launch event pair of kind `kind` around `launch` when timing is on.
template <class F>
static cudaError_t timed_launch(oxpt_ctx* c, int kind, F&& launch) {
    oxpt_ctx::Timed t{nullptr, nullptr, kind};
    if (c->timing) {
        cudaEventCreate(&t.a);
        cudaEventCreate(&t.b);
        cudaEventRecord(t.a, c->stream);
    }
    cudaError_t e = launch();
    if (c->timing) {
        cudaEventRecord(t.b, c->stream);
        c->timed.push_back(t);
    }
    return e;
}

extern "C" {

oxpt_status oxpt_nrc_refine(oxpt_nrc* r, oxpt_ctx* c, uint32_t first, uint32_t count, const oxpt_nrc_config* cfg,
                            float* loss) {
    if (!r || !c || !cfg) return fail(c, OXPT_E_INVALID, "null argument");
    if (r->device != c->device) return fail(c, OXPT_E_INVALID, "the cache lives on another device");
    if (count == 0) return OXPT_OK;
    if (!cfg->enabled) {
        oxpt_frame f{first, count, 0, c->h};
        return oxpt_dispatch(c, &f);
    }
    if (cfg->train_one_in == 0 || (cfg->train_one_in & (cfg->train_one_in - 1)) != 0)
        return fail(c, OXPT_E_INVALID, "train_one_in must be a power of two");
    oxpt_status s = set_device(c);
    if (s) return s;
    if ((s = ready(c))) return s;
    const uint64_t npix = (uint64_t)c->w * c->h;
    if (npix > c->wave_items) return fail(c, OXPT_E_LIMIT, "a cache frame must fit one launch (width x height <= wave_items)");
    const uint32_t P = (uint32_t)npix;  // every path of a frame in flight at once
    const uint32_t max_train = std::max(cfg->max_train, 1u);
    // Frames traced as one wavefront: refill takes the next frame's paths
    // into the slots the previous frame's paths free, so a frame's tail of
    // nearly empty iterations overlaps the next frame's first bounces.
    const uint32_t G = std::max(cfg->frames_per_wave, 1u);
    if (G > 64) return fail(c, OXPT_E_INVALID, "frames_per_wave above 64");
    if (npix * G > c->wave_items) return fail(c, OXPT_E_LIMIT, "frames_per_wave x width x height exceeds wave_items");
    if (cfg->train_suffix > 64) return fail(c, OXPT_E_INVALID, "train_suffix above 64");
    if (!(cfg->spread >= 0.0f) || !std::isfinite(cfg->spread))
        return fail(c, OXPT_E_INVALID, "spread must be finite and not negative");
    if ((s = nrc_buffers(c, r, npix * G, max_train, P))) return s;
    if ((s = oxd::nrc::ensure_scratch(r, max_train))) return s;
    if ((s = ensure_out(c, npix * G))) return s;
    uint32_t saved_mode = c->mode, saved_slots = c->wave_slots;
    c->mode = OXPT_MODE_WAVEFRONT_SPLIT;
    c->wave_slots = P;  // the cache's per-slot state holds one frame's paths
    for (uint32_t i = 0; i < count && !s; i += G) {
        const uint32_t g = std::min(G, count - i);
        const uint64_t items = npix * g;
        cudaError_t ce = cudaMemsetAsync(r->counts, 0, 8, c->stream);
        if (ce) {
            s = cuda_fail(c, ce, "cache counters");
            break;
        }
        oxd::TraceArgs ta;
        ta.s = scene_view(c);
        ta.first = first + i;
        ta.count = g;
        ta.y0 = 0;
        ta.rows = c->h;
        ta.npix = (uint32_t)npix;
        ta.total = items;
        ta.out = c->out;
        ta.counters = nullptr;
        ta.err = c->dev_err;
        oxd::NrcWave nw{};
        nw.on = 1;
        nw.query_k = cfg->query_bounce;
        nw.train_mask = cfg->train_one_in - 1;
        nw.q_cap = (uint32_t)items;
        nw.t_cap = max_train;
        nw.counts = r->counts;
        nw.q_in = r->q_in;
        nw.q_beta = r->q_beta;
        nw.q_item = r->q_item;
        nw.t_in = r->t_in;
        nw.t_target = r->t_target;
        nw.s_pre = r->s_pre;
        nw.s_beta = r->s_beta;
        nw.s_tidx = r->s_tidx;
        nw.t_tail = r->t_tail;
        nw.suffix = cfg->train_suffix;
        nw.spread = cfg->spread;
        nw.s_spread = r->s_spread;
        nw.s_tail = r->s_tail;
        if ((s = run_wave(c, ta, false, &nw))) break;
        // The cache's predictions complete the rendering paths.
        oxd::nrc::Args a = oxd::nrc::base_args(r);
        a.in = r->q_in;
        a.n = (uint32_t)items;
        a.n_dev = r->counts;
        a.query_beta = r->q_beta;
        a.query_item = r->q_item;
        a.query_out = c->out;
        a.pred = r->q_pred;
        if ((ce = timed_launch(c, 7, [&] { return oxd::nrc::launch_forward(a, c->sms, c->stream); }))) {
            s = cuda_fail(c, ce, "cache inference");
            break;
        }
        oxd::ReduceArgs ra{c->accum, c->out, c->w, 0, (uint32_t)npix, g};
        if ((ce = oxd::launch_reduce(ra, c->stream))) {
            s = cuda_fail(c, ce, "reduce");
            break;
        }
        c->launches += 2;
        if (cfg->train) {
            ce = cudaMemsetAsync(r->grad, 0, oxd::nrc::PARAMS * 4, c->stream);
            if (!ce) ce = cudaMemsetAsync(r->loss, 0, 4, c->stream);
            oxd::nrc::Args b = oxd::nrc::base_args(r);
            b.in = r->t_in;
            b.n = max_train;
            b.n_dev = r->counts + 1;
            b.target = r->t_target;
            b.acts = r->acts;
            b.dy = r->dy;
            b.grad_scale = 0.0f;
            if (!ce && cfg->train_suffix)
                ce = oxd::nrc::launch_tail_targets(r->counts, max_train, (uint32_t)items, r->t_tail, r->q_pred,
                                                   r->t_target, c->stream);
            if (!ce) ce = timed_launch(c, 8, [&] { return oxd::nrc::launch_forward(b, c->sms, c->stream); });
            if (!ce) ce = timed_launch(c, 9, [&] { return oxd::nrc::launch_backward(b, c->sms, c->stream); });
            if (!ce) ce = oxd::nrc::adam_step(r, c->stream);
            if (ce) {
                s = cuda_fail(c, ce, "cache training");
                break;
            }
            c->launches += 3;
        }
    }
    c->mode = saved_mode;
    c->wave_slots = saved_slots;
    if (s) return s;
    if (loss) {
        float l = 0.0f;
        uint32_t n[2] = {0, 0};
        CK(c, cudaMemcpyAsync(&l, r->loss, 4, cudaMemcpyDeviceToHost, c->stream), "cache loss");
        CK(c, cudaMemcpyAsync(n, r->counts, 8, cudaMemcpyDeviceToHost, c->stream), "cache counters");
        CK(c, cudaStreamSynchronize(c->stream), "cache loss");
        uint32_t m = std::min(n[1], max_train);
        *loss = m ? l / (3.0f * (float)m) : 0.0f;
    }
    return OXPT_OK;
}

oxpt_status oxpt_nrc_frame_counts(oxpt_nrc* r, uint32_t* queries, uint32_t* samples) {
    if (!r || !r->counts) return OXPT_E_INVALID;
    uint32_t n[2] = {0, 0};
    if (cudaSetDevice(r->device) != cudaSuccess) return OXPT_E_CUDA;
    if (cudaDeviceSynchronize() != cudaSuccess || cudaMemcpy(n, r->counts, 8, cudaMemcpyDeviceToHost) != cudaSuccess)
        return OXPT_E_CUDA;
    if (queries) *queries = n[0];
    if (samples) *samples = n[1];
    return OXPT_OK;
}

}  // extern "C"
