// Traversal kernels of the wavefront plans with on-chip walk storage
// (walk.cuh): short per-lane stacks in shared memory, the binary tree's top
// levels staged in shared memory, alpha tests out of line. Persistent grids
// over the ray queues with the lane refill of wave_extend / wave_shadow
// (wavefront.cu), and the same per-ray steps, so every result, counter and
// error bit equals theirs. Chosen by trace_variant 3-5 (occupancy targets
// of 6, 8 and 10 resident blocks per SM). How many stack entries per lane
// live in shared memory and how many top nodes a CTA stages are launch
// parameters (shared memory taken from L1: more on chip is not always
// faster), set per context (oxpt_diag_set_walk).
#include "kernels.cuh"
#include "walk.cuh"
#include "wavefront.cuh"

namespace oxd {

namespace {

constexpr uint32_t NT = WAVE_TRAVERSE_THREADS;
constexpr unsigned FULL = 0xffffffffu;
constexpr int STEPS = 4;        // walk steps between refill checks
// Most stack entries per lane a walk keeps in shared memory (the launch
// may keep fewer): binary walk (3 words an entry), four-wide any-hit walk
// (1 word), four-wide closest-hit walk (2 words).
constexpr int SS2 = 16;
constexpr int SS4 = 16;
constexpr int SS4C = 16;
constexpr uint32_t SM_SHARED = 228u * 1024u;  // shared memory per SM (sm_100)
constexpr uint32_t CTA_RESERVED = 1024u;      // per resident CTA, reserved by the runtime

// Shared-memory bytes of `lim` stack entries per lane.
__host__ __device__ constexpr uint32_t stack_bytes_of(uint32_t words_per_entry, uint32_t lim) {
    return words_per_entry * lim * NT * 4u;
}

extern __shared__ __align__(16) uint32_t walk_smem[];

// Copies the first `staged` float4 words of the scene's geom (top nodes)
// into shared memory after the stack columns.
__device__ __forceinline__ WalkShared stage_nodes(const Scene& s, uint32_t stack_bytes, uint32_t staged,
                                                  uint32_t lim) {
    WalkShared sh;
    sh.words = walk_smem;
    sh.lim = lim;
    float4* nodes = reinterpret_cast<float4*>(reinterpret_cast<char*>(walk_smem) + stack_bytes);
    for (uint32_t i = threadIdx.x; i < staged; i += NT) nodes[i] = geomv(s, i);
    __syncthreads();
    sh.nodes = nodes;
    sh.staged = staged;
    return sh;
}

template <bool COUNT, int MINB, int SD, bool BATCH>
__global__ void __launch_bounds__(NT, MINB) walk_extend(const __grid_constant__ WaveArgs a, uint32_t staged, uint32_t lim) {
    Cnt cnt;
    if (COUNT)
        for (int k = 0; k < C_N; k++) cnt.c[k] = 0;
    const WalkShared sh = stage_nodes(a.s, stack_bytes_of(3u, lim), staged, lim);
    const uint32_t n = *((volatile uint32_t*)&a.ctr[0]);
    bool active = false, warp_drained = false;
    uint32_t i = 0u, k = 0u, path_seed = 0u;
    const Scene* sc = &a.s;
    Ray r;
    Walk2S<SS2, SD> w;
    for (;;) {
        const unsigned act = __ballot_sync(FULL, active);
        if (act == 0u && warp_drained) break;
        if (!warp_drained && 32 - __popc(act) >= (act ? a.refill : 1u)) {
            bool none_left = false;
            if (!active) {
                uint32_t q = append(&a.ctr[5]);
                if (q < n) {
                    i = a.q.ext[q];
                    if (BATCH) sc = &a.frames[a.st.frame[i]].s;
                    float4 o = a.st.org[i], d = a.st.dir[i];
                    uint4 sd = a.st.seed[i];
                    path_seed = sd.z;
                    k = sd.w;
                    bump<COUNT>(cnt, C_PATH_RAYS);
                    r = make_ray(xyz(o), xyz(d));
                    if (walk2s_begin<COUNT, SS2, SD>(*sc, sh, r, INF, w, cnt)) active = true;
                    else a.st.hit[i] = make_uint4(NONE, 0u, 0u, 0u);
                } else {
                    none_left = true;
                }
            }
            warp_drained = __any_sync(FULL, none_left);
        }
#pragma unroll 1
        for (int st = 0; st < STEPS && active; st++) {
            if (walk2s_step<COUNT, SS2, SD, NT>(sc, sh, r, path_seed, k << 16u, k == 0u, false, NONE, w, cnt,
                                                a.err)) {
                active = false;
                if (w.hit_any) {
                    const Hit& h = w.best;
                    a.st.hit[i] = make_uint4(h.slot, __float_as_uint(h.t), __float_as_uint(h.b.y),
                                             __float_as_uint(h.b.z));
                    a.st.hmeta[i] = w.best_mat | (h.front ? 0x80000000u : 0u);
                } else {
                    a.st.hit[i] = make_uint4(NONE, 0u, 0u, 0u);
                }
            }
        }
    }
    if (COUNT)
        for (int c = 0; c < C_N; c++)
            if (cnt.c[c]) atomicAdd(a.counters + c, cnt.c[c]);
}

// Closest hits over the four-wide tree (the tolerance plan: the closest
// hit equals the binary walk's except near-ties, see walk4c_step).
template <bool COUNT, int MINB, int SD, bool BATCH>
__global__ void __launch_bounds__(NT, MINB) walk_extend4(const __grid_constant__ WaveArgs a, uint32_t lim) {
    Cnt cnt;
    if (COUNT)
        for (int k = 0; k < C_N; k++) cnt.c[k] = 0;
    const uint32_t n = *((volatile uint32_t*)&a.ctr[0]);
    bool active = false, warp_drained = false;
    uint32_t i = 0u, k = 0u, path_seed = 0u;
    const Scene* sc = &a.s;
    Ray r;
    Walk4C<SS4C, SD> w;
    for (;;) {
        const unsigned act = __ballot_sync(FULL, active);
        if (act == 0u && warp_drained) break;
        if (!warp_drained && 32 - __popc(act) >= (act ? a.refill : 1u)) {
            bool none_left = false;
            if (!active) {
                uint32_t q = append(&a.ctr[5]);
                if (q < n) {
                    i = a.q.ext[q];
                    if (BATCH) sc = &a.frames[a.st.frame[i]].s;
                    float4 o = a.st.org[i], d = a.st.dir[i];
                    uint4 sd = a.st.seed[i];
                    path_seed = sd.z;
                    k = sd.w;
                    bump<COUNT>(cnt, C_PATH_RAYS);
                    r = make_ray(xyz(o), xyz(d));
                    if (walk4c_begin<SS4C, SD>(*sc, r, INF, w)) active = true;
                    else a.st.hit[i] = make_uint4(NONE, 0u, 0u, 0u);
                } else {
                    none_left = true;
                }
            }
            warp_drained = __any_sync(FULL, none_left);
        }
#pragma unroll 1
        for (int st = 0; st < STEPS && active; st++) {
            if (walk4c_step<COUNT, SS4C, SD, NT>(sc, walk_smem, lim, r, path_seed, k << 16u, k == 0u, NONE, w, cnt,
                                                 a.err)) {
                active = false;
                if (w.hit_any) {
                    const Hit& h = w.best;
                    a.st.hit[i] = make_uint4(h.slot, __float_as_uint(h.t), __float_as_uint(h.b.y),
                                             __float_as_uint(h.b.z));
                    a.st.hmeta[i] = w.best_mat | (h.front ? 0x80000000u : 0u);
                } else {
                    a.st.hit[i] = make_uint4(NONE, 0u, 0u, 0u);
                }
            }
        }
    }
    if (COUNT)
        for (int c = 0; c < C_N; c++)
            if (cnt.c[c]) atomicAdd(a.counters + c, cnt.c[c]);
}

template <int SD, bool FOUR>
struct ShadowState {
    Walk2S<SS2, SD> w;
};
template <int SD>
struct ShadowState<SD, true> {
    Walk4S<SS4, SD> w;
};

template <bool COUNT, int MINB, int SD, bool FOUR, bool BATCH>
__global__ void __launch_bounds__(NT, MINB) walk_shadow(const __grid_constant__ WaveArgs a, uint32_t staged, uint32_t lim) {
    Cnt cnt;
    if (COUNT)
        for (int k = 0; k < C_N; k++) cnt.c[k] = 0;
    const WalkShared sh = stage_nodes(a.s, stack_bytes_of(FOUR ? 1u : 3u, lim), FOUR ? 0u : staged, lim);
    const uint32_t n = *((volatile uint32_t*)&a.ctr[1]);
    bool active = false, warp_drained = false;
    uint32_t slot = 0u, job = 0u, rid = 0u, skip = NONE, path_seed = 0u;
    const Scene* sc = &a.s;
    Ray r;
    ShadowState<SD, FOUR> ss;
    for (;;) {
        const unsigned act = __ballot_sync(FULL, active);
        if (act == 0u && warp_drained) break;
        if (!warp_drained && 32 - __popc(act) >= (act ? a.refill : 1u)) {
            bool none_left = false;
            if (!active) {
                uint32_t q = append(&a.ctr[6]);
                if (q < n) {
                    if (a.ray_order & 2u) q = a.q.sh_perm[q];
                    float4 o = a.q.sh_o[q], d = a.q.sh_d[q];
                    uint4 m = a.q.sh_m[q];
                    slot = m.x;
                    job = m.y;
                    rid = m.z;
                    path_seed = m.w;
                    skip = __float_as_uint(d.w);
                    if (BATCH) sc = &a.frames[a.st.frame[slot]].s;
                    bump<COUNT>(cnt, C_SHADOW_RAYS);
                    r = make_ray(xyz(o), xyz(d));
                    bool started;
                    if constexpr (FOUR) started = walk4s_begin<SS4, SD>(*sc, r, o.w, ss.w);
                    else started = walk2s_begin<COUNT, SS2, SD>(*sc, sh, r, o.w, ss.w, cnt);
                    if (started) active = true;
                    else mark_visible(a.st, a.jobs, slot, job);  // nothing in the way
                } else {
                    none_left = true;
                }
            }
            warp_drained = __any_sync(FULL, none_left);
        }
#pragma unroll 1
        for (int st = 0; st < STEPS && active; st++) {
            bool done;
            if constexpr (FOUR)
                done = walk4s_step<COUNT, SS4, SD, NT>(sc, walk_smem, sh.lim, r, path_seed, rid, false, skip,
                                                      ss.w, cnt, a.err);
            else
                done = walk2s_step<COUNT, SS2, SD, NT>(sc, sh, r, path_seed, rid, false, true, skip, ss.w, cnt,
                                                       a.err);
            if (done) {
                active = false;
                if (!ss.w.hit_any) mark_visible(a.st, a.jobs, slot, job);
            }
        }
    }
    if (COUNT)
        for (int c = 0; c < C_N; c++)
            if (cnt.c[c]) atomicAdd(a.counters + c, cnt.c[c]);
}

// Shadow rays over the four-wide tree with postponed leaves (walk4p_step):
// per step the warp takes node steps while any lane has node work, and a
// leaf step (every parked leaf tested) when none has.
template <bool COUNT, int MINB, int SD, bool BATCH>
__global__ void __launch_bounds__(NT, MINB) walk_shadow4p(const __grid_constant__ WaveArgs a, uint32_t staged,
                                                          uint32_t lim) {
    Cnt cnt;
    if (COUNT)
        for (int k = 0; k < C_N; k++) cnt.c[k] = 0;
    (void)staged;
    const uint32_t n = *((volatile uint32_t*)&a.ctr[1]);
    bool active = false, warp_drained = false;
    uint32_t slot = 0u, job = 0u, rid = 0u, skip = NONE, path_seed = 0u;
    const Scene* sc = &a.s;
    Ray r;
    Walk4P<SS4, SD> w;
    for (;;) {
        const unsigned act = __ballot_sync(FULL, active);
        if (act == 0u && warp_drained) break;
        if (!warp_drained && 32 - __popc(act) >= (act ? a.refill : 1u)) {
            bool none_left = false;
            if (!active) {
                uint32_t q = append(&a.ctr[6]);
                if (q < n) {
                    if (a.ray_order & 2u) q = a.q.sh_perm[q];
                    float4 o = a.q.sh_o[q], d = a.q.sh_d[q];
                    uint4 m = a.q.sh_m[q];
                    slot = m.x;
                    job = m.y;
                    rid = m.z;
                    path_seed = m.w;
                    skip = __float_as_uint(d.w);
                    if (BATCH) sc = &a.frames[a.st.frame[slot]].s;
                    bump<COUNT>(cnt, C_SHADOW_RAYS);
                    r = make_ray(xyz(o), xyz(d));
                    if (walk4p_begin<SS4, SD>(*sc, r, o.w, w)) active = true;
                    else mark_visible(a.st, a.jobs, slot, job);  // nothing in the way
                } else {
                    none_left = true;
                }
            }
            warp_drained = __any_sync(FULL, none_left);
        }
#pragma unroll 1
        for (int st = 0; st < STEPS; st++) {
            const bool leaf_step = __ballot_sync(FULL, active && walk4p_node_work(w)) == 0u;
            if (!active) continue;
            if (walk4p_step<COUNT, SS4, SD, NT>(sc, walk_smem, lim, r, path_seed, rid, false, skip, leaf_step, w, cnt,
                                                a.err)) {
                active = false;
                if (!w.hit_any) mark_visible(a.st, a.jobs, slot, job);
            }
        }
    }
    if (COUNT)
        for (int c = 0; c < C_N; c++)
            if (cnt.c[c]) atomicAdd(a.counters + c, cnt.c[c]);
}

template <bool C, int SD, bool B>
void* shadow4p_fn(int v) {
    if (v == 0) return (void*)walk_shadow4p<C, 6, SD, B>;
    if (v == 1) return (void*)walk_shadow4p<C, 8, SD, B>;
    return (void*)walk_shadow4p<C, 10, SD, B>;
}

template <bool C, int SD, bool B>
void* ext_fn(int v) {
    if (v == 0) return (void*)walk_extend<C, 6, SD, B>;
    if (v == 1) return (void*)walk_extend<C, 8, SD, B>;
    return (void*)walk_extend<C, 10, SD, B>;
}

template <bool C, int SD, bool B>
void* ext4_fn(int v) {
    if (v == 0) return (void*)walk_extend4<C, 6, SD, B>;
    if (v == 1) return (void*)walk_extend4<C, 8, SD, B>;
    return (void*)walk_extend4<C, 10, SD, B>;
}

template <bool C, int SD, bool FOUR, bool B>
void* shadow_fn(int v) {
    if (v == 0) return (void*)walk_shadow<C, 6, SD, FOUR, B>;
    if (v == 1) return (void*)walk_shadow<C, 8, SD, FOUR, B>;
    return (void*)walk_shadow<C, 10, SD, FOUR, B>;
}

template <bool C, bool B>
void* kernel_c(bool ext, bool four, bool post, int v, int sd) {
    if (ext && four) return sd <= 32 ? ext4_fn<C, 32, B>(v) : ext4_fn<C, 64, B>(v);
    if (four && post) return sd <= 32 ? shadow4p_fn<C, 32, B>(v) : shadow4p_fn<C, 64, B>(v);
    if (ext) return sd <= 32 ? ext_fn<C, 32, B>(v) : ext_fn<C, 64, B>(v);
    if (four) return sd <= 32 ? shadow_fn<C, 32, true, B>(v) : shadow_fn<C, 64, true, B>(v);
    return sd <= 32 ? shadow_fn<C, 32, false, B>(v) : shadow_fn<C, 64, false, B>(v);
}

void* kernel_of(bool count, bool batch, bool ext, bool four, bool post, int v, int sd) {
    if (batch) return count ? nullptr : kernel_c<false, true>(ext, four, post, v, sd);
    return count ? kernel_c<true, false>(ext, four, post, v, sd) : kernel_c<false, false>(ext, four, post, v, sd);
}

const int TARGET_BLOCKS[3] = {6, 8, 10};

}  // namespace

// ext && four: closest hits over the four-wide tree (walk_extend4);
// !ext && four && a.shadow_post: shadow rays with postponed leaves.
// variant 0..2: 6 / 8 / 10 resident blocks per SM targeted. a.walk_lim
// stack entries per lane (at most the walk's SS) live in shared memory;
// binary walks of launches over one scene (a plain launch, or a batch
// whose frames all trace the same node words) also stage up to
// a.walk_stage top nodes, within what the targeted number of blocks leaves
// each block.
cudaError_t launch_walk(const WaveArgs& a, bool count, bool ext, bool four, int variant, int sd, int sms,
                        cudaStream_t st) {
    variant = variant < 0 ? 0 : (variant > 2 ? 2 : variant);
    void* fn = kernel_of(count, a.nframes > 0, ext, four, a.shadow_post != 0u, variant, sd);
    if (!fn) return cudaErrorInvalidValue;
    const uint32_t target = (uint32_t)TARGET_BLOCKS[variant];
    const uint32_t words = four ? (ext ? 2u : 1u) : 3u;
    const uint32_t cap = four ? (ext ? (uint32_t)SS4C : (uint32_t)SS4) : (uint32_t)SS2;
    uint32_t lim = a.walk_lim < cap ? a.walk_lim : cap;
    const uint32_t stack_bytes = stack_bytes_of(words, lim);
    uint32_t per_block = SM_SHARED / target - CTA_RESERVED;
    if (per_block > 48u * 1024u) per_block = 48u * 1024u;
    uint32_t staged = 0u;  // float4 words of staged top nodes (binary walks)
    if (!four && (a.nframes == 0 || a.one_scene) && per_block > stack_bytes) {
        uint64_t nodes = (per_block - stack_bytes) / 32u;
        if (nodes > a.walk_stage) nodes = a.walk_stage;
        if (nodes > a.s.P.env[3]) nodes = a.s.P.env[3];
        if (2 * nodes > a.s.geom_vec4) nodes = a.s.geom_vec4 / 2;
        staged = (uint32_t)(2 * nodes);
    }
    const uint32_t smem = stack_bytes + staged * 16u;
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, NT, smem);
    if (e != cudaSuccess) return e;
    unsigned blocks = (unsigned)(sms * (per_sm > 0 ? per_sm : 1));
    WaveArgs copy = a;
    void* args3[] = {&copy, &staged, &lim};
    void* args2[] = {&copy, &lim};
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(blocks);
    cfg.blockDim = dim3(NT);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    // The tree nodes this walk reads as persisting L2 lines, so that the
    // wavefront state and attributes streaming through L2 between walks do
    // not evict them (a hint: results do not depend on it).
    cudaLaunchAttribute attr[1];
    const float4* base = four ? a.s.bvh4 : a.s.geom;
    const uint64_t bytes = four ? (uint64_t)a.s.bvh4_nodes * 128u : (uint64_t)a.s.P.env[3] * 32u;
    if (a.l2_share && a.l2_max_window && base && bytes && (a.nframes == 0 || a.one_scene)) {
        const uint64_t win = bytes < a.l2_max_window ? bytes : a.l2_max_window;
        const double ratio = (double)a.l2_share / (double)win;
        attr[0].id = cudaLaunchAttributeAccessPolicyWindow;
        attr[0].val.accessPolicyWindow.base_ptr = (void*)base;
        attr[0].val.accessPolicyWindow.num_bytes = (size_t)win;
        attr[0].val.accessPolicyWindow.hitRatio = ratio < 1.0 ? (float)ratio : 1.0f;
        attr[0].val.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
        attr[0].val.accessPolicyWindow.missProp = cudaAccessPropertyNormal;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
    }
    return cudaLaunchKernelExC(&cfg, fn, (ext && four) ? args2 : args3);
}

}  // namespace oxd
