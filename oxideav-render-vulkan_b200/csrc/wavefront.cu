// Wavefront path tracing for sm_100a (Laine, Karras & Aila 2013,
// "Megakernels considered harmful").
//
// The megakernel (trace.cu) interleaves traversal, texture filtering,
// the layered BSDF and light sampling in one divergent loop: its code does
// not fit the instruction cache and a warp's lanes sit at different stages.
// Here a path is a slot of SoA state in HBM and every bounce is three
// launches:
//   wave_logic   one thread per slot: adds the previous vertex's visible NEE
//                contributions in job order, processes the continuation
//                ray's hit (emission, material, BSDF), evaluates every NEE
//                job of the new vertex at once (their shadow rays go to a
//                queue), samples the BSDF and queues the next continuation
//                ray; finished slots take the next (pixel, sample) item from
//                a global counter (path regeneration);
//   wave_extend  closest-hit traversal of the queued continuation rays;
//   wave_shadow  any-hit traversal of the queued shadow rays.
// The traversal kernels hold nothing but the ray and the stack, so they run
// at high occupancy with coherent code. Each path's radiance receives the
// same contributions in the same order as in the megakernel (emission, the
// unoccluded NEE terms in job order, the next ray's findings), so results
// are bit-identical; finished paths land in the per-launch result buffer
// that reduce_frame adds to the accumulator in sample order.
#include <cooperative_groups.h>

#include "kernels.cuh"
#include "path.cuh"
#include "shade.cuh"
#include "traverse.cuh"
#include "wavefront.cuh"

namespace cg = cooperative_groups;

namespace oxd {

enum : uint32_t { ST_EMPTY = 0, ST_TRACING = 1, ST_ENDING = 2 };

__device__ __forceinline__ void load_core(const WaveArgs& a, uint32_t i, PathCore* pc, Sampler* smp, uint32_t* flags) {
    uint4 sd = a.st.seed[i];
    float4 b = a.st.beta[i], r = a.st.rad[i], d = a.st.dir[i], pp = a.st.prev[i], sg = a.st.sigma[i];
    smp->pixel_seed = sd.x;
    smp->index = sd.y;
    smp->path_seed = sd.z;
    pc->k = sd.w;
    pc->beta = xyz(b);
    pc->prev_pdf = b.w;
    pc->radiance = xyz(r);
    *flags = __float_as_uint(r.w);
    pc->in_medium = (*flags & 4u) != 0u;
    pc->d = xyz(d);
    pc->prev_pos = xyz(pp);
    pc->sigma = xyz(sg);
}

__device__ __forceinline__ void store_core(const WaveArgs& a, uint32_t i, const PathCore& pc, const Sampler& smp,
                                           uint32_t stage) {
    a.st.seed[i] = make_uint4(smp.pixel_seed, smp.index, smp.path_seed, pc.k);
    a.st.beta[i] = make_float4(pc.beta.x, pc.beta.y, pc.beta.z, pc.prev_pdf);
    uint32_t flags = stage | (pc.in_medium ? 4u : 0u);
    a.st.rad[i] = make_float4(pc.radiance.x, pc.radiance.y, pc.radiance.z, __uint_as_float(flags));
    a.st.dir[i] = make_float4(pc.d.x, pc.d.y, pc.d.z, 0.0f);
    a.st.prev[i] = make_float4(pc.prev_pos.x, pc.prev_pos.y, pc.prev_pos.z, 0.0f);
    a.st.sigma[i] = make_float4(pc.sigma.x, pc.sigma.y, pc.sigma.z, 0.0f);
}

__device__ __forceinline__ void set_stage(const WaveArgs& a, uint32_t i, uint32_t flags_other, uint32_t stage) {
    float4 r = a.st.rad[i];
    r.w = __uint_as_float(stage | flags_other);
    a.st.rad[i] = r;
}

// The frame of launch item `item` in a batched launch (frames ordered by
// base, none empty).
__device__ __forceinline__ uint32_t frame_of(const WaveArgs& a, unsigned long long item) {
    uint32_t lo = 0u, hi = a.nframes;
    while (hi - lo > 1u) {
        uint32_t mid = (lo + hi) >> 1;
        if (a.frames[mid].base <= item) lo = mid;
        else hi = mid;
    }
    return lo;
}

// The scene of slot i: the launch's own, or in a batched launch that of the
// frame the slot's path belongs to.
template <bool BATCH>
__device__ __forceinline__ const Scene& scene_of(const WaveArgs& a, uint32_t i) {
    return BATCH ? a.frames[a.st.frame[i]].s : a.s;
}

// Starts the path of launch item `item` in slot i (camera ray queued).
template <bool BATCH>
__device__ __forceinline__ void start_item(const WaveArgs& a, const uint32_t* s_sobol, uint32_t i,
                                           unsigned long long item, PathCore* pc, Sampler* smp) {
    uint32_t f = BATCH ? frame_of(a, item) : 0u;
    const Scene& s = BATCH ? a.frames[f].s : a.s;
    unsigned long long local = BATCH ? item - a.frames[f].base : item;
    uint32_t npix = BATCH ? a.frames[f].npix : a.npix;
    uint32_t y0 = BATCH ? a.frames[f].y0 : a.y0, first = BATCH ? a.frames[f].first : a.first;
    uint32_t it = (uint32_t)(local / npix);
    uint32_t q = (uint32_t)(local - (unsigned long long)it * npix);
    uint32_t yy = q / s.P.dims[0];
    f3 o = start_path(s, s_sobol, q - yy * s.P.dims[0], y0 + yy, first + it, smp, pc);
    a.st.item[i] = item;
    if (BATCH) a.st.frame[i] = f;
    store_core(a, i, *pc, *smp, ST_TRACING);
    a.st.org[i] = make_float4(o.x, o.y, o.z, 0.0f);
    a.q.ext[append(&a.ctr[0])] = i;
}

// The tables staged in shared memory (Sobol' direction numbers, sheen
// albedo) are the same words in every scene; a batched launch checks this
// on the host and stages the first frame's.
template <bool BATCH>
__device__ __forceinline__ const Scene& table_scene(const WaveArgs& a) {
    return BATCH ? a.frames[0].s : a.s;
}

template <bool COUNT, int MINB, bool BATCH>
__global__ void __launch_bounds__(128, MINB) wave_logic(const __grid_constant__ WaveArgs a) {
    __shared__ uint32_t s_sobol[128];
    __shared__ float s_sheen[512];
    {
        const Scene& s0 = table_scene<BATCH>(a);
        for (uint32_t i = threadIdx.x; i < 128u; i += blockDim.x) s_sobol[i] = tw(s0, s0.P.offs0[0] + i);
        for (uint32_t i = threadIdx.x; i < 512u; i += blockDim.x) s_sheen[i] = tf(s0, s0.P.offs0[1] + i);
    }
    __syncthreads();
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.slots) return;
    const uint32_t J = a.jobs;
    unsigned long long paths = 0, shaded = 0;

    PathCore pc;
    Sampler smp;
    uint32_t flags = __float_as_uint(a.st.rad[i].w);
    uint32_t stage = flags & 3u;
    bool need_new = stage == ST_EMPTY;
    if (!need_new) {
        const Scene& s = scene_of<BATCH>(a, i);
        const uint32_t Js = BATCH ? s.P.cfg[2] + 1u : J;  // this scene's NEE jobs
        load_core(a, i, &pc, &smp, &flags);
        // The previous vertex's NEE terms, in job order.
        uint32_t n = a.st.nee_n[i];
        for (uint32_t j = 0; j < n; j++) {
            float4 pe = a.st.pend[(uint64_t)i * J + j];
            if (pe.w == 2.0f) pc.radiance = pc.radiance + xyz(pe);
        }
        a.st.nee_n[i] = 0u;
        bool covered = true, finished = false;
        if (stage == ST_ENDING) {
            finished = true;
        } else {
            uint4 hb = a.st.hit[i];
            uint32_t hm = a.st.hmeta[i];
            Hit hit;
            hit.slot = hb.x;
            bool got = hb.x != NONE;
            uint32_t hmat = hm & 0x7fffffffu;
            hit.t = __uint_as_float(hb.y);
            float u = __uint_as_float(hb.z), v = __uint_as_float(hb.w);
            hit.b = mk(1.0f - u - v, u, v);
            hit.front = (hm >> 31) != 0u;
            Vertex vx;
            int outcome = on_path_hit<COUNT>(s, s_sheen, s_sobol, smp, pc, got, hit, hmat, &vx, &shaded);
            if (outcome != PATH_VERTEX) {
                finished = true;
                covered = outcome != PATH_UNCOVERED;
            } else {
                uint32_t armed = 0;
                for (uint32_t j = 0; j < Js; j++) {
                    ShadowRay sr;
                    float4 pe = make_float4(0.f, 0.f, 0.f, 0.f);
                    if (nee_job(s, s_sheen, pc, vx, j, &sr)) {
                        pe = make_float4(sr.pending.x, sr.pending.y, sr.pending.z, 1.0f);
                        uint32_t q = append(&a.ctr[1]);
                        a.q.sh_o[q] = make_float4(sr.o.x, sr.o.y, sr.o.z, sr.tmax);
                        a.q.sh_d[q] = make_float4(sr.d.x, sr.d.y, sr.d.z, __uint_as_float(sr.skip));
                        a.q.sh_m[q] = make_uint4(i, j, sr.rid, smp.path_seed);
                        armed = j + 1;
                    }
                    a.st.pend[(uint64_t)i * J + j] = pe;
                }
                a.st.nee_n[i] = armed;
                f3 o;
                if (continue_path(s, s_sheen, s_sobol, smp, pc, vx, &o)) {
                    store_core(a, i, pc, smp, ST_TRACING);
                    a.st.org[i] = make_float4(o.x, o.y, o.z, 0.0f);
                    a.q.ext[append(&a.ctr[0])] = i;
                } else if (armed) {
                    store_core(a, i, pc, smp, ST_ENDING);
                } else {
                    finished = true;
                }
            }
        }
        if (finished) {
            a.out[a.st.item[i]] = path_result(pc, covered);
            need_new = true;
        }
    }
    if (need_new) {
        unsigned long long item = fetch_item(a.work);
        if (item < a.total) {
            start_item<BATCH>(a, s_sobol, i, item, &pc, &smp);
            paths = 1;
        } else {
            if (stage != ST_EMPTY) set_stage(a, i, 0u, ST_EMPTY);
            stage = ST_EMPTY;
            if (COUNT) {
                if (shaded) atomicAdd(a.counters + C_SHADED, shaded);
            }
            return;
        }
    }
    append(&a.ctr[2]);  // one more slot still active
    if (COUNT) {
        if (paths) atomicAdd(a.counters + C_PATHS, paths);
        if (shaded) atomicAdd(a.counters + C_SHADED, shaded);
    }
}

// Traversal kernels: persistent grids over the ray queues, one walk per
// lane. A lane whose ray is finished takes the next queued ray (warp-
// aggregated fetch from a queue head) while the other lanes of its warp
// keep walking, once at least `a.refill` lanes of the warp are idle (1:
// at once; 32: only when the whole warp is idle), so warps are not held
// by their longest ray (Aila & Laine 2009, "Understanding the efficiency
// of ray traversal on GPUs": persistent threads, replacing terminated
// rays). The warp checks for idle lanes every STEPS walk steps. Each walk
// performs the same steps as a single-ray loop.
constexpr unsigned FULL_WARP = 0xffffffffu;
constexpr int STEPS = 4;

template <bool COUNT, int MINB, int SD, bool BATCH>
__global__ void __launch_bounds__(WAVE_TRAVERSE_THREADS, MINB) wave_extend(const __grid_constant__ WaveArgs a) {
    Cnt cnt;
    if (COUNT)
        for (int k = 0; k < C_N; k++) cnt.c[k] = 0;
    const uint32_t n = *((volatile uint32_t*)&a.ctr[0]);
    bool active = false, warp_drained = false;
    uint32_t i = 0u, k = 0u;
    const Scene* sc = &a.s;
    Ray r;
    Sampler smp{0u, 0u, 0u};
    Walk2<SD> w;
    for (;;) {
        const unsigned act = __ballot_sync(FULL_WARP, active);
        if (act == 0u && warp_drained) break;
        if (!warp_drained && 32 - __popc(act) >= (act ? a.refill : 1u)) {
            bool none_left = false;
            if (!active) {
                uint32_t q = append(&a.ctr[5]);
                if (q < n) {
                    i = a.q.ext[q];
                    sc = BATCH ? &a.frames[a.st.frame[i]].s : &a.s;
                    float4 o = a.st.org[i], d = a.st.dir[i];
                    uint4 sd = a.st.seed[i];
                    smp = Sampler{sd.x, sd.y, sd.z};
                    k = sd.w;
                    bump<COUNT>(cnt, C_PATH_RAYS);
                    r = make_ray(xyz(o), xyz(d));
                    if (walk2_begin<COUNT, SD>(*sc, r, INF, w, cnt)) active = true;
                    else a.st.hit[i] = make_uint4(NONE, 0u, 0u, 0u);
                } else {
                    none_left = true;
                }
            }
            warp_drained = __any_sync(FULL_WARP, none_left);
        }
#pragma unroll 1
        for (int st = 0; st < STEPS && active; st++) {
            if (walk2_step<COUNT, SD>(*sc, r, smp, k << 16u, k == 0u, false, NONE, w, cnt, a.err)) {
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

// FOUR: walk the four-wide tree (same occlusion as the binary walk); a
// batched launch uses it only when every frame's scene has one.
template <int SD, bool FOUR>
struct ShadowWalk {
    Walk2<SD> w;
};
template <int SD>
struct ShadowWalk<SD, true> {
    Walk4<SD> w;
};

template <bool COUNT, int MINB, int SD, bool FOUR, bool BATCH>
__global__ void __launch_bounds__(WAVE_TRAVERSE_THREADS, MINB) wave_shadow(const __grid_constant__ WaveArgs a) {
    Cnt cnt;
    if (COUNT)
        for (int k = 0; k < C_N; k++) cnt.c[k] = 0;
    const uint32_t n = *((volatile uint32_t*)&a.ctr[1]);
    bool active = false, warp_drained = false;
    uint32_t slot = 0u, job = 0u, rid = 0u, skip = NONE;
    const Scene* sc = &a.s;
    Ray r;
    Sampler smp{0u, 0u, 0u};
    ShadowWalk<SD, FOUR> sw;
    for (;;) {
        const unsigned act = __ballot_sync(FULL_WARP, active);
        if (act == 0u && warp_drained) break;
        if (!warp_drained && 32 - __popc(act) >= (act ? a.refill : 1u)) {
            bool none_left = false;
            if (!active) {
                uint32_t q = append(&a.ctr[6]);
                if (q < n) {
                    float4 o = a.q.sh_o[q], d = a.q.sh_d[q];
                    uint4 m = a.q.sh_m[q];
                    slot = m.x;
                    job = m.y;
                    rid = m.z;
                    skip = __float_as_uint(d.w);
                    smp = Sampler{0u, 0u, m.w};
                    sc = BATCH ? &a.frames[a.st.frame[slot]].s : &a.s;
                    bump<COUNT>(cnt, C_SHADOW_RAYS);
                    r = make_ray(xyz(o), xyz(d));
                    bool started;
                    if constexpr (FOUR) started = walk4_begin<SD>(*sc, r, o.w, sw.w);
                    else started = walk2_begin<COUNT, SD>(*sc, r, o.w, sw.w, cnt);
                    if (started) active = true;
                    else mark_visible(a.st, a.jobs, slot, job);  // nothing in the way
                } else {
                    none_left = true;
                }
            }
            warp_drained = __any_sync(FULL_WARP, none_left);
        }
#pragma unroll 1
        for (int st = 0; st < STEPS && active; st++) {
            bool done;
            if constexpr (FOUR) done = walk4_step<COUNT, SD>(*sc, r, smp, rid, false, skip, sw.w, cnt, a.err);
            else done = walk2_step<COUNT, SD>(*sc, r, smp, rid, false, true, skip, sw.w, cnt, a.err);
            if (done) {
                active = false;
                if (!sw.w.hit_any) mark_visible(a.st, a.jobs, slot, job);
            }
        }
    }
    if (COUNT)
        for (int c = 0; c < C_N; c++)
            if (cnt.c[c]) atomicAdd(a.counters + c, cnt.c[c]);
}

// Compiled variants: logic kernel occupancy targets 2 / 3 / 4 resident
// blocks per SM, traversal kernels 6 / 8 / 10 blocks with a 32- or 64-deep
// stack; batched launches have no counting build. The tuner picks one; all
// give the same results.
template <bool C, bool B>
static cudaError_t logic_v(const WaveArgs& a, int v, unsigned blocks, cudaStream_t st) {
    switch (v) {
        case 0: wave_logic<C, 2, B><<<blocks, 128, 0, st>>>(a); break;
        case 1: wave_logic<C, 3, B><<<blocks, 128, 0, st>>>(a); break;
        default: wave_logic<C, 4, B><<<blocks, 128, 0, st>>>(a); break;
    }
    return cudaGetLastError();
}

template <bool C, int SD, bool B>
static void* ext_fn(int v) {
    if (v == 0) return (void*)wave_extend<C, 6, SD, B>;
    if (v == 1) return (void*)wave_extend<C, 8, SD, B>;
    return (void*)wave_extend<C, 10, SD, B>;
}

template <bool C, int SD, bool FOUR, bool B>
static void* shadow_fn(int v) {
    if (v == 0) return (void*)wave_shadow<C, 6, SD, FOUR, B>;
    if (v == 1) return (void*)wave_shadow<C, 8, SD, FOUR, B>;
    return (void*)wave_shadow<C, 10, SD, FOUR, B>;
}

template <bool C, bool B>
static void* trav_kernel_c(bool ext, bool four, int v, int sd) {
    if (ext) return sd <= 32 ? ext_fn<C, 32, B>(v) : ext_fn<C, 64, B>(v);
    if (four) return sd <= 32 ? shadow_fn<C, 32, true, B>(v) : shadow_fn<C, 64, true, B>(v);
    return sd <= 32 ? shadow_fn<C, 32, false, B>(v) : shadow_fn<C, 64, false, B>(v);
}

static void* trav_kernel(bool count, bool batch, bool ext, bool four, int v, int sd) {
    if (batch) return count ? nullptr : trav_kernel_c<false, true>(ext, four, v, sd);
    return count ? trav_kernel_c<true, false>(ext, four, v, sd) : trav_kernel_c<false, false>(ext, four, v, sd);
}

cudaError_t launch_wave_logic(const WaveArgs& a, bool count, int variant, cudaStream_t st) {
    unsigned blocks = (a.slots + 127u) / 128u;
    variant = variant < 0 ? 0 : (variant > 2 ? 2 : variant);
    if (a.nframes) return count ? cudaErrorInvalidValue : logic_v<false, true>(a, variant, blocks, st);
    return count ? logic_v<true, false>(a, variant, blocks, st) : logic_v<false, false>(a, variant, blocks, st);
}

static cudaError_t launch_trav(const WaveArgs& a, bool count, bool ext, bool four, int variant, int sd, int sms,
                               cudaStream_t st) {
    variant = variant < 0 ? 0 : (variant > 2 ? 2 : variant);
    void* fn = trav_kernel(count, a.nframes > 0, ext, four, variant, sd);
    if (!fn) return cudaErrorInvalidValue;
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, WAVE_TRAVERSE_THREADS, 0);
    unsigned blocks = (unsigned)(sms * (per_sm > 0 ? per_sm : 1));
    WaveArgs copy = a;
    void* args[] = {&copy};
    return cudaLaunchKernel(fn, dim3(blocks), dim3(WAVE_TRAVERSE_THREADS), args, 0, st);
}

// ctr[10] counts the iterations of the current run (zeroed with the run's
// counters; the per-iteration queue reset clears ctr[0..7] only).
__global__ void wave_continue(cudaGraphConditionalHandle h, uint32_t* ctr, uint32_t cap, uint32_t* err,
                              unsigned long long* tally, uint32_t kernels) {
    uint32_t it = ctr[10] + 1u;
    ctr[10] = it;
    bool more = ctr[2] != 0u;
    if (more && it >= cap) {
        atomicOr(err, 8u);
        more = false;
    }
    tally[0] += kernels;
    tally[1] += 1ull;
    cudaGraphSetConditional(h, more ? 1u : 0u);
}

cudaError_t launch_wave_continue(cudaGraphConditionalHandle h, uint32_t* ctr, uint32_t cap, uint32_t* err,
                                 unsigned long long* tally, uint32_t kernels, cudaStream_t st) {
    wave_continue<<<1, 1, 0, st>>>(h, ctr, cap, err, tally, kernels);
    return cudaGetLastError();
}

cudaError_t launch_wave_extend(const WaveArgs& a, bool count, int variant, int stack, int sms, cudaStream_t st) {
    if (variant >= 3) return launch_walk(a, count, true, a.closest4 != 0u, variant - 3, stack, sms, st);
    return launch_trav(a, count, true, false, variant, stack, sms, st);
}

cudaError_t launch_wave_shadow(const WaveArgs& a, bool count, bool four, int variant, int stack, int sms,
                               cudaStream_t st) {
    if (variant >= 3) return launch_walk(a, count, false, four, variant - 3, stack, sms, st);
    return launch_trav(a, count, false, four, variant, stack, sms, st);
}

}  // namespace oxd
