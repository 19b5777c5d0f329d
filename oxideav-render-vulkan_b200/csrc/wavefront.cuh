// Wavefront path-state layout and launch entry points (see wavefront.cu).
#pragma once

#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "device.cuh"

namespace oxd {

// Warp-aggregated append: one atomic per converged group.
__device__ __forceinline__ uint32_t append(uint32_t* ctr) {
    namespace cg = cooperative_groups;
    cg::coalesced_group g = cg::coalesced_threads();
    uint32_t base = 0;
    if (g.thread_rank() == 0) base = atomicAdd(ctr, g.size());
    return g.shfl(base, 0) + g.thread_rank();
}
__device__ __forceinline__ unsigned long long fetch_item(unsigned long long* ctr) {
    namespace cg = cooperative_groups;
    cg::coalesced_group g = cg::coalesced_threads();
    unsigned long long base = 0;
    if (g.thread_rank() == 0) base = atomicAdd(ctr, (unsigned long long)g.size());
    return g.shfl(base, 0) + g.thread_rank();
}

constexpr uint32_t WAVE_TRAVERSE_THREADS = 128;

// Path slots, structure-of-arrays in HBM (16-byte records: one vector load
// per field, coalesced across consecutive slots).
struct WaveState {
    unsigned long long* item;  // work item of the slot
    uint4* seed;               // pixel seed, sample index, path seed, bounce k
    float4* beta;              // beta.xyz, previous BSDF pdf
    float4* rad;               // radiance.xyz, flags (stage | in_medium << 2)
    float4* dir;               // continuation direction
    float4* org;               // continuation origin
    float4* prev;              // previous vertex position
    float4* sigma;             // medium extinction
    uint4* hit;                // slot (0xffffffff = miss), t, u, v
    uint32_t* hmeta;           // material | front << 31
    uint32_t* nee_n;           // NEE jobs of the last vertex to add (0..J)
    float4* pend;              // slots x J: contribution.xyz, 0 none / 1 queued / 2 visible
    uint32_t* frame;           // batched launches: the slot's frame
    // split plan with at most 32 NEE jobs (else null): per slot, bit j set
    // when job j's shadow ray found nothing in the way; pend then holds
    // only the queued jobs' contributions and its w is not used
    uint32_t* vis;
};

// Job `job` of `slot` is unoccluded: its contribution is added.
__device__ __forceinline__ void mark_visible(const WaveState& st, uint32_t jobs, uint32_t slot, uint32_t job) {
    if (st.vis) atomicOr(st.vis + slot, 1u << job);
    else st.pend[(uint64_t)slot * jobs + job].w = 2.0f;
}

// One frame of a batched launch: a scene's samples [first, first + count)
// over npix pixels from row y0, as the launch's items [base, base + total).
// Every path keeps its pixel, sample index and scene, so its result is the
// one the frame's own launch gives.
struct BatchFrame {
    Scene s;
    unsigned long long base, total;
    uint32_t first, y0, npix, pad;
};

// Default paths per wavefront launch round: a 1920x1080 frame of 64 spp
// (133 M paths) in one round, so its regeneration tail comes once instead
// of once per round; the per-path result buffer holds one round (16 bytes a
// path, at most 2 GiB, less for smaller refines).
constexpr uint64_t DEFAULT_WAVE_ITEMS = 1ull << 27;

// Radiance-cache frame (split plan only; `on` = 0 otherwise): paths that
// are not training paths end with a cache query (features, throughput,
// result index) at their first vertex at or after bounce `query_k` whose
// path spread passes the heuristic (`spread` = 0: exactly at query_k);
// training paths (path seed & train_mask == 0) record, at that vertex, the
// inputs and, when they finish, the radiance they gathered from there on
// divided by their throughput there: the cache's target. A training path
// ends into the cache `suffix` bounces later (0: never): its target then
// adds the cache's prediction there (scaled by the throughput ratio),
// filled in after inference.
struct NrcWave {
    uint32_t on, query_k, train_mask, q_cap, t_cap, suffix;
    float spread;                  // path-spread constant (0: end exactly at query_k)
    uint32_t pad;
    uint32_t* counts;              // [0] queries, [1] training samples
    float4* q_in;                  // q_cap x 3 float4 inputs
    float4* q_beta;                // throughput at the query vertex
    unsigned long long* q_item;    // path result index
    float4* t_in;                  // t_cap x 3 float4 inputs
    float4* t_target;              // rgb target per training sample
    float4* s_pre;                 // per slot: radiance before the training vertex's reflected light
    float4* s_beta;                // per slot: throughput at the training vertex
    uint32_t* s_tidx;              // per slot: training sample index, or 0xffffffff
    uint4* t_tail;                 // per training sample: tail query, throughput ratio (float bits)
    float2* s_spread;              // per slot: primary spread a0, sum of sqrt(t^2 / (pdf |cos|))
    uint32_t* s_tail;              // per slot: bounce where a training path's suffix ends, or
                                   // 0xfffffffe after its training vertex without a suffix, or
                                   // 0xffffffff before it
};

struct WaveQueues {
    uint32_t* ext;  // slot ids with a continuation ray
    float4* sh_o;   // shadow ray origin, t_max
    float4* sh_d;   // shadow ray direction, skip id bits
    uint4* sh_m;    // slot, job, ray id, path seed
    // split wavefront (wave_split.cu)
    uint32_t* shade;  // slot ids with a surface hit to shade
    uint32_t* vslot;  // vertex record -> slot
    float4* vrec;     // vertex records, 13 float4 fields, field-major
    // continuation-ray reordering (ray_order.cu): the queue sorted, and per
    // entry its bucket and rank; bucket counts / offsets (2^15)
    uint32_t* ext_sorted;
    uint32_t* sh_perm;  // shadow queue order (sorted position -> entry)
    uint32_t* ord_key;
    uint32_t* ord_rank;
    uint32_t* ord_hist;
};

struct WaveArgs {
    Scene s;
    WaveState st;
    WaveQueues q;
    uint32_t slots, jobs, vcap;
    uint32_t first, y0, npix;
    unsigned long long total;   // items of this launch (npix x samples)
    unsigned long long* work;   // next item
    uint32_t* ctr;              // [0] continuation rays, [1] shadow rays, [2] active slots,
                                // [3] hits to shade, [4] vertex records, [5] / [6] next
                                // continuation / shadow ray to walk
    uint32_t refill;            // traversal: idle lanes of a warp that take new rays
    float4* out;
    unsigned long long* counters;
    uint32_t* err;
    // batched launches (null / 0 otherwise): frames ordered by base; `s`,
    // first, y0 and npix are then unused, `jobs` is the largest NEE job
    // count of the frames and out is indexed by launch item.
    const BatchFrame* frames;
    uint32_t nframes;
    NrcWave nrc;
    // traversal variants 3-5: walk-stack entries per lane kept in shared
    // memory (capped by the kernel's columns; deeper ones in local memory),
    // and top nodes of the binary tree a CTA stages in shared memory
    // (defaults measured on the 1.05 M-triangle scene: 2 entries and no
    // staged nodes; more on chip only took L1 from the node fetches)
    uint32_t walk_lim = 2u;
    uint32_t walk_stage = 0u;
    // batched launches whose frames all trace one scene (the same node
    // words): `s` is then that scene, for the traversal kernels' staged
    // top nodes
    uint32_t one_scene = 0u;
    // continuation rays walk the four-wide tree (traversal variants 3-5;
    // the tolerance plan: closest hits equal except near-ties)
    uint32_t closest4 = 0u;
    // four-wide shadow walks of variants 3-5 park leaves until the warp
    // has no node work (same occlusion, fewer mixed node/leaf steps)
    uint32_t shadow_post = 0u;
    // bit 0: the continuation queue is reordered by origin cell and
    // direction octant before the closest-hit walk; bit 1: the shadow queue
    // by light and origin cell, read through q.sh_perm by the short-stack
    // shadow walks (same results, other warps)
    uint32_t ray_order = 0u;
    // traversal variants 3-5 of one-scene launches: bytes of the L2's
    // persisting set-aside each walk may claim for the tree nodes it reads
    // (an access-policy window on its launch; 0: none), and the largest
    // window the device takes
    unsigned long long l2_share = 0ull, l2_max_window = 0ull;
};

// Reorders a.q.ext into a.q.ext_sorted / the shadow queue into
// a.q.sh_perm (ray_order.cu).
cudaError_t launch_order_ext(const WaveArgs& a, int sms, cudaStream_t st);
cudaError_t launch_order_shadow(const WaveArgs& a, int sms, cudaStream_t st);

// `variant`: 0..2, the occupancy target of the compiled kernel (logic 2 / 3
// / 4 blocks per SM; traversal 6 / 8 / 10); traversal variants 3..5 run the
// on-chip-stack kernels of wave_walk.cu (6 / 8 / 10 blocks per SM);
// `stack`: 32 or 64 entries.
// With a.nframes > 0 the batched kernels run (count must then be false).
cudaError_t launch_wave_logic(const WaveArgs& a, bool count, int variant, cudaStream_t st);
cudaError_t launch_wave_extend(const WaveArgs& a, bool count, int variant, int stack, int sms, cudaStream_t st);
// four: any-hit walk over the four-wide tree (Scene::bvh4) instead of the
// binary one; stack: 32 or 64 entries, enough for the tree walked.
cudaError_t launch_wave_shadow(const WaveArgs& a, bool count, bool four, int variant, int stack, int sms,
                               cudaStream_t st);
// wave_walk.cu: traversal with shared-memory short stacks and staged top
// nodes; ext = closest hit of the continuation queue, else the shadow queue
// (four: the four-wide tree); variant 0..2 targets 6 / 8 / 10 blocks per SM.
cudaError_t launch_walk(const WaveArgs& a, bool count, bool ext, bool four, int variant, int sd, int sms,
                        cudaStream_t st);
// Graph-resident loop: after an iteration, sets the enclosing while node's
// condition to "slots still active and fewer than `cap` iterations"; on
// reaching the bound it sets bit 3 of *err instead. tally[0] += kernels
// (the iteration's launches, this one included), tally[1] += 1.
cudaError_t launch_wave_continue(cudaGraphConditionalHandle h, uint32_t* ctr, uint32_t cap, uint32_t* err,
                                 unsigned long long* tally, uint32_t kernels, cudaStream_t st);
// Split wavefront (wave_split.cu); shade variants 2 / 3 / 4 blocks per SM,
// NEE variants 4 / 5 / 6.
cudaError_t launch_split_logic(const WaveArgs& a, bool count, cudaStream_t st);
cudaError_t launch_split_shade(const WaveArgs& a, bool count, int variant, int sms, cudaStream_t st);
cudaError_t launch_split_nee(const WaveArgs& a, bool count, int variant, int sms, cudaStream_t st);
// The same three kernels built a second time with FMA contraction,
// approximate division and square root and the CUDA library's
// transcendentals (wave_split.cu with OXPT_FAST): the shading of the
// tolerance plan, held to image PSNR against the oracle instead of bits.
namespace fast {
cudaError_t launch_split_logic(const WaveArgs& a, bool count, cudaStream_t st);
cudaError_t launch_split_shade(const WaveArgs& a, bool count, int variant, int sms, cudaStream_t st);
cudaError_t launch_split_nee(const WaveArgs& a, bool count, int variant, int sms, cudaStream_t st);
}  // namespace fast

}  // namespace oxd
