// Short-stack BVH walkers for the wavefront traversal kernels (wave_walk.cu).
//
// The same walks as traverse.cuh — the reference's ordered binary walk
// (pathtrace.wgsl:646-735: near child first, the far child pushed with its
// entry distance, pops culled against t_max, a 64-entry stack that drops
// the far child on overflow) and the exact four-wide any-hit walk — with
// the storage moved on chip:
//
// * Walk stacks: the first `lim` entries (at most SS) of each lane's stack
//   live in shared memory as columns (entry k of lane j at word k * NT + j,
//   one block of lim * NT words per field), so the 32 lanes of a warp push
//   and pop with one conflict-free shared-memory access; deeper entries go
//   to local memory. Near-first walks of the
//   scenes here rarely go deeper than a handful of entries, so the per-
//   thread local stack (512-768 bytes per lane, more than L1 holds at
//   traversal occupancy) is no longer touched on the common path.
// * Top of the binary tree: nodes are numbered level by level, so nodes
//   [0, K) are the tree's top levels; a CTA copies them into shared memory
//   once and fetches child pairs below K from there.
// * Alpha-tested acceptance (MASK / BLEND materials sample the base-colour
//   texture) is an out-of-line call, so the texture code does not reserve
//   registers for the whole walk loop; opaque materials never make it.
//
// Every step performs the operations of the corresponding traverse.cuh
// step in the same order, so hits, counters and error bits are identical.
#pragma once

#include "kernels.cuh"
#include "shade.cuh"
#include "traverse.cuh"

namespace oxd {

// Alpha acceptance of a MASK (mode 1) or BLEND (mode 2, 3) hit
// (pathtrace.wgsl:621-636), out of line.
static __device__ __noinline__ bool alpha_accept(const Scene* s, uint32_t slot, uint32_t m, uint32_t gid, float b0,
                                                 float b1, float b2, uint32_t path_seed, uint32_t ray_id,
                                                 uint32_t mode) {
    f3 b = mk(b0, b1, b2);
    if (mode == 1u) return hit_alpha(*s, slot, m, b) >= tf(*s, mat_off(*s, m) + 11u);
    Sampler smp{0u, 0u, path_seed};
    return coin(smp, ray_id, gid) < hit_alpha(*s, slot, m, b);
}

// accept() of traverse.cuh with the alpha test out of line.
__device__ __forceinline__ bool accept_ol(const Scene* s, uint32_t slot, uint32_t m, uint32_t gid, const Hit& h,
                                          uint32_t path_seed, uint32_t ray_id, bool primary) {
    uint32_t fl = mat_flags(*s, m);
    if (primary && !h.front && (fl & 4u) == 0u) return false;
    uint32_t mode = fl & 3u;
    if (mode == 0u) return true;
    return alpha_accept(s, slot, m, gid, h.b.x, h.b.y, h.b.z, path_seed, ray_id, mode);
}

// Shared-memory view of a CTA's walk storage. `nodes` holds the first
// `staged` float4 words of the scene's geom (whole nodes, top levels);
// stack entries below `lim` (at most the columns' SS) use the columns.
struct WalkShared {
    uint32_t* words;       // stack columns
    const float4* nodes;   // staged top nodes (2 float4 per node)
    uint32_t staged;       // float4 words staged (2 x nodes staged)
    uint32_t lim;          // stack entries kept in shared memory
};

__device__ __forceinline__ float4 node_vec(const Scene& s, const WalkShared& sh, uint64_t i) {
    return i < sh.staged ? sh.nodes[i] : geomv(s, i);
}

// ---------------------------------------------------------------------
// Ordered binary walk with a short shared stack: entries (first, count, t)
// in three column blocks of sh.lim x NT words; entries from sh.lim on in
// local memory. SD is the full depth (64 as the reference, or 32 when the tree
// has at most 32 levels).
// ---------------------------------------------------------------------
template <int SS, int SD>
struct Walk2S {
    float t_max;
    uint32_t cur_first, cur_count, sp, guard;
    bool hit_any;
    uint32_t best_mat;
    Hit best;
    uint2 deep_fc[SD];
    float deep_t[SD];
};

template <bool COUNT, int SS, int SD>
__device__ __forceinline__ bool walk2s_begin(const Scene& s, const WalkShared& sh, const Ray& r, float t_max,
                                             Walk2S<SS, SD>& w, Cnt& cnt) {
    w.best.slot = NONE;
    w.hit_any = false;
    w.best_mat = 0u;
    uint32_t node_count = s.P.env[3];
    if (node_count == 0u || !r.valid) return false;
    float4 rlo = node_vec(s, sh, 0), rhi = node_vec(s, sh, 1);
    bump<COUNT>(cnt, C_BOXES);
    if (slab(r, rlo, rhi, t_max) < 0.0f) return false;
    w.t_max = t_max;
    w.cur_first = __float_as_uint(rlo.w);
    w.cur_count = __float_as_uint(rhi.w);
    w.sp = 0u;
    w.guard = node_count + 8u;
    return true;
}

template <bool COUNT, int SS, int SD, int NT>
__device__ __forceinline__ bool walk2s_step(const Scene* sp_, const WalkShared& sh, const Ray& r, uint32_t path_seed,
                                            uint32_t ray_id, bool primary, bool any, uint32_t skip,
                                            Walk2S<SS, SD>& w, Cnt& cnt, uint32_t* err) {
    const Scene& s = *sp_;
    const uint32_t lane = threadIdx.x;
    uint32_t* col_f = sh.words;
    uint32_t* col_c = sh.words + sh.lim * NT;
    float* col_t = reinterpret_cast<float*>(sh.words + 2 * sh.lim * NT);
    if (w.guard-- == 0u) {
        atomicOr(err, 1u);
        w.best.slot = NONE;
        w.hit_any = false;
        return true;
    }
    if (w.cur_count > 0u) {
        bump<COUNT>(cnt, C_LEAVES);
        if ((uint64_t)w.cur_first + w.cur_count > s.slot_count) {
            atomicOr(err, 2u);
            w.best.slot = NONE;
            w.hit_any = false;
            return true;
        }
        uint32_t end = w.cur_first + w.cur_count;
        for (uint32_t slot = w.cur_first; slot < end; slot++) {
            bump<COUNT>(cnt, C_TRIS);
            uint64_t tb = tri_base(s, slot);
            float4 q0 = geomv(s, tb), q1 = geomv(s, tb + 1), q2 = geomv(s, tb + 2);
            Hit h;
            if (!intersect(r, q0, q1, q2, w.t_max, &h)) continue;
            uint32_t gid = __float_as_uint(q0.w);
            if (gid == skip) continue;
            uint32_t m = __float_as_uint(q2.w);
            if (!accept_ol(sp_, slot, m, gid, h, path_seed, ray_id, primary)) continue;
            h.slot = slot;
            w.best = h;
            w.best_mat = m;
            w.hit_any = true;
            if (any) return true;
            w.t_max = h.t;
        }
    } else {
        bump<COUNT>(cnt, C_BOXES, 2);
        uint64_t l = w.cur_first;
        float4 alo = node_vec(s, sh, 2 * l), ahi = node_vec(s, sh, 2 * l + 1);
        float4 blo = node_vec(s, sh, 2 * l + 2), bhi = node_vec(s, sh, 2 * l + 3);
        float tl = slab(r, alo, ahi, w.t_max);
        float tr = slab(r, blo, bhi, w.t_max);
        if (tl >= 0.0f && tr >= 0.0f) {
            bool swap = tl > tr;
            uint32_t nf = swap ? __float_as_uint(blo.w) : __float_as_uint(alo.w);
            uint32_t nc = swap ? __float_as_uint(bhi.w) : __float_as_uint(ahi.w);
            uint32_t ff = swap ? __float_as_uint(alo.w) : __float_as_uint(blo.w);
            uint32_t fc = swap ? __float_as_uint(ahi.w) : __float_as_uint(bhi.w);
            float ft = swap ? tl : tr;
            if (w.sp < (uint32_t)SD) {
                if (w.sp < sh.lim) {
                    col_f[w.sp * NT + lane] = ff;
                    col_c[w.sp * NT + lane] = fc;
                    col_t[w.sp * NT + lane] = ft;
                } else {
                    w.deep_fc[w.sp] = make_uint2(ff, fc);
                    w.deep_t[w.sp] = ft;
                }
                w.sp++;
            }
            w.cur_first = nf;
            w.cur_count = nc;
            return false;
        } else if (tl >= 0.0f) {
            w.cur_first = __float_as_uint(alo.w);
            w.cur_count = __float_as_uint(ahi.w);
            return false;
        } else if (tr >= 0.0f) {
            w.cur_first = __float_as_uint(blo.w);
            w.cur_count = __float_as_uint(bhi.w);
            return false;
        }
    }
    while (w.sp != 0u) {
        w.sp--;
        bump<COUNT>(cnt, C_POPS);
        float t;
        uint32_t f, c;
        if (w.sp < sh.lim) {
            t = col_t[w.sp * NT + lane];
            f = col_f[w.sp * NT + lane];
            c = col_c[w.sp * NT + lane];
        } else {
            t = w.deep_t[w.sp];
            f = w.deep_fc[w.sp].x;
            c = w.deep_fc[w.sp].y;
        }
        if (t <= w.t_max) {
            w.cur_first = f;
            w.cur_count = c;
            return false;
        }
    }
    return true;
}

// ---------------------------------------------------------------------
// Four-wide any-hit walk with a short shared stack of child references
// (SS x NT words), entries from `lim` on in local memory; SD at least the
// tree's stack need (checked on upload).
// ---------------------------------------------------------------------
template <int SS, int SD>
struct Walk4S {
    float t_max;
    uint32_t cur, sp, guard;
    bool hit_any;
    uint32_t deep[SD];
};

template <int SS, int SD>
__device__ __forceinline__ bool walk4s_begin(const Scene& s, const Ray& r, float t_max, Walk4S<SS, SD>& w) {
    w.hit_any = false;
    if (!r.valid || s.bvh4_root == NONE) return false;
    w.t_max = t_max;
    w.cur = s.bvh4_root;
    w.sp = 0u;
    w.guard = 4u * s.bvh4_nodes + 8u;
    return true;
}

template <bool COUNT, int SS, int SD, int NT>
__device__ __forceinline__ bool walk4s_step(const Scene* sp_, uint32_t* stack_words, uint32_t lim, const Ray& r,
                                            uint32_t path_seed, uint32_t ray_id, bool primary, uint32_t skip,
                                            Walk4S<SS, SD>& w, Cnt& cnt, uint32_t* err) {
    const Scene& s = *sp_;
    const uint32_t lane = threadIdx.x;
    if (w.guard-- == 0u) {
        atomicOr(err, 1u);
        return true;
    }
    const uint32_t cur = w.cur;
    if (cur & 0x80000000u) {
        bump<COUNT>(cnt, C_LEAVES);
        uint32_t first = cur & 0x07ffffffu, end = first + ((cur >> 27) & 15u) + 1u;
        if ((uint64_t)end > s.slot_count) {
            atomicOr(err, 2u);
            return true;
        }
        for (uint32_t slot = first; slot < end; slot++) {
            bump<COUNT>(cnt, C_TRIS);
            uint64_t tb = tri_base(s, slot);
            float4 q0 = geomv(s, tb), q1 = geomv(s, tb + 1), q2 = geomv(s, tb + 2);
            Hit h;
            if (!intersect(r, q0, q1, q2, w.t_max, &h)) continue;
            uint32_t gid = __float_as_uint(q0.w);
            if (gid == skip) continue;
            uint32_t m = __float_as_uint(q2.w);
            if (!accept_ol(sp_, slot, m, gid, h, path_seed, ray_id, primary)) continue;
            w.hit_any = true;
            return true;
        }
    } else {
        if (cur >= s.bvh4_nodes) {
            atomicOr(err, 1u);
            return true;
        }
        bump<COUNT>(cnt, C_BOXES, 4);
        const float4* nd = s.bvh4 + (uint64_t)cur * 8u;
        float4 lx = __ldg(nd), ly = __ldg(nd + 1), lz = __ldg(nd + 2);
        float4 hx = __ldg(nd + 3), hy = __ldg(nd + 4), hz = __ldg(nd + 5);
        uint4 rf = __ldg(reinterpret_cast<const uint4*>(nd) + 6);
        uint32_t ref[4] = {rf.x, rf.y, rf.z, rf.w};
        float t[4];
        t[0] = rf.x == NONE ? -1.0f : slab6(r, lx.x, ly.x, lz.x, hx.x, hy.x, hz.x, w.t_max);
        t[1] = rf.y == NONE ? -1.0f : slab6(r, lx.y, ly.y, lz.y, hx.y, hy.y, hz.y, w.t_max);
        t[2] = rf.z == NONE ? -1.0f : slab6(r, lx.z, ly.z, lz.z, hx.z, hy.z, hz.z, w.t_max);
        t[3] = rf.w == NONE ? -1.0f : slab6(r, lx.w, ly.w, lz.w, hx.w, hy.w, hz.w, w.t_max);
        int best = -1;
        float bt = 0.0f;
        uint32_t bref = NONE;
#pragma unroll
        for (int k = 0; k < 4; k++)
            if (t[k] >= 0.0f && (best < 0 || t[k] < bt)) {
                best = k;
                bt = t[k];
                bref = ref[k];
            }
        if (best >= 0) {
#pragma unroll
            for (int k = 0; k < 4; k++) {
                if (k == best || !(t[k] >= 0.0f)) continue;
                if (w.sp >= (uint32_t)SD) {  // excluded on upload
                    atomicOr(err, 4u);
                    return true;
                }
                if (w.sp < lim) stack_words[w.sp * NT + lane] = ref[k];
                else w.deep[w.sp] = ref[k];
                w.sp++;
            }
            w.cur = bref;
            return false;
        }
    }
    if (w.sp == 0u) return true;
    bump<COUNT>(cnt, C_POPS);
    --w.sp;
    w.cur = w.sp < lim ? stack_words[w.sp * NT + lane] : w.deep[w.sp];
    return false;
}

// ---------------------------------------------------------------------
// Four-wide any-hit walk with postponed leaves (Aila & Laine 2009,
// "Understanding the efficiency of ray traversal on GPUs": speculative
// traversal). A lane that reaches a leaf parks it and goes on with inner
// nodes; the warp tests leaves only in steps where no lane has node work
// left (every lane has parked a leaf and met a second one, or has run out
// of nodes), so node steps and leaf steps are not interleaved within a
// warp. Occlusion is order-free, so the answer is walk4s_step's; only
// steps that visit a node or test a leaf count against the guard (a lane
// waiting for the leaf step is not walking).
// ---------------------------------------------------------------------
template <int SS, int SD>
struct Walk4P {
    float t_max;
    uint32_t cur, pend, sp, guard;
    bool hit_any;
    uint32_t deep[SD];
};

template <int SS, int SD>
__device__ __forceinline__ bool walk4p_begin(const Scene& s, const Ray& r, float t_max, Walk4P<SS, SD>& w) {
    w.hit_any = false;
    if (!r.valid || s.bvh4_root == NONE) return false;
    w.t_max = t_max;
    w.cur = s.bvh4_root;
    w.pend = NONE;
    w.sp = 0u;
    w.guard = 4u * s.bvh4_nodes + 8u;
    return true;
}

// Whether the lane can take a node step now.
template <int SS, int SD>
__device__ __forceinline__ bool walk4p_node_work(const Walk4P<SS, SD>& w) {
    return w.cur != NONE && !((w.cur & 0x80000000u) && w.pend != NONE);
}

template <bool COUNT, int SS, int SD, int NT>
__device__ __forceinline__ bool walk4p_step(const Scene* sp_, uint32_t* stack_words, uint32_t lim, const Ray& r,
                                            uint32_t path_seed, uint32_t ray_id, bool primary, uint32_t skip,
                                            bool leaf_step, Walk4P<SS, SD>& w, Cnt& cnt, uint32_t* err) {
    const Scene& s = *sp_;
    const uint32_t lane = threadIdx.x;
    if (leaf_step) {
        if (w.pend != NONE) {
            if (w.guard-- == 0u) {
                atomicOr(err, 1u);
                return true;
            }
            bump<COUNT>(cnt, C_LEAVES);
            const uint32_t lf = w.pend;
            w.pend = NONE;
            uint32_t first = lf & 0x07ffffffu, end = first + ((lf >> 27) & 15u) + 1u;
            if ((uint64_t)end > s.slot_count) {
                atomicOr(err, 2u);
                return true;
            }
            for (uint32_t slot = first; slot < end; slot++) {
                bump<COUNT>(cnt, C_TRIS);
                uint64_t tb = tri_base(s, slot);
                float4 q0 = geomv(s, tb), q1 = geomv(s, tb + 1), q2 = geomv(s, tb + 2);
                Hit h;
                if (!intersect(r, q0, q1, q2, w.t_max, &h)) continue;
                uint32_t gid = __float_as_uint(q0.w);
                if (gid == skip) continue;
                uint32_t m = __float_as_uint(q2.w);
                if (!accept_ol(sp_, slot, m, gid, h, path_seed, ray_id, primary)) continue;
                w.hit_any = true;
                return true;
            }
        }
        return w.cur == NONE && w.pend == NONE;
    }
    uint32_t cur = w.cur;
    if (cur == NONE) return w.pend == NONE;
    if (cur & 0x80000000u) {
        if (w.pend != NONE) return false;  // parked: waits for the leaf step
        w.pend = cur;
    } else {
        if (w.guard-- == 0u) {
            atomicOr(err, 1u);
            return true;
        }
        if (cur >= s.bvh4_nodes) {
            atomicOr(err, 1u);
            return true;
        }
        bump<COUNT>(cnt, C_BOXES, 4);
        const float4* nd = s.bvh4 + (uint64_t)cur * 8u;
        float4 lx = __ldg(nd), ly = __ldg(nd + 1), lz = __ldg(nd + 2);
        float4 hx = __ldg(nd + 3), hy = __ldg(nd + 4), hz = __ldg(nd + 5);
        uint4 rf = __ldg(reinterpret_cast<const uint4*>(nd) + 6);
        uint32_t ref[4] = {rf.x, rf.y, rf.z, rf.w};
        float t[4];
        t[0] = rf.x == NONE ? -1.0f : slab6(r, lx.x, ly.x, lz.x, hx.x, hy.x, hz.x, w.t_max);
        t[1] = rf.y == NONE ? -1.0f : slab6(r, lx.y, ly.y, lz.y, hx.y, hy.y, hz.y, w.t_max);
        t[2] = rf.z == NONE ? -1.0f : slab6(r, lx.z, ly.z, lz.z, hx.z, hy.z, hz.z, w.t_max);
        t[3] = rf.w == NONE ? -1.0f : slab6(r, lx.w, ly.w, lz.w, hx.w, hy.w, hz.w, w.t_max);
        int best = -1;
        float bt = 0.0f;
        uint32_t bref = NONE;
#pragma unroll
        for (int k = 0; k < 4; k++)
            if (t[k] >= 0.0f && (best < 0 || t[k] < bt)) {
                best = k;
                bt = t[k];
                bref = ref[k];
            }
        if (best >= 0) {
#pragma unroll
            for (int k = 0; k < 4; k++) {
                if (k == best || !(t[k] >= 0.0f)) continue;
                if (w.sp >= (uint32_t)SD) {  // excluded on upload
                    atomicOr(err, 4u);
                    return true;
                }
                if (w.sp < lim) stack_words[w.sp * NT + lane] = ref[k];
                else w.deep[w.sp] = ref[k];
                w.sp++;
            }
            // A leaf child is parked at once when the lane has none parked.
            if ((bref & 0x80000000u) && w.pend == NONE) w.pend = bref;
            else {
                w.cur = bref;
                return false;
            }
        }
    }
    // Next node (or leaf) from the stack; none left: only the parked leaf.
    if (w.sp == 0u) {
        w.cur = NONE;
        return w.pend == NONE;
    }
    bump<COUNT>(cnt, C_POPS);
    --w.sp;
    w.cur = w.sp < lim ? stack_words[w.sp * NT + lane] : w.deep[w.sp];
    return false;
}

// ---------------------------------------------------------------------
// Four-wide closest-hit walk (the tolerance plan, not the reference's
// order). Per inner node the four child boxes are slab-tested against the
// current t_max; the nearest passing child is taken next and the others
// pushed with their entry distances, farthest first, so pops come back in
// near-to-far order; a popped entry farther than t_max is culled. With
// every child box inside its parent's it reaches every leaf the binary
// walk could need, so the closest hit is the binary walk's except where
// two candidate hits lie within rounding of each other (exact ties, and a
// leaf whose box entry rounds past a contained hit at nearly the same
// distance): there the order decides, and it differs. Stack entries are
// (reference, entry distance) in two column blocks of lim x NT words.
// ---------------------------------------------------------------------
template <int SS, int SD>
struct Walk4C {
    float t_max;
    uint32_t cur, sp, guard;
    bool hit_any;
    uint32_t best_mat;
    Hit best;
    uint32_t deep_ref[SD];
    float deep_t[SD];
};

template <int SS, int SD>
__device__ __forceinline__ bool walk4c_begin(const Scene& s, const Ray& r, float t_max, Walk4C<SS, SD>& w) {
    w.best.slot = NONE;
    w.hit_any = false;
    w.best_mat = 0u;
    if (!r.valid || s.bvh4_root == NONE || s.P.env[3] == 0u) return false;
    w.t_max = t_max;
    w.cur = s.bvh4_root;
    w.sp = 0u;
    w.guard = 4u * s.bvh4_nodes + 8u;
    return true;
}

template <bool COUNT, int SS, int SD, int NT>
__device__ __forceinline__ bool walk4c_step(const Scene* sp_, uint32_t* words, uint32_t lim, const Ray& r,
                                            uint32_t path_seed, uint32_t ray_id, bool primary, uint32_t skip,
                                            Walk4C<SS, SD>& w, Cnt& cnt, uint32_t* err) {
    const Scene& s = *sp_;
    const uint32_t lane = threadIdx.x;
    uint32_t* col_ref = words;
    float* col_t = reinterpret_cast<float*>(words + lim * NT);
    if (w.guard-- == 0u) {
        atomicOr(err, 1u);
        w.best.slot = NONE;
        w.hit_any = false;
        return true;
    }
    const uint32_t cur = w.cur;
    if (cur & 0x80000000u) {
        bump<COUNT>(cnt, C_LEAVES);
        uint32_t first = cur & 0x07ffffffu, end = first + ((cur >> 27) & 15u) + 1u;
        if ((uint64_t)end > s.slot_count) {
            atomicOr(err, 2u);
            w.best.slot = NONE;
            w.hit_any = false;
            return true;
        }
        for (uint32_t slot = first; slot < end; slot++) {
            bump<COUNT>(cnt, C_TRIS);
            uint64_t tb = tri_base(s, slot);
            float4 q0 = geomv(s, tb), q1 = geomv(s, tb + 1), q2 = geomv(s, tb + 2);
            Hit h;
            if (!intersect(r, q0, q1, q2, w.t_max, &h)) continue;
            uint32_t gid = __float_as_uint(q0.w);
            if (gid == skip) continue;
            uint32_t m = __float_as_uint(q2.w);
            if (!accept_ol(sp_, slot, m, gid, h, path_seed, ray_id, primary)) continue;
            h.slot = slot;
            w.best = h;
            w.best_mat = m;
            w.hit_any = true;
            w.t_max = h.t;
        }
    } else {
        if (cur >= s.bvh4_nodes) {
            atomicOr(err, 1u);
            w.best.slot = NONE;
            w.hit_any = false;
            return true;
        }
        bump<COUNT>(cnt, C_BOXES, 4);
        const float4* nd = s.bvh4 + (uint64_t)cur * 8u;
        float4 lx = __ldg(nd), ly = __ldg(nd + 1), lz = __ldg(nd + 2);
        float4 hx = __ldg(nd + 3), hy = __ldg(nd + 4), hz = __ldg(nd + 5);
        uint4 rf = __ldg(reinterpret_cast<const uint4*>(nd) + 6);
        uint32_t ref[4] = {rf.x, rf.y, rf.z, rf.w};
        float t[4];
        t[0] = rf.x == NONE ? -1.0f : slab6(r, lx.x, ly.x, lz.x, hx.x, hy.x, hz.x, w.t_max);
        t[1] = rf.y == NONE ? -1.0f : slab6(r, lx.y, ly.y, lz.y, hx.y, hy.y, hz.y, w.t_max);
        t[2] = rf.z == NONE ? -1.0f : slab6(r, lx.z, ly.z, lz.z, hx.z, hy.z, hz.z, w.t_max);
        t[3] = rf.w == NONE ? -1.0f : slab6(r, lx.w, ly.w, lz.w, hx.w, hy.w, hz.w, w.t_max);
        // Order the passing children near to far (ties by child index).
        uint32_t ord[4] = {0u, 1u, 2u, 3u};
        uint32_t n = 0u;
#pragma unroll
        for (int k = 0; k < 4; k++)
            if (t[k] >= 0.0f) ord[n++] = (uint32_t)k;
#pragma unroll
        for (int i = 1; i < 4; i++) {
#pragma unroll
            for (int j = i; j > 0; j--) {
                if ((uint32_t)j >= n) continue;
                uint32_t a = ord[j - 1], b = ord[j];
                if (t[b] < t[a]) {
                    ord[j - 1] = b;
                    ord[j] = a;
                }
            }
        }
        if (n > 0u) {
            // Push all but the nearest, farthest first.
            for (uint32_t q = n - 1u; q >= 1u; q--) {
                if (w.sp >= (uint32_t)SD) {  // excluded on upload
                    atomicOr(err, 4u);
                    w.best.slot = NONE;
                    w.hit_any = false;
                    return true;
                }
                uint32_t k = ord[q];
                if (w.sp < lim) {
                    col_ref[w.sp * NT + lane] = ref[k];
                    col_t[w.sp * NT + lane] = t[k];
                } else {
                    w.deep_ref[w.sp] = ref[k];
                    w.deep_t[w.sp] = t[k];
                }
                w.sp++;
            }
            w.cur = ref[ord[0]];
            return false;
        }
    }
    while (w.sp != 0u) {
        w.sp--;
        bump<COUNT>(cnt, C_POPS);
        float te;
        uint32_t rr;
        if (w.sp < lim) {
            te = col_t[w.sp * NT + lane];
            rr = col_ref[w.sp * NT + lane];
        } else {
            te = w.deep_t[w.sp];
            rr = w.deep_ref[w.sp];
        }
        if (te <= w.t_max) {
            w.cur = rr;
            return false;
        }
    }
    return true;
}

}  // namespace oxd
