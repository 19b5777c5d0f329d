// BVH traversal shared by the megakernel and the wavefront kernels.
//
// The reference's ordered walk (near child first, far child pushed with
// its entry distance, pops culled against t_max; pathtrace.wgsl:646-735)
// over the same node layout, with the two children of an inner node
// fetched as one 64-byte pair, the chosen child carried in registers and
// (first, count) pushed instead of a node index: one dependent fetch per
// inner node instead of three. Any-hit acceptance follows
// pathtrace.wgsl:621-636.
#pragma once

#include "kernels.cuh"
#include "shade.cuh"

namespace oxd {

struct Cnt {
    unsigned long long c[C_N];
};

template <bool COUNT>
__device__ __forceinline__ void bump(Cnt& c, int k, unsigned long long v = 1) {
    if (COUNT) c.c[k] += v;
}

// Any-hit acceptance (pathtrace.wgsl:621-636).
__device__ __forceinline__ bool accept(const Scene& s, uint32_t slot, uint32_t m, uint32_t gid, const Hit& h,
                                       const Sampler& smp, uint32_t ray_id, bool primary) {
    uint32_t fl = mat_flags(s, m);
    if (primary && !h.front && (fl & 4u) == 0u) return false;
    uint32_t mode = fl & 3u;
    if (mode == 0u) return true;
    if (mode == 1u) return hit_alpha(s, slot, m, h.b) >= tf(s, mat_off(s, m) + 11u);
    return coin(smp, ray_id, gid) < hit_alpha(s, slot, m, h.b);
}

// The walks are written as resumable state machines: begin() sets a ray's
// walk up, step() advances it by one loop iteration of the reference's
// walk (one inner node or one leaf, then the pops that follow) and says
// whether it is over. A thread that loops step() to the end performs
// exactly the operations of a single loop; the wavefront traversal kernels
// instead interleave walks, giving an idle lane a new ray while the other
// lanes of its warp are still walking theirs. Results do not depend on the
// interleaving.

// Ordered binary walk (pathtrace.wgsl:646-735): closest hit (any = false)
// or first accepted hit (any = true). SD is the stack depth: the
// reference's 64 (an overflow drops the far child, pathtrace.wgsl:700-704),
// or any depth at least the BVH's, which never overflows and so gives the
// same walk with less local memory.
template <int SD>
struct Walk2 {
    float t_max;
    uint32_t cur_first, cur_count, sp, guard;
    bool hit_any;
    uint32_t best_mat;
    Hit best;
    uint2 st_fc[SD];
    float st_t[SD];
};

// False when the query is answered before any node is visited (no hit).
template <bool COUNT, int SD>
__device__ __forceinline__ bool walk2_begin(const Scene& s, const Ray& r, float t_max, Walk2<SD>& w, Cnt& cnt) {
    w.best.slot = NONE;
    w.hit_any = false;
    w.best_mat = 0u;
    uint32_t node_count = s.P.env[3];
    if (node_count == 0u || !r.valid) return false;
    float4 rlo = geomv(s, 0), rhi = geomv(s, 1);
    bump<COUNT>(cnt, C_BOXES);
    if (slab(r, rlo, rhi, t_max) < 0.0f) return false;
    w.t_max = t_max;
    w.cur_first = __float_as_uint(rlo.w);
    w.cur_count = __float_as_uint(rhi.w);
    w.sp = 0u;
    // A tree visits each node at most once; anything longer is a malformed
    // BVH, reported through the error word instead of looping.
    w.guard = node_count + 8u;
    return true;
}

// True when the walk is over; the answer is then w.hit_any, w.best and
// w.best_mat.
template <bool COUNT, int SD>
__device__ __forceinline__ bool walk2_step(const Scene& s, const Ray& r, const Sampler& smp, uint32_t ray_id,
                                           bool primary, bool any, uint32_t skip, Walk2<SD>& w, Cnt& cnt,
                                           uint32_t* err) {
    if (w.guard-- == 0u) {
        atomicOr(err, 1u);
        w.best.slot = NONE;
        w.hit_any = false;
        return true;
    }
    if (w.cur_count > 0u) {
        bump<COUNT>(cnt, C_LEAVES);
        if ((uint64_t)w.cur_first + w.cur_count > s.slot_count) {  // malformed leaf
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
            if (!accept(s, slot, m, gid, h, smp, ray_id, primary)) continue;
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
        float4 alo = geomv(s, 2 * l), ahi = geomv(s, 2 * l + 1);
        float4 blo = geomv(s, 2 * l + 2), bhi = geomv(s, 2 * l + 3);
        float tl = slab(r, alo, ahi, w.t_max);
        float tr = slab(r, blo, bhi, w.t_max);
        if (tl >= 0.0f && tr >= 0.0f) {
            bool swap = tl > tr;
            uint2 nearfc = swap ? make_uint2(__float_as_uint(blo.w), __float_as_uint(bhi.w))
                                : make_uint2(__float_as_uint(alo.w), __float_as_uint(ahi.w));
            uint2 farfc = swap ? make_uint2(__float_as_uint(alo.w), __float_as_uint(ahi.w))
                               : make_uint2(__float_as_uint(blo.w), __float_as_uint(bhi.w));
            if (w.sp < (uint32_t)SD) {
                w.st_fc[w.sp] = farfc;
                w.st_t[w.sp] = swap ? tl : tr;
                w.sp++;
            }
            w.cur_first = nearfc.x;
            w.cur_count = nearfc.y;
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
        if (w.st_t[w.sp] <= w.t_max) {
            w.cur_first = w.st_fc[w.sp].x;
            w.cur_count = w.st_fc[w.sp].y;
            return false;
        }
    }
    return true;
}

// The whole query in one call. Returns whether something was hit; *best
// holds the hit and *best_mat its material.
template <bool COUNT, int SD = STACK>
__device__ bool traverse(const Scene& s, const Ray& r, float t_max, const Sampler& smp, uint32_t ray_id,
                         bool primary, bool any, uint32_t skip, Hit* best, uint32_t* best_mat, Cnt& cnt,
                         uint32_t* err) {
    Walk2<SD> w;
    if (walk2_begin<COUNT, SD>(s, r, t_max, w, cnt))
        while (!walk2_step<COUNT, SD>(s, r, smp, ray_id, primary, any, skip, w, cnt, err)) {
        }
    *best = w.best;
    if (w.hit_any) *best_mat = w.best_mat;
    return w.hit_any;
}

// Any-hit walk over the four-wide tree built on upload (host/bvh4.cpp):
// 128-byte nodes holding four child boxes as x/y/z planes and four child
// references, one node per cache line. Whether a ray is occluded does not
// depend on the order its candidate triangles are tested in (acceptance is
// a function of the ray and the triangle alone), and with every child box
// inside its parent's the slab test passes a leaf's box only if it passes
// all its ancestors', so this walk tests exactly the leaves the binary walk
// reaches and returns the same answer with half the dependent fetches.
// The nearest passing child is taken next and the others pushed without
// their distances (order only changes how early an occluder is found). SD
// is at least the tree's stack need, checked on upload.
template <int SD>
struct Walk4 {
    float t_max;
    uint32_t cur, sp, guard;
    bool hit_any;
    uint32_t best_mat;
    Hit best;
    uint32_t stack[SD];
};

template <int SD>
__device__ __forceinline__ bool walk4_begin(const Scene& s, const Ray& r, float t_max, Walk4<SD>& w) {
    w.best.slot = NONE;
    w.hit_any = false;
    w.best_mat = 0u;
    if (!r.valid || s.bvh4_root == NONE) return false;
    w.t_max = t_max;
    w.cur = s.bvh4_root;
    w.sp = 0u;
    w.guard = 4u * s.bvh4_nodes + 8u;
    return true;
}

template <bool COUNT, int SD>
__device__ __forceinline__ bool walk4_step(const Scene& s, const Ray& r, const Sampler& smp, uint32_t ray_id,
                                           bool primary, uint32_t skip, Walk4<SD>& w, Cnt& cnt, uint32_t* err) {
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
            if (!accept(s, slot, m, gid, h, smp, ray_id, primary)) continue;
            h.slot = slot;
            w.best = h;
            w.best_mat = m;
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
                w.stack[w.sp++] = ref[k];
            }
            w.cur = bref;
            return false;
        }
    }
    if (w.sp == 0u) return true;
    bump<COUNT>(cnt, C_POPS);
    w.cur = w.stack[--w.sp];
    return false;
}

// The whole four-wide query in one call; *hit is the accepted triangle.
template <bool COUNT, int SD>
__device__ bool occluded4(const Scene& s, const Ray& r, float t_max, const Sampler& smp, uint32_t ray_id,
                          bool primary, uint32_t skip, Hit* hit, uint32_t* hit_mat, Cnt& cnt, uint32_t* err) {
    Walk4<SD> w;
    if (walk4_begin<SD>(s, r, t_max, w))
        while (!walk4_step<COUNT, SD>(s, r, smp, ray_id, primary, skip, w, cnt, err)) {
        }
    *hit = w.best;
    if (w.hit_any) *hit_mat = w.best_mat;
    return w.hit_any;
}

}  // namespace oxd
