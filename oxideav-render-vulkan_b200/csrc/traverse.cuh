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

// Closest-hit (any = false) or any-hit (any = true) query. Returns whether
// something was hit; *best holds the hit and *best_mat its material.
// SD is the stack depth: the reference's 64 (an overflow drops the far
// child, pathtrace.wgsl:700-704), or any depth at least the BVH's, which
// never overflows and so gives the same walk with less local memory.
template <bool COUNT, int SD = STACK>
__device__ bool traverse(const Scene& s, const Ray& r, float t_max, const Sampler& smp, uint32_t ray_id,
                         bool primary, bool any, uint32_t skip, Hit* best, uint32_t* best_mat, Cnt& cnt,
                         uint32_t* err) {
    best->slot = NONE;
    uint32_t node_count = s.P.env[3];
    if (node_count == 0u || !r.valid) return false;
    float4 rlo = geomv(s, 0), rhi = geomv(s, 1);
    bump<COUNT>(cnt, C_BOXES);
    if (slab(r, rlo, rhi, t_max) < 0.0f) return false;
    uint32_t cur_first = __float_as_uint(rlo.w), cur_count = __float_as_uint(rhi.w);
    uint2 st_fc[SD];
    float st_t[SD];
    uint32_t sp = 0u;
    // A tree visits each node at most once; anything longer is a malformed
    // BVH, reported through the error word instead of looping.
    uint32_t guard = node_count + 8u;
    bool hit_any = false;
    for (;;) {
        if (guard-- == 0u) {
            atomicOr(err, 1u);
            best->slot = NONE;
            return false;
        }
        if (cur_count > 0u) {
            bump<COUNT>(cnt, C_LEAVES);
            if ((uint64_t)cur_first + cur_count > s.slot_count) {  // malformed leaf
                atomicOr(err, 2u);
                best->slot = NONE;
                return false;
            }
            uint32_t end = cur_first + cur_count;
            for (uint32_t slot = cur_first; slot < end; slot++) {
                bump<COUNT>(cnt, C_TRIS);
                uint64_t tb = tri_base(s, slot);
                float4 q0 = geomv(s, tb), q1 = geomv(s, tb + 1), q2 = geomv(s, tb + 2);
                Hit h;
                if (!intersect(r, q0, q1, q2, t_max, &h)) continue;
                uint32_t gid = __float_as_uint(q0.w);
                if (gid == skip) continue;
                uint32_t m = __float_as_uint(q2.w);
                if (!accept(s, slot, m, gid, h, smp, ray_id, primary)) continue;
                h.slot = slot;
                *best = h;
                *best_mat = m;
                hit_any = true;
                if (any) return true;
                t_max = h.t;
            }
        } else {
            bump<COUNT>(cnt, C_BOXES, 2);
            uint64_t l = cur_first;
            float4 alo = geomv(s, 2 * l), ahi = geomv(s, 2 * l + 1);
            float4 blo = geomv(s, 2 * l + 2), bhi = geomv(s, 2 * l + 3);
            float tl = slab(r, alo, ahi, t_max);
            float tr = slab(r, blo, bhi, t_max);
            if (tl >= 0.0f && tr >= 0.0f) {
                bool swap = tl > tr;
                uint2 nearfc = swap ? make_uint2(__float_as_uint(blo.w), __float_as_uint(bhi.w))
                                    : make_uint2(__float_as_uint(alo.w), __float_as_uint(ahi.w));
                uint2 farfc = swap ? make_uint2(__float_as_uint(alo.w), __float_as_uint(ahi.w))
                                   : make_uint2(__float_as_uint(blo.w), __float_as_uint(bhi.w));
                if (sp < (uint32_t)SD) {
                    st_fc[sp] = farfc;
                    st_t[sp] = swap ? tl : tr;
                    sp++;
                }
                cur_first = nearfc.x;
                cur_count = nearfc.y;
                continue;
            } else if (tl >= 0.0f) {
                cur_first = __float_as_uint(alo.w);
                cur_count = __float_as_uint(ahi.w);
                continue;
            } else if (tr >= 0.0f) {
                cur_first = __float_as_uint(blo.w);
                cur_count = __float_as_uint(bhi.w);
                continue;
            }
        }
        bool found = false;
        while (sp != 0u) {
            sp--;
            bump<COUNT>(cnt, C_POPS);
            if (st_t[sp] <= t_max) {
                cur_first = st_fc[sp].x;
                cur_count = st_fc[sp].y;
                found = true;
                break;
            }
        }
        if (!found) break;
    }
    return hit_any;
}

}  // namespace oxd
