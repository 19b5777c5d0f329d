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

// Any-hit query over the four-wide tree built on upload (host/bvh4.cpp):
// 128-byte nodes holding four child boxes as x/y/z planes and four child
// references, one node per cache line. Whether a ray is occluded does not
// depend on the order its candidate triangles are tested in (acceptance is
// a function of the ray and the triangle alone), and with every child box
// inside its parent's the slab test passes a leaf's box only if it passes
// all its ancestors', so this walk tests exactly the leaves the binary walk
// reaches and returns the same answer with half the dependent fetches.
// The nearest passing child is taken next and the others pushed without
// their distances (order only changes how early an occluder is found). SD
// is at least the tree's stack need, checked on upload; *hit is the
// accepted triangle.
template <bool COUNT, int SD>
__device__ bool occluded4(const Scene& s, const Ray& r, float t_max, const Sampler& smp, uint32_t ray_id,
                          bool primary, uint32_t skip, Hit* hit, uint32_t* hit_mat, Cnt& cnt, uint32_t* err) {
    hit->slot = NONE;
    if (!r.valid || s.bvh4_root == NONE) return false;
    uint32_t stack[SD];
    uint32_t sp = 0u, cur = s.bvh4_root;
    uint32_t guard = 4u * s.bvh4_nodes + 8u;
    for (;;) {
        if (guard-- == 0u) {
            atomicOr(err, 1u);
            return false;
        }
        if (cur & 0x80000000u) {
            bump<COUNT>(cnt, C_LEAVES);
            uint32_t first = cur & 0x07ffffffu, end = first + ((cur >> 27) & 15u) + 1u;
            if ((uint64_t)end > s.slot_count) {
                atomicOr(err, 2u);
                return false;
            }
            for (uint32_t slot = first; slot < end; slot++) {
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
                *hit = h;
                *hit_mat = m;
                return true;
            }
        } else {
            if (cur >= s.bvh4_nodes) {
                atomicOr(err, 1u);
                return false;
            }
            bump<COUNT>(cnt, C_BOXES, 4);
            const float4* nd = s.bvh4 + (uint64_t)cur * 8u;
            float4 lx = __ldg(nd), ly = __ldg(nd + 1), lz = __ldg(nd + 2);
            float4 hx = __ldg(nd + 3), hy = __ldg(nd + 4), hz = __ldg(nd + 5);
            uint4 rf = __ldg(reinterpret_cast<const uint4*>(nd) + 6);
            uint32_t ref[4] = {rf.x, rf.y, rf.z, rf.w};
            float t[4];
            t[0] = rf.x == NONE ? -1.0f : slab6(r, lx.x, ly.x, lz.x, hx.x, hy.x, hz.x, t_max);
            t[1] = rf.y == NONE ? -1.0f : slab6(r, lx.y, ly.y, lz.y, hx.y, hy.y, hz.y, t_max);
            t[2] = rf.z == NONE ? -1.0f : slab6(r, lx.z, ly.z, lz.z, hx.z, hy.z, hz.z, t_max);
            t[3] = rf.w == NONE ? -1.0f : slab6(r, lx.w, ly.w, lz.w, hx.w, hy.w, hz.w, t_max);
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
                    if (sp >= (uint32_t)SD) {  // excluded on upload
                        atomicOr(err, 4u);
                        return false;
                    }
                    stack[sp++] = ref[k];
                }
                cur = bref;
                continue;
            }
        }
        if (sp == 0u) return false;
        bump<COUNT>(cnt, C_POPS);
        cur = stack[--sp];
    }
}

}  // namespace oxd
