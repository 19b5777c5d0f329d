// Binned-SAH BVH build on the GPU, producing the same node words and slot
// order as the host builder (host/bvh.cpp: level-order, stable partitions,
// 32 bins per axis, unit SAH costs, leaves of at most 8 triangles).
//
// Per level of the tree:
//   decide_small   one thread per node of at most LARGE triangles: bounds,
//                  binning and the SAH sweep exactly as the host writes
//                  them, then the stable partition of its triangle ids;
//   decide_large   one CTA per larger node: bounds and bins reduced in
//                  shared memory (float min / max as order-preserving
//                  integers, so any order gives the host's bits), the SAH
//                  sweep by one thread, then a stable partition chunk by
//                  chunk with block scans;
//   scan / emit    child pairs are numbered by an exclusive scan over the
//                  level's split flags in node order (the host allocates
//                  them in that order), node words are written and the next
//                  level's nodes listed.
// Every float operation (box growth, areas, costs, bin indices) is the
// host's, in the host's order, without contraction.
#include <cfloat>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <string>
#include <vector>

#include "../../include/oxpt_diag.h"
#include "../host/bvh_gpu.hpp"

namespace oxd {
namespace bvhb {

constexpr int BINS = 32;
constexpr uint32_t MAX_LEAF = 8;
// Work per node by its triangle count: a thread (<= SMALL_MAX), a warp
// (<= LARGE), a CTA (<= HUGE_N), or CTAs over CHUNK-triangle chunks.
constexpr uint32_t SMALL_MAX = 32;
constexpr uint32_t LARGE = 1024;
constexpr uint32_t HUGE_N = 16384;
constexpr uint32_t CHUNK = 4096;
constexpr uint32_t CTA = 512;
constexpr int WN = 8;  // nodes (warps) per CTA of decide_warp

struct Job {
    uint32_t node, begin, end, pad;
};
struct Decision {
    float lo[3], hi[3];
    uint32_t split, mid, pad0, pad1;
};

__device__ __forceinline__ float area(const float* lo, const float* hi) {
    float ex = hi[0] - lo[0], ey = hi[1] - lo[1], ez = hi[2] - lo[2];
    if (ex < 0 || ey < 0 || ez < 0) return 0.0f;
    return 2.0f * (ex * ey + ey * ez + ez * ex);
}

__device__ __forceinline__ int bin_of(float c, float lo, float scale) {
    int b = (int)((c - lo) * scale);
    return min(max(b, 0), BINS - 1);
}

// Order-preserving integer image of a float (for atomic min / max).
__device__ __forceinline__ int fkey(float f) {
    int b = __float_as_int(f);
    return b >= 0 ? b : b ^ 0x7fffffff;
}
__device__ __forceinline__ float funkey(int k) { return __int_as_float(k >= 0 ? k : k ^ 0x7fffffff); }

__global__ void tri_prep(const float* pos, uint32_t n, float4* blo, float4* bhi, float4* cen, uint32_t* ids) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int v = 0; v < 3; v++)
        for (int k = 0; k < 3; k++) {
            float x = pos[(size_t)i * 9 + v * 3 + k] + 0.0f;
            lo[k] = fminf(lo[k], x);
            hi[k] = fmaxf(hi[k], x);
        }
    blo[i] = make_float4(lo[0], lo[1], lo[2], 0.0f);
    bhi[i] = make_float4(hi[0], hi[1], hi[2], 0.0f);
    cen[i] = make_float4((lo[0] + hi[0]) * 0.5f, (lo[1] + hi[1]) * 0.5f, (lo[2] + hi[2]) * 0.5f, 0.0f);
    ids[i] = i;
}

struct Tri {
    const float4 *blo, *bhi, *cen;
};

// One axis of the host's SAH sweep (host/bvh.cpp) over binned boxes and
// counts given by accessors: the cheapest split after bin `split` (first
// minimum in bin order), or split -1 when the axis has no candidate.
template <class Lo, class Hi, class Cnt>
__device__ void axis_sweep(Lo blo, Hi bhi, Cnt bc, float* cost_out, int* split_out) {
    float right_area[BINS];
    uint32_t right_count[BINS];
    float alo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, ahi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    uint32_t nn = 0;
    for (int b = BINS - 1; b > 0; b--) {
        for (int k = 0; k < 3; k++) {
            alo[k] = fminf(alo[k], blo(b, k));
            ahi[k] = fmaxf(ahi[k], bhi(b, k));
        }
        nn += bc(b);
        right_area[b] = area(alo, ahi);
        right_count[b] = nn;
    }
    float llo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, lhi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    uint32_t ln = 0;
    float best = FLT_MAX;
    int split = -1;
    for (int b = 0; b < BINS - 1; b++) {
        for (int k = 0; k < 3; k++) {
            llo[k] = fminf(llo[k], blo(b, k));
            lhi[k] = fmaxf(lhi[k], bhi(b, k));
        }
        ln += bc(b);
        if (ln == 0 || right_count[b + 1] == 0) continue;
        float cost = area(llo, lhi) * (float)ln + right_area[b + 1] * (float)right_count[b + 1];
        if (cost < best) {
            best = cost;
            split = b;
        }
    }
    *cost_out = best;
    *split_out = split;
}

// The host's leaf / split decision from the best axis (-1: none).
__device__ void finish_decision(int best_axis, int best_split, float best_cost, const float* clo, const float* chi,
                                const float* lo, const float* hi, uint32_t begin, uint32_t count, Decision* d,
                                int* axis_out, int* split_out, float* plo, float* pscale) {
    for (int k = 0; k < 3; k++) {
        d->lo[k] = lo[k];
        d->hi[k] = hi[k];
    }
    float parent_area = area(lo, hi);
    float leaf_cost = (float)count;
    float split_cost = parent_area > 0 ? 1.0f + best_cost / parent_area : FLT_MAX;
    *axis_out = -1;
    if (best_axis < 0) {
        if (count <= MAX_LEAF) {
            d->split = 0;
            return;
        }
        d->split = 1;
        d->mid = begin + count / 2;  // coincident centroids: halves, no reordering
        return;
    }
    if (count <= MAX_LEAF && leaf_cost <= split_cost) {
        d->split = 0;
        return;
    }
    d->split = 1;
    *axis_out = best_axis;
    *split_out = best_split;
    *plo = clo[best_axis];
    *pscale = BINS / (chi[best_axis] - clo[best_axis]);
}

// The host's SAH sweep over binned boxes / counts; returns the decision.
// Axes in order, a later axis taking over only when strictly cheaper.
__device__ void sah(const float (*blo)[BINS][3], const float (*bhi)[BINS][3], const uint32_t (*bc)[BINS],
                    const float* clo, const float* chi, const float* lo, const float* hi, uint32_t begin,
                    uint32_t count, Decision* d, int* axis_out, int* split_out, float* plo, float* pscale) {
    float best_cost = FLT_MAX;
    int best_axis = -1, best_split = -1;
    for (int axis = 0; axis < 3; axis++) {
        if (!(chi[axis] > clo[axis])) continue;
        float c;
        int sp;
        axis_sweep([&](int b, int k) { return blo[axis][b][k]; }, [&](int b, int k) { return bhi[axis][b][k]; },
                   [&](int b) { return bc[axis][b]; }, &c, &sp);
        if (sp >= 0 && c < best_cost) {
            best_cost = c;
            best_axis = axis;
            best_split = sp;
        }
    }
    finish_decision(best_axis, best_split, best_cost, clo, chi, lo, hi, begin, count, d, axis_out, split_out, plo,
                    pscale);
}

__global__ void decide_small(const Job* jobs, uint32_t K, Tri tr, const uint32_t* ids, uint32_t* ids_next,
                             Decision* dec) {
    uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= K) return;
    Job jb = jobs[j];
    uint32_t count = jb.end - jb.begin;
    if (count > SMALL_MAX) return;
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    float clo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, chi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (uint32_t i = jb.begin; i < jb.end; i++) {
        uint32_t t = ids[i];
        float4 a = tr.blo[t], b = tr.bhi[t], c = tr.cen[t];
        lo[0] = fminf(lo[0], a.x); lo[1] = fminf(lo[1], a.y); lo[2] = fminf(lo[2], a.z);
        hi[0] = fmaxf(hi[0], b.x); hi[1] = fmaxf(hi[1], b.y); hi[2] = fmaxf(hi[2], b.z);
        clo[0] = fminf(clo[0], c.x); clo[1] = fminf(clo[1], c.y); clo[2] = fminf(clo[2], c.z);
        chi[0] = fmaxf(chi[0], c.x); chi[1] = fmaxf(chi[1], c.y); chi[2] = fmaxf(chi[2], c.z);
    }
    Decision d;
    d.mid = jb.begin;
    d.pad0 = d.pad1 = 0;
    int axis = -1, split = -1;
    float plo = 0.0f, pscale = 0.0f;
    if (count <= 1) {
        for (int k = 0; k < 3; k++) {
            d.lo[k] = lo[k];
            d.hi[k] = hi[k];
        }
        d.split = 0;
    } else {
        float blo[3][BINS][3], bhi[3][BINS][3];
        uint32_t bc[3][BINS];
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < BINS; b++) {
                bc[a][b] = 0;
                for (int k = 0; k < 3; k++) {
                    blo[a][b][k] = FLT_MAX;
                    bhi[a][b][k] = -FLT_MAX;
                }
            }
        for (int a = 0; a < 3; a++) {
            if (!(chi[a] > clo[a])) continue;
            float scale = BINS / (chi[a] - clo[a]);
            for (uint32_t i = jb.begin; i < jb.end; i++) {
                uint32_t t = ids[i];
                float4 c = tr.cen[t], x = tr.blo[t], y = tr.bhi[t];
                float cv = a == 0 ? c.x : (a == 1 ? c.y : c.z);
                int b = bin_of(cv, clo[a], scale);
                bc[a][b]++;
                blo[a][b][0] = fminf(blo[a][b][0], x.x); blo[a][b][1] = fminf(blo[a][b][1], x.y);
                blo[a][b][2] = fminf(blo[a][b][2], x.z);
                bhi[a][b][0] = fmaxf(bhi[a][b][0], y.x); bhi[a][b][1] = fmaxf(bhi[a][b][1], y.y);
                bhi[a][b][2] = fmaxf(bhi[a][b][2], y.z);
            }
        }
        sah(blo, bhi, bc, clo, chi, lo, hi, jb.begin, count, &d, &axis, &split, &plo, &pscale);
    }
    // Stable partition (or a copy).
    if (axis >= 0) {
        uint32_t w = jb.begin;
        for (uint32_t i = jb.begin; i < jb.end; i++) {
            uint32_t t = ids[i];
            float4 c = tr.cen[t];
            float cv = axis == 0 ? c.x : (axis == 1 ? c.y : c.z);
            if (bin_of(cv, plo, pscale) <= split) ids_next[w++] = t;
        }
        uint32_t mid = w;
        for (uint32_t i = jb.begin; i < jb.end; i++) {
            uint32_t t = ids[i];
            float4 c = tr.cen[t];
            float cv = axis == 0 ? c.x : (axis == 1 ? c.y : c.z);
            if (bin_of(cv, plo, pscale) > split) ids_next[w++] = t;
        }
        d.mid = (mid == jb.begin || mid == jb.end) ? jb.begin + count / 2 : mid;
    } else {
        for (uint32_t i = jb.begin; i < jb.end; i++) ids_next[i] = ids[i];
    }
    dec[j] = d;
}

__global__ void __launch_bounds__(CTA) decide_large(const Job* jobs, const uint32_t* list, uint32_t L, Tri tr,
                                                    const uint32_t* ids, uint32_t* ids_next, Decision* dec) {
    if (blockIdx.x >= L) return;
    const uint32_t j = list[blockIdx.x];
    const Job jb = jobs[j];
    const uint32_t count = jb.end - jb.begin;
    __shared__ int s_box[12];                // lo xyz, hi xyz, clo xyz, chi xyz (keys)
    __shared__ int s_blo[3][BINS][3], s_bhi[3][BINS][3];
    __shared__ uint32_t s_bc[3][BINS];
    __shared__ uint32_t s_scan[CTA / 32 + 1];
    __shared__ int s_axis, s_split;
    __shared__ float s_plo, s_pscale;
    __shared__ uint32_t s_left, s_base_left, s_base_right;
    const uint32_t t = threadIdx.x;
    if (t < 12) s_box[t] = (t % 6) < 3 ? fkey(FLT_MAX) : fkey(-FLT_MAX);
    for (uint32_t i = t; i < 3 * BINS; i += CTA) {
        int a = i / BINS, b = i % BINS;
        s_bc[a][b] = 0;
        for (int k = 0; k < 3; k++) {
            s_blo[a][b][k] = fkey(FLT_MAX);
            s_bhi[a][b][k] = fkey(-FLT_MAX);
        }
    }
    __syncthreads();
    // Bounds and centroid bounds.
    {
        float v[12];
        for (int k = 0; k < 12; k++) v[k] = (k % 6) < 3 ? FLT_MAX : -FLT_MAX;
        for (uint32_t i = jb.begin + t; i < jb.end; i += CTA) {
            uint32_t id = ids[i];
            float4 a = tr.blo[id], b = tr.bhi[id], c = tr.cen[id];
            v[0] = fminf(v[0], a.x); v[1] = fminf(v[1], a.y); v[2] = fminf(v[2], a.z);
            v[3] = fmaxf(v[3], b.x); v[4] = fmaxf(v[4], b.y); v[5] = fmaxf(v[5], b.z);
            v[6] = fminf(v[6], c.x); v[7] = fminf(v[7], c.y); v[8] = fminf(v[8], c.z);
            v[9] = fmaxf(v[9], c.x); v[10] = fmaxf(v[10], c.y); v[11] = fmaxf(v[11], c.z);
        }
        for (int k = 0; k < 12; k++) {
            if ((k % 6) < 3) atomicMin(&s_box[k], fkey(v[k]));
            else atomicMax(&s_box[k], fkey(v[k]));
        }
    }
    __syncthreads();
    float lo[3], hi[3], clo[3], chi[3];
    for (int k = 0; k < 3; k++) {
        lo[k] = funkey(s_box[k]);
        hi[k] = funkey(s_box[3 + k]);
        clo[k] = funkey(s_box[6 + k]);
        chi[k] = funkey(s_box[9 + k]);
    }
    // Bins.
    for (uint32_t i = jb.begin + t; i < jb.end; i += CTA) {
        uint32_t id = ids[i];
        float4 c = tr.cen[id], x = tr.blo[id], y = tr.bhi[id];
        const float cv[3] = {c.x, c.y, c.z};
        for (int a = 0; a < 3; a++) {
            if (!(chi[a] > clo[a])) continue;
            float scale = BINS / (chi[a] - clo[a]);
            int b = bin_of(cv[a], clo[a], scale);
            atomicAdd(&s_bc[a][b], 1u);
            atomicMin(&s_blo[a][b][0], fkey(x.x));
            atomicMin(&s_blo[a][b][1], fkey(x.y));
            atomicMin(&s_blo[a][b][2], fkey(x.z));
            atomicMax(&s_bhi[a][b][0], fkey(y.x));
            atomicMax(&s_bhi[a][b][1], fkey(y.y));
            atomicMax(&s_bhi[a][b][2], fkey(y.z));
        }
    }
    __syncthreads();
    if (t == 0) {
        float blo[3][BINS][3], bhi[3][BINS][3];
        uint32_t bc[3][BINS];
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < BINS; b++) {
                bc[a][b] = s_bc[a][b];
                for (int k = 0; k < 3; k++) {
                    blo[a][b][k] = funkey(s_blo[a][b][k]);
                    bhi[a][b][k] = funkey(s_bhi[a][b][k]);
                }
            }
        Decision d;
        d.mid = jb.begin;
        d.pad0 = d.pad1 = 0;
        int axis = -1, split = -1;
        float plo = 0.0f, pscale = 0.0f;
        sah(blo, bhi, bc, clo, chi, lo, hi, jb.begin, count, &d, &axis, &split, &plo, &pscale);
        dec[j] = d;
        s_axis = axis;
        s_split = split;
        s_plo = plo;
        s_pscale = pscale;
        uint32_t left = 0;
        if (axis >= 0)
            for (int b = 0; b <= split; b++) left += bc[axis][b];
        s_left = left;
        s_base_left = 0;
        s_base_right = 0;
    }
    __syncthreads();
    const int axis = s_axis, split = s_split;
    const float plo = s_plo, pscale = s_pscale;
    if (axis < 0) {
        for (uint32_t i = jb.begin + t; i < jb.end; i += CTA) ids_next[i] = ids[i];
        return;
    }
    // Stable partition, one chunk of CTA ids at a time.
    const uint32_t left_total = s_left;
    const uint32_t lane = t & 31, warp = t >> 5;
    for (uint32_t c0 = jb.begin; c0 < jb.end; c0 += CTA) {
        uint32_t i = c0 + t;
        bool valid = i < jb.end;
        uint32_t id = valid ? ids[i] : 0u;
        bool goes_left = false;
        if (valid) {
            float4 c = tr.cen[id];
            float cv = axis == 0 ? c.x : (axis == 1 ? c.y : c.z);
            goes_left = bin_of(cv, plo, pscale) <= split;
        }
        unsigned ballot = __ballot_sync(0xffffffffu, goes_left);
        uint32_t in_warp = __popc(ballot & ((1u << lane) - 1u));
        if (lane == 31) s_scan[warp] = __popc(ballot);
        __syncthreads();
        if (t == 0) {
            uint32_t acc = 0;
            for (uint32_t w = 0; w < CTA / 32; w++) {
                uint32_t v = s_scan[w];
                s_scan[w] = acc;
                acc += v;
            }
            s_scan[CTA / 32] = acc;
        }
        __syncthreads();
        uint32_t lefts_before = s_scan[warp] + in_warp;
        uint32_t chunk_left = s_scan[CTA / 32];
        uint32_t base_l = s_base_left, base_r = s_base_right;
        if (valid) {
            if (goes_left) ids_next[jb.begin + base_l + lefts_before] = id;
            else ids_next[jb.begin + left_total + base_r + (t - lefts_before)] = id;
        }
        __syncthreads();
        if (t == 0) {
            uint32_t n_in_chunk = min(CTA, jb.end - c0);
            s_base_left = base_l + chunk_left;
            s_base_right = base_r + (n_in_chunk - chunk_left);
        }
        __syncthreads();
    }
    if (t == 0) {
        uint32_t mid = jb.begin + left_total;
        if (mid == jb.begin || mid == jb.end) dec[j].mid = jb.begin + count / 2;
        else dec[j].mid = mid;
    }
}

// One warp per node of SMALL_MAX < count <= LARGE triangles (nodes from
// `list`): bounds by warp shuffles, bins in the warp's shared memory (int
// keys, so any order gives the host's bits), the three axis sweeps on lanes
// 0-2 combined in axis order as sah() does, and a stable partition 32 ids
// at a time by ballot.
__global__ void __launch_bounds__(WN * 32) decide_warp(const Job* jobs, const uint32_t* list, uint32_t M, Tri tr,
                                                       const uint32_t* ids, uint32_t* ids_next, Decision* dec) {
    __shared__ int s_lo[WN][3][BINS][3], s_hi[WN][3][BINS][3];
    __shared__ uint32_t s_bc[WN][3][BINS];
    const uint32_t w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t li = blockIdx.x * WN + w;
    if (li >= M) return;  // whole warps
    const uint32_t FULL = 0xffffffffu;
    const uint32_t j = list[li];
    const Job jb = jobs[j];
    const uint32_t count = jb.end - jb.begin;
    float v[12];
    for (int k = 0; k < 12; k++) v[k] = (k % 6) < 3 ? FLT_MAX : -FLT_MAX;
    for (uint32_t i = jb.begin + lane; i < jb.end; i += 32) {
        uint32_t id = ids[i];
        float4 a = tr.blo[id], b = tr.bhi[id], c = tr.cen[id];
        v[0] = fminf(v[0], a.x); v[1] = fminf(v[1], a.y); v[2] = fminf(v[2], a.z);
        v[3] = fmaxf(v[3], b.x); v[4] = fmaxf(v[4], b.y); v[5] = fmaxf(v[5], b.z);
        v[6] = fminf(v[6], c.x); v[7] = fminf(v[7], c.y); v[8] = fminf(v[8], c.z);
        v[9] = fmaxf(v[9], c.x); v[10] = fmaxf(v[10], c.y); v[11] = fmaxf(v[11], c.z);
    }
    for (int off = 16; off; off >>= 1)
        for (int k = 0; k < 12; k++) {
            float o = __shfl_xor_sync(FULL, v[k], off);
            v[k] = (k % 6) < 3 ? fminf(v[k], o) : fmaxf(v[k], o);
        }
    const float lo[3] = {v[0], v[1], v[2]}, hi[3] = {v[3], v[4], v[5]};
    const float clo[3] = {v[6], v[7], v[8]}, chi[3] = {v[9], v[10], v[11]};
    for (uint32_t x = lane; x < 3 * BINS; x += 32) {
        int a = x / BINS, b = x % BINS;
        s_bc[w][a][b] = 0;
        for (int k = 0; k < 3; k++) {
            s_lo[w][a][b][k] = fkey(FLT_MAX);
            s_hi[w][a][b][k] = fkey(-FLT_MAX);
        }
    }
    __syncwarp();
    for (uint32_t i = jb.begin + lane; i < jb.end; i += 32) {
        uint32_t id = ids[i];
        float4 c = tr.cen[id], x = tr.blo[id], y = tr.bhi[id];
        const float cv[3] = {c.x, c.y, c.z};
        for (int a = 0; a < 3; a++) {
            if (!(chi[a] > clo[a])) continue;
            float scale = BINS / (chi[a] - clo[a]);
            int b = bin_of(cv[a], clo[a], scale);
            atomicAdd(&s_bc[w][a][b], 1u);
            atomicMin(&s_lo[w][a][b][0], fkey(x.x));
            atomicMin(&s_lo[w][a][b][1], fkey(x.y));
            atomicMin(&s_lo[w][a][b][2], fkey(x.z));
            atomicMax(&s_hi[w][a][b][0], fkey(y.x));
            atomicMax(&s_hi[w][a][b][1], fkey(y.y));
            atomicMax(&s_hi[w][a][b][2], fkey(y.z));
        }
    }
    __syncwarp();
    float cost = FLT_MAX;
    int sp = -1;
    if (lane < 3 && chi[lane] > clo[lane]) {
        const int a = (int)lane;
        axis_sweep([&](int b, int k) { return funkey(s_lo[w][a][b][k]); },
                   [&](int b, int k) { return funkey(s_hi[w][a][b][k]); }, [&](int b) { return s_bc[w][a][b]; },
                   &cost, &sp);
    }
    float best_cost = FLT_MAX;
    int best_axis = -1, best_split = -1;
    for (int a = 0; a < 3; a++) {
        float c = __shfl_sync(FULL, cost, a);
        int b = __shfl_sync(FULL, sp, a);
        if (b >= 0 && c < best_cost) {
            best_cost = c;
            best_axis = a;
            best_split = b;
        }
    }
    Decision d;
    d.mid = jb.begin;
    d.pad0 = d.pad1 = 0;
    int axis = -1, split = -1;
    float plo = 0.0f, pscale = 0.0f;
    finish_decision(best_axis, best_split, best_cost, clo, chi, lo, hi, jb.begin, count, &d, &axis, &split, &plo,
                    &pscale);
    if (axis >= 0) {
        uint32_t left_total = 0;
        for (int b = 0; b <= split; b++) left_total += s_bc[w][axis][b];
        uint32_t base_l = 0, base_r = 0;
        for (uint32_t c0 = jb.begin; c0 < jb.end; c0 += 32) {
            uint32_t i = c0 + lane;
            bool valid = i < jb.end;
            uint32_t id = valid ? ids[i] : 0u;
            bool goes_left = false;
            if (valid) {
                float4 c = tr.cen[id];
                float cv = axis == 0 ? c.x : (axis == 1 ? c.y : c.z);
                goes_left = bin_of(cv, plo, pscale) <= split;
            }
            unsigned ballot = __ballot_sync(FULL, goes_left);
            uint32_t before = __popc(ballot & ((1u << lane) - 1u));
            if (valid) {
                if (goes_left) ids_next[jb.begin + base_l + before] = id;
                else ids_next[jb.begin + left_total + base_r + (lane - before)] = id;
            }
            uint32_t nl = __popc(ballot), nin = min(32u, jb.end - c0);
            base_l += nl;
            base_r += nin - nl;
        }
        uint32_t mid = jb.begin + left_total;
        d.mid = (mid == jb.begin || mid == jb.end) ? jb.begin + count / 2 : mid;
    } else {
        for (uint32_t i = jb.begin + lane; i < jb.end; i += 32) ids_next[i] = ids[i];
    }
    if (lane == 0) dec[j] = d;
}

// Nodes of more than HUGE_N triangles: CHUNK-triangle chunks, one CTA each,
// reduce into per-node accumulators (int keys and counts, so any order gives
// the host's bits); one thread per node decides; chunks count their left
// ids, a per-node scan places them, and each chunk partitions stably.
struct HugeNode {
    uint32_t job, begin, end, chunk0;  // chunk0: the node's first chunk
    int axis, split;
    float plo, pscale;
    uint32_t left_total, pad0, pad1, pad2;
};
struct HugeAcc {
    int box[12];  // lo xyz, hi xyz, clo xyz, chi xyz
    int lo[3][BINS][3], hi[3][BINS][3];
    uint32_t bc[3][BINS];
};

__global__ void huge_setup(const Job* jobs, const uint32_t* list, uint32_t H, HugeNode* hn, HugeAcc* acc,
                           uint32_t* total_chunks) {
    if (threadIdx.x == 0) {
        uint32_t c = 0;
        for (uint32_t h = 0; h < H; h++) {
            Job jb = jobs[list[h]];
            HugeNode x{};
            x.job = list[h];
            x.begin = jb.begin;
            x.end = jb.end;
            x.chunk0 = c;
            x.axis = -1;
            hn[h] = x;
            c += (jb.end - jb.begin + CHUNK - 1) / CHUNK;
        }
        *total_chunks = c;
    }
    const uint32_t per = sizeof(HugeAcc) / 4;
    for (uint32_t x = threadIdx.x; x < H * per; x += blockDim.x) {
        uint32_t h = x / per, k = x % per;
        int* a = reinterpret_cast<int*>(&acc[h]);
        int val;
        if (k < 12) val = (k % 6) < 3 ? fkey(FLT_MAX) : fkey(-FLT_MAX);
        else if (k < 12 + 3 * BINS * 3) val = fkey(FLT_MAX);
        else if (k < 12 + 6 * BINS * 3) val = fkey(-FLT_MAX);
        else val = 0;
        a[k] = val;
    }
}

// The node and triangle range of chunk c (false: past the last chunk).
__device__ bool huge_chunk(const HugeNode* hn, uint32_t H, uint32_t total, uint32_t c, uint32_t* h_out, uint32_t* i0,
                           uint32_t* i1) {
    if (c >= total) return false;
    uint32_t lo = 0, hi = H;
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (hn[mid].chunk0 <= c) lo = mid;
        else hi = mid;
    }
    *h_out = lo;
    *i0 = hn[lo].begin + (c - hn[lo].chunk0) * CHUNK;
    *i1 = min(hn[lo].end, *i0 + CHUNK);
    return true;
}

__global__ void __launch_bounds__(CTA) huge_bounds(const HugeNode* hn, uint32_t H, const uint32_t* total_chunks, Tri tr,
                                                   const uint32_t* ids, HugeAcc* acc) {
    __shared__ int s_box[12];
    uint32_t h, i0, i1;
    if (!huge_chunk(hn, H, *total_chunks, blockIdx.x, &h, &i0, &i1)) return;
    const uint32_t t = threadIdx.x;
    if (t < 12) s_box[t] = (t % 6) < 3 ? fkey(FLT_MAX) : fkey(-FLT_MAX);
    __syncthreads();
    float v[12];
    for (int k = 0; k < 12; k++) v[k] = (k % 6) < 3 ? FLT_MAX : -FLT_MAX;
    for (uint32_t i = i0 + t; i < i1; i += CTA) {
        uint32_t id = ids[i];
        float4 a = tr.blo[id], b = tr.bhi[id], c = tr.cen[id];
        v[0] = fminf(v[0], a.x); v[1] = fminf(v[1], a.y); v[2] = fminf(v[2], a.z);
        v[3] = fmaxf(v[3], b.x); v[4] = fmaxf(v[4], b.y); v[5] = fmaxf(v[5], b.z);
        v[6] = fminf(v[6], c.x); v[7] = fminf(v[7], c.y); v[8] = fminf(v[8], c.z);
        v[9] = fmaxf(v[9], c.x); v[10] = fmaxf(v[10], c.y); v[11] = fmaxf(v[11], c.z);
    }
    for (int off = 16; off; off >>= 1)
        for (int k = 0; k < 12; k++) {
            float o = __shfl_xor_sync(0xffffffffu, v[k], off);
            v[k] = (k % 6) < 3 ? fminf(v[k], o) : fmaxf(v[k], o);
        }
    if ((t & 31) == 0)
        for (int k = 0; k < 12; k++) {
            if ((k % 6) < 3) atomicMin(&s_box[k], fkey(v[k]));
            else atomicMax(&s_box[k], fkey(v[k]));
        }
    __syncthreads();
    if (t < 12) {
        if ((t % 6) < 3) atomicMin(&acc[h].box[t], s_box[t]);
        else atomicMax(&acc[h].box[t], s_box[t]);
    }
}

__global__ void __launch_bounds__(CTA) huge_bins(const HugeNode* hn, uint32_t H, const uint32_t* total_chunks, Tri tr,
                                                 const uint32_t* ids, HugeAcc* acc) {
    __shared__ int s_lo[3][BINS][3], s_hi[3][BINS][3];
    __shared__ uint32_t s_bc[3][BINS];
    uint32_t h, i0, i1;
    if (!huge_chunk(hn, H, *total_chunks, blockIdx.x, &h, &i0, &i1)) return;
    const uint32_t t = threadIdx.x;
    for (uint32_t x = t; x < 3 * BINS; x += CTA) {
        int a = x / BINS, b = x % BINS;
        s_bc[a][b] = 0;
        for (int k = 0; k < 3; k++) {
            s_lo[a][b][k] = fkey(FLT_MAX);
            s_hi[a][b][k] = fkey(-FLT_MAX);
        }
    }
    float clo[3], chi[3];
    for (int k = 0; k < 3; k++) {
        clo[k] = funkey(acc[h].box[6 + k]);
        chi[k] = funkey(acc[h].box[9 + k]);
    }
    __syncthreads();
    for (uint32_t i = i0 + t; i < i1; i += CTA) {
        uint32_t id = ids[i];
        float4 c = tr.cen[id], x = tr.blo[id], y = tr.bhi[id];
        const float cv[3] = {c.x, c.y, c.z};
        for (int a = 0; a < 3; a++) {
            if (!(chi[a] > clo[a])) continue;
            float scale = BINS / (chi[a] - clo[a]);
            int b = bin_of(cv[a], clo[a], scale);
            atomicAdd(&s_bc[a][b], 1u);
            atomicMin(&s_lo[a][b][0], fkey(x.x));
            atomicMin(&s_lo[a][b][1], fkey(x.y));
            atomicMin(&s_lo[a][b][2], fkey(x.z));
            atomicMax(&s_hi[a][b][0], fkey(y.x));
            atomicMax(&s_hi[a][b][1], fkey(y.y));
            atomicMax(&s_hi[a][b][2], fkey(y.z));
        }
    }
    __syncthreads();
    for (uint32_t x = t; x < 3 * BINS; x += CTA) {
        int a = x / BINS, b = x % BINS;
        if (!s_bc[a][b]) continue;
        atomicAdd(&acc[h].bc[a][b], s_bc[a][b]);
        for (int k = 0; k < 3; k++) {
            atomicMin(&acc[h].lo[a][b][k], s_lo[a][b][k]);
            atomicMax(&acc[h].hi[a][b][k], s_hi[a][b][k]);
        }
    }
}

__global__ void huge_decide(HugeNode* hn, uint32_t H, const HugeAcc* acc, Decision* dec) {
    uint32_t h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= H) return;
    HugeNode x = hn[h];
    const HugeAcc& A = acc[h];
    float lo[3], hi[3], clo[3], chi[3];
    for (int k = 0; k < 3; k++) {
        lo[k] = funkey(A.box[k]);
        hi[k] = funkey(A.box[3 + k]);
        clo[k] = funkey(A.box[6 + k]);
        chi[k] = funkey(A.box[9 + k]);
    }
    float blo[3][BINS][3], bhi[3][BINS][3];
    uint32_t bc[3][BINS];
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < BINS; b++) {
            bc[a][b] = A.bc[a][b];
            for (int k = 0; k < 3; k++) {
                blo[a][b][k] = funkey(A.lo[a][b][k]);
                bhi[a][b][k] = funkey(A.hi[a][b][k]);
            }
        }
    const uint32_t count = x.end - x.begin;
    Decision d;
    d.mid = x.begin;
    d.pad0 = d.pad1 = 0;
    int axis = -1, split = -1;
    float plo = 0.0f, pscale = 0.0f;
    sah(blo, bhi, bc, clo, chi, lo, hi, x.begin, count, &d, &axis, &split, &plo, &pscale);
    uint32_t left = 0;
    if (axis >= 0) {
        for (int b = 0; b <= split; b++) left += bc[axis][b];
        uint32_t mid = x.begin + left;
        d.mid = (mid == x.begin || mid == x.end) ? x.begin + count / 2 : mid;
    }
    dec[x.job] = d;
    hn[h].axis = axis;
    hn[h].split = split;
    hn[h].plo = plo;
    hn[h].pscale = pscale;
    hn[h].left_total = left;
}

__device__ __forceinline__ bool huge_goes_left(const HugeNode& x, Tri tr, uint32_t id) {
    float4 c = tr.cen[id];
    float cv = x.axis == 0 ? c.x : (x.axis == 1 ? c.y : c.z);
    return bin_of(cv, x.plo, x.pscale) <= x.split;
}

__global__ void __launch_bounds__(CTA) huge_count(const HugeNode* hn, uint32_t H, const uint32_t* total_chunks, Tri tr,
                                                  const uint32_t* ids, uint32_t* chunk_left) {
    __shared__ uint32_t s_n;
    uint32_t h, i0, i1;
    if (!huge_chunk(hn, H, *total_chunks, blockIdx.x, &h, &i0, &i1)) return;
    const HugeNode x = hn[h];
    if (threadIdx.x == 0) s_n = 0;
    __syncthreads();
    uint32_t n = 0;
    if (x.axis >= 0)
        for (uint32_t i = i0 + threadIdx.x; i < i1; i += CTA) n += huge_goes_left(x, tr, ids[i]) ? 1u : 0u;
    for (int off = 16; off; off >>= 1) n += __shfl_xor_sync(0xffffffffu, n, off);
    if ((threadIdx.x & 31) == 0) atomicAdd(&s_n, n);
    __syncthreads();
    if (threadIdx.x == 0) chunk_left[blockIdx.x] = s_n;
}

// Per node, the exclusive scan of its chunks' left counts (in place).
__global__ void huge_scan(const HugeNode* hn, uint32_t H, uint32_t* chunk_left) {
    uint32_t h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= H) return;
    const HugeNode x = hn[h];
    uint32_t chunks = (x.end - x.begin + CHUNK - 1) / CHUNK, acc = 0;
    for (uint32_t c = 0; c < chunks; c++) {
        uint32_t v = chunk_left[x.chunk0 + c];
        chunk_left[x.chunk0 + c] = acc;
        acc += v;
    }
}

__global__ void __launch_bounds__(CTA) huge_scatter(const HugeNode* hn, uint32_t H, const uint32_t* total_chunks,
                                                    Tri tr, const uint32_t* ids, uint32_t* ids_next,
                                                    const uint32_t* chunk_left) {
    __shared__ uint32_t s_scan[CTA / 32 + 1];
    uint32_t h, i0, i1;
    if (!huge_chunk(hn, H, *total_chunks, blockIdx.x, &h, &i0, &i1)) return;
    const HugeNode x = hn[h];
    const uint32_t t = threadIdx.x, lane = t & 31, warp = t >> 5;
    if (x.axis < 0) {
        for (uint32_t i = i0 + t; i < i1; i += CTA) ids_next[i] = ids[i];
        return;
    }
    const uint32_t lefts_before_chunk = chunk_left[blockIdx.x];
    uint32_t base_l = x.begin + lefts_before_chunk;
    uint32_t base_r = x.begin + x.left_total + ((i0 - x.begin) - lefts_before_chunk);
    for (uint32_t c0 = i0; c0 < i1; c0 += CTA) {
        uint32_t i = c0 + t;
        bool valid = i < i1;
        uint32_t id = valid ? ids[i] : 0u;
        bool goes_left = valid && huge_goes_left(x, tr, id);
        unsigned ballot = __ballot_sync(0xffffffffu, goes_left);
        uint32_t in_warp = __popc(ballot & ((1u << lane) - 1u));
        if (lane == 31) s_scan[warp] = __popc(ballot);
        __syncthreads();
        if (t == 0) {
            uint32_t acc = 0;
            for (uint32_t w = 0; w < CTA / 32; w++) {
                uint32_t v = s_scan[w];
                s_scan[w] = acc;
                acc += v;
            }
            s_scan[CTA / 32] = acc;
        }
        __syncthreads();
        uint32_t lefts_before = s_scan[warp] + in_warp;
        uint32_t chunk_lefts = s_scan[CTA / 32];
        if (valid) {
            if (goes_left) ids_next[base_l + lefts_before] = id;
            else ids_next[base_r + (t - lefts_before)] = id;
        }
        uint32_t n_in = min(CTA, i1 - c0);
        base_l += chunk_lefts;
        base_r += n_in - chunk_lefts;
        __syncthreads();
    }
}

// Exclusive scan of the split flags: per-block scans, then block offsets.
__global__ void scan_blocks(const Decision* dec, uint32_t K, uint32_t* excl, uint32_t* block_sums) {
    __shared__ uint32_t s[1024];
    uint32_t i = blockIdx.x * 1024 + threadIdx.x;
    uint32_t v = i < K ? dec[i].split : 0u;
    s[threadIdx.x] = v;
    __syncthreads();
    for (uint32_t off = 1; off < 1024; off <<= 1) {
        uint32_t x = threadIdx.x >= off ? s[threadIdx.x - off] : 0u;
        __syncthreads();
        s[threadIdx.x] += x;
        __syncthreads();
    }
    if (i < K) excl[i] = s[threadIdx.x] - v;
    if (threadIdx.x == 1023) block_sums[blockIdx.x] = s[1023];
}

__global__ void scan_sums(uint32_t* block_sums, uint32_t nb, uint32_t* total) {
    __shared__ uint32_t s[1024];
    uint32_t v = threadIdx.x < nb ? block_sums[threadIdx.x] : 0u;
    s[threadIdx.x] = v;
    __syncthreads();
    for (uint32_t off = 1; off < 1024; off <<= 1) {
        uint32_t x = threadIdx.x >= off ? s[threadIdx.x - off] : 0u;
        __syncthreads();
        s[threadIdx.x] += x;
        __syncthreads();
    }
    if (threadIdx.x < nb) block_sums[threadIdx.x] = s[threadIdx.x] - v;
    if (threadIdx.x == 1023) *total = s[1023];
}

// Class lists of the next level's nodes (by triangle count); index order
// within a list does not matter, every node is decided on its own.
struct Lists {
    uint32_t *medium, *large, *huge;
    uint32_t* counts;  // medium, large, huge
};

__device__ __forceinline__ void classify(const Lists& l, uint32_t idx, uint32_t count) {
    if (count > HUGE_N) l.huge[atomicAdd(&l.counts[2], 1u)] = idx;
    else if (count > LARGE) l.large[atomicAdd(&l.counts[1], 1u)] = idx;
    else if (count > SMALL_MAX) l.medium[atomicAdd(&l.counts[0], 1u)] = idx;
}

// Wide levels (more than 1024 blocks of 1024): the block sums are scanned
// in place by blocks of 1024 as well, and those blocks' offsets added back.
__global__ void scan_u32(uint32_t* v, uint32_t K, uint32_t* block_sums) {
    __shared__ uint32_t s[1024];
    uint32_t i = blockIdx.x * 1024 + threadIdx.x;
    uint32_t x = i < K ? v[i] : 0u;
    s[threadIdx.x] = x;
    __syncthreads();
    for (uint32_t off = 1; off < 1024; off <<= 1) {
        uint32_t y = threadIdx.x >= off ? s[threadIdx.x - off] : 0u;
        __syncthreads();
        s[threadIdx.x] += y;
        __syncthreads();
    }
    if (i < K) v[i] = s[threadIdx.x] - x;
    if (threadIdx.x == 1023) block_sums[blockIdx.x] = s[1023];
}

__global__ void add_offsets(uint32_t* v, uint32_t K, const uint32_t* offs) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < K) v[i] += offs[i / 1024];
}

__global__ void emit(const Job* jobs, uint32_t K, const Decision* dec, const uint32_t* excl, const uint32_t* block_sums,
                     uint32_t nodes_before, uint32_t* words, Job* next, Lists lists) {
    uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= K) return;
    Job jb = jobs[j];
    Decision d = dec[j];
    uint32_t* w = words + (size_t)jb.node * 8;
    for (int k = 0; k < 3; k++) {
        w[k] = __float_as_uint(d.lo[k]);
        w[4 + k] = __float_as_uint(d.hi[k]);
    }
    if (!d.split) {
        w[3] = jb.begin;
        w[7] = jb.end - jb.begin;
        return;
    }
    uint32_t e = excl[j] + block_sums[j / 1024];
    uint32_t first = nodes_before + 2 * e;
    w[3] = first;
    w[7] = 0;
    next[2 * e] = Job{first, jb.begin, d.mid, 0};
    next[2 * e + 1] = Job{first + 1, d.mid, jb.end, 0};
    classify(lists, 2 * e, d.mid - jb.begin);
    classify(lists, 2 * e + 1, jb.end - d.mid);
}

}  // namespace bvhb
}  // namespace oxd

namespace oxd {
namespace bvhb {

#define BK(expr)                                                         \
    do {                                                                 \
        cudaError_t e_ = (expr);                                         \
        if (e_ != cudaSuccess) {                                         \
            if (err) *err = std::string("bvh build: ") + cudaGetErrorString(e_); \
            ok = false;                                                  \
            goto done;                                                   \
        }                                                                \
    } while (0)

bool build_on_device(const float* pos, uint32_t n, cudaStream_t st, uint32_t** words_out, uint32_t** slots_out,
                     uint32_t* nodes_out, uint32_t* depth_out, uint32_t* launches_out, std::string* err) {
    *words_out = *slots_out = nullptr;
    *nodes_out = *depth_out = 0;
    if (launches_out) *launches_out = 0;
    if (n == 0) return true;
    if (n > (1u << 30)) {
        if (err) *err = "bvh build: too many triangles";
        return false;
    }
    bool ok = true;
    float4 *blo = nullptr, *bhi = nullptr, *cen = nullptr;
    uint32_t *ids = nullptr, *ids2 = nullptr, *words = nullptr, *excl = nullptr, *sums = nullptr, *ctr = nullptr;
    uint32_t* sums2 = nullptr;  // block offsets of the block sums (levels wider than 1024 x 1024)
    uint32_t *l_medium = nullptr, *l_large = nullptr, *l_huge = nullptr, *chunk_left = nullptr, *total_chunks = nullptr;
    HugeNode* hn = nullptr;
    HugeAcc* acc = nullptr;
    uint32_t hctr[4] = {0, 0, 0, 0};  // pageable: the copy completes before the sync returns
    Job *jobs = nullptr, *next = nullptr;
    Decision* dec = nullptr;
    const size_t max_nodes = 2 * (size_t)n;
    const size_t max_jobs = (size_t)n;  // nodes of one level
    const size_t max_large = n / LARGE + 2, max_huge = n / HUGE_N + 2, max_chunks = n / CHUNK + max_huge + 1;
    uint32_t K = 1, nodes = 1, levels = 0, launches = 0;
    uint32_t M = 0, Lg = 0, H = 0;  // this level's medium / large / huge nodes
    BK(cudaMallocAsync((void**)&blo, (size_t)n * 16, st));
    BK(cudaMallocAsync((void**)&bhi, (size_t)n * 16, st));
    BK(cudaMallocAsync((void**)&cen, (size_t)n * 16, st));
    BK(cudaMallocAsync((void**)&ids, (size_t)n * 4, st));
    BK(cudaMallocAsync((void**)&ids2, (size_t)n * 4, st));
    BK(cudaMallocAsync((void**)&words, max_nodes * 32, st));
    BK(cudaMallocAsync((void**)&jobs, max_jobs * sizeof(Job), st));
    BK(cudaMallocAsync((void**)&next, max_jobs * sizeof(Job), st));
    BK(cudaMallocAsync((void**)&dec, max_jobs * sizeof(Decision), st));
    BK(cudaMallocAsync((void**)&excl, max_jobs * 4, st));
    BK(cudaMallocAsync((void**)&sums, ((max_jobs + 1023) / 1024) * 4, st));
    BK(cudaMallocAsync((void**)&sums2, 1024 * 4, st));
    BK(cudaMallocAsync((void**)&ctr, 4 * 4, st));
    BK(cudaMallocAsync((void**)&l_medium, max_jobs * 4, st));
    BK(cudaMallocAsync((void**)&l_large, max_large * 4, st));
    BK(cudaMallocAsync((void**)&l_huge, max_huge * 4, st));
    BK(cudaMallocAsync((void**)&hn, max_huge * sizeof(HugeNode), st));
    BK(cudaMallocAsync((void**)&acc, max_huge * sizeof(HugeAcc), st));
    BK(cudaMallocAsync((void**)&chunk_left, max_chunks * 4, st));
    BK(cudaMallocAsync((void**)&total_chunks, 4, st));
    tri_prep<<<(n + 255) / 256, 256, 0, st>>>(pos, n, blo, bhi, cen, ids);
    BK(cudaGetLastError());
    launches++;
    {
        Job root{0, 0, n, 0};
        BK(cudaMemcpyAsync(jobs, &root, sizeof(Job), cudaMemcpyHostToDevice, st));
        // The root's class list holds job 0.
        if (n > HUGE_N) H = 1;
        else if (n > LARGE) Lg = 1;
        else if (n > SMALL_MAX) M = 1;
        uint32_t* l = H ? l_huge : (Lg ? l_large : l_medium);
        BK(cudaMemsetAsync(l, 0, 4, st));
    }
    while (K > 0) {
        levels++;
        Tri tr{blo, bhi, cen};
        decide_small<<<(K + 127) / 128, 128, 0, st>>>(jobs, K, tr, ids, ids2, dec);
        BK(cudaGetLastError());
        launches++;
        if (M) {
            decide_warp<<<(M + WN - 1) / WN, WN * 32, 0, st>>>(jobs, l_medium, M, tr, ids, ids2, dec);
            BK(cudaGetLastError());
            launches++;
        }
        if (Lg) {
            decide_large<<<Lg, CTA, 0, st>>>(jobs, l_large, Lg, tr, ids, ids2, dec);
            BK(cudaGetLastError());
            launches++;
        }
        if (H) {
            const uint32_t grid = (uint32_t)std::min<size_t>(max_chunks, (size_t)n / CHUNK + H + 1);
            huge_setup<<<1, 256, 0, st>>>(jobs, l_huge, H, hn, acc, total_chunks);
            huge_bounds<<<grid, CTA, 0, st>>>(hn, H, total_chunks, tr, ids, acc);
            huge_bins<<<grid, CTA, 0, st>>>(hn, H, total_chunks, tr, ids, acc);
            huge_decide<<<(H + 127) / 128, 128, 0, st>>>(hn, H, acc, dec);
            huge_count<<<grid, CTA, 0, st>>>(hn, H, total_chunks, tr, ids, chunk_left);
            huge_scan<<<(H + 127) / 128, 128, 0, st>>>(hn, H, chunk_left);
            huge_scatter<<<grid, CTA, 0, st>>>(hn, H, total_chunks, tr, ids, ids2, chunk_left);
            BK(cudaGetLastError());
            launches += 7;
        }
        uint32_t nb = (K + 1023) / 1024;
        scan_blocks<<<nb, 1024, 0, st>>>(dec, K, excl, sums);
        BK(cudaGetLastError());
        if (nb <= 1024) {
            scan_sums<<<1, 1024, 0, st>>>(sums, nb, ctr);
        } else {  // K <= n <= 2^30, so nb <= 2^20 and one more level suffices
            uint32_t nb2 = (nb + 1023) / 1024;
            scan_u32<<<nb2, 1024, 0, st>>>(sums, nb, sums2);
            scan_sums<<<1, 1024, 0, st>>>(sums2, nb2, ctr);
            add_offsets<<<(nb + 255) / 256, 256, 0, st>>>(sums, nb, sums2);
            launches += 3;
        }
        BK(cudaGetLastError());
        BK(cudaMemsetAsync(ctr + 1, 0, 12, st));
        emit<<<(K + 127) / 128, 128, 0, st>>>(jobs, K, dec, excl, sums, nodes, words, next,
                                              Lists{l_medium, l_large, l_huge, ctr + 1});
        BK(cudaGetLastError());
        launches += 3;
        BK(cudaMemcpyAsync(hctr, ctr, 16, cudaMemcpyDeviceToHost, st));
        BK(cudaStreamSynchronize(st));
        nodes += 2 * hctr[0];
        K = 2 * hctr[0];
        M = hctr[1];
        Lg = hctr[2];
        H = hctr[3];
        std::swap(jobs, next);
        std::swap(ids, ids2);
    }
    *words_out = words;
    *slots_out = ids;
    words = ids = nullptr;
    *nodes_out = nodes;
    *depth_out = levels;
    if (launches_out) *launches_out = launches;
done:
    void* ptrs[] = {blo, bhi, cen, ids, ids2, words, excl, sums, sums2, ctr, jobs, next, dec,
                    l_medium, l_large, l_huge, hn, acc, chunk_left, total_chunks};
    for (void* p : ptrs)
        if (p) cudaFreeAsync(p, st);  // stream-ordered: no device-wide synchronisation
    if (!ok) cudaStreamSynchronize(st);
    return ok;
}

}  // namespace bvhb
}  // namespace oxd

namespace oxpt {

bool build_bvh_device(int device, const std::vector<float>& tri_pos, BvhBuild* out, std::string* err) {
    const uint32_t n = (uint32_t)(tri_pos.size() / 9);
    *out = BvhBuild{};
    if (n == 0) return true;
    bool ok = true;
    float* pos = nullptr;
    uint32_t *words = nullptr, *slots = nullptr, nodes = 0, depth = 0;
    cudaStream_t st = nullptr;
    BK(cudaSetDevice(device));
    BK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    BK(cudaMalloc((void**)&pos, tri_pos.size() * 4));
    BK(cudaMemcpyAsync(pos, tri_pos.data(), tri_pos.size() * 4, cudaMemcpyHostToDevice, st));
    if (!oxd::bvhb::build_on_device(pos, n, st, &words, &slots, &nodes, &depth, nullptr, err)) {
        ok = false;
        goto done;
    }
    out->node_words.resize((size_t)nodes * 8);
    out->slots.resize(n);
    BK(cudaMemcpyAsync(out->node_words.data(), words, (size_t)nodes * 32, cudaMemcpyDeviceToHost, st));
    BK(cudaMemcpyAsync(out->slots.data(), slots, (size_t)n * 4, cudaMemcpyDeviceToHost, st));
    BK(cudaStreamSynchronize(st));
    out->depth = depth;
done:
    if (st) cudaStreamSynchronize(st);
    if (pos) cudaFree(pos);
    if (words) cudaFreeAsync(words, st);
    if (slots) cudaFreeAsync(slots, st);
    if (st) {
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
    }
    if (!ok) *out = BvhBuild{};
    return ok;
}

}  // namespace oxpt

extern "C" oxpt_status oxpt_diag_bvh_build(int device, const float* tri_pos, uint32_t n, int on_gpu, uint32_t* words,
                                           uint32_t* slots, uint32_t* node_count, uint32_t* depth) {
    if ((n && !tri_pos) || !words || !slots || !node_count || !depth) return OXPT_E_INVALID;
    std::vector<float> pos(tri_pos, tri_pos + (size_t)n * 9);
    oxpt::BvhBuild b;
    if (on_gpu) {
        std::string e;
        if (!oxpt::build_bvh_device(device, pos, &b, &e)) return OXPT_E_CUDA;
    } else {
        b = oxpt::build_bvh(pos);
    }
    std::copy(b.node_words.begin(), b.node_words.end(), words);
    std::copy(b.slots.begin(), b.slots.end(), slots);
    *node_count = (uint32_t)(b.node_words.size() / 8);
    *depth = b.depth;
    return OXPT_OK;
}
