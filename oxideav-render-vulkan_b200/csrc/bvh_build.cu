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
constexpr uint32_t LARGE = 1024;   // nodes above this many triangles take the CTA path
constexpr uint32_t CTA = 512;

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

// The host's SAH sweep over binned boxes / counts; returns the decision.
__device__ void sah(const float (*blo)[BINS][3], const float (*bhi)[BINS][3], const uint32_t (*bc)[BINS],
                    const float* clo, const float* chi, const float* lo, const float* hi, uint32_t begin,
                    uint32_t count, Decision* d, int* axis_out, int* split_out, float* plo, float* pscale) {
    float best_cost = FLT_MAX;
    int best_axis = -1, best_split = -1;
    for (int axis = 0; axis < 3; axis++) {
        if (!(chi[axis] > clo[axis])) continue;
        float right_area[BINS];
        uint32_t right_count[BINS];
        float alo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, ahi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
        uint32_t nn = 0;
        for (int b = BINS - 1; b > 0; b--) {
            for (int k = 0; k < 3; k++) {
                alo[k] = fminf(alo[k], blo[axis][b][k]);
                ahi[k] = fmaxf(ahi[k], bhi[axis][b][k]);
            }
            nn += bc[axis][b];
            right_area[b] = area(alo, ahi);
            right_count[b] = nn;
        }
        float llo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, lhi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
        uint32_t ln = 0;
        for (int b = 0; b < BINS - 1; b++) {
            for (int k = 0; k < 3; k++) {
                llo[k] = fminf(llo[k], blo[axis][b][k]);
                lhi[k] = fmaxf(lhi[k], bhi[axis][b][k]);
            }
            ln += bc[axis][b];
            if (ln == 0 || right_count[b + 1] == 0) continue;
            float cost = area(llo, lhi) * (float)ln + right_area[b + 1] * (float)right_count[b + 1];
            if (cost < best_cost) {
                best_cost = cost;
                best_axis = axis;
                best_split = b;
            }
        }
    }
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

__global__ void decide_small(const Job* jobs, uint32_t K, Tri tr, const uint32_t* ids, uint32_t* ids_next,
                             Decision* dec) {
    uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= K) return;
    Job jb = jobs[j];
    uint32_t count = jb.end - jb.begin;
    if (count > LARGE) return;
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

__global__ void __launch_bounds__(CTA) decide_large(const Job* jobs, uint32_t K, Tri tr, const uint32_t* ids,
                                                    uint32_t* ids_next, Decision* dec) {
    const uint32_t j = blockIdx.x;
    if (j >= K) return;
    const Job jb = jobs[j];
    const uint32_t count = jb.end - jb.begin;
    if (count <= LARGE) return;
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

__global__ void emit(const Job* jobs, uint32_t K, const Decision* dec, const uint32_t* excl, const uint32_t* block_sums,
                     uint32_t nodes_before, uint32_t* words, Job* next) {
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
                     uint32_t* nodes_out, uint32_t* depth_out, std::string* err) {
    *words_out = *slots_out = nullptr;
    *nodes_out = *depth_out = 0;
    if (n == 0) return true;
    if (n > (1u << 30)) {
        if (err) *err = "bvh build: too many triangles";
        return false;
    }
    bool ok = true;
    float4 *blo = nullptr, *bhi = nullptr, *cen = nullptr;
    uint32_t *ids = nullptr, *ids2 = nullptr, *words = nullptr, *excl = nullptr, *sums = nullptr, *total = nullptr;
    uint32_t splits_host = 0;  // pageable: the copy completes before the sync returns
    Job *jobs = nullptr, *next = nullptr;
    Decision* dec = nullptr;
    const size_t max_nodes = 2 * (size_t)n;
    const size_t max_jobs = (size_t)n;  // nodes of one level
    uint32_t K = 1, nodes = 1, levels = 0;
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
    BK(cudaMallocAsync((void**)&sums, 1024 * 4, st));
    BK(cudaMallocAsync((void**)&total, 4, st));
    tri_prep<<<(n + 255) / 256, 256, 0, st>>>(pos, n, blo, bhi, cen, ids);
    BK(cudaGetLastError());
    {
        Job root{0, 0, n, 0};
        BK(cudaMemcpyAsync(jobs, &root, sizeof(Job), cudaMemcpyHostToDevice, st));
    }
    while (K > 0) {
        if (K > 1024u * 1024u) {
            if (err) *err = "bvh build: a level wider than the scan supports";
            ok = false;
            goto done;
        }
        levels++;
        Tri tr{blo, bhi, cen};
        decide_small<<<(K + 127) / 128, 128, 0, st>>>(jobs, K, tr, ids, ids2, dec);
        BK(cudaGetLastError());
        // One CTA per node; nodes of at most LARGE triangles leave at once.
        decide_large<<<K, CTA, 0, st>>>(jobs, K, tr, ids, ids2, dec);
        BK(cudaGetLastError());
        uint32_t nb = (K + 1023) / 1024;
        scan_blocks<<<nb, 1024, 0, st>>>(dec, K, excl, sums);
        BK(cudaGetLastError());
        scan_sums<<<1, 1024, 0, st>>>(sums, nb, total);
        BK(cudaGetLastError());
        emit<<<(K + 127) / 128, 128, 0, st>>>(jobs, K, dec, excl, sums, nodes, words, next);
        BK(cudaGetLastError());
        BK(cudaMemcpyAsync(&splits_host, total, 4, cudaMemcpyDeviceToHost, st));
        BK(cudaStreamSynchronize(st));
        nodes += 2 * splits_host;
        K = 2 * splits_host;
        std::swap(jobs, next);
        std::swap(ids, ids2);
    }
    *words_out = words;
    *slots_out = ids;
    words = ids = nullptr;
    *nodes_out = nodes;
    *depth_out = levels;
done:
    void* ptrs[] = {blo, bhi, cen, ids, ids2, words, excl, sums, total, jobs, next, dec};
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
    if (!oxd::bvhb::build_on_device(pos, n, st, &words, &slots, &nodes, &depth, err)) {
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
