// Reordering of the ray queues before the walks.
//
// The traversal kernels hand each warp the next queue entries; the order
// of the queue decides which rays a warp walks together. A ray's walk and
// its hit do not depend on that order (each ray is walked alone by one
// lane), so any permutation of the queue gives the same results. This pass
// groups rays that start in the same region of the scene and go the same
// way, so the lanes of a warp visit the same nodes: a counting sort of the
// continuation queue's slot ids on a 15-bit key (3 bits of direction
// octant above 12 bits of a Morton code of the origin, 16 cells per axis of
// the scene's root box), and of the shadow queue's entries on a 17-bit key
// (the NEE job, i.e. the light, above the origin's Morton code), written
// as a permutation the shadow walk reads the queue through. Order within a bucket is whatever the
// atomics give; it does not matter. Device-side counts only, so the three
// kernels capture into the per-step CUDA graph.
#include "kernels.cuh"
#include "wavefront.cuh"

namespace oxd {

namespace {

constexpr uint32_t BUCKETS = 1u << 15;
constexpr uint32_t SH_BUCKETS = 1u << 17;
constexpr uint32_t SCAN_THREADS = 1024;

__device__ __forceinline__ uint32_t spread3(uint32_t v) {  // 4 bits -> every third bit
    v &= 0xfu;
    v = (v | (v << 4)) & 0x0c3u;
    v = (v | (v << 2)) & 0x249u;
    return v;
}

__device__ __forceinline__ uint32_t cell(float x, float lo, float hi) {
    float f = (x - lo) / (hi - lo);
    if (!(f > 0.0f)) return 0u;  // below, or NaN
    return f >= 1.0f ? 15u : (uint32_t)(f * 16.0f);
}

__device__ __forceinline__ uint32_t morton12(const Scene& s, float4 o) {
    const float4 lo = geomv(s, 0), hi = geomv(s, 1);
    return spread3(cell(o.x, lo.x, hi.x)) | (spread3(cell(o.y, lo.y, hi.y)) << 1) |
           (spread3(cell(o.z, lo.z, hi.z)) << 2);
}

template <bool BATCH>
__global__ void order_count(const __grid_constant__ WaveArgs a) {
    const uint32_t n = *((volatile uint32_t*)&a.ctr[0]);
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const uint32_t i = a.q.ext[q];
        const Scene& s = BATCH ? a.frames[a.st.frame[i]].s : a.s;
        const float4 o = a.st.org[i], d = a.st.dir[i];
        const uint32_t m = morton12(s, o);
        const uint32_t oct = (d.x < 0.0f ? 1u : 0u) | (d.y < 0.0f ? 2u : 0u) | (d.z < 0.0f ? 4u : 0u);
        const uint32_t key = (oct << 12) | m;
        a.q.ord_key[q] = key;
        a.q.ord_rank[q] = atomicAdd(a.q.ord_hist + key, 1u);
    }
}

template <bool BATCH>
__global__ void order_count_shadow(const __grid_constant__ WaveArgs a) {
    const uint32_t n = *((volatile uint32_t*)&a.ctr[1]);
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const uint4 m = a.q.sh_m[q];
        const Scene& s = BATCH ? a.frames[a.st.frame[m.x]].s : a.s;
        const uint32_t key = ((m.y & 31u) << 12) | morton12(s, a.q.sh_o[q]);
        a.q.ord_key[q] = key;
        a.q.ord_rank[q] = atomicAdd(a.q.ord_hist + key, 1u);
    }
}

// Exclusive prefix sums of the bucket counts, in place (one block).
template <uint32_t NB>
__global__ void __launch_bounds__(SCAN_THREADS) order_scan(uint32_t* hist) {
    __shared__ uint32_t part[SCAN_THREADS];
    constexpr uint32_t PER = NB / SCAN_THREADS;
    const uint32_t t = threadIdx.x;
    uint32_t sum = 0u;
    for (uint32_t k = 0; k < PER; k++) sum += hist[t * PER + k];
    part[t] = sum;
    __syncthreads();
    for (uint32_t off = 1; off < SCAN_THREADS; off <<= 1) {
        uint32_t v = t >= off ? part[t - off] : 0u;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    uint32_t run = t ? part[t - 1] : 0u;
    for (uint32_t k = 0; k < PER; k++) {
        uint32_t c = hist[t * PER + k];
        hist[t * PER + k] = run;
        run += c;
    }
}

__global__ void order_scatter(const __grid_constant__ WaveArgs a) {
    const uint32_t n = *((volatile uint32_t*)&a.ctr[0]);
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const uint32_t dst = a.q.ord_hist[a.q.ord_key[q]] + a.q.ord_rank[q];  // < n: the counts sum to n
        a.q.ext_sorted[dst] = a.q.ext[q];
    }
}

__global__ void order_scatter_shadow(const __grid_constant__ WaveArgs a) {
    const uint32_t n = *((volatile uint32_t*)&a.ctr[1]);
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const uint32_t dst = a.q.ord_hist[a.q.ord_key[q]] + a.q.ord_rank[q];  // < n
        a.q.sh_perm[dst] = q;
    }
}

}  // namespace

cudaError_t launch_order_ext(const WaveArgs& a, int sms, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(a.q.ord_hist, 0, BUCKETS * sizeof(uint32_t), st);
    if (e) return e;
    const unsigned grid = (unsigned)(sms > 0 ? sms * 8 : 1024);
    if (a.nframes) order_count<true><<<grid, 256, 0, st>>>(a);
    else order_count<false><<<grid, 256, 0, st>>>(a);
    if ((e = cudaGetLastError())) return e;
    order_scan<BUCKETS><<<1, SCAN_THREADS, 0, st>>>(a.q.ord_hist);
    if ((e = cudaGetLastError())) return e;
    order_scatter<<<grid, 256, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_order_shadow(const WaveArgs& a, int sms, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(a.q.ord_hist, 0, SH_BUCKETS * sizeof(uint32_t), st);
    if (e) return e;
    const unsigned grid = (unsigned)(sms > 0 ? sms * 8 : 1024);
    if (a.nframes) order_count_shadow<true><<<grid, 256, 0, st>>>(a);
    else order_count_shadow<false><<<grid, 256, 0, st>>>(a);
    if ((e = cudaGetLastError())) return e;
    order_scan<SH_BUCKETS><<<1, SCAN_THREADS, 0, st>>>(a.q.ord_hist);
    if ((e = cudaGetLastError())) return e;
    order_scatter_shadow<<<grid, 256, 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace oxd
