// Path-tracing kernels for sm_100a.
//
// trace_paths: a persistent megakernel. The grid is sized to the resident
// capacity of the GPU; each thread owns one path slot and, whenever its
// path ends, regenerates the slot with its next (pixel, sample) item
// (grid-stride over samples-major, pixels-minor items, so that the lanes
// of a warp start on neighbouring pixels of the same sample). Every loop
// iteration traces exactly one ray — the path's continuation ray or one
// NEE shadow ray — through a single traversal call site, as the reference
// megakernel does (pathtrace.wgsl:1702-2045), so lanes that are shading,
// shadowing or starting a new camera ray all meet at the same traversal.
// The result of every path is written to a per-launch buffer and
// reduce_frame then adds them into the accumulator in sample order,
// which keeps each pixel's float summation identical to the reference's
// per-pixel loop (pathtrace.wgsl:2064-2072) whatever the launch split.
//
// Traversal (traverse.cuh) is shared with the wavefront kernels.
#include "kernels.cuh"
#include "shade.cuh"
#include "traverse.cuh"
#include "walk.cuh"
#include "path.cuh"

namespace oxd {

template <bool COUNT>
__global__ void __launch_bounds__(TRACE_THREADS) trace_paths(const __grid_constant__ TraceArgs a) {
    __shared__ uint32_t s_sobol[128];
    __shared__ float s_sheen[512];
    const Scene& s = a.s;
    for (uint32_t i = threadIdx.x; i < 128u; i += blockDim.x) s_sobol[i] = tw(s, s.P.offs0[0] + i);
    for (uint32_t i = threadIdx.x; i < 512u; i += blockDim.x) s_sheen[i] = tf(s, s.P.offs0[1] + i);
    __syncthreads();

    Cnt cnt;
    if (COUNT)
        for (int k = 0; k < C_N; k++) cnt.c[k] = 0;
    const uint32_t W = s.P.dims[0];
    const uint32_t n_punct = s.P.cfg[2];
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;

    uint64_t item = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    bool live = false, shadow = false;
    Sampler smp{0u, 0u, 0u};
    PathCore pc;
    Vertex v;
    uint32_t job = 0u, r_id = 0u, r_skip = NONE;
    f3 r_o = sp(0.0f), r_d = sp(0.0f), pending = sp(0.0f);
    float r_tmax = INF;

    for (;;) {
        if (!live) {
            if (item >= a.total) break;
            uint32_t i = (uint32_t)(item / a.npix);
            uint32_t q = (uint32_t)(item - (uint64_t)i * a.npix);
            uint32_t yy = q / W;
            r_o = start_path(s, s_sobol, q - yy * W, a.y0 + yy, a.first + i, &smp, &pc);
            r_d = pc.d;
            r_tmax = INF;
            r_id = 0u;
            r_skip = NONE;
            shadow = false;
            live = true;
            bump<COUNT>(cnt, C_PATHS);
        }
        bump<COUNT>(cnt, shadow ? C_SHADOW_RAYS : C_PATH_RAYS);
        Hit hit;
        uint32_t hmat = 0u;
        bool got = traverse<COUNT>(s, make_ray(r_o, r_d), r_tmax, smp, r_id, !shadow && pc.k == 0u, shadow, r_skip,
                                   &hit, &hmat, cnt, a.err);
        int outcome = PATH_VERTEX;
        if (shadow) {
            if (!got) pc.radiance = pc.radiance + pending;
            job += 1u;
        } else {
            outcome = on_path_hit<COUNT>(s, s_sheen, s_sobol, smp, pc, got, hit, hmat, &v, &cnt.c[C_SHADED]);
            job = 0u;
        }
        if (outcome == PATH_VERTEX) {
            bool armed = false;
            for (; job <= n_punct; job++) {
                ShadowRay sr;
                if (nee_job(s, s_sheen, pc, v, job, &sr)) {
                    pending = sr.pending;
                    r_o = sr.o;
                    r_d = sr.d;
                    r_tmax = sr.tmax;
                    r_id = sr.rid;
                    r_skip = sr.skip;
                    armed = true;
                    break;
                }
            }
            if (armed) {
                shadow = true;
                continue;
            }
            if (continue_path(s, s_sheen, s_sobol, smp, pc, v, &r_o)) {
                shadow = false;
                r_d = pc.d;
                r_tmax = INF;
                r_id = pc.k << 16u;
                r_skip = NONE;
                continue;
            }
            outcome = PATH_DONE;
        }
        a.out[item] = path_result(pc, outcome != PATH_UNCOVERED);
        item += stride;
        live = false;
    }
    if (COUNT) {
        for (int c = 0; c < C_N; c++) {
            unsigned long long x = cnt.c[c];
            for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
            if ((threadIdx.x & 31u) == 0u && x) atomicAdd(a.counters + c, x);
        }
    }
}

// Ordered accumulation: samples of one launch added to each pixel in
// sample order (pathtrace.wgsl:2065-2072).
__global__ void reduce_frame(const ReduceArgs a) {
    uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= a.npix) return;
    uint64_t idx = (uint64_t)a.y0 * a.w + q;
    float4 acc = a.accum[idx];
    for (uint32_t i = 0; i < a.count; i++) {
        float4 r = __ldcs(a.out + (uint64_t)i * a.npix + q);
        if (r.w > 0.0f) acc = make_float4(acc.x + r.x, acc.y + r.y, acc.z + r.z, acc.w + 1.0f);
    }
    a.accum[idx] = acc;
}

template <bool COUNT>
__global__ void __launch_bounds__(128) trace_rays(const __grid_constant__ RayArgs a) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    Cnt cnt;
    if (COUNT)
        for (int k = 0; k < C_N; k++) cnt.c[k] = 0;
    if (i < a.n) {
        const float* r = a.rays + i * 8;
        Sampler smp{0u, 0u, 0u};
        Hit h;
        uint32_t m = 0;
        Ray ray = make_ray(mk(r[0], r[1], r[2]), mk(r[4], r[5], r[6]));
        bool primary = (a.flags & 2u) != 0u;
        bool got;
        if ((a.flags & 9u) == 8u) {
            // Closest hit over the four-wide tree (the tolerance plan's walk),
            // its whole stack in local memory.
            __shared__ uint32_t unused_columns[1];
            Walk4C<1, STACK> w;
            got = false;
            if (walk4c_begin<1, STACK>(a.s, ray, r[3], w)) {
                while (!walk4c_step<COUNT, 1, STACK, 128>(&a.s, unused_columns, 0u, ray, 0u, 0u, primary,
                                                          __float_as_uint(r[7]), w, cnt, a.err)) {
                }
            }
            got = w.hit_any;
            h = w.best;
        } else {
            got = (a.flags & 5u) == 5u
                      ? occluded4<COUNT, STACK>(a.s, ray, r[3], smp, 0u, primary, __float_as_uint(r[7]), &h, &m,
                                                cnt, a.err)
                      : traverse<COUNT>(a.s, ray, r[3], smp, 0u, primary, (a.flags & 1u) != 0u,
                                        __float_as_uint(r[7]), &h, &m, cnt, a.err);
        }
        if (a.slot) a.slot[i] = got ? h.slot : NONE;
        if (a.gid) a.gid[i] = got ? tri_word(a.s, h.slot, 0u) : NONE;
        if (a.t) a.t[i] = got ? h.t : 0.0f;
        if (a.bary) {
            a.bary[i * 3] = got ? h.b.x : 0.0f;
            a.bary[i * 3 + 1] = got ? h.b.y : 0.0f;
            a.bary[i * 3 + 2] = got ? h.b.z : 0.0f;
        }
    }
    if (COUNT)
        for (int c = 0; c < C_N; c++)
            if (cnt.c[c]) atomicAdd(a.counters + c, cnt.c[c]);
}

__global__ void sobol_points(const uint32_t* dirs, uint32_t seed, uint64_t n, const uint32_t* x, const uint32_t* y,
                             const uint32_t* idx, const uint32_t* pat, uint32_t* out) {
    __shared__ uint32_t sd[128];
    for (uint32_t i = threadIdx.x; i < 128u; i += blockDim.x) sd[i] = dirs[i];
    __syncthreads();
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Sampler smp = make_sampler(seed, x[i], y[i], idx[i]);
    uint32_t u[4];
    pattern_u(sd, smp, pat[i], u);
    reinterpret_cast<uint4*>(out)[i] = make_uint4(u[0], u[1], u[2], u[3]);
}

__global__ void math_kernel(int op, uint64_t n, const float* a, const float* b, float* out) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float x = a[i], y = b ? b[i] : 0.0f, r = 0.0f;
    switch (op) {
        case 0: r = fm_sin(x); break;
        case 1: r = fm_cos(x); break;
        case 2: r = fm_acos(x); break;
        case 3: r = fm_atan2(x, y); break;
        case 4: r = fm_exp(x); break;
        case 5: r = fm_log(x); break;
        case 6: r = fm_log2(x); break;
        case 7: r = fm_pow(x, y); break;
        default: r = 0.0f;
    }
    out[i] = r;
}

cudaError_t launch_trace(const TraceArgs& a, bool count, uint32_t blocks, uint32_t threads, cudaStream_t st) {
    if (count) trace_paths<true><<<blocks, threads, 0, st>>>(a);
    else trace_paths<false><<<blocks, threads, 0, st>>>(a);
    return cudaGetLastError();
}

int trace_blocks_per_sm(uint32_t threads, bool count) {
    int n = 0;
    if (count) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, trace_paths<true>, (int)threads, 0);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, trace_paths<false>, (int)threads, 0);
    return n;
}

cudaError_t launch_reduce(const ReduceArgs& a, cudaStream_t st) {
    uint32_t blocks = (a.npix + 255u) / 256u;
    reduce_frame<<<blocks, 256, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_rays(const RayArgs& a, cudaStream_t st) {
    if (a.n == 0) return cudaSuccess;
    uint64_t blocks = (a.n + 127) / 128;
    if (a.counters) trace_rays<true><<<(unsigned)blocks, 128, 0, st>>>(a);
    else trace_rays<false><<<(unsigned)blocks, 128, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_sobol(const uint32_t* dirs, uint32_t seed, uint64_t n, const uint32_t* x, const uint32_t* y,
                         const uint32_t* idx, const uint32_t* pat, uint32_t* out, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    sobol_points<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(dirs, seed, n, x, y, idx, pat, out);
    return cudaGetLastError();
}

cudaError_t launch_math(int op, uint64_t n, const float* a, const float* b, float* out, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    math_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(op, n, a, b, out);
    return cudaGetLastError();
}

}  // namespace oxd
