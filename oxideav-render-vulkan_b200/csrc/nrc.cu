// Neural radiance cache: a 5-layer MLP (256 -> 64 -> 64 -> 64 -> 64 -> 3,
// ReLU, no biases) with BF16 weights and activations and FP32 accumulation
// on the fifth-generation tensor cores, trained online with Adam.
//
// The reference has no learned component; this follows the neural
// radiance cache of Mueller, Rousselle, Novak and Keller (2021, "Real-time
// neural radiance caching for path tracing"): inputs are a surface
// vertex's position (normalised to the scene bounds), outgoing direction,
// shading normal and roughness, encoded by 12 sine / cosine frequencies
// each; the loss is the relative L2 (y - t)^2 / (sg(y)^2 + 0.01).
//
// Kernels (128 samples per tile, persistent grids):
//   nrc_forward   two warpgroups per CTA on alternate tiles, each with its
//                 own operand tiles and TMEM columns, so one issues MMAs
//                 while the other encodes and activates; a warpgroup
//                 encodes a tile into shared memory, then per layer issues
//                 tcgen05.mma over the K slices (A = activations, B = the
//                 layer's weights, both resident in shared memory), waits
//                 on an mbarrier, reads the 128 x N FP32 accumulator from
//                 TMEM (one row per thread), applies ReLU and writes the
//                 next layer's BF16 operand. Inference writes predictions
//                 (or adds beta * max(prediction, 0) into path results);
//                 training also stores the hidden activations and the loss
//                 gradient.
//   nrc_backward  propagates the gradient down the layers with tcgen05
//                 (delta_{l-1} = delta_l x W_l through W_l^T, masked by
//                 ReLU) and accumulates the weight gradients a^T x delta
//                 with tcgen05 too, in TMEM across all of the CTA's tiles
//                 (512 columns: one accumulator per layer); each CTA then
//                 writes one row of partial sums and nrc_grad_reduce adds
//                 the rows in CTA order (no atomics, deterministic).
//   nrc_adam      Adam on the FP32 master weights; rewrites the BF16
//                 operand copies (forward and transposed layouts).
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "nrc.cuh"
#include "umma.cuh"

namespace oxd {
namespace nrc {

using umma::cm_offset;

// ---------------------------------------------------------------------
// Shared-memory plans.
// ---------------------------------------------------------------------
// Forward: the weights once, then per warpgroup (two per CTA) its own
// 128 x 256 encoded-input tile and 128 x 64 hidden tile.
constexpr uint32_t FWD_W = W_BYTES;                 // forward weights, all layers
constexpr uint32_t FWD_WG = TILE * IN * 2 + TILE * HID * 2;
__host__ __device__ constexpr uint32_t fwd_a0(uint32_t wg) { return FWD_W + wg * FWD_WG; }
__host__ __device__ constexpr uint32_t fwd_h(uint32_t wg) { return fwd_a0(wg) + TILE * IN * 2; }
constexpr uint32_t FWD_BAR = FWD_W + 2 * FWD_WG;     // two mbarriers, then the TMEM slot
constexpr uint32_t FWD_SMEM = FWD_BAR + 64;
constexpr uint32_t FWD_THREADS = 2 * TILE;

constexpr uint32_t BWD_WT = 0;                             // transposed weights, layers 1..4
constexpr uint32_t BWD_GCM = BWD_WT + WT_BYTES;            // gradient operand: rows = samples, 128 x 64
constexpr uint32_t BWD_GT = BWD_GCM + TILE * HID * 2;      // gradient^T operand: rows = outputs, 64 x 128
constexpr uint32_t BWD_ACTT = BWD_GT + HID * TILE * 2;     // h^T operand: rows = features, 128 (64 used) x 128
constexpr uint32_t BWD_A0T = BWD_ACTT + TILE * TILE * 2;   // encoded inputs^T: 2 x (128 features x 128)
constexpr uint32_t BWD_BAR = BWD_A0T + 2 * TILE * TILE * 2;
constexpr uint32_t BWD_SMEM = BWD_BAR + 64;

constexpr uint32_t WAIT_LIMIT = 1u << 26;

// ---------------------------------------------------------------------
// Encoding: 10 inputs x 12 frequencies x (sin, cos), the raw inputs, 1.
// ---------------------------------------------------------------------
__device__ __forceinline__ void encode(const float4* in, uint32_t s, uint32_t n, float* f /* IN */) {
    float x[RAW];
    if (s < n) {
        float4 a = in[3 * (size_t)s], b = in[3 * (size_t)s + 1], c = in[3 * (size_t)s + 2];
        x[0] = a.x; x[1] = a.y; x[2] = a.z; x[3] = a.w;
        x[4] = b.x; x[5] = b.y; x[6] = b.z; x[7] = b.w;
        x[8] = c.x; x[9] = c.y; x[10] = c.z; x[11] = c.w;
    } else {
        for (int i = 0; i < RAW; i++) x[i] = 0.0f;
    }
#pragma unroll
    for (int i = 0; i < USED; i++) {
        float scale = 1.0f;
#pragma unroll
        for (int j = 0; j < FREQS; j++) {
            float sv, cv;
            sincospif(x[i] * scale, &sv, &cv);
            f[2 * FREQS * i + 2 * j] = sv;
            f[2 * FREQS * i + 2 * j + 1] = cv;
            scale *= 2.0f;
        }
    }
#pragma unroll
    for (int i = 0; i < USED; i++) f[2 * FREQS * USED + i] = x[i];
    f[2 * FREQS * USED + USED] = 1.0f;
#pragma unroll
    for (int i = 2 * FREQS * USED + USED + 1; i < IN; i++) f[i] = 0.0f;
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t*>(&h);
}
__device__ __forceinline__ float bf16_lo(uint32_t v) { return __uint_as_float(v << 16); }
__device__ __forceinline__ float bf16_hi(uint32_t v) { return __uint_as_float(v & 0xffff0000u); }

// Row r (K values in f) into a K-major core-matrix tile.
template <int K>
__device__ __forceinline__ void put_row(char* tile, uint32_t r, const float* f) {
#pragma unroll
    for (int kb = 0; kb < K / 8; kb++) {
        uint4 v = make_uint4(pack_bf16(f[8 * kb], f[8 * kb + 1]), pack_bf16(f[8 * kb + 2], f[8 * kb + 3]),
                             pack_bf16(f[8 * kb + 4], f[8 * kb + 5]), pack_bf16(f[8 * kb + 6], f[8 * kb + 7]));
        *reinterpret_cast<uint4*>(tile + cm_offset(r, 8 * kb, K)) = v;
    }
}

// Issues D = A x B^T over K (multiple of 16) with one thread and commits
// to `bar`. A is 128 x K at `a`, B is N x K at `b`, both core-matrix tiles.
__device__ __forceinline__ void layer_mma(uint32_t tmem, uint32_t a, uint32_t b, uint32_t K, uint32_t N,
                                          uint64_t* bar) {
    const uint32_t idesc = umma::idesc_bf16(TILE, N);
    const uint32_t sbo = (K / 8) * 128;
    for (uint32_t kk = 0; kk < K / 16; kk++)
        umma::mma_bf16(tmem, umma::smem_desc(a + kk * 256, 128, sbo), umma::smem_desc(b + kk * 256, 128, sbo), idesc,
                       kk > 0);
    umma::commit(bar);
}

// Everyone: make shared-memory writes visible to the tensor core and
// order them before the MMA thread's issue.
__device__ __forceinline__ void publish_smem() {
    umma::fence_smem_to_async();
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
}

// Waits for the MMA batch; all threads see the same result.
__device__ __forceinline__ bool await_mma(uint64_t* bar, uint32_t* phase, uint32_t* err) {
    bool ok = umma::bar_wait(bar, *phase, WAIT_LIMIT);
    *phase ^= 1u;
    umma::fence_after_sync();
    if (!ok) atomicOr(err, 16u);
    return __syncthreads_and(ok ? 1 : 0) != 0;
}

// Samples of this launch: a.n, or fewer when the count is on the device.
__device__ __forceinline__ uint32_t count_of(const Args& a) {
    if (!a.n_dev) return a.n;
    uint32_t d = *((volatile const uint32_t*)a.n_dev);
    return d < a.n ? d : a.n;
}

// This thread's TMEM row: `cols` FP32 values starting at column 0.
__device__ __forceinline__ void read_row(uint32_t tmem, uint32_t cols, float* v) {
    const uint32_t warp = threadIdx.x >> 5;
    const uint32_t base = tmem + ((warp * 32u) << 16);
    for (uint32_t c = 0; c < cols; c += 16) umma::tmem_ld16(base + c, v + c);
}

// Warpgroup-local synchronisation (named barriers 1 and 2; 0 is the CTA's).
__device__ __forceinline__ void wg_sync(uint32_t id) { asm volatile("bar.sync %0, 128;" ::"r"(id) : "memory"); }
__device__ __forceinline__ bool wg_all(uint32_t id, bool v) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\tbar.red.and.pred q, %2, 128, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}\n"
        : "=r"(r)
        : "r"((uint32_t)v), "r"(id)
        : "memory");
    return r != 0u;
}
__device__ __forceinline__ void publish_smem_wg(uint32_t id) {
    umma::fence_smem_to_async();
    umma::fence_before_sync();
    wg_sync(id);
    umma::fence_after_sync();
}
__device__ __forceinline__ bool await_mma_wg(uint32_t id, uint64_t* bar, uint32_t* phase, uint32_t* err) {
    bool ok = umma::bar_wait(bar, *phase, WAIT_LIMIT);
    *phase ^= 1u;
    umma::fence_after_sync();
    if (!ok) atomicOr(err, 16u);
    return wg_all(id, ok);
}

// Two warpgroups per CTA take alternate tiles, each with its own operand
// tiles, mbarrier and 64 TMEM columns: while one waits for its MMAs the
// other encodes, reads back and activates, so the tensor core and the
// CUDA cores work on different tiles at once. Warp w reads TMEM lanes
// 32 (w mod 4) .. +31, the rows of its warpgroup's tile.
__global__ void __launch_bounds__(FWD_THREADS, 1) nrc_forward(const __grid_constant__ Args a) {
    extern __shared__ __align__(1024) char smem[];
    uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + FWD_BAR + 16);
    const uint32_t wg = threadIdx.x >> 7, t = threadIdx.x & 127u;
    const uint32_t bid = 1u + wg;  // this warpgroup's named barrier
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + FWD_BAR) + wg;
    // Weights: a straight copy of the core-matrix image.
    for (uint32_t i = threadIdx.x; i < FWD_W / 16; i += FWD_THREADS)
        reinterpret_cast<uint4*>(smem)[i] = reinterpret_cast<const uint4*>(a.wf)[i];
    if (t == 0) umma::bar_init(bar, 1);
    if (threadIdx.x < 32) umma::tmem_alloc(tslot, 128);
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tmem = *tslot + wg * 64u;
    const uint32_t lanes = ((threadIdx.x >> 5) & 3u) * 32u;
    const uint32_t s_w = umma::smem_addr(smem), s_a0 = s_w + fwd_a0(wg), s_h = s_w + fwd_h(wg);
    char* a0_tile = smem + fwd_a0(wg);
    char* h_tile = smem + fwd_h(wg);
    uint32_t phase = 0;
    const uint32_t n = count_of(a);
    const float grad_scale = a.grad_scale != 0.0f ? a.grad_scale : 1.0f / (3.0f * (float)(n ? n : 1u));
    const uint32_t tiles = (n + TILE - 1) / TILE;
    for (uint32_t tile = 2u * blockIdx.x + wg; tile < tiles; tile += 2u * gridDim.x) {
        const uint32_t s = tile * TILE + t;
        float f[IN];
        encode(a.in, s, n, f);
        put_row<IN>(a0_tile, t, f);
        publish_smem_wg(bid);
        bool ok = true;
        float v[HID];
        for (int l = 0; l < LAYERS && ok; l++) {
            const uint32_t K = l == 0 ? IN : HID, N = l == LAYERS - 1 ? OUT_PAD : HID;
            if (t == 0) layer_mma(tmem, l == 0 ? s_a0 : s_h, s_w + W_OFF(l), K, N, bar);
            ok = await_mma_wg(bid, bar, &phase, a.err);
            if (!ok) break;
            for (uint32_t c = 0; c < N; c += 16) umma::tmem_ld16(tmem + (lanes << 16) + c, v + c);
            if (l < LAYERS - 1) {
#pragma unroll
                for (int k = 0; k < HID; k++) v[k] = fmaxf(v[k], 0.0f);
                umma::fence_before_sync();
                wg_sync(bid);  // every row read before the next MMA overwrites D
                put_row<HID>(h_tile, t, v);
                if (a.acts && s < n) {
                    uint4* dst = reinterpret_cast<uint4*>(a.acts + ((size_t)s * (LAYERS - 1) + l) * HID);
#pragma unroll
                    for (int kb = 0; kb < HID / 8; kb++)
                        dst[kb] = make_uint4(pack_bf16(v[8 * kb], v[8 * kb + 1]), pack_bf16(v[8 * kb + 2], v[8 * kb + 3]),
                                             pack_bf16(v[8 * kb + 4], v[8 * kb + 5]),
                                             pack_bf16(v[8 * kb + 6], v[8 * kb + 7]));
                }
                publish_smem_wg(bid);
            }
        }
        if (!ok) break;
        // Outputs: v[0..2] radiance.
        if (s < n) {
            if (a.pred) a.pred[s] = make_float4(v[0], v[1], v[2], 0.0f);
            if (a.query_out) {
                float4 b = a.query_beta[s];
                unsigned long long item = a.query_item[s];
                float4 o = a.query_out[item];
                o.x += b.x * fmaxf(v[0], 0.0f);
                o.y += b.y * fmaxf(v[1], 0.0f);
                o.z += b.z * fmaxf(v[2], 0.0f);
                a.query_out[item] = o;
            }
        }
        if (a.target) {
            float loss = 0.0f;
            float g[OUT_PAD];
#pragma unroll
            for (int c = 0; c < OUT_PAD; c++) g[c] = 0.0f;
            if (s < n) {
                float4 tg = a.target[s];
                const float tv[3] = {tg.x, tg.y, tg.z};
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    float d = v[c] - tv[c];
                    float w = 1.0f / (v[c] * v[c] + 0.01f);
                    loss += d * d * w;
                    g[c] = 2.0f * d * w * grad_scale;
                }
                float4* dst = reinterpret_cast<float4*>(a.dy + (size_t)s * OUT_PAD);
#pragma unroll
                for (int q = 0; q < OUT_PAD / 4; q++) dst[q] = make_float4(g[4 * q], g[4 * q + 1], g[4 * q + 2], g[4 * q + 3]);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) loss += __shfl_xor_sync(0xffffffffu, loss, o);
            if ((t & 31) == 0 && loss != 0.0f) atomicAdd(a.loss, loss);
        }
        umma::fence_before_sync();
        wg_sync(bid);  // D and A0 are reused by this warpgroup's next tile
        umma::fence_after_sync();
    }
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    if (threadIdx.x < 32) umma::tmem_free(*tslot, 128);
}

// Writes column r (one sample) of a K-major core-matrix tile whose rows
// are features and whose K dimension is the 128 samples of the tile.
__device__ __forceinline__ void put_col(char* tile, uint32_t r, uint32_t rows, const float* f) {
    for (uint32_t k = 0; k < rows; k++)
        *reinterpret_cast<__nv_bfloat16*>(tile + cm_offset(k, r, TILE)) = __float2bfloat16_rn(f[k]);
}

// TMEM columns of the backward kernel: the gradient propagation product,
// then each layer's weight-gradient accumulator (transposed: lane = input
// feature, column = output), which lives across the CTA's tiles.
constexpr uint32_t TC_D = 0;
__host__ __device__ constexpr uint32_t tc_dw(int l) {
    return l == 0 ? 64u : (l == 1 ? 192u : (l == 2 ? 256u : (l == 3 ? 320u : 384u)));
}

__global__ void __launch_bounds__(TILE, 1) nrc_backward(const __grid_constant__ Args a) {
    extern __shared__ __align__(1024) char smem[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + BWD_BAR);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + BWD_BAR + 8);
    const uint32_t t = threadIdx.x;
    for (uint32_t i = t; i < WT_BYTES / 16; i += TILE)
        reinterpret_cast<uint4*>(smem + BWD_WT)[i] = reinterpret_cast<const uint4*>(a.wt)[i];
    if (t == 0) umma::bar_init(bar, 1);
    if (t < 32) umma::tmem_alloc(tslot, 512);
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tmem = *tslot;
    const uint32_t sb = umma::smem_addr(smem);
    uint32_t phase = 0;
    bool first = true;  // first tile of this CTA: the weight-gradient accumulators start at zero
    bool ok = true;
    const uint32_t n = count_of(a);
    const uint32_t tiles = (n + TILE - 1) / TILE;
    for (uint32_t tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
        const uint32_t s = tile * TILE + t;
        const bool live = s < n;
        // Output gradient, N = 16: row t of the propagation operand, column t
        // of the weight-gradient operand.
        float g[HID];
        for (int c = 0; c < HID; c++) g[c] = (live && c < (int)OUT_PAD) ? a.dy[(size_t)s * OUT_PAD + c] : 0.0f;
        put_row<OUT_PAD>(smem + BWD_GCM, t, g);
        put_col(smem + BWD_GT, t, OUT_PAD, g);
        for (int l = LAYERS - 1; l >= 1 && ok; l--) {
            const uint32_t N = l == LAYERS - 1 ? OUT_PAD : HID;
            // h_{l-1}, the input of layer l, for this sample.
            float h[HID];
            {
                const uint4* src = reinterpret_cast<const uint4*>(a.acts + ((size_t)s * (LAYERS - 1) + (l - 1)) * HID);
                for (int q = 0; q < HID / 8; q++) {
                    uint4 v = live ? src[q] : make_uint4(0, 0, 0, 0);
                    h[8 * q + 0] = bf16_lo(v.x); h[8 * q + 1] = bf16_hi(v.x);
                    h[8 * q + 2] = bf16_lo(v.y); h[8 * q + 3] = bf16_hi(v.y);
                    h[8 * q + 4] = bf16_lo(v.z); h[8 * q + 5] = bf16_hi(v.z);
                    h[8 * q + 6] = bf16_lo(v.w); h[8 * q + 7] = bf16_hi(v.w);
                }
            }
            put_col(smem + BWD_ACTT, t, HID, h);
            publish_smem();
            if (t == 0) {
                // delta_{l-1} = G x W_l (B = W_l^T), and dW_l^T += h_{l-1}^T x G.
                const uint32_t sbo_g = (N / 8) * 128;
                const uint32_t id = umma::idesc_bf16(TILE, HID);
                for (uint32_t kk = 0; kk < N / 16; kk++)
                    umma::mma_bf16(tmem + TC_D, umma::smem_desc(sb + BWD_GCM + kk * 256, 128, sbo_g),
                                   umma::smem_desc(sb + BWD_WT + WT_OFF(l) + kk * 256, 128, sbo_g), id, kk > 0);
                const uint32_t idw = umma::idesc_bf16(TILE, N), sbo_t = (TILE / 8) * 128;
                for (uint32_t kk = 0; kk < TILE / 16; kk++)
                    umma::mma_bf16(tmem + tc_dw(l), umma::smem_desc(sb + BWD_ACTT + kk * 256, 128, sbo_t),
                                   umma::smem_desc(sb + BWD_GT + kk * 256, 128, sbo_t), idw, !first || kk > 0);
                umma::commit(bar);
            }
            ok = await_mma(bar, &phase, a.err);
            if (!ok) break;
            float d[HID];
            read_row(tmem + TC_D, HID, d);
            for (int k = 0; k < HID; k++) d[k] = h[k] > 0.0f ? d[k] : 0.0f;
            umma::fence_before_sync();
            __syncthreads();  // products read, operands free
            put_row<HID>(smem + BWD_GCM, t, d);
            put_col(smem + BWD_GT, t, HID, d);
        }
        if (!ok) break;
        // dW_0^T += encoded inputs^T x delta_0, two 128-feature halves.
        {
            float f[IN];
            encode(a.in, s, n, f);
            put_col(smem + BWD_A0T, t, TILE, f);
            put_col(smem + BWD_A0T + TILE * TILE * 2, t, TILE, f + TILE);
        }
        publish_smem();
        if (t == 0) {
            const uint32_t idw = umma::idesc_bf16(TILE, HID), sbo_t = (TILE / 8) * 128;
            for (uint32_t half = 0; half < 2; half++)
                for (uint32_t kk = 0; kk < TILE / 16; kk++)
                    umma::mma_bf16(tmem + tc_dw(0) + half * HID,
                                   umma::smem_desc(sb + BWD_A0T + half * TILE * TILE * 2 + kk * 256, 128, sbo_t),
                                   umma::smem_desc(sb + BWD_GT + kk * 256, 128, sbo_t), idw, !first || kk > 0);
            umma::commit(bar);
        }
        ok = await_mma(bar, &phase, a.err);
        first = false;
        umma::fence_before_sync();
        __syncthreads();
        umma::fence_after_sync();
    }
    // This CTA's weight gradients, one row of partial sums per CTA.
    if (ok && !first) {
        float* part = a.grad_part + (size_t)blockIdx.x * PARAMS;
        float v[HID];
        for (uint32_t half = 0; half < 2; half++) {
            read_row(tmem + tc_dw(0) + half * HID, HID, v);
            const uint32_t f = half * TILE + t;
            for (uint32_t o = 0; o < HID; o++) part[P_OFF(0) + o * IN + f] = v[o];
        }
        for (int l = 1; l < LAYERS; l++) {
            const uint32_t N = l == LAYERS - 1 ? OUT_PAD : HID;
            read_row(tmem + tc_dw(l), N, v);
            if (t < HID)
                for (uint32_t o = 0; o < N; o++) part[P_OFF(l) + o * HID + t] = v[o];
        }
    } else if (!first || !ok) {
        // nothing traced, or gave up: no contribution
    }
    if (first) {  // no tile: an all-zero partial
        float* part = a.grad_part + (size_t)blockIdx.x * PARAMS;
        for (uint32_t i = t; i < PARAMS; i += TILE) part[i] = 0.0f;
    }
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    if (t < 32) umma::tmem_free(tmem, 512);
}

// grad[i] = sum over the backward CTAs' partial rows, in CTA order.
__global__ void nrc_grad_reduce(const float* part, uint32_t rows, float* grad) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= PARAMS) return;
    float acc = 0.0f;
    for (uint32_t r = 0; r < rows; r++) acc += part[(size_t)r * PARAMS + i];
    grad[i] = acc;
}

// Layer, row (output) and column (input) of parameter i.
__device__ __forceinline__ void locate(uint32_t i, int* l, uint32_t* n, uint32_t* k) {
    int L = 0;
    while (L < LAYERS - 1 && i >= P_OFF(L + 1)) L++;
    uint32_t K = L == 0 ? IN : HID, j = i - P_OFF(L);
    *l = L;
    *n = j / K;
    *k = j % K;
}

// BF16 operand images of parameter i (value w).
__device__ __forceinline__ void publish_weight(const Args& a, uint32_t i, float w) {
    int l;
    uint32_t n, k;
    locate(i, &l, &n, &k);
    const uint32_t K = l == 0 ? IN : HID, N = l == LAYERS - 1 ? OUT_PAD : HID;
    __nv_bfloat16 h = __float2bfloat16_rn(w);
    *reinterpret_cast<__nv_bfloat16*>(reinterpret_cast<char*>(a.wf) + W_OFF(l) + cm_offset(n, k, K)) = h;
    if (l >= 1)  // W_l^T: rows = inputs k, K dimension = outputs n
        *reinterpret_cast<__nv_bfloat16*>(reinterpret_cast<char*>(a.wt) + WT_OFF(l) + cm_offset(k, n, N)) = h;
}

__global__ void nrc_adam(const __grid_constant__ Args a, AdamStep st) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= PARAMS) return;
    float w = a.master[i];
    if (st.apply) {
        float g = a.grad[i];
        float m = st.b1 * a.m1[i] + (1.0f - st.b1) * g;
        float v = st.b2 * a.m2[i] + (1.0f - st.b2) * g * g;
        a.m1[i] = m;
        a.m2[i] = v;
        w -= st.lr * (m * st.c1) / (sqrtf(v * st.c2) + st.eps);
        a.master[i] = w;
    }
    publish_weight(a, i, w);
}

// Targets of training samples whose suffix ended into the cache: add the
// cache's (non-negative) prediction there times the throughput ratio.
__global__ void nrc_tail_targets(const uint32_t* counts, uint32_t t_cap, uint32_t q_cap, const uint4* tail,
                                 const float4* pred, float4* target) {
    uint32_t n = counts[1] < t_cap ? counts[1] : t_cap;
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint4 t = tail[i];
    if (t.x == 0xffffffffu || t.x >= q_cap) return;
    float4 p = pred[t.x], g = target[i];
    g.x += __uint_as_float(t.y) * fmaxf(p.x, 0.0f);
    g.y += __uint_as_float(t.z) * fmaxf(p.y, 0.0f);
    g.z += __uint_as_float(t.w) * fmaxf(p.z, 0.0f);
    target[i] = g;
}

cudaError_t launch_tail_targets(const uint32_t* counts, uint32_t t_cap, uint32_t q_cap, const uint4* tail,
                                const float4* pred, float4* target, cudaStream_t st) {
    if (t_cap == 0) return cudaSuccess;
    nrc_tail_targets<<<(t_cap + 255) / 256, 256, 0, st>>>(counts, t_cap, q_cap, tail, pred, target);
    return cudaGetLastError();
}

cudaError_t launch_forward(const Args& a, int sms, cudaStream_t st) {
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(nrc_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, FWD_SMEM);
        if (e) return e;
        attr = true;
    }
    uint32_t tiles = (a.n + TILE - 1) / TILE;
    if (tiles == 0) return cudaSuccess;
    uint32_t pairs = (tiles + 1) / 2;
    uint32_t grid = pairs < (uint32_t)sms ? pairs : (uint32_t)sms;
    nrc_forward<<<grid, FWD_THREADS, FWD_SMEM, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_backward(const Args& a, int sms, cudaStream_t st) {
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(nrc_backward, cudaFuncAttributeMaxDynamicSharedMemorySize, BWD_SMEM);
        if (e) return e;
        attr = true;
    }
    // The grid is the SM count (a partial-sum row per CTA; CTAs without a
    // tile write zeros), so the reduce order does not depend on n.
    if (a.n == 0) return cudaSuccess;
    const uint32_t grid = (uint32_t)sms;
    nrc_backward<<<grid, TILE, BWD_SMEM, st>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e) return e;
    nrc_grad_reduce<<<(PARAMS + 255) / 256, 256, 0, st>>>(a.grad_part, grid, a.grad);
    return cudaGetLastError();
}

cudaError_t launch_adam(const Args& a, const AdamStep& s, cudaStream_t st) {
    nrc_adam<<<(PARAMS + 255) / 256, 256, 0, st>>>(a, s);
    return cudaGetLastError();
}

}  // namespace nrc
}  // namespace oxd
