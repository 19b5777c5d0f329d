// Neural radiance cache: network shape, parameter and operand layouts,
// kernel arguments (nrc.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace oxd {
namespace nrc {

constexpr uint32_t TILE = 128;     // samples per CTA tile (MMA M)
constexpr uint32_t RAW = 12;       // input floats per sample (3 float4)
constexpr uint32_t USED = 10;      // position 3, direction 3, normal 3, roughness 1
constexpr uint32_t FREQS = 12;     // sine / cosine frequencies per input
constexpr uint32_t IN = 256;       // encoded width: 240 + 10 raw + 1 constant + padding
constexpr uint32_t HID = 64;       // hidden width
constexpr uint32_t OUT_PAD = 16;   // output rows (3 used: RGB)
constexpr int LAYERS = 5;

// FP32 master parameters, row-major [out][in] per layer, concatenated.
__host__ __device__ constexpr uint32_t p_off(int l) {
    return l == 0 ? 0u : (l == 1 ? 16384u : (l == 2 ? 20480u : (l == 3 ? 24576u : (l == 4 ? 28672u : 29696u))));
}
constexpr uint32_t PARAMS = 29696;
// Byte offsets of each layer's BF16 K-major core-matrix image (forward:
// rows = outputs, K = inputs) and of W^T for layers 1..4 (rows = inputs,
// K = outputs).
__host__ __device__ constexpr uint32_t w_off(int l) {
    return l == 0 ? 0u : (l == 1 ? 32768u : (l == 2 ? 40960u : (l == 3 ? 49152u : 57344u)));
}
constexpr uint32_t W_BYTES = 59392;
__host__ __device__ constexpr uint32_t wt_off(int l) {
    return l <= 1 ? 0u : (l == 2 ? 8192u : (l == 3 ? 16384u : 24576u));
}
constexpr uint32_t WT_BYTES = 26624;

#define P_OFF(l) p_off(l)
#define W_OFF(l) w_off(l)
#define WT_OFF(l) wt_off(l)

struct Args {
    uint16_t* wf;                 // forward operand image (W_BYTES)
    uint16_t* wt;                 // transposed operand image (WT_BYTES)
    const float4* in;             // n x 3 float4 inputs
    uint32_t n;                   // samples (capacity of the arrays when n_dev is set)
    const uint32_t* n_dev;        // optional: the sample count in device memory (min with n)
    float4* pred;                 // inference: n predictions (rgb, 0), or null
    const float4* query_beta;     // path queries: throughput per sample, or null
    const unsigned long long* query_item;  // path result index per sample
    float4* query_out;            // path results: += beta * max(prediction, 0)
    const float4* target;         // training targets (rgb), or null
    uint16_t* acts;               // training: n x 4 x 64 bf16 hidden activations
    float* dy;                    // training: n x 16 loss gradient w.r.t. outputs
    float* loss;                  // training: summed relative L2 loss
    float grad_scale;             // 1 / (3 n): the loss is a mean over samples and channels (0: from n)
    float* grad;                  // PARAMS gradient
    float* grad_part;             // backward: one row of PARAMS partial sums per CTA (SM count rows)
    float* master;                // PARAMS FP32 weights
    float* m1;                    // Adam first moments
    float* m2;                    // Adam second moments
    uint32_t* err;                // bit 4: an MMA wait gave up
};

struct AdamStep {
    float lr, b1, b2, eps;
    float c1, c2;                 // 1 / (1 - b1^t), 1 / (1 - b2^t)
    int apply;                    // 0: only rewrite the BF16 images
};

cudaError_t launch_forward(const Args& a, int sms, cudaStream_t st);
cudaError_t launch_backward(const Args& a, int sms, cudaStream_t st);
cudaError_t launch_adam(const Args& a, const AdamStep& s, cudaStream_t st);
cudaError_t launch_tail_targets(const uint32_t* counts, uint32_t t_cap, uint32_t q_cap, const uint4* tail,
                                const float4* pred, float4* target, cudaStream_t st);

}  // namespace nrc
}  // namespace oxd
