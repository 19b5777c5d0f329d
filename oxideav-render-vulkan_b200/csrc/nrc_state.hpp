// State of a radiance cache (include/oxpt_nrc.h), shared by its C ABI
// (nrc_api.cu) and the cache-frame driver in capi.cu.
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "../../include/oxpt.h"

struct oxpt_nrc {
    oxpt_ctx* ctx = nullptr;
    int device = 0, sms = 1;
    cudaStream_t stream = nullptr;  // owned: host-buffer calls
    std::string err;
    float *master = nullptr, *m1 = nullptr, *m2 = nullptr, *grad = nullptr, *loss = nullptr;
    float* grad_part = nullptr;  // SM count x PARAMS partial sums of the backward kernel
    uint16_t *wf = nullptr, *wt = nullptr;
    uint32_t* err_dev = nullptr;
    // scratch of the host-buffer calls
    float4 *in = nullptr, *pred = nullptr, *target = nullptr;
    uint16_t* acts = nullptr;
    float* dy = nullptr;
    size_t cap = 0;
    // radiance-cache frames (oxpt_nrc_refine)
    uint32_t* counts = nullptr;                       // queries, training samples
    float4 *q_in = nullptr, *q_beta = nullptr;
    unsigned long long* q_item = nullptr;
    size_t q_cap = 0;
    float4 *t_in = nullptr, *t_target = nullptr;
    uint4* t_tail = nullptr;
    size_t t_cap = 0;
    float4* q_pred = nullptr;
    float4 *s_pre = nullptr, *s_beta = nullptr;
    uint32_t* s_tidx = nullptr;
    float2* s_spread = nullptr;
    uint32_t* s_tail = nullptr;
    size_t s_cap = 0;
    float lr = 1e-2f, b1 = 0.9f, b2 = 0.99f, eps = 1e-8f;
    uint64_t step = 0;
};

namespace oxd {
namespace nrc {
struct Args;
// Arguments for a launch on this cache's buffers (weights, moments, error word).
Args base_args(oxpt_nrc* c);
// Grows the training scratch (activations, output gradients) to n samples.
oxpt_status ensure_scratch(oxpt_nrc* c, size_t n);
// One Adam update from the accumulated gradient (advances the step count).
cudaError_t adam_step(oxpt_nrc* c, cudaStream_t st);
}  // namespace nrc
}  // namespace oxd
