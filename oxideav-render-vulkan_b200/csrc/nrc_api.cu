// C ABI of the neural radiance cache (include/oxpt_nrc.h): weights, Adam
// state and scratch on the device of a tracer context, launches on its
// stream.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/oxpt_nrc.h"
#include "../../include/oxpt_serve.h"
#include "nrc.cuh"
#include "nrc_state.hpp"

using namespace oxd::nrc;


namespace {

oxpt_status nfail(oxpt_nrc* c, oxpt_status s, const std::string& m) {
    if (c) c->err = m;
    return s;
}
oxpt_status ncuda(oxpt_nrc* c, cudaError_t e, const char* what) {
    (void)cudaGetLastError();
    return nfail(c, e == cudaErrorMemoryAllocation ? OXPT_E_NOMEM : OXPT_E_CUDA,
                 std::string("cuda: ") + what + ": " + cudaGetErrorString(e));
}
#define NK(c, expr, what)                                   \
    do {                                                    \
        cudaError_t e_ = (expr);                            \
        if (e_ != cudaSuccess) return ncuda(c, e_, what);   \
    } while (0)

}  // namespace

Args oxd::nrc::base_args(oxpt_nrc* c) {
    Args a;
    std::memset(&a, 0, sizeof(a));
    a.wf = c->wf;
    a.wt = c->wt;
    a.grad = c->grad;
    a.grad_part = c->grad_part;
    a.master = c->master;
    a.m1 = c->m1;
    a.m2 = c->m2;
    a.loss = c->loss;
    a.err = c->err_dev;
    return a;
}

oxpt_status oxd::nrc::ensure_scratch(oxpt_nrc* c, size_t n) {
    if (n <= c->cap) return OXPT_OK;
    void* ptrs[] = {c->in, c->pred, c->target, c->acts, c->dy};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    c->in = c->pred = c->target = nullptr;
    c->acts = nullptr;
    c->dy = nullptr;
    c->cap = 0;
    NK(c, cudaMalloc((void**)&c->in, n * 3 * sizeof(float4)), "nrc inputs");
    NK(c, cudaMalloc((void**)&c->pred, n * sizeof(float4)), "nrc predictions");
    NK(c, cudaMalloc((void**)&c->target, n * sizeof(float4)), "nrc targets");
    NK(c, cudaMalloc((void**)&c->acts, n * (LAYERS - 1) * HID * 2), "nrc activations");
    NK(c, cudaMalloc((void**)&c->dy, n * OUT_PAD * sizeof(float)), "nrc output gradient");
    c->cap = n;
    return OXPT_OK;
}

cudaError_t oxd::nrc::adam_step(oxpt_nrc* c, cudaStream_t st) {
    c->step++;
    AdamStep a;
    a.lr = c->lr;
    a.b1 = c->b1;
    a.b2 = c->b2;
    a.eps = c->eps;
    a.c1 = (float)(1.0 / (1.0 - std::pow((double)c->b1, (double)c->step)));
    a.c2 = (float)(1.0 / (1.0 - std::pow((double)c->b2, (double)c->step)));
    a.apply = 1;
    return launch_adam(base_args(c), a, st);
}

namespace {

// Rewrites the BF16 operand images from the FP32 master weights.
oxpt_status publish(oxpt_nrc* c) {
    AdamStep st{};
    st.apply = 0;
    NK(c, launch_adam(base_args(c), st, c->stream), "nrc publish");
    return OXPT_OK;
}

oxpt_status check_err(oxpt_nrc* c) {
    uint32_t e = 0;
    NK(c, cudaMemcpyAsync(&e, c->err_dev, 4, cudaMemcpyDeviceToHost, c->stream), "nrc error word");
    NK(c, cudaStreamSynchronize(c->stream), "nrc sync");
    if (e) {
        cudaMemsetAsync(c->err_dev, 0, 4, c->stream);
        return nfail(c, OXPT_E_TIMEOUT, "a tensor-core wait gave up");
    }
    return OXPT_OK;
}

// splitmix64
uint64_t mix(uint64_t* s) {
    uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

}  // namespace

extern "C" {

oxpt_status oxpt_nrc_create(oxpt_ctx* ctx, uint64_t seed, oxpt_nrc** out) {
    if (!ctx || !out) return OXPT_E_INVALID;
    *out = nullptr;
    auto* c = new oxpt_nrc();
    c->ctx = ctx;
    c->device = oxpt_ctx_device(ctx);
    // Its own stream for the host-buffer calls: the cache may outlive the
    // context it was made on (cache frames run on the rendering context's).
    if (cudaSetDevice(c->device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return OXPT_E_NODEV;
    }
    cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, c->device);
    bool ok = cudaMalloc((void**)&c->master, PARAMS * 4) == cudaSuccess &&
              cudaMalloc((void**)&c->m1, PARAMS * 4) == cudaSuccess &&
              cudaMalloc((void**)&c->m2, PARAMS * 4) == cudaSuccess &&
              cudaMalloc((void**)&c->grad, PARAMS * 4) == cudaSuccess &&
              cudaMalloc((void**)&c->loss, 16) == cudaSuccess && cudaMalloc((void**)&c->wf, W_BYTES) == cudaSuccess &&
              cudaMalloc((void**)&c->wt, WT_BYTES) == cudaSuccess &&
              cudaMalloc((void**)&c->err_dev, 4) == cudaSuccess &&
              cudaMalloc((void**)&c->grad_part, (size_t)c->sms * PARAMS * 4) == cudaSuccess;
    if (!ok) {
        oxpt_nrc_destroy(c);
        return OXPT_E_NOMEM;
    }
    cudaMemset(c->wf, 0, W_BYTES);
    cudaMemset(c->wt, 0, WT_BYTES);
    cudaMemset(c->err_dev, 0, 4);
    // Uniform He initialisation; output rows 3..15 stay zero.
    std::vector<float> w(PARAMS, 0.0f);
    uint64_t s = seed;
    for (int l = 0; l < LAYERS; l++) {
        uint32_t K = l == 0 ? IN : HID, N = l == LAYERS - 1 ? 3u : HID;
        float a = std::sqrt(6.0f / (float)K);
        for (uint32_t n = 0; n < N; n++)
            for (uint32_t k = 0; k < K; k++) {
                double u = (double)(mix(&s) >> 11) * (1.0 / 9007199254740992.0);
                w[p_off(l) + n * K + k] = (float)((2.0 * u - 1.0) * a);
            }
    }
    *out = c;
    oxpt_status st = oxpt_nrc_set_weights(c, w.data());
    if (st) {
        oxpt_nrc_destroy(c);
        *out = nullptr;
    }
    return st;
}

void oxpt_nrc_destroy(oxpt_nrc* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) {
        cudaStreamSynchronize(c->stream);
        cudaStreamDestroy(c->stream);
    }
    void* ptrs[] = {c->master, c->m1, c->m2, c->grad, c->grad_part, c->loss, c->wf, c->wt, c->err_dev,
                    c->in, c->pred, c->target, c->acts, c->dy, c->counts, c->q_in, c->q_beta, c->q_item,
                    c->t_in, c->t_target, c->s_pre, c->s_beta, c->s_tidx, c->t_tail, c->q_pred,
                    c->s_spread, c->s_tail};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    delete c;
}

const char* oxpt_nrc_last_error(const oxpt_nrc* c) { return c ? c->err.c_str() : "null cache"; }

oxpt_status oxpt_nrc_get_weights(oxpt_nrc* c, float* out) {
    if (!c || !out) return OXPT_E_INVALID;
    NK(c, cudaSetDevice(c->device), "device");
    NK(c, cudaMemcpyAsync(out, c->master, PARAMS * 4, cudaMemcpyDeviceToHost, c->stream), "weights");
    NK(c, cudaStreamSynchronize(c->stream), "weights");
    return OXPT_OK;
}

oxpt_status oxpt_nrc_set_weights(oxpt_nrc* c, const float* w) {
    if (!c || !w) return OXPT_E_INVALID;
    NK(c, cudaSetDevice(c->device), "device");
    NK(c, cudaMemcpyAsync(c->master, w, PARAMS * 4, cudaMemcpyHostToDevice, c->stream), "weights");
    NK(c, cudaMemsetAsync(c->m1, 0, PARAMS * 4, c->stream), "adam state");
    NK(c, cudaMemsetAsync(c->m2, 0, PARAMS * 4, c->stream), "adam state");
    c->step = 0;
    oxpt_status s = publish(c);
    if (s) return s;
    NK(c, cudaStreamSynchronize(c->stream), "weights");
    return OXPT_OK;
}

oxpt_status oxpt_nrc_set_adam(oxpt_nrc* c, float lr, float b1, float b2, float eps) {
    if (!c || !(lr >= 0.0f) || !(b1 >= 0.0f && b1 < 1.0f) || !(b2 >= 0.0f && b2 < 1.0f) || !(eps > 0.0f))
        return nfail(c, OXPT_E_INVALID, "Adam needs lr >= 0, 0 <= beta < 1, eps > 0");
    c->lr = lr;
    c->b1 = b1;
    c->b2 = b2;
    c->eps = eps;
    return OXPT_OK;
}

oxpt_status oxpt_nrc_infer(oxpt_nrc* c, const float* inputs, uint32_t n, float* out) {
    if (!c || (n && (!inputs || !out))) return OXPT_E_INVALID;
    if (n == 0) return OXPT_OK;
    NK(c, cudaSetDevice(c->device), "device");
    oxpt_status s = ensure_scratch(c, n);
    if (s) return s;
    NK(c, cudaMemcpyAsync(c->in, inputs, (size_t)n * RAW * 4, cudaMemcpyHostToDevice, c->stream), "inputs");
    Args a = base_args(c);
    a.in = c->in;
    a.n = n;
    a.pred = c->pred;
    NK(c, launch_forward(a, c->sms, c->stream), "nrc forward");
    NK(c, cudaMemcpyAsync(out, c->pred, (size_t)n * 16, cudaMemcpyDeviceToHost, c->stream), "predictions");
    return check_err(c);
}

oxpt_status oxpt_nrc_train(oxpt_nrc* c, const float* inputs, const float* targets, uint32_t n, int apply, float* loss,
                           float* grad) {
    if (!c || !inputs || !targets || n == 0) return nfail(c, OXPT_E_INVALID, "training needs inputs and targets");
    NK(c, cudaSetDevice(c->device), "device");
    oxpt_status s = ensure_scratch(c, n);
    if (s) return s;
    NK(c, cudaMemcpyAsync(c->in, inputs, (size_t)n * RAW * 4, cudaMemcpyHostToDevice, c->stream), "inputs");
    NK(c, cudaMemcpyAsync(c->target, targets, (size_t)n * 16, cudaMemcpyHostToDevice, c->stream), "targets");
    NK(c, cudaMemsetAsync(c->grad, 0, PARAMS * 4, c->stream), "gradient");
    NK(c, cudaMemsetAsync(c->loss, 0, 4, c->stream), "loss");
    Args a = base_args(c);
    a.in = c->in;
    a.n = n;
    a.target = c->target;
    a.acts = c->acts;
    a.dy = c->dy;
    a.grad_scale = 1.0f / (3.0f * (float)n);
    NK(c, launch_forward(a, c->sms, c->stream), "nrc forward");
    NK(c, launch_backward(a, c->sms, c->stream), "nrc backward");
    if (apply) NK(c, adam_step(c, c->stream), "nrc adam");
    float l = 0.0f;
    NK(c, cudaMemcpyAsync(&l, c->loss, 4, cudaMemcpyDeviceToHost, c->stream), "loss");
    if (grad) NK(c, cudaMemcpyAsync(grad, c->grad, PARAMS * 4, cudaMemcpyDeviceToHost, c->stream), "gradient");
    s = check_err(c);
    if (s) return s;
    if (loss) *loss = l / (3.0f * (float)n);
    return OXPT_OK;
}

}  // extern "C"
