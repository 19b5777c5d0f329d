// Kernel argument blocks and launch entry points shared by the C ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "device.cuh"

namespace oxd {

// Traversal / path counters of the counting build (oxpt_diag.h order).
enum { C_PATHS = 0, C_PATH_RAYS, C_SHADOW_RAYS, C_BOXES, C_LEAVES, C_TRIS, C_SHADED, C_POPS, C_N };

struct TraceArgs {
    Scene s;
    uint32_t first, count, y0, rows;
    uint32_t npix;          // w * rows
    uint64_t total;         // npix * count
    float4* out;            // per path: rgb, covered (1) / uncovered (0)
    unsigned long long* counters;
    uint32_t* err;          // bit 0: traversal guard tripped
};

struct ReduceArgs {
    float4* accum;
    const float4* out;
    uint32_t w, y0, npix, count;
};

struct RayArgs {
    Scene s;
    uint64_t n;
    const float* rays;
    uint32_t flags;
    uint32_t* slot;
    uint32_t* gid;
    float* t;
    float* bary;
    unsigned long long* counters;
    uint32_t* err;
};

struct ResolveArgs {
    const float4* accum;
    uint32_t w, h;
    oxpt_resolve_params p;
    int hdr;
    void* out;
};

cudaError_t launch_trace(const TraceArgs& a, bool count, uint32_t blocks, uint32_t threads, cudaStream_t st);
cudaError_t launch_reduce(const ReduceArgs& a, cudaStream_t st);
cudaError_t launch_rays(const RayArgs& a, cudaStream_t st);
cudaError_t launch_resolve(const ResolveArgs& a, cudaStream_t st);
cudaError_t launch_sobol(const uint32_t* dirs, uint32_t seed, uint64_t n, const uint32_t* x, const uint32_t* y,
                         const uint32_t* idx, const uint32_t* pat, uint32_t* out, cudaStream_t st);
cudaError_t launch_math(int op, uint64_t n, const float* a, const float* b, float* out, cudaStream_t st);
// Occupancy of the trace kernel for `threads` per block.
int trace_blocks_per_sm(uint32_t threads, bool count);
constexpr uint32_t TRACE_THREADS = 128;

}  // namespace oxd
