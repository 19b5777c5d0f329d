// oxpt_dispatch_noalloc: one trace dispatch that allocates nothing.
//
// Some callers cannot let a library call cudaMalloc or cudaFree: a host
// application that owns every byte of device memory through its own
// allocator (a renderer that budgets its frame's memory up front and hands
// each plugin the buffers it may use), or one that must not block in the
// middle of a frame, since allocation and freeing can synchronise the
// device. They pass their own device buffers for the scene and the
// accumulator. The dispatch still needs scratch memory for the per-path
// results that are added to the accumulator in sample order; it uses the
// file-scope array below instead of an allocation. The array is created
// when the library is loaded onto a device and lives until the process
// exits (NOALLOC_MAX_PATHS x 16 bytes = 4 MiB, plus one 16-byte word for the
// traversal error flag) on every GPU that loads the library.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/oxpt.h"
#include "kernels.cuh"

namespace {

constexpr uint32_t NOALLOC_MAX_PATHS = OXPT_NOALLOC_MAX_PATHS;

// Per-path results of one launch; the last element holds the error word.
static __device__ __align__(256) float4 g_noalloc_scratch[NOALLOC_MAX_PATHS + 1];

constexpr int MAX_DEVICES = 64;
struct DeviceSetup {
    bool ready = false;
    float4* scratch = nullptr;  // device address of g_noalloc_scratch
    void* context = nullptr;    // the CUDA context the address belongs to
    int sms = 0;
    int blocks_per_sm = 0;
};
DeviceSetup g_setup[MAX_DEVICES];
std::mutex g_setup_lock;

// The calling thread's current CUDA context (driver cuCtxGetCurrent, reached
// through the runtime's entry-point query so the library need not link the
// driver library), or null when it cannot be asked.
void* current_context() {
    typedef int (*GetCurrent)(void**);
    static GetCurrent fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        (void)cudaGetLastError();
        return (GetCurrent)p;
    }();
    void* ctx = nullptr;
    if (!fn || fn(&ctx) != 0) return nullptr;
    return ctx;
}

// Device addresses of the scratch array, looked up once per device with
// that device current. In host code `g_noalloc_scratch` names a host-side
// shadow, not device memory, so kernels only ever get the looked-up address.
// A device reset (cudaDeviceReset, or a reset of the primary context) loads
// the module again, possibly elsewhere: the lookup is redone whenever the
// current context is no longer the one the address was taken in.
oxpt_status setup_device(int dev, DeviceSetup** out) {
    if (dev < 0 || dev >= MAX_DEVICES) return OXPT_E_NODEV;
    std::lock_guard<std::mutex> lock(g_setup_lock);
    DeviceSetup& d = g_setup[dev];
    void* ctx = current_context();
    if (d.ready && ctx && ctx != d.context) d.ready = false;
    if (!d.ready) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
            (void)cudaGetLastError();
            return OXPT_E_CUDA;
        }
        int sms = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) {
            (void)cudaGetLastError();
            return OXPT_E_CUDA;
        }
        d.scratch = (float4*)p;
        d.context = current_context();  // made current by the lookup above
        d.sms = sms;
        d.blocks_per_sm = oxd::trace_blocks_per_sm(oxd::TRACE_THREADS, false);
        if (d.blocks_per_sm <= 0) d.blocks_per_sm = 1;
        d.ready = true;
    }
    *out = &d;
    return OXPT_OK;
}

}  // namespace

extern "C" oxpt_status oxpt_dispatch_noalloc(const oxpt_device_scene* scene, const oxpt_params* params,
                                             const oxpt_frame* frame, float* accum, void* stream) {
    if (!scene || !params || !frame || !accum) return OXPT_E_INVALID;
    if (!scene->geom || scene->geom_words < 8 || scene->geom_words % 4 != 0) return OXPT_E_INVALID;
    if (!scene->attrs || scene->attr_floats < 48 || scene->attr_floats % 48 != 0) return OXPT_E_INVALID;
    if (!scene->tables || scene->table_words == 0) return OXPT_E_INVALID;
    if (!scene->atlas || scene->atlas_side == 0 || scene->atlas_layers == 0) return OXPT_E_INVALID;
    const uint32_t w = params->dims[0], h = params->dims[1];
    if (w == 0 || h == 0) return OXPT_E_INVALID;
    // An empty frame is a no-op wherever it lies, as for oxpt_dispatch.
    if (frame->count == 0 || frame->rows == 0) return OXPT_OK;
    if (frame->y0 >= h || frame->rows > h - frame->y0) return OXPT_E_INVALID;
    if (frame->count > 0xffffffffu - frame->first) return OXPT_E_INVALID;
    // The unit of work per launch is whole rows: one row must fit.
    if (w > NOALLOC_MAX_PATHS) return OXPT_E_LIMIT;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        (void)cudaGetLastError();
        return OXPT_E_NODEV;
    }
    DeviceSetup* d = nullptr;
    oxpt_status st = setup_device(dev, &d);
    if (st != OXPT_OK) return st;
    cudaStream_t s = (cudaStream_t)stream;

    oxd::TraceArgs ta;
    ta.s.geom = (const float4*)scene->geom;
    ta.s.geom_vec4 = scene->geom_words / 4;
    ta.s.attrs = (const float4*)scene->attrs;
    ta.s.slot_count = scene->attr_floats / 48;
    ta.s.tables = (const uint32_t*)scene->tables;
    ta.s.table_words = scene->table_words;
    ta.s.atlas = (const uint2*)scene->atlas;
    ta.s.side = scene->atlas_side;
    ta.s.layers = scene->atlas_layers;
    ta.s.P = *params;
    ta.out = d->scratch;
    ta.counters = nullptr;
    ta.err = (uint32_t*)(d->scratch + NOALLOC_MAX_PATHS);
    // The shared error word keeps the last call's value: clear it.
    if (cudaMemsetAsync(ta.err, 0, sizeof(uint32_t), s) != cudaSuccess) {
        (void)cudaGetLastError();
        return OXPT_E_CUDA;
    }
    // Launches of at most NOALLOC_MAX_PATHS paths: whole rows, and as many
    // consecutive samples of them as fit. Results are added to the caller's
    // accumulator in sample order, as by oxpt_dispatch.
    uint64_t row_paths = (uint64_t)w * frame->rows;
    uint32_t rows_per = frame->rows, per = frame->count;
    if (row_paths > NOALLOC_MAX_PATHS) {
        rows_per = NOALLOC_MAX_PATHS / w;
        per = 1;
    } else {
        uint64_t fit = NOALLOC_MAX_PATHS / row_paths;
        per = (uint32_t)(fit < frame->count ? fit : frame->count);
    }
    for (uint32_t s0 = 0; s0 < frame->count; s0 += per) {
        uint32_t n = per < frame->count - s0 ? per : frame->count - s0;
        for (uint32_t r0 = 0; r0 < frame->rows; r0 += rows_per) {
            uint32_t rows = rows_per < frame->rows - r0 ? rows_per : frame->rows - r0;
            ta.first = frame->first + s0;
            ta.count = n;
            ta.y0 = frame->y0 + r0;
            ta.rows = rows;
            ta.npix = w * rows;
            ta.total = (uint64_t)ta.npix * n;
            uint64_t need = (ta.total + oxd::TRACE_THREADS - 1) / oxd::TRACE_THREADS;
            uint64_t grid = (uint64_t)d->sms * d->blocks_per_sm;
            uint32_t blocks = (uint32_t)(need < grid ? need : grid);
            if (oxd::launch_trace(ta, false, blocks ? blocks : 1, oxd::TRACE_THREADS, s) != cudaSuccess) {
                (void)cudaGetLastError();
                return OXPT_E_CUDA;
            }
            oxd::ReduceArgs ra{(float4*)accum, d->scratch, w, ta.y0, ta.npix, n};
            if (oxd::launch_reduce(ra, s) != cudaSuccess) {
                (void)cudaGetLastError();
                return OXPT_E_CUDA;
            }
        }
    }
    return OXPT_OK;
}
