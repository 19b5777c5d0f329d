// Stream-ordered scratch memory of the library's device passes (BVH build,
// four-wide collapse, depth walk) from a memory pool of its own per device.
// The device's default pool returns freed memory to the driver at every
// synchronisation (release threshold 0), so a pass repeated on each scene
// upload would map and unmap its scratch every time, and those driver
// calls stall behind other work; this pool keeps up to 4 GiB of freed
// scratch mapped instead. It leaves the default pool's settings alone.
#pragma once

#include <cuda_runtime.h>

#include <mutex>

namespace oxd {

// Allocates on `st` from the pool of the current device; free with
// cudaFreeAsync as usual.
inline cudaError_t scratch_alloc(void** p, size_t bytes, cudaStream_t st) {
    static std::mutex mu;
    static cudaMemPool_t pools[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaMallocAsync(p, bytes, st);
    cudaMemPool_t pool;
    {
        std::lock_guard<std::mutex> g(mu);
        if (!pools[dev]) {
            cudaMemPoolProps props = {};
            props.allocType = cudaMemAllocationTypePinned;
            props.handleTypes = cudaMemHandleTypeNone;
            props.location.type = cudaMemLocationTypeDevice;
            props.location.id = dev;
            cudaMemPool_t created = nullptr;
            if ((e = cudaMemPoolCreate(&created, &props)) != cudaSuccess) return e;
            uint64_t keep = 4ull << 30;
            cudaMemPoolSetAttribute(created, cudaMemPoolAttrReleaseThreshold, &keep);
            pools[dev] = created;  // kept for the life of the process
        }
        pool = pools[dev];
    }
    return cudaMallocFromPoolAsync(p, bytes, pool, st);
}

}  // namespace oxd
