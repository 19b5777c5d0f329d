// Scene preparation on the device (scene_prep.cu, bvh_build.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/oxpt.h"

namespace oxd {
namespace bvhb {

// Binned-SAH BVH over n triangles whose positions (9 floats each) are in
// device memory, built on stream st. On success *words (nodes x 8 words)
// and *slots (leaf slot -> triangle, n entries) are stream-ordered device
// allocations (cudaMallocAsync on st) that the caller frees with
// cudaFreeAsync. Scratch is stream-ordered too, so the build never waits
// for other streams' work. False with *err when an allocation or launch
// fails.
bool build_on_device(const float* pos, uint32_t n, cudaStream_t st, uint32_t** words, uint32_t** slots,
                     uint32_t* nodes, uint32_t* depth, uint32_t* launches, std::string* err);

}  // namespace bvhb

// Four-wide any-hit tree collapsed on the device from binary node words in
// device memory (bvh4_build.cu): the host collapse's words (host/bvh4.cpp),
// node for node. BUILT: *out holds n4 x 32 words (the caller's buffer of
// *out_cap bytes when large enough, else a new cudaMalloc that replaces
// it; untouched when the root is a leaf), *root_ref and *need are set. REFUSED: the host collapse
// refuses the tree too (keep the binary walk). UNSUPPORTED: deeper than
// 64 four-wide levels (collapse on the host). FAILED: a CUDA error.
enum class Collapse { BUILT, REFUSED, UNSUPPORTED, FAILED };
Collapse collapse4_device(const uint32_t* words, uint32_t nodes, cudaStream_t st, uint32_t** out, size_t* out_cap,
                          uint32_t* n4,
                          uint32_t* root_ref, uint32_t* need, std::string* err);
// Levels of the binary tree (65 when deeper than 64 or malformed), as the
// host's depth walk counts them.
bool binary_depth_device(const uint32_t* words, uint32_t nodes, cudaStream_t st, uint32_t* depth, std::string* err);

namespace prep {

// Device buffers of one prepared scene, owned by the caller afterwards.
struct DeviceScene {
    float4* geom = nullptr;   // nodes, then triangles in leaf-slot order
    size_t geom_vec4 = 0;
    float4* attrs = nullptr;  // 12 float4 per slot
    size_t slot_count = 0;
    uint2* atlas = nullptr;   // side x side x layers RGBA16F texels
    uint32_t node_count = 0, depth = 0;

    // Device time of the phases (CUDA events): source upload, BVH, slot
    // flattening, atlas (texel upload + mip chains, on its own stream).
    float phase_ms[4] = {0, 0, 0, 0};
    uint32_t launches = 0;  // kernels this build launched
};

// Builds every buffer of `src` on st (oxpt_build_scene). On failure nothing
// stays allocated and *err says why.
oxpt_status build_scene(const oxpt_scene_src& src, cudaStream_t st, DeviceScene* out, uint32_t* light_slots,
                        std::string* err);

}  // namespace prep
}  // namespace oxd
