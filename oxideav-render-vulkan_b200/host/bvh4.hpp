// Four-wide BVH for any-hit queries (bvh4.cpp).
#pragma once

#include <cstdint>
#include <vector>

namespace oxpt {

constexpr uint32_t BVH4_EMPTY = 0xffffffffu;  // child slot unused
constexpr uint32_t BVH4_LEAF = 0x80000000u;   // | (count - 1) << 27 | first slot
constexpr uint32_t BVH4_NODE_WORDS = 32;      // 128 bytes

// Collapses the binary node words of a scene (node i at words 8i..8i+7)
// into 4-wide nodes; *root_ref is a node index, a leaf reference, or
// BVH4_EMPTY. False: keep the binary walk.
bool build_bvh4(const uint32_t* geom, uint32_t nodes, std::vector<uint32_t>* out, uint32_t* root_ref);

// Stack entries an any-hit walk needs when it pushes every passing child
// but the one it descends into.
uint32_t bvh4_stack_need(const std::vector<uint32_t>& nodes, uint32_t root_ref);

}  // namespace oxpt
