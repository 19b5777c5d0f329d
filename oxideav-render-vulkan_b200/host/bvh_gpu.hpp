// GPU build of the binned-SAH BVH (csrc/bvh_build.cu): the same node words
// and slot order as build_bvh (host/bvh.cpp).
#pragma once

#include <string>
#include <vector>

#include "model.hpp"

namespace oxpt {

// False (with *err) when the device or an allocation fails; the caller
// then builds on the host.
bool build_bvh_device(int device, const std::vector<float>& tri_pos, BvhBuild* out, std::string* err);

}  // namespace oxpt
