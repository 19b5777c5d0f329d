// Round planning of batched refinement (batch.cpp).
#pragma once

#include <cstdint>
#include <vector>

namespace oxpt {

// A frame to trace: samples [first, first + count) over rows [y0, y0 + rows)
// of an image `w` pixels wide.
struct BatchInput {
    uint32_t w, first, count, y0, rows;
};

// One piece of a round: frame `frame`'s samples [first, first + count) over
// rows [y0, y0 + rows), as the round's items [base, base + w * rows * count).
struct BatchPiece {
    uint32_t frame, first, count, y0, rows;
    uint64_t base;
};

// Packs the frames into rounds of at most `cap` items (cap >= every w).
// Frames wider than a round are cut into row bands; each band's samples
// go out in increasing order, so reducing the rounds in order adds every
// pixel's samples in sample order.
std::vector<std::vector<BatchPiece>> plan_batch(const std::vector<BatchInput>& in, uint64_t cap);

}  // namespace oxpt
