// Round planning of batched refinement.
//
// A batched refine traces the frames of several scenes as one wavefront.
// Each round's per-path results must fit the result buffer (`cap` items),
// so the frames are cut into row bands of at most `cap` pixels and each
// band's samples into chunks, packed first-fit in frame order: a round
// takes, from every band that still has samples, as many whole samples as
// fit. Within a band, chunks leave in sample order and rounds are reduced
// in order, which keeps every pixel's accumulation order that of a single
// frame's refine.
#include "batch.hpp"

#include <algorithm>

namespace oxpt {

std::vector<std::vector<BatchPiece>> plan_batch(const std::vector<BatchInput>& in, uint64_t cap) {
    struct Band {
        uint32_t frame, y0, rows, next, left;
        uint64_t npix;
    };
    std::vector<Band> bands;
    for (uint32_t f = 0; f < in.size(); f++) {
        const BatchInput& b = in[f];
        if (b.count == 0 || b.rows == 0 || b.w == 0) continue;
        uint32_t per = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(b.rows, cap / b.w));
        for (uint32_t r = 0; r < b.rows; r += per) {
            uint32_t rows = std::min(per, b.rows - r);
            bands.push_back({f, b.y0 + r, rows, b.first, b.count, (uint64_t)b.w * rows});
        }
    }
    std::vector<std::vector<BatchPiece>> rounds;
    for (;;) {
        std::vector<BatchPiece> round;
        uint64_t room = cap, base = 0;
        for (Band& b : bands) {
            if (b.left == 0 || b.npix > room) continue;
            uint32_t n = (uint32_t)std::min<uint64_t>(b.left, room / b.npix);
            round.push_back({b.frame, b.next, n, b.y0, b.rows, base});
            base += b.npix * n;
            room -= b.npix * n;
            b.next += n;
            b.left -= n;
        }
        if (round.empty()) break;
        rounds.push_back(std::move(round));
    }
    return rounds;
}

}  // namespace oxpt
