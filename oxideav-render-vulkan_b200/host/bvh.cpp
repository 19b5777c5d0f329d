// Binned-SAH BVH builder.
//
// The reference consumes oxideav_mesh3d's binned-SAH Bvh through
// `node_words()` and `triangles` (src/pathtrace.rs:974-977) and reads it in
// pathtrace.wgsl:638-735: 32-byte nodes {lo.xyz, first | hi.xyz, count};
// count > 0 = leaf over slots [first, first + count); otherwise the two
// children are nodes `first` and `first + 1`; node 0 is the root. The
// external builder's exact split rules are not available, so this builder
// is this project's own (Wald 2007 binning, 32 bins per axis, SAH with unit
// traversal and intersection costs, leaves of at most 8 triangles). It
// writes the same node format.
//
// The build is defined level by level so that the GPU builder
// (csrc/bvh_build.cu) can produce the same words: the nodes of a level are
// split in order, each split allocates its child pair next, partitions are
// stable, and a triangle's box has its zeros made positive (so that min /
// max over any order give the same bits).
#include <algorithm>
#include <cfloat>
#include <cstring>

#include "model.hpp"

namespace oxpt {

namespace {

struct Box {
    V3 lo{FLT_MAX, FLT_MAX, FLT_MAX}, hi{-FLT_MAX, -FLT_MAX, -FLT_MAX};
    void grow(V3 p) {
        lo = vmin(lo, p);
        hi = vmax(hi, p);
    }
    void grow(const Box& b) {
        lo = vmin(lo, b.lo);
        hi = vmax(hi, b.hi);
    }
    float area() const {
        V3 e = hi - lo;
        if (e.x < 0 || e.y < 0 || e.z < 0) return 0.0f;
        return 2.0f * (e.x * e.y + e.y * e.z + e.z * e.x);
    }
};

constexpr int BINS = 32;
constexpr uint32_t MAX_LEAF = 8;

struct Builder {
    std::vector<Box> tri_box;
    std::vector<V3> centroid;
    std::vector<uint32_t> ids;
    std::vector<uint32_t> words;
    uint32_t max_depth = 0;

    uint32_t alloc_pair() {
        uint32_t n = (uint32_t)(words.size() / 8);
        words.resize(words.size() + 16, 0);
        return n;
    }

    void set_node(uint32_t n, const Box& b, uint32_t first, uint32_t count) {
        uint32_t* w = &words[(size_t)n * 8];
        std::memcpy(&w[0], &b.lo.x, 4);
        std::memcpy(&w[1], &b.lo.y, 4);
        std::memcpy(&w[2], &b.lo.z, 4);
        w[3] = first;
        std::memcpy(&w[4], &b.hi.x, 4);
        std::memcpy(&w[5], &b.hi.y, 4);
        std::memcpy(&w[6], &b.hi.z, 4);
        w[7] = count;
    }

    // Level-order build from the root over ids[begin0, end0).
    void build(uint32_t root_node, uint32_t begin0, uint32_t end0) {
        struct Job {
            uint32_t node, begin, end;
        };
        std::vector<Job> level{{root_node, begin0, end0}}, next;
        while (!level.empty()) {
            max_depth++;
            next.clear();
            for (const Job& j : level) {
                Box bounds, cbounds;
                for (uint32_t i = j.begin; i < j.end; i++) {
                    bounds.grow(tri_box[ids[i]]);
                    cbounds.grow(centroid[ids[i]]);
                }
                uint32_t count = j.end - j.begin;
                if (count <= 1) {
                    set_node(j.node, bounds, j.begin, count);
                    continue;
                }
                // Binned SAH over the three axes.
                float best_cost = FLT_MAX;
                int best_axis = -1, best_split = -1;
                for (int axis = 0; axis < 3; axis++) {
                    float lo = cbounds.lo[axis], hi = cbounds.hi[axis];
                    if (!(hi > lo)) continue;
                    float scale = BINS / (hi - lo);
                    Box bb[BINS];
                    uint32_t bc[BINS] = {0};
                    for (uint32_t i = j.begin; i < j.end; i++) {
                        int b = (int)((centroid[ids[i]][axis] - lo) * scale);
                        b = std::min(std::max(b, 0), BINS - 1);
                        bc[b]++;
                        bb[b].grow(tri_box[ids[i]]);
                    }
                    float right_area[BINS];
                    uint32_t right_count[BINS];
                    Box acc;
                    uint32_t n = 0;
                    for (int b = BINS - 1; b > 0; b--) {
                        acc.grow(bb[b]);
                        n += bc[b];
                        right_area[b] = acc.area();
                        right_count[b] = n;
                    }
                    Box lacc;
                    uint32_t ln = 0;
                    for (int b = 0; b < BINS - 1; b++) {
                        lacc.grow(bb[b]);
                        ln += bc[b];
                        if (ln == 0 || right_count[b + 1] == 0) continue;
                        float cost = lacc.area() * ln + right_area[b + 1] * right_count[b + 1];
                        if (cost < best_cost) {
                            best_cost = cost;
                            best_axis = axis;
                            best_split = b;
                        }
                    }
                }
                float parent_area = bounds.area();
                float leaf_cost = (float)count;
                float split_cost = parent_area > 0 ? 1.0f + best_cost / parent_area : FLT_MAX;
                uint32_t mid;
                if (best_axis < 0) {
                    // Coincident centroids: leaf if small, else split in half.
                    if (count <= MAX_LEAF) {
                        set_node(j.node, bounds, j.begin, count);
                        continue;
                    }
                    mid = j.begin + count / 2;
                } else {
                    if (count <= MAX_LEAF && leaf_cost <= split_cost) {
                        set_node(j.node, bounds, j.begin, count);
                        continue;
                    }
                    float lo = cbounds.lo[best_axis];
                    float scale = BINS / (cbounds.hi[best_axis] - lo);
                    auto it = std::stable_partition(ids.begin() + j.begin, ids.begin() + j.end, [&](uint32_t t) {
                        int b = (int)((centroid[t][best_axis] - lo) * scale);
                        b = std::min(std::max(b, 0), BINS - 1);
                        return b <= best_split;
                    });
                    mid = (uint32_t)(it - ids.begin());
                    if (mid == j.begin || mid == j.end) mid = j.begin + count / 2;
                }
                uint32_t first = alloc_pair();
                set_node(j.node, bounds, first, 0);
                next.push_back({first, j.begin, mid});
                next.push_back({first + 1, mid, j.end});
            }
            std::swap(level, next);
        }
    }
};

}  // namespace

BvhBuild build_bvh(const std::vector<float>& tri_pos) {
    BvhBuild out;
    size_t n = tri_pos.size() / 9;
    if (n == 0) return out;
    Builder b;
    b.tri_box.resize(n);
    b.centroid.resize(n);
    b.ids.resize(n);
    for (size_t i = 0; i < n; i++) {
        Box bx;
        for (int v = 0; v < 3; v++)  // + 0.0f: -0 becomes +0
            bx.grow(V3{tri_pos[i * 9 + v * 3] + 0.0f, tri_pos[i * 9 + v * 3 + 1] + 0.0f,
                       tri_pos[i * 9 + v * 3 + 2] + 0.0f});
        b.tri_box[i] = bx;
        b.centroid[i] = (bx.lo + bx.hi) * 0.5f;
        b.ids[i] = (uint32_t)i;
    }
    b.words.resize(8, 0);  // root
    b.build(0, 0, (uint32_t)n);
    out.node_words = std::move(b.words);
    out.slots = std::move(b.ids);
    out.depth = b.max_depth;
    return out;
}

}  // namespace oxpt
