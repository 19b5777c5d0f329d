// Four-wide BVH for any-hit (shadow) queries, collapsed from the binary
// node words of the uploaded scene.
//
// Each binary inner node becomes a 4-wide node whose children are up to
// four of its descendants: start from its two children and, while fewer
// than four, replace the inner child of largest surface area by its two
// children. Every leaf of the binary tree is reached under exactly the same
// boxes or a subset of them, and a float slab test cannot pass a box that
// its parent's test failed (the entry and exit distances are monotone in
// the box planes), so an any-hit walk over this tree tests the same leaves
// the binary walk can reach and returns the same occlusion. Node: 128 bytes
// = child boxes as lo.x[4], lo.y[4], lo.z[4], hi.x[4], hi.y[4], hi.z[4],
// then four child references (bit 31 set: leaf, bits 27..30 count - 1, bits
// 0..26 first slot; otherwise a node index; 0xffffffff: empty), then 16
// bytes of padding.
#include <algorithm>
#include <cstring>
#include <vector>

#include "bvh4.hpp"

namespace oxpt {

namespace {

struct BNode {
    float lo[3], hi[3];
    uint32_t first, count;
};

inline BNode bnode(const uint32_t* g, uint32_t i) {
    BNode n;
    std::memcpy(n.lo, &g[(size_t)i * 8], 12);
    n.first = g[(size_t)i * 8 + 3];
    std::memcpy(n.hi, &g[(size_t)i * 8 + 4], 12);
    n.count = g[(size_t)i * 8 + 7];
    return n;
}

// Boxes the monotonicity argument covers: finite, ordered, and small enough
// that a shading point minus a corner cannot overflow.
inline bool sane(const BNode& n) {
    for (int a = 0; a < 3; a++)
        if (!(n.lo[a] <= n.hi[a]) || !(n.lo[a] >= -1.0e37f) || !(n.hi[a] <= 1.0e37f)) return false;
    return true;
}

inline bool inside(const BNode& c, const BNode& p) {
    for (int a = 0; a < 3; a++)
        if (!(c.lo[a] >= p.lo[a]) || !(c.hi[a] <= p.hi[a])) return false;
    return sane(c);
}

inline float area(const BNode& n) {
    float e0 = n.hi[0] - n.lo[0], e1 = n.hi[1] - n.lo[1], e2 = n.hi[2] - n.lo[2];
    return e0 * e1 + e1 * e2 + e2 * e0;
}

}  // namespace

// Returns false when the binary tree is malformed, a child box is not
// inside its parent's, or a leaf does not fit the encoding (more than 16
// triangles or a first slot >= 2^27); the caller then keeps the binary walk.
bool build_bvh4(const uint32_t* geom, uint32_t nodes, std::vector<uint32_t>* out, uint32_t* root_ref) {
    out->clear();
    if (nodes == 0) {
        *root_ref = BVH4_EMPTY;
        return true;
    }
    auto leaf_ref = [](const BNode& n, uint32_t* ref) {
        if (n.count == 0 || n.count > 16 || n.first >= (1u << 27)) return false;
        *ref = BVH4_LEAF | ((n.count - 1) << 27) | n.first;
        return true;
    };
    BNode root = bnode(geom, 0);
    if (root.count > 0) return leaf_ref(root, root_ref);
    // Every 4-wide node stands for a distinct binary inner node, and a
    // binary tree of `nodes` nodes has at most nodes / 2 inner ones.
    const size_t cap = (size_t)nodes / 2 + 1;
    out->resize(cap * 32);  // zero-filled: padding words and unused child boxes stay 0
    uint32_t* o = out->data();
    size_t used = 1;
    // Work list of (binary node, 4-wide node index to fill).
    struct Item {
        uint32_t b, dst;
    };
    std::vector<Item> work;
    work.reserve(256);
    work.push_back({0u, 0u});
    *root_ref = 0u;
    uint64_t guard = 0;
    while (!work.empty()) {
        Item it = work.back();
        work.pop_back();
        if (++guard > nodes) return false;
        BNode n = bnode(geom, it.b);
        if (n.count > 0 || (uint64_t)n.first + 1 >= nodes) return false;
        uint32_t kid[4] = {n.first, n.first + 1, 0, 0};
        BNode kn[4];
        kn[0] = bnode(geom, kid[0]);
        kn[1] = bnode(geom, kid[1]);
        if (!sane(n) || !inside(kn[0], n) || !inside(kn[1], n)) return false;
        int nk = 2;
        while (nk < 4) {
            // Open the inner child of largest area (the first on ties).
            int best = -1;
            float best_a = -1.0f;
            for (int k = 0; k < nk; k++) {
                if (kn[k].count != 0) continue;
                float a = area(kn[k]);
                if (a > best_a) {
                    best_a = a;
                    best = k;
                }
            }
            if (best < 0) break;
            const BNode c = kn[best];
            if ((uint64_t)c.first + 1 >= nodes) return false;
            BNode c0 = bnode(geom, c.first), c1 = bnode(geom, c.first + 1);
            if (!sane(c) || !inside(c0, c) || !inside(c1, c)) return false;
            for (int k = nk; k > best + 1; k--) {
                kid[k] = kid[k - 1];
                kn[k] = kn[k - 1];
            }
            kid[best] = c.first;
            kn[best] = c0;
            kid[best + 1] = c.first + 1;
            kn[best + 1] = c1;
            nk++;
        }
        float* f = reinterpret_cast<float*>(o + (size_t)it.dst * 32);
        uint32_t* r = o + (size_t)it.dst * 32 + 24;
        for (int k = 0; k < 4; k++) {
            if (k >= nk) {
                r[k] = BVH4_EMPTY;  // empty child: skipped by its reference (its box is unused, 0)
                continue;
            }
            for (int a = 0; a < 3; a++) {
                f[a * 4 + k] = kn[k].lo[a];
                f[12 + a * 4 + k] = kn[k].hi[a];
            }
            if (kn[k].count > 0) {
                if (!leaf_ref(kn[k], &r[k])) return false;
            } else {
                if (used >= cap) return false;
                r[k] = (uint32_t)used;
                work.push_back({kid[k], (uint32_t)used});
                used++;
            }
        }
    }
    out->resize(used * 32);
    return true;
}

// Largest number of stack entries an any-hit walk that pushes every passing
// child can hold: the maximum over root-to-leaf paths of the children pushed
// along the way (at most three per level besides the one taken).
uint32_t bvh4_stack_need(const std::vector<uint32_t>& nodes, uint32_t root_ref) {
    if (root_ref & BVH4_LEAF || root_ref == BVH4_EMPTY) return 1;
    std::vector<std::pair<uint32_t, uint32_t>> st = {{root_ref, 0u}};
    uint32_t need = 0;
    while (!st.empty()) {
        auto [n, acc] = st.back();
        st.pop_back();
        const uint32_t* r = nodes.data() + (size_t)n * 32 + 24;
        uint32_t kids = 0;
        for (int k = 0; k < 4; k++) kids += r[k] != BVH4_EMPTY;
        uint32_t here = acc + (kids > 0 ? kids - 1 : 0) + 1;
        need = std::max(need, here);
        for (int k = 0; k < 4; k++)
            if (r[k] != BVH4_EMPTY && !(r[k] & BVH4_LEAF)) st.push_back({r[k], acc + (kids > 0 ? kids - 1 : 0)});
    }
    return need;
}

}  // namespace oxpt
