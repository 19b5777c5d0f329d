// Four-wide any-hit tree and binary depth on the device, from binary node
// words already in device memory: the same words as the host collapse
// (host/bvh4.cpp), node for node, without a host round trip.
//
// The host collapse walks a LIFO work list: a 4-wide node picks up to four
// descendants greedily (open the inner child of largest area, first on
// ties), numbers its inner kids consecutively at the current count `u`,
// and the last kid's subtree is numbered first. Here the same tree is
// built level by level:
//   expand  one thread per 4-wide node of the level: the greedy pick and
//           every check of the host (sane boxes, children inside their
//           parent, encodable leaves, indices in range);
//   scan    of the inner-kid counts gives the next level's items, each
//           knowing its parent and its position among the parent's kids;
//   sizes   bottom up, D(x) = number of 4-wide nodes below x;
//   place   top down, the host numbering: kid j of x (u_x, m_x inner kids)
//           gets index u_x + j and starts numbering at
//           u_x + m_x + sum of D over the kids after j; the node's words
//           and the stack bound (max over nodes of acc + kids) are written.
// A tree deeper than 64 four-wide levels is left to the host collapse.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <string>
#include <vector>

#include "scene_prep.cuh"

namespace oxd {
namespace bvh4b {

constexpr uint32_t NONE = 0xffffffffu;
constexpr uint32_t LEAF = 0x80000000u;

struct Item {
    uint32_t b;             // binary node this 4-wide node stands for
    uint32_t nk, m;         // kids, inner kids
    uint32_t first_child;   // item index of the first inner kid (the kids are contiguous)
    uint32_t kid[4];        // binary node ids of the kids, in order
    uint32_t D;             // 4-wide nodes below
    uint32_t idx, u, acc;   // output index, numbering start, stack entries above
};

struct BN {
    float lo[3], hi[3];
    uint32_t first, count;
};

__device__ __forceinline__ BN load(const uint32_t* w, uint32_t i) {
    const uint4 a = reinterpret_cast<const uint4*>(w)[(size_t)i * 2];
    const uint4 b = reinterpret_cast<const uint4*>(w)[(size_t)i * 2 + 1];
    BN n;
    n.lo[0] = __uint_as_float(a.x);
    n.lo[1] = __uint_as_float(a.y);
    n.lo[2] = __uint_as_float(a.z);
    n.first = a.w;
    n.hi[0] = __uint_as_float(b.x);
    n.hi[1] = __uint_as_float(b.y);
    n.hi[2] = __uint_as_float(b.z);
    n.count = b.w;
    return n;
}

// The host's checks (host/bvh4.cpp: sane, inside, area).
__device__ __forceinline__ bool sane(const BN& n) {
    for (int a = 0; a < 3; a++)
        if (!(n.lo[a] <= n.hi[a]) || !(n.lo[a] >= -1.0e37f) || !(n.hi[a] <= 1.0e37f)) return false;
    return true;
}
__device__ __forceinline__ bool inside(const BN& c, const BN& p) {
    for (int a = 0; a < 3; a++)
        if (!(c.lo[a] >= p.lo[a]) || !(c.hi[a] <= p.hi[a])) return false;
    return sane(c);
}
__device__ __forceinline__ float area(const BN& n) {
    float e0 = n.hi[0] - n.lo[0], e1 = n.hi[1] - n.lo[1], e2 = n.hi[2] - n.lo[2];
    return e0 * e1 + e1 * e2 + e2 * e0;
}
__device__ __forceinline__ bool leaf_ok(const BN& n) { return n.count != 0 && n.count <= 16 && n.first < (1u << 27); }

__global__ void expand(Item* items, uint32_t s, uint32_t e, const uint32_t* w, uint32_t nodes, uint32_t* counts,
                       uint32_t* bad) {
    uint32_t i = s + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= e) return;
    Item it = items[i];
    BN n = load(w, it.b);
    if (n.count > 0 || (uint64_t)n.first + 1 >= nodes) {
        atomicOr(bad, 1u);
        items[i].nk = items[i].m = 0;
        for (int k = 0; k < 4; k++) items[i].kid[k] = NONE;
        counts[i - s] = 0;
        return;
    }
    uint32_t kid[4] = {n.first, n.first + 1, 0, 0};
    BN kn[4];
    kn[0] = load(w, kid[0]);
    kn[1] = load(w, kid[1]);
    bool ok = sane(n) && inside(kn[0], n) && inside(kn[1], n);
    int nk = 2;
    while (ok && nk < 4) {
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
        const BN c = kn[best];
        if ((uint64_t)c.first + 1 >= nodes) {
            ok = false;
            break;
        }
        BN c0 = load(w, c.first), c1 = load(w, c.first + 1);
        if (!sane(c) || !inside(c0, c) || !inside(c1, c)) {
            ok = false;
            break;
        }
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
    uint32_t m = 0;
    for (int k = 0; ok && k < nk; k++) {
        if (kn[k].count > 0) ok = leaf_ok(kn[k]);
        else m++;
    }
    if (!ok) {
        atomicOr(bad, 1u);
        m = 0;
    }
    items[i].nk = (uint32_t)nk;
    items[i].m = m;
    items[i].D = 0;
    for (int k = 0; k < 4; k++) items[i].kid[k] = k < nk ? kid[k] : NONE;
    counts[i - s] = m;
}

// Exclusive scan of the counts: per-block scans, then block offsets (for more
// than 1024 blocks the block sums are scanned the same way and their
// offsets added back).
__global__ void scan_blocks(uint32_t* v, uint32_t K, uint32_t* block_sums) {
    __shared__ uint32_t s[1024];
    uint32_t i = blockIdx.x * 1024 + threadIdx.x;
    uint32_t x = i < K ? v[i] : 0u;
    s[threadIdx.x] = x;
    __syncthreads();
    for (uint32_t off = 1; off < 1024; off <<= 1) {
        uint32_t y = threadIdx.x >= off ? s[threadIdx.x - off] : 0u;
        __syncthreads();
        s[threadIdx.x] += y;
        __syncthreads();
    }
    if (i < K) v[i] = s[threadIdx.x] - x;
    if (threadIdx.x == 1023) block_sums[blockIdx.x] = s[1023];
}

__global__ void add_offsets(uint32_t* v, uint32_t K, const uint32_t* offs) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < K) v[i] += offs[i / 1024];
}

__global__ void scan_sums(uint32_t* block_sums, uint32_t nb, uint32_t* total) {
    __shared__ uint32_t s[1024];
    uint32_t x = threadIdx.x < nb ? block_sums[threadIdx.x] : 0u;
    s[threadIdx.x] = x;
    __syncthreads();
    for (uint32_t off = 1; off < 1024; off <<= 1) {
        uint32_t y = threadIdx.x >= off ? s[threadIdx.x - off] : 0u;
        __syncthreads();
        s[threadIdx.x] += y;
        __syncthreads();
    }
    if (threadIdx.x < nb) block_sums[threadIdx.x] = s[threadIdx.x] - x;
    if (threadIdx.x == 1023) *total = s[1023];
}

// The next level's items from the scanned inner-kid counts.
__global__ void link(Item* items, uint32_t s, uint32_t e, const uint32_t* offs, const uint32_t* block_sums,
                     const uint32_t* w, uint32_t cap) {
    uint32_t i = s + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= e) return;
    const uint32_t r = i - s;
    const uint32_t first = e + offs[r] + block_sums[r / 1024];
    items[i].first_child = first;
    uint32_t j = 0;
    const uint32_t m = items[i].m;
    for (int k = 0; k < 4 && j < m; k++) {
        uint32_t b = items[i].kid[k];
        if (b == NONE) break;
        if (w[(size_t)b * 8 + 7] != 0) continue;  // leaf kid
        if (first + j < cap) items[first + j].b = b;
        j++;
    }
}

__global__ void sizes(Item* items, uint32_t s, uint32_t e) {
    uint32_t i = s + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= e) return;
    uint32_t m = items[i].m, f = items[i].first_child, d = 0;
    for (uint32_t j = 0; j < m; j++) d += 1 + items[f + j].D;
    items[i].D = d;
}

__global__ void place(Item* items, uint32_t s, uint32_t e, const uint32_t* w, uint4* out, uint32_t n4,
                      uint32_t* need) {
    uint32_t i = s + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= e) return;
    const Item it = items[i];
    if (it.idx >= n4 || (uint64_t)it.first_child + it.m > n4) return;  // cannot happen for a counted tree
    // Kids' numbering, the last kid's subtree first (the host's LIFO order).
    uint32_t suffix = 0;
    for (int j = (int)it.m - 1; j >= 0; j--) {
        Item& c = items[it.first_child + j];
        c.idx = it.u + (uint32_t)j;
        c.u = it.u + it.m + suffix;
        c.acc = it.acc + (it.nk - 1);
        suffix += c.D;
    }
    float lo[3][4], hi[3][4];
    uint32_t ref[4];
    uint32_t j = 0;
    for (int k = 0; k < 4; k++) {
        if (k >= (int)it.nk) {
            for (int a = 0; a < 3; a++) lo[a][k] = hi[a][k] = 0.0f;
            ref[k] = NONE;
            continue;
        }
        BN c = load(w, it.kid[k]);
        for (int a = 0; a < 3; a++) {
            lo[a][k] = c.lo[a];
            hi[a][k] = c.hi[a];
        }
        if (c.count > 0) ref[k] = LEAF | ((c.count - 1) << 27) | c.first;
        else ref[k] = it.u + j++;
    }
    uint4* o = out + (size_t)it.idx * 8;
    for (int a = 0; a < 3; a++) {
        o[a] = make_uint4(__float_as_uint(lo[a][0]), __float_as_uint(lo[a][1]), __float_as_uint(lo[a][2]),
                          __float_as_uint(lo[a][3]));
        o[3 + a] = make_uint4(__float_as_uint(hi[a][0]), __float_as_uint(hi[a][1]), __float_as_uint(hi[a][2]),
                              __float_as_uint(hi[a][3]));
    }
    o[6] = make_uint4(ref[0], ref[1], ref[2], ref[3]);
    o[7] = make_uint4(0u, 0u, 0u, 0u);
    atomicMax(need, it.acc + (it.nk - 1) + 1);
}

// Binary depth, level by level (the host's bvh_depth_of: 65 for a tree
// deeper than 64 levels or malformed).
__global__ void depth_level(const uint32_t* frontier, uint32_t K, const uint32_t* w, uint32_t nodes, uint32_t* next,
                            uint32_t cap, uint32_t* ctr) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= K) return;
    uint32_t node = frontier[i];
    uint32_t first = w[(size_t)node * 8 + 3], count = w[(size_t)node * 8 + 7];
    if (count != 0) return;
    if ((uint64_t)first + 1 >= nodes) {
        atomicOr(&ctr[1], 1u);
        return;
    }
    uint32_t at = atomicAdd(&ctr[0], 2u);
    if (at + 1 < cap) {
        next[at] = first;
        next[at + 1] = first + 1;
    }
}

unsigned blocks(uint32_t n, unsigned t) { return (n + t - 1) / t; }

}  // namespace bvh4b

// ---------------------------------------------------------------------
// Host drivers.
// ---------------------------------------------------------------------

#define CK4(expr)                                                              \
    do {                                                                       \
        cudaError_t e_ = (expr);                                               \
        if (e_ != cudaSuccess) {                                               \
            *err = std::string("four-wide tree: ") + cudaGetErrorString(e_);   \
            res = Collapse::FAILED;                                            \
            goto done;                                                         \
        }                                                                      \
    } while (0)

Collapse collapse4_device(const uint32_t* w, uint32_t nodes, cudaStream_t st, uint32_t** out, size_t* out_cap, uint32_t* n4,
                          uint32_t* root_ref, uint32_t* need, std::string* err) {
    using namespace bvh4b;
    *n4 = 0;
    *need = 1;
    if (nodes == 0) {
        *root_ref = NONE;
        return Collapse::BUILT;
    }
    uint32_t root_words[8];
    Collapse res = Collapse::BUILT;
    Item* items = nullptr;
    uint32_t *counts = nullptr, *sums = nullptr, *sums2 = nullptr, *ctr = nullptr;
    std::vector<uint32_t> level_start;
    uint32_t h[2] = {0, 0};
    const uint32_t cap = nodes / 2 + 1;
    if (cudaMemcpyAsync(root_words, w, 32, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        *err = "four-wide tree: root readback";
        return Collapse::FAILED;
    }
    if (root_words[7] > 0) {  // a leaf root
        uint32_t count = root_words[7], first = root_words[3];
        if (count > 16 || first >= (1u << 27)) return Collapse::REFUSED;
        *root_ref = LEAF | ((count - 1) << 27) | first;
        return Collapse::BUILT;
    }
    *root_ref = 0;
    CK4(cudaMallocAsync((void**)&items, (size_t)cap * sizeof(Item), st));
    CK4(cudaMallocAsync((void**)&counts, (size_t)cap * 4, st));
    CK4(cudaMallocAsync((void**)&sums, (size_t)blocks(cap, 1024) * 4, st));
    CK4(cudaMallocAsync((void**)&sums2, 1024 * 4, st));
    CK4(cudaMallocAsync((void**)&ctr, 8, st));  // total, bad
    {
        Item root{};
        root.b = 0;
        root.idx = 0;
        root.u = 1;
        root.acc = 0;
        CK4(cudaMemcpyAsync(items, &root, sizeof(Item), cudaMemcpyHostToDevice, st));
    }
    CK4(cudaMemsetAsync(ctr, 0, 8, st));
    level_start = {0u, 1u};
    for (;;) {
        uint32_t s = level_start[level_start.size() - 2], e = level_start.back(), K = e - s;
        if (level_start.size() > 66) {
            res = Collapse::UNSUPPORTED;
            goto done;
        }
        expand<<<blocks(K, 128), 128, 0, st>>>(items, s, e, w, nodes, counts, ctr + 1);
        const uint32_t nb = blocks(K, 1024);
        scan_blocks<<<nb, 1024, 0, st>>>(counts, K, sums);
        if (nb <= 1024) {
            scan_sums<<<1, 1024, 0, st>>>(sums, nb, ctr);
        } else {  // K <= cap <= 2^29 + 1, so one more level of blocks suffices
            const uint32_t nb2 = blocks(nb, 1024);
            scan_blocks<<<nb2, 1024, 0, st>>>(sums, nb, sums2);
            scan_sums<<<1, 1024, 0, st>>>(sums2, nb2, ctr);
            add_offsets<<<blocks(nb, 256), 256, 0, st>>>(sums, nb, sums2);
        }
        link<<<blocks(K, 128), 128, 0, st>>>(items, s, e, counts, sums, w, cap);
        CK4(cudaGetLastError());
        CK4(cudaMemcpyAsync(h, ctr, 8, cudaMemcpyDeviceToHost, st));
        CK4(cudaStreamSynchronize(st));
        if (h[1]) {
            res = Collapse::REFUSED;  // the host collapse refuses the same tree
            goto done;
        }
        if (h[0] == 0) break;
        if ((uint64_t)e + h[0] > cap) {
            res = Collapse::REFUSED;  // more 4-wide nodes than inner binary nodes: malformed
            goto done;
        }
        level_start.push_back(e + h[0]);
    }
    *n4 = level_start.back();
    for (size_t l = level_start.size() - 1; l-- > 0;) {
        uint32_t s = level_start[l], e = level_start[l + 1];
        sizes<<<blocks(e - s, 128), 128, 0, st>>>(items, s, e);
    }
    CK4(cudaGetLastError());
    if (!*out || *out_cap < (size_t)*n4 * 128) {  // the caller's buffer, when it is large enough
        if (*out) cudaFree(*out);
        *out = nullptr;
        *out_cap = 0;
        CK4(cudaMalloc((void**)out, (size_t)*n4 * 128));
        *out_cap = (size_t)*n4 * 128;
    }
    CK4(cudaMemsetAsync(ctr, 0, 4, st));
    for (size_t l = 0; l + 1 < level_start.size(); l++) {
        uint32_t s = level_start[l], e = level_start[l + 1];
        place<<<blocks(e - s, 128), 128, 0, st>>>(items, s, e, w, reinterpret_cast<uint4*>(*out), *n4, ctr);
    }
    CK4(cudaGetLastError());
    CK4(cudaMemcpyAsync(h, ctr, 4, cudaMemcpyDeviceToHost, st));
    CK4(cudaStreamSynchronize(st));
    *need = h[0];
done:
    for (void* p : {(void*)items, (void*)counts, (void*)sums, (void*)sums2, (void*)ctr})
        if (p) cudaFreeAsync(p, st);
    if (res != Collapse::BUILT) {
        cudaStreamSynchronize(st);
        *n4 = 0;
    }
    return res;
}

#define CKD(expr)                                                            \
    do {                                                                     \
        cudaError_t e_ = (expr);                                             \
        if (e_ != cudaSuccess) {                                             \
            *err = std::string("binary depth: ") + cudaGetErrorString(e_);   \
            ok = false;                                                      \
            goto done;                                                       \
        }                                                                    \
    } while (0)

bool binary_depth_device(const uint32_t* w, uint32_t nodes, cudaStream_t st, uint32_t* depth, std::string* err) {
    using namespace bvh4b;
    *depth = 0;
    if (nodes == 0) return true;
    bool ok = true;
    uint32_t *a = nullptr, *b = nullptr, *ctr = nullptr;
    uint32_t h[2] = {0, 0}, K = 1, levels = 0;
    const uint32_t cap = nodes + 2;
    CKD(cudaMallocAsync((void**)&a, (size_t)cap * 4, st));
    CKD(cudaMallocAsync((void**)&b, (size_t)cap * 4, st));
    CKD(cudaMallocAsync((void**)&ctr, 8, st));
    CKD(cudaMemsetAsync(a, 0, 4, st));  // the root
    CKD(cudaMemsetAsync(ctr, 0, 8, st));
    {
        uint64_t visits = 1;
        while (K > 0) {
            levels++;
            if (levels > 64) {
                levels = 65;
                break;
            }
            CKD(cudaMemsetAsync(ctr, 0, 4, st));
            depth_level<<<blocks(K, 256), 256, 0, st>>>(a, K, w, nodes, b, cap, ctr);
            CKD(cudaGetLastError());
            CKD(cudaMemcpyAsync(h, ctr, 8, cudaMemcpyDeviceToHost, st));
            CKD(cudaStreamSynchronize(st));
            if (h[1]) {
                levels = 65;
                break;
            }
            visits += h[0];
            if (visits > nodes || h[0] > cap) {  // a node reached twice: malformed
                levels = 65;
                break;
            }
            K = h[0];
            std::swap(a, b);
        }
    }
    *depth = levels;
done:
    for (void* p : {(void*)a, (void*)b, (void*)ctr})
        if (p) cudaFreeAsync(p, st);
    if (!ok) cudaStreamSynchronize(st);
    return ok;
}
#undef CKD
#undef CK4

}  // namespace oxd
