// Scene preparation on the device (oxpt_build_scene): the host passes of
// upload (src/pathtrace.rs:970-1239) moved to the GPU.
//
//   * Sources go up once, through two pinned staging chunks that alternate
//     (host memcpy into one while the other is in flight), merged into one
//     copy per contiguous run: positions in global triangle order, then
//     every mesh's optional attribute streams.
//   * BVH: bvh_build.cu on the device positions (the host builder's tree).
//   * Slot flattening: one thread per output vec4 (3 triangle vec4 + 12
//     attribute vec4 per leaf slot), in the word layout of the triangle
//     records (pos.xyz + global id / light index / material) and of
//     push_attrs (:1274-1315): normals + flags, tangents, uv0 / uv1,
//     colours (absent streams: 0, colours 1).
//   * Atlas (on a host thread and stream of its own, overlapping all of the
//     above): per mip chain, level 0 is staged as f32 RGBA, decoded from
//     sRGB in place when asked (fm_srgb_decode), then each level is the 2x2
//     box of the previous one with clamped taps, summed in the host's order
//     and scaled by 1/4, and the packed levels are converted with
//     fm_f32_to_f16 straight into their shelf rectangles.
// Every float operation is the host's, in the host's order, without
// contraction, so the buffers equal the host preparation's word for word.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "f16pack.h"
#include "scene_prep.cuh"

namespace oxd {
namespace prep {
namespace {

constexpr uint32_t NONE = 0xffffffffu;
constexpr unsigned long long ABSENT = ~0ull;

struct MeshRec {
    uint32_t tri_base, material, flags, pad;
    unsigned long long off[5];  // nrm, tan, uv0, uv1, col: float offsets into the stream buffer
};

struct Pack {
    uint32_t layer, x, y, on;
};

// ---------------------------------------------------------------------
// Kernels.
// ---------------------------------------------------------------------

__global__ void scatter_lights(const uint32_t* light_tris, uint32_t n_lights, uint32_t* light_of) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n_lights) light_of[light_tris[i]] = i;
}

__global__ void light_slot_of(const uint32_t* slots, uint32_t n, const uint32_t* light_of, uint32_t* light_slots) {
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    uint32_t li = light_of[slots[s]];
    if (li != NONE) light_slots[li] = s;
}

__device__ __forceinline__ float4 ld4(const float* p) { return make_float4(p[0], p[1], p[2], p[3]); }

__global__ void emit_slots(uint32_t n, const uint32_t* __restrict__ slots, const float* __restrict__ pos,
                           const float* __restrict__ src, const MeshRec* __restrict__ meshes,
                           const uint32_t* __restrict__ bases, uint32_t n_meshes, const uint32_t* __restrict__ light_of,
                           uint4* __restrict__ tris, float4* __restrict__ attrs) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)n * 15) return;
    uint32_t s = (uint32_t)(i / 15), k = (uint32_t)(i % 15);
    uint32_t g = slots[s];
    uint32_t lo = 0, hi = n_meshes;  // the last mesh whose first triangle is <= g
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (bases[mid] <= g) lo = mid;
        else hi = mid;
    }
    const MeshRec& m = meshes[lo];
    size_t t = g - m.tri_base;
    if (k < 3) {
        const float* p = pos + (size_t)g * 9 + k * 3;
        uint32_t w = k == 0 ? g : (k == 1 ? light_of[g] : m.material);
        tris[(size_t)s * 3 + k] = make_uint4(__float_as_uint(p[0]), __float_as_uint(p[1]), __float_as_uint(p[2]), w);
        return;
    }
    uint32_t a = k - 3, v = a % 3;
    float4 o;
    switch (a / 3) {
    case 0: {  // normal + flags word on vertex 0
        float f = v == 0 ? __uint_as_float(m.flags) : 0.0f;
        if (m.off[0] != ABSENT) {
            const float* q = src + m.off[0] + t * 9 + v * 3;
            o = make_float4(q[0], q[1], q[2], f);
        } else {
            o = make_float4(0.0f, 0.0f, 0.0f, f);
        }
        break;
    }
    case 1:  // tangent
        o = m.off[1] != ABSENT ? ld4(src + m.off[1] + t * 12 + v * 4) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        break;
    case 2: {  // uv0, uv1
        o = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (m.off[2] != ABSENT) {
            o.x = src[m.off[2] + t * 6 + v * 2];
            o.y = src[m.off[2] + t * 6 + v * 2 + 1];
        }
        if (m.off[3] != ABSENT) {
            o.z = src[m.off[3] + t * 6 + v * 2];
            o.w = src[m.off[3] + t * 6 + v * 2 + 1];
        }
        break;
    }
    default:  // colour
        o = m.off[4] != ABSENT ? ld4(src + m.off[4] + t * 12 + v * 4) : make_float4(1.0f, 1.0f, 1.0f, 1.0f);
        break;
    }
    attrs[(size_t)s * 12 + a] = o;
}

__device__ __forceinline__ uint2 pack_half4(float4 v) {
    return make_uint2((uint32_t)fm_f32_to_f16(v.x) | (uint32_t)fm_f32_to_f16(v.y) << 16,
                      (uint32_t)fm_f32_to_f16(v.z) | (uint32_t)fm_f32_to_f16(v.w) << 16);
}

__device__ __forceinline__ size_t atlas_at(const Pack& p, uint32_t side, uint32_t row, uint32_t col) {
    return ((size_t)p.layer * side + p.y + row) * side + p.x + col;
}

// Level 0: optional in-place sRGB decode of RGB, then the packed copy.
__global__ void chain_level0(float4* tex, uint32_t w, uint32_t h, int decode, uint2* atlas, uint32_t side, Pack p) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)w * h) return;
    float4 v = tex[i];
    if (decode) {
        v.x = fm_srgb_decode(v.x);
        v.y = fm_srgb_decode(v.y);
        v.z = fm_srgb_decode(v.z);
        tex[i] = v;
    }
    if (p.on) atlas[atlas_at(p, side, (uint32_t)(i / w), (uint32_t)(i % w))] = pack_half4(v);
}

// One level down: the 2x2 box of `a` with clamped taps.
__global__ void chain_down(const float4* __restrict__ a, uint32_t aw, uint32_t ah, float4* __restrict__ b, uint32_t bw,
                           uint32_t bh, uint2* __restrict__ atlas, uint32_t side, Pack p) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)bw * bh) return;
    uint32_t y = (uint32_t)(i / bw), x = (uint32_t)(i % bw);
    uint32_t x0 = min(2 * x, aw - 1), x1 = min(2 * x + 1, aw - 1);
    uint32_t y0 = min(2 * y, ah - 1), y1 = min(2 * y + 1, ah - 1);
    float4 q00 = a[(size_t)y0 * aw + x0], q01 = a[(size_t)y0 * aw + x1];
    float4 q10 = a[(size_t)y1 * aw + x0], q11 = a[(size_t)y1 * aw + x1];
    float4 r;
    r.x = (((q00.x + q01.x) + q10.x) + q11.x) * 0.25f;
    r.y = (((q00.y + q01.y) + q10.y) + q11.y) * 0.25f;
    r.z = (((q00.z + q01.z) + q10.z) + q11.z) * 0.25f;
    r.w = (((q00.w + q01.w) + q10.w) + q11.w) * 0.25f;
    b[i] = r;
    if (p.on) atlas[atlas_at(p, side, y, x)] = pack_half4(r);
}

// ---------------------------------------------------------------------
// Host side.
// ---------------------------------------------------------------------

// Pinned staging chunks, kept for the life of the process: page-locking
// 32 MiB costs milliseconds, so builds take chunks from here and give them
// back instead of allocating their own.
class PinnedPool {
  public:
    static PinnedPool& get() {
        static PinnedPool* p = new PinnedPool();  // never destroyed: no CUDA calls at exit
        return *p;
    }
    cudaError_t take(char** out, size_t bytes) {
        {
            std::lock_guard<std::mutex> g(mu_);
            if (!free_.empty()) {
                *out = free_.back();
                free_.pop_back();
                return cudaSuccess;
            }
        }
        return cudaMallocHost((void**)out, bytes);
    }
    void give(char* b) {
        std::lock_guard<std::mutex> g(mu_);
        free_.push_back(b);
    }

  private:
    std::mutex mu_;
    std::vector<char*> free_;
};

// memcpy on several host threads: one thread reaches a fraction of the
// memory bandwidth that staging into pinned memory can use.
void copy_host(char* dst, const char* src, size_t bytes) {
    static const unsigned hw = std::max(1u, std::min(8u, std::thread::hardware_concurrency() / 2));
    const size_t PART = 4u << 20;
    unsigned parts = (unsigned)std::min<size_t>(hw, bytes / PART);
    if (parts <= 1) {
        std::memcpy(dst, src, bytes);
        return;
    }
    size_t each = (bytes + parts - 1) / parts;
    std::vector<std::thread> th;
    th.reserve(parts - 1);
    for (unsigned i = 1; i < parts; i++) {
        size_t a = i * each, n = std::min(bytes - a, each);
        th.emplace_back([=] { std::memcpy(dst + a, src + a, n); });
    }
    std::memcpy(dst, src, each);
    for (auto& t : th) t.join();
}

// Pinned double-buffered upload: copy into one chunk while the other's
// copies run. Consecutive puts into the same allocation (`region`, its base
// pointer) at contiguous offsets merge into one copy; a copy never spans
// two allocations, even adjacent ones.
class Stager {
  public:
    explicit Stager(cudaStream_t st) : st_(st) {}
    ~Stager() { release(); }
    cudaError_t init() {
        for (int i = 0; i < 2; i++) {
            cudaError_t e = PinnedPool::get().take(&buf_[i], CHUNK);
            if (e != cudaSuccess) {
                buf_[i] = nullptr;
                return e;
            }
            e = cudaEventCreateWithFlags(&ev_[i], cudaEventDisableTiming);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    }
    cudaError_t put(const void* region, void* dst, const void* src, size_t bytes) {
        char* d = (char*)dst;
        const char* s = (const char*)src;
        while (bytes) {
            cudaError_t e;
            if (fill_ == CHUNK && (e = next_chunk()) != cudaSuccess) return e;
            size_t take = std::min(bytes, CHUNK - fill_);
            copy_host(buf_[cur_] + fill_, s, take);
            if (run_len_ && run_region_ == region && run_dst_ + run_len_ == d && run_off_ + run_len_ == fill_) {
                run_len_ += take;
            } else {
                if ((e = issue()) != cudaSuccess) return e;
                run_region_ = region;
                run_dst_ = d;
                run_off_ = fill_;
                run_len_ = take;
            }
            fill_ += take;
            d += take;
            s += take;
            bytes -= take;
        }
        return cudaSuccess;
    }
    cudaError_t flush() { return issue(); }
    void release() {
        if (run_len_) issue();
        if (buf_[0] || buf_[1]) cudaStreamSynchronize(st_);
        for (int i = 0; i < 2; i++) {
            if (buf_[i]) PinnedPool::get().give(buf_[i]);
            if (ev_[i]) cudaEventDestroy(ev_[i]);
            buf_[i] = nullptr;
            ev_[i] = nullptr;
        }
    }

  private:
    static constexpr size_t CHUNK = 32u << 20;
    cudaError_t issue() {
        if (!run_len_) return cudaSuccess;
        cudaError_t e = cudaMemcpyAsync(run_dst_, buf_[cur_] + run_off_, run_len_, cudaMemcpyHostToDevice, st_);
        run_len_ = 0;
        return e;
    }
    cudaError_t next_chunk() {
        cudaError_t e = issue();
        if (e != cudaSuccess) return e;
        if ((e = cudaEventRecord(ev_[cur_], st_)) != cudaSuccess) return e;
        used_[cur_] = true;
        cur_ ^= 1;
        if (used_[cur_] && (e = cudaEventSynchronize(ev_[cur_])) != cudaSuccess) return e;
        fill_ = 0;
        return cudaSuccess;
    }
    cudaStream_t st_;
    char* buf_[2] = {nullptr, nullptr};
    cudaEvent_t ev_[2] = {nullptr, nullptr};
    bool used_[2] = {false, false};
    int cur_ = 0;
    size_t fill_ = 0;
    const void* run_region_ = nullptr;
    char* run_dst_ = nullptr;
    size_t run_off_ = 0, run_len_ = 0;
};

void level_dims(uint32_t w, uint32_t h, uint32_t level, uint32_t* lw, uint32_t* lh) {
    for (uint32_t l = 0; l < level; l++) {
        w = std::max(1u, w / 2);
        h = std::max(1u, h / 2);
    }
    *lw = w;
    *lh = h;
}

uint32_t level_count(uint32_t w, uint32_t h) {
    uint32_t n = 1;
    while (w > 1 || h > 1) {
        w = std::max(1u, w / 2);
        h = std::max(1u, h / 2);
        n++;
    }
    return n;
}

oxpt_status check_src(const oxpt_scene_src& src, const uint32_t* light_slots, uint64_t* ntri_out,
                      uint64_t* stream_floats, std::string* err) {
    auto bad = [&](const std::string& m) {
        *err = m;
        return OXPT_E_INVALID;
    };
    if (src.n_meshes && !src.meshes) return bad("meshes missing");
    uint64_t ntri = 0, floats = 0;
    for (uint32_t i = 0; i < src.n_meshes; i++) {
        const oxpt_mesh_src& m = src.meshes[i];
        if (m.ntri && !m.pos) return bad("mesh " + std::to_string(i) + " has no positions");
        ntri += m.ntri;
        floats += (uint64_t)m.ntri * ((m.nrm ? 9 : 0) + (m.tan ? 12 : 0) + (m.uv0 ? 6 : 0) + (m.uv1 ? 6 : 0) +
                                      (m.col ? 12 : 0));
    }
    if (ntri == 0) return bad("a device-built scene needs at least one triangle");
    if (ntri > (1ull << 30)) {
        *err = "more than 2^30 triangles";
        return OXPT_E_LIMIT;
    }
    if (src.n_lights && (!src.light_tris || !light_slots)) return bad("light triangles or light_slots missing");
    for (uint32_t i = 0; i < src.n_lights; i++) {
        if (src.light_tris[i] >= ntri) return bad("light triangle id out of range");
        if (i && src.light_tris[i] <= src.light_tris[i - 1]) return bad("light triangle ids must increase");
    }
    if (src.atlas_side == 0 || src.atlas_layers == 0) return bad("atlas must have at least one layer");
    if (src.atlas_side > 16384) {
        *err = "atlas layer side above 16384";
        return OXPT_E_LIMIT;
    }
    if (src.n_chains && !src.chains) return bad("chains missing");
    for (uint32_t c = 0; c < src.n_chains; c++) {
        const oxpt_chain_src& ch = src.chains[c];
        if (!ch.width || !ch.height || !ch.rgba) return bad("chain " + std::to_string(c) + " has no texels");
        if (ch.width > 65535 || ch.height > 65535) {
            *err = "texture side above 65535";
            return OXPT_E_LIMIT;
        }
        uint32_t levels = level_count(ch.width, ch.height);
        if ((uint64_t)ch.skip + ch.n_rects > levels) return bad("chain " + std::to_string(c) + " packs levels it does not have");
        if (ch.n_rects && !ch.rects) return bad("chain rectangles missing");
        for (uint32_t r = 0; r < ch.n_rects; r++) {
            const uint32_t* q = ch.rects + 4 * r;
            uint32_t lw, lh;
            level_dims(ch.width, ch.height, ch.skip + r, &lw, &lh);
            if ((q[3] & 0xffffu) != lw || (q[3] >> 16) != lh)
                return bad("chain " + std::to_string(c) + " rectangle size differs from its level");
            if (q[0] >= src.atlas_layers || (uint64_t)q[1] + lw > src.atlas_side || (uint64_t)q[2] + lh > src.atlas_side)
                return bad("chain " + std::to_string(c) + " rectangle outside the atlas");
        }
    }
    *ntri_out = ntri;
    *stream_floats = floats;
    return OXPT_OK;
}

unsigned grid_of(size_t n, unsigned block) { return (unsigned)((n + block - 1) / block); }

// The atlas half of a build: texel staging and mip kernels for every chain
// on its own stream and host thread, overlapping the geometry half.
struct AtlasJob {
    const oxpt_scene_src* src = nullptr;
    int device = 0;
    cudaStream_t st = nullptr;
    uint2* atlas = nullptr;
    float4 *tex = nullptr, *lvl_a = nullptr, *lvl_b = nullptr;  // level-0 staging, ping-pong levels
    cudaEvent_t begin = nullptr, end = nullptr;
    cudaError_t e = cudaSuccess;
    std::string what;
    uint32_t launches = 0;  // kernels launched
};

void atlas_work(AtlasJob* j) {
    const oxpt_scene_src& src = *j->src;
    auto ck = [&](cudaError_t e, const char* what) {
        if (e != cudaSuccess && j->e == cudaSuccess) {
            j->e = e;
            j->what = what;
        }
        return e == cudaSuccess;
    };
    if (!ck(cudaSetDevice(j->device), "texture thread device")) return;
    Stager stage(j->st);
    if (!ck(stage.init(), "texture staging")) return;
    if (!ck(cudaEventRecord(j->begin, j->st), "atlas timing")) return;
    if (!ck(cudaMemsetAsync(j->atlas, 0, (size_t)src.atlas_side * src.atlas_side * src.atlas_layers * 8, j->st),
            "texture atlas"))
        return;
    const float* staged = nullptr;  // texels now in `tex` (undecoded)
    uint32_t staged_w = 0, staged_h = 0;
    for (uint32_t c = 0; c < src.n_chains; c++) {
        const oxpt_chain_src& ch = src.chains[c];
        const uint32_t w = ch.width, h = ch.height, levels = level_count(w, h);
        if (!(staged == ch.rgba && staged_w == w && staged_h == h)) {
            if (!ck(stage.put(j->tex, j->tex, ch.rgba, (size_t)w * h * 16), "texel upload")) return;
            if (!ck(stage.flush(), "texel upload")) return;
        }
        staged = ch.srgb_decode ? nullptr : ch.rgba;
        staged_w = w;
        staged_h = h;
        auto pack_of = [&](uint32_t level) {
            Pack p{0, 0, 0, 0};
            if (level >= ch.skip && level < ch.skip + ch.n_rects) {
                const uint32_t* q = ch.rects + 4 * (level - ch.skip);
                p = Pack{q[0], q[1], q[2], 1};
            }
            return p;
        };
        chain_level0<<<grid_of((size_t)w * h, 256), 256, 0, j->st>>>(j->tex, w, h, ch.srgb_decode ? 1 : 0, j->atlas,
                                                                      src.atlas_side, pack_of(0));
        if (!ck(cudaGetLastError(), "mip level 0")) return;
        const float4* a = j->tex;
        uint32_t aw = w, ah = h;
        float4* out_buf[2] = {j->lvl_a, j->lvl_b};
        for (uint32_t l = 1; l < levels; l++) {
            uint32_t bw = std::max(1u, aw / 2), bh = std::max(1u, ah / 2);
            float4* b = out_buf[(l - 1) & 1];
            chain_down<<<grid_of((size_t)bw * bh, 256), 256, 0, j->st>>>(a, aw, ah, b, bw, bh, j->atlas,
                                                                         src.atlas_side, pack_of(l));
            if (!ck(cudaGetLastError(), "mip level")) return;
            a = b;
            aw = bw;
            ah = bh;
        }
    }
    j->launches = 0;
    for (uint32_t c = 0; c < src.n_chains; c++) j->launches += level_count(src.chains[c].width, src.chains[c].height);
    ck(cudaEventRecord(j->end, j->st), "atlas timing");
    stage.release();  // waits for the stream
}

}  // namespace

oxpt_status build_scene(const oxpt_scene_src& src, cudaStream_t st, DeviceScene* out, uint32_t* light_slots,
                        std::string* err) {
    *out = DeviceScene{};
    uint64_t ntri64 = 0, stream_floats = 0;
    oxpt_status status = check_src(src, light_slots, &ntri64, &stream_floats, err);
    if (status) return status;
    const uint32_t n = (uint32_t)ntri64;

    float *pos = nullptr, *streams = nullptr;
    MeshRec* recs = nullptr;
    uint32_t *bases = nullptr, *light_of = nullptr, *lights = nullptr, *lslots = nullptr;
    uint32_t *words = nullptr, *slots = nullptr;
    DeviceScene ds;
    Stager stage(st);
    cudaError_t e = cudaSuccess;
    std::vector<MeshRec> hrec;
    std::vector<uint32_t> hbase;
    uint64_t max_tex = 0, max_lvl1 = 0;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    AtlasJob job;
    std::thread worker;
    bool working = false;
    uint32_t bvh_launches = 0;

#define PK(expr, what)                                            \
    do {                                                          \
        e = (expr);                                               \
        if (e != cudaSuccess) {                                   \
            *err = std::string("scene build: ") + what + ": " + cudaGetErrorString(e); \
            goto fail;                                            \
        }                                                         \
    } while (0)

    for (auto& x : ev) PK(cudaEventCreate(&x), "timing events");
    // Atlas: buffers here, the work on a thread and stream of its own.
    PK(cudaGetDevice(&job.device), "device");
    job.src = &src;
    for (uint32_t c = 0; c < src.n_chains; c++) {
        const oxpt_chain_src& ch = src.chains[c];
        max_tex = std::max<uint64_t>(max_tex, (uint64_t)ch.width * ch.height);
        uint32_t w1, h1;
        level_dims(ch.width, ch.height, 1, &w1, &h1);
        max_lvl1 = std::max<uint64_t>(max_lvl1, (uint64_t)w1 * h1);
    }
    PK(cudaMalloc((void**)&ds.atlas, (size_t)src.atlas_side * src.atlas_side * src.atlas_layers * 8), "texture atlas");
    job.atlas = ds.atlas;
    if (src.n_chains) {
        PK(cudaMalloc((void**)&job.tex, max_tex * 16), "texture staging");
        PK(cudaMalloc((void**)&job.lvl_a, max_lvl1 * 16), "mip level");
        PK(cudaMalloc((void**)&job.lvl_b, max_lvl1 * 16), "mip level");
    }
    PK(cudaStreamCreateWithFlags(&job.st, cudaStreamNonBlocking), "texture stream");
    PK(cudaEventCreate(&job.begin), "timing events");
    PK(cudaEventCreate(&job.end), "timing events");
    // Device buffers of the geometry half.
    PK(cudaMalloc((void**)&pos, (size_t)n * 36), "positions");
    PK(cudaMalloc((void**)&streams, std::max<uint64_t>(stream_floats, 1) * 4), "attribute streams");
    PK(cudaMalloc((void**)&light_of, (size_t)n * 4), "light lookup");
    PK(cudaMalloc((void**)&lslots, std::max(src.n_lights, 1u) * 4), "light slots");
    if (src.n_lights) PK(cudaMalloc((void**)&lights, (size_t)src.n_lights * 4), "light list");
    {
        uint32_t non_empty = 0;
        for (uint32_t i = 0; i < src.n_meshes; i++) non_empty += src.meshes[i].ntri ? 1 : 0;
        PK(cudaMalloc((void**)&recs, (size_t)non_empty * sizeof(MeshRec)), "mesh records");
        PK(cudaMalloc((void**)&bases, (size_t)non_empty * 4), "mesh bases");
    }
    worker = std::thread(atlas_work, &job);
    working = true;

    PK(stage.init(), "pinned staging");
    PK(cudaEventRecord(ev[0], st), "timing");
    // Mesh records (non-empty meshes) and the sources.
    {
        uint64_t base = 0, off = 0;
        for (uint32_t i = 0; i < src.n_meshes; i++) {
            const oxpt_mesh_src& m = src.meshes[i];
            if (!m.ntri) continue;
            MeshRec r{};
            r.tri_base = (uint32_t)base;
            r.material = m.material;
            r.flags = (m.nrm ? 1u : 0u) | (m.tan ? 1u : 0u) << 1 | (m.col ? 1u : 0u) << 2 | (m.uv0 ? 1u : 0u) << 3 |
                      (m.uv1 ? 1u : 0u) << 4;
            const float* ptr[5] = {m.nrm, m.tan, m.uv0, m.uv1, m.col};
            const uint32_t per[5] = {9, 12, 6, 6, 12};
            PK(stage.put(pos, pos + base * 9, m.pos, (size_t)m.ntri * 36), "position upload");
            for (int k = 0; k < 5; k++) {
                if (!ptr[k]) {
                    r.off[k] = ABSENT;
                    continue;
                }
                r.off[k] = off;
                PK(stage.put(streams, streams + off, ptr[k], (size_t)m.ntri * per[k] * 4), "attribute upload");
                off += (uint64_t)m.ntri * per[k];
            }
            hrec.push_back(r);
            hbase.push_back(r.tri_base);
            base += m.ntri;
        }
    }
    PK(stage.put(recs, recs, hrec.data(), hrec.size() * sizeof(MeshRec)), "mesh record upload");
    PK(stage.put(bases, bases, hbase.data(), hbase.size() * 4), "mesh base upload");
    PK(cudaMemsetAsync(light_of, 0xff, (size_t)n * 4, st), "light lookup");
    if (src.n_lights) PK(stage.put(lights, lights, src.light_tris, (size_t)src.n_lights * 4), "light list upload");
    PK(stage.flush(), "upload");
    if (src.n_lights) {
        scatter_lights<<<grid_of(src.n_lights, 256), 256, 0, st>>>(lights, src.n_lights, light_of);
        PK(cudaGetLastError(), "light lookup");
    }
    PK(cudaEventRecord(ev[1], st), "timing");
    // BVH (syncs the stream once per level).
    if (!bvhb::build_on_device(pos, n, st, &words, &slots, &ds.node_count, &ds.depth, &bvh_launches, err)) {
        status = err->find("out of memory") != std::string::npos ? OXPT_E_NOMEM : OXPT_E_CUDA;
        goto fail_status;
    }
    PK(cudaEventRecord(ev[2], st), "timing");
    ds.slot_count = n;
    ds.geom_vec4 = (size_t)ds.node_count * 2 + (size_t)n * 3;
    PK(cudaMalloc((void**)&ds.geom, ds.geom_vec4 * 16), "geom buffer");
    PK(cudaMalloc((void**)&ds.attrs, (size_t)n * 12 * 16), "attribute buffer");
    PK(cudaMemcpyAsync(ds.geom, words, (size_t)ds.node_count * 32, cudaMemcpyDeviceToDevice, st), "node copy");
    emit_slots<<<grid_of((size_t)n * 15, 256), 256, 0, st>>>(n, slots, pos, streams, recs, bases, (uint32_t)hrec.size(),
                                                              light_of, (uint4*)(ds.geom + (size_t)ds.node_count * 2),
                                                              ds.attrs);
    PK(cudaGetLastError(), "slot flattening");
    if (src.n_lights) {
        PK(cudaMemsetAsync(lslots, 0xff, (size_t)src.n_lights * 4, st), "light slots");
        light_slot_of<<<grid_of(n, 256), 256, 0, st>>>(slots, n, light_of, lslots);
        PK(cudaGetLastError(), "light slots");
    }
    PK(cudaEventRecord(ev[3], st), "timing");
    if (src.n_lights)
        PK(cudaMemcpyAsync(light_slots, lslots, (size_t)src.n_lights * 4, cudaMemcpyDeviceToHost, st), "light slots");
    PK(cudaStreamSynchronize(st), "scene build");
    worker.join();
    working = false;
    if (job.e != cudaSuccess) {
        e = job.e;
        *err = "scene build: " + job.what + ": " + cudaGetErrorString(job.e);
        goto fail;
    }
    cudaEventElapsedTime(&ds.phase_ms[0], ev[0], ev[1]);
    cudaEventElapsedTime(&ds.phase_ms[1], ev[1], ev[2]);
    cudaEventElapsedTime(&ds.phase_ms[2], ev[2], ev[3]);
    if (cudaEventElapsedTime(&ds.phase_ms[3], job.begin, job.end) != cudaSuccess) ds.phase_ms[3] = 0.0f;
    // the BVH's, flattening (+ two for lights), mip levels
    ds.launches = bvh_launches + 1 + (src.n_lights ? 2 : 0) + job.launches;
    (void)cudaGetLastError();
    cudaFreeAsync(words, st);
    cudaFreeAsync(slots, st);
    {
        void* temps[] = {pos, streams, job.tex, job.lvl_a, job.lvl_b, recs, bases, light_of, lights, lslots};
        for (void* p : temps)
            if (p) cudaFree(p);
    }
    for (auto x : ev) cudaEventDestroy(x);
    cudaEventDestroy(job.begin);
    cudaEventDestroy(job.end);
    cudaStreamDestroy(job.st);
    stage.release();
    *out = std::move(ds);
    return OXPT_OK;
#undef PK

fail:
    status = e == cudaErrorMemoryAllocation ? OXPT_E_NOMEM : OXPT_E_CUDA;
fail_status:
    if (working) worker.join();
    (void)cudaGetLastError();
    cudaStreamSynchronize(st);
    if (job.st) cudaStreamSynchronize(job.st);
    stage.release();
    if (words) cudaFreeAsync(words, st);
    if (slots) cudaFreeAsync(slots, st);
    cudaStreamSynchronize(st);
    {
        void* temps[] = {pos, streams, job.tex, job.lvl_a, job.lvl_b, recs, bases, light_of, lights, lslots,
                         ds.geom, ds.attrs, ds.atlas};
        for (void* p : temps)
            if (p) cudaFree(p);
    }
    for (auto x : ev)
        if (x) cudaEventDestroy(x);
    if (job.begin) cudaEventDestroy(job.begin);
    if (job.end) cudaEventDestroy(job.end);
    if (job.st) cudaStreamDestroy(job.st);
    return status;
}

}  // namespace prep
}  // namespace oxd
