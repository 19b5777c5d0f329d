// Split wavefront: the shading work of a bounce in three small kernels.
//
// The single wavefront logic kernel (wavefront.cu) carries texture
// filtering, the layered BSDF, light sampling and path bookkeeping in one
// body whose code does not fit the instruction cache. Here a bounce is
//   split_logic  one thread per slot: adds the previous vertex's visible NEE
//                terms in job order, attenuates in a medium, handles misses
//                (environment / ambient), finalises finished paths and
//                regenerates their slots; surface hits go to a shade queue;
//   split_shade  one thread per queued hit: emission, material, BSDF of the
//                vertex (written to a vertex record for split_nee), BSDF
//                sampling and roulette; queues the continuation ray;
//   split_nee    one thread per (vertex, NEE job), job-major so that a warp
//                evaluates the same light for 32 vertices;
// followed by the same extension and shadow traversal kernels. Every path
// still receives its contributions in the reference's order: the vertex's
// NEE terms are added by the next split_logic before anything the next
// continuation ray finds.
#include <cooperative_groups.h>

#include "kernels.cuh"
#include "path.cuh"
#include "shade.cuh"
#include "traverse.cuh"
#include "wavefront.cuh"

namespace cg = cooperative_groups;

namespace oxd {
// Built twice: exactly (the launchers in oxd) and with OXPT_FAST and fast
// math (the tolerance plan's shading; the launchers in oxd::fast).
#ifdef OXPT_FAST
namespace fast {
#endif

namespace {

enum : uint32_t { ST_EMPTY = 0, ST_TRACING = 1, ST_ENDING = 2 };

__device__ __forceinline__ uint32_t append1(uint32_t* ctr) {
    cg::coalesced_group g = cg::coalesced_threads();
    uint32_t base = 0;
    if (g.thread_rank() == 0) base = atomicAdd(ctr, g.size());
    return g.shfl(base, 0) + g.thread_rank();
}
__device__ __forceinline__ unsigned long long fetch1(unsigned long long* ctr) {
    cg::coalesced_group g = cg::coalesced_threads();
    unsigned long long base = 0;
    if (g.thread_rank() == 0) base = atomicAdd(ctr, (unsigned long long)g.size());
    return g.shfl(base, 0) + g.thread_rank();
}

__device__ __forceinline__ void load_state(const WaveArgs& a, uint32_t i, PathCore* pc, Sampler* smp) {
    uint4 sd = a.st.seed[i];
    float4 b = a.st.beta[i], r = a.st.rad[i], d = a.st.dir[i], pp = a.st.prev[i], sg = a.st.sigma[i];
    smp->pixel_seed = sd.x;
    smp->index = sd.y;
    smp->path_seed = sd.z;
    pc->k = sd.w;
    pc->beta = xyz(b);
    pc->prev_pdf = b.w;
    pc->radiance = xyz(r);
    pc->in_medium = (__float_as_uint(r.w) & 4u) != 0u;
    pc->d = xyz(d);
    pc->prev_pos = xyz(pp);
    pc->sigma = xyz(sg);
}

__device__ __forceinline__ void save_state(const WaveArgs& a, uint32_t i, const PathCore& pc, const Sampler& smp,
                                           uint32_t stage) {
    a.st.seed[i] = make_uint4(smp.pixel_seed, smp.index, smp.path_seed, pc.k);
    a.st.beta[i] = make_float4(pc.beta.x, pc.beta.y, pc.beta.z, pc.prev_pdf);
    a.st.rad[i] = make_float4(pc.radiance.x, pc.radiance.y, pc.radiance.z,
                              __uint_as_float(stage | (pc.in_medium ? 4u : 0u)));
    a.st.dir[i] = make_float4(pc.d.x, pc.d.y, pc.d.z, 0.0f);
    a.st.prev[i] = make_float4(pc.prev_pos.x, pc.prev_pos.y, pc.prev_pos.z, 0.0f);
    a.st.sigma[i] = make_float4(pc.sigma.x, pc.sigma.y, pc.sigma.z, 0.0f);
}

__device__ __forceinline__ Hit load_hit(const WaveArgs& a, uint32_t i, uint32_t* hmat) {
    uint4 hb = a.st.hit[i];
    uint32_t hm = a.st.hmeta[i];
    Hit h;
    h.slot = hb.x;
    h.t = __uint_as_float(hb.y);
    float u = __uint_as_float(hb.z), v = __uint_as_float(hb.w);
    h.b = mk(1.0f - u - v, u, v);
    h.front = (hm >> 31) != 0u;
    *hmat = hm & 0x7fffffffu;
    return h;
}

// Vertex record, 13 float4 fields stored field-major (a warp's loads of one
// field are contiguous).
constexpr uint32_t VREC = 13;

__device__ __forceinline__ void put_vertex(const WaveArgs& a, uint32_t v, const Vertex& x, const PathCore& pc,
                                           uint32_t path_seed) {
    const uint32_t P = a.vcap;
    const Bsdf& b = x.bsdf;
    float4* r = a.q.vrec;
    r[0 * P + v] = make_float4(b.v.x, b.v.y, b.v.z, b.metallic);
    r[1 * P + v] = make_float4(b.n.x, b.n.y, b.n.z, b.alpha);
    r[2 * P + v] = make_float4(b.ng.x, b.ng.y, b.ng.z, b.specular);
    r[3 * P + v] = make_float4(b.ncc.x, b.ncc.y, b.ncc.z, b.transmission);
    r[4 * P + v] = make_float4(b.base.x, b.base.y, b.base.z, b.clearcoat);
    r[5 * P + v] = make_float4(b.f0d.x, b.f0d.y, b.f0d.z, b.cc_alpha);
    r[6 * P + v] = make_float4(b.sheen.x, b.sheen.y, b.sheen.z, b.sheen_rough);
    r[7 * P + v] = make_float4(b.eta_i, b.eta_t, b.sheen_alpha, b.w_cc);
    r[8 * P + v] = make_float4(b.p0, b.p1, b.p2, b.p3);
    r[9 * P + v] = make_float4(b.p4, __uint_as_float(b.thin ? 1u : 0u), __uint_as_float(pc.k), __uint_as_float(path_seed));
    r[10 * P + v] = make_float4(x.p.x, x.p.y, x.p.z, 0.0f);
    r[11 * P + v] = make_float4(pc.beta.x, pc.beta.y, pc.beta.z, 0.0f);
    r[12 * P + v] = x.pl_u;
}

__device__ __forceinline__ void get_vertex(const WaveArgs& a, uint32_t v, Vertex* x, PathCore* pc,
                                           uint32_t* path_seed) {
    const uint32_t P = a.vcap;
    const float4* r = a.q.vrec;
    Bsdf& b = x->bsdf;
    float4 f;
    f = r[0 * P + v]; b.v = xyz(f); b.metallic = f.w;
    f = r[1 * P + v]; b.n = xyz(f); b.alpha = f.w;
    f = r[2 * P + v]; b.ng = xyz(f); b.specular = f.w;
    f = r[3 * P + v]; b.ncc = xyz(f); b.transmission = f.w;
    f = r[4 * P + v]; b.base = xyz(f); b.clearcoat = f.w;
    f = r[5 * P + v]; b.f0d = xyz(f); b.cc_alpha = f.w;
    f = r[6 * P + v]; b.sheen = xyz(f); b.sheen_rough = f.w;
    f = r[7 * P + v]; b.eta_i = f.x; b.eta_t = f.y; b.sheen_alpha = f.z; b.w_cc = f.w;
    f = r[8 * P + v]; b.p0 = f.x; b.p1 = f.y; b.p2 = f.z; b.p3 = f.w;
    f = r[9 * P + v];
    b.p4 = f.x;
    b.thin = __float_as_uint(f.y) != 0u;
    pc->k = __float_as_uint(f.z);
    *path_seed = __float_as_uint(f.w);
    f = r[10 * P + v]; x->p = xyz(f);
    f = r[11 * P + v]; pc->beta = xyz(f);
    x->pl_u = r[12 * P + v];
    x->ng = b.ng;
}

// Batched launches (frames of several scenes in one wavefront): the frame
// of a launch item, and the scene of a slot.
__device__ __forceinline__ uint32_t frame_of1(const WaveArgs& a, unsigned long long item) {
    uint32_t lo = 0u, hi = a.nframes;
    while (hi - lo > 1u) {
        uint32_t mid = (lo + hi) >> 1;
        if (a.frames[mid].base <= item) lo = mid;
        else hi = mid;
    }
    return lo;
}

template <bool BATCH>
__device__ __forceinline__ const Scene& slot_scene(const WaveArgs& a, uint32_t i) {
    return BATCH ? a.frames[a.st.frame[i]].s : a.s;
}

// Shared-memory tables come from the first frame in a batched launch (the
// host checks that every scene holds the same words).
template <bool BATCH>
__device__ __forceinline__ const Scene& tables_of(const WaveArgs& a) {
    return BATCH ? a.frames[0].s : a.s;
}

// Radiance-cache inputs of a vertex: position normalised to the scene's
// root box, outgoing direction and shading normal mapped to [0, 1], GGX
// alpha; three float4 (pos.xyz, alpha | dir.xyz, 0 | normal.xyz, 0).
__device__ __forceinline__ void nrc_features(const Scene& s, const Vertex& vx, float4* out) {
    float4 lo = geomv(s, 0), hi = geomv(s, 1);
    f3 ext = mk(fmaxf(hi.x - lo.x, 1e-20f), fmaxf(hi.y - lo.y, 1e-20f), fmaxf(hi.z - lo.z, 1e-20f));
    f3 p = vx.p;
    const Bsdf& b = vx.bsdf;
    out[0] = make_float4(clampf((p.x - lo.x) / ext.x, 0.0f, 1.0f), clampf((p.y - lo.y) / ext.y, 0.0f, 1.0f),
                         clampf((p.z - lo.z) / ext.z, 0.0f, 1.0f), clampf(b.alpha, 0.0f, 1.0f));
    out[1] = make_float4(0.5f * (b.v.x + 1.0f), 0.5f * (b.v.y + 1.0f), 0.5f * (b.v.z + 1.0f), 0.0f);
    out[2] = make_float4(0.5f * (b.n.x + 1.0f), 0.5f * (b.n.y + 1.0f), 0.5f * (b.n.z + 1.0f), 0.0f);
}

// A finished training path: its target is the radiance gathered after the
// recorded vertex, per unit throughput there.
__device__ __forceinline__ void nrc_finish(const WaveArgs& a, uint32_t i, const PathCore& pc) {
    uint32_t ti = a.nrc.s_tidx[i];
    if (ti == NONE) return;
    a.nrc.s_tidx[i] = NONE;
    float4 pre = a.nrc.s_pre[i], b = a.nrc.s_beta[i];
    f3 d = pc.radiance - xyz(pre);
    float t[3] = {d.x, d.y, d.z}, bb[3] = {b.x, b.y, b.z};
    for (int c = 0; c < 3; c++) {
        float v = bb[c] > 0.0f ? t[c] / bb[c] : 0.0f;
        t[c] = finite(v) ? fmaxf(v, 0.0f) : 0.0f;
    }
    a.nrc.t_target[ti] = make_float4(t[0], t[1], t[2], 1.0f);
}

}  // namespace

template <bool COUNT, bool BATCH>
__global__ void __launch_bounds__(128, 4) split_logic(const __grid_constant__ WaveArgs a) {
    __shared__ uint32_t s_sobol[128];
    {
        const Scene& s0 = tables_of<BATCH>(a);
        for (uint32_t i = threadIdx.x; i < 128u; i += blockDim.x) s_sobol[i] = tw(s0, s0.P.offs0[0] + i);
    }
    __syncthreads();
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.slots) return;
    const uint32_t J = a.jobs;
    PathCore pc;
    Sampler smp;
    uint32_t stage = __float_as_uint(a.st.rad[i].w) & 3u;
    bool need_new = stage == ST_EMPTY;
    if (!need_new) {
        const Scene& s = slot_scene<BATCH>(a, i);
        load_state(a, i, &pc, &smp);
        uint32_t n = a.st.nee_n[i];
        if (a.st.vis) {
            // The unoccluded jobs' contributions, in job order.
            uint32_t m = n ? a.st.vis[i] : 0u;
            while (m) {
                uint32_t j = __ffs(m) - 1u;
                m &= m - 1u;
                if (j < n) pc.radiance = pc.radiance + xyz(a.st.pend[(uint64_t)i * J + j]);
            }
        } else {
            for (uint32_t j = 0; j < n; j++) {
                float4 pe = a.st.pend[(uint64_t)i * J + j];
                if (pe.w == 2.0f) pc.radiance = pc.radiance + xyz(pe);
            }
        }
        if (n) a.st.nee_n[i] = 0u;
        int r = PATH_DONE;
        if (stage == ST_TRACING) {
            uint32_t hmat;
            Hit hit = load_hit(a, i, &hmat);
            r = after_ray(s, pc, hit.slot != NONE, hit);
        }
        if (r == PATH_SURFACE) {
            save_state(a, i, pc, smp, ST_TRACING);
            a.q.shade[append1(&a.ctr[3])] = i;
            append1(&a.ctr[2]);
            return;
        }
        a.out[a.st.item[i]] = path_result(pc, r != PATH_UNCOVERED);
        if (a.nrc.on) nrc_finish(a, i, pc);
        need_new = true;
    }
    unsigned long long item = fetch1(a.work);
    if (item < a.total) {
        uint32_t f = BATCH ? frame_of1(a, item) : 0u;
        const Scene& s = BATCH ? a.frames[f].s : a.s;
        unsigned long long local = BATCH ? item - a.frames[f].base : item;
        uint32_t npix = BATCH ? a.frames[f].npix : a.npix;
        uint32_t y0 = BATCH ? a.frames[f].y0 : a.y0, first = BATCH ? a.frames[f].first : a.first;
        uint32_t it = (uint32_t)(local / npix);
        uint32_t q = (uint32_t)(local - (unsigned long long)it * npix);
        uint32_t yy = q / s.P.dims[0];
        f3 o = start_path(s, s_sobol, q - yy * s.P.dims[0], y0 + yy, first + it, &smp, &pc);
        a.st.item[i] = item;
        if (BATCH) a.st.frame[i] = f;
        if (a.nrc.on) {
            a.nrc.s_tidx[i] = NONE;
            a.nrc.s_tail[i] = NONE;
        }
        save_state(a, i, pc, smp, ST_TRACING);
        a.st.org[i] = make_float4(o.x, o.y, o.z, 0.0f);
        a.q.ext[append1(&a.ctr[0])] = i;
        append1(&a.ctr[2]);
        if (COUNT) atomicAdd(a.counters + C_PATHS, 1ull);
    } else if (stage != ST_EMPTY) {
        float4 r = a.st.rad[i];
        r.w = __uint_as_float(ST_EMPTY);
        a.st.rad[i] = r;
    }
}

template <bool COUNT, int MINB, bool BATCH>
__global__ void __launch_bounds__(128, MINB) split_shade(const __grid_constant__ WaveArgs a) {
    __shared__ uint32_t s_sobol[128];
    __shared__ float s_sheen[512];
    {
        const Scene& s0 = tables_of<BATCH>(a);
        for (uint32_t i = threadIdx.x; i < 128u; i += blockDim.x) s_sobol[i] = tw(s0, s0.P.offs0[0] + i);
        for (uint32_t i = threadIdx.x; i < 512u; i += blockDim.x) s_sheen[i] = tf(s0, s0.P.offs0[1] + i);
    }
    __syncthreads();
    const uint32_t n = *((volatile uint32_t*)&a.ctr[3]);
    unsigned long long shaded = 0;
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        uint32_t i = a.q.shade[q];
        const Scene& s = slot_scene<BATCH>(a, i);
        PathCore pc;
        Sampler smp;
        load_state(a, i, &pc, &smp);
        uint32_t hmat;
        Hit hit = load_hit(a, i, &hmat);
        Vertex vx;
        int r = shade_hit<COUNT>(s, s_sheen, s_sobol, smp, pc, hit, hmat, &vx, &shaded);
        if (r != PATH_VERTEX) {
            save_state(a, i, pc, smp, ST_ENDING);
            continue;
        }
        bool spread_ok = true;
        if (a.nrc.on) {
            // Path spread (Mueller et al. 2021): a0 = t^2 / (4 pi |cos|) at the
            // primary vertex, then the sum of sqrt(t^2 / (pdf |cos|)) over bounces.
            const float cosv = fabsf(dot(vx.ng, pc.d));
            float2 sp = pc.k == 0u ? make_float2(0.0f, 0.0f) : a.nrc.s_spread[i];
            if (pc.k == 0u) sp.x = hit.t * hit.t / (4.0f * PI * fmaxf(cosv, 1e-6f));
            else if (pc.prev_pdf > 0.0f && cosv > 0.0f) sp.y += sqrtf(hit.t * hit.t / (pc.prev_pdf * cosv));
            a.nrc.s_spread[i] = sp;
            spread_ok = a.nrc.spread <= 0.0f || sp.y * sp.y > a.nrc.spread * sp.x;
        }
        const uint32_t tail = a.nrc.on ? a.nrc.s_tail[i] : NONE;
        if (a.nrc.on && tail == pc.k && (smp.path_seed & a.nrc.train_mask) == 0u) {
            // A training path's suffix ends here, into the cache.
            float4 f[3];
            nrc_features(s, vx, f);
            uint32_t q = atomicAdd(&a.nrc.counts[0], 1u);
            if (q < a.nrc.q_cap) {
                a.nrc.q_in[3 * (size_t)q] = f[0];
                a.nrc.q_in[3 * (size_t)q + 1] = f[1];
                a.nrc.q_in[3 * (size_t)q + 2] = f[2];
                a.nrc.q_beta[q] = make_float4(pc.beta.x, pc.beta.y, pc.beta.z, 0.0f);
                a.nrc.q_item[q] = a.st.item[i];
                uint32_t ti = a.nrc.s_tidx[i];
                if (ti != NONE) {
                    float4 b0 = a.nrc.s_beta[i];
                    float rx = b0.x > 0.0f ? pc.beta.x / b0.x : 0.0f;
                    float ry = b0.y > 0.0f ? pc.beta.y / b0.y : 0.0f;
                    float rz = b0.z > 0.0f ? pc.beta.z / b0.z : 0.0f;
                    a.nrc.t_tail[ti] = make_uint4(q, __float_as_uint(rx), __float_as_uint(ry), __float_as_uint(rz));
                }
            }
            a.st.nee_n[i] = 0u;
            save_state(a, i, pc, smp, ST_ENDING);
            continue;
        }
        if (a.nrc.on && pc.k >= a.nrc.query_k && tail == NONE && spread_ok) {
            float4 f[3];
            nrc_features(s, vx, f);
            if ((smp.path_seed & a.nrc.train_mask) != 0u) {
                // A rendering path ends here: the cache supplies the rest.
                uint32_t q = atomicAdd(&a.nrc.counts[0], 1u);
                if (q < a.nrc.q_cap) {
                    a.nrc.q_in[3 * (size_t)q] = f[0];
                    a.nrc.q_in[3 * (size_t)q + 1] = f[1];
                    a.nrc.q_in[3 * (size_t)q + 2] = f[2];
                    a.nrc.q_beta[q] = make_float4(pc.beta.x, pc.beta.y, pc.beta.z, 0.0f);
                    a.nrc.q_item[q] = a.st.item[i];
                }
                a.st.nee_n[i] = 0u;
                save_state(a, i, pc, smp, ST_ENDING);
                continue;
            }
            a.nrc.s_tail[i] = a.nrc.suffix ? pc.k + a.nrc.suffix : 0xfffffffeu;
            uint32_t ti = atomicAdd(&a.nrc.counts[1], 1u);
            if (ti < a.nrc.t_cap) {
                a.nrc.t_in[3 * (size_t)ti] = f[0];
                a.nrc.t_in[3 * (size_t)ti + 1] = f[1];
                a.nrc.t_in[3 * (size_t)ti + 2] = f[2];
                a.nrc.t_target[ti] = make_float4(0.f, 0.f, 0.f, 0.f);
                a.nrc.t_tail[ti] = make_uint4(NONE, 0u, 0u, 0u);
                a.nrc.s_pre[i] = make_float4(pc.radiance.x, pc.radiance.y, pc.radiance.z, 0.0f);
                a.nrc.s_beta[i] = make_float4(pc.beta.x, pc.beta.y, pc.beta.z, 0.0f);
                a.nrc.s_tidx[i] = ti;
            }
        }
        uint32_t v = append1(&a.ctr[4]);
        put_vertex(a, v, vx, pc, smp.path_seed);
        a.q.vslot[v] = i;
        a.st.nee_n[i] = BATCH ? s.P.cfg[2] + 1u : a.jobs;
        f3 o;
        if (continue_path(s, s_sheen, s_sobol, smp, pc, vx, &o)) {
            save_state(a, i, pc, smp, ST_TRACING);
            a.st.org[i] = make_float4(o.x, o.y, o.z, 0.0f);
            a.q.ext[append1(&a.ctr[0])] = i;
        } else {
            save_state(a, i, pc, smp, ST_ENDING);
        }
    }
    if (COUNT && shaded) atomicAdd(a.counters + C_SHADED, shaded);
}

template <bool COUNT, int MINB, bool BATCH>
__global__ void __launch_bounds__(128, MINB) split_nee(const __grid_constant__ WaveArgs a) {
    __shared__ float s_sheen[512];
    {
        const Scene& s0 = tables_of<BATCH>(a);
        for (uint32_t i = threadIdx.x; i < 512u; i += blockDim.x) s_sheen[i] = tf(s0, s0.P.offs0[1] + i);
    }
    __syncthreads();
    const uint32_t nv = *((volatile uint32_t*)&a.ctr[4]);
    const uint64_t total = (uint64_t)nv * a.jobs;
    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t j = (uint32_t)(t / nv);
        uint32_t v = (uint32_t)(t - (uint64_t)j * nv);
        uint32_t slot = a.q.vslot[v];
        const Scene& s = slot_scene<BATCH>(a, slot);
        if (BATCH && j > s.P.cfg[2]) continue;  // beyond this scene's NEE jobs (its nee_n stops short)
        Vertex vx;
        PathCore pc;
        uint32_t path_seed;
        get_vertex(a, v, &vx, &pc, &path_seed);
        ShadowRay sr;
        float4 pe = make_float4(0.f, 0.f, 0.f, 0.f);
        if (a.st.vis && j == 0u) a.st.vis[slot] = 0u;
        bool queued = nee_job(s, s_sheen, pc, vx, j, &sr);
        if (queued) {
            pe = make_float4(sr.pending.x, sr.pending.y, sr.pending.z, 1.0f);
            uint32_t q = append1(&a.ctr[1]);
            a.q.sh_o[q] = make_float4(sr.o.x, sr.o.y, sr.o.z, sr.tmax);
            a.q.sh_d[q] = make_float4(sr.d.x, sr.d.y, sr.d.z, __uint_as_float(sr.skip));
            a.q.sh_m[q] = make_uint4(slot, j, sr.rid, path_seed);
        }
        if (queued || !a.st.vis) a.st.pend[(uint64_t)slot * a.jobs + j] = pe;
    }
}

// The same NEE jobs vertex-major: one thread per vertex loads its record
// once and runs every job in order, so the lanes of a warp still evaluate
// the same light together while the vertex array is read once instead of
// once per job. Each (vertex, job) computes what split_nee computes; only
// the order of the shadow queue changes (warp-sized runs per light).
template <bool COUNT, int MINB, bool BATCH>
__global__ void __launch_bounds__(128, MINB) split_nee_v(const __grid_constant__ WaveArgs a) {
    __shared__ float s_sheen[512];
    {
        const Scene& s0 = tables_of<BATCH>(a);
        for (uint32_t i = threadIdx.x; i < 512u; i += blockDim.x) s_sheen[i] = tf(s0, s0.P.offs0[1] + i);
    }
    __syncthreads();
    const uint32_t nv = *((volatile uint32_t*)&a.ctr[4]);
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
        uint32_t slot = a.q.vslot[v];
        const Scene& s = slot_scene<BATCH>(a, slot);
        const uint32_t J = BATCH ? min(a.jobs, s.P.cfg[2] + 1u) : a.jobs;  // this scene's NEE jobs
        Vertex vx;
        PathCore pc;
        uint32_t path_seed;
        get_vertex(a, v, &vx, &pc, &path_seed);
        if (a.st.vis) a.st.vis[slot] = 0u;
        for (uint32_t j = 0; j < J; j++) {
            ShadowRay sr;
            float4 pe = make_float4(0.f, 0.f, 0.f, 0.f);
            bool queued = nee_job(s, s_sheen, pc, vx, j, &sr);
            if (queued) {
                pe = make_float4(sr.pending.x, sr.pending.y, sr.pending.z, 1.0f);
                uint32_t q = append1(&a.ctr[1]);
                a.q.sh_o[q] = make_float4(sr.o.x, sr.o.y, sr.o.z, sr.tmax);
                a.q.sh_d[q] = make_float4(sr.d.x, sr.d.y, sr.d.z, __uint_as_float(sr.skip));
                a.q.sh_m[q] = make_uint4(slot, j, sr.rid, path_seed);
            }
            if (queued || !a.st.vis) a.st.pend[(uint64_t)slot * a.jobs + j] = pe;
        }
    }
}

// Variants: shade kernel for 2 / 3 / 4 resident blocks per SM; the NEE
// kernel job-major (0-2) or vertex-major (3-5) for 4 / 5 / 6.
template <bool C, bool B>
static void* shade_fn(int v) {
    if (v == 0) return (void*)split_shade<C, 2, B>;
    if (v == 1) return (void*)split_shade<C, 3, B>;
    return (void*)split_shade<C, 4, B>;
}
template <bool C, bool B>
static void* nee_fn(int v) {
    if (v == 0) return (void*)split_nee<C, 4, B>;
    if (v == 1) return (void*)split_nee<C, 5, B>;
    if (v == 2) return (void*)split_nee<C, 6, B>;
    if (v == 3) return (void*)split_nee_v<C, 4, B>;
    if (v == 4) return (void*)split_nee_v<C, 5, B>;
    return (void*)split_nee_v<C, 6, B>;
}

static cudaError_t persistent(void* fn, const WaveArgs& a, int sms, cudaStream_t st) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 128, 0);
    WaveArgs copy = a;
    void* args[] = {&copy};
    return cudaLaunchKernel(fn, dim3((unsigned)(sms * (per_sm > 0 ? per_sm : 1))), dim3(128), args, 0, st);
}

// Batched launches (a.nframes > 0) have no counting build.
cudaError_t launch_split_logic(const WaveArgs& a, bool count, cudaStream_t st) {
    unsigned blocks = (a.slots + 127u) / 128u;
    if (a.nframes) {
        if (count) return cudaErrorInvalidValue;
        split_logic<false, true><<<blocks, 128, 0, st>>>(a);
    } else if (count) {
        split_logic<true, false><<<blocks, 128, 0, st>>>(a);
    } else {
        split_logic<false, false><<<blocks, 128, 0, st>>>(a);
    }
    return cudaGetLastError();
}

cudaError_t launch_split_shade(const WaveArgs& a, bool count, int variant, int sms, cudaStream_t st) {
    variant = variant < 0 ? 0 : (variant > 2 ? 2 : variant);
    if (a.nframes) return count ? cudaErrorInvalidValue : persistent(shade_fn<false, true>(variant), a, sms, st);
    return persistent(count ? shade_fn<true, false>(variant) : shade_fn<false, false>(variant), a, sms, st);
}

cudaError_t launch_split_nee(const WaveArgs& a, bool count, int variant, int sms, cudaStream_t st) {
    variant = variant < 0 ? 0 : (variant > 5 ? 5 : variant);
    if (a.nframes) return count ? cudaErrorInvalidValue : persistent(nee_fn<false, true>(variant), a, sms, st);
    return persistent(count ? nee_fn<true, false>(variant) : nee_fn<false, false>(variant), a, sms, st);
}

#ifdef OXPT_FAST
}  // namespace fast
#endif
}  // namespace oxd
