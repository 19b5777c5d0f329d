// Path-tracing kernels for sm_100a.
//
// trace_paths: a persistent megakernel. The grid is sized to the resident
// capacity of the GPU; each thread owns one path slot and, whenever its
// path ends, regenerates the slot with its next (pixel, sample) item
// (grid-stride over samples-major, pixels-minor items, so that the lanes
// of a warp start on neighbouring pixels of the same sample). Every loop
// iteration traces exactly one ray — the path's continuation ray or one
// NEE shadow ray — through a single traversal call site, as the reference
// megakernel does (pathtrace.wgsl:1702-2045), so lanes that are shading,
// shadowing or starting a new camera ray all meet at the same traversal.
// The result of every path is written to a per-launch buffer and
// reduce_frame then adds them into the accumulator in sample order,
// which keeps each pixel's float summation identical to the reference's
// per-pixel loop (pathtrace.wgsl:2064-2072) whatever the launch split.
//
// Traversal follows the reference's ordered walk (near child first, far
// child pushed with its entry distance, pops culled against t_max;
// pathtrace.wgsl:651-735) over the same node layout, but fetches the two
// children of an inner node as one 64-byte pair, carries the chosen child
// in registers and pushes (first, count) instead of a node index, so an
// inner node costs one dependent fetch instead of three.
#include "kernels.cuh"
#include "shade.cuh"

namespace oxd {

struct Cnt {
    unsigned long long c[C_N];
};

template <bool COUNT>
__device__ __forceinline__ void bump(Cnt& c, int k, unsigned long long v = 1) {
    if (COUNT) c.c[k] += v;
}

// Any-hit acceptance (pathtrace.wgsl:621-636).
__device__ __forceinline__ bool accept(const Scene& s, uint32_t slot, uint32_t m, uint32_t gid, const Hit& h,
                                       const Sampler& smp, uint32_t ray_id, bool primary) {
    uint32_t fl = mat_flags(s, m);
    if (primary && !h.front && (fl & 4u) == 0u) return false;
    uint32_t mode = fl & 3u;
    if (mode == 0u) return true;
    if (mode == 1u) return hit_alpha(s, slot, m, h.b) >= tf(s, mat_off(s, m) + 11u);
    return coin(smp, ray_id, gid) < hit_alpha(s, slot, m, h.b);
}

// Closest-hit (any = false) or any-hit (any = true) query. Returns whether
// something was hit; *best holds the hit and *best_mat its material.
template <bool COUNT>
__device__ bool traverse(const Scene& s, const Ray& r, float t_max, const Sampler& smp, uint32_t ray_id,
                         bool primary, bool any, uint32_t skip, Hit* best, uint32_t* best_mat, Cnt& cnt,
                         uint32_t* err) {
    best->slot = NONE;
    uint32_t node_count = s.P.env[3];
    if (node_count == 0u || !r.valid) return false;
    float4 rlo = geomv(s, 0), rhi = geomv(s, 1);
    bump<COUNT>(cnt, C_BOXES);
    if (slab(r, rlo, rhi, t_max) < 0.0f) return false;
    uint32_t cur_first = __float_as_uint(rlo.w), cur_count = __float_as_uint(rhi.w);
    uint2 st_fc[STACK];
    float st_t[STACK];
    uint32_t sp = 0u;
    // A tree visits each node at most once; anything longer is a malformed
    // BVH, reported through the error word instead of looping.
    uint32_t guard = node_count + 8u;
    bool hit_any = false;
    for (;;) {
        if (guard-- == 0u) {
            atomicOr(err, 1u);
            best->slot = NONE;
            return false;
        }
        if (cur_count > 0u) {
            bump<COUNT>(cnt, C_LEAVES);
            if ((uint64_t)cur_first + cur_count > s.slot_count) {  // malformed leaf
                atomicOr(err, 2u);
                best->slot = NONE;
                return false;
            }
            uint32_t end = cur_first + cur_count;
            for (uint32_t slot = cur_first; slot < end; slot++) {
                bump<COUNT>(cnt, C_TRIS);
                uint64_t tb = tri_base(s, slot);
                float4 q0 = geomv(s, tb), q1 = geomv(s, tb + 1), q2 = geomv(s, tb + 2);
                Hit h;
                if (!intersect(r, q0, q1, q2, t_max, &h)) continue;
                uint32_t gid = __float_as_uint(q0.w);
                if (gid == skip) continue;
                uint32_t m = __float_as_uint(q2.w);
                if (!accept(s, slot, m, gid, h, smp, ray_id, primary)) continue;
                h.slot = slot;
                *best = h;
                *best_mat = m;
                hit_any = true;
                if (any) return true;
                t_max = h.t;
            }
        } else {
            bump<COUNT>(cnt, C_BOXES, 2);
            uint64_t l = cur_first;
            float4 alo = geomv(s, 2 * l), ahi = geomv(s, 2 * l + 1);
            float4 blo = geomv(s, 2 * l + 2), bhi = geomv(s, 2 * l + 3);
            float tl = slab(r, alo, ahi, t_max);
            float tr = slab(r, blo, bhi, t_max);
            if (tl >= 0.0f && tr >= 0.0f) {
                bool swap = tl > tr;
                uint2 nearfc = swap ? make_uint2(__float_as_uint(blo.w), __float_as_uint(bhi.w))
                                    : make_uint2(__float_as_uint(alo.w), __float_as_uint(ahi.w));
                uint2 farfc = swap ? make_uint2(__float_as_uint(alo.w), __float_as_uint(ahi.w))
                                   : make_uint2(__float_as_uint(blo.w), __float_as_uint(bhi.w));
                if (sp < (uint32_t)STACK) {
                    st_fc[sp] = farfc;
                    st_t[sp] = swap ? tl : tr;
                    sp++;
                }
                cur_first = nearfc.x;
                cur_count = nearfc.y;
                continue;
            } else if (tl >= 0.0f) {
                cur_first = __float_as_uint(alo.w);
                cur_count = __float_as_uint(ahi.w);
                continue;
            } else if (tr >= 0.0f) {
                cur_first = __float_as_uint(blo.w);
                cur_count = __float_as_uint(bhi.w);
                continue;
            }
        }
        bool found = false;
        while (sp != 0u) {
            sp--;
            bump<COUNT>(cnt, C_POPS);
            if (st_t[sp] <= t_max) {
                cur_first = st_fc[sp].x;
                cur_count = st_fc[sp].y;
                found = true;
                break;
            }
        }
        if (!found) break;
    }
    return hit_any;
}

template <bool COUNT>
__global__ void __launch_bounds__(TRACE_THREADS) trace_paths(const __grid_constant__ TraceArgs a) {
    __shared__ uint32_t s_sobol[128];
    __shared__ float s_sheen[512];
    const Scene& s = a.s;
    for (uint32_t i = threadIdx.x; i < 128u; i += blockDim.x) s_sobol[i] = tw(s, s.P.offs0[0] + i);
    for (uint32_t i = threadIdx.x; i < 512u; i += blockDim.x) s_sheen[i] = tf(s, s.P.offs0[1] + i);
    __syncthreads();

    Cnt cnt;
    if (COUNT)
        for (int k = 0; k < C_N; k++) cnt.c[k] = 0;

    const uint32_t W = s.P.dims[0];
    const uint32_t strategy = s.P.cfg[1];
    const bool has_env = s.P.env[2] != 0u;
    const uint32_t n_elights = s.P.cfg[3], n_punct = s.P.cfg[2];
    const bool orthographic = s.P.eye[3] > 0.5f;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;

    uint64_t item = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    bool live = false;
    // Path state (trace_sample's locals, pathtrace.wgsl:1715-1764).
    Sampler smp{0u, 0u, 0u};
    f3 d = sp(0.0f), beta = sp(1.0f), radiance = sp(0.0f), prev_pos = sp(0.0f), sigma = sp(0.0f);
    float prev_pdf = 0.0f;
    bool in_medium = false, shadow = false;
    uint32_t k = 0u, r_id = 0u, r_skip = NONE, job = 0u;
    f3 r_o = sp(0.0f), r_d = sp(0.0f), pending = sp(0.0f);
    float r_tmax = INF;
    Bsdf bsdf;
    f3 p = sp(0.0f), ng = sp(0.0f), atten_color = sp(1.0f);
    float thickness = 0.0f, transmission = 0.0f, atten_dist = -1.0f;
    bool front = true;
    float4 pl_u = make_float4(0.f, 0.f, 0.f, 0.f);

    for (;;) {
        if (!live) {
            if (item >= a.total) break;
            uint32_t i = (uint32_t)(item / a.npix);
            uint32_t q = (uint32_t)(item - (uint64_t)i * a.npix);
            uint32_t yy = q / W;
            uint32_t x = q - yy * W, y = a.y0 + yy;
            smp = make_sampler(s.P.dims[2], x, y, a.first + i);
            float4 p0 = pattern(s_sobol, smp, 0u);
            float width = (float)s.P.dims[0], height = (float)s.P.dims[1];
            float ndc_x = (((float)x + p0.x) / fmaxf(width, 1.0f)) * 2.0f - 1.0f;
            float ndc_y = 1.0f - (((float)y + p0.y) / fmaxf(height, 1.0f)) * 2.0f;
            f3 eye = mk(s.P.eye[0], s.P.eye[1], s.P.eye[2]);
            f3 fwd = mk(s.P.forward[0], s.P.forward[1], s.P.forward[2]);
            f3 side = mk(s.P.side[0], s.P.side[1], s.P.side[2]);
            f3 up = mk(s.P.up[0], s.P.up[1], s.P.up[2]);
            float half_w = s.P.forward[3], half_h = s.P.side[3];
            if (orthographic) {
                r_o = eye + (side * (ndc_x * half_w) + up * (ndc_y * half_h));
                d = fwd;
            } else {
                r_o = eye;
                d = nrm(side * (ndc_x * half_w) + up * (ndc_y * half_h) + fwd);
            }
            beta = sp(1.0f);
            radiance = sp(0.0f);
            prev_pdf = 0.0f;
            prev_pos = sp(0.0f);
            in_medium = false;
            sigma = sp(0.0f);
            k = 0u;
            shadow = false;
            r_d = d;
            r_tmax = INF;
            r_id = 0u;
            r_skip = NONE;
            pending = sp(0.0f);
            p = sp(0.0f);
            ng = sp(0.0f);
            thickness = 0.0f;
            transmission = 0.0f;
            atten_color = sp(1.0f);
            atten_dist = -1.0f;
            front = true;
            pl_u = make_float4(0.f, 0.f, 0.f, 0.f);
            job = 0u;
            live = true;
            bump<COUNT>(cnt, C_PATHS);
        }

        bump<COUNT>(cnt, shadow ? C_SHADOW_RAYS : C_PATH_RAYS);
        Hit hit;
        uint32_t hmat = 0u;
        bool got = traverse<COUNT>(s, make_ray(r_o, r_d), r_tmax, smp, r_id, !shadow && k == 0u, shadow, r_skip,
                                   &hit, &hmat, cnt, a.err);
        bool done = false, covered = true;
        if (shadow) {
            if (!got) radiance = radiance + pending;
            job += 1u;
        } else {
            if (in_medium) {
                if (!got) {
                    done = true;
                } else {
                    f3 ex = -sigma * hit.t;
                    beta = beta * mk(fm_exp(ex.x), fm_exp(ex.y), fm_exp(ex.z));
                }
            }
            if (!done && !got) {
                if (k == 0u) {
                    covered = false;
                } else {
                    f3 le = sp(s.P.fparams[0]);
                    float w = 1.0f;
                    if (has_env) {
                        Texel t = env_texel(s, d);
                        le = env_radiance_at(s, t);
                        if (strategy == 0u) w = power_heuristic(prev_pdf, s.P.fparams[2] * env_pdf_at(s, t));
                        else if (strategy == 1u) w = 0.0f;
                    }
                    if (w > 0.0f) radiance = radiance + clamp_c(s, beta * le * w);
                }
                done = true;
            }
            if (!done) {
                bump<COUNT>(cnt, C_SHADED);
                Surface surf = surface(s, hit.slot, hit.b);
                uint32_t mflags = mat_flags(s, hmat);
                bool double_sided = (mflags & 4u) != 0u;
                Lod lod = base_lod();
                if (k == 0u) {
                    float cw = orthographic ? s.P.up[3] : s.P.up[3] * hit.t;
                    lod = {cw, d};
                }
                bool flip = !hit.front && double_sided;
                Mat mat = material(s, hit.slot, hmat, hit.b, surf.sn, lod, flip);
                if (flip) {
                    mat.normal = -mat.normal;
                    mat.cc_normal = -mat.cc_normal;
                }
                if ((hit.front || double_sided) && !is_black(mat.emission)) {
                    f3 le = mat.emission;
                    if (k == 0u) {
                        radiance = radiance + beta * le;
                    } else {
                        uint32_t li = tri_word(s, hit.slot, 1u);
                        float pl = li == NONE ? 0.0f : tri_pdf(s, li, hit.slot, prev_pos, surf.position);
                        float w = 1.0f;
                        if (pl > 0.0f) {
                            if (strategy == 0u) w = power_heuristic(prev_pdf, pl);
                            else if (strategy == 1u) w = 0.0f;
                        }
                        if (w > 0.0f) radiance = radiance + clamp_c(s, beta * le * w);
                    }
                }
                if (mat.unlit) {
                    f3 contrib = beta * xyz(mat.base);
                    radiance = radiance + (k == 0u ? contrib : clamp_c(s, contrib));
                    done = true;
                } else if (k >= s.P.dims[3]) {
                    done = true;
                } else {
                    bsdf = make_bsdf(s_sheen, mat, -d, surf.ng, hit.front);
                    if (bsdf_black(bsdf)) {
                        done = true;
                    } else {
                        p = surf.position;
                        ng = bsdf.ng;
                        thickness = mat.thickness;
                        transmission = mat.transmission;
                        atten_color = mat.atten_color;
                        atten_dist = mat.atten_dist;
                        front = hit.front;
                        pl_u = pattern(s_sobol, smp, 2u + 2u * k);
                        job = 0u;
                    }
                }
            }
        }

        if (!done) {
            // Next NEE shadow ray: punctual lights in order, then the
            // area / environment sample (pathtrace.wgsl:1863-1997).
            bool armed = false;
            uint32_t ray_id = k << 16u;
            while (job <= n_punct) {
                bool ok = false;
                f3 l = sp(0.0f);
                float tmax = INF;
                uint32_t rid = ray_id | 0xffffu, skip = NONE;
                f3 le = sp(0.0f);
                float pl = -1.0f;
                if (job < n_punct) {
                    LightSample ls = punctual_sample(s, job, p);
                    if (ls.ok) {
                        ok = true;
                        l = ls.l;
                        if (ls.distance >= 0.0f) tmax = ls.distance * (1.0f - 1.0e-4f);
                        rid = ray_id | 0x8000u | (job & 0x7fffu);
                        le = ls.radiance;
                    }
                } else if (strategy != 2u && (has_env || n_elights > 0u)) {
                    float pe = s.P.fparams[2];
                    if (pl_u.z < pe) {
                        if (has_env) {
                            EnvSample es = env_sample(s, pl_u.x, pl_u.y);
                            if (es.ok && pe * es.pdf > 0.0f) {
                                ok = true;
                                l = es.d;
                                le = es.le;
                                pl = pe * es.pdf;
                            }
                        }
                    } else if (n_elights > 0u) {
                        float us = pl_u.z;
                        if (pe > 0.0f) us = clampf((pl_u.z - pe) / (1.0f - pe), 0.0f, 0.999999f);
                        uint32_t li = partition_point(s, s.P.offs1[0], n_elights, us, 4u);
                        li = li < n_elights - 1u ? li : n_elights - 1u;
                        uint32_t lslot = tw(s, s.P.offs1[0] + 4u * li + 3u);
                        f3 ta = tri_pos(s, lslot, 0u), tb = tri_pos(s, lslot, 1u), tc = tri_pos(s, lslot, 2u);
                        bool has_target = false;
                        f3 q = sp(0.0f);
                        if (triangle_solid_angle(p, ta, tb, tc) >= MIN_SPHERICAL_SOLID_ANGLE) {
                            f3 sl = sample_spherical_triangle(p, ta, tb, tc, pl_u.x, pl_u.y);
                            if (dot(sl, sl) > 0.0f) {
                                f3 n = cross(tb - ta, tc - ta);
                                float dn = dot(sl, n);
                                if (dn != 0.0f) {
                                    float t = dot(ta - p, n) / dn;
                                    if (t > 0.0f && finite(t)) {
                                        q = p + sl * t;
                                        has_target = true;
                                    }
                                }
                            }
                        } else {
                            float su = sqrtf(pl_u.x);
                            f3 w3 = mk(1.0f - su, su * (1.0f - pl_u.y), su * pl_u.y);
                            q = ta * w3.x + tb * w3.y + tc * w3.z;
                            has_target = true;
                        }
                        if (has_target) {
                            f3 e1 = tb - ta, e2 = tc - ta, rr = q - ta;
                            float d11 = dot(e1, e1), d12 = dot(e1, e2), d22 = dot(e2, e2);
                            float r1 = dot(rr, e1), r2 = dot(rr, e2);
                            float det = d11 * d22 - d12 * d12;
                            f3 to = q - p;
                            float dist2 = dot(to, to);
                            if (finite(det) && fabsf(det) > 1.17549435e-38f && dist2 > 1.0e-12f) {
                                float bu = (d22 * r1 - d12 * r2) / det;
                                float bv = (d11 * r2 - d12 * r1) / det;
                                f3 lb = vmin(vmax(mk(1.0f - bu - bv, bu, bv), sp(0.0f)), sp(1.0f));
                                f3 lng = surface(s, lslot, lb).ng;
                                uint32_t lm = tri_word(s, lslot, 2u);
                                bool lds = (mat_flags(s, lm) & 4u) != 0u;
                                float dist = sqrtf(dist2);
                                f3 ld = to / dist;
                                float cos_l = -dot(lng, ld);
                                float tp = tri_pdf(s, li, lslot, p, q);
                                if ((cos_l > 0.0f || (lds && cos_l < 0.0f)) && tp > 0.0f && finite(tp)) {
                                    ok = true;
                                    l = ld;
                                    le = emission_of(s, lslot, lm, lb);
                                    pl = tp;
                                    tmax = fmaxf(dist * (1.0f - 1.0e-4f), 0.0f);
                                    skip = tri_word(s, lslot, 0u);
                                }
                            }
                        }
                    }
                }
                if (ok) {
                    Eval e = bsdf_eval(s_sheen, bsdf, l);
                    if (!is_black(e.f) && !is_black(le)) {
                        if (pl < 0.0f) {
                            pending = clamp_c(s, beta * e.f * le);
                        } else {
                            float w = strategy == 0u ? power_heuristic(pl, e.pdf) : 1.0f;
                            pending = clamp_c(s, beta * e.f * le * (w / pl));
                        }
                        r_o = spawn(p, ng, l);
                        r_d = l;
                        r_tmax = tmax;
                        r_id = rid;
                        r_skip = skip;
                        armed = true;
                        break;
                    }
                }
                job += 1u;
            }
            if (armed) {
                shadow = true;
            } else {
                // BSDF sampling -> next path ray (pathtrace.wgsl:1999-2039).
                float4 pb_u = pattern(s_sobol, smp, 1u + 2u * k);
                BSample bs = bsdf_sample(s_sheen, bsdf, pb_u.x, pb_u.y, pb_u.z);
                if (!bs.ok) {
                    done = true;
                } else {
                    beta = beta * (bs.f * (1.0f / bs.pdf));
                    if (!finite3(beta)) {
                        done = true;
                    } else {
                        prev_pdf = bs.pdf;
                        prev_pos = p;
                        if (dot(bs.l, ng) < 0.0f && thickness > 0.0f && transmission > 0.0f) {
                            if (front && atten_dist >= 0.0f) {
                                f3 la = vmax(atten_color, sp(1.0e-6f));
                                sigma = -mk(fm_log(la.x), fm_log(la.y), fm_log(la.z)) / atten_dist;
                                in_medium = true;
                            } else {
                                in_medium = false;
                            }
                        }
                        if (k + 1u >= s.P.cfg[0]) {
                            float qq = clampf(max3(beta), 0.05f, 1.0f);
                            if (qq < 1.0f) {
                                if (pb_u.w >= qq) done = true;
                                else beta = beta * (1.0f / qq);
                            }
                        }
                        if (!done) {
                            k += 1u;
                            d = bs.l;
                            shadow = false;
                            r_o = spawn(p, ng, bs.l);
                            r_d = d;
                            r_tmax = INF;
                            r_id = k << 16u;
                            r_skip = NONE;
                        }
                    }
                }
            }
        }

        if (done) {
            float4 res = make_float4(0.f, 0.f, 0.f, 0.f);
            if (covered) {
                if (finite3(radiance)) res = make_float4(radiance.x, radiance.y, radiance.z, 1.0f);
                else res = make_float4(0.f, 0.f, 0.f, 1.0f);
            }
            a.out[item] = res;
            item += stride;
            live = false;
        }
    }
    if (COUNT) {
        for (int c = 0; c < C_N; c++) {
            unsigned long long v = cnt.c[c];
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
            if ((threadIdx.x & 31u) == 0u && v) atomicAdd(a.counters + c, v);
        }
    }
}

// Ordered accumulation: samples of one launch added to each pixel in
// sample order (pathtrace.wgsl:2065-2072).
__global__ void reduce_frame(const ReduceArgs a) {
    uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= a.npix) return;
    uint64_t idx = (uint64_t)a.y0 * a.w + q;
    float4 acc = a.accum[idx];
    for (uint32_t i = 0; i < a.count; i++) {
        float4 r = __ldcs(a.out + (uint64_t)i * a.npix + q);
        if (r.w > 0.0f) acc = make_float4(acc.x + r.x, acc.y + r.y, acc.z + r.z, acc.w + 1.0f);
    }
    a.accum[idx] = acc;
}

template <bool COUNT>
__global__ void __launch_bounds__(128) trace_rays(const __grid_constant__ RayArgs a) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    Cnt cnt;
    if (COUNT)
        for (int k = 0; k < C_N; k++) cnt.c[k] = 0;
    if (i < a.n) {
        const float* r = a.rays + i * 8;
        Sampler smp{0u, 0u, 0u};
        Hit h;
        uint32_t m = 0;
        bool got = traverse<COUNT>(a.s, make_ray(mk(r[0], r[1], r[2]), mk(r[4], r[5], r[6])), r[3], smp, 0u,
                                   (a.flags & 2u) != 0u, (a.flags & 1u) != 0u, __float_as_uint(r[7]), &h, &m, cnt,
                                   a.err);
        if (a.slot) a.slot[i] = got ? h.slot : NONE;
        if (a.gid) a.gid[i] = got ? tri_word(a.s, h.slot, 0u) : NONE;
        if (a.t) a.t[i] = got ? h.t : 0.0f;
        if (a.bary) {
            a.bary[i * 3] = got ? h.b.x : 0.0f;
            a.bary[i * 3 + 1] = got ? h.b.y : 0.0f;
            a.bary[i * 3 + 2] = got ? h.b.z : 0.0f;
        }
    }
    if (COUNT)
        for (int c = 0; c < C_N; c++)
            if (cnt.c[c]) atomicAdd(a.counters + c, cnt.c[c]);
}

__global__ void sobol_points(const uint32_t* dirs, uint32_t seed, uint64_t n, const uint32_t* x, const uint32_t* y,
                             const uint32_t* idx, const uint32_t* pat, uint32_t* out) {
    __shared__ uint32_t sd[128];
    for (uint32_t i = threadIdx.x; i < 128u; i += blockDim.x) sd[i] = dirs[i];
    __syncthreads();
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Sampler smp = make_sampler(seed, x[i], y[i], idx[i]);
    uint32_t u[4];
    pattern_u(sd, smp, pat[i], u);
    reinterpret_cast<uint4*>(out)[i] = make_uint4(u[0], u[1], u[2], u[3]);
}

__global__ void math_kernel(int op, uint64_t n, const float* a, const float* b, float* out) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float x = a[i], y = b ? b[i] : 0.0f, r = 0.0f;
    switch (op) {
        case 0: r = fm_sin(x); break;
        case 1: r = fm_cos(x); break;
        case 2: r = fm_acos(x); break;
        case 3: r = fm_atan2(x, y); break;
        case 4: r = fm_exp(x); break;
        case 5: r = fm_log(x); break;
        case 6: r = fm_log2(x); break;
        case 7: r = fm_pow(x, y); break;
        default: r = 0.0f;
    }
    out[i] = r;
}

cudaError_t launch_trace(const TraceArgs& a, bool count, uint32_t blocks, uint32_t threads, cudaStream_t st) {
    if (count) trace_paths<true><<<blocks, threads, 0, st>>>(a);
    else trace_paths<false><<<blocks, threads, 0, st>>>(a);
    return cudaGetLastError();
}

int trace_blocks_per_sm(uint32_t threads, bool count) {
    int n = 0;
    if (count) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, trace_paths<true>, (int)threads, 0);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, trace_paths<false>, (int)threads, 0);
    return n;
}

cudaError_t launch_reduce(const ReduceArgs& a, cudaStream_t st) {
    uint32_t blocks = (a.npix + 255u) / 256u;
    reduce_frame<<<blocks, 256, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_rays(const RayArgs& a, cudaStream_t st) {
    if (a.n == 0) return cudaSuccess;
    uint64_t blocks = (a.n + 127) / 128;
    if (a.counters) trace_rays<true><<<(unsigned)blocks, 128, 0, st>>>(a);
    else trace_rays<false><<<(unsigned)blocks, 128, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_sobol(const uint32_t* dirs, uint32_t seed, uint64_t n, const uint32_t* x, const uint32_t* y,
                         const uint32_t* idx, const uint32_t* pat, uint32_t* out, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    sobol_points<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(dirs, seed, n, x, y, idx, pat, out);
    return cudaGetLastError();
}

cudaError_t launch_math(int op, uint64_t n, const float* a, const float* b, float* out, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    math_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(op, n, a, b, out);
    return cudaGetLastError();
}

}  // namespace oxd
