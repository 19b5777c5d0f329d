// One path of the estimator, cut at its ray boundaries.
//
// trace_sample (pathtrace.wgsl:1714-2045) restated as four steps so that the
// megakernel (one thread runs all steps of a path in a loop) and the
// wavefront kernels (each step a separate launch over many paths, with the
// path state in HBM between launches) run the same arithmetic:
//   start_path     camera ray of sample `index` of pixel (x, y);
//   on_path_hit    the PATH branch after a continuation ray: medium
//                  attenuation, miss (environment / ambient), emission with
//                  MIS, unlit, the bounce limit, the BSDF of the vertex;
//   nee_job        one NEE job of a vertex (punctual light j, or the area /
//                  environment sample when j = n_punct): its contribution
//                  and shadow ray, if any;
//   continue_path  BSDF sampling, the medium transition and roulette.
// Radiance contributions are added in the reference's order: emission at a
// hit, then each unoccluded NEE contribution in job order, then whatever
// the next continuation ray finds.
#pragma once

#include "shade.cuh"

namespace oxd {

struct PathCore {
    f3 beta, radiance, prev_pos, sigma, d;
    float prev_pdf;
    uint32_t k;
    bool in_medium;
};

struct Vertex {
    Bsdf bsdf;
    f3 p, ng, atten_color;
    float thickness, transmission, atten_dist;
    bool front;
    float4 pl_u;
};

struct ShadowRay {
    f3 o, d, pending;
    float tmax;
    uint32_t rid, skip;
};

// Camera ray (pathtrace.wgsl:1715-1732). Returns the ray origin; the
// direction is pc->d.
__device__ __forceinline__ f3 start_path(const Scene& s, const uint32_t* sobol, uint32_t x, uint32_t y,
                                         uint32_t index, Sampler* smp, PathCore* pc) {
    *smp = make_sampler(s.P.dims[2], x, y, index);
    float4 p0 = pattern(sobol, *smp, 0u);
    float width = (float)s.P.dims[0], height = (float)s.P.dims[1];
    float ndc_x = (((float)x + p0.x) / fmaxf(width, 1.0f)) * 2.0f - 1.0f;
    float ndc_y = 1.0f - (((float)y + p0.y) / fmaxf(height, 1.0f)) * 2.0f;
    f3 eye = mk(s.P.eye[0], s.P.eye[1], s.P.eye[2]);
    f3 fwd = mk(s.P.forward[0], s.P.forward[1], s.P.forward[2]);
    f3 side = mk(s.P.side[0], s.P.side[1], s.P.side[2]);
    f3 up = mk(s.P.up[0], s.P.up[1], s.P.up[2]);
    float half_w = s.P.forward[3], half_h = s.P.side[3];
    f3 o;
    if (s.P.eye[3] > 0.5f) {
        o = eye + (side * (ndc_x * half_w) + up * (ndc_y * half_h));
        pc->d = fwd;
    } else {
        o = eye;
        pc->d = nrm(side * (ndc_x * half_w) + up * (ndc_y * half_h) + fwd);
    }
    pc->beta = sp(1.0f);
    pc->radiance = sp(0.0f);
    pc->prev_pdf = 0.0f;
    pc->prev_pos = sp(0.0f);
    pc->in_medium = false;
    pc->sigma = sp(0.0f);
    pc->k = 0u;
    return o;
}

enum HitOutcome { PATH_DONE = 0, PATH_UNCOVERED = 1, PATH_VERTEX = 2, PATH_SURFACE = 3 };

// The start of the PATH branch (pathtrace.wgsl:1773-1798): medium
// attenuation, then a miss (environment / ambient with MIS). PATH_SURFACE:
// a surface was hit and shade_hit follows.
__device__ __forceinline__ int after_ray(const Scene& s, PathCore& pc, bool got, const Hit& hit) {
    const uint32_t strategy = s.P.cfg[1];
    if (pc.in_medium) {
        if (!got) return PATH_DONE;
        f3 ex = -pc.sigma * hit.t;
        pc.beta = pc.beta * mk(fm_exp(ex.x), fm_exp(ex.y), fm_exp(ex.z));
    }
    if (!got) {
        if (pc.k == 0u) return PATH_UNCOVERED;
        f3 le = sp(s.P.fparams[0]);
        float w = 1.0f;
        if (s.P.env[2] != 0u) {
            Texel t = env_texel(s, pc.d);
            le = env_radiance_at(s, t);
            if (strategy == 0u) w = power_heuristic(pc.prev_pdf, s.P.fparams[2] * env_pdf_at(s, t));
            else if (strategy == 1u) w = 0.0f;
        }
        if (w > 0.0f) pc.radiance = pc.radiance + clamp_c(s, pc.beta * le * w);
        return PATH_DONE;
    }
    return PATH_SURFACE;
}

// The rest of the PATH branch at a surface hit (pathtrace.wgsl:1799-1861):
// emission with MIS, unlit, the bounce limit and the vertex's BSDF.
// PATH_VERTEX: *v holds the vertex and NEE / BSDF sampling follow.
template <bool COUNT>
__device__ __forceinline__ int shade_hit(const Scene& s, const float* sheen, const uint32_t* sobol,
                                         const Sampler& smp, PathCore& pc, const Hit& hit, uint32_t hmat,
                                         Vertex* v, unsigned long long* shaded) {
    const uint32_t strategy = s.P.cfg[1];
    if (COUNT) *shaded += 1;
    Surface surf = surface(s, hit.slot, hit.b);
    uint32_t mflags = mat_flags(s, hmat);
    bool double_sided = (mflags & 4u) != 0u;
    Lod lod = base_lod();
    if (pc.k == 0u) {
        float cw = s.P.eye[3] > 0.5f ? s.P.up[3] : s.P.up[3] * hit.t;
        lod = {cw, pc.d};
    }
    bool flip = !hit.front && double_sided;
    Mat mat = material(s, hit.slot, hmat, hit.b, surf.sn, lod, flip);
    if (flip) {
        mat.normal = -mat.normal;
        mat.cc_normal = -mat.cc_normal;
    }
    if ((hit.front || double_sided) && !is_black(mat.emission)) {
        f3 le = mat.emission;
        if (pc.k == 0u) {
            pc.radiance = pc.radiance + pc.beta * le;
        } else {
            uint32_t li = tri_word(s, hit.slot, 1u);
            float pl = li == NONE ? 0.0f : tri_pdf(s, li, hit.slot, pc.prev_pos, surf.position);
            float w = 1.0f;
            if (pl > 0.0f) {
                if (strategy == 0u) w = power_heuristic(pc.prev_pdf, pl);
                else if (strategy == 1u) w = 0.0f;
            }
            if (w > 0.0f) pc.radiance = pc.radiance + clamp_c(s, pc.beta * le * w);
        }
    }
    if (mat.unlit) {
        f3 contrib = pc.beta * xyz(mat.base);
        pc.radiance = pc.radiance + (pc.k == 0u ? contrib : clamp_c(s, contrib));
        return PATH_DONE;
    }
    if (pc.k >= s.P.dims[3]) return PATH_DONE;
    v->bsdf = make_bsdf(sheen, mat, -pc.d, surf.ng, hit.front);
    if (bsdf_black(v->bsdf)) return PATH_DONE;
    v->p = surf.position;
    v->ng = v->bsdf.ng;
    v->thickness = mat.thickness;
    v->transmission = mat.transmission;
    v->atten_color = mat.atten_color;
    v->atten_dist = mat.atten_dist;
    v->front = hit.front;
    v->pl_u = pattern(sobol, smp, 2u + 2u * pc.k);
    return PATH_VERTEX;
}

// The whole PATH branch after a continuation ray.
template <bool COUNT>
__device__ __forceinline__ int on_path_hit(const Scene& s, const float* sheen, const uint32_t* sobol,
                                           const Sampler& smp, PathCore& pc, bool got, const Hit& hit,
                                           uint32_t hmat, Vertex* v, unsigned long long* shaded) {
    int r = after_ray(s, pc, got, hit);
    if (r != PATH_SURFACE) return r;
    return shade_hit<COUNT>(s, sheen, sobol, smp, pc, hit, hmat, v, shaded);
}

// NEE job `job` of vertex v (pathtrace.wgsl:1863-1993). True when it arms
// a shadow ray whose pending contribution is sr->pending.
__device__ __forceinline__ bool nee_job(const Scene& s, const float* sheen, const PathCore& pc, const Vertex& v,
                                        uint32_t job, ShadowRay* sr) {
    const uint32_t strategy = s.P.cfg[1];
    const bool has_env = s.P.env[2] != 0u;
    const uint32_t n_elights = s.P.cfg[3], n_punct = s.P.cfg[2];
    const uint32_t ray_id = pc.k << 16u;
    bool ok = false;
    f3 l = sp(0.0f);
    float tmax = INF;
    uint32_t rid = ray_id | 0xffffu, skip = NONE;
    f3 le = sp(0.0f);
    float pl = -1.0f;
    const f3 p = v.p;
    const float4 pl_u = v.pl_u;
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
    if (!ok) return false;
    Eval e = bsdf_eval(sheen, v.bsdf, l);
    if (is_black(e.f) || is_black(le)) return false;
    if (pl < 0.0f) {
        sr->pending = clamp_c(s, pc.beta * e.f * le);
    } else {
        float w = strategy == 0u ? power_heuristic(pl, e.pdf) : 1.0f;
        sr->pending = clamp_c(s, pc.beta * e.f * le * (w / pl));
    }
    sr->o = spawn(p, v.ng, l);
    sr->d = l;
    sr->tmax = tmax;
    sr->rid = rid;
    sr->skip = skip;
    return true;
}

// BSDF sampling, medium transition and roulette (pathtrace.wgsl:1999-2039).
// False when the path ends; otherwise pc.d is the new direction, pc.k the
// new bounce and the new ray origin is returned through *origin.
__device__ __forceinline__ bool continue_path(const Scene& s, const float* sheen, const uint32_t* sobol,
                                              const Sampler& smp, PathCore& pc, const Vertex& v, f3* origin) {
    float4 pb_u = pattern(sobol, smp, 1u + 2u * pc.k);
    BSample bs = bsdf_sample(sheen, v.bsdf, pb_u.x, pb_u.y, pb_u.z);
    if (!bs.ok) return false;
    pc.beta = pc.beta * (bs.f * (1.0f / bs.pdf));
    if (!finite3(pc.beta)) return false;
    pc.prev_pdf = bs.pdf;
    pc.prev_pos = v.p;
    if (dot(bs.l, v.ng) < 0.0f && v.thickness > 0.0f && v.transmission > 0.0f) {
        if (v.front && v.atten_dist >= 0.0f) {
            f3 la = vmax(v.atten_color, sp(1.0e-6f));
            pc.sigma = -mk(fm_log(la.x), fm_log(la.y), fm_log(la.z)) / v.atten_dist;
            pc.in_medium = true;
        } else {
            pc.in_medium = false;
        }
    }
    if (pc.k + 1u >= s.P.cfg[0]) {
        float q = clampf(max3(pc.beta), 0.05f, 1.0f);
        if (q < 1.0f) {
            if (pb_u.w >= q) return false;
            pc.beta = pc.beta * (1.0f / q);
        }
    }
    pc.k += 1u;
    pc.d = bs.l;
    *origin = spawn(v.p, v.ng, bs.l);
    return true;
}

// The accumulated value of a finished path (pathtrace.wgsl:2041-2044).
__device__ __forceinline__ float4 path_result(const PathCore& pc, bool covered) {
    if (!covered) return make_float4(0.f, 0.f, 0.f, 0.f);
    if (finite3(pc.radiance)) return make_float4(pc.radiance.x, pc.radiance.y, pc.radiance.z, 1.0f);
    return make_float4(0.f, 0.f, 0.f, 1.0f);
}

}  // namespace oxd
