// Device shading: surface, material, layered BSDF and light sampling
// (pathtrace.wgsl:765-1654), same arithmetic as the reference estimator.
#pragma once

#include "device.cuh"

namespace oxd {

struct Surface {
    f3 position, ng, sn;
};
static __device__ Surface surface(const Scene& s, uint32_t slot, f3 b) {
    f3 p0 = tri_pos(s, slot, 0u), p1 = tri_pos(s, slot, 1u), p2 = tri_pos(s, slot, 2u);
    Surface o;
    o.position = p0 * b.x + p1 * b.y + p2 * b.z;
    f3 cr = cross(p1 - p0, p2 - p0);
    float len = sqrtf(dot(cr, cr));
    o.ng = len > 0.0f ? cr / len : mk(0.0f, 0.0f, 1.0f);
    o.sn = o.ng;
    if ((attr_flags(s, slot) & F_NORMALS) != 0u) {
        f3 n = nrm(interp3a(s, slot, 0u, b));
        if (dot(n, n) > 0.5f) o.sn = n;
    }
    return o;
}

struct Mat {
    float4 base;
    float metallic, roughness;
    f3 normal;
    bool unlit;
    f3 emission;
    float ior, specular;
    f3 specular_color;
    float transmission, thickness;
    f3 atten_color;
    float atten_dist, clearcoat, cc_rough;
    f3 cc_normal, sheen;
    float sheen_rough;
};

static __device__ f3 perturb(const Scene& s, uint32_t slot, f3 b, f3 n, float4 t, float scale) {
    if ((attr_flags(s, slot) & F_TANGENTS) == 0u) return n;
    float4 tg = interp4a(s, slot, 3u, b);
    float w = attr(s, slot, 3u).w < 0.0f ? -1.0f : 1.0f;
    f3 t3 = xyz(tg);
    float d = dot(n, t3);
    f3 tt = nrm(t3 - n * d);
    if (dot(tt, tt) < 0.5f) return n;
    f3 bt = cross(n, tt) * w;
    f3 ts = mk((t.x * 2.0f - 1.0f) * scale, (t.y * 2.0f - 1.0f) * scale, t.z * 2.0f - 1.0f);
    f3 nn = nrm(tt * ts.x + bt * ts.y + n * ts.z);
    return dot(nn, nn) > 0.5f ? nn : n;
}

// material() (pathtrace.wgsl:842-902). Slots are sampled in order; an
// absent slot is white. `m` is the hit's material index.
static __device__ OXD_HEAVY Mat material(const Scene& s, uint32_t slot, uint32_t m, f3 b, f3 sn_in, const Lod& lod, bool flip) {
    f3 sn = flip ? -sn_in : sn_in;
    uint32_t o = mat_off(s, m);
    float4 tex[13];
    uint32_t present = 0u;
    // Fast path: one word per slot tells whether any texture is bound.
#pragma unroll 1
    for (uint32_t si = 0; si < 13u; si++) {
        tex[si] = make_float4(1.f, 1.f, 1.f, 1.f);
        if (slot_present(s, m, si, slot)) {
            present |= 1u << si;
            tex[si] = slot_sample(s, m, si, slot, b, si == S_EMISSIVE ? base_lod() : lod);
        }
    }
    Mat r;
    float4 col = mul4(tv4(s, o), tex[S_BASE]);
    if ((attr_flags(s, slot) & F_COLORS) != 0u) col = mul4(col, interp4a(s, slot, 9u, b));
    r.base = col;
    r.metallic = clampf(tf(s, o + 8u) * tex[S_MR].z, 0.0f, 1.0f);
    r.roughness = clampf(tf(s, o + 9u) * tex[S_MR].y, 0.0f, 1.0f);
    r.normal = sn;
    if ((present & (1u << S_NORMAL)) != 0u) r.normal = perturb(s, slot, b, sn, tex[S_NORMAL], tf(s, o + 10u));
    r.unlit = (tw(s, o + M_FLAGS) & 8u) != 0u;
    r.emission = sp(0.0f);
    f3 e = tv3(s, o + 4u);
    if (!r.unlit && !is_black(e)) r.emission = e * xyz(tex[S_EMISSIVE]);
    r.ior = tf(s, o + 12u);
    r.specular = tf(s, o + 13u) * tex[S_SPEC].w;
    r.specular_color = tv3(s, o + 14u) * xyz(tex[S_SPEC_COLOR]);
    r.transmission = tf(s, o + 17u) * tex[S_TRANSMISSION].x;
    r.thickness = tf(s, o + 18u) * tex[S_THICKNESS].y;
    r.atten_color = tv3(s, o + 19u);
    r.atten_dist = tf(s, o + 22u);
    r.clearcoat = tf(s, o + 23u) * tex[S_CC].x;
    r.cc_rough = tf(s, o + 24u) * tex[S_CC_ROUGH].y;
    r.cc_normal = sn;
    if ((present & (1u << S_CC_NORMAL)) != 0u) r.cc_normal = perturb(s, slot, b, sn, tex[S_CC_NORMAL], tf(s, o + 25u));
    r.sheen = tv3(s, o + 26u) * xyz(tex[S_SHEEN_COLOR]);
    r.sheen_rough = tf(s, o + 29u) * tex[S_SHEEN_ROUGH].w;
    return r;
}

static __device__ f3 emission_of(const Scene& s, uint32_t slot, uint32_t m, f3 b) {
    uint32_t o = mat_off(s, m);
    f3 e = tv3(s, o + 4u);
    if ((tw(s, o + M_FLAGS) & 8u) != 0u || is_black(e)) return sp(0.0f);
    if (slot_present(s, m, S_EMISSIVE, slot)) return e * xyz(slot_sample(s, m, S_EMISSIVE, slot, b, base_lod()));
    return e;
}

// ---- §4 BSDF
__device__ __forceinline__ float d_ggx(float n_dot_h, float a) {
    if (n_dot_h <= 0.0f) return 0.0f;
    float a2 = a * a;
    float d = n_dot_h * n_dot_h * (a2 - 1.0f) + 1.0f;
    return a2 / (PI * d * d);
}
__device__ __forceinline__ float lambda(float c_in, float a) {
    float c = fmaxf(fabsf(c_in), 1.0e-7f);
    float a2 = a * a;
    return (sqrtf(a2 + (1.0f - a2) * c * c) / c - 1.0f) * 0.5f;
}
__device__ __forceinline__ float g1(float c, float a) { return 1.0f / (1.0f + lambda(c, a)); }
__device__ __forceinline__ float g2(float cv, float cl, float a) { return 1.0f / (1.0f + lambda(cv, a) + lambda(cl, a)); }
__device__ __forceinline__ f3 schlick(f3 f0, float c) {
    float x = 1.0f - clampf(c, 0.0f, 1.0f);
    float k = x * x * x * x * x;
    return f0 + (sp(1.0f) - f0) * k;
}
static __device__ f3 sample_vndf(f3 v, float a, float u0, float u1) {
    f3 vh = nrm(mk(a * v.x, a * v.y, v.z));
    float lensq = vh.x * vh.x + vh.y * vh.y;
    f3 t1 = mk(1.0f, 0.0f, 0.0f);
    if (lensq > 0.0f) {
        float il = 1.0f / sqrtf(lensq);
        t1 = mk(-vh.y * il, vh.x * il, 0.0f);
    }
    f3 t2 = cross(vh, t1);
    float r = sqrtf(u0);
    float phi = 2.0f * PI * u1;
    float p1 = r * fm_cos(phi);
    float p2 = r * fm_sin(phi);
    float sc = 0.5f * (1.0f + vh.z);
    p2 = (1.0f - sc) * sqrtf(fmaxf(1.0f - p1 * p1, 0.0f)) + sc * p2;
    float pz = sqrtf(fmaxf(1.0f - p1 * p1 - p2 * p2, 0.0f));
    f3 nh = t1 * p1 + t2 * p2 + vh * pz;
    return nrm(mk(a * nh.x, a * nh.y, fmaxf(nh.z, 1.0e-6f)));
}
__device__ __forceinline__ float vndf_reflect_pdf(f3 n, f3 v, f3 h, float a) {
    float nv = dot(n, v), nh = dot(n, h);
    if (nv <= 0.0f || nh <= 0.0f || dot(v, h) <= 0.0f) return 0.0f;
    return g1(nv, a) * d_ggx(nh, a) / (4.0f * nv);
}
__device__ __forceinline__ f3 reflect_h(f3 v, f3 h) { return 2.0f * dot(v, h) * h - v; }
__device__ __forceinline__ float d_charlie(float n_dot_h, float a) {
    float inv = 1.0f / fmaxf(a, 1.0e-3f);
    float sin2 = fmaxf(1.0f - n_dot_h * n_dot_h, 0.0f);
    if (sin2 <= 0.0f) return 0.0f;
    return (2.0f + inv) * fm_pow(sin2, inv * 0.5f) / (2.0f * PI);
}
__device__ __forceinline__ float v_neubelt(float nl, float nv) { return 1.0f / fmaxf(4.0f * (nl + nv - nl * nv), 1.0e-6f); }
__device__ __forceinline__ float sheen_albedo(const float* lut, float c, float rough) {
    float x = clampf(clampf(c, 0.0f, 1.0f) * (float)SHEEN_COS - 0.5f, 0.0f, (float)(SHEEN_COS - 1u));
    float y = clampf(clampf(rough, 0.0f, 1.0f) * (float)(SHEEN_ROUGH - 1u), 0.0f, (float)(SHEEN_ROUGH - 1u));
    uint32_t x0 = to_u32(floorf(x)), y0 = to_u32(floorf(y));
    uint32_t x1 = x0 + 1u < SHEEN_COS - 1u ? x0 + 1u : SHEEN_COS - 1u;
    uint32_t y1 = y0 + 1u < SHEEN_ROUGH - 1u ? y0 + 1u : SHEEN_ROUGH - 1u;
    float fx = x - (float)x0, fy = y - (float)y0;
    float a00 = lut[y0 * SHEEN_COS + x0], a10 = lut[y0 * SHEEN_COS + x1];
    float a01 = lut[y1 * SHEEN_COS + x0], a11 = lut[y1 * SHEEN_COS + x1];
    float a = a00 + (a10 - a00) * fx;
    float bb = a01 + (a11 - a01) * fx;
    return a + (bb - a) * fy;
}
__device__ __forceinline__ void basis(f3 n, f3* t, f3* b) {
    float sign = sign_of(n.z);
    float a = -1.0f / (sign + n.z);
    float bb = n.x * n.y * a;
    *t = mk(1.0f + sign * n.x * n.x * a, sign * bb, -sign * n.x);
    *b = mk(bb, sign + n.y * n.y * a, -n.y);
}
static __device__ f3 cosine_hemisphere(float u0, float u1) {
    float a = 2.0f * u0 - 1.0f, b = 2.0f * u1 - 1.0f;
    float r = 0.0f, phi = 0.0f;
    if (a == 0.0f && b == 0.0f) {
        r = 0.0f;
        phi = 0.0f;
    } else if (fabsf(a) > fabsf(b)) {
        r = a;
        phi = (PI / 4.0f) * (b / a);
    } else {
        r = b;
        phi = PI / 2.0f - (PI / 4.0f) * (a / b);
    }
    float x = r * fm_cos(phi), y = r * fm_sin(phi);
    return mk(x, y, sqrtf(fmaxf(1.0f - x * x - y * y, 0.0f)));
}

struct Bsdf {
    f3 v, n, ng, ncc, base;
    float metallic, alpha, specular;
    f3 f0d;
    float transmission;
    bool thin;
    float eta_i, eta_t, clearcoat, cc_alpha;
    f3 sheen;
    float sheen_rough, sheen_alpha, w_cc;
    float p0, p1, p2, p3, p4;
};
__device__ __forceinline__ f3 fresnel_d(const Bsdf& bs, float c) {
    if (bs.eta_i > bs.eta_t) {
        float eta = bs.eta_i / bs.eta_t;
        float s2 = eta * eta * fmaxf(1.0f - c * c, 0.0f);
        if (s2 >= 1.0f) return sp(1.0f);
        return schlick(bs.f0d, sqrtf(1.0f - s2));
    }
    return schlick(bs.f0d, c);
}
static __device__ OXD_HEAVY Bsdf make_bsdf(const float* lut, const Mat& m, f3 v, f3 ng_in, bool front) {
    float fl = front ? 1.0f : -1.0f;
    f3 ng = ng_in * fl;
    f3 n = m.normal * fl;
    if (dot(n, v) <= 1.0e-4f) n = ng;
    f3 ncc = m.cc_normal * fl;
    if (dot(ncc, v) <= 1.0e-4f) ncc = n;
    bool thin = m.thickness <= 0.0f;
    float ior = (finite(m.ior) && m.ior >= 1.0f) ? m.ior : 1.5f;
    float eta_i = ior, eta_t = 1.0f;
    if (thin || front) {
        eta_i = 1.0f;
        eta_t = ior;
    }
    bool inside = !thin && !front;
    float q = (ior - 1.0f) / (ior + 1.0f);
    float r0 = q * q;
    Bsdf b;
    b.v = v;
    b.n = n;
    b.ng = ng;
    b.ncc = ncc;
    b.base = xyz(m.base);
    b.metallic = m.metallic;
    b.alpha = fmaxf(m.roughness * m.roughness, MIN_ALPHA);
    b.specular = clampf(m.specular, 0.0f, 1.0f);
    b.f0d = vmin(r0 * m.specular_color, sp(1.0f));
    b.transmission = m.transmission;
    b.thin = thin;
    b.eta_i = eta_i;
    b.eta_t = eta_t;
    b.clearcoat = inside ? 0.0f : m.clearcoat;
    b.sheen = inside ? sp(0.0f) : m.sheen;
    b.cc_alpha = fmaxf(m.cc_rough * m.cc_rough, MIN_ALPHA);
    b.sheen_rough = m.sheen_rough;
    b.sheen_alpha = fmaxf(m.sheen_rough * m.sheen_rough, 1.0e-3f);
    float cv = fmaxf(dot(n, v), 1.0e-4f);
    b.w_cc = 0.0f;
    if (b.clearcoat > 0.0f) b.w_cc = b.clearcoat * schlick(sp(0.04f), dot(ncc, v)).x;
    float sheen_max = max3(b.sheen);
    float e_v = sheen_max > 0.0f ? sheen_albedo(lut, cv, b.sheen_rough) : 0.0f;
    float s_scale = (1.0f - b.w_cc) * (1.0f - sheen_max * e_v);
    float fd = b.specular * max3(fresnel_d(b, cv));
    float fm = mean3(schlick(b.base, cv));
    float mm = b.metallic;
    float base_mean = fmaxf(mean3(b.base), 0.0f);
    float p0 = s_scale * (1.0f - mm) * (1.0f - b.transmission) * (1.0f - fd) * base_mean;
    float p1 = s_scale * ((1.0f - mm) * fd + mm * fm);
    float p2 = s_scale * (1.0f - mm) * b.transmission * (1.0f - fd) * base_mean;
    float p3 = b.w_cc;
    float p4 = (1.0f - b.w_cc) * sheen_max * e_v;
    float sum = p0 + p1 + p2 + p3 + p4;
    if (sum > 0.0f && finite(sum)) {
        b.p0 = p0 / sum;
        b.p1 = p1 / sum;
        b.p2 = p2 / sum;
        b.p3 = p3 / sum;
        b.p4 = p4 / sum;
    } else {
        b.p0 = b.p1 = b.p2 = b.p3 = b.p4 = 0.0f;
    }
    return b;
}
__device__ __forceinline__ bool bsdf_black(const Bsdf& b) {
    return b.p0 <= 0.0f && b.p1 <= 0.0f && b.p2 <= 0.0f && b.p3 <= 0.0f && b.p4 <= 0.0f;
}
__device__ __forceinline__ float lobe_p(const Bsdf& b, uint32_t i) {
    return i == 0u ? b.p0 : (i == 1u ? b.p1 : (i == 2u ? b.p2 : (i == 3u ? b.p3 : b.p4)));
}

struct Eval {
    f3 f;
    float pdf;
};
static __device__ OXD_HEAVY Eval bsdf_eval(const float* lut, const Bsdf& b, f3 l) {
    f3 v = b.v, n = b.n;
    float nv = fmaxf(dot(n, v), 1.0e-4f);
    if (dot(b.ng, l) > 0.0f) {
        float nl = dot(n, l);
        f3 h = nrm(v + l);
        float vh = fmaxf(dot(v, h), 0.0f);
        float nh = dot(n, h);
        f3 f = sp(0.0f);
        float pdf = 0.0f;
        if (nl > 0.0f) {
            f3 fd = fresnel_d(b, vh);
            f3 fm = schlick(b.base, vh);
            float spec_c = d_ggx(nh, b.alpha) * g2(nv, nl, b.alpha) / (4.0f * nv * nl);
            float m = b.metallic;
            float diff_k = (1.0f - m) * (1.0f - b.transmission) * (1.0f - b.specular * max3(fd)) / PI;
            f3 layer = spec_c * ((1.0f - m) * b.specular * fd + m * fm) + diff_k * b.base;
            float smax = max3(b.sheen);
            if (smax > 0.0f) {
                float scale = fminf(1.0f - smax * sheen_albedo(lut, nv, b.sheen_rough),
                                    1.0f - smax * sheen_albedo(lut, nl, b.sheen_rough));
                float sh = d_charlie(nh, b.sheen_alpha) * v_neubelt(nl, nv);
                layer = layer * scale + b.sheen * sh;
            }
            f = layer * (1.0f - b.w_cc);
            pdf += (b.p0 + b.p4) * nl / PI;
            pdf += b.p1 * vndf_reflect_pdf(n, v, h, b.alpha);
        }
        if (b.clearcoat > 0.0f) {
            float cnv = fmaxf(dot(b.ncc, v), 1.0e-4f);
            float cnl = dot(b.ncc, l);
            if (cnl > 0.0f) {
                float cnh = dot(b.ncc, h);
                float c = b.w_cc * d_ggx(cnh, b.cc_alpha) * g2(cnv, cnl, b.cc_alpha) / (4.0f * cnv * cnl);
                f = f + sp(c);
                pdf += b.p3 * vndf_reflect_pdf(b.ncc, v, h, b.cc_alpha);
            }
        }
        return {f * fmaxf(nl, 0.0f), pdf};
    }
    if (b.transmission <= 0.0f || b.metallic >= 1.0f) return {sp(0.0f), 0.0f};
    float nl = -dot(n, l);
    if (nl <= 0.0f) return {sp(0.0f), 0.0f};
    float smax = max3(b.sheen);
    float sheen_scale = smax > 0.0f ? 1.0f - smax * sheen_albedo(lut, nv, b.sheen_rough) : 1.0f;
    float w = (1.0f - b.metallic) * b.transmission * (1.0f - b.w_cc) * sheen_scale;
    float val, pdf_t;
    if (b.thin) {
        f3 lm = l + n * (2.0f * nl);
        f3 h = nrm(v + lm);
        float vh = dot(v, h), nh = dot(n, h);
        if (vh <= 0.0f || nh <= 0.0f) return {sp(0.0f), 0.0f};
        float fd = b.specular * max3(fresnel_d(b, vh));
        val = d_ggx(nh, b.alpha) * g2(nv, nl, b.alpha) / (4.0f * nv * nl) * (1.0f - fd);
        pdf_t = vndf_reflect_pdf(n, v, h, b.alpha);
    } else {
        float ei = b.eta_i, et = b.eta_t;
        f3 h = nrm(-(ei * v + et * l));
        if (dot(h, n) < 0.0f) h = -h;
        float vh = dot(v, h), lh = dot(l, h), nh = dot(n, h);
        if (vh <= 0.0f || lh >= 0.0f || nh <= 0.0f) return {sp(0.0f), 0.0f};
        float denom = ei * vh + et * lh;
        if (fabsf(denom) < 1.0e-6f) return {sp(0.0f), 0.0f};
        float d = d_ggx(nh, b.alpha);
        float fd = b.specular * max3(fresnel_d(b, vh));
        float jac = et * et * fabsf(lh) / (denom * denom);
        val = vh * fabsf(lh) * d * g2(nv, nl, b.alpha) * et * et * (1.0f - fd) / (nv * nl * denom * denom);
        pdf_t = g1(nv, b.alpha) * vh * d / nv * jac;
    }
    return {b.base * (w * val * nl), b.p2 * pdf_t};
}

struct BSample {
    bool ok;
    f3 l, f;
    float pdf;
};
static __device__ OXD_HEAVY BSample bsdf_sample(const float* lut, const Bsdf& b, float ux, float uy, float uz) {
    BSample res;
    res.ok = false;
    float acc = 0.0f;
    uint32_t lobe = NONE;
#pragma unroll
    for (uint32_t i = 0; i < 5u; i++) {
        float p = lobe_p(b, i);
        acc += p;
        if (lobe == NONE && p > 0.0f && uz < acc) lobe = i;
    }
    if (lobe == NONE) {
#pragma unroll
        for (uint32_t i = 0; i < 5u; i++)
            if (lobe_p(b, i) > 0.0f) lobe = i;
        if (lobe == NONE) return res;
    }
    f3 v = b.v;
    f3 l;
    if (lobe == 0u || lobe == 4u) {
        f3 t, bb;
        basis(b.n, &t, &bb);
        f3 c = cosine_hemisphere(ux, uy);
        l = t * c.x + bb * c.y + b.n * c.z;
    } else {
        f3 nn = lobe == 3u ? b.ncc : b.n;
        float a = lobe == 3u ? b.cc_alpha : b.alpha;
        f3 t, bb;
        basis(nn, &t, &bb);
        f3 vl = mk(dot(v, t), dot(v, bb), dot(v, nn));
        if (vl.z <= 0.0f) return res;
        f3 hl = sample_vndf(vl, a, ux, uy);
        f3 h = t * hl.x + bb * hl.y + nn * hl.z;
        if (lobe != 2u) {
            l = reflect_h(v, h);
        } else if (b.thin) {
            f3 r = reflect_h(v, h);
            float d = dot(r, b.n);
            l = r + b.n * (-2.0f * d);
        } else {
            float eta = b.eta_i / b.eta_t;
            float ci = dot(v, h);
            float s2 = eta * eta * fmaxf(1.0f - ci * ci, 0.0f);
            if (s2 >= 1.0f) return res;
            float ct = sqrtf(1.0f - s2);
            float k = eta * ci - ct;
            l = nrm(-eta * v + k * h);
        }
    }
    if (!finite3(l) || dot(l, l) < 0.5f) return res;
    bool reflection = dot(b.ng, l) > 0.0f;
    if (reflection == (lobe == 2u)) return res;
    Eval e = bsdf_eval(lut, b, l);
    if (e.pdf <= 0.0f || !finite(e.pdf) || is_black(e.f) || !finite3(e.f)) return res;
    res.ok = true;
    res.l = l;
    res.f = e.f;
    res.pdf = e.pdf;
    return res;
}

// ---- lights
struct LightSample {
    bool ok;
    f3 l;
    float distance;
    f3 radiance;
};
static __device__ LightSample punctual_sample(const Scene& s, uint32_t j, f3 p) {
    uint32_t o = s.P.offs0[3] + 16u * j;
    LightSample r;
    r.ok = false;
    uint32_t kind = tw(s, o + 3u);
    f3 base = tv3(s, o + 8u), dir = tv3(s, o + 4u);
    if (kind == 0u) {
        r.ok = true;
        r.l = -dir;
        r.distance = -1.0f;
        r.radiance = base;
        return r;
    }
    f3 to = tv3(s, o) - p;
    float d2 = dot(to, to);
    if (!(d2 > 1.0e-12f)) return r;
    float d = sqrtf(d2);
    f3 l = to / d;
    float att = 1.0f / d2;
    float range = tf(s, o + 7u);
    if (range > 0.0f) {
        float x = d / range;
        att *= clampf(1.0f - x * x * x * x, 0.0f, 1.0f);
    }
    if (kind == 2u) {
        float cd = dot(dir, -l);
        float a = clampf(cd * tf(s, o + 12u) + tf(s, o + 13u), 0.0f, 1.0f);
        att *= a * a;
    }
    if (att <= 0.0f) return r;
    r.ok = true;
    r.l = l;
    r.distance = d;
    r.radiance = base * att;
    return r;
}
__device__ __forceinline__ uint32_t partition_point(const Scene& s, uint32_t o, uint32_t n, float u, uint32_t stride) {
    uint32_t lo = 0u, hi = n;
    while (lo < hi) {
        uint32_t mid = (lo + hi) / 2u;
        if (tf(s, o + stride * mid) <= u) lo = mid + 1u;
        else hi = mid;
    }
    return lo;
}
__device__ __forceinline__ float triangle_solid_angle(f3 p, f3 a0, f3 b0, f3 c0) {
    f3 a = nrm_any(a0 - p), b = nrm_any(b0 - p), c = nrm_any(c0 - p);
    float num = fabsf(dot(a, cross(b, c)));
    float den = 1.0f + dot(a, b) + dot(b, c) + dot(c, a);
    float o = 2.0f * fm_atan2(num, den);
    return finite(o) ? fmaxf(o, 0.0f) : 0.0f;
}
static __device__ OXD_HEAVY f3 sample_spherical_triangle(f3 p, f3 a0, f3 b0, f3 c0, float u0, float u1) {
    f3 zero = sp(0.0f);
    f3 a = nrm_any(a0 - p), b = nrm_any(b0 - p), c = nrm_any(c0 - p);
    f3 nab = nrm_any(cross(a, b)), nbc = nrm_any(cross(b, c)), nca = nrm_any(cross(c, a));
    if (dot(a, a) == 0.0f || dot(b, b) == 0.0f || dot(c, c) == 0.0f || dot(nab, nab) == 0.0f ||
        dot(nbc, nbc) == 0.0f || dot(nca, nca) == 0.0f)
        return zero;
    float alpha = fm_acos(clampf(-dot(nab, nca), -1.0f, 1.0f));
    float beta = fm_acos(clampf(-dot(nbc, nab), -1.0f, 1.0f));
    float gamma = fm_acos(clampf(-dot(nca, nbc), -1.0f, 1.0f));
    float area = alpha + beta + gamma - PI;
    if (!(area > 0.0f)) return zero;
    float ap = u0 * area;
    float sn = fm_sin(ap - alpha), t = fm_cos(ap - alpha);
    float sa = fm_sin(alpha), ca = fm_cos(alpha);
    float cos_c = dot(a, b);
    float uu = t - ca;
    float vv = sn + sa * cos_c;
    float den = (vv * sn + uu * t) * sa;
    if (fabsf(den) < 1.0e-30f) return zero;
    float q = clampf(((vv * t - uu * sn) * ca - vv) / den, -1.0f, 1.0f);
    f3 ca_perp = nrm_any(c - dot(c, a) * a);
    if (dot(ca_perp, ca_perp) == 0.0f) return zero;
    float r = sqrtf(fmaxf(1.0f - q * q, 0.0f));
    f3 cp = q * a + r * ca_perp;
    float z = 1.0f - u1 * (1.0f - dot(cp, b));
    f3 cb_perp = nrm_any(cp - dot(cp, b) * b);
    float w = sqrtf(fmaxf(1.0f - z * z, 0.0f));
    f3 d = b;
    if (dot(cb_perp, cb_perp) > 0.0f) d = z * b + w * cb_perp;
    return nrm_any(d);
}
static __device__ float tri_pdf(const Scene& s, uint32_t li, uint32_t slot, f3 p, f3 q) {
    f3 a = tri_pos(s, slot, 0u), b = tri_pos(s, slot, 1u), c = tri_pos(s, slot, 2u);
    float sel = (1.0f - s.P.fparams[2]) * tf(s, s.P.offs1[0] + 4u * li + 1u);
    float omega = triangle_solid_angle(p, a, b, c);
    if (omega >= MIN_SPHERICAL_SOLID_ANGLE) return sel / omega;
    f3 cr = cross(b - a, c - a);
    float len = sqrtf(dot(cr, cr));
    f3 to = q - p;
    float d2 = dot(to, to);
    if (len <= 0.0f || d2 <= 0.0f) return 0.0f;
    float cs = fabsf(dot(cr, to) / (len * sqrtf(d2)));
    if (cs <= 0.0f) return 0.0f;
    return sel * d2 / (0.5f * len * cs);
}
struct Texel {
    uint32_t x, y;
    float st;
};
__device__ __forceinline__ Texel env_texel(const Scene& s, f3 d) {
    uint32_t w = s.P.env[0], h = s.P.env[1];
    float u = 0.5f + fm_atan2(d.x, -d.z) / (2.0f * PI);
    float th = fm_acos(clampf(d.y, -1.0f, 1.0f));
    float v = th / PI;
    uint32_t x = to_u32(fmaxf(u * (float)w, 0.0f));
    uint32_t y = to_u32(fmaxf(v * (float)h, 0.0f));
    x = x < w - 1u ? x : w - 1u;
    y = y < h - 1u ? y : h - 1u;
    return {x, y, fm_sin(th)};
}
__device__ __forceinline__ f3 env_radiance_at(const Scene& s, const Texel& t) {
    return tv3(s, s.P.offs2[1] + 3u * (t.y * s.P.env[0] + t.x));
}
__device__ __forceinline__ float env_pdf_at(const Scene& s, const Texel& t) {
    if (t.st <= 1.0e-6f) return 0.0f;
    uint32_t w = s.P.env[0], h = s.P.env[1];
    return tf(s, s.P.offs2[0] + t.y * w + t.x) * (float)(w * h) / (2.0f * PI * PI * t.st);
}
struct EnvSample {
    bool ok;
    f3 d, le;
    float pdf;
};
static __device__ OXD_HEAVY EnvSample env_sample(const Scene& s, float u0, float u1) {
    EnvSample r;
    r.ok = false;
    uint32_t w = s.P.env[0], h = s.P.env[1];
    uint32_t marg = s.P.offs1[2];
    uint32_t pp = partition_point(s, marg, h + 1u, u0, 1u);
    uint32_t y = (pp < 1u ? 1u : (pp > h ? h : pp)) - 1u;
    uint32_t row = s.P.offs1[3] + y * (w + 1u);
    uint32_t px = partition_point(s, row, w + 1u, u1, 1u);
    uint32_t x = (px < 1u ? 1u : (px > w ? w : px)) - 1u;
    float my = (u0 - tf(s, marg + y)) / fmaxf(tf(s, marg + y + 1u) - tf(s, marg + y), 1.0e-12f);
    float mx = (u1 - tf(s, row + x)) / fmaxf(tf(s, row + x + 1u) - tf(s, row + x), 1.0e-12f);
    float u = ((float)x + clampf(mx, 0.0f, 0.99999f)) / (float)w;
    float v = ((float)y + clampf(my, 0.0f, 0.99999f)) / (float)h;
    float phi = 2.0f * PI * (u - 0.5f);
    float th = PI * v;
    float st = fm_sin(th), ct = fm_cos(th);
    f3 d = mk(st * fm_sin(phi), ct, -st * fm_cos(phi));
    Texel t = env_texel(s, d);
    float pdf = env_pdf_at(s, t);
    if (pdf <= 0.0f || !finite(pdf)) return r;
    r.ok = true;
    r.d = d;
    r.le = env_radiance_at(s, t);
    r.pdf = pdf;
    return r;
}
__device__ __forceinline__ float power_heuristic(float a, float b) {
    float a2 = a * a, b2 = b * b;
    if (a2 + b2 > 0.0f && finite(a2 + b2)) return a2 / (a2 + b2);
    if (!finite(a) && a > 0.0f) return 1.0f;
    return 0.0f;
}
__device__ __forceinline__ f3 clamp_c(const Scene& s, f3 c) {
    float m = max3(c);
    float cl = s.P.fparams[1];
    if (cl > 0.0f && m > cl) return c * (cl / m);
    return c;
}

}  // namespace oxd
