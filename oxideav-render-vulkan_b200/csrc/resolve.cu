// Resolve: accumulator -> RGBA8 (sRGB-encoded) or RGBA32F (scene-linear).
//
// fs_resolve_pt (resolve.wgsl:151-188) as an element-wise compute kernel
// writing a device buffer instead of a render target. HBM-bound: 16 bytes
// read and 4 (or 16) written per pixel; each thread handles one pixel with
// 16-byte loads and a single 4- or 16-byte store.
#include "kernels.cuh"

namespace oxd {

__device__ __forceinline__ float srgb_to_linear(float c) {
    if (c <= 0.04045f) return c / 12.92f;
    return fm_pow((c + 0.055f) / 1.055f, 2.4f);
}
__device__ __forceinline__ float linear_to_srgb(float c) {
    float x = clampf(c, 0.0f, 1.0f);
    if (x <= 0.0031308f) return 12.92f * x;
    return 1.055f * fm_pow(x, 1.0f / 2.4f) - 0.055f;
}
__device__ __forceinline__ float aces(float x) {
    float y = x * 0.6f;
    return clampf((y * (2.51f * y + 0.03f)) / (y * (2.43f * y + 0.59f) + 0.14f), 0.0f, 1.0f);
}
__device__ __forceinline__ f3 tone_map(f3 rgb_in, uint32_t op) {
    f3 rgb = vmax(rgb_in, sp(0.0f));
    if (op == 1u) {
        float l = dot(rgb, mk(0.2126f, 0.7152f, 0.0722f));
        if (l <= 0.0f) return sp(0.0f);
        return vmin(rgb / (1.0f + l), sp(1.0f));
    }
    if (op == 2u) return mk(aces(rgb.x), aces(rgb.y), aces(rgb.z));
    return vmin(rgb, sp(1.0f));
}
__device__ __forceinline__ uint32_t unorm8(float v) {
    float x = clampf(v, 0.0f, 1.0f);
    return (uint32_t)(x * 255.0f + 0.5f);
}

__global__ void __launch_bounds__(256) resolve_kernel(const __grid_constant__ ResolveArgs a) {
    uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= a.w || y >= a.h) return;
    uint64_t idx = (uint64_t)y * a.w + x;
    const bool hdr = a.hdr != 0;
    f3 bg_lin = mk(srgb_to_linear(a.p.background[0]), srgb_to_linear(a.p.background[1]),
                   srgb_to_linear(a.p.background[2]));
    float ba = a.p.background[3];
    float n = a.p.exposure[1];
    float4 acc = __ldcs(a.accum + idx);
    float4 o;
    if (acc.w <= 0.0f || n <= 0.0f) {
        o = make_float4(bg_lin.x, bg_lin.y, bg_lin.z, ba);
    } else {
        f3 m = mk(acc.x, acc.y, acc.z) / acc.w;
        float f = clampf(acc.w / n, 0.0f, 1.0f);
        f3 c = hdr ? m : tone_map(m * a.p.exposure[0], a.p.cfg[2]);
        if (f >= 1.0f) {
            o = make_float4(c.x, c.y, c.z, 1.0f);
        } else {
            float a_sum = f + (1.0f - f) * ba;
            if (a_sum > 0.0f) {
                f3 r = (f * c + (1.0f - f) * bg_lin * ba) / a_sum;
                o = make_float4(r.x, r.y, r.z, a_sum);
            } else {
                f3 r = f * c + (1.0f - f) * bg_lin;
                o = make_float4(r.x, r.y, r.z, 0.0f);
            }
        }
    }
    if (hdr) {
        reinterpret_cast<float4*>(a.out)[idx] = o;
    } else {
        uint32_t px = unorm8(linear_to_srgb(o.x)) | unorm8(linear_to_srgb(o.y)) << 8 |
                      unorm8(linear_to_srgb(o.z)) << 16 | unorm8(o.w) << 24;
        reinterpret_cast<uint32_t*>(a.out)[idx] = px;
    }
}

cudaError_t launch_resolve(const ResolveArgs& a, cudaStream_t st) {
    if (a.w == 0 || a.h == 0) return cudaSuccess;
    dim3 grid((a.w + 255u) / 256u, a.h);
    resolve_kernel<<<grid, 256, 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace oxd
