// Display transform on the device: exposure and sanitising
// (Renderer.cpp:149-161), the tone-mapping operators of ToneMapping.hpp:45-279
// (Raw, Standard, AgX with the allenwp curve, Khronos PBR Neutral), and the
// 8-bit quantisation of Renderer.cpp:169-171. ACES, which the reference does
// not have, is added as K. Narkowicz's published fit (2015):
// f(x) = x(2.51x + 0.03) / (x(2.43x + 0.59) + 0.14), clamped, then sRGB.
//
// One thread per pixel, 12 bytes in and 3 (or 12) out: a streaming, HBM-bound
// kernel; the allenwp constants are formed once on the host with the
// reference's float arithmetic and passed in.
#include "prr_internal.h"

#include <cmath>

namespace prr {
namespace {

struct Allenwp {
    float contrast, toe_a, slope, w, shoulder_max, output_max;
};
constexpr float kCrossover = 0.1841865f;

// AllenwpParams(1.25, 16, 1) (ToneMapping.hpp:125-147), on the host.
Allenwp allenwp_params() {
    Allenwp p;
    const float contrast = 1.25f, output_max = 1.0f;
    p.contrast = contrast;
    p.output_max = output_max;
    const float high_clip = std::max(16.0f, output_max);
    p.toe_a = ((1.f / kCrossover) - 1.f) * std::pow(kCrossover, contrast);
    const float denom = std::pow(kCrossover, contrast) + p.toe_a;
    p.slope = (contrast * std::pow(kCrossover, contrast - 1.f) * p.toe_a) / (denom * denom);
    p.shoulder_max = output_max - kCrossover;
    p.w = high_clip - kCrossover;
    p.w = p.w * p.w;
    p.w = p.w / p.shoulder_max;
    p.w = p.w * p.slope;
    return p;
}

__device__ __forceinline__ float dmax(float a, float b) { return (a < b) ? b : a; }
__device__ __forceinline__ float dmin(float a, float b) { return (b < a) ? b : a; }
__device__ __forceinline__ float dclamp(float x, float lo, float hi) {
    return x < lo ? lo : (hi < x ? hi : x);
}

__device__ __forceinline__ float srgb_oetf(float x) { // ToneMapping.hpp:45-48
    x = dclamp(x, 0.f, 1.f);
    return x < 0.0031308f ? 12.92f * x : 1.055f * powf(x, 1.f / 2.4f) - 0.055f;
}

__device__ __forceinline__ float allenwp(float x, const Allenwp &p) { // :151-166
    x = dmax(x, 0.f);
    if (x < kCrossover) {
        const float t = powf(x, p.contrast);
        return t / (t + p.toe_a);
    }
    float s = x - kCrossover;
    const float slope_s = p.slope * s;
    s = slope_s * (1.f + s / p.w) / (1.f + (slope_s / p.shoulder_max));
    s += kCrossover;
    return s;
}

__device__ __forceinline__ float3 agx(float3 c, const Allenwp &p) { // :172-214
    c.x = dmax(c.x, 0.f);
    c.y = dmax(c.y, 0.f);
    c.z = dmax(c.z, 0.f);
    float3 i;
    i.x = 0.544814746488245f * c.x + 0.373787398372697f * c.y + 0.0813978551390581f * c.z;
    i.y = 0.140416948464053f * c.x + 0.754137554567394f * c.y + 0.105445496968552f * c.z;
    i.z = 0.0888104196149096f * c.x + 0.178871756420858f * c.y + 0.732317823964232f * c.z;
    i.x = dmin(1.0f, allenwp(i.x, p));
    i.y = dmin(1.0f, allenwp(i.y, p));
    i.z = dmin(1.0f, allenwp(i.z, p));
    float3 o;
    o.x = 1.96488741169489f * i.x + -0.855988495690215f * i.y + -0.108898916004672f * i.z;
    o.y = -0.299313364904742f * i.x + 1.32639796461980f * i.y + -0.0270845997150571f * i.z;
    o.z = -0.164352742528393f * i.x + -0.238183969428088f * i.y + 1.40253671195648f * i.z;
    return make_float3(srgb_oetf(dclamp(o.x, 0.f, 1.f)), srgb_oetf(dclamp(o.y, 0.f, 1.f)),
                       srgb_oetf(dclamp(o.z, 0.f, 1.f)));
}

__device__ __forceinline__ float3 pbr_neutral(float3 c) { // :234-262
    const float start = 0.8f - 0.04f;
    const float desat = 0.15f;
    const float x = dmin(c.x, dmin(c.y, c.z));
    const float offset = x < 0.08f ? x - 6.25f * x * x : 0.04f;
    c.x -= offset;
    c.y -= offset;
    c.z -= offset;
    const float peak = dmax(c.x, dmax(c.y, c.z));
    if (peak < start)
        return make_float3(srgb_oetf(c.x), srgb_oetf(c.y), srgb_oetf(c.z));
    const float d = 1.f - start;
    const float new_peak = 1.f - d * d / (peak + d - start);
    const float scale = new_peak / peak;
    c.x *= scale;
    c.y *= scale;
    c.z *= scale;
    const float g = 1.f - 1.f / (desat * (peak - new_peak) + 1.f);
    c.x = c.x * (1.f - g) + new_peak * g;
    c.y = c.y * (1.f - g) + new_peak * g;
    c.z = c.z * (1.f - g) + new_peak * g;
    return make_float3(srgb_oetf(c.x), srgb_oetf(c.y), srgb_oetf(c.z));
}

__device__ __forceinline__ float aces(float x) {
    const float n = x * (2.51f * x + 0.03f);
    const float d = x * (2.43f * x + 0.59f) + 0.14f;
    return dclamp(n / d, 0.f, 1.f);
}

__global__ void k_tonemap(int mapper, float exposure, Allenwp params, const float *__restrict__ in,
                          int64_t n, float *__restrict__ out_f, uint8_t *__restrict__ out_u8) {
    const int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    float3 c = make_float3(in[i * 3] * exposure, in[i * 3 + 1] * exposure, in[i * 3 + 2] * exposure);
    if (!isfinite(c.x))
        c.x = 0.f;
    if (!isfinite(c.y))
        c.y = 0.f;
    if (!isfinite(c.z))
        c.z = 0.f;
    c.x = dmax(0.f, c.x);
    c.y = dmax(0.f, c.y);
    c.z = dmax(0.f, c.z);
    float3 r;
    switch (mapper) {
    case PRR_TONEMAP_RAW:
        r = make_float3(dclamp(c.x, 0.f, 1.f), dclamp(c.y, 0.f, 1.f), dclamp(c.z, 0.f, 1.f));
        break;
    case PRR_TONEMAP_STANDARD:
        r = make_float3(srgb_oetf(c.x), srgb_oetf(c.y), srgb_oetf(c.z));
        break;
    case PRR_TONEMAP_AGX:
        r = agx(c, params);
        break;
    case PRR_TONEMAP_PBR_NEUTRAL:
        r = pbr_neutral(c);
        break;
    default:
        r = make_float3(srgb_oetf(aces(c.x)), srgb_oetf(aces(c.y)), srgb_oetf(aces(c.z)));
        break;
    }
    if (out_f) {
        out_f[i * 3] = r.x;
        out_f[i * 3 + 1] = r.y;
        out_f[i * 3 + 2] = r.z;
    }
    if (out_u8) {
        out_u8[i * 3] = (uint8_t) (dclamp(r.x, 0.f, 1.f) * 255.f + 0.5f);
        out_u8[i * 3 + 1] = (uint8_t) (dclamp(r.y, 0.f, 1.f) * 255.f + 0.5f);
        out_u8[i * 3 + 2] = (uint8_t) (dclamp(r.z, 0.f, 1.f) * 255.f + 0.5f);
    }
}

} // namespace
} // namespace prr

extern "C" int prr_tonemap(int mapper, float exposure, const float *rgb, int64_t n,
                           float *out_rgb, uint8_t *out_u8, void *stream) {
    using namespace prr;
    if (mapper < PRR_TONEMAP_RAW || mapper > PRR_TONEMAP_ACES)
        return fail(PRR_ERR_INVALID_ARGUMENT, "unknown tone mapper");
    if (n < 0 || (n > 0 && (!rgb || (!out_rgb && !out_u8))))
        return fail(PRR_ERR_INVALID_ARGUMENT, "bad tone-map arguments");
    if (n == 0)
        return PRR_OK;
    static const Allenwp params = allenwp_params();
    k_tonemap<<<(unsigned) ((n + 255) / 256), 256, 0, (cudaStream_t) stream>>>(
        mapper, exposure, params, rgb, n, out_rgb, out_u8);
    PRR_CUDA_TRY(cudaGetLastError());
    return PRR_OK;
}
