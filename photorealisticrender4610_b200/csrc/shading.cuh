// Device shading: the reference's vector helpers, RNG stream, camera, BRDF
// utilities, materials, environment map and emitter sampling.
//
// Every function keeps the reference's operation order (compiled without
// multiply-add contraction), so everything that is +, -, *, / or sqrt rounds
// exactly as the reference's IEEE build does. Transcendentals (sin, cos, pow,
// atan2, acos) are CUDA's own and may differ from the host libm in the last
// ulp; paths therefore agree with the reference sample by sample except where
// such an ulp flips a branch.
#pragma once
#include "device_types.h"
#include "trace.cuh"

namespace prr {

#define PRR_PI 3.141592653589793f  // global.hpp:10 (float)
#define PRR_EPS 1e-3f              // global.hpp:12

// ---------------------------------------------------------------- vectors
struct V3 {
    float x, y, z;
};
__device__ __forceinline__ V3 v3(float x, float y, float z) { return V3{x, y, z}; }
__device__ __forceinline__ V3 v3(float s) { return V3{s, s, s}; }
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ V3 operator-(V3 a) { return v3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ V3 operator*(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
// Vector3f * float and float * Vector3f both compute v.c * r (Vector.hpp:18-20, :61-63)
__device__ __forceinline__ V3 operator*(V3 a, float r) { return v3(a.x * r, a.y * r, a.z * r); }
__device__ __forceinline__ V3 operator*(float r, V3 a) { return v3(a.x * r, a.y * r, a.z * r); }
__device__ __forceinline__ V3 operator/(V3 a, float r) { return v3(a.x / r, a.y / r, a.z / r); }
__device__ __forceinline__ float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 cross(V3 a, V3 b) {
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
// normalize() (Vector.hpp:103-111): multiply by 1/sqrtf(|v|^2)
__device__ __forceinline__ V3 normalize(V3 v) {
    const float m2 = v.x * v.x + v.y * v.y + v.z * v.z;
    if (m2 > 0) {
        const float inv = 1 / sqrtf(m2);
        return v3(v.x * inv, v.y * inv, v.z * inv);
    }
    return v;
}
// Vector3f::normalized() (Vector.hpp:28-31): divide by the norm
__device__ __forceinline__ V3 normalized(V3 v) {
    const float n = sqrtf(v.x * v.x + v.y * v.y + v.z * v.z);
    return v3(v.x / n, v.y / n, v.z / n);
}
__device__ __forceinline__ float norm(V3 v) { return sqrtf(v.x * v.x + v.y * v.y + v.z * v.z); }
__device__ __forceinline__ float smax(float a, float b) { return (a < b) ? b : a; }
__device__ __forceinline__ float smin(float a, float b) { return (b < a) ? b : a; }
__device__ __forceinline__ float max3(V3 v) { return smax(smax(v.x, v.y), v.z); }
__device__ __forceinline__ bool finite3(V3 v) {
    return isfinite(v.x) && isfinite(v.y) && isfinite(v.z);
}

// ---------------------------------------------------------------- RNG
// The counter-keyed replacement of get_random_float (global.hpp:35-50): a
// SplitMix64 stream whose state is derived from (seed, stream, index), with
// the reference generator's output form (top 24 bits times 2^-24).
__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
__host__ __device__ __forceinline__ uint64_t path_state(uint64_t seed, uint32_t stream,
                                                        uint32_t index) {
    return mix64(mix64(seed ^ 0x6A09E667F3BCC909ULL) ^ (((uint64_t) stream << 32) | index));
}
struct Rng {
    uint64_t s;
    __device__ __forceinline__ float next() {
        s += 0x9E3779B97F4A7C15ULL;
        const uint64_t z = mix64(s);
        return (float) (z >> 40) * 0x1p-24f;
    }
};

// ---------------------------------------------------------------- camera
struct Ray3 {
    V3 o, d;
};

__device__ __forceinline__ V3 sample_disc(float u, float v) { // Camera.hpp:58-73
    const float a = 2.0f * u - 1.0f;
    const float b = 2.0f * v - 1.0f;
    if (a == 0.0f && b == 0.0f)
        return v3(0.f);
    float r, phi;
    if (fabsf(a) > fabsf(b)) {
        r = a;
        phi = (PRR_PI / 4.0f) * (b / a);
    } else {
        r = b;
        phi = (PRR_PI / 2.0f) - (PRR_PI / 4.0f) * (a / b);
    }
    return v3(r * cosf(phi), r * sinf(phi), 0.0f);
}

// Camera::generateRay (Camera.hpp:75-95); the focal length in pixels and the
// frame are computed once on the host by Camera::init's arithmetic.
__device__ __forceinline__ Ray3 generate_ray(const DevCamera &c, int i, int j, float xo, float yo,
                                             Rng &rng) {
    const V3 fwd = v3(c.forward[0], c.forward[1], c.forward[2]);
    const V3 right = v3(c.right[0], c.right[1], c.right[2]);
    const V3 up = v3(c.up[0], c.up[1], c.up[2]);
    const V3 eye = v3(c.eye[0], c.eye[1], c.eye[2]);
    const float x = ((float) i + xo - (float) c.width * 0.5f) / c.focal_px;
    const float y = ((float) (c.height - j) + yo - (float) c.height * 0.5f) / c.focal_px;
    const V3 dir = normalize(fwd + x * right + y * up);
    if (c.aperture <= 0.0f)
        return Ray3{eye, dir};
    const V3 focus = eye + dir * (c.focus_distance / dot(dir, fwd));
    const float u = rng.next();
    const float v = rng.next();
    const V3 lo = sample_disc(u, v);
    const V3 lens = eye + c.aperture * (lo.x * right + lo.y * up);
    return Ray3{lens, normalize(focus - lens)};
}

// ---------------------------------------------------------------- BRDF utils
struct Frame {
    V3 T, B, N;
};
// buildTBN (BRDFUtils.hpp:15-30)
__device__ __forceinline__ Frame build_tbn(V3 N) {
    Frame f;
    if (fabsf(N.x) > fabsf(N.y)) {
        const float inv = 1.0f / sqrtf(N.x * N.x + N.z * N.z);
        f.T = v3(N.z * inv, 0.0f, -N.x * inv);
    } else {
        const float inv = 1.0f / sqrtf(N.y * N.y + N.z * N.z);
        f.T = v3(0.0f, N.z * inv, -N.y * inv);
    }
    f.B = cross(N, f.T);
    f.N = N;
    return f;
}
__device__ __forceinline__ V3 to_local(const Frame &f, V3 w) { // BRDFUtils.hpp:45-49
    return v3(dot(w, f.T), dot(w, f.B), dot(w, f.N));
}
__device__ __forceinline__ V3 to_world(const Frame &f, V3 l) { // BRDFUtils.hpp:35-39
    return l.x * f.T + l.y * f.B + l.z * f.N;
}
__device__ __forceinline__ V3 reflect(V3 wo, V3 N) { // BRDFUtils.hpp:56-58
    return 2.f * dot(wo, N) * N - wo;
}
__device__ __forceinline__ float pdf_cosine(float ndotwi) { // BRDFUtils.hpp:79-81
    return smax(0.f, ndotwi) / PRR_PI;
}
__device__ __forceinline__ float d_ggx(float ndoth, float alpha) { // BRDFUtils.hpp:90-94
    const float a2 = alpha * alpha;
    const float den = ndoth * ndoth * (a2 - 1.f) + 1.f;
    return a2 / (PRR_PI * den * den);
}
__device__ __forceinline__ float smith_lambda(float ndotv, float alpha) { // :102-106
    const float c2 = ndotv * ndotv;
    const float t2 = (1.f - c2) / smax(c2, 1e-6f);
    return 0.5f * (-1.f + sqrtf(1.f + alpha * alpha * t2));
}
__device__ __forceinline__ float g1_ggx(float ndotv, float alpha) { // :112-114
    return 1.f / (1.f + smith_lambda(ndotv, alpha));
}
__device__ __forceinline__ float g2_ggx(float ndotwo, float ndotwi, float alpha) { // :121-123
    return 1.f / (1.f + smith_lambda(ndotwo, alpha) + smith_lambda(ndotwi, alpha));
}
__device__ __forceinline__ V3 f_schlick(float wodoth, V3 f0) { // :143-146
    const float t = powf(smax(0.f, 1.f - wodoth), 5.f);
    return f0 + (v3(1.f) - f0) * t;
}
// sampleGGX_VNDF (BRDFUtils.hpp:163-181), Heitz 2018
__device__ __forceinline__ V3 sample_vndf(V3 wo, float alpha, float u1, float u2) {
    const V3 vh = normalize(v3(alpha * wo.x, alpha * wo.y, wo.z));
    const float lensq = vh.x * vh.x + vh.y * vh.y;
    const V3 T1 = lensq > 0.f ? v3(-vh.y, vh.x, 0.f) / sqrtf(lensq) : v3(1.f, 0.f, 0.f);
    const V3 T2 = cross(vh, T1);
    const float r = sqrtf(u1);
    const float phi = 2.f * PRR_PI * u2;
    const float t1 = r * cosf(phi);
    float t2 = r * sinf(phi);
    const float s = 0.5f * (1.f + vh.z);
    t2 = (1.f - s) * sqrtf(1.f - t1 * t1) + s * t2;
    const V3 nh = t1 * T1 + t2 * T2 + sqrtf(smax(0.f, 1.f - t1 * t1 - t2 * t2)) * vh;
    return normalize(v3(alpha * nh.x, alpha * nh.y, smax(0.f, nh.z)));
}
__device__ __forceinline__ float pdf_vndf(float ndotwo, float ndoth, float wodoth,
                                          float alpha) { // :195-204
    const float D = d_ggx(ndoth, alpha);
    const float G1 = g1_ggx(ndotwo, alpha);
    return D * G1 * smax(0.f, wodoth) / (smax(1e-6f, ndotwo) * 4.f * smax(1e-4f, wodoth));
}
// global clamp(lo, hi, v) (global.hpp:14-16)
__device__ __forceinline__ float gclamp(float lo, float hi, float v) { return smax(lo, smin(hi, v)); }
__device__ __forceinline__ V3 refract(V3 I, V3 N, float ior) { // :232-245
    float cosi = gclamp(-1.f, 1.f, dot(I, N));
    float etai = 1.f, etat = ior;
    V3 n = N;
    if (cosi < 0.f) {
        cosi = -cosi;
    } else {
        const float tmp = etai;
        etai = etat;
        etat = tmp;
        n = -N;
    }
    const float eta = etai / etat;
    const float k = 1.f - eta * eta * (1.f - cosi * cosi);
    return k < 0.f ? v3(0.f) : eta * I + (eta * cosi - sqrtf(k)) * n;
}
__device__ __forceinline__ float fresnel(V3 I, V3 N, float ior) { // :247-260
    float cosi = gclamp(-1.f, 1.f, dot(I, N));
    float etai = 1.f, etat = ior;
    if (cosi > 0.f) {
        const float tmp = etai;
        etai = etat;
        etat = tmp;
    }
    const float sint = etai / etat * sqrtf(smax(0.f, 1.f - cosi * cosi));
    if (sint >= 1.f)
        return 1.f;
    const float cost = sqrtf(smax(0.f, 1.f - sint * sint));
    cosi = fabsf(cosi);
    const float Rs = ((etat * cosi) - (etai * cost)) / ((etat * cosi) + (etai * cost));
    const float Rp = ((etai * cosi) - (etat * cost)) / ((etai * cosi) + (etat * cost));
    return (Rs * Rs + Rp * Rp) * 0.5f;
}

// ---------------------------------------------------------------- textures
// TextureUtils.hpp:22-136: bilinear with wrap-around on 8-bit texels.
__device__ __forceinline__ void uv_to_texel(float u, float v, int w, int h, int &x0, int &y0,
                                            int &x1, int &y1, float &fx, float &fy) {
    u = u - floorf(u);
    v = v - floorf(v);
    const float px = u * (float) w;
    const float py = v * (float) h;
    x0 = (int) px % w;
    y0 = (int) py % h;
    x1 = (x0 + 1) % w;
    y1 = (y0 + 1) % h;
    fx = px - floorf(px);
    fy = py - floorf(py);
}
__device__ __forceinline__ float texel(const DevTexture &t, int x, int y, int c) {
    return (float) t.data[(y * t.width + x) * t.channels + c] / 255.f;
}
__device__ __forceinline__ V3 fetch_rgb(const DevTexture &t, int x, int y) {
    return v3(texel(t, x, y, 0), texel(t, x, y, 1), texel(t, x, y, 2));
}
__device__ __forceinline__ V3 bilerp(V3 c00, V3 c10, V3 c01, V3 c11, float fx, float fy) {
    const V3 top = c00 + (c10 - c00) * fx;
    const V3 bottom = c01 + (c11 - c01) * fx;
    return top + (bottom - top) * fy;
}
__device__ __forceinline__ float srgb_to_linear(float x) {
    x = smax(0.f, x);
    return x <= 0.04045f ? x / 12.92f : powf((x + 0.055f) / 1.055f, 2.4f);
}
// sampleBaseColor (TextureUtils.hpp:76-88)
__device__ __forceinline__ V3 sample_base_color(const DevTexture &t, float u, float v) {
    int x0, y0, x1, y1;
    float fx, fy;
    uv_to_texel(u, v, t.width, t.height, x0, y0, x1, y1, fx, fy);
    const V3 c = bilerp(fetch_rgb(t, x0, y0), fetch_rgb(t, x1, y0), fetch_rgb(t, x0, y1),
                        fetch_rgb(t, x1, y1), fx, fy);
    return v3(srgb_to_linear(c.x), srgb_to_linear(c.y), srgb_to_linear(c.z));
}
// sampleNormalMap (TextureUtils.hpp:90-106)
__device__ __forceinline__ V3 sample_normal_map(const DevTexture &t, float u, float v) {
    int x0, y0, x1, y1;
    float fx, fy;
    uv_to_texel(u, v, t.width, t.height, x0, y0, x1, y1, fx, fy);
    auto fetch = [&](int x, int y) {
        return v3(texel(t, x, y, 0) * 2.f - 1.f, texel(t, x, y, 1) * 2.f - 1.f,
                  texel(t, x, y, 2) * 2.f - 1.f);
    };
    return normalize(bilerp(fetch(x0, y0), fetch(x1, y0), fetch(x0, y1), fetch(x1, y1), fx, fy));
}
// sampleMetallicRoughness (TextureUtils.hpp:108-126): (G = roughness, B = metallic)
__device__ __forceinline__ void sample_mr(const DevTexture &t, float u, float v, float &rough,
                                          float &metal) {
    int x0, y0, x1, y1;
    float fx, fy;
    uv_to_texel(u, v, t.width, t.height, x0, y0, x1, y1, fx, fy);
    auto lerp = [](float a, float b, float s) { return a + (b - a) * s; };
    const float r0 = lerp(texel(t, x0, y0, 1), texel(t, x1, y0, 1), fx);
    const float r1 = lerp(texel(t, x0, y1, 1), texel(t, x1, y1, 1), fx);
    const float m0 = lerp(texel(t, x0, y0, 2), texel(t, x1, y0, 2), fx);
    const float m1 = lerp(texel(t, x0, y1, 2), texel(t, x1, y1, 2), fx);
    rough = lerp(r0, r1, fy);
    metal = lerp(m0, m1, fy);
}

// Out-of-line forms of the samplers, for kernels whose common path reads no
// texture: there the calls are rare, and inlined the samplers' code crowds
// the instruction cache (the caustic sample kernel: 2.87 -> 2.80 ms).
static __device__ __noinline__ V3 sample_base_color_ool(const DevTexture &t, float u, float v) {
    return sample_base_color(t, u, v);
}
static __device__ __noinline__ V3 sample_normal_map_ool(const DevTexture &t, float u, float v) {
    return sample_normal_map(t, u, v);
}
static __device__ __noinline__ void sample_mr_ool(const DevTexture &t, float u, float v,
                                                  float &rough, float &metal) {
    sample_mr(t, u, v, rough, metal);
}

// ---------------------------------------------------------------- materials
// Interpolated surface data of a hit (Intersection::tcoords, tangent,
// tangentHandedness, hasTangent; Intersection.hpp:26-30).
struct SurfAttr {
    float u, v;
    V3 tan;
    float hand;
    int has_tan;
};
__device__ __forceinline__ SurfAttr no_attr() { return SurfAttr{0.f, 0.f, v3(0.f), 1.f, 0}; }

// ShadingData (Material.cpp:3-26 and the glTF-tangent overload of
// Material.hpp:57-70): the frame T, B from the hit's tangent (Gram-Schmidt
// against Ng, B = cross(Ng, T) * handedness) or from buildTBN(Ng); base
// colour and metallic / roughness from their textures or factors, roughness
// floored at 0.08; N from the normal map in that frame, else Ng. The BSDF
// frame is buildTBN(N), as toLocal / toWorld build it (BRDFUtils.hpp:35-49).
struct Shading {
    Frame f;
    V3 base;
    float roughness, metallic;
};
// kOutline: the texture samplers called out of line (see above).
template <bool kOutline = false>
__device__ __forceinline__ Shading build_shading(const DevScene &S, const DevMaterial &m, V3 Ng,
                                                 const SurfAttr &a) {
    Shading sd;
    if (m.tex_base >= 0)
        sd.base = kOutline ? sample_base_color_ool(S.textures[m.tex_base], a.u, a.v)
                           : sample_base_color(S.textures[m.tex_base], a.u, a.v);
    else
        sd.base = v3(m.base[0], m.base[1], m.base[2]);
    float rough = m.roughness, metal = m.metallic;
    if (m.tex_mr >= 0) {
        if (kOutline)
            sample_mr_ool(S.textures[m.tex_mr], a.u, a.v, rough, metal);
        else
            sample_mr(S.textures[m.tex_mr], a.u, a.v, rough, metal);
    }
    sd.roughness = smax(rough, 0.08f);
    sd.metallic = metal;
    V3 N = Ng;
    if (m.tex_normal >= 0) {
        Frame tb;
        bool basis = false;
        if (a.has_tan) {
            const V3 tg = normalize(a.tan);
            const V3 T = tg - dot(Ng, tg) * Ng;
            const float tlen = sqrtf(T.x * T.x + T.y * T.y + T.z * T.z);
            if (!(tlen < 1e-6f)) {
                tb.T = T / tlen;
                tb.B = cross(Ng, tb.T) * a.hand;
                basis = true;
            }
        }
        if (!basis)
            tb = build_tbn(Ng);
        const V3 tn = kOutline ? sample_normal_map_ool(S.textures[m.tex_normal], a.u, a.v)
                               : sample_normal_map(S.textures[m.tex_normal], a.u, a.v);
        N = normalize(tn.x * tb.T + tn.y * tb.B + tn.z * Ng);
    }
    sd.f = build_tbn(N);
    return sd;
}

struct BSDFSample {
    V3 wi, f;
    float pdf;
};

// Material::computeF0 (Material.hpp:113-117)
__device__ __forceinline__ V3 compute_f0(float ior, float metallic, V3 color) {
    float f0 = (ior - 1.0f) / (ior + 1.0f);
    f0 *= f0;
    return v3(f0) * (1 - metallic) + color * metallic;
}

// DiffuseMaterial::eval + pdf with LOBE_ALL (Material.cpp:63-158), sharing
// the local-frame set-up; f includes N.wi.
__device__ __forceinline__ void diffuse_eval_pdf(const DevMaterial &m, const Shading &sd, V3 wi,
                                                 V3 wo, V3 *f_out, float *pdf_out) {
    const float alpha = sd.roughness * sd.roughness;
    const V3 F0 = compute_f0(m.ior, sd.metallic, sd.base);
    const V3 wl = to_local(sd.f, wi);
    const V3 ol = to_local(sd.f, wo);
    const float ndwi = wl.z, ndwo = ol.z;
    if (ndwi <= 0.f || ndwo <= 0.f) {
        if (f_out)
            *f_out = v3(0.f);
        if (pdf_out)
            *pdf_out = 0.f;
        return;
    }
    V3 H = wl + ol;
    if (dot(H, H) < 1e-8f) {
        if (f_out)
            *f_out = v3(0.f);
        if (pdf_out)
            *pdf_out = 0.f;
        return;
    }
    H = normalize(H);
    if (H.z < 0.f)
        H = -H;
    const float ndh = smax(0.f, H.z);
    const float wodh = smax(0.f, dot(ol, H));
    if (f_out) {
        const V3 F = f_schlick(wodh, F0);
        const float D = d_ggx(ndh, alpha);
        const float G = g2_ggx(ndwo, ndwi, alpha);
        const float den = 4.f * smax(ndwo, 1e-4f) * smax(ndwi, 1e-4f);
        const V3 spec = D * G * F / den;
        const V3 kD = (v3(1.f) - F) * (1.f - sd.metallic);
        const V3 diff = kD * sd.base / PRR_PI;
        *f_out = (diff + spec) * ndwi;
    }
    if (pdf_out) {
        const float F0max = max3(F0);
        const float sw = sd.metallic + (1.f - sd.metallic) * F0max;
        const float ps = pdf_vndf(ndwo, ndh, wodh, alpha);
        const float pd = pdf_cosine(ndwi);
        *pdf_out = sw * ps + (1.f - sw) * pd;
    }
}

// eval / pdf through the material's dynamic type, as the integrator's calls
// through Material* dispatch (EmissiveMaterial, Mirror and Glass return 0).
__device__ __forceinline__ void mat_eval_pdf(const DevMaterial &m, const Shading &sd, V3 wi, V3 wo,
                                             V3 *f, float *pdf) {
    if (m.kind == kMatDiffuse) {
        diffuse_eval_pdf(m, sd, wi, wo, f, pdf);
    } else {
        if (f)
            *f = v3(0.f);
        if (pdf)
            *pdf = 0.f;
    }
}

// DiffuseMaterial::sample (Material.cpp:28-61): draws three numbers once the
// outgoing direction is above the surface.
__device__ __forceinline__ BSDFSample diffuse_sample(const DevMaterial &m, const Shading &sd, V3 wo,
                                                     Rng &rng) {
    BSDFSample s;
    s.wi = v3(0.f);
    s.f = v3(0.f);
    s.pdf = 0.f;
    const float alpha = sd.roughness * sd.roughness;
    const V3 F0 = compute_f0(m.ior, sd.metallic, sd.base);
    const float F0max = max3(F0);
    const float sw = sd.metallic + (1.f - sd.metallic) * F0max;
    const V3 wol = to_local(sd.f, wo);
    if (wol.z <= 0.f)
        return s;
    const float u0 = rng.next();
    const float u1 = rng.next();
    const float u2 = rng.next();
    V3 wil;
    if (u0 < sw) {
        const V3 H = sample_vndf(wol, alpha, u1, u2);
        if (dot(H, H) < 1e-8f)
            return s;
        wil = reflect(wol, H);
    } else {
        const float r = sqrtf(u1);
        const float phi = 2.f * PRR_PI * u2;
        wil = v3(r * cosf(phi), r * sinf(phi), sqrtf(smax(0.f, 1.f - u1)));
    }
    if (wil.z <= 0.f)
        return s;
    const V3 wi = to_world(sd.f, wil);
    s.wi = wi;
    float pdf;
    diffuse_eval_pdf(m, sd, wi, wo, nullptr, &pdf);
    s.pdf = pdf;
    if (pdf > 1e-6f)
        diffuse_eval_pdf(m, sd, wi, wo, &s.f, nullptr);
    return s;
}

// MirrorMaterial::sample / GlassMaterial::sample (Material.cpp:160-191).
__device__ __forceinline__ BSDFSample delta_sample(const DevMaterial &m, const Shading &sd, V3 wo,
                                                   Rng &rng) {
    BSDFSample s;
    s.pdf = 1.0f;
    const V3 N = sd.f.N;
    if (m.kind == kMatMirror) {
        s.wi = normalize(reflect(wo, N));
        s.f = v3(m.base[0], m.base[1], m.base[2]);
        return s;
    }
    const V3 inc = -wo;
    const float kr = fresnel(inc, N, m.ior);
    const V3 refr = refract(inc, N, m.ior);
    const bool tir = norm(refr) < 1e-6f;
    const bool entering = dot(inc, N) < 0.f;
    const float eta = entering ? (1.0f / m.ior) : m.ior;
    if (rng.next() < kr || tir) {
        s.wi = normalize(reflect(wo, N));
        s.f = v3(1.0f);
    } else {
        s.wi = normalize(refr);
        s.f = v3(eta * eta);
    }
    return s;
}

// ---------------------------------------------------------------- env map
__device__ __forceinline__ float luminance(V3 c) { // EnvMap.hpp:181-183
    return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z;
}
__device__ __forceinline__ void dir_to_uv(V3 d, float &u, float &v) { // EnvMap.hpp:71-75
    const float phi = atan2f(d.z, d.x);
    const float theta = acosf(smax(-1.f, smin(1.f, d.y)));
    u = (phi + PRR_PI) / (2.f * PRR_PI);
    v = theta / PRR_PI;
}
__device__ __forceinline__ V3 uv_to_dir(float u, float v) { // EnvMap.hpp:84-89
    const float phi = u * 2.f * PRR_PI - PRR_PI;
    const float theta = v * PRR_PI;
    const float st = sinf(theta);
    return v3(st * cosf(phi), cosf(theta), st * sinf(phi));
}
__device__ __forceinline__ V3 env_px(const DevEnv &e, int x, int y) {
    const float4 p = __ldg(&e.pixels[(size_t) y * e.width + x]);
    return v3(p.x, p.y, p.z);
}
// EnvMap::sample (EnvMap.hpp:97-113): bilinear at uv * (size - 1)
__device__ __forceinline__ V3 env_lookup(const DevEnv &e, V3 dir) {
    if (!e.loaded)
        return v3(0.f);
    float u, v;
    dir_to_uv(dir, u, v);
    const float px = smax(0.f, u * (e.width - 1));
    const float py = smax(0.f, v * (e.height - 1));
    const int x0 = (int) px, y0 = (int) py;
    const int x1 = min(x0 + 1, e.width - 1);
    const int y1 = min(y0 + 1, e.height - 1);
    const float fx = px - x0, fy = py - y0;
    const V3 p00 = env_px(e, x0, y0), p10 = env_px(e, x1, y0);
    const V3 p01 = env_px(e, x0, y1), p11 = env_px(e, x1, y1);
    const V3 top = p00 + (p10 - p00) * fx;
    const V3 bot = p01 + (p11 - p01) * fx;
    return top + (bot - top) * fy;
}
// EnvMap::importanceSamplePdf (EnvMap.hpp:124-133)
__device__ __forceinline__ float env_pdf(const DevEnv &e, V3 dir) {
    float u, v;
    dir_to_uv(dir, u, v);
    const int col = min((int) (u * e.width), e.width - 1);
    const int row = min((int) (v * e.height), e.height - 1);
    const float theta = v * PRR_PI;
    const float st = smax(1e-4f, sinf(theta));
    const float lum = luminance(env_px(e, col, row));
    return (lum * st / (e.total + 1e-6f)) * ((float) (e.width * e.height) / (2.f * PRR_PI * PRR_PI * st));
}
// std::lower_bound over [first, first + n): first index with !(a[i] < x)
__device__ __forceinline__ int lower_bound(const float *a, int n, float x) {
    int lo = 0, len = n;
    while (len > 0) {
        const int half = len >> 1;
        if (__ldg(a + lo + half) < x) {
            lo += half + 1;
            len -= half + 1;
        } else {
            len = half;
        }
    }
    return lo;
}
// lower_bound over a non-decreasing CDF, started from its guide table: for u
// in [k/G, (k+1)/G) the answer lies in [guide[k], guide[k+1]] (lower_bound is
// monotone in the searched value), and the search of that sub-range returns
// the same index as the search of the whole array, in a few steps instead of
// log2(n). u * G is exact (G a power of two, u in [0, 1)).
__device__ __forceinline__ int guided_lower_bound(const float *a, int n, float u,
                                                  const int32_t *g, int G) {
    if (G > 0 && __ldg(g) >= 0) {
        const int k = min((int) (u * (float) G), G - 1);
        const int lo = __ldg(g + k), hi = __ldg(g + k + 1);
        return lo + lower_bound(a + lo, hi - lo, u);
    }
    return lower_bound(a, n, u);
}
// EnvMap::importanceSample (EnvMap.hpp:145-169)
__device__ __forceinline__ V3 env_importance(const DevEnv &e, Rng &rng, float &pdf) {
    const float r1 = rng.next();
    const float r2 = rng.next();
    const int G = e.guide_n;
    int row = guided_lower_bound(e.marginal, e.height, r1, e.guide, G);
    row = min(row, e.height - 1);
    int col = guided_lower_bound(e.cdf + (size_t) row * e.width, e.width, r2,
                                 G > 0 ? e.guide + (size_t) (row + 1) * (G + 1) : nullptr, G);
    col = min(col, e.width - 1);
    const float u = (col + 0.5f) / (float) e.width;
    const float v = (row + 0.5f) / (float) e.height;
    const V3 dir = uv_to_dir(u, v);
    const float lum = luminance(env_px(e, col, row));
    pdf = (lum / (e.total + 1e-6f)) * ((float) (e.width * e.height) / (2.f * PRR_PI * PRR_PI));
    pdf = smax(1e-6f, pdf);
    return dir;
}

// ---------------------------------------------------------------- emitters
struct LightPoint {
    V3 p, n;
    int material;
};

// BVHAccel::Sample -> getSample -> Triangle::Sample (BVH.cpp:478-514,
// Triangle.hpp:98-103) on one mesh.
__device__ __forceinline__ LightPoint mesh_sample(const DevScene &S, const DevObject &o, Rng &rng) {
    float p = sqrtf(rng.next()) * o.bvh_area;
    uint32_t ref = o.root;
    uint32_t tri = 0;
    for (;;) {
        if (ref & kLeafBit) {
            const uint32_t first = leaf_first(ref), cnt = leaf_count(ref);
            tri = first + cnt - 1;
            for (uint32_t i = 0; i < cnt; i++) {
                p -= __ldg(&S.tri_meta[first + i].area);
                if (p <= 0.f || i == cnt - 1) {
                    tri = first + i;
                    break;
                }
            }
            break;
        }
        const WNode &n = S.nodes[ref];
        const float la = __ldg(&n.left_area);
        if (p < la) {
            ref = __ldg(&n.left);
        } else {
            p -= la;
            ref = __ldg(&n.right);
        }
    }
    const float *v = S.verts + (size_t) tri * 9;
    const V3 v0 = v3(v[0], v[1], v[2]), v1 = v3(v[3], v[4], v[5]), v2 = v3(v[6], v[7], v[8]);
    const float x = sqrtf(rng.next());
    const float y = rng.next();
    LightPoint lp;
    lp.p = v0 * (1.0f - x) + v1 * (x * (1.0f - y)) + v2 * (x * y);
    lp.n = v3(S.normals[(size_t) tri * 3], S.normals[(size_t) tri * 3 + 1],
              S.normals[(size_t) tri * 3 + 2]);
    lp.material = o.material;
    return lp;
}

// Sphere::Sample (Sphere.hpp:54-63): theta is formed in double because the
// reference writes 2.0 * M_PI * u.
__device__ __forceinline__ LightPoint sphere_sample(const DevObject &o, Rng &rng) {
    const float theta = (float) (2.0 * (double) PRR_PI * (double) rng.next());
    const float phi = PRR_PI * rng.next();
    const V3 dir = v3(cosf(phi), sinf(phi) * cosf(theta), sinf(phi) * sinf(theta));
    LightPoint lp;
    lp.p = v3(o.cx, o.cy, o.cz) + o.radius * dir;
    lp.n = dir;
    lp.material = o.material;
    return lp;
}

// Scene::sampleLight (Scene.cpp:37-58): pick an emitter by area, then a point
// on it; the reported pdf is always 1 / totalEmitArea.
__device__ __forceinline__ LightPoint sample_light(const DevScene &S, Rng &rng) {
    const float p = rng.next() * S.total_emit_area;
    float acc = 0.f;
    int pick = S.emissives[S.n_emissives - 1];
    for (int k = 0; k < S.n_emissives; k++) {
        const int obj = S.emissives[k];
        acc += S.objects[obj].area;
        if (p <= acc) {
            pick = obj;
            break;
        }
    }
    const DevObject &o = S.objects[pick];
    return o.kind == kObjMesh ? mesh_sample(S, o, rng) : sphere_sample(o, rng);
}

} // namespace prr
