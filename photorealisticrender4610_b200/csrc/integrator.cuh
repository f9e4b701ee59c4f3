// The path integrator: Integrator::castRay (Integrator.cpp:104-263) with its
// light-sampling helpers (sampleDirectLight :14-34, sampleEnvironmentMap
// :39-66, evalLightSample :78-87, evalEnvironmentSample :93-102, mis
// Integrator.hpp:30-32), restated for one device thread.
#pragma once
#include "shading.cuh"

namespace prr {

// The part of Intersection the integrator reads (Intersection.hpp:12-34).
struct Inter {
    bool hit;
    V3 p, n;
    int mat;
    SurfAttr a;
};

// Triangle::finalize (Triangle.cpp:34-59) for meshes with per-corner data:
// the hit's barycentrics (re-derived by the same Moller-Trumbore test the
// traversal ran), w0 = 1 - u - v, interpolated uv, smooth normal and tangent
// with its handedness.
__device__ __forceinline__ void finalize_attr(const DevScene &S, const DevObject &o, int tri,
                                              const RayD &r, V3 &n, SurfAttr &a) {
    a = no_attr();
    if (!o.attr)
        return;
    float t, u, v;
    tri_hit(load_tri(S, (uint32_t) tri), r, t, u, v);
    const float w0 = 1.f - u - v;
    const float *R = S.attr + (size_t) (o.attr_base + (tri - o.tri_base)) * kAttrFloats;
    if (o.attr & kAttrUV) {
        a.u = R[9] * w0 + R[11] * u + R[13] * v;
        a.v = R[10] * w0 + R[12] * u + R[14] * v;
    }
    if (o.attr & kAttrNormals)
        n = normalize(v3(R[0], R[1], R[2]) * w0 + v3(R[3], R[4], R[5]) * u +
                      v3(R[6], R[7], R[8]) * v);
    if (o.attr & kAttrTangents) {
        a.tan = normalize(v3(R[15], R[16], R[17]) * w0 + v3(R[18], R[19], R[20]) * u +
                          v3(R[21], R[22], R[23]) * v);
        const float w = R[24] * w0 + R[25] * u + R[26] * v;
        a.hand = w >= 0.f ? 1.f : -1.f;
        a.has_tan = 1;
    }
}

__device__ __forceinline__ Inter intersect(const DevScene &S, const Ray3 &ray, SmemStack &tst,
                                           SmemStack &bst) {
    RayD r{ray.o.x, ray.o.y, ray.o.z, ray.d.x, ray.d.y, ray.d.z};
    const RayPre p = precompute(r);
    const SceneHit h = scene_closest(S, r, p, tst, bst);
    Inter in;
    in.hit = h.obj >= 0;
    in.a = no_attr();
    if (!in.hit) {
        in.p = in.n = v3(0.f);
        in.mat = -1;
        return in;
    }
    const DevObject &o = S.objects[h.obj];
    in.mat = o.material;
    if (o.kind == kObjMesh) {
        // Triangle::finalize (Triangle.cpp:34-59): origin + t * direction, face normal
        in.p = ray.o + h.t * ray.d;
        in.n = v3(S.normals[(size_t) h.tri * 3], S.normals[(size_t) h.tri * 3 + 1],
                  S.normals[(size_t) h.tri * 3 + 2]);
        finalize_attr(S, o, h.tri, r, in.n, in.a);
    } else {
        // Sphere::getIntersection (Sphere.hpp:37-39)
        in.p = ray.o + ray.d * h.t;
        in.n = normalize(in.p - v3(o.cx, o.cy, o.cz));
    }
    return in;
}

__device__ __forceinline__ bool occluded(const DevScene &S, V3 o, V3 d, float tmax, SmemStack &tst,
                                         SmemStack &bst) {
    RayD r{o.x, o.y, o.z, d.x, d.y, d.z};
    const RayPre p = precompute(r);
    return scene_occluded(S, r, p, tst, bst, tmax);
}

__device__ __forceinline__ float mis(float a, float b) { return (a * a) / (a * a + b * b + 1e-6f); }

__device__ __forceinline__ V3 clamp_indirect(V3 c, float clamp) {
    if (clamp <= 0.f)
        return c;
    const float lum = (c.x + c.y + c.z) / 3;
    return (lum > clamp) ? c * (clamp / lum) : c;
}

struct PathCounters {
    uint32_t closest, shadow; // rays traced by this path
};

// Integrator::castRay. `rng` must be positioned after the camera draws.
static __device__ V3 cast_ray(const DevScene &S, Ray3 ray, int max_depth, float clamp, Rng &rng,
                       SmemStack &tst, SmemStack &bst, PathCounters &cnt) {
    V3 L = v3(0.f), beta = v3(1.f);
    Ray3 cur = ray;
    bool specular = false;
    const DevEnv &env = S.env;
    const V3 bg = v3(S.background[0], S.background[1], S.background[2]);
    Inter in = intersect(S, cur, tst, bst);
    cnt.closest++;
    for (int bounce = 0; bounce < max_depth; bounce++) {
        if (bounce == 0 || specular) {
            if (!in.hit) {
                const V3 b = env.loaded ? env_lookup(env, cur.d) : bg;
                const V3 c = beta * b;
                L = L + ((bounce > 0) ? clamp_indirect(c, clamp) : c);
            } else if (S.materials[in.mat].kind == kMatEmissive) {
                const DevMaterial &m = S.materials[in.mat];
                const V3 c = beta * v3(m.emission[0], m.emission[1], m.emission[2]);
                L = L + ((bounce > 0) ? clamp_indirect(c, clamp) : c);
            }
        }
        if (!in.hit || bounce >= max_depth)
            break;
        const DevMaterial &m = S.materials[in.mat];
        const V3 hp = in.p;
        const V3 gn = in.n;
        if (m.kind == kMatMirror || m.kind == kMatGlass) {
            // delta chain (Integrator.cpp:143-169)
            const Shading sd = build_shading(S, m, gn, in.a);
            const BSDFSample bs = delta_sample(m, sd, -cur.d, rng);
            if (bs.pdf < 1e-6f)
                break;
            beta = beta * bs.f / bs.pdf;
            const bool trans = dot(bs.wi, gn) < 0.f;
            const V3 off = trans ? -gn : gn;
            cur = Ray3{hp + off * PRR_EPS, bs.wi};
            in = intersect(S, cur, tst, bst);
            cnt.closest++;
            if (trans)
                beta = beta * sd.base;
            specular = true;
            continue;
        }
        specular = false;
        const V3 sn = dot(cur.d, gn) < 0.f ? gn : -gn;
        const Shading sd = build_shading(S, m, sn, in.a);
        const V3 wo = -cur.d;
        const bool indirect = bounce > 0;

        // NEE towards area emitters (sampleDirectLight + evalLightSample)
        if (S.total_emit_area > 0.f) {
            const LightPoint lp = sample_light(S, rng);
            const float pdf_area = 1.0f / S.total_emit_area;
            const V3 to = lp.p - hp;
            const float dist2 = dot(to, to);
            const float dist = sqrtf(dist2);
            const V3 wi = to / dist;
            const float cos_l = smax(0.f, dot(-wi, normalized(lp.n)));
            // evalLightSample is formed before the visibility test (it has no
            // side effects); a zero contribution needs no shadow ray because
            // castRay would add exactly zero either way
            V3 c = v3(0.f);
            if (cos_l > 0.f) {
                const float pdf_sa = pdf_area * dist2 / cos_l;
                V3 f;
                float bp;
                mat_eval_pdf(m, sd, wi, wo, &f, &bp);
                const float w = mis(pdf_sa, bp);
                const DevMaterial &lm = S.materials[lp.material];
                c = beta * (w * v3(lm.emission[0], lm.emission[1], lm.emission[2]) * f / pdf_sa);
                if (!(c.x == 0.f && c.y == 0.f && c.z == 0.f)) {
                    cnt.shadow++;
                    if (occluded(S, hp + wi * PRR_EPS, wi, dist - 2.f * PRR_EPS, tst, bst))
                        c = v3(0.f);
                }
            }
            L = L + (indirect ? clamp_indirect(c, clamp) : c);
        }
        // NEE towards the environment (sampleEnvironmentMap + evalEnvironmentSample)
        if (env.loaded) {
            float pdf;
            const V3 dir = env_importance(env, rng, pdf);
            V3 c = v3(0.f);
            if (!(pdf < 1e-6f)) {
                const V3 em = env_lookup(env, dir);
                V3 f;
                float bp;
                mat_eval_pdf(m, sd, dir, wo, &f, &bp);
                const float w = mis(pdf, bp);
                c = beta * (w * em * f / (pdf + 1e-6f));
                if (!(c.x == 0.f && c.y == 0.f && c.z == 0.f)) {
                    cnt.shadow++;
                    if (occluded(S, hp + dir * PRR_EPS, dir, kInf, tst, bst))
                        c = v3(0.f);
                }
            }
            L = L + (indirect ? clamp_indirect(c, clamp) : c);
        }
        // BSDF sampling (Integrator.cpp:198-244)
        BSDFSample bs;
        if (m.kind == kMatDiffuse) {
            bs = diffuse_sample(m, sd, wo, rng);
        } else {
            bs.pdf = 0.f; // EmissiveMaterial::sample
        }
        if (bs.pdf < 1e-6f)
            break;
        const V3 scale = bs.f / bs.pdf;
        const V3 off = dot(bs.wi, sd.f.N) >= 0.f ? sd.f.N : -sd.f.N;
        cur = Ray3{hp + off * PRR_EPS, bs.wi};
        in = intersect(S, cur, tst, bst);
        cnt.closest++;
        if (!in.hit) {
            V3 c;
            if (env.loaded) {
                const V3 el = env_lookup(env, bs.wi);
                const float ep = env_pdf(env, bs.wi);
                const float w = mis(bs.pdf, ep);
                c = beta * scale * w * el;
            } else {
                c = beta * scale * bg;
            }
            L = L + (indirect ? clamp_indirect(c, clamp) : c);
            break;
        }
        if (S.materials[in.mat].kind == kMatEmissive) {
            const DevMaterial &lm = S.materials[in.mat];
            const float cos_l = smax(0.f, dot(-bs.wi, normalized(in.n)));
            const V3 dd = in.p - hp;
            const float hd2 = dot(dd, dd);
            const float pdf_area = S.total_emit_area > 0.f ? 1.f / S.total_emit_area : 0.f;
            const float pdf_sa = pdf_area * hd2 / smax(cos_l, 1e-4f);
            const float w = mis(bs.pdf, pdf_sa);
            const V3 c = beta * scale * w * v3(lm.emission[0], lm.emission[1], lm.emission[2]);
            L = L + (indirect ? clamp_indirect(c, clamp) : c);
            break;
        }
        beta = beta * scale;
        if (!finite3(beta))
            break;
        // Russian roulette from bounce 3 (Integrator.cpp:250-256)
        if (bounce >= 3) {
            const float mc = max3(beta);
            const float q = smax(0.05f, 1.f - mc);
            if (rng.next() < q)
                break;
            beta = beta * (1.f / (1.f - q));
        }
    }
    if (!finite3(L))
        return v3(0.f);
    return L;
}

// Welford online mean / variance and the 95% confidence stop of the
// adaptive sampler (Renderer.hpp:14-40), with the reference's float steps.
struct Welford {
    int n = 0;
    float mean = 0.f, M2 = 0.f;
    __device__ void update(float x) {
        n++;
        const float delta = x - mean;
        mean += delta / (float) n;
        M2 += delta * (x - mean);
    }
    __device__ float variance() const { return n < 2 ? 0.f : M2 / (float) (n - 1); }
    __device__ float ci() const {
        if (n < 2 || fabsf(mean) < 1e-6f)
            return 1.f;
        return 1.96f * sqrtf(variance() / (float) n) / fabsf(mean);
    }
};

} // namespace prr
