// Homogeneous participating medium and the Henyey-Greenstein phase function
// (Volume.hpp:7-63, Volume.cpp:3-28). The reference's integrator never reads
// them (Scene::medium is not used by Integrator::castRay); they are device
// functions here, reached through the batch calls of k_medium.cu.
#pragma once
#include "shading.cuh"

namespace prr {

struct DevMedium {
    float sigma_a, sigma_s, sigma_t, g;
    int bounded;
    float lo[3], hi[3];
};

// Medium::intersect (Volume.hpp:17-45): slab entry and exit of the medium's
// box (all of space when unbounded). The box corner and the ray origin are
// read through Vector3f's const operator[], which returns double
// (Vector.hpp:67,78-80), so each slab distance is a double product rounded
// once to float. The per-axis swap follows the reference's flag, which is set
// for POSITIVE directions; std::max / std::min keep their operand order.
__device__ __forceinline__ bool medium_intersect(const DevMedium &m, V3 o, V3 d, float &t_enter,
                                                 float &t_exit) {
    if (!m.bounded) {
        t_enter = 0.0f;
        t_exit = __int_as_float(0x7f800000);
        return true;
    }
    const float oo[3] = {o.x, o.y, o.z};
    const float dd[3] = {d.x, d.y, d.z};
    float te = -3.402823466e+38f, tx = 3.402823466e+38f;
#pragma unroll
    for (int i = 0; i < 3; i++) {
        const float inv = 1.0f / dd[i];
        float a = (float) (((double) m.lo[i] - (double) oo[i]) * (double) inv);
        float b = (float) (((double) m.hi[i] - (double) oo[i]) * (double) inv);
        if (!(dd[i] > 0)) {
            const float t = a;
            a = b;
            b = t;
        }
        te = smax(a, te);
        tx = smin(b, tx);
    }
    if (te > tx || tx < 0.0f)
        return false;
    t_enter = te;
    t_exit = tx;
    return true;
}

// phaseHG (Volume.cpp:3-6), in float throughout (the reference's M_PI is a
// float, global.hpp:9-10); the 1.5 power is evaluated in double and rounded
// once, which is what a correctly rounded powf returns.
__device__ __forceinline__ float phase_hg(float cos_theta, float g) {
    const float denom = 1.0f + g * g - 2.0f * g * cos_theta;
    const float p = (float) pow((double) denom, 1.5);
    return (1.0f - g * g) / (4.0f * PRR_PI * p);
}

// samplePhaseHG (Volume.cpp:8-28): one draw for cos(theta) (uniform when
// |g| < 1e-3, else the inverted HG CDF), one for phi = 2*pi*u (float); the
// direction is built in buildTBN(wo)'s frame and normalized. The float cosine
// and sine of phi are taken in double and rounded once.
__device__ __forceinline__ V3 sample_phase_hg(V3 wo, float g, Rng &rng) {
    float cos_theta;
    if (fabsf(g) < 1e-3f) {
        cos_theta = 1.0f - 2.0f * rng.next();
    } else {
        const float u = rng.next();
        const float sqr = (1.0f - g * g) / (1.0f - g + 2.0f * g * u);
        cos_theta = (1.0f + g * g - sqr * sqr) / (2.0f * g);
    }
    const float sin_theta = sqrtf(smax(0.0f, 1.0f - cos_theta * cos_theta));
    const float phi = 2.0f * PRR_PI * rng.next();
    const Frame f = build_tbn(wo);
    const float cp = (float) cos((double) phi), sp = (float) sin((double) phi);
    return normalize((sin_theta * cp) * f.T + (sin_theta * sp) * f.B + cos_theta * wo);
}

} // namespace prr
