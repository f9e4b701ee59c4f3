// Batch calls over the participating-medium functions of medium.cuh
// (Volume.hpp / Volume.cpp): box entry/exit, HG phase values and HG direction
// samples, each one thread per item.
#include "medium.cuh"
#include "prr_internal.h"

namespace prr {
namespace {

DevMedium to_dev(const prr_medium &m) {
    DevMedium d;
    d.sigma_a = m.sigma_a;
    d.sigma_s = m.sigma_s;
    d.sigma_t = m.sigma_t;
    d.g = m.g;
    d.bounded = m.bounded;
    for (int i = 0; i < 3; i++) {
        d.lo[i] = m.bounds_min[i];
        d.hi[i] = m.bounds_max[i];
    }
    return d;
}

__global__ void k_medium_intersect(DevMedium m, const float *o, const float *d, int64_t n,
                                   float *t_enter, float *t_exit, uint8_t *hit) {
    const int64_t k = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n)
        return;
    const V3 ro = v3(o[k * 3], o[k * 3 + 1], o[k * 3 + 2]);
    const V3 rd = v3(d[k * 3], d[k * 3 + 1], d[k * 3 + 2]);
    float te = 0.f, tx = 0.f;
    const bool h = medium_intersect(m, ro, rd, te, tx);
    hit[k] = h ? 1 : 0;
    t_enter[k] = h ? te : 0.f;
    t_exit[k] = h ? tx : 0.f;
}

__global__ void k_phase_hg(const float *c, int64_t n, float g, float *out) {
    const int64_t k = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n)
        out[k] = phase_hg(c[k], g);
}

__global__ void k_phase_hg_sample(const float *wo, int64_t n, float g, uint64_t seed,
                                  float *out) {
    const int64_t k = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n)
        return;
    Rng rng{path_state(seed, (uint32_t) k, 0u)};
    const V3 w = sample_phase_hg(v3(wo[k * 3], wo[k * 3 + 1], wo[k * 3 + 2]), g, rng);
    out[k * 3] = w.x;
    out[k * 3 + 1] = w.y;
    out[k * 3 + 2] = w.z;
}

int grid(int64_t n) { return (int) ((n + 255) / 256); }

} // namespace
} // namespace prr

using namespace prr;

extern "C" {

int prr_medium_preset(int which, prr_medium *out) {
    if (!out)
        return fail(PRR_ERR_INVALID_ARGUMENT, "out is NULL");
    prr_medium m{};
    if (which == PRR_MEDIUM_DUST) { // Medium::dust() (Volume.hpp:47-54)
        m.sigma_s = 0.05f;
        m.sigma_a = 0.005f;
        m.g = 0.6f;
    } else if (which == PRR_MEDIUM_FOG) { // Medium::fog() (Volume.hpp:56-63)
        m.sigma_s = 0.1f;
        m.sigma_a = 0.01f;
        m.g = 0.0f;
    } else {
        return fail(PRR_ERR_INVALID_ARGUMENT, "unknown medium preset");
    }
    m.sigma_t = m.sigma_s + m.sigma_a;
    *out = m;
    return PRR_OK;
}

int prr_medium_intersect(const prr_medium *medium, const float *o, const float *d, int64_t n,
                         float *out_t_enter, float *out_t_exit, uint8_t *out_hit, void *stream) {
    if (!medium || n < 0)
        return fail(PRR_ERR_INVALID_ARGUMENT, "medium and a count >= 0 are required");
    if (n == 0)
        return PRR_OK;
    if (!o || !d || !out_t_enter || !out_t_exit || !out_hit)
        return fail(PRR_ERR_INVALID_ARGUMENT, "ray and output arrays are required");
    k_medium_intersect<<<grid(n), 256, 0, (cudaStream_t) stream>>>(
        to_dev(*medium), o, d, n, out_t_enter, out_t_exit, out_hit);
    PRR_CUDA_TRY(cudaGetLastError());
    return PRR_OK;
}

int prr_phase_hg(const float *cos_theta, int64_t n, float g, float *out, void *stream) {
    if (n < 0 || (n > 0 && (!cos_theta || !out)))
        return fail(PRR_ERR_INVALID_ARGUMENT, "input and output arrays are required");
    if (n == 0)
        return PRR_OK;
    k_phase_hg<<<grid(n), 256, 0, (cudaStream_t) stream>>>(cos_theta, n, g, out);
    PRR_CUDA_TRY(cudaGetLastError());
    return PRR_OK;
}

int prr_phase_hg_sample(const float *wo, int64_t n, float g, uint64_t seed, float *out_dirs,
                        void *stream) {
    if (n < 0 || (n > 0 && (!wo || !out_dirs)))
        return fail(PRR_ERR_INVALID_ARGUMENT, "input and output arrays are required");
    if (n == 0)
        return PRR_OK;
    k_phase_hg_sample<<<grid(n), 256, 0, (cudaStream_t) stream>>>(wo, n, g, seed, out_dirs);
    PRR_CUDA_TRY(cudaGetLastError());
    return PRR_OK;
}

} // extern "C"
