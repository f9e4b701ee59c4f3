// Batched forms of the reference's per-call methods that the integrator is
// built from, for callers that want them on their own and for unit parity:
//   Integrator::castRay per (pixel, sample)   Integrator.cpp:104-263
//   Camera::generateRay                        Camera.hpp:75-95
//   Scene::sampleLight                         Scene.cpp:37-58
//   EnvMap::sample / importanceSamplePdf       EnvMap.hpp:97-133
//   EnvMap::importanceSample                   EnvMap.hpp:145-169
#include "integrator.cuh"
#include "prr_internal.h"

namespace prr {
namespace {

__global__ void k_cast_samples(DevScene S, const int32_t *__restrict__ px,
                               const int32_t *__restrict__ py, const int32_t *__restrict__ sample,
                               int64_t n, uint64_t seed, int max_depth, float clamp,
                               float *__restrict__ out, int tlas_cap) {
    extern __shared__ uint2 smem[];
    SmemStack tst{smem + threadIdx.x, (int) blockDim.x, 0, S.tlas_depth + 1, S.check};
    SmemStack bst{smem + (size_t) tlas_cap * blockDim.x + threadIdx.x, (int) blockDim.x, 0,
                  S.blas_depth + 1, S.check};
    const int64_t k = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n)
        return;
    const int i = px[k], j = py[k];
    const uint32_t m = (uint32_t) i + (uint32_t) j * (uint32_t) S.camera.width;
    Rng rng{path_state(seed, m, (uint32_t) sample[k])};
    const float xo = rng.next();
    const float yo = rng.next();
    const Ray3 ray = generate_ray(S.camera, i, j, xo, yo, rng);
    PathCounters cnt{0, 0};
    V3 s = cast_ray(S, ray, max_depth, clamp, rng, tst, bst, cnt);
    if (isnan(s.x) || isnan(s.y) || isnan(s.z))
        s = v3(0.f);
    out[k * 3 + 0] = s.x;
    out[k * 3 + 1] = s.y;
    out[k * 3 + 2] = s.z;
}

__global__ void k_cast_rays(DevScene S, const float *__restrict__ O, const float *__restrict__ D,
                            int64_t n, uint64_t seed, int max_depth, float clamp,
                            float *__restrict__ out, int tlas_cap) {
    extern __shared__ uint2 smem[];
    SmemStack tst{smem + threadIdx.x, (int) blockDim.x, 0, S.tlas_depth + 1, S.check};
    SmemStack bst{smem + (size_t) tlas_cap * blockDim.x + threadIdx.x, (int) blockDim.x, 0,
                  S.blas_depth + 1, S.check};
    const int64_t k = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n)
        return;
    Rng rng{path_state(seed, (uint32_t) k, 0u)};
    const Ray3 ray{v3(O[k * 3], O[k * 3 + 1], O[k * 3 + 2]), v3(D[k * 3], D[k * 3 + 1], D[k * 3 + 2])};
    PathCounters cnt{0, 0};
    const V3 s = cast_ray(S, ray, max_depth, clamp, rng, tst, bst, cnt);
    out[k * 3 + 0] = s.x;
    out[k * 3 + 1] = s.y;
    out[k * 3 + 2] = s.z;
}

__global__ void k_camera_rays(DevCamera cam, const int32_t *px, const int32_t *py, const float *xo,
                              const float *yo, int64_t n, float *o, float *d) {
    const int64_t k = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n)
        return;
    Rng rng{0};
    const Ray3 r = generate_ray(cam, px[k], py[k], xo[k], yo[k], rng);
    o[k * 3 + 0] = r.o.x;
    o[k * 3 + 1] = r.o.y;
    o[k * 3 + 2] = r.o.z;
    d[k * 3 + 0] = r.d.x;
    d[k * 3 + 1] = r.d.y;
    d[k * 3 + 2] = r.d.z;
}

__global__ void k_sample_light(DevScene S, uint64_t seed, int64_t n, float *pos, float *nrm,
                               float *pdf) {
    const int64_t k = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n)
        return;
    Rng rng{path_state(seed, (uint32_t) k, 0u)};
    const LightPoint lp = sample_light(S, rng);
    pos[k * 3 + 0] = lp.p.x;
    pos[k * 3 + 1] = lp.p.y;
    pos[k * 3 + 2] = lp.p.z;
    nrm[k * 3 + 0] = lp.n.x;
    nrm[k * 3 + 1] = lp.n.y;
    nrm[k * 3 + 2] = lp.n.z;
    pdf[k] = 1.0f / S.total_emit_area;
}

__global__ void k_env_eval(DevEnv e, const float *dirs, int64_t n, float *rgb, float *pdf) {
    const int64_t k = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n)
        return;
    const V3 d = v3(dirs[k * 3], dirs[k * 3 + 1], dirs[k * 3 + 2]);
    const V3 c = env_lookup(e, d);
    rgb[k * 3 + 0] = c.x;
    rgb[k * 3 + 1] = c.y;
    rgb[k * 3 + 2] = c.z;
    pdf[k] = env_pdf(e, d);
}

__global__ void k_env_importance(DevEnv e, uint64_t seed, int64_t n, float *dirs, float *pdf) {
    const int64_t k = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n)
        return;
    Rng rng{path_state(seed, (uint32_t) k, 0u)};
    float p;
    const V3 d = env_importance(e, rng, p);
    dirs[k * 3 + 0] = d.x;
    dirs[k * 3 + 1] = d.y;
    dirs[k * 3 + 2] = d.z;
    pdf[k] = p;
}

int blocks(int64_t n, int b) { return (int) ((n + b - 1) / b); }

const Scene *built(const prr_scene *s) {
    if (!s) {
        fail(PRR_ERR_INVALID_ARGUMENT, "scene is NULL");
        return nullptr;
    }
    const Scene *sc = reinterpret_cast<const Scene *>(s);
    if (!sc->built) {
        fail(PRR_ERR_NOT_BUILT, "scene not built (call prr_scene_build)");
        return nullptr;
    }
    return sc;
}

} // namespace
} // namespace prr

using namespace prr;

extern "C" {

int prr_cast_samples(const prr_scene *scene, const int32_t *px, const int32_t *py,
                     const int32_t *sample, int64_t n, uint64_t seed, int max_depth,
                     float indirect_clamp, float *out_rgb, void *stream) {
    const Scene *s = built(scene);
    if (!s)
        return PRR_ERR_INVALID_ARGUMENT;
    if (!s->camera_set)
        return fail(PRR_ERR_INVALID_ARGUMENT, "scene has no camera");
    if (n < 0 || (n > 0 && (!px || !py || !sample || !out_rgb)) || max_depth < 1)
        return fail(PRR_ERR_INVALID_ARGUMENT, "bad arguments");
    if (n == 0)
        return PRR_OK;
    const int block = 128;
    const int tcap = s->dev.tlas_depth + 1, bcap = s->dev.blas_depth + 1;
    const size_t smem = (size_t) (tcap + bcap) * block * sizeof(uint2);
    if (smem > 200 * 1024)
        return fail(PRR_ERR_UNSUPPORTED, "BVH too deep for the shared-memory stacks");
    if (smem > 48 * 1024)
        PRR_CUDA_TRY(cudaFuncSetAttribute(k_cast_samples,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
    k_cast_samples<<<blocks(n, block), block, smem, (cudaStream_t) stream>>>(
        s->dev, px, py, sample, n, seed, max_depth, indirect_clamp, out_rgb, tcap);
    PRR_CUDA_TRY(cudaGetLastError());
    return PRR_OK;
}

int prr_cast_rays(const prr_scene *scene, const float *o, const float *d, int64_t n,
                  uint64_t seed, int max_depth, float indirect_clamp, float *out_rgb,
                  void *stream) {
    const Scene *s = built(scene);
    if (!s)
        return PRR_ERR_INVALID_ARGUMENT;
    if (n < 0 || (n > 0 && (!o || !d || !out_rgb)) || max_depth < 1)
        return fail(PRR_ERR_INVALID_ARGUMENT, "bad arguments");
    if (n == 0)
        return PRR_OK;
    const int block = 128;
    const int tcap = s->dev.tlas_depth + 1, bcap = s->dev.blas_depth + 1;
    const size_t smem = (size_t) (tcap + bcap) * block * sizeof(uint2);
    if (smem > 200 * 1024)
        return fail(PRR_ERR_UNSUPPORTED, "BVH too deep for the shared-memory stacks");
    if (smem > 48 * 1024)
        PRR_CUDA_TRY(cudaFuncSetAttribute(k_cast_rays, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int) smem));
    k_cast_rays<<<blocks(n, block), block, smem, (cudaStream_t) stream>>>(
        s->dev, o, d, n, seed, max_depth, indirect_clamp, out_rgb, tcap);
    PRR_CUDA_TRY(cudaGetLastError());
    return PRR_OK;
}

int prr_camera_rays(const prr_scene *scene, const int32_t *px, const int32_t *py,
                    const float *xo, const float *yo, int64_t n, float *out_o, float *out_d,
                    void *stream) {
    const Scene *s = built(scene);
    if (!s)
        return PRR_ERR_INVALID_ARGUMENT;
    if (!s->camera_set || n < 0)
        return fail(PRR_ERR_INVALID_ARGUMENT, "no camera or bad count");
    if (n == 0)
        return PRR_OK;
    k_camera_rays<<<blocks(n, 256), 256, 0, (cudaStream_t) stream>>>(s->dev.camera, px, py, xo,
                                                                      yo, n, out_o, out_d);
    PRR_CUDA_TRY(cudaGetLastError());
    return PRR_OK;
}

int prr_scene_sample_light(const prr_scene *scene, uint64_t seed, int64_t n, float *out_pos,
                           float *out_normal, float *out_pdf, void *stream) {
    const Scene *s = built(scene);
    if (!s)
        return PRR_ERR_INVALID_ARGUMENT;
    if (s->dev.n_emissives == 0 || !(s->dev.total_emit_area > 0.f))
        return fail(PRR_ERR_INVALID_ARGUMENT, "scene has no emitters");
    if (n <= 0)
        return n == 0 ? PRR_OK : fail(PRR_ERR_INVALID_ARGUMENT, "bad count");
    k_sample_light<<<blocks(n, 256), 256, 0, (cudaStream_t) stream>>>(s->dev, seed, n, out_pos,
                                                                       out_normal, out_pdf);
    PRR_CUDA_TRY(cudaGetLastError());
    return PRR_OK;
}

int prr_env_eval(const prr_scene *scene, const float *dirs, int64_t n, float *out_rgb,
                 float *out_pdf, void *stream) {
    const Scene *s = built(scene);
    if (!s)
        return PRR_ERR_INVALID_ARGUMENT;
    if (!s->dev.env.loaded)
        return fail(PRR_ERR_INVALID_ARGUMENT, "scene has no environment map");
    if (n <= 0)
        return n == 0 ? PRR_OK : fail(PRR_ERR_INVALID_ARGUMENT, "bad count");
    k_env_eval<<<blocks(n, 256), 256, 0, (cudaStream_t) stream>>>(s->dev.env, dirs, n, out_rgb,
                                                                   out_pdf);
    PRR_CUDA_TRY(cudaGetLastError());
    return PRR_OK;
}

int prr_env_importance_sample(const prr_scene *scene, uint64_t seed, int64_t n, float *out_dirs,
                              float *out_pdf, void *stream) {
    const Scene *s = built(scene);
    if (!s)
        return PRR_ERR_INVALID_ARGUMENT;
    if (!s->dev.env.loaded)
        return fail(PRR_ERR_INVALID_ARGUMENT, "scene has no environment map");
    if (n <= 0)
        return n == 0 ? PRR_OK : fail(PRR_ERR_INVALID_ARGUMENT, "bad count");
    k_env_importance<<<blocks(n, 256), 256, 0, (cudaStream_t) stream>>>(s->dev.env, seed, n,
                                                                         out_dirs, out_pdf);
    PRR_CUDA_TRY(cudaGetLastError());
    return PRR_OK;
}

int prr_env_export(const prr_scene *scene, float *cdf, float *marginal, float *total) {
    const Scene *s = built(scene);
    if (!s)
        return PRR_ERR_INVALID_ARGUMENT;
    if (!s->dev.env.loaded)
        return fail(PRR_ERR_INVALID_ARGUMENT, "scene has no environment map");
    const size_t w = s->env_w, h = s->env_h;
    if (cdf)
        PRR_CUDA_TRY(cudaMemcpy(cdf, s->dev.env.cdf, w * h * sizeof(float), cudaMemcpyDeviceToHost));
    if (marginal)
        PRR_CUDA_TRY(cudaMemcpy(marginal, s->dev.env.marginal, h * sizeof(float),
                                cudaMemcpyDeviceToHost));
    if (total)
        *total = s->dev.env.total;
    return PRR_OK;
}

} // extern "C"
