// Plain megakernel renderer: the per-pixel sample loop of Renderer::Render
// (Renderer.cpp:63-99) around Integrator::castRay, one thread per
// (pixel, slice of its samples).
//
// Pixel m = i + j*W draws its n-th sample from the stream (seed, m, n), so
// any split of the samples over threads, launches or requests sees the same
// random numbers. In the fixed-spp mode the samples of a pixel are split into
// `slices` contiguous ranges, each summed in sample order by one thread, and a
// resolve kernel adds the slice sums in slice order: the result does not
// depend on scheduling. In the adaptive mode (minSPP < maxSPP) one thread runs
// the reference's Welford loop (Renderer.hpp:14-40) for the pixel.
#include "integrator.cuh"
#include "prr_internal.h"

#include <algorithm>
#include <mutex>
#include <string>

namespace prr {
namespace {

constexpr int kTileW = 16, kTileH = 8; // 128-thread blocks cover 16x8 pixel tiles

struct RenderArgs {
    int W, H;
    int x0, y0, ww, wh;
    int spp_begin, spp_end; // samples [begin, end) of the fixed mode
    int slices;
    int min_spp, max_spp;
    float threshold;
    int max_depth;
    float clamp;
    uint64_t seed;
    int tlas_cap;
    float3 *partial;        // [slices][ww*wh]
    int32_t *spp_out;
    unsigned long long *rays; // [2]: closest, shadow
};

__device__ __forceinline__ void count_rays(unsigned long long *rays, const PathCounters &c) {
    if (!rays)
        return;
    unsigned long long a = c.closest, b = c.shadow;
    for (int off = 16; off > 0; off >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, off);
        b += __shfl_down_sync(0xffffffffu, b, off);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(rays, a);
        atomicAdd(rays + 1, b);
    }
}

__global__ void __launch_bounds__(kTileW *kTileH) k_render_plain(DevScene S, RenderArgs a) {
    extern __shared__ uint2 smem[];
    SmemStack tst{smem + threadIdx.x, (int) blockDim.x, 0, S.tlas_depth + 1, S.check};
    SmemStack bst{smem + (size_t) a.tlas_cap * blockDim.x + threadIdx.x, (int) blockDim.x, 0,
                  S.blas_depth + 1, S.check};
    const int tiles_x = (a.ww + kTileW - 1) / kTileW;
    const int tile = blockIdx.x;
    const int lx = (tile % tiles_x) * kTileW + (int) (threadIdx.x % kTileW);
    const int ly = (tile / tiles_x) * kTileH + (int) (threadIdx.x / kTileW);
    const bool active = lx < a.ww && ly < a.wh;
    PathCounters cnt{0, 0};
    if (active) {
        const int i = a.x0 + lx, j = a.y0 + ly;
        const uint32_t m = (uint32_t) i + (uint32_t) j * (uint32_t) a.W;
        const int q = lx + ly * a.ww;
        const int slice = blockIdx.y;
        const int total = a.spp_end - a.spp_begin;
        const int s0 = a.spp_begin + (int) ((int64_t) total * slice / a.slices);
        const int s1 = a.spp_begin + (int) ((int64_t) total * (slice + 1) / a.slices);
        V3 acc = v3(0.f);
        for (int n = s0; n < s1; n++) {
            Rng rng{path_state(a.seed, m, (uint32_t) n)};
            const float xo = rng.next();
            const float yo = rng.next();
            const Ray3 ray = generate_ray(S.camera, i, j, xo, yo, rng);
            V3 s = cast_ray(S, ray, a.max_depth, a.clamp, rng, tst, bst, cnt);
            if (isnan(s.x) || isnan(s.y) || isnan(s.z))
                s = v3(0.f);
            acc = acc + s;
        }
        a.partial[(size_t) slice * a.ww * a.wh + q] = make_float3(acc.x, acc.y, acc.z);
    }
    count_rays(a.rays, cnt);
}

__global__ void __launch_bounds__(kTileW *kTileH) k_render_adaptive(DevScene S, RenderArgs a) {
    extern __shared__ uint2 smem[];
    SmemStack tst{smem + threadIdx.x, (int) blockDim.x, 0, S.tlas_depth + 1, S.check};
    SmemStack bst{smem + (size_t) a.tlas_cap * blockDim.x + threadIdx.x, (int) blockDim.x, 0,
                  S.blas_depth + 1, S.check};
    const int tiles_x = (a.ww + kTileW - 1) / kTileW;
    const int tile = blockIdx.x;
    const int lx = (tile % tiles_x) * kTileW + (int) (threadIdx.x % kTileW);
    const int ly = (tile / tiles_x) * kTileH + (int) (threadIdx.x / kTileW);
    PathCounters cnt{0, 0};
    if (lx < a.ww && ly < a.wh) {
        const int i = a.x0 + lx, j = a.y0 + ly;
        const uint32_t m = (uint32_t) i + (uint32_t) j * (uint32_t) a.W;
        const int q = lx + ly * a.ww;
        Welford wr, wg, wb;
        V3 acc = v3(0.f);
        int n = 0;
        while (n < a.max_spp) {
            Rng rng{path_state(a.seed, m, (uint32_t) (a.spp_begin + n))};
            const float xo = rng.next();
            const float yo = rng.next();
            const Ray3 ray = generate_ray(S.camera, i, j, xo, yo, rng);
            V3 s = cast_ray(S, ray, a.max_depth, a.clamp, rng, tst, bst, cnt);
            if (isnan(s.x) || isnan(s.y) || isnan(s.z))
                s = v3(0.f);
            acc = acc + s;
            n++;
            wr.update(s.x);
            wg.update(s.y);
            wb.update(s.z);
            if (n >= a.min_spp && wr.ci() < a.threshold && wg.ci() < a.threshold &&
                wb.ci() < a.threshold)
                break;
        }
        a.partial[q] = make_float3(acc.x, acc.y, acc.z);
        if (a.spp_out)
            a.spp_out[q] = n;
    }
    count_rays(a.rays, cnt);
}

// mean = (sum of slice sums) / n (Renderer.cpp:98)
__global__ void k_render_resolve(const float3 *__restrict__ partial, int npix, int slices,
                                 const int32_t *__restrict__ spp, int fixed_n,
                                 float *__restrict__ out, int32_t *spp_out) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= npix)
        return;
    float3 s = partial[q];
    for (int k = 1; k < slices; k++) {
        const float3 p = partial[(size_t) k * npix + q];
        s.x += p.x;
        s.y += p.y;
        s.z += p.z;
    }
    const int n = spp ? spp[q] : fixed_n;
    out[(size_t) q * 3 + 0] = s.x / (float) n;
    out[(size_t) q * 3 + 1] = s.y / (float) n;
    out[(size_t) q * 3 + 2] = s.z / (float) n;
    if (spp_out && !spp)
        spp_out[q] = n;
}

} // namespace

int render_plain(Scene &s, const prr_render_settings &rs, float *out_rgb, int32_t *out_spp,
                 unsigned long long *out_rays, cudaStream_t st) {
    const DevScene &S = s.dev;
    RenderArgs a{};
    a.W = s.width;
    a.H = s.height;
    a.x0 = rs.x0;
    a.y0 = rs.y0;
    a.ww = rs.x1 - rs.x0;
    a.wh = rs.y1 - rs.y0;
    a.min_spp = rs.min_spp;
    a.max_spp = rs.max_spp;
    a.threshold = rs.variance_threshold;
    a.max_depth = rs.max_depth;
    a.clamp = rs.indirect_clamp;
    a.seed = rs.seed;
    a.spp_begin = rs.sample_offset;
    a.spp_end = rs.sample_offset + rs.max_spp;
    a.rays = out_rays;
    const bool adaptive = rs.min_spp < rs.max_spp;
    const int npix = a.ww * a.wh;
    int slices = 1;
    if (!adaptive) {
        slices = rs.slices > 0 ? rs.slices : 1;
        if (rs.slices <= 0) {
            // enough threads to fill the GPU a few times over
            const int64_t want = (int64_t) device_sm_count() * 1024 * 2;
            while ((int64_t) npix * slices < want && slices * 2 <= rs.max_spp)
                slices *= 2;
        }
        slices = std::max(1, std::min(slices, rs.max_spp));
    }
    a.slices = slices;
    a.tlas_cap = S.tlas_depth + 1;
    const int bcap = S.blas_depth + 1;
    const size_t smem = (size_t) (a.tlas_cap + bcap) * kTileW * kTileH * sizeof(uint2);
    if (smem > 200 * 1024)
        return fail(PRR_ERR_UNSUPPORTED, "BVH too deep for the shared-memory stacks");
    PRR_CUDA_TRY(s.d_render.ensure((size_t) slices * npix * sizeof(float3)));
    a.partial = s.d_render.as<float3>();
    if (adaptive) {
        PRR_CUDA_TRY(s.d_render_spp.ensure((size_t) npix * sizeof(int32_t)));
        a.spp_out = s.d_render_spp.as<int32_t>();
    }
    if (out_rays)
        PRR_CUDA_TRY(cudaMemsetAsync(out_rays, 0, 2 * sizeof(unsigned long long), st));
    const int tiles = ((a.ww + kTileW - 1) / kTileW) * ((a.wh + kTileH - 1) / kTileH);
    const void *fn = adaptive ? (const void *) k_render_adaptive : (const void *) k_render_plain;
    if (smem > 48 * 1024)
        PRR_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
    if (adaptive)
        k_render_adaptive<<<tiles, kTileW * kTileH, smem, st>>>(S, a);
    else
        k_render_plain<<<dim3(tiles, slices), kTileW * kTileH, smem, st>>>(S, a);
    PRR_CUDA_TRY(cudaGetLastError());
    k_render_resolve<<<(npix + 255) / 256, 256, 0, st>>>(a.partial, npix, slices,
                                                          adaptive ? a.spp_out : nullptr,
                                                          rs.max_spp, out_rgb, out_spp);
    PRR_CUDA_TRY(cudaGetLastError());
    if (adaptive && out_spp)
        PRR_CUDA_TRY(cudaMemcpyAsync(out_spp, a.spp_out, (size_t) npix * sizeof(int32_t),
                                     cudaMemcpyDeviceToDevice, st));
    s.last_launches = 2;
    return PRR_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free rendering.
//
// Some callers of this library cannot call cudaMalloc while they render: a
// host application whose device memory is owned and budgeted by another
// allocator, or a caller that must not enter the CUDA allocator (or its
// implicit device synchronisation) on its frame loop. prr_render_noalloc
// serves them: it runs the same plain megakernel and resolve kernels as
// prr_render in its fixed-spp mode, but the per-slice partial sums live in the
// file-scope array below instead of memory obtained from cudaMalloc.
//
// The array holds kNoAllocPartials float3 partial sums (pixels x slices,
// 24 MiB). Every GPU on which the library's render module is loaded keeps
// this memory until the process exits. All calls on a device share the one
// array: calls whose kernels overlap on the GPU race on it, so callers must
// order them (one stream, or events between streams). Each call writes every
// partial sum it later reads, so nothing needs clearing between calls.
// ---------------------------------------------------------------------------
constexpr int64_t kNoAllocPartials = int64_t(1) << 21;
static __device__ __align__(256) float3 g_noalloc_partials[kNoAllocPartials];

namespace {

// The array's device address, looked up once per device with that device
// current (in host code the array's name is only a host-side stand-in).
int noalloc_partials(float3 **out) {
    static std::mutex mu;
    static float3 *addr[256] = {};
    int dev = 0;
    PRR_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 256)
        return fail(PRR_ERR_UNSUPPORTED, "device ordinal out of range");
    std::lock_guard<std::mutex> g(mu);
    if (!addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials);
        if (e != cudaSuccess || !p)
            return fail(PRR_ERR_CUDA, std::string("cudaGetSymbolAddress(partial sums): ") +
                                          cudaGetErrorString(e));
        addr[dev] = (float3 *) p;
    }
    *out = addr[dev];
    return PRR_OK;
}

} // namespace
} // namespace prr

extern "C" int prr_render_noalloc(prr_scene *scene, const prr_render_settings *settings,
                                  float *out_rgb, uint64_t *out_rays, void *stream) {
    using namespace prr;
    if (!scene || !settings || !out_rgb)
        return fail(PRR_ERR_INVALID_ARGUMENT, "scene, settings and out_rgb are required");
    Scene &s = *reinterpret_cast<Scene *>(scene);
    if (!s.built)
        return fail(PRR_ERR_NOT_BUILT, "scene not built (call prr_scene_build)");
    prr_render_settings rs = *settings;
    if (int rc = validate_render(s, rs))
        return rc;
    if (rs.mode != PRR_RENDER_PLAIN)
        return fail(PRR_ERR_UNSUPPORTED, "prr_render_noalloc renders with the plain kernel only");
    if (rs.min_spp < rs.max_spp)
        return fail(PRR_ERR_UNSUPPORTED, "prr_render_noalloc supports fixed spp only "
                                         "(min_spp == max_spp)");
    const int ww = rs.x1 - rs.x0, wh = rs.y1 - rs.y0;
    const int64_t npix = (int64_t) ww * wh;
    if (npix > kNoAllocPartials)
        return fail(PRR_ERR_INVALID_ARGUMENT,
                    "window of " + std::to_string(npix) + " pixels exceeds the " +
                        std::to_string(kNoAllocPartials) +
                        " partial sums of the allocation-free renderer");
    const DevScene &S = s.dev;
    RenderArgs a{};
    a.W = s.width;
    a.H = s.height;
    a.x0 = rs.x0;
    a.y0 = rs.y0;
    a.ww = ww;
    a.wh = wh;
    a.min_spp = rs.min_spp;
    a.max_spp = rs.max_spp;
    a.threshold = rs.variance_threshold;
    a.max_depth = rs.max_depth;
    a.clamp = rs.indirect_clamp;
    a.seed = rs.seed;
    a.spp_begin = rs.sample_offset;
    a.spp_end = rs.sample_offset + rs.max_spp;
    a.rays = (unsigned long long *) out_rays;
    int slices = rs.slices > 0 ? rs.slices : 1;
    if (rs.slices <= 0) {
        const int64_t want = (int64_t) device_sm_count() * 1024 * 2;
        while (npix * slices < want && slices * 2 <= rs.max_spp)
            slices *= 2;
    }
    slices = std::max(1, std::min(slices, rs.max_spp));
    if (npix * slices > kNoAllocPartials) {
        // an explicit slice count fixes the summation order, so it is not cut
        // silently; the automatic choice only aims to fill the GPU
        if (rs.slices > 0)
            return fail(PRR_ERR_INVALID_ARGUMENT,
                        std::to_string(slices) + " slices of " + std::to_string(npix) +
                            " pixels exceed the " + std::to_string(kNoAllocPartials) +
                            " partial sums of the allocation-free renderer");
        slices = (int) (kNoAllocPartials / npix);
    }
    a.slices = slices;
    a.tlas_cap = S.tlas_depth + 1;
    const int bcap = S.blas_depth + 1;
    const size_t smem = (size_t) (a.tlas_cap + bcap) * kTileW * kTileH * sizeof(uint2);
    if (smem > 200 * 1024)
        return fail(PRR_ERR_UNSUPPORTED, "BVH too deep for the shared-memory stacks");
    float3 *partial = nullptr;
    if (int rc = noalloc_partials(&partial))
        return rc;
    a.partial = partial;
    cudaStream_t st = (cudaStream_t) stream;
    std::lock_guard<std::mutex> g(s.mu);
    if (out_rays)
        PRR_CUDA_TRY(cudaMemsetAsync(out_rays, 0, 2 * sizeof(uint64_t), st));
    if (smem > 48 * 1024)
        PRR_CUDA_TRY(cudaFuncSetAttribute(k_render_plain,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
    const int tiles = ((ww + kTileW - 1) / kTileW) * ((wh + kTileH - 1) / kTileH);
    k_render_plain<<<dim3(tiles, slices), kTileW * kTileH, smem, st>>>(S, a);
    PRR_CUDA_TRY(cudaGetLastError());
    k_render_resolve<<<(int) ((npix + 255) / 256), 256, 0, st>>>(partial, (int) npix, slices,
                                                                  nullptr, rs.max_spp, out_rgb,
                                                                  nullptr);
    PRR_CUDA_TRY(cudaGetLastError());
    return PRR_OK;
}

