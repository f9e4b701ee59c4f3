// Device side of the render server's megakernel steps (the server's other
// step kind runs on the wavefront integrator, k_wavefront.cu): one launch
// renders the next sample chunk of every admitted request at once. Each block takes one work item -- a
// (request, 16x8 pixel tile) pair -- from a table the host fills per step, so
// requests of different scenes, sizes and sample counts share the launch.
// Scenes stay resident: every request points at its scene's DevScene, kept in
// device memory by the server.
//
// A request's samples are processed in fixed chunks (its own chunk size, fixed
// at admission), each pixel summing its chunk's samples in order, and chunk
// sums are added to the film in chunk order: a request's image therefore does
// not depend on which other requests shared its launches.
#include "integrator.cuh"
#include "prr_internal.h"
#include "serve.h"

namespace prr {
namespace {

constexpr int kTileW = 16, kTileH = 8;

__global__ void __launch_bounds__(kTileW *kTileH)
    k_serve_step(const ServeItem *__restrict__ items, ServeReq *reqs, int tlas_cap) {
    extern __shared__ uint2 smem[];
    SmemStack tst{smem + threadIdx.x, (int) blockDim.x, 0};
    SmemStack bst{smem + (size_t) tlas_cap * blockDim.x + threadIdx.x, (int) blockDim.x, 0};
    const ServeItem it = items[blockIdx.x];
    const ServeReq &r = reqs[it.req];
    const DevScene &S = *r.scene;
    const int tiles_x = (r.ww + kTileW - 1) / kTileW;
    const int lx = (it.tile % tiles_x) * kTileW + (int) (threadIdx.x % kTileW);
    const int ly = (it.tile / tiles_x) * kTileH + (int) (threadIdx.x / kTileW);
    PathCounters cnt{0, 0};
    if (lx < r.ww && ly < r.wh) {
        const int i = r.x0 + lx, j = r.y0 + ly;
        const uint32_t m = (uint32_t) i + (uint32_t) j * (uint32_t) r.camera.width;
        V3 acc = v3(0.f);
        for (int n = r.s0; n < r.s1; n++) {
            Rng rng{path_state(r.seed, m, (uint32_t) n)};
            const float xo = rng.next();
            const float yo = rng.next();
            const Ray3 ray = generate_ray(r.camera, i, j, xo, yo, rng);
            V3 s = cast_ray(S, ray, r.max_depth, r.clamp, rng, tst, bst, cnt);
            if (isnan(s.x) || isnan(s.y) || isnan(s.z))
                s = v3(0.f);
            acc = acc + s;
        }
        float3 &f = r.film[lx + ly * r.ww];
        f.x += acc.x;
        f.y += acc.y;
        f.z += acc.z;
    }
    unsigned long long a = cnt.closest + cnt.shadow;
    for (int off = 16; off > 0; off >>= 1)
        a += __shfl_down_sync(0xffffffffu, a, off);
    if ((threadIdx.x & 31) == 0 && a)
        atomicAdd(&reqs[it.req].rays, a);
}

__global__ void k_serve_resolve(const float3 *__restrict__ film, int npix, int n, float *out) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= npix)
        return;
    const float3 f = film[q];
    out[(size_t) q * 3 + 0] = f.x / (float) n;
    out[(size_t) q * 3 + 1] = f.y / (float) n;
    out[(size_t) q * 3 + 2] = f.z / (float) n;
}

} // namespace

int serve_launch_step(const ServeItem *d_items, int n_items, ServeReq *d_reqs, int tlas_cap,
                      int blas_cap, cudaStream_t st) {
    if (n_items == 0)
        return PRR_OK;
    const size_t smem = (size_t) (tlas_cap + blas_cap) * kTileW * kTileH * sizeof(uint2);
    if (smem > 200 * 1024)
        return fail(PRR_ERR_UNSUPPORTED, "BVH too deep for the shared-memory stacks");
    if (smem > 48 * 1024)
        PRR_CUDA_TRY(cudaFuncSetAttribute(k_serve_step, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int) smem));
    k_serve_step<<<n_items, kTileW * kTileH, smem, st>>>(d_items, d_reqs, tlas_cap);
    PRR_CUDA_TRY(cudaGetLastError());
    return PRR_OK;
}

int serve_resolve(const float3 *film, int npix, int n, float *out, cudaStream_t st) {
    k_serve_resolve<<<(npix + 255) / 256, 256, 0, st>>>(film, npix, n, out);
    PRR_CUDA_TRY(cudaGetLastError());
    return PRR_OK;
}

int serve_tiles(int ww, int wh) {
    return ((ww + kTileW - 1) / kTileW) * ((wh + kTileH - 1) / kTileH);
}

} // namespace prr
