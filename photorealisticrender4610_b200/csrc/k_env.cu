// Environment-map importance-sampling tables on the device: the restatement of
// EnvMap::buildCDF (EnvMap.hpp:189-224).
//
// Each row's conditional CDF is a running float sum of luminance * sin(theta)
// over the row. Float addition is not associative, so to reproduce the
// reference's CDF to the bit the running sum is taken in column order by one
// thread per row; the row's pixels are first staged through shared memory
// with coalesced loads, and the normalisation and write-back are spread over
// the block. Rows run in parallel, one block each. The marginal CDF over the
// row sums is the same sequential sum over rows. Guide tables for the
// samplers' searches are built last.
#include "prr_internal.h"

namespace prr {
namespace {

constexpr int kEnvBlock = 256;

__global__ void k_env_rows(const float4 *__restrict__ px, const float *__restrict__ row_sin,
                           int w, int h, float *__restrict__ cdf, float *__restrict__ row_sums) {
    extern __shared__ float lum[]; // w floats
    const int row = blockIdx.x;
    if (row >= h)
        return;
    const float sin_t = row_sin[row];
    const float4 *src = px + (size_t) row * w;
    for (int c = threadIdx.x; c < w; c += blockDim.x) {
        const float4 p = src[c];
        // EnvMap::luminance (EnvMap.hpp:181-183) times sin(theta)
        lum[c] = (0.2126f * p.x + 0.7152f * p.y + 0.0722f * p.z) * sin_t;
    }
    __syncthreads();
    __shared__ float total;
    if (threadIdx.x == 0) {
        float s = 0.f;
        for (int c = 0; c < w; c++) {
            s += lum[c];
            lum[c] = s;
        }
        total = s;
        row_sums[row] = s;
    }
    __syncthreads();
    const float s = total;
    float *dst = cdf + (size_t) row * w;
    for (int c = threadIdx.x; c < w; c += blockDim.x)
        dst[c] = (s > 0.f) ? lum[c] / s : lum[c];
}

__global__ void k_env_marginal(const float *__restrict__ row_sums, int h,
                               float *__restrict__ marginal, float *__restrict__ total_out) {
    extern __shared__ float acc[]; // h floats
    for (int r = threadIdx.x; r < h; r += blockDim.x)
        acc[r] = row_sums[r];
    __syncthreads();
    __shared__ float total;
    if (threadIdx.x == 0) {
        float t = 0.f;
        for (int r = 0; r < h; r++) {
            t += acc[r];
            acc[r] = t;
        }
        total = t;
        *total_out = t;
    }
    __syncthreads();
    const float t = total;
    for (int r = threadIdx.x; r < h; r += blockDim.x)
        marginal[r] = (t > 0.f) ? acc[r] / t : acc[r];
}

// One block per table (block 0: the marginal, block r + 1: row r): entry k
// = lower_bound(cdf, k / G), by the same search the samplers run; the
// table's first entry becomes -1 when its CDF is not non-decreasing (NaN or
// a decrease), so that the samplers search it whole.
__global__ void k_env_guide(const float *__restrict__ cdf, const float *__restrict__ marginal,
                            int w, int h, int G, int32_t *__restrict__ guide) {
    const int b = blockIdx.x;
    const float *a = b == 0 ? marginal : cdf + (size_t) (b - 1) * w;
    const int n = b == 0 ? h : w;
    int32_t *g = guide + (size_t) b * (G + 1);
    __shared__ int bad;
    if (threadIdx.x == 0)
        bad = 0;
    __syncthreads();
    for (int i = threadIdx.x; i + 1 < n; i += blockDim.x)
        if (!(a[i] <= a[i + 1]))
            bad = 1;
    if (threadIdx.x == 0 && !(a[0] >= 0.f))
        bad = 1;
    for (int k = threadIdx.x; k <= G; k += blockDim.x) {
        const float t = (float) k / (float) G;
        int lo = 0, len = n;
        while (len > 0) {
            const int half = len >> 1;
            if (a[lo + half] < t) {
                lo += half + 1;
                len -= half + 1;
            } else {
                len = half;
            }
        }
        g[k] = lo;
    }
    __syncthreads();
    if (threadIdx.x == 0 && bad)
        g[0] = -1;
}

} // namespace

int launch_env_cdf(Scene &s, cudaStream_t st) {
    const int w = s.env_w, h = s.env_h;
    const size_t row_smem = (size_t) w * sizeof(float);
    const size_t col_smem = (size_t) h * sizeof(float);
    if (row_smem > 200 * 1024 || col_smem > 200 * 1024)
        return fail(PRR_ERR_UNSUPPORTED, "environment map too large for the CDF kernels");
    if (row_smem > 48 * 1024)
        PRR_CUDA_TRY(cudaFuncSetAttribute(k_env_rows, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int) row_smem));
    if (col_smem > 48 * 1024)
        PRR_CUDA_TRY(cudaFuncSetAttribute(k_env_marginal,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int) col_smem));
    DevBuf sums;
    PRR_CUDA_TRY(sums.alloc((size_t) (h + 1) * sizeof(float)));
    k_env_rows<<<h, kEnvBlock, row_smem, st>>>(s.d_env_px.as<float4>(), s.d_env_rowsin.as<float>(),
                                               w, h, s.d_env_cdf.as<float>(), sums.as<float>());
    PRR_CUDA_TRY(cudaGetLastError());
    k_env_marginal<<<1, kEnvBlock, col_smem, st>>>(sums.as<float>(), h,
                                                   s.d_env_marginal.as<float>(),
                                                   sums.as<float>() + h);
    PRR_CUDA_TRY(cudaGetLastError());
    k_env_guide<<<h + 1, kEnvBlock, 0, st>>>(s.d_env_cdf.as<float>(), s.d_env_marginal.as<float>(),
                                             w, h, kEnvGuide, s.d_env_guide.as<int32_t>());
    PRR_CUDA_TRY(cudaGetLastError());
    float total = 0.f;
    PRR_CUDA_TRY(cudaMemcpyAsync(&total, sums.as<float>() + h, sizeof(float),
                                 cudaMemcpyDeviceToHost, st));
    PRR_CUDA_TRY(cudaStreamSynchronize(st));
    s.dev.env.total = total;
    return PRR_OK;
}

} // namespace prr
