// Caustic photons on the device: PhotonMap::emit / trace (Photon.cpp:96-188),
// PhotonGrid::build (Photon.cpp:24-53) and the fixed-radius
// PhotonMap::estimateIrradiance (Photon.cpp:55-94), plus a k-nearest-capped
// gather and a caustic render of the first diffuse camera hit.
//
// Emission: photon i draws from stream (seed, i, 0xFFFFFFFF) and is traced by
// one thread with the recursion of PhotonMap::trace unrolled into a loop.
// Stored records are appended with a key (photon index, record number) and
// then sorted, so the photon array is in the canonical order (by photon, then
// by trace order) no matter how the appends interleaved.
//
// Grid: the reference bins photons into an unordered_map keyed by cell index
// with per-cell vectors in insertion order, and a query walks the cell box in
// x, y, z order. Here cells are numbered in that walk order (x slowest, z
// fastest) and photons sorted by (cell, position in the photon array) --
// unique keys, so the order is fully determined. A table of lower bounds
// (for each cell, the first sorted slot of that cell or a later one) replaces
// the hash map: the cells (cx, cy, z0..z1) of a query box are consecutive, so
// a column of the box is one slot range, read with two lookups. A query
// therefore adds the same photons in the same order as the reference and gets
// the same float sum.
//
// Sorting: an in-house bitonic sort over 64-bit keys (global passes for long
// strides, shared-memory passes for strides below 2048), in one cooperative
// launch when the device holds all of its blocks at once.
#include "integrator.cuh"
#include "prr_internal.h"

#include <cooperative_groups.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

namespace cg = cooperative_groups;

namespace prr {

struct PhotonMap {
    DevBuf rec;      // n x 9 floats: position, direction, power (canonical order)
    DevBuf owner;    // n int32: emitting photon
    int64_t n = 0;
    // grid
    bool built = false;
    float radius = 0.01f; // PhotonMap::photon_radius default (Photon.hpp:36)
    float inside_sq = 1e-4f; // the largest float s with sqrtf(s) <= radius
    int res = 0;
    float bmin[3] = {0, 0, 0}, cs[3] = {1, 1, 1};
    DevBuf order;    // n int32: photon index, sorted by (cell, index)
    DevBuf first;    // res^3 + 1 int32: first sorted slot of each cell or a later one
                     // (cells in the walk's order: x slowest, z fastest), n past the last
    DevBuf tiles;    // suffix minima of the cell table's tiles (build scratch)
    DevBuf sorted;   // n x 2 float4 in `order`: position + power r, then power g b + the
                     // slot's cell as int bits (gathers read a cell's photons
                     // contiguously and stop where the cell changes)
    DevBuf params;   // device copy of the grid parameters
    DevBuf scratch;
    // kernels launched by calls on this map (emit, build, gather, caustic
    // render); renders take the map read-only, hence mutable
    mutable std::atomic<int64_t> launches{0};
};

namespace {

constexpr float kPhotonEps = 1e-3f; // EPSILON (global.hpp:12)

struct PhotonRecord {
    V3 pos, dir, power;
};

// ---------------------------------------------------------------- emission
struct EmitArgs {
    int64_t n_photons;
    uint64_t seed;
    int max_depth;
    float *rec;                 // capacity x 9
    unsigned long long *keys;   // capacity: (photon << 5 | record) << 32 | slot
    unsigned *count;
    int64_t capacity;
    int tlas_cap;
};

// sampleCosineHemisphere (BRDFUtils.hpp:66-73)
__device__ __forceinline__ V3 sample_cosine(V3 N, Rng &rng) {
    const float r1 = rng.next();
    const float r2 = rng.next();
    const float r = sqrtf(r1);
    const float phi = 2.f * PRR_PI * r2;
    return to_world(build_tbn(N), v3(r * cosf(phi), r * sinf(phi), sqrtf(smax(0.f, 1.f - r1))));
}

__global__ void k_photon_emit(DevScene S, EmitArgs a) {
    extern __shared__ uint2 smem[];
    SmemStack tst{smem + threadIdx.x, (int) blockDim.x, 0, S.tlas_depth + 1, S.check};
    SmemStack bst{smem + (size_t) a.tlas_cap * blockDim.x + threadIdx.x, (int) blockDim.x, 0,
                  S.blas_depth + 1, S.check};
    const int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n_photons)
        return;
    Rng rng{path_state(a.seed, (uint32_t) i, 0xFFFFFFFFu)};
    // PhotonMap::emit body (Photon.cpp:166-180)
    const LightPoint lp = sample_light(S, rng);
    const float light_pdf = 1.0f / S.total_emit_area;
    const float area = 1.0f / light_pdf;
    const V3 dir0 = sample_cosine(lp.n, rng);
    const DevMaterial &lm = S.materials[lp.material];
    V3 power = v3(lm.emission[0], lm.emission[1], lm.emission[2]) * area / (float) a.n_photons;
    V3 pos = lp.p + lp.n * kPhotonEps;
    V3 dir = dir0;
    bool caustic = false;
    int stored = 0;
    // PhotonMap::trace (Photon.cpp:96-154), tail recursion as a loop
    for (int depth = 0; depth <= a.max_depth; depth++) {
        const Inter hit = intersect(S, Ray3{pos, dir}, tst, bst);
        if (!hit.hit)
            break;
        const DevMaterial &m = S.materials[hit.mat];
        if (m.kind == kMatEmissive)
            break;
        const V3 gn = dot(dir, hit.n) < 0.0f ? hit.n : -hit.n;
        if (m.kind == kMatMirror || m.kind == kMatGlass) {
            Shading sd;
            sd.f.N = gn; // trace fills only Ng and N (Photon.cpp:108-110)
            const BSDFSample bs = delta_sample(m, sd, -dir, rng);
            caustic = true;
            power = power * bs.f;
            dir = bs.wi;
            pos = hit.p + (dot(bs.wi, gn) > 0.0f ? gn : -gn) * kPhotonEps;
            continue;
        }
        if (depth > 0 && caustic) {
            const unsigned slot = atomicAdd(a.count, 1u);
            if ((int64_t) slot < a.capacity) {
                float *r = a.rec + (size_t) slot * 9;
                r[0] = hit.p.x;
                r[1] = hit.p.y;
                r[2] = hit.p.z;
                r[3] = dir.x;
                r[4] = dir.y;
                r[5] = dir.z;
                r[6] = power.x;
                r[7] = power.y;
                r[8] = power.z;
                a.keys[slot] = ((((unsigned long long) i << 5) | (unsigned) stored) << 32) | slot;
            }
            stored++;
        }
        const float survival = smin(1.0f, max3(power));
        if (!(rng.next() < survival && depth < a.max_depth))
            break;
        const Shading sd = build_shading(S, m, gn, hit.a);
        const V3 wo = -dir;
        const BSDFSample bs = diffuse_sample(m, sd, wo, rng);
        if (bs.pdf < 1e-6f)
            break;
        const float cos_t = smax(0.0f, dot(bs.wi, gn));
        const V3 weight = bs.f * cos_t / bs.pdf;
        power = power * weight;
        const float s2 = smin(1.0f, max3(power));
        if (rng.next() > s2)
            break;
        power = power / s2;
        pos = hit.p + gn * kPhotonEps;
        dir = bs.wi;
    }
}

// ---------------------------------------------------------------- sorting
__global__ void k_fill_keys(unsigned long long *keys, int64_t from, int64_t to) {
    const int64_t i = from + (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (i < to)
        keys[i] = ~0ull;
}

__global__ void k_bitonic_global(unsigned long long *keys, int64_t j, int64_t k, int64_t n) {
    const int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const int64_t l = i ^ j;
    if (l <= i)
        return;
    const bool up = (i & k) == 0;
    const unsigned long long a = keys[i], b = keys[l];
    if ((a > b) == up) {
        keys[i] = b;
        keys[l] = a;
    }
}

// strides j0, j0/2, ..., 1 of stage k inside 2048-element tiles
__global__ void k_bitonic_shared(unsigned long long *keys, int64_t k, int j0) {
    __shared__ unsigned long long t[2048];
    const int64_t base = (int64_t) blockIdx.x * 2048;
    t[threadIdx.x] = keys[base + threadIdx.x];
    t[threadIdx.x + 1024] = keys[base + threadIdx.x + 1024];
    __syncthreads();
    for (int j = j0; j > 0; j >>= 1) {
        for (int h = 0; h < 2; h++) {
            const int i = (int) threadIdx.x + h * 1024;
            const int l = i ^ j;
            if (l > i) {
                const bool up = ((base + i) & k) == 0;
                const unsigned long long a = t[i], b = t[l];
                if ((a > b) == up) {
                    t[i] = b;
                    t[l] = a;
                }
            }
        }
        __syncthreads();
    }
    keys[base + threadIdx.x] = t[threadIdx.x];
    keys[base + threadIdx.x + 1024] = t[threadIdx.x + 1024];
}

// The whole bitonic sort of n2 keys in one cooperative launch of n2 / 2048
// blocks: block b keeps keys [2048 b, 2048 b + 2048) in shared memory for the
// strides below 2048 of every stage, and the strides of 2048 and more run on
// global memory between grid-wide barriers (the launch guarantees that all
// blocks are resident, so the barriers complete). The same compare-exchange
// network as k_bitonic_global + k_bitonic_shared, in the same order.
__global__ void __launch_bounds__(1024) k_bitonic_coop(unsigned long long *keys, int64_t n2) {
    cg::grid_group grid = cg::this_grid();
    __shared__ unsigned long long t[2048];
    const int64_t base = (int64_t) blockIdx.x * 2048;
    const int64_t nthreads = (int64_t) gridDim.x * blockDim.x;
    const int64_t gtid = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
    t[threadIdx.x] = keys[base + threadIdx.x];
    t[threadIdx.x + 1024] = keys[base + threadIdx.x + 1024];
    __syncthreads();
    for (int64_t k = 2; k <= n2; k <<= 1) {
        int64_t j = k >> 1;
        if (j >= 2048) {
            keys[base + threadIdx.x] = t[threadIdx.x];
            keys[base + threadIdx.x + 1024] = t[threadIdx.x + 1024];
            grid.sync();
            for (; j >= 2048; j >>= 1) {
                for (int64_t i = gtid; i < n2; i += nthreads) {
                    const int64_t l = i ^ j;
                    if (l > i) {
                        const bool up = (i & k) == 0;
                        const unsigned long long a = keys[i], b = keys[l];
                        if ((a > b) == up) {
                            keys[i] = b;
                            keys[l] = a;
                        }
                    }
                }
                grid.sync();
            }
            t[threadIdx.x] = keys[base + threadIdx.x];
            t[threadIdx.x + 1024] = keys[base + threadIdx.x + 1024];
            __syncthreads();
        }
        for (; j > 0; j >>= 1) {
            for (int h = 0; h < 2; h++) {
                const int i = (int) threadIdx.x + h * 1024;
                const int l = i ^ (int) j;
                if (l > i) {
                    const bool up = ((base + i) & k) == 0;
                    const unsigned long long a = t[i], b = t[l];
                    if ((a > b) == up) {
                        t[i] = b;
                        t[l] = a;
                    }
                }
            }
            __syncthreads();
        }
    }
    keys[base + threadIdx.x] = t[threadIdx.x];
    keys[base + threadIdx.x + 1024] = t[threadIdx.x + 1024];
}

// Blocks of k_bitonic_coop that can be resident at once on this device (0:
// no cooperative launch).
int64_t coop_sort_blocks() {
    static const int64_t blocks = [] {
        int dev = 0, coop = 0, per_sm = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess ||
            !coop ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_bitonic_coop, 1024, 0) !=
                cudaSuccess) {
            cudaGetLastError();
            return int64_t(0);
        }
        return (int64_t) per_sm * device_sm_count();
    }();
    return blocks;
}

// Sorts keys[0, n2) ascending; n2 is a power of two >= 2048. One cooperative
// launch when the device holds all n2 / 2048 blocks at once, else a launch
// per stage (and per large stride). Adds its kernel launches to *launches.
int bitonic_sort(unsigned long long *keys, int64_t n2, cudaStream_t st,
                 std::atomic<int64_t> *launches) {
    if (n2 / 2048 <= coop_sort_blocks()) {
        void *args[] = {(void *) &keys, (void *) &n2};
        PRR_CUDA_TRY(cudaLaunchCooperativeKernel((const void *) k_bitonic_coop,
                                                 dim3((unsigned) (n2 / 2048)), dim3(1024), args,
                                                 0, st));
        *launches += 1;
        return PRR_OK;
    }
    const int tb = 256;
    const unsigned grid = (unsigned) ((n2 + tb - 1) / tb);
    int64_t count = 0;
    for (int64_t k = 2; k <= n2; k <<= 1) {
        int64_t j = k >> 1;
        for (; j >= 1024; j >>= 1, count++)
            k_bitonic_global<<<grid, tb, 0, st>>>(keys, j, k, n2);
        k_bitonic_shared<<<(unsigned) (n2 / 2048), 1024, 0, st>>>(keys, k, (int) j);
        count++;
    }
    *launches += count;
    PRR_CUDA_TRY(cudaGetLastError());
    return PRR_OK;
}

// The largest float s with sqrtf(s) <= r (r finite and > 0): the threshold
// on a squared distance that decides `sqrtf(d.d) <= r` without the square
// root (IEEE sqrt is correctly rounded and monotone, on the host as on the
// device built with IEEE sqrt).
float inside_square(float r) {
    if (!std::isfinite(r))
        return r;
    float t = r * r;
    while (t > 0.f && std::sqrt(t) > r)
        t = std::nextafter(t, 0.f);
    for (;;) {
        const float n = std::nextafter(t, INFINITY);
        if (!(std::sqrt(n) <= r))
            break;
        t = n;
    }
    return t;
}

int64_t pow2_at_least(int64_t n) {
    int64_t p = 2048;
    while (p < n)
        p <<= 1;
    return p;
}

__global__ void k_gather_records(const unsigned long long *keys, const float *src, int64_t n,
                                 float *dst, int32_t *owner) {
    const int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const unsigned long long k = keys[i];
    const unsigned slot = (unsigned) (k & 0xffffffffu);
    for (int q = 0; q < 9; q++)
        dst[i * 9 + q] = src[(size_t) slot * 9 + q];
    owner[i] = (int32_t) ((k >> 32) >> 5);
}

// ---------------------------------------------------------------- grid
// kOccWords 32-bit words hold one bit per slab of an axis (res <= kMaxRes)
constexpr int kMaxRes = 200; // PhotonGrid::build's resolution cap (Photon.cpp:44-46)
constexpr int kOccWords = 7;

struct GridParams {
    float bmin[3], bmax[3], cs[3];
    int res;
    // occupancy of the grid's slabs along x, y and z: bit c of occ[a] is set
    // when some photon lies in a cell whose coordinate on axis a is c. A cell
    // can hold photons only if its three slabs are occupied, so the gathers
    // skip the other cells without reading the cell table (the same cells in
    // the same order as the reference's walk, minus ones known to be empty).
    uint32_t occ[3][kOccWords];
};

__global__ void k_bounds(const float *rec, int64_t n, float *partial) {
    // per block min/max of positions; exact in any order
    __shared__ float s[6][256];
    float mn[3] = {kInf, kInf, kInf}, mx[3] = {-kInf, -kInf, -kInf};
    for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t) gridDim.x * blockDim.x)
        for (int k = 0; k < 3; k++) {
            const float v = rec[i * 9 + k];
            mn[k] = fminf(mn[k], v);
            mx[k] = fmaxf(mx[k], v);
        }
    for (int k = 0; k < 3; k++) {
        s[k][threadIdx.x] = mn[k];
        s[3 + k][threadIdx.x] = mx[k];
    }
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int) threadIdx.x < w)
            for (int k = 0; k < 3; k++) {
                s[k][threadIdx.x] = fminf(s[k][threadIdx.x], s[k][threadIdx.x + w]);
                s[3 + k][threadIdx.x] = fmaxf(s[3 + k][threadIdx.x], s[3 + k][threadIdx.x + w]);
            }
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int k = 0; k < 6; k++)
            partial[blockIdx.x * 6 + k] = s[k][0];
}

// PhotonGrid::build's parameters (Photon.cpp:27-46): one block folds the
// per-block bounds (min and max are exact in any order), its first thread
// derives the grid.
__global__ void __launch_bounds__(256) k_grid_params(const float *partial, int nb, float radius,
                                                     GridParams *g) {
    __shared__ float s[6][256];
    float mn[3] = {kInf, kInf, kInf}, mx[3] = {-kInf, -kInf, -kInf};
    for (int b = threadIdx.x; b < nb; b += blockDim.x)
        for (int k = 0; k < 3; k++) {
            mn[k] = fminf(mn[k], partial[b * 6 + k]);
            mx[k] = fmaxf(mx[k], partial[b * 6 + 3 + k]);
        }
    for (int k = 0; k < 3; k++) {
        s[k][threadIdx.x] = mn[k];
        s[3 + k][threadIdx.x] = mx[k];
    }
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int) threadIdx.x < w)
            for (int k = 0; k < 3; k++) {
                s[k][threadIdx.x] = fminf(s[k][threadIdx.x], s[k][threadIdx.x + w]);
                s[3 + k][threadIdx.x] = fmaxf(s[3 + k][threadIdx.x], s[3 + k][threadIdx.x + w]);
            }
        __syncthreads();
    }
    if (threadIdx.x != 0)
        return;
    for (int k = 0; k < 3; k++) {
        mn[k] = s[k][0];
        mx[k] = s[3 + k][0];
    }
    for (int k = 0; k < 3; k++) {
        g->bmin[k] = mn[k] - 0.01f;
        g->bmax[k] = mx[k] + 0.01f;
        for (int w = 0; w < kOccWords; w++)
            g->occ[k][w] = 0u;
    }
    const float ex = g->bmax[0] - g->bmin[0], ey = g->bmax[1] - g->bmin[1],
                ez = g->bmax[2] - g->bmin[2];
    int res = (int) (sqrtf(ex * ex + ey * ey + ez * ez) / radius);
    res = max(10, min(kMaxRes, res));
    g->res = res;
    g->cs[0] = ex / (float) res;
    g->cs[1] = ey / (float) res;
    g->cs[2] = ez / (float) res;
}

// cell of each photon through worldToCell / cellToIndex (Photon.cpp:8-22)
__global__ void k_cell_keys(const float *rec, int64_t n, const GridParams *g,
                            unsigned long long *keys) {
    const int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const int res = g->res;
    const int cx = (int) (float) (int) ((rec[i * 9 + 0] - g->bmin[0]) / g->cs[0]);
    const int cy = (int) (float) (int) ((rec[i * 9 + 1] - g->bmin[1]) / g->cs[1]);
    const int cz = (int) (float) (int) ((rec[i * 9 + 2] - g->bmin[2]) / g->cs[2]);
    // cells numbered in the walk's order (x slowest, z fastest), so the cells
    // (cx, cy, z0..z1) of one column are consecutive keys
    const unsigned cell = (unsigned) (cz + cy * res + cx * res * res);
    keys[i] = ((unsigned long long) cell << 32) | (unsigned long long) i;
}

// the slabs each photon's cell occupies (one atomic per axis per photon whose
// cell differs from its predecessor's in the sorted order)
__global__ void k_cell_occupancy(const unsigned long long *keys, int64_t n, GridParams *g) {
    const int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const unsigned cell = (unsigned) (keys[i] >> 32);
    if (i > 0 && (unsigned) (keys[i - 1] >> 32) == cell)
        return;
    const unsigned res = (unsigned) g->res;
    const unsigned c[3] = {cell / (res * res), (cell / res) % res, cell % res};
    for (int a = 0; a < 3; a++)
        atomicOr(&g->occ[a][c[a] >> 5], 1u << (c[a] & 31));
}

// The sorted copy and, at the first slot of each occupied cell, that slot in
// the cell's entry of `first` (the other entries hold a value above any slot;
// k_first_* then turn the table into lower bounds).
__global__ void k_cell_table(const unsigned long long *keys, const float *rec, int64_t n,
                             int32_t *order, int32_t *first, float4 *sorted) {
    const int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const unsigned cell = (unsigned) (keys[i] >> 32);
    const int32_t o = (int32_t) (keys[i] & 0xffffffffu);
    order[i] = o;
    const float *p = rec + (size_t) o * 9;
    sorted[2 * i] = make_float4(p[0], p[1], p[2], p[6]);
    sorted[2 * i + 1] = make_float4(p[7], p[8], 0.f, 0.f);
    if (i == 0 || (unsigned) (keys[i - 1] >> 32) != cell)
        first[cell] = (int32_t) i;
}

// Lower bounds over the cell table: first[c] becomes the first sorted slot
// whose cell is c or later (n when there is none), by a suffix minimum over
// the cells in tiles of 4096: within each tile here, across tiles in
// k_first_tile_mins, both applied in k_first_apply.
constexpr int kFirstTile = 4096;

// Suffix minimum over the threads of a block: thread t gets the minimum of v
// over threads t + 1 .. blockDim.x - 1 (INT_MAX for the last); *total = the
// minimum over all threads.
__device__ int block_suffix_min_excl(int v, int *total) {
    __shared__ int warp_suf[32];
    __shared__ int thread_suf[1024];
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_down_sync(full, v, o);
        if (lane + o < 32)
            v = min(v, y);
    }
    if (lane == 0)
        warp_suf[wid] = v;
    __syncthreads();
    if (wid == 0) {
        int w = lane < nw ? warp_suf[lane] : INT_MAX;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_down_sync(full, w, o);
            if (lane + o < 32)
                w = min(w, y);
        }
        warp_suf[lane] = w;
    }
    __syncthreads();
    thread_suf[threadIdx.x] = min(v, wid + 1 < nw ? warp_suf[wid + 1] : INT_MAX);
    __syncthreads();
    const int excl =
        threadIdx.x + 1 < blockDim.x ? thread_suf[threadIdx.x + 1] : INT_MAX;
    *total = warp_suf[0];
    __syncthreads();
    return excl;
}

// Cells of the table for the grid's resolution (one past the last cell).
__device__ __forceinline__ int64_t table_cells(const GridParams *g) {
    const int64_t r = g->res;
    return r * r * r + 1;
}

// Launched for the largest table; blocks past this grid's table return.
__global__ void __launch_bounds__(1024) k_first_tiles(int32_t *first, const GridParams *g,
                                                      int32_t *tile_min) {
    const int64_t m = table_cells(g);
    if ((int64_t) blockIdx.x * kFirstTile >= m)
        return;
    const int64_t base = (int64_t) blockIdx.x * kFirstTile + (int64_t) threadIdx.x * 4;
    int x[4];
    for (int q = 0; q < 4; q++)
        x[q] = base + q < m ? first[base + q] : INT_MAX;
    x[2] = min(x[2], x[3]);
    x[1] = min(x[1], x[2]);
    x[0] = min(x[0], x[1]);
    int total;
    const int later = block_suffix_min_excl(x[0], &total);
    for (int q = 0; q < 4; q++)
        if (base + q < m)
            first[base + q] = min(x[q], later);
    if (threadIdx.x == 0)
        tile_min[blockIdx.x] = total;
}

// tile_min[b] <- the minimum over the tiles after b (INT_MAX for the last);
// one block, at most 4 * 1024 tiles.
__global__ void __launch_bounds__(1024) k_first_tile_mins(int32_t *tile_min,
                                                          const GridParams *g) {
    const int ntiles = (int) ((table_cells(g) + kFirstTile - 1) / kFirstTile);
    const int base = (int) threadIdx.x * 4;
    int y[4];
    for (int q = 0; q < 4; q++)
        y[q] = base + q < ntiles ? tile_min[base + q] : INT_MAX;
    int suf[4];
    suf[3] = y[3];
    suf[2] = min(y[2], suf[3]);
    suf[1] = min(y[1], suf[2]);
    suf[0] = min(y[0], suf[1]);
    int total;
    const int later = block_suffix_min_excl(suf[0], &total);
    for (int q = 0; q < 4; q++)
        if (base + q < ntiles)
            tile_min[base + q] = min(q < 3 ? suf[q + 1] : INT_MAX, later);
}

__global__ void k_first_apply(int32_t *first, const GridParams *g, const int32_t *after,
                              int32_t n) {
    const int64_t c = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (c < table_cells(g))
        first[c] = min(min(first[c], after[c / kFirstTile]), n);
}

// ---------------------------------------------------------------- gather
struct GridView {
    const float *rec;
    const float4 *sorted;
    const int32_t *order;
    // first[c]: the first sorted slot whose cell is c or later (cells in the
    // walk's order), n when there is none; res^3 + 1 entries
    const int32_t *first;
    const GridParams *g;
    int64_t n;
    float radius;
    // the largest float s with sqrtf(s) <= radius: sqrtf is correctly
    // rounded and monotone, so |d| <= radius exactly when d.d <= inside_sq
    float inside_sq;
};

// pi r^2 as estimateIrradiance computes it (Photon.cpp:87): all in float,
// since the reference redefines M_PI as a float literal (global.hpp:9-10).
__device__ __forceinline__ float disc_area(float r) {
    return PRR_PI * r * r;
}

// The first occupied slab of an axis in [c, hi], or hi + 1.
__device__ __forceinline__ int next_slab(const uint32_t *occ, int c, int hi) {
    while (c <= hi) {
        const uint32_t w = occ[c >> 5] >> (c & 31);
        if (w) {
            c += __ffs(w) - 1;
            return c <= hi ? c : hi + 1;
        }
        c = (c | 31) + 1;
    }
    return hi + 1;
}

// Calls col(a, b) for each column (cx, cy) of the box [x0,x1] x [y0,y1] x
// [z0,z1] whose x and y slabs hold photons, in the reference query's order
// (by x, then y): the sorted slots [a, b) are the photons of the column's
// cells cz = z0..z1, cell after cell, each cell's in photon order -- the
// order the reference's walk over cells by x, then y, then z takes them.
template <class C>
__device__ __forceinline__ void walk_columns(const GridView &v, const GridParams &g, int x0,
                                             int x1, int y0, int y1, int z0, int z1, C &&col) {
    for (int cx = next_slab(g.occ[0], x0, x1); cx <= x1; cx = next_slab(g.occ[0], cx + 1, x1))
        for (int cy = next_slab(g.occ[1], y0, y1); cy <= y1;
             cy = next_slab(g.occ[1], cy + 1, y1)) {
            const int k0 = z0 + cy * g.res + cx * g.res * g.res;
            const int a = v.first[k0];
            const int b = v.first[k0 + (z1 - z0) + 1];
            if (a < b)
                col(a, b);
        }
}

// Calls f(s) for every photon of the cells in the box, in the reference
// query's order (s indexes the cell-sorted arrays).
template <class F>
__device__ __forceinline__ void walk_cells(const GridView &v, const GridParams &g, int x0, int x1,
                                           int y0, int y1, int z0, int z1, F &&f) {
    walk_columns(v, g, x0, x1, y0, y1, z0, z1, [&](int a, int b) {
        for (int s = a; s < b; s++)
            f(s);
    });
}

// The cell box of a query at pos (PhotonGrid::query, Photon.cpp:58-72).
struct GatherBox {
    int x0, x1, y0, y1, z0, z1;
};

__device__ __forceinline__ GatherBox gather_box(const GridParams &g, V3 pos, float r) {
    GatherBox b;
    b.x0 = (int) ((pos.x - r - g.bmin[0]) / g.cs[0]);
    b.y0 = (int) ((pos.y - r - g.bmin[1]) / g.cs[1]);
    b.z0 = (int) ((pos.z - r - g.bmin[2]) / g.cs[2]);
    b.x1 = (int) ((pos.x + r - g.bmin[0]) / g.cs[0]);
    b.y1 = (int) ((pos.y + r - g.bmin[1]) / g.cs[1]);
    b.z1 = (int) ((pos.z + r - g.bmin[2]) / g.cs[2]);
    b.x0 = max(0, b.x0);
    b.x1 = min(g.res - 1, b.x1);
    b.y0 = max(0, b.y0);
    b.y1 = min(g.res - 1, b.y1);
    b.z0 = max(0, b.z0);
    b.z1 = min(g.res - 1, b.z1);
    return b;
}

// Pass 1 of a gather: the sum of the powers within the radius and their
// number, in the reference query's order.
template <bool COUNT = false>
__device__ __forceinline__ V3 radius_sum(const GridView &v, const GatherBox &b, V3 pos,
                                         int &found, unsigned *tested = nullptr,
                                         unsigned *inside = nullptr) {
    V3 e = v3(0.f);
    found = 0;
    walk_cells(v, *v.g, b.x0, b.x1, b.y0, b.y1, b.z0, b.z1, [&](int s) {
        const float4 pa = v.sorted[2 * s];
        const V3 d = v3(pa.x, pa.y, pa.z) - pos;
        // sqrtf(d.d) <= r, decided on d.d
        const float dd = d.x * d.x + d.y * d.y + d.z * d.z;
        if constexpr (COUNT)
            (*tested)++;
        if (dd <= v.inside_sq) {
            if constexpr (COUNT)
                (*inside)++;
            const float4 pb = v.sorted[2 * s + 1];
            e = e + v3(pa.w, pb.x, pb.y);
            found++;
        }
    });
    return e;
}

// Passes 2 and 3 of a gather with more than k photons inside: the k smallest
// (distance, photon index) pairs in a max-heap (the largest kept pair at its
// root), then the powers of the photons at or below the root pair added in
// the walk's order, over the disc through the k-th. Kept out of line: in the
// caustic sample kernel it runs only when the dense-gather queue is full, and
// inlined there its heap code crowded the instruction cache (render 2.97 ->
// 2.87 ms out of line).
__device__ __noinline__ V3 knn_estimate(const GridView &v, const GatherBox &b, V3 pos,
                                        int k_nearest, float *kd, int *kc) {
    const float r = v.radius;
    auto below = [](float da, int ia, float db, int ib) {
        return da < db || (da == db && ia < ib);
    };
    int kept = 0;
    walk_cells(v, *v.g, b.x0, b.x1, b.y0, b.y1, b.z0, b.z1, [&](int s) {
        const float4 pa = v.sorted[2 * s];
        const V3 d = v3(pa.x, pa.y, pa.z) - pos;
        const float dist = sqrtf(d.x * d.x + d.y * d.y + d.z * d.z);
        if (!(dist <= r) || (kept == k_nearest && dist > kd[0]))
            return;
        const int idx = v.order[s];
        if (kept < k_nearest) { // push and sift up
            int c = kept++;
            while (c > 0) {
                const int up = (c - 1) >> 1;
                if (!below(kd[up], kc[up], dist, idx))
                    break;
                kd[c] = kd[up];
                kc[c] = kc[up];
                c = up;
            }
            kd[c] = dist;
            kc[c] = idx;
        } else if (below(dist, idx, kd[0], kc[0])) { // replace the root and sift down
            int c = 0;
            for (;;) {
                int m = 2 * c + 1;
                if (m >= k_nearest)
                    break;
                if (m + 1 < k_nearest && below(kd[m], kc[m], kd[m + 1], kc[m + 1]))
                    m++;
                if (!below(dist, idx, kd[m], kc[m]))
                    break;
                kd[c] = kd[m];
                kc[c] = kc[m];
                c = m;
            }
            kd[c] = dist;
            kc[c] = idx;
        }
    });
    const float rk = kd[0];
    const int ik = kc[0];
    V3 ek = v3(0.f);
    walk_cells(v, *v.g, b.x0, b.x1, b.y0, b.y1, b.z0, b.z1, [&](int s) {
        const float4 pa = v.sorted[2 * s];
        const V3 d = v3(pa.x, pa.y, pa.z) - pos;
        const float dist = sqrtf(d.x * d.x + d.y * d.y + d.z * d.z);
        if (dist < rk || (dist == rk && v.order[s] <= ik)) {
            const float4 pb = v.sorted[2 * s + 1];
            ek = ek + v3(pa.w, pb.x, pb.y);
        }
    });
    return ek / disc_area(rk);
}

// PhotonGrid::query + PhotonMap::estimateIrradiance (Photon.cpp:55-94). With
// k_nearest > 0 and more than k photons inside the radius, the estimate uses
// the k nearest -- the k smallest (distance, photon index) pairs, so ties at
// the k-th distance keep the lower photon index whatever the walk order --
// and the disc through the k-th one: sum / (pi r_k^2), the kept photons added
// in the order the query walks them (as estimateIrradiance adds its photons).
__device__ V3 irradiance(const GridView &v, V3 pos, int k_nearest, float *kd, int *kc) {
    const GatherBox b = gather_box(*v.g, pos, v.radius);
    int found = 0;
    const V3 e = radius_sum(v, b, pos, found);
    if (found == 0)
        return v3(0.f);
    if (!kd || found <= k_nearest)
        return e / disc_area(v.radius);
    return knn_estimate(v, b, pos, k_nearest, kd, kc);
}

constexpr int kMaxK = 64;

__global__ void k_photon_gather(GridView v, const float *q, int64_t n, int k_nearest, float *out) {
    const int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    float kd[kMaxK];
    int kc[kMaxK];
    const V3 e = irradiance(v, v3(q[i * 3], q[i * 3 + 1], q[i * 3 + 2]), k_nearest,
                            k_nearest > 0 ? kd : nullptr, kc);
    out[i * 3] = e.x;
    out[i * 3 + 1] = e.y;
    out[i * 3 + 2] = e.z;
}

// Caustic render: per (pixel, sample), follow the camera ray through the
// specular chain as castRay does (Integrator.cpp:143-169) and, at the first
// non-delta hit, estimate the caustic radiance baseColor/pi * E(x).
struct CausticArgs {
    int W, x0, y0, ww, wh, spp, max_depth, k_nearest, tlas_cap;
    uint64_t seed;
    int sample_offset;
    float *out;
    float4 *samples; // npix x chunk contributions, sample-major
    float4 *acc;     // npix running sums across chunks
    int s0, chunk;   // this launch's samples [s0, s0 + chunk) of each pixel
    unsigned long long *stats; // counting variant: camera hits, gathers, photons
                               // tested, photons inside the radius, dense gathers
    unsigned long long *next;  // work counter of this launch (zeroed before it)
    // gathers with more than k photons inside, selected by k_caustic_dense:
    // 2 float4 per entry (hit point + item index bits, beta * baseColor / pi
    // + the number of photons inside the radius as int bits)
    float4 *dense;
    unsigned *dense_count;     // entries queued (zeroed before each launch)
    int64_t dense_cap;
    unsigned long long *dense_next; // k_caustic_dense's work counter (zeroed too)
};

// walk_cells with the photons of each column shared out over a warp: lane l
// takes the column's photons l, l + 32, ... (every lane walks the same
// columns).
template <class F>
__device__ __forceinline__ void walk_cells_warp(const GridView &v, const GatherBox &b, int lane,
                                                F &&f) {
    walk_columns(v, *v.g, b.x0, b.x1, b.y0, b.y1, b.z0, b.z1, [&](int a, int e) {
        for (int s = a + lane; s < e; s += 32)
            f(s);
    });
}

// The value of rank `want` (1-based) among the candidates' 32-bit keys, by a
// radix select over the key's bytes from the top: each pass histograms one
// byte of the candidates that match the bytes found so far into the warp's
// 256 shared-memory bins and keeps the bin holding the wanted rank. On
// return want is the rank within the candidates whose key equals the result,
// and *equal is how many have that key. walk(f) calls f(s) for this lane's
// share of the items; key_of(s, key) gives item s's key (false: not a
// candidate).
template <class Walk, class K>
__device__ uint32_t warp_radix_select(Walk &&walk, int lane, unsigned *bins, int &want,
                                      int *equal, K &&key_of) {
    const unsigned full = 0xffffffffu;
    uint32_t prefix = 0, mask = 0;
    for (int shift = 24; shift >= 0; shift -= 8) {
        for (int q = lane; q < 256; q += 32)
            bins[q] = 0u;
        __syncwarp();
        walk([&](int s) {
            uint32_t key;
            if (key_of(s, key) && (key & mask) == prefix)
                atomicAdd(&bins[(key >> shift) & 255u], 1u);
        });
        __syncwarp();
        // the bin holding rank `want`: each lane sums 8 bins, a warp scan
        // finds the lane, the lane finds the bin
        unsigned own = 0;
        for (int q = 0; q < 8; q++)
            own += bins[lane * 8 + q];
        unsigned incl = own;
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned y = __shfl_up_sync(full, incl, o);
            if (lane >= o)
                incl += y;
        }
        const unsigned before = incl - own;
        const bool holds = before < (unsigned) want && (unsigned) want <= incl;
        const int src = __ffs(__ballot_sync(full, holds)) - 1;
        int bin = 0;
        unsigned below = 0, in_bin = 0;
        if (holds) {
            unsigned run = before;
            for (int q = 0; q < 8; q++) {
                const unsigned c = bins[lane * 8 + q];
                if ((unsigned) want <= run + c) {
                    bin = lane * 8 + q;
                    below = run;
                    in_bin = c;
                    break;
                }
                run += c;
            }
        }
        bin = __shfl_sync(full, bin, src);
        below = __shfl_sync(full, below, src);
        in_bin = __shfl_sync(full, in_bin, src);
        want -= (int) below;
        prefix |= (uint32_t) bin << shift;
        mask |= 255u << shift;
        *equal = (int) in_bin;
        __syncwarp();
    }
    return prefix;
}

// Candidates per warp that k_caustic_dense holds in shared memory (4 KB; at
// 1,024 the 36 KB blocks left 6 resident per SM, at 512 the 20 KB blocks are
// held to 7 by registers: 4% faster on the caustics frame).
constexpr int kDenseCands = 512;
// Collection walks k_caustic_dense tries before it selects by walking cells.
constexpr int kDenseTries = 4;

// The cells of `big` that can hold photons within t of pos: the cell box of
// the disc of radius t, one cell wider on every side (so rounding in the cell
// arithmetic cannot leave such a photon out), cut to `big`. Walked in the
// same nested x, y, z order, its cells come in the order `big` visits them.
__device__ __forceinline__ GatherBox sub_box(const GridParams &g, const GatherBox &big, V3 pos,
                                             float t) {
    const GatherBox s = gather_box(g, pos, t);
    GatherBox b;
    b.x0 = max(big.x0, s.x0 - 1);
    b.x1 = min(big.x1, s.x1 + 1);
    b.y0 = max(big.y0, s.y0 - 1);
    b.y1 = min(big.y1, s.y1 + 1);
    b.z0 = max(big.z0, s.z0 - 1);
    b.z1 = min(big.z1, s.z1 + 1);
    return b;
}

// The dense gathers of one launch, one warp each (4 per block of 128, the
// next entry from a counter). The k-th smallest (distance, photon index)
// pair, then the kept photons -- at or below that pair -- added in the
// walk's order, as knn_estimate adds them; the item gets scale * E(x), the
// product the render kernel forms for the other items.
//
// Collection first: one walk over the cells that can hold photons within a
// threshold t <= r stores every photon at distance <= t, in walk order, as
// (distance bits, sorted slot) in the warp's shared memory. When at least k
// photons lie within t, the k nearest within r are the k nearest of these
// (any pair at or below the k-th has distance <= t), so the selection and
// the ordered sum run over shared memory. t starts where about 3k of the
// `found` photons inside r would lie if they were spread evenly over the
// disc, and is widened (fewer than k within t) or narrowed (more than the
// warp holds) for up to kDenseTries walks. Failing that the warp selects by
// radix passes that walk the cells of the whole query box: one per byte of
// the distance's bits (non-negative floats order as their bit patterns), one
// more per byte of the photon index when several photons share the k-th
// distance, and the ordered sum in a last walk, 32 photons tested per round.
__global__ void __launch_bounds__(128) k_caustic_dense(GridView v, CausticArgs a) {
    __shared__ unsigned bins_all[4][256];
    __shared__ uint2 cand_all[4][kDenseCands];
    unsigned *bins = bins_all[threadIdx.x >> 5];
    uint2 *cand = cand_all[threadIdx.x >> 5];
    const int64_t n = min((int64_t) *a.dense_count, a.dense_cap);
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const float r = v.radius;
    const int k = a.k_nearest;
    const GridParams &g = *v.g;
    for (;;) {
        unsigned long long e = 0;
        if (lane == 0)
            e = atomicAdd(a.dense_next, 1ull);
        e = __shfl_sync(full, e, 0);
        if ((int64_t) e >= n)
            break;
        const float4 p = a.dense[2 * e], sc = a.dense[2 * e + 1];
        const V3 pos = v3(p.x, p.y, p.z);
        const int found = __float_as_int(sc.w); // photons inside r (> k)
        const GatherBox big = gather_box(g, pos, r);
        auto dist_of = [&](int s) {
            const float4 pa = v.sorted[2 * s];
            const V3 d = v3(pa.x, pa.y, pa.z) - pos;
            return sqrtf(d.x * d.x + d.y * d.y + d.z * d.z);
        };
        float t = r * sqrtf(fminf(1.f, 3.f * (float) k / (float) found));
        int count = -1; // photons collected in shared memory (-1: none usable)
        for (int attempt = 0; attempt < kDenseTries; attempt++) {
            const GatherBox b = sub_box(g, big, pos, t);
            int c = 0;
            walk_columns(v, g, b.x0, b.x1, b.y0, b.y1, b.z0, b.z1, [&](int a0, int e0) {
                for (int base = a0; base < e0; base += 32) {
                    const int s = base + lane;
                    float dist = 0.f;
                    bool take = false;
                    if (s < e0) {
                        dist = dist_of(s);
                        take = dist <= t;
                    }
                    const unsigned m = __ballot_sync(full, take);
                    const int at = c + __popc(m & ((1u << lane) - 1u));
                    if (take && at < kDenseCands)
                        cand[at] = make_uint2(__float_as_uint(dist), (unsigned) s);
                    c += __popc(m);
                }
            });
            __syncwarp();
            if (c >= k && c <= kDenseCands) {
                count = c;
                break;
            }
            if (c < k) {
                if (t >= r)
                    break; // cannot happen while found > k
                t = fminf(r, t * sqrtf(2.f * (float) k / (float) max(c, 1)));
            } else {
                t = t * sqrtf(0.5f * (float) kDenseCands / (float) c);
            }
        }
        int want = k, equal = 0;
        uint32_t dk;
        int ik = 0x7fffffff;
        V3 ek = v3(0.f);
        if (count >= 0) {
            auto walk = [&](auto &&f) {
                for (int q = lane; q < count; q += 32)
                    f(q);
            };
            dk = warp_radix_select(walk, lane, bins, want, &equal, [&](int q, uint32_t &key) {
                key = cand[q].x;
                return true;
            });
            // of the photons at the k-th distance, keep the lowest `want` indices
            if (equal > want) {
                int eq2 = 0;
                ik = (int) warp_radix_select(walk, lane, bins, want, &eq2,
                                             [&](int q, uint32_t &key) {
                                                 key = (uint32_t) v.order[cand[q].y];
                                                 return cand[q].x == dk;
                                             });
            }
            // the ordered sum of the kept powers (lane 0 holds it)
            for (int base = 0; base < count; base += 32) {
                const int q = base + lane;
                bool keep = false;
                V3 pw = v3(0.f);
                if (q < count) {
                    const uint2 cq = cand[q];
                    keep = cq.x < dk || (cq.x == dk && v.order[cq.y] <= ik);
                    if (keep) {
                        const float4 pa = v.sorted[2 * cq.y];
                        const float4 pb = v.sorted[2 * cq.y + 1];
                        pw = v3(pa.w, pb.x, pb.y);
                    }
                }
                for (unsigned km = __ballot_sync(full, keep); km; km &= km - 1) {
                    const int l = __ffs(km) - 1;
                    const V3 w = v3(__shfl_sync(full, pw.x, l), __shfl_sync(full, pw.y, l),
                                    __shfl_sync(full, pw.z, l));
                    ek = ek + w;
                }
            }
        } else {
            const GatherBox &b = big;
            auto walk = [&](auto &&f) { walk_cells_warp(v, b, lane, f); };
            dk = warp_radix_select(walk, lane, bins, want, &equal, [&](int s, uint32_t &key) {
                const float dist = dist_of(s);
                key = __float_as_uint(dist);
                return dist <= r;
            });
            if (equal > want) {
                int eq2 = 0;
                ik = (int) warp_radix_select(walk, lane, bins, want, &eq2,
                                             [&](int s, uint32_t &key) {
                                                 key = (uint32_t) v.order[s];
                                                 return __float_as_uint(dist_of(s)) == dk;
                                             });
            }
            const float rk = __uint_as_float(dk);
            walk_columns(v, g, b.x0, b.x1, b.y0, b.y1, b.z0, b.z1, [&](int a0, int e0) {
                for (int base = a0; base < e0; base += 32) {
                    const int s = base + lane;
                    bool keep = false;
                    V3 pw = v3(0.f);
                    if (s < e0) {
                        const float dist = dist_of(s);
                        keep = dist < rk || (dist == rk && v.order[s] <= ik);
                        if (keep) {
                            const float4 pa = v.sorted[2 * s];
                            const float4 pb = v.sorted[2 * s + 1];
                            pw = v3(pa.w, pb.x, pb.y);
                        }
                    }
                    for (unsigned km = __ballot_sync(full, keep); km; km &= km - 1) {
                        const int l = __ffs(km) - 1;
                        const V3 w = v3(__shfl_sync(full, pw.x, l), __shfl_sync(full, pw.y, l),
                                        __shfl_sync(full, pw.z, l));
                        ek = ek + w;
                    }
                }
            });
        }
        if (lane == 0) {
            const V3 c = v3(sc.x, sc.y, sc.z) * (ek / disc_area(__uint_as_float(dk)));
            a.samples[__float_as_int(p.w)] = make_float4(c.x, c.y, c.z, 0.f);
        }
        __syncwarp();
    }
}

// One (pixel, sample) item per thread at a time: sample n of window pixel q is
// item n * npix + q, so a warp's lanes trace neighbouring pixels; its result
// goes to slot n * npix + q, so the image does not depend on which thread
// took which item. Held to 64 registers (8 resident blocks of 128 instead of
// 7; the in-place k-nearest arrays live in local memory either way).
template <bool COUNT>
__global__ void __launch_bounds__(128, 8) k_caustic_samples(DevScene S, GridView v, CausticArgs a) {
    extern __shared__ uint2 smem[];
    SmemStack tst{smem + threadIdx.x, (int) blockDim.x, 0, S.tlas_depth + 1, S.check};
    SmemStack bst{smem + (size_t) a.tlas_cap * blockDim.x + threadIdx.x, (int) blockDim.x, 0,
                  S.blas_depth + 1, S.check};
    const int64_t npix = (int64_t) a.ww * a.wh;
    const int64_t total = npix * a.chunk;
    float kd[kMaxK];
    int kc[kMaxK];
    unsigned cnt_[5] = {0, 0, 0, 0, 0}; // hits, gathers, photons tested, photons inside,
                                        // gathers with more than k inside
    // Persistent warps take the next 32 items from the launch's counter: a
    // sample through the glass sphere or with a dense k-nearest gather costs
    // many times a plain floor hit, so a fixed share per thread would leave
    // most warps waiting on a few slow ones.
    const int lane = threadIdx.x & 31;
    for (;;) {
        unsigned long long base = 0;
        if (lane == 0)
            base = atomicAdd(a.next, 32ull);
        base = __shfl_sync(0xffffffffu, base, 0);
        if ((int64_t) base >= total)
            break;
        const int64_t t = (int64_t) base + lane;
        if (t >= total)
            continue;
        const int nc = (int) (t / npix);
        const int q = (int) (t - (int64_t) nc * npix);
        const int n = a.s0 + nc;
        const int i = a.x0 + q % a.ww, j = a.y0 + q / a.ww;
        const uint32_t m = (uint32_t) i + (uint32_t) j * (uint32_t) a.W;
        Rng rng{path_state(a.seed, m, (uint32_t) (a.sample_offset + n))};
        const float xo = rng.next();
        const float yo = rng.next();
        Ray3 ray = generate_ray(S.camera, i, j, xo, yo, rng);
        V3 beta = v3(1.f);
        V3 c = v3(0.f);
        bool deferred = false;
        for (int d = 0; d < a.max_depth; d++) {
            tst.sp = 0;
            bst.sp = 0;
            const Inter in = intersect(S, ray, tst, bst);
            if (!in.hit)
                break;
            if constexpr (COUNT)
                cnt_[0]++;
            const DevMaterial &mt = S.materials[in.mat];
            if (mt.kind == kMatEmissive)
                break;
            if (mt.kind == kMatMirror || mt.kind == kMatGlass) {
                const Shading sd = build_shading<true>(S, mt, in.n, in.a);
                const BSDFSample bs = delta_sample(mt, sd, -ray.d, rng);
                if (bs.pdf < 1e-6f)
                    break;
                beta = beta * bs.f / bs.pdf;
                const bool trans = dot(bs.wi, in.n) < 0.f;
                ray = Ray3{in.p + (trans ? -in.n : in.n) * PRR_EPS, bs.wi};
                if (trans)
                    beta = beta * sd.base;
                continue;
            }
            if constexpr (COUNT)
                cnt_[1]++;
            const V3 albedo = mt.tex_base >= 0
                                  ? sample_base_color_ool(S.textures[mt.tex_base], in.a.u, in.a.v)
                                  : v3(mt.base[0], mt.base[1], mt.base[2]);
            const V3 scale = beta * (albedo / PRR_PI);
            const GatherBox b = gather_box(*v.g, in.p, v.radius);
            int found = 0;
            V3 e = radius_sum<COUNT>(v, b, in.p, found, cnt_ + 2, cnt_ + 3);
            if (found == 0) {
                e = v3(0.f);
            } else if (a.k_nearest == 0 || found <= a.k_nearest) {
                e = e / disc_area(v.radius);
            } else {
                if constexpr (COUNT)
                    cnt_[4]++;
                // more than k inside: the selection goes to the dense queue,
                // whose kernel runs such gathers side by side (here one lane
                // would hold its warp); a full queue selects in place
                const unsigned slot = atomicAdd(a.dense_count, 1u);
                if ((int64_t) slot < a.dense_cap) {
                    a.dense[2 * (size_t) slot] =
                        make_float4(in.p.x, in.p.y, in.p.z, __int_as_float((int) t));
                    a.dense[2 * (size_t) slot + 1] =
                        make_float4(scale.x, scale.y, scale.z, __int_as_float(found));
                    deferred = true;
                    break;
                }
                e = knn_estimate(v, b, in.p, a.k_nearest, kd, kc);
            }
            c = scale * e;
            break;
        }
        if (!deferred)
            a.samples[t] = make_float4(c.x, c.y, c.z, 0.f);
    }
    if constexpr (COUNT) {
        for (int k = 0; k < 5; k++) {
            unsigned long long x = cnt_[k];
            for (int off = 16; off > 0; off >>= 1)
                x += __shfl_down_sync(0xffffffffu, x, off);
            if ((threadIdx.x & 31) == 0 && x)
                atomicAdd(a.stats + k, x);
        }
    }
}

// The pixel's sum: the chunk's samples added in sample order to the sums of
// the chunks before (a sample without a diffuse hit adds zero, which leaves
// the non-negative sum unchanged), so the image is the one a per-pixel loop
// over its samples produces; the last chunk writes the mean.
__global__ void k_caustic_film(CausticArgs a) {
    const int64_t npix = (int64_t) a.ww * a.wh;
    const int64_t q = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= npix)
        return;
    V3 acc = v3(0.f);
    if (a.s0 > 0) {
        const float4 p = a.acc[q];
        acc = v3(p.x, p.y, p.z);
    }
    for (int n = 0; n < a.chunk; n++) {
        const float4 c = a.samples[(int64_t) n * npix + q];
        acc = acc + v3(c.x, c.y, c.z);
    }
    if (a.s0 + a.chunk < a.spp) {
        a.acc[q] = make_float4(acc.x, acc.y, acc.z, 0.f);
        return;
    }
    a.out[q * 3] = acc.x / (float) a.spp;
    a.out[q * 3 + 1] = acc.y / (float) a.spp;
    a.out[q * 3 + 2] = acc.z / (float) a.spp;
}

// Contributions held at once per call (16 bytes each): larger renders run in
// chunks of whole samples per pixel.
constexpr int64_t kCausticItems = int64_t(1) << 28;

PhotonMap *PM(prr_photon_map *p) { return reinterpret_cast<PhotonMap *>(p); }
const PhotonMap *PM(const prr_photon_map *p) { return reinterpret_cast<const PhotonMap *>(p); }

GridView view(const PhotonMap &pm) {
    GridView v;
    v.rec = pm.rec.as<float>();
    v.sorted = pm.sorted.as<float4>();
    v.order = pm.order.as<int32_t>();
    v.first = pm.first.as<int32_t>();
    v.g = pm.params.as<GridParams>();
    v.n = pm.n;
    v.radius = pm.radius;
    v.inside_sq = pm.inside_sq;
    return v;
}

} // namespace
} // namespace prr

using namespace prr;

namespace prr {
namespace {

int render_caustics(const prr_scene *scene, const prr_photon_map *pmap,
                    const prr_render_settings *settings, int k_nearest, float *out_rgb,
                    unsigned long long *stats, cudaStream_t st) {
    if (!scene || !pmap || !settings || !out_rgb || k_nearest < 0 || k_nearest > kMaxK)
        return fail(PRR_ERR_INVALID_ARGUMENT, "bad caustic render arguments");
    const Scene &s = *reinterpret_cast<const Scene *>(scene);
    if (!s.built)
        return fail(PRR_ERR_NOT_BUILT, "scene not built (call prr_scene_build)");
    const PhotonMap &pm = *PM(pmap);
    if (!pm.built || pm.n == 0)
        return fail(PRR_ERR_NOT_BUILT, "photon map empty or not built");
    prr_render_settings rs = *settings;
    rs.mode = PRR_RENDER_PLAIN;
    rs.min_spp = rs.max_spp;
    if (int rc = validate_render(s, rs))
        return rc;
    CausticArgs a{};
    a.W = s.width;
    a.x0 = rs.x0;
    a.y0 = rs.y0;
    a.ww = rs.x1 - rs.x0;
    a.wh = rs.y1 - rs.y0;
    a.spp = rs.max_spp;
    a.max_depth = rs.max_depth;
    a.k_nearest = k_nearest;
    a.seed = rs.seed;
    a.sample_offset = rs.sample_offset;
    a.out = out_rgb;
    a.stats = stats;
    a.tlas_cap = s.dev.tlas_depth + 1;
    const int block = 128;
    const size_t smem = (size_t) (a.tlas_cap + s.dev.blas_depth + 1) * block * sizeof(uint2);
    if (smem > 200 * 1024)
        return fail(PRR_ERR_UNSUPPORTED, "BVH too deep for the shared-memory stacks");
    auto kern = stats ? k_caustic_samples<true> : k_caustic_samples<false>;
    if (smem > 48 * 1024)
        PRR_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int) smem));
    const int64_t npix = (int64_t) a.ww * a.wh;
    const int chunk = (int) std::max<int64_t>(1, std::min<int64_t>(a.spp, kCausticItems / npix));
    const int64_t items = npix * chunk;
    // per-call contributions (and, when chunked, running sums) from the
    // library's stream-ordered pool: concurrent calls on other streams get
    // their own
    // (and the dense-gather queue: room for an eighth of the items, 32 B each;
    // a launch with more dense gathers selects the rest in place)
    char *scratch = nullptr;
    const size_t acc_bytes = chunk < a.spp ? (size_t) npix * sizeof(float4) : 0;
    a.dense_cap = k_nearest > 0 ? std::max<int64_t>(1024, items / 8) : 0;
    const size_t dense_bytes = (size_t) a.dense_cap * 2 * sizeof(float4);
    cudaMemPool_t pool;
    PRR_CUDA_TRY(library_pool(&pool));
    PRR_CUDA_TRY(cudaMallocFromPoolAsync(
        (void **) &scratch, (size_t) items * sizeof(float4) + acc_bytes + dense_bytes + 256, pool,
        st));
    a.samples = reinterpret_cast<float4 *>(scratch);
    a.acc = acc_bytes ? reinterpret_cast<float4 *>(scratch + (size_t) items * sizeof(float4))
                      : nullptr;
    a.dense = reinterpret_cast<float4 *>(scratch + (size_t) items * sizeof(float4) + acc_bytes);
    char *tail = scratch + (size_t) items * sizeof(float4) + acc_bytes + dense_bytes;
    a.next = reinterpret_cast<unsigned long long *>(tail);
    a.dense_count = reinterpret_cast<unsigned *>(tail + sizeof(unsigned long long));
    a.dense_next = reinterpret_cast<unsigned long long *>(tail + 2 * sizeof(unsigned long long));
    int bps = 1, dense_bps = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kern, block, smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&dense_bps, k_caustic_dense, 128, 0);
    dense_bps = std::max(1, dense_bps);
    cudaError_t e = cudaSuccess;
    for (int s0 = 0; s0 < a.spp && e == cudaSuccess; s0 += chunk) {
        a.s0 = s0;
        a.chunk = std::min(chunk, a.spp - s0);
        const int64_t total = npix * a.chunk;
        const int64_t grid = std::min<int64_t>((total + block - 1) / block,
                                               (int64_t) device_sm_count() * std::max(1, bps));
        e = cudaMemsetAsync(tail, 0, 3 * sizeof(unsigned long long), st);
        if (e == cudaSuccess) {
            kern<<<(unsigned) grid, block, smem, st>>>(s.dev, view(pm), a);
            pm.launches++;
            e = cudaGetLastError();
        }
        if (e == cudaSuccess && a.dense_cap > 0) {
            k_caustic_dense<<<(unsigned) (device_sm_count() * dense_bps), 128, 0, st>>>(view(pm),
                                                                                       a);
            pm.launches++;
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) {
            k_caustic_film<<<(unsigned) ((npix + 255) / 256), 256, 0, st>>>(a);
            pm.launches++;
            e = cudaGetLastError();
        }
    }
    cudaFreeAsync(scratch, st);
    if (e != cudaSuccess)
        return fail(PRR_ERR_CUDA, std::string("caustic render: ") + cudaGetErrorString(e));
    return PRR_OK;
}

} // namespace
} // namespace prr

extern "C" {

int prr_photon_map_create(prr_photon_map **out) {
    if (!out)
        return fail(PRR_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = reinterpret_cast<prr_photon_map *>(new PhotonMap());
    return PRR_OK;
}

int prr_photon_map_destroy(prr_photon_map *pm) {
    delete PM(pm);
    return PRR_OK;
}

int prr_photon_emit(prr_photon_map *pmap, const prr_scene *scene, int64_t num_photons,
                    uint64_t seed, int max_depth, void *stream) {
    if (!pmap || !scene)
        return fail(PRR_ERR_INVALID_ARGUMENT, "photon map and scene are required");
    const Scene &s = *reinterpret_cast<const Scene *>(scene);
    if (!s.built)
        return fail(PRR_ERR_NOT_BUILT, "scene not built (call prr_scene_build)");
    if (s.dev.n_emissives == 0 || !(s.dev.total_emit_area > 0.f))
        return fail(PRR_ERR_INVALID_ARGUMENT, "scene has no area emitters");
    if (num_photons <= 0 || num_photons >= (int64_t) 1 << 27 || max_depth < 0 || max_depth > 30)
        return fail(PRR_ERR_INVALID_ARGUMENT, "need 0 < num_photons < 2^27, 0 <= max_depth <= 30");
    PhotonMap &pm = *PM(pmap);
    cudaStream_t st = (cudaStream_t) stream;
    const int block = 128;
    const int tcap = s.dev.tlas_depth + 1, bcap = s.dev.blas_depth + 1;
    const size_t smem = (size_t) (tcap + bcap) * block * sizeof(uint2);
    if (smem > 200 * 1024)
        return fail(PRR_ERR_UNSUPPORTED, "BVH too deep for the shared-memory stacks");
    if (smem > 48 * 1024)
        PRR_CUDA_TRY(cudaFuncSetAttribute(k_photon_emit,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
    int64_t capacity = std::max<int64_t>(num_photons, 1 << 16);
    for (int attempt = 0; attempt < 2; attempt++) {
        const int64_t n2 = pow2_at_least(capacity);
        PRR_CUDA_TRY(pm.scratch.ensure((size_t) capacity * 9 * sizeof(float) + n2 * 8 + 64));
        float *rec = pm.scratch.as<float>();
        unsigned long long *keys =
            reinterpret_cast<unsigned long long *>((char *) pm.scratch.ptr + capacity * 9 * 4);
        unsigned *count = reinterpret_cast<unsigned *>((char *) keys + n2 * 8);
        PRR_CUDA_TRY(cudaMemsetAsync(count, 0, sizeof(unsigned), st));
        EmitArgs a{num_photons, seed, max_depth, rec, keys, count, capacity, tcap};
        k_photon_emit<<<(unsigned) ((num_photons + block - 1) / block), block, smem, st>>>(s.dev, a);
        pm.launches++;
        PRR_CUDA_TRY(cudaGetLastError());
        unsigned stored = 0;
        PRR_CUDA_TRY(cudaMemcpyAsync(&stored, count, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
        PRR_CUDA_TRY(cudaStreamSynchronize(st));
        if ((int64_t) stored > capacity) { // rerun with room for every record
            capacity = (int64_t) stored + (stored >> 3) + 1024;
            continue;
        }
        const int64_t n = stored;
        const int64_t np2 = pow2_at_least(std::max<int64_t>(n, 1));
        if (np2 > n) {
            k_fill_keys<<<(unsigned) ((np2 - n + 255) / 256), 256, 0, st>>>(keys, n, np2);
            pm.launches++;
        }
        if (int rc = bitonic_sort(keys, np2, st, &pm.launches))
            return rc;
        PRR_CUDA_TRY(pm.rec.ensure((size_t) std::max<int64_t>(n, 1) * 9 * sizeof(float)));
        PRR_CUDA_TRY(pm.owner.ensure((size_t) std::max<int64_t>(n, 1) * sizeof(int32_t)));
        if (n > 0) {
            k_gather_records<<<(unsigned) ((n + 255) / 256), 256, 0, st>>>(
                keys, rec, n, pm.rec.as<float>(), pm.owner.as<int32_t>());
            pm.launches++;
        }
        PRR_CUDA_TRY(cudaGetLastError());
        PRR_CUDA_TRY(cudaStreamSynchronize(st));
        pm.n = n;
        pm.built = false;
        return PRR_OK;
    }
    return fail(PRR_ERR_INTERNAL, "photon record buffer overflow");
}

int prr_photon_set(prr_photon_map *pmap, const float *records, int64_t n, void *stream) {
    if (!pmap || n < 0 || (n > 0 && !records))
        return fail(PRR_ERR_INVALID_ARGUMENT, "bad photon array");
    PhotonMap &pm = *PM(pmap);
    cudaStream_t st = (cudaStream_t) stream;
    PRR_CUDA_TRY(pm.rec.ensure((size_t) std::max<int64_t>(n, 1) * 9 * sizeof(float)));
    PRR_CUDA_TRY(pm.owner.ensure((size_t) std::max<int64_t>(n, 1) * sizeof(int32_t)));
    if (n > 0) {
        PRR_CUDA_TRY(cudaMemcpyAsync(pm.rec.ptr, records, (size_t) n * 9 * sizeof(float),
                                     cudaMemcpyDefault, st));
        PRR_CUDA_TRY(cudaMemsetAsync(pm.owner.ptr, 0xff, (size_t) n * sizeof(int32_t), st));
    }
    PRR_CUDA_TRY(cudaStreamSynchronize(st));
    pm.n = n;
    pm.built = false;
    return PRR_OK;
}

int prr_photon_build(prr_photon_map *pmap, float radius, void *stream) {
    if (!pmap || !(radius > 0.f))
        return fail(PRR_ERR_INVALID_ARGUMENT, "need a photon map and radius > 0");
    PhotonMap &pm = *PM(pmap);
    cudaStream_t st = (cudaStream_t) stream;
    pm.radius = radius;
    pm.inside_sq = inside_square(radius);
    PRR_CUDA_TRY(pm.params.ensure(sizeof(GridParams)));
    if (pm.n == 0) {
        pm.built = true;
        pm.res = 0;
        return PRR_OK;
    }
    const int64_t n = pm.n;
    const int nb = (int) std::min<int64_t>(1024, (n + 255) / 256);
    const int64_t n2 = pow2_at_least(n);
    PRR_CUDA_TRY(pm.scratch.ensure((size_t) n2 * 8 + (size_t) nb * 6 * 4 + 64));
    unsigned long long *keys = pm.scratch.as<unsigned long long>();
    float *partial = reinterpret_cast<float *>((char *) pm.scratch.ptr + n2 * 8);
    k_bounds<<<nb, 256, 0, st>>>(pm.rec.as<float>(), n, partial);
    k_grid_params<<<1, 256, 0, st>>>(partial, nb, radius, pm.params.as<GridParams>());
    k_cell_keys<<<(unsigned) ((n + 255) / 256), 256, 0, st>>>(pm.rec.as<float>(), n,
                                                              pm.params.as<GridParams>(), keys);
    pm.launches += 3;
    if (n2 > n) {
        k_fill_keys<<<(unsigned) ((n2 - n + 255) / 256), 256, 0, st>>>(keys, n, n2);
        pm.launches++;
    }
    PRR_CUDA_TRY(cudaGetLastError());
    if (int rc = bitonic_sort(keys, n2, st, &pm.launches))
        return rc;
    // the cell table with one entry past the last cell (a column's end), its
    // entries above every slot until k_cell_table marks the occupied cells;
    // sized and cleared for the largest resolution, so that the host need not
    // wait for the grid's own before it launches the rest of the build
    const int64_t m = (int64_t) kMaxRes * kMaxRes * kMaxRes + 1;
    const int ntiles = (int) ((m + kFirstTile - 1) / kFirstTile);
    PRR_CUDA_TRY(pm.order.ensure((size_t) n * sizeof(int32_t)));
    PRR_CUDA_TRY(pm.first.ensure((size_t) m * sizeof(int32_t)));
    PRR_CUDA_TRY(pm.tiles.ensure((size_t) ntiles * sizeof(int32_t)));
    PRR_CUDA_TRY(cudaMemsetAsync(pm.first.ptr, 0x7f, (size_t) m * sizeof(int32_t), st));
    PRR_CUDA_TRY(pm.sorted.ensure((size_t) n * 2 * sizeof(float4)));
    k_cell_table<<<(unsigned) ((n + 255) / 256), 256, 0, st>>>(
        keys, pm.rec.as<float>(), n, pm.order.as<int32_t>(),
        pm.first.as<int32_t>(), pm.sorted.as<float4>());
    k_cell_occupancy<<<(unsigned) ((n + 255) / 256), 256, 0, st>>>(keys, n,
                                                                     pm.params.as<GridParams>());
    const GridParams *dg = pm.params.as<GridParams>();
    k_first_tiles<<<ntiles, 1024, 0, st>>>(pm.first.as<int32_t>(), dg, pm.tiles.as<int32_t>());
    k_first_tile_mins<<<1, 1024, 0, st>>>(pm.tiles.as<int32_t>(), dg);
    k_first_apply<<<(unsigned) ((m + 255) / 256), 256, 0, st>>>(
        pm.first.as<int32_t>(), dg, pm.tiles.as<int32_t>(), (int32_t) n);
    pm.launches += 5;
    PRR_CUDA_TRY(cudaGetLastError());
    GridParams g;
    PRR_CUDA_TRY(cudaMemcpyAsync(&g, pm.params.ptr, sizeof(g), cudaMemcpyDeviceToHost, st));
    PRR_CUDA_TRY(cudaStreamSynchronize(st));
    pm.res = g.res;
    std::memcpy(pm.bmin, g.bmin, sizeof(pm.bmin));
    std::memcpy(pm.cs, g.cs, sizeof(pm.cs));
    pm.built = true;
    return PRR_OK;
}

int prr_photon_info(const prr_photon_map *pmap, int64_t *count, int32_t *grid_res) {
    if (!pmap)
        return fail(PRR_ERR_INVALID_ARGUMENT, "photon map is NULL");
    const PhotonMap &pm = *PM(pmap);
    if (count)
        *count = pm.n;
    if (grid_res)
        *grid_res = pm.res;
    return PRR_OK;
}

int prr_photon_launches(const prr_photon_map *pmap, int64_t *out) {
    if (!pmap || !out)
        return fail(PRR_ERR_INVALID_ARGUMENT, "photon map or out is NULL");
    *out = PM(pmap)->launches.load();
    return PRR_OK;
}

int prr_photon_export(const prr_photon_map *pmap, float *records, int32_t *owner, void *stream) {
    if (!pmap)
        return fail(PRR_ERR_INVALID_ARGUMENT, "photon map is NULL");
    const PhotonMap &pm = *PM(pmap);
    cudaStream_t st = (cudaStream_t) stream;
    if (pm.n > 0 && records)
        PRR_CUDA_TRY(cudaMemcpyAsync(records, pm.rec.ptr, (size_t) pm.n * 9 * sizeof(float),
                                     cudaMemcpyDefault, st));
    if (pm.n > 0 && owner)
        PRR_CUDA_TRY(cudaMemcpyAsync(owner, pm.owner.ptr, (size_t) pm.n * sizeof(int32_t),
                                     cudaMemcpyDefault, st));
    PRR_CUDA_TRY(cudaStreamSynchronize(st));
    return PRR_OK;
}

int prr_photon_gather(const prr_photon_map *pmap, const float *points, int64_t n, int k_nearest,
                      float *out_rgb, void *stream) {
    if (!pmap || n < 0 || (n > 0 && (!points || !out_rgb)) || k_nearest < 0 || k_nearest > kMaxK)
        return fail(PRR_ERR_INVALID_ARGUMENT, "bad gather arguments (k_nearest <= 64)");
    const PhotonMap &pm = *PM(pmap);
    if (!pm.built)
        return fail(PRR_ERR_NOT_BUILT, "photon map not built (call prr_photon_build)");
    cudaStream_t st = (cudaStream_t) stream;
    if (n == 0)
        return PRR_OK;
    if (pm.n == 0) {
        PRR_CUDA_TRY(cudaMemsetAsync(out_rgb, 0, (size_t) n * 3 * sizeof(float), st));
        return PRR_OK;
    }
    k_photon_gather<<<(unsigned) ((n + 127) / 128), 128, 0, st>>>(view(pm), points, n, k_nearest,
                                                                   out_rgb);
    pm.launches++;
    PRR_CUDA_TRY(cudaGetLastError());
    return PRR_OK;
}

int prr_render_caustics(const prr_scene *scene, const prr_photon_map *pmap,
                        const prr_render_settings *settings, int k_nearest, float *out_rgb,
                        void *stream) {
    return render_caustics(scene, pmap, settings, k_nearest, out_rgb, nullptr,
                           (cudaStream_t) stream);
}

int prr_render_caustics_counts(const prr_scene *scene, const prr_photon_map *pmap,
                               const prr_render_settings *settings, int k_nearest,
                               float *out_rgb, uint64_t out[5], void *stream) {
    if (!out)
        return fail(PRR_ERR_INVALID_ARGUMENT, "out is required");
    cudaStream_t st = (cudaStream_t) stream;
    DevBuf buf;
    PRR_CUDA_TRY(buf.alloc(5 * sizeof(unsigned long long)));
    PRR_CUDA_TRY(cudaMemsetAsync(buf.ptr, 0, 5 * sizeof(unsigned long long), st));
    if (int rc = render_caustics(scene, pmap, settings, k_nearest, out_rgb,
                                 buf.as<unsigned long long>(), st))
        return rc;
    PRR_CUDA_TRY(cudaMemcpyAsync(out, buf.ptr, 5 * sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
    PRR_CUDA_TRY(cudaStreamSynchronize(st));
    return PRR_OK;
}

} // extern "C"
