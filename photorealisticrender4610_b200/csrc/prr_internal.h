// Internal host-side state behind the C ABI (include/prr.h).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/prr.h"
#include "bvh_build.h"
#include "device_types.h"

namespace prr {

// ---- error reporting: every ABI call returns a status and leaves a message
void set_error(const std::string &msg);
int fail(int code, const std::string &msg);

// The library's stream-ordered memory pool of the current device (per-call
// scratch of the caustic render and of ray reordering): freed blocks stay in
// it for later calls. Created on first use, one per device.
cudaError_t library_pool(cudaMemPool_t *out);

// 64-bit traversal counters of a counting wavefront render (prr_render_counts)
constexpr int kWfStatSlots = 9;
// A failed allocation (cudaMalloc, a pool allocation) reports
// PRR_ERR_OUT_OF_MEMORY; every other CUDA error PRR_ERR_CUDA.
#define PRR_CUDA_TRY(expr)                                                                        \
    do {                                                                                         \
        cudaError_t e__ = (expr);                                                                \
        if (e__ != cudaSuccess)                                                                  \
            return ::prr::fail(e__ == cudaErrorMemoryAllocation ? PRR_ERR_OUT_OF_MEMORY           \
                                                                : PRR_ERR_CUDA,                   \
                               std::string(#expr) + ": " + cudaGetErrorString(e__));             \
    } while (0)

// Owning device allocation.
struct DevBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (ptr)
            cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
    }
    cudaError_t alloc(size_t n) {
        release();
        if (n == 0)
            return cudaSuccess;
        cudaError_t e = cudaMalloc(&ptr, n);
        if (e == cudaSuccess)
            bytes = n;
        return e;
    }
    cudaError_t ensure(size_t n) { return n <= bytes ? cudaSuccess : alloc(n); }
    template <class T> T *as() const { return (T *) ptr; }
};

struct HostMaterial {
    int kind;
    float params[9]; // baseColor[3], roughness, metallic, ior, emission[3]
    int tex[4] = {-1, -1, -1, -1}; // base colour, metallic-roughness, normal, emissive
};

struct HostTexture {
    int width = 0, height = 0, channels = 0;
    std::vector<uint8_t> texels;
};

struct HostObject {
    int kind;          // kObjMesh / kObjSphere
    int material;
    std::vector<float> verts; // mesh: n x 9 input triangles
    // mesh per-corner data (empty when absent): n x 9 normals, n x 6 uvs,
    // n x 12 tangents (xyz + handedness w per corner)
    std::vector<float> cnormals, cuvs, ctangents;
    float center[3] = {0, 0, 0};
    float radius = 0.f;
    // filled by build
    FlatBVH bvh;
    PrimBox bounds{};
    float area = 0.f;
    int tri_base = 0;
    uint32_t root = 0;
};

struct WavefrontPlan;

struct Scene {
    std::mutex mu;
    std::vector<HostMaterial> materials;
    std::vector<HostObject> objects;
    float background[3] = {0.235294f, 0.67451f, 0.843137f}; // Scene.hpp:17
    std::vector<float> env_rgb;
    int env_w = 0, env_h = 0;
    prr_camera camera{};
    int width = 0, height = 0;
    bool camera_set = false;

    bool built = false;
    FlatBVH tlas;
    DevScene dev{};   // device pointers + scalars, passed to kernels by value
    int64_t n_tris = 0;
    size_t device_bytes = 0;

    DevBuf d_nodes, d_tris, d_tri_e2z, d_tri_meta, d_verts, d_normals, d_objects, d_materials,
        d_emissives;
    std::vector<HostTexture> textures;
    DevBuf d_attr, d_texels, d_textures;
    DevBuf d_env_px, d_env_cdf, d_env_marginal, d_env_rowsin, d_env_guide;
    DevBuf d_scratch;      // staging for host-buffer entry points
    DevBuf d_render, d_render_spp; // per-slice partial sums / adaptive spp
    DevBuf d_counter;      // persistent-kernel work counters
    DevBuf d_check;        // status words of the checked build's device-side tests
    DevBuf d_wavefront;    // wavefront path state, queues and film
    std::shared_ptr<WavefrontPlan> wf_plan; // captured pass graph
    int64_t wf_paths = 0;  // paths in flight per pass (0 = automatic)
    int wf_block = 0;      // extend / shadow block size (0 = 128)
    int wf_refill = 0;     // idle lanes that trigger a refill (0 = 8)
    bool wf_graphs = true; // replay passes from a captured CUDA graph
    int wf_stack = 0;      // mesh-stack entries per thread in shared memory (0 = whole stack)
    bool wf_ordered = false; // queues rebuilt in path order by a stable partition
    DevBuf d_wf_spill;     // global part of the traversal stacks
    unsigned long long *wf_stats = nullptr; // set by prr_render_counts: count traversal work
    int64_t last_launches = 0; // kernels the last prr_render launched
    // Renders reuse the scratch above; each render waits for the previous
    // one's event before touching it, whatever stream either ran on.
    cudaEvent_t scratch_done = nullptr;
    // host-buffer pipeline of prr_mesh_intersect_host: streams and events
    // created on first use
    static constexpr int kHostBufs = 3;
    cudaStream_t host_streams[kHostBufs] = {};
    cudaEvent_t host_events[kHostBufs + 1] = {};
    ~Scene() {
        if (scratch_done)
            cudaEventDestroy(scratch_done);
        for (cudaEvent_t e : host_events)
            if (e)
                cudaEventDestroy(e);
        for (cudaStream_t h : host_streams)
            if (h)
                cudaStreamDestroy(h);
    }
};

// Kernel launchers (k_*.cu). All return a status; launch errors are checked.
int launch_mesh_closest(const Scene &s, int object, const float *o, const float *d, int64_t n,
                        int32_t *id, float *t, double *t64, unsigned *counter,
                        const prr_trace_config *cfg, cudaStream_t st);
int launch_mesh_occluded(const Scene &s, int object, const float *o, const float *d,
                         const float *tmax, int64_t n, uint8_t *hit, cudaStream_t st);
int launch_scene_closest(const Scene &s, const float *o, const float *d, int64_t n,
                         int32_t *obj, int32_t *prim, float *t, float *geo, cudaStream_t st);
int launch_scene_occluded(const Scene &s, const float *o, const float *d, const float *tmax,
                          int64_t n, uint8_t *hit, cudaStream_t st);
// Buckets of the env CDF guide tables (a power of two: k / kEnvGuide and
// u * kEnvGuide are exact in float).
constexpr int kEnvGuide = 256;
int launch_env_cdf(Scene &s, cudaStream_t st);
int render_plain(Scene &s, const prr_render_settings &rs, float *out_rgb, int32_t *out_spp,
                 unsigned long long *out_rays, cudaStream_t st);
int validate_render(const Scene &s, prr_render_settings &rs);
int render_wavefront(Scene &s, const prr_render_settings &rs, float *out_rgb, int32_t *out_spp,
                     unsigned long long *out_rays, cudaStream_t st);

// One request of a render-server step on the wavefront integrator: samples
// [s0, s0 + nspp) of every pixel of its window, summed into `film`.
struct WfStepReq {
    const DevScene *scene; // the scene's resident descriptor (device memory)
    DevCamera camera;      // the scene's camera at the request's resolution
    int x0, y0, ww, wh;    // pixel window
    int s0, nspp;
    int max_depth;
    float clamp;
    uint64_t seed;
    float3 *film; // ww*wh running sums (device)
};
// Buffers a server keeps across its wavefront steps: path state, stack
// spill, and the request table (device, and pinned host for the upload).
struct WfMultiState {
    DevBuf state, spill, reqs;
    void *h_table = nullptr;
    size_t h_cap = 0;
    WfMultiState() = default;
    WfMultiState(const WfMultiState &) = delete;
    WfMultiState &operator=(const WfMultiState &) = delete;
    ~WfMultiState() {
        if (h_table)
            cudaFreeHost(h_table);
    }
};
// Traces one step of n requests: consecutive requests of at most
// paths_per_launch paths share one set of ordered ray queues (a request
// alone may exceed it). Per request, rays_host[2k], rays_host[2k+1] receive
// the closest and shadow rays it traced (valid once the stream has drained);
// `launches` the kernel count. The step is ordered on `st`; the host does not
// wait for it.
int wavefront_step_multi(WfMultiState &ms, const WfStepReq *reqs, int n,
                         int64_t paths_per_launch, int tlas_cap, int blas_cap,
                         unsigned long long *rays_host, cudaStream_t st, int64_t *launches);

int device_sm_count();
DevCamera make_camera(const prr_camera &c, int width, int height);

} // namespace prr
