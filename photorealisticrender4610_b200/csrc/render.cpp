// C ABI of the renderer (Renderer::Render, Renderer.cpp:24-212, up to the
// linear framebuffer), its argument checks, and the wavefront autotuner.
#include "prr_internal.h"

#include <algorithm>

namespace prr {

int validate_render(const Scene &s, prr_render_settings &rs) {
    if (!s.camera_set)
        return fail(PRR_ERR_INVALID_ARGUMENT, "scene has no camera");
    if (rs.width != s.width || rs.height != s.height)
        return fail(PRR_ERR_INVALID_ARGUMENT, "settings size differs from the camera's");
    if (rs.x1 <= 0 || rs.y1 <= 0) {
        rs.x0 = rs.y0 = 0;
        rs.x1 = rs.width;
        rs.y1 = rs.height;
    }
    if (rs.x0 < 0 || rs.y0 < 0 || rs.x1 > rs.width || rs.y1 > rs.height || rs.x0 >= rs.x1 ||
        rs.y0 >= rs.y1)
        return fail(PRR_ERR_INVALID_ARGUMENT, "bad pixel window");
    if (rs.max_spp < 1 || rs.min_spp < 1 || rs.min_spp > rs.max_spp)
        return fail(PRR_ERR_INVALID_ARGUMENT, "need 1 <= min_spp <= max_spp");
    if (rs.max_depth < 1 || rs.max_depth > 1024)
        return fail(PRR_ERR_INVALID_ARGUMENT, "max_depth out of range");
    if (rs.sample_offset < 0)
        return fail(PRR_ERR_INVALID_ARGUMENT, "negative sample offset");
    if ((int64_t) rs.width * rs.height > (int64_t) 1 << 31)
        return fail(PRR_ERR_INVALID_ARGUMENT, "image too large");
    if (rs.mode != PRR_RENDER_PLAIN && rs.mode != PRR_RENDER_WAVEFRONT)
        return fail(PRR_ERR_INVALID_ARGUMENT, "unknown render mode");
    return PRR_OK;
}

} // namespace prr

using namespace prr;

extern "C" int prr_render(prr_scene *scene, const prr_render_settings *settings, float *out_rgb,
                          int32_t *out_spp, uint64_t *out_rays, void *stream) {
    if (!scene || !settings || !out_rgb)
        return fail(PRR_ERR_INVALID_ARGUMENT, "scene, settings and out_rgb are required");
    Scene &s = *reinterpret_cast<Scene *>(scene);
    if (!s.built)
        return fail(PRR_ERR_NOT_BUILT, "scene not built (call prr_scene_build)");
    prr_render_settings rs = *settings;
    if (int rc = validate_render(s, rs))
        return rc;
    std::lock_guard<std::mutex> g(s.mu);
    cudaStream_t st = (cudaStream_t) stream;
    if (!s.scratch_done)
        PRR_CUDA_TRY(cudaEventCreateWithFlags(&s.scratch_done, cudaEventDisableTiming));
    else
        PRR_CUDA_TRY(cudaStreamWaitEvent(st, s.scratch_done, 0));
    int rc;
    if (rs.mode == PRR_RENDER_WAVEFRONT)
        rc = render_wavefront(s, rs, out_rgb, out_spp, (unsigned long long *) out_rays, st);
    else
        rc = render_plain(s, rs, out_rgb, out_spp, (unsigned long long *) out_rays, st);
    PRR_CUDA_TRY(cudaEventRecord(s.scratch_done, st));
    return rc;
}

extern "C" int prr_render_counts(prr_scene *scene, const prr_render_settings *settings,
                                 float *out_rgb, prr_render_count *out, void *stream) {
    if (!scene || !settings || !out_rgb || !out)
        return fail(PRR_ERR_INVALID_ARGUMENT, "scene, settings, out_rgb and out are required");
    Scene &s = *reinterpret_cast<Scene *>(scene);
    if (!s.built)
        return fail(PRR_ERR_NOT_BUILT, "scene not built (call prr_scene_build)");
    prr_render_settings rs = *settings;
    rs.mode = PRR_RENDER_WAVEFRONT;
    if (int rc = validate_render(s, rs))
        return rc;
    std::lock_guard<std::mutex> g(s.mu);
    cudaStream_t st = (cudaStream_t) stream;
    if (!s.scratch_done)
        PRR_CUDA_TRY(cudaEventCreateWithFlags(&s.scratch_done, cudaEventDisableTiming));
    else
        PRR_CUDA_TRY(cudaStreamWaitEvent(st, s.scratch_done, 0));
    DevBuf buf;
    PRR_CUDA_TRY(buf.alloc((kWfStatSlots + 2) * sizeof(unsigned long long)));
    PRR_CUDA_TRY(cudaMemsetAsync(buf.ptr, 0, (kWfStatSlots + 2) * sizeof(unsigned long long), st));
    unsigned long long *stats = buf.as<unsigned long long>();
    s.wf_stats = stats;
    const int rc = render_wavefront(s, rs, out_rgb, nullptr, stats + kWfStatSlots, st);
    s.wf_stats = nullptr;
    PRR_CUDA_TRY(cudaEventRecord(s.scratch_done, st));
    if (rc)
        return rc;
    unsigned long long h[kWfStatSlots + 2];
    PRR_CUDA_TRY(cudaMemcpyAsync(h, stats, sizeof(h), cudaMemcpyDeviceToHost, st));
    PRR_CUDA_TRY(cudaStreamSynchronize(st));
    out->closest_rays = h[kWfStatSlots];
    out->closest_nodes = h[0];
    out->closest_tris = h[1];
    out->closest_objects = h[2];
    out->shadow_rays = h[kWfStatSlots + 1];
    out->shadow_nodes = h[3];
    out->shadow_tris = h[4];
    out->shadow_objects = h[5];
    out->misses = h[6];
    out->delta_hits = h[7];
    out->surface_hits = h[8];
    return PRR_OK;
}

extern "C" int prr_scene_set_wavefront(prr_scene *scene, const prr_wavefront_config *config) {
    if (!scene || !config)
        return fail(PRR_ERR_INVALID_ARGUMENT, "scene and config are required");
    if (config->paths_per_pass < 0 || config->paths_per_pass > (int64_t(1) << 30) ||
        config->block_size < 0 || config->block_size % 32 != 0 || config->block_size > 512 ||
        config->stack_smem < 0 || config->refill < 0 || config->refill > 32)
        return fail(PRR_ERR_INVALID_ARGUMENT,
                    "bad wavefront config (paths_per_pass <= 2^30, block_size a multiple of "
                    "32 up to 512, stack_smem >= 0, refill 0..32)");
    Scene &s = *reinterpret_cast<Scene *>(scene);
    std::lock_guard<std::mutex> g(s.mu);
    s.wf_paths = config->paths_per_pass;
    s.wf_block = config->block_size;
    s.wf_graphs = config->use_graphs != 0;
    s.wf_stack = config->stack_smem;
    s.wf_ordered = config->ordered != 0;
    s.wf_refill = config->refill;
    return PRR_OK;
}

extern "C" int prr_autotune(prr_scene *scene, const prr_render_settings *settings,
                            prr_wavefront_config *out_best, void *stream) {
    if (!scene || !settings)
        return fail(PRR_ERR_INVALID_ARGUMENT, "scene and settings are required");
    Scene &s = *reinterpret_cast<Scene *>(scene);
    if (!s.built)
        return fail(PRR_ERR_NOT_BUILT, "scene not built (call prr_scene_build)");
    prr_render_settings rs = *settings;
    rs.mode = PRR_RENDER_WAVEFRONT;
    rs.min_spp = rs.max_spp;
    if (int rc = validate_render(s, rs))
        return rc;
    cudaStream_t st = (cudaStream_t) stream;
    const int64_t npix = (int64_t) (rs.x1 - rs.x0) * (rs.y1 - rs.y0);
    DevBuf out;
    PRR_CUDA_TRY(out.alloc((size_t) npix * 3 * sizeof(float)));
    cudaEvent_t a, b;
    PRR_CUDA_TRY(cudaEventCreate(&a));
    PRR_CUDA_TRY(cudaEventCreate(&b));
    const int64_t paths[] = {int64_t(1) << 20, int64_t(1) << 21, int64_t(1) << 22,
                             int64_t(1) << 23, int64_t(1) << 24, int64_t(1) << 25,
                             int64_t(1) << 26};
    const int blocks[] = {64, 128, 256};
    float best_ms = 1e30f;
    prr_wavefront_config best{0, 0, 1, 0, 1, 0};
    int rc = PRR_OK;
    std::lock_guard<std::mutex> g(s.mu);
    auto trial = [&](const prr_wavefront_config &c) {
        s.wf_paths = c.paths_per_pass;
        s.wf_block = c.block_size;
        s.wf_graphs = true;
        s.wf_stack = c.stack_smem;
        s.wf_ordered = c.ordered != 0;
        s.wf_refill = c.refill;
        float ms_min = 1e30f;
        for (int rep = 0; rep < 2 && rc == PRR_OK; rep++) {
            cudaEventRecord(a, st);
            rc = render_wavefront(s, rs, out.as<float>(), nullptr, nullptr, st);
            cudaEventRecord(b, st);
            if (cudaEventSynchronize(b) != cudaSuccess && rc == PRR_OK)
                rc = fail(PRR_ERR_CUDA, "autotune render failed");
            float ms = 0.f;
            cudaEventElapsedTime(&ms, a, b);
            if (rep > 0) // the first run captures the graph
                ms_min = std::min(ms_min, ms);
        }
        if (rc == PRR_OK && ms_min < best_ms) {
            best_ms = ms_min;
            best = c;
        }
    };
    // stage 1: paths per pass x block size, ordered queues, 8 shared stack
    // entries (the rest of the L1 caches nodes and triangles)
    const int stack1 = std::min(8, s.dev.blas_depth + 1);
    int64_t last = -1;
    for (int64_t cand : paths) {
        // a pass never holds more than the whole render
        const int64_t pp = std::min<int64_t>(cand, npix * rs.max_spp);
        if (pp == last)
            continue;
        last = pp;
        for (int bl : blocks)
            if (rc == PRR_OK)
                trial(prr_wavefront_config{pp, bl, 1, stack1, 1, 0});
    }
    // stage 2: at that shape, other shared stack depths (0: the whole stack)
    const prr_wavefront_config shape = best;
    for (int sk : {0, 16, 4, 2})
        if (rc == PRR_OK && sk < s.dev.blas_depth + 1 && sk != stack1)
            trial(prr_wavefront_config{shape.paths_per_pass, shape.block_size, 1, sk, 1, 0});
    // stage 3: append-order queues
    const prr_wavefront_config shape2 = best;
    if (rc == PRR_OK)
        trial(prr_wavefront_config{shape2.paths_per_pass, shape2.block_size, 1,
                                   shape2.stack_smem, 0, 0});
    // stage 4: the refill threshold of the traversal stages
    const prr_wavefront_config shape3 = best;
    for (int rf : {4, 12, 16})
        if (rc == PRR_OK)
            trial(prr_wavefront_config{shape3.paths_per_pass, shape3.block_size, 1,
                                       shape3.stack_smem, shape3.ordered, rf});
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (rc)
        return rc;
    s.wf_paths = best.paths_per_pass;
    s.wf_block = best.block_size;
    s.wf_graphs = true;
    s.wf_stack = best.stack_smem;
    s.wf_ordered = best.ordered != 0;
    s.wf_refill = best.refill;
    if (out_best)
        *out_best = best;
    return PRR_OK;
}
