// C ABI of the renderer (Renderer::Render, Renderer.cpp:24-212, up to the
// linear framebuffer) and its argument checks.
#include "prr_internal.h"

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
