// Wavefront integrator (placeholder until the staged kernels land).
#include "prr_internal.h"

namespace prr {

int render_wavefront(Scene &, const prr_render_settings &, float *, int32_t *,
                     unsigned long long *, cudaStream_t) {
    return fail(PRR_ERR_UNSUPPORTED, "wavefront mode not available in this build");
}

} // namespace prr
