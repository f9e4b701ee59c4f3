// Test infrastructure only: exercises include/prr_bridge.hpp on scenes built
// with the reference renderer's own classes (by harness.cpp), so a test can
// check that the bridge hands libprr the same scene the reference built.
// Compiled into _ref/libprr_ref_bridge.so together with the reference sources
// and the harness, and linked against libprr.so.
#include "Material.hpp"
#include "Renderer.hpp"
#include "Scene.hpp"
#include "Sphere.hpp"
#include "Triangle.hpp"

#include "prr_bridge.hpp"

extern "C" void *prr_ref_scene_object(void *h, int *width, int *height);

extern "C" int prr_ref_bridge_render(void *h, int max_depth, int min_spp, int max_spp,
                                     float threshold, uint64_t seed, int mode, int mapper,
                                     float exposure, float *out_rgb, int32_t *out_spp,
                                     uint8_t *out_u8, int64_t *report8) {
    int w = 0, hh = 0;
    const Scene &scene = *(const Scene *) prr_ref_scene_object(h, &w, &hh);
    RenderSettings s;
    s.width = w;
    s.height = hh;
    s.minSPP = min_spp;
    s.maxSPP = max_spp;
    s.maxDepth = max_depth;
    s.varianceThreshold = threshold;
    s.exposure = exposure;
    s.toneMapper = (tonemap::ToneMapper) mapper;
    prr_bridge::Report rep;
    try {
        prr_bridge::Output out = prr_bridge::render(scene, s, max_depth, seed, mode, 10.0f, &rep);
        std::copy(out.linear.begin(), out.linear.end(), out_rgb);
        std::copy(out.spp.begin(), out.spp.end(), out_spp);
        std::copy(out.rgb8.begin(), out.rgb8.end(), out_u8);
    } catch (const std::exception &e) {
        std::fprintf(stderr, "prr_ref_bridge_render: %s\n", e.what());
        return -1;
    }
    const int64_t r[8] = {rep.meshes,   rep.spheres,           rep.triangles,
                          rep.materials, rep.textures,          rep.attributed_meshes,
                          rep.skipped_objects, rep.dropped};
    std::copy(r, r + 8, report8);
    return 0;
}
