// prr_bridge.hpp -- hands a scene built with the reference renderer's OWN
// classes (its GLTF loader, MeshTriangle, Sphere, the four materials, EnvMap,
// Camera) to libprr and renders it on the GPU. This is the integration for a
// program that keeps the reference's scene setup and replaces only
// Renderer::Render (Renderer.cpp:24-212): include this header after the
// reference's Renderer.hpp and call prr_bridge::render instead of
// Renderer::Render.
//
// What is read from the reference objects (reference file:line):
//   Scene::objects, backgroundColor, envMap, camera   Scene.hpp:17-22
//   MeshTriangle::triangles (v0, v1, v2), m            Triangle.hpp:15, :166-170
//   Sphere::center, radius, m                          Sphere.hpp:15-17
//   Material::baseColor, roughness, metallic, ior, m_emission, and the
//   concrete class (Diffuse / Emissive / Mirror / Glass)
//                                                      Material.hpp:38-183
//   EnvMap::pixels, width, height, loaded               EnvMap.hpp:19-27
//   Camera::eye, target, up, fovv, fovh, aperture, focusDistance
//                                                      Camera.hpp:9-15
//   RenderSettings                                     Renderer.hpp:42-55
//
// Not carried over (Report counts them so a caller can refuse the scene):
// textures (Material::*Tex), per-vertex smooth normals and tangents, and any
// Object subclass other than MeshTriangle and Sphere.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "prr.h"

namespace prr_bridge {

inline void check(int rc) {
    if (rc < 0) {
        char buf[512];
        prr_last_error(buf, sizeof(buf));
        throw std::runtime_error(std::string("libprr: ") + buf);
    }
}

struct Report {
    int64_t meshes = 0, spheres = 0, triangles = 0, materials = 0;
    int64_t textured_materials = 0;      // textures are not sampled by libprr
    int64_t smooth_normal_triangles = 0; // shaded with the face normal instead
    int64_t skipped_objects = 0;         // Object subclasses libprr does not know
};

// Owns the libprr scene built from a reference Scene.
class GpuScene {
  public:
    GpuScene() { check(prr_scene_create(&h_)); }
    ~GpuScene() { if (h_) prr_scene_destroy(h_); }
    GpuScene(const GpuScene &) = delete;
    GpuScene &operator=(const GpuScene &) = delete;
    GpuScene(GpuScene &&o) noexcept : h_(o.h_) { o.h_ = nullptr; }
    prr_scene *get() const { return h_; }

  private:
    prr_scene *h_ = nullptr;
};

inline int material_kind(const Material *m) {
    if (dynamic_cast<const EmissiveMaterial *>(m)) return PRR_MAT_EMISSIVE;
    if (dynamic_cast<const MirrorMaterial *>(m)) return PRR_MAT_MIRROR;
    if (dynamic_cast<const GlassMaterial *>(m)) return PRR_MAT_GLASS;
    return PRR_MAT_DIFFUSE;
}

inline void put3(float *dst, const Vector3f &v) {
    dst[0] = v.x;
    dst[1] = v.y;
    dst[2] = v.z;
}

// Scene::Add order is kept, so object k here is objects[k] there (the scene
// BVH and the emitter list depend on it).
inline GpuScene upload(const Scene &scene, int width, int height, Report *report = nullptr) {
    Report rep;
    GpuScene gs;
    prr_scene *h = gs.get();
    std::unordered_map<const Material *, int> ids;
    auto material = [&](const Material *m) {
        auto it = ids.find(m);
        if (it != ids.end()) return it->second;
        float p[9];
        put3(p, m->baseColor);
        p[3] = m->roughness;
        p[4] = m->metallic;
        p[5] = m->ior;
        put3(p + 6, m->m_emission);
        if (!m->baseColorTex.empty() || !m->emissiveTex.empty() || !m->normalTex.empty() ||
            !m->metallicRoughnessTex.empty())
            rep.textured_materials++;
        int id = -1;
        check(prr_scene_add_material(h, material_kind(m), p, &id));
        ids.emplace(m, id);
        rep.materials++;
        return id;
    };
    std::vector<float> verts;
    for (const Object *o : scene.objects) {
        int obj = -1;
        if (auto *mesh = dynamic_cast<const MeshTriangle *>(o)) {
            verts.resize(mesh->triangles.size() * 9);
            float *v = verts.data();
            for (const Triangle &t : mesh->triangles) {
                put3(v, t.v0);
                put3(v + 3, t.v1);
                put3(v + 6, t.v2);
                v += 9;
                if (t.hasSmoothNormals) rep.smooth_normal_triangles++;
            }
            check(prr_scene_add_mesh(h, verts.data(), (int64_t) mesh->triangles.size(),
                                     material(mesh->m), &obj));
            rep.meshes++;
            rep.triangles += (int64_t) mesh->triangles.size();
        } else if (auto *sph = dynamic_cast<const Sphere *>(o)) {
            float c[3];
            put3(c, sph->center);
            check(prr_scene_add_sphere(h, c, sph->radius, material(sph->m), &obj));
            rep.spheres++;
        } else {
            rep.skipped_objects++;
        }
    }
    float bg[3];
    put3(bg, scene.backgroundColor);
    check(prr_scene_set_background(h, bg));
    if (scene.envMap.loaded) {
        const EnvMap &env = scene.envMap;
        std::vector<float> px((size_t) env.width * env.height * 3);
        for (size_t i = 0; i < (size_t) env.width * env.height; ++i)
            put3(&px[i * 3], env.pixels[i]);
        check(prr_scene_set_env(h, px.data(), env.width, env.height));
    }
    const Camera &cam = scene.camera;
    prr_camera pc{};
    put3(pc.eye, cam.eye);
    put3(pc.target, cam.target);
    put3(pc.up, cam.up);
    pc.fovv = cam.fovv;
    pc.fovh = cam.fovh;
    pc.aperture = cam.aperture;
    pc.focus_distance = cam.focusDistance;
    check(prr_scene_set_camera(h, &pc, width, height));
    check(prr_scene_build(h, nullptr));
    if (report) *report = rep;
    return gs;
}

struct Output {
    std::vector<float> linear;       // width x height x 3, the reference's framebuffer
    std::vector<int32_t> spp;        // samples taken per pixel
    std::vector<unsigned char> rgb8; // tone-mapped 8-bit image (Renderer.cpp:149-171)
};

// Renderer::Render on the GPU: the sample loop of Renderer.cpp:63-110 (fixed
// or adaptive spp), the path loop of Integrator::castRay, and the display
// transform. max_depth is the value given to the Integrator's constructor.
// Pixel m = i + j*W, sample n draws random stream (seed, m, n).
inline Output render(const Scene &scene, const RenderSettings &s, int max_depth,
                     uint64_t seed = 1, int mode = PRR_RENDER_WAVEFRONT,
                     float indirect_clamp = 10.0f, Report *report = nullptr) {
    GpuScene gs = upload(scene, s.width, s.height, report);
    prr_render_settings rs{};
    rs.width = s.width;
    rs.height = s.height;
    rs.min_spp = s.minSPP;
    rs.max_spp = s.maxSPP;
    rs.max_depth = max_depth;
    rs.variance_threshold = s.varianceThreshold;
    rs.indirect_clamp = indirect_clamp;
    rs.mode = mode;
    rs.seed = seed;
    const size_t n = (size_t) s.width * s.height;
    float *d_rgb = nullptr;
    int32_t *d_spp = nullptr;
    uint8_t *d_u8 = nullptr;
    auto release = [&] {
        cudaFree(d_rgb);
        cudaFree(d_spp);
        cudaFree(d_u8);
    };
    if (cudaMalloc(&d_rgb, n * 12) != cudaSuccess || cudaMalloc(&d_spp, n * 4) != cudaSuccess ||
        cudaMalloc(&d_u8, n * 3) != cudaSuccess) {
        release();
        throw std::runtime_error("prr_bridge: cudaMalloc failed");
    }
    Output out;
    try {
        check(prr_render(gs.get(), &rs, d_rgb, d_spp, nullptr, nullptr));
        check(prr_tonemap((int) s.toneMapper, s.exposure, d_rgb, (int64_t) n, nullptr, d_u8,
                          nullptr));
        out.linear.resize(n * 3);
        out.spp.resize(n);
        out.rgb8.resize(n * 3);
        if (cudaMemcpy(out.linear.data(), d_rgb, n * 12, cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemcpy(out.spp.data(), d_spp, n * 4, cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemcpy(out.rgb8.data(), d_u8, n * 3, cudaMemcpyDeviceToHost) != cudaSuccess)
            throw std::runtime_error("prr_bridge: cudaMemcpy failed");
    } catch (...) {
        release();
        throw;
    }
    release();
    return out;
}

} // namespace prr_bridge
