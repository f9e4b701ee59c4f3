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
//   Triangle::n0..n2, t0..t2, tan0..tan2, tangentW*, hasSmoothNormals,
//   hasTangents                                        Triangle.hpp:17-23
//   Material::baseColorTex, metallicRoughnessTex, normalTex, emissiveTex
//                                                      Material.hpp:45-48
//
// Not carried over (Report counts them so a caller can refuse the scene): any
// Object subclass other than MeshTriangle and Sphere, per-corner data on a
// mesh where only some triangles have it, and texture data that is not
// width x height x channels bytes.
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
    int64_t textures = 0;          // textures carried over
    int64_t attributed_meshes = 0; // meshes carried with per-corner data
    int64_t skipped_objects = 0;   // Object subclasses libprr does not know
    int64_t dropped = 0;           // per-corner data or textures left out (see above)
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
        int id = -1;
        check(prr_scene_add_material(h, material_kind(m), p, &id));
        const Texture *tex[4] = {&m->baseColorTex, &m->metallicRoughnessTex, &m->normalTex,
                                 &m->emissiveTex};
        int tid[4] = {-1, -1, -1, -1};
        for (int k = 0; k < 4; k++) {
            const Texture &t = *tex[k];
            if (t.empty())
                continue;
            if ((t.channels != 3 && t.channels != 4) ||
                t.data.size() != (size_t) t.width * t.height * t.channels) {
                rep.dropped++;
                continue;
            }
            check(prr_scene_add_texture(h, t.data.data(), t.width, t.height, t.channels, &tid[k]));
            rep.textures++;
        }
        if (tid[0] >= 0 || tid[1] >= 0 || tid[2] >= 0 || tid[3] >= 0)
            check(prr_scene_set_material_textures(h, id, tid[0], tid[1], tid[2], tid[3]));
        ids.emplace(m, id);
        rep.materials++;
        return id;
    };
    std::vector<float> verts, nrm, uvs, tan;
    for (const Object *o : scene.objects) {
        int obj = -1;
        if (auto *mesh = dynamic_cast<const MeshTriangle *>(o)) {
            const size_t n = mesh->triangles.size();
            size_t with_n = 0, with_t = 0;
            bool any_uv = false;
            verts.resize(n * 9);
            nrm.resize(n * 9);
            uvs.resize(n * 6);
            tan.resize(n * 12);
            for (size_t i = 0; i < n; i++) {
                const Triangle &t = mesh->triangles[i];
                put3(&verts[i * 9], t.v0);
                put3(&verts[i * 9 + 3], t.v1);
                put3(&verts[i * 9 + 6], t.v2);
                put3(&nrm[i * 9], t.n0);
                put3(&nrm[i * 9 + 3], t.n1);
                put3(&nrm[i * 9 + 6], t.n2);
                const Vector2f *uv[3] = {&t.t0, &t.t1, &t.t2};
                const Vector3f *tg[3] = {&t.tan0, &t.tan1, &t.tan2};
                const float tw[3] = {t.tangentW0, t.tangentW1, t.tangentW2};
                for (int q = 0; q < 3; q++) {
                    uvs[i * 6 + q * 2] = uv[q]->x;
                    uvs[i * 6 + q * 2 + 1] = uv[q]->y;
                    any_uv = any_uv || uv[q]->x != 0.f || uv[q]->y != 0.f;
                    put3(&tan[i * 12 + q * 4], *tg[q]);
                    tan[i * 12 + q * 4 + 3] = tw[q];
                }
                with_n += t.hasSmoothNormals ? 1 : 0;
                with_t += t.hasTangents ? 1 : 0;
            }
            const bool use_n = with_n == n && n > 0, use_t = with_t == n && n > 0;
            if ((with_n && !use_n) || (with_t && !use_t))
                rep.dropped++;
            if (use_n || use_t || any_uv) {
                check(prr_scene_add_mesh_attr(h, verts.data(), use_n ? nrm.data() : nullptr,
                                              any_uv ? uvs.data() : nullptr,
                                              use_t ? tan.data() : nullptr, (int64_t) n,
                                              material(mesh->m), &obj));
                rep.attributed_meshes++;
            } else {
                check(prr_scene_add_mesh(h, verts.data(), (int64_t) n, material(mesh->m), &obj));
            }
            rep.meshes++;
            rep.triangles += (int64_t) n;
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
