// prr_dropin.hpp -- C++ classes with the reference renderer's names and
// method signatures, forwarding to libprr's C ABI (prr.h). A program written
// against the reference's Scene / MeshTriangle / Sphere / Material / Camera /
// Integrator / Renderer / tonemap switches by including this header instead
// of the reference headers and linking libprr.so.
//
// Mirrored interfaces (reference file:line):
//   Vector3f, Vector2f            Vector.hpp:12-97 (arithmetic subset)
//   Ray(origin, direction)        Ray.hpp:8-28
//   Material + Diffuse/Emissive/Mirror/GlassMaterial (public fields)
//                                 Material.hpp:38-183
//   Triangle(v0, v1, v2, m)       Triangle.hpp:27-32
//   MeshTriangle(tris, bounds, m) Triangle.hpp:116-124
//   MeshTriangle(filename, offset, m) (OBJ)
//                                 Triangle.cpp:4-32
//   Sphere(center, radius, m)     Sphere.hpp:14-16
//   Texture; Triangle's per-corner data; Material textures
//                                 TextureUtils.hpp:9-18, Triangle.hpp:17-23,
//                                 Material.hpp:45-48
//   GLTFLoader::load(file, MaterialType, override)
//                                 GLTFLoader.hpp:10-26
//   Camera::create / fromBlender / init
//                                 Camera.hpp:23-56
//   Scene::Add / buildBVH / intersect / intersectP, envMap, camera,
//   backgroundColor, medium       Scene.hpp:15-41
//   Medium (dust, fog, active, intersect)
//                                 Volume.hpp:7-63
//   Integrator(scene, maxDepth, rr), castRay
//                                 Integrator.hpp:15-23
//   RenderSettings, Renderer::Render
//                                 Renderer.hpp:42-59
//   tonemap::ToneMapper / apply   ToneMapping.hpp:32-37, :267-279
//
// The per-ray calls (Scene::intersect, Integrator::castRay) run a one-ray
// batch and exist for compatibility; the batch entry points of prr.h are the
// hot path. Renderer::Render renders on the GPU, keeps the linear framebuffer
// (framebuffer()), and writes output, output_raw and sample_count as .png and
// .ppm like the reference (Renderer.cpp:163-211).
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

#include "prr.h"

namespace prr_detail {
inline void check(int rc) {
    if (rc < 0) {
        char buf[512];
        prr_last_error(buf, sizeof(buf));
        throw std::runtime_error(std::string("libprr: ") + buf);
    }
}
template <class T> struct DeviceArray {
    T *p = nullptr;
    size_t n = 0;
    explicit DeviceArray(size_t count) : n(count) {
        if (cudaMalloc(&p, sizeof(T) * (count ? count : 1)) != cudaSuccess)
            throw std::runtime_error("cudaMalloc failed");
    }
    ~DeviceArray() { cudaFree(p); }
    void put(const T *h) { cudaMemcpy(p, h, sizeof(T) * n, cudaMemcpyHostToDevice); }
    void get(T *h) const { cudaMemcpy(h, p, sizeof(T) * n, cudaMemcpyDeviceToHost); }
};
} // namespace prr_detail

struct Vector3f {
    float x = 0, y = 0, z = 0;
    Vector3f() = default;
    Vector3f(float v) : x(v), y(v), z(v) {}
    Vector3f(float a, float b, float c) : x(a), y(b), z(c) {}
    Vector3f operator+(const Vector3f &v) const { return {x + v.x, y + v.y, z + v.z}; }
    Vector3f operator-(const Vector3f &v) const { return {x - v.x, y - v.y, z - v.z}; }
    Vector3f operator*(const Vector3f &v) const { return {x * v.x, y * v.y, z * v.z}; }
    Vector3f operator*(float r) const { return {x * r, y * r, z * r}; }
    Vector3f operator/(float r) const { return {x / r, y / r, z / r}; }
    Vector3f operator-() const { return {-x, -y, -z}; }
    float norm() const { return std::sqrt(x * x + y * y + z * z); }
};
inline Vector3f operator*(float r, const Vector3f &v) { return {v.x * r, v.y * r, v.z * r}; }

struct Vector2f {
    float x = 0, y = 0;
    Vector2f() = default;
    Vector2f(float a, float b) : x(a), y(b) {}
};

struct Ray {
    Vector3f origin, direction;
    Ray(const Vector3f &o, const Vector3f &d) : origin(o), direction(d) {}
};

struct Bounds3 {
    Vector3f pMin, pMax;
    Bounds3() = default;
    Bounds3(const Vector3f &a, const Vector3f &b) : pMin(a), pMax(b) {}
};

// Texture (TextureUtils.hpp:9-18): 8-bit texels, row-major.
struct Texture {
    std::vector<unsigned char> data;
    int width = 0;
    int height = 0;
    int channels = 4;
    bool empty() const { return data.empty(); }
};

class Material {
  public:
    Vector3f m_emission = Vector3f(0.0f);
    Vector3f baseColor = Vector3f(0.8f, 0.8f, 0.8f);
    float roughness = 0.5f;
    float metallic = 0.0f;
    float ior = 1.5f;
    Texture emissiveTex;
    Texture baseColorTex;
    Texture normalTex;
    Texture metallicRoughnessTex;
    virtual ~Material() = default;
    virtual int kind() const = 0;
    virtual bool isDelta() const { return false; }
    virtual bool isEmissive() const { return false; }
};
class DiffuseMaterial : public Material {
  public:
    int kind() const override { return PRR_MAT_DIFFUSE; }
};
class EmissiveMaterial : public Material {
  public:
    int kind() const override { return PRR_MAT_EMISSIVE; }
    bool isEmissive() const override { return true; }
};
class MirrorMaterial : public Material {
  public:
    int kind() const override { return PRR_MAT_MIRROR; }
    bool isDelta() const override { return true; }
};
class GlassMaterial : public Material {
  public:
    int kind() const override { return PRR_MAT_GLASS; }
    bool isDelta() const override { return true; }
};

class Object {
  public:
    virtual ~Object() = default;
    Material *m = nullptr;
};

class Triangle {
  public:
    Vector3f v0, v1, v2;
    Vector2f t0, t1, t2;       // per-corner texture coordinates
    Vector3f tan0, tan1, tan2; // per-corner tangents
    float tangentW0 = 1.f, tangentW1 = 1.f, tangentW2 = 1.f;
    bool hasTangents = false;
    Vector3f n0, n1, n2; // per-corner smooth normals
    bool hasSmoothNormals = false;
    Material *m;
    Triangle(Vector3f a, Vector3f b, Vector3f c, Material *mat = nullptr)
        : v0(a), v1(b), v2(c), m(mat) {}
};

class MeshTriangle : public Object {
  public:
    std::vector<Triangle> triangles;
    Bounds3 bounding_box;
    MeshTriangle(std::vector<Triangle> tris, Bounds3 bounds, Material *mt)
        : triangles(std::move(tris)), bounding_box(bounds) {
        m = mt;
    }
    // MeshTriangle(filename, offset, m) (Triangle.cpp:4-32): the OBJ file's
    // one mesh as the reference's bundled loader reads it, shifted by offset.
    MeshTriangle(const std::string &filename, Vector3f offset, Material *mt);
};

class Sphere : public Object {
  public:
    Vector3f center;
    float radius;
    Sphere(const Vector3f &c, const float &r, Material *mt) : center(c), radius(r) { m = mt; }
};

inline MeshTriangle::MeshTriangle(const std::string &filename, Vector3f offset, Material *mt) {
    m = mt;
    const float off[3] = {offset.x, offset.y, offset.z};
    int64_t nt = 0;
    prr_detail::check(prr_obj_read(filename.c_str(), off, nullptr, 0, &nt));
    std::vector<float> v((size_t) nt * 9);
    prr_detail::check(prr_obj_read(filename.c_str(), off, v.data(), nt, &nt));
    const float inf = std::numeric_limits<float>::infinity();
    Vector3f lo(inf, inf, inf), hi(-inf, -inf, -inf);
    triangles.reserve((size_t) nt);
    for (int64_t i = 0; i < nt; i++) {
        Vector3f c[3];
        for (int j = 0; j < 3; j++) {
            c[j] = Vector3f(v[i * 9 + j * 3], v[i * 9 + j * 3 + 1], v[i * 9 + j * 3 + 2]);
            lo = Vector3f(std::min(lo.x, c[j].x), std::min(lo.y, c[j].y), std::min(lo.z, c[j].z));
            hi = Vector3f(std::max(hi.x, c[j].x), std::max(hi.y, c[j].y), std::max(hi.z, c[j].z));
        }
        triangles.emplace_back(c[0], c[1], c[2], mt);
    }
    bounding_box = Bounds3(lo, hi);
}

enum class MaterialType { Diffuse, Glass, Mirror, Emit }; // GLTFLoader.hpp:10

// GLTFLoader::load (GLTFLoader.cpp:140-281): one heap-allocated MeshTriangle
// per triangle primitive, with its per-corner data and a new material per
// primitive (or overrideMat for all). Parsed by libprr's glTF reader.
class GLTFLoader {
  public:
    static std::vector<MeshTriangle *> load(const std::string &filename, MaterialType matType,
                                            Material *overrideMat = nullptr) {
        prr_scene *tmp = nullptr;
        prr_detail::check(prr_scene_create(&tmp));
        std::vector<MeshTriangle *> out;
        try {
            int first = -1, count = 0, undecoded = 0;
            int over = -1;
            if (overrideMat) {
                const float p[9] = {0.8f, 0.8f, 0.8f, 0.5f, 0.f, 1.5f, 0.f, 0.f, 0.f};
                prr_detail::check(prr_scene_add_material(tmp, PRR_MAT_DIFFUSE, p, &over));
            }
            prr_detail::check(prr_scene_add_gltf(tmp, filename.c_str(), (int) matType, over,
                                                 &first, &count, &undecoded));
            for (int k = 0; k < count; k++) {
                const int obj = first + k;
                int64_t nt = 0;
                int attr = 0;
                prr_detail::check(prr_scene_export_mesh(tmp, obj, &nt, &attr, nullptr, nullptr,
                                                        nullptr, nullptr));
                std::vector<float> v(nt * 9), n(nt * 9), uv(nt * 6), tg(nt * 12);
                prr_detail::check(prr_scene_export_mesh(tmp, obj, nullptr, nullptr, v.data(),
                                                        n.data(), uv.data(), tg.data()));
                Material *mat = overrideMat ? overrideMat : export_material(tmp, over < 0 ? k : -1);
                std::vector<Triangle> tris;
                Vector3f lo(std::numeric_limits<float>::infinity());
                Vector3f hi(-std::numeric_limits<float>::infinity());
                for (int64_t i = 0; i < nt; i++) {
                    const float *p = &v[i * 9];
                    Triangle t(Vector3f(p[0], p[1], p[2]), Vector3f(p[3], p[4], p[5]),
                               Vector3f(p[6], p[7], p[8]), mat);
                    for (int q = 0; q < 3; q++) {
                        lo = Vector3f(std::min(lo.x, p[q * 3]), std::min(lo.y, p[q * 3 + 1]),
                                      std::min(lo.z, p[q * 3 + 2]));
                        hi = Vector3f(std::max(hi.x, p[q * 3]), std::max(hi.y, p[q * 3 + 1]),
                                      std::max(hi.z, p[q * 3 + 2]));
                    }
                    if (attr & 1) {
                        const float *c = &n[i * 9];
                        t.n0 = Vector3f(c[0], c[1], c[2]);
                        t.n1 = Vector3f(c[3], c[4], c[5]);
                        t.n2 = Vector3f(c[6], c[7], c[8]);
                        t.hasSmoothNormals = true;
                    }
                    if (attr & 2) {
                        const float *c = &uv[i * 6];
                        t.t0 = Vector2f(c[0], c[1]);
                        t.t1 = Vector2f(c[2], c[3]);
                        t.t2 = Vector2f(c[4], c[5]);
                    }
                    if (attr & 4) {
                        const float *c = &tg[i * 12];
                        t.tan0 = Vector3f(c[0], c[1], c[2]);
                        t.tan1 = Vector3f(c[4], c[5], c[6]);
                        t.tan2 = Vector3f(c[8], c[9], c[10]);
                        t.tangentW0 = c[3];
                        t.tangentW1 = c[7];
                        t.tangentW2 = c[11];
                        t.hasTangents = true;
                    }
                    tris.push_back(t);
                }
                out.push_back(new MeshTriangle(std::move(tris), Bounds3(lo, hi), mat));
            }
        } catch (...) {
            prr_scene_destroy(tmp);
            throw;
        }
        prr_scene_destroy(tmp);
        return out;
    }

  private:
    static Material *export_material(prr_scene *tmp, int id) {
        int kind = 0, tex[4];
        float p[9];
        prr_detail::check(prr_scene_export_material(tmp, id, &kind, p, tex));
        Material *m = kind == PRR_MAT_GLASS      ? (Material *) new GlassMaterial()
                      : kind == PRR_MAT_MIRROR   ? (Material *) new MirrorMaterial()
                      : kind == PRR_MAT_EMISSIVE ? (Material *) new EmissiveMaterial()
                                                 : (Material *) new DiffuseMaterial();
        m->baseColor = Vector3f(p[0], p[1], p[2]);
        m->roughness = p[3];
        m->metallic = p[4];
        m->ior = p[5];
        m->m_emission = Vector3f(p[6], p[7], p[8]);
        Texture *slots[4] = {&m->baseColorTex, &m->metallicRoughnessTex, &m->normalTex,
                             &m->emissiveTex};
        for (int k = 0; k < 4; k++) {
            if (tex[k] < 0)
                continue;
            int w = 0, h = 0, c = 0;
            prr_detail::check(prr_scene_export_texture(tmp, tex[k], &w, &h, &c, nullptr));
            slots[k]->data.resize((size_t) w * h * c);
            slots[k]->width = w;
            slots[k]->height = h;
            slots[k]->channels = c;
            prr_detail::check(
                prr_scene_export_texture(tmp, tex[k], nullptr, nullptr, nullptr, slots[k]->data.data()));
        }
        return m;
    }
};

struct Camera {
    Vector3f eye = Vector3f(0, 0, -1), target = Vector3f(0, 0, 0), up = Vector3f(0, 1, 0);
    float fovv = 40.0f, fovh = 40.0f, aperture = 0.0f, focusDistance = -1.0f;
    int width = 0, height = 0;
    static Camera create(Vector3f eye_, Vector3f target_, Vector3f up_, float fovv_, float fovh_) {
        Camera c;
        c.eye = eye_;
        c.target = target_;
        c.up = up_;
        c.fovv = fovv_;
        c.fovh = fovh_;
        return c;
    }
    static Camera fromBlender(Vector3f eye_, Vector3f target_, Vector3f up_, float fovh_,
                              float fovv_, float focusDist_) { // Camera.hpp:31-41
        Camera c;
        c.eye = Vector3f(eye_.x, eye_.z, -eye_.y);
        c.target = Vector3f(target_.x, target_.z, -target_.y);
        Vector3f u(up_.x, up_.z, -up_.y);
        const float m2 = u.x * u.x + u.y * u.y + u.z * u.z;
        if (m2 > 0) {
            const float inv = 1 / sqrtf(m2);
            u = Vector3f(u.x * inv, u.y * inv, u.z * inv);
        }
        c.up = u;
        c.fovv = fovv_;
        c.fovh = fovh_;
        c.focusDistance = focusDist_;
        return c;
    }
    void init(int w, int h) {
        width = w;
        height = h;
    }
};

struct EnvMap {
    std::vector<float> rgb; // decoded pixels, row-major RGB
    int width = 0, height = 0;
    bool empty() const { return rgb.empty(); }
    void set(const float *pixels, int w, int h) {
        rgb.assign(pixels, pixels + (size_t) w * h * 3);
        width = w;
        height = h;
    }
};

struct Intersection {
    bool happened = false;
    Vector3f coords, normal;
    double tnear = std::numeric_limits<double>::max();
    int object = -1;    // index in Scene::objects
    int primitive = -1; // triangle index within the mesh
};

// Medium (Volume.hpp:7-63): a homogeneous medium; like the reference's
// integrator, rendering does not read Scene::medium. intersect is a one-ray
// batch of prr_medium_intersect.
struct Medium {
    float sigma_a = 0.0f;
    float sigma_s = 0.0f;
    float sigma_t = 0.0f;
    float g = 0.0f;
    bool bounded = false;
    Bounds3 bounds;
    bool active() const { return sigma_t > 1e-6f; }
    bool intersect(const Ray &ray, float &t_enter, float &t_exit) const {
        prr_medium m{};
        m.sigma_a = sigma_a;
        m.sigma_s = sigma_s;
        m.sigma_t = sigma_t;
        m.g = g;
        m.bounded = bounded ? 1 : 0;
        const float lo[3] = {bounds.pMin.x, bounds.pMin.y, bounds.pMin.z};
        const float hi[3] = {bounds.pMax.x, bounds.pMax.y, bounds.pMax.z};
        std::copy(lo, lo + 3, m.bounds_min);
        std::copy(hi, hi + 3, m.bounds_max);
        const float o[3] = {ray.origin.x, ray.origin.y, ray.origin.z};
        const float d[3] = {ray.direction.x, ray.direction.y, ray.direction.z};
        prr_detail::DeviceArray<float> dO(3), dD(3), dE(1), dX(1);
        prr_detail::DeviceArray<uint8_t> dH(1);
        dO.put(o);
        dD.put(d);
        prr_detail::check(prr_medium_intersect(&m, dO.p, dD.p, 1, dE.p, dX.p, dH.p, nullptr));
        uint8_t hit;
        dH.get(&hit);
        if (hit) {
            dE.get(&t_enter);
            dX.get(&t_exit);
        }
        return hit != 0;
    }
    static Medium preset(int which) {
        prr_medium p{};
        prr_detail::check(prr_medium_preset(which, &p));
        Medium m;
        m.sigma_a = p.sigma_a;
        m.sigma_s = p.sigma_s;
        m.sigma_t = p.sigma_t;
        m.g = p.g;
        return m;
    }
    static Medium dust() { return preset(PRR_MEDIUM_DUST); }
    static Medium fog() { return preset(PRR_MEDIUM_FOG); }
};

class Scene {
  public:
    Vector3f backgroundColor = Vector3f(0.235294f, 0.67451f, 0.843137f);
    std::vector<Object *> objects;
    EnvMap envMap;
    Camera camera;
    Medium medium; // Scene.hpp:25; not read by rendering, as in the reference

    Scene() { prr_detail::check(prr_scene_create(&h_)); }
    ~Scene() { prr_scene_destroy(h_); }
    Scene(const Scene &) = delete;
    Scene &operator=(const Scene &) = delete;

    void Add(Object *object) { objects.push_back(object); }

    // Scene::buildBVH (Scene.cpp:15-27): uploads everything and builds on the GPU.
    void buildBVH() {
        std::vector<Material *> mats;
        std::vector<int> mat_ids;
        auto mat_id = [&](Material *m) {
            for (size_t k = 0; k < mats.size(); k++)
                if (mats[k] == m)
                    return mat_ids[k];
            const float p[9] = {m->baseColor.x, m->baseColor.y, m->baseColor.z, m->roughness,
                                m->metallic,    m->ior,         m->m_emission.x, m->m_emission.y,
                                m->m_emission.z};
            int id = -1;
            prr_detail::check(prr_scene_add_material(h_, m->kind(), p, &id));
            const Texture *tex[4] = {&m->baseColorTex, &m->metallicRoughnessTex, &m->normalTex,
                                     &m->emissiveTex};
            int tid[4] = {-1, -1, -1, -1};
            for (int k = 0; k < 4; k++)
                if (!tex[k]->empty())
                    prr_detail::check(prr_scene_add_texture(h_, tex[k]->data.data(),
                                                            tex[k]->width, tex[k]->height,
                                                            tex[k]->channels, &tid[k]));
            if (tid[0] >= 0 || tid[1] >= 0 || tid[2] >= 0 || tid[3] >= 0)
                prr_detail::check(
                    prr_scene_set_material_textures(h_, id, tid[0], tid[1], tid[2], tid[3]));
            mats.push_back(m);
            mat_ids.push_back(id);
            return id;
        };
        for (Object *o : objects) {
            const int mid = mat_id(o->m);
            if (auto *mesh = dynamic_cast<MeshTriangle *>(o)) {
                const size_t n = mesh->triangles.size();
                std::vector<float> v, nrm, uv, tg;
                bool has_n = n > 0, has_t = n > 0, has_uv = false;
                for (const Triangle &t : mesh->triangles) {
                    has_n = has_n && t.hasSmoothNormals;
                    has_t = has_t && t.hasTangents;
                    for (const Vector2f *q : {&t.t0, &t.t1, &t.t2})
                        has_uv = has_uv || q->x != 0.f || q->y != 0.f;
                }
                for (const Triangle &t : mesh->triangles) {
                    for (const Vector3f &p : {t.v0, t.v1, t.v2})
                        v.insert(v.end(), {p.x, p.y, p.z});
                    if (has_n)
                        for (const Vector3f &p : {t.n0, t.n1, t.n2})
                            nrm.insert(nrm.end(), {p.x, p.y, p.z});
                    if (has_uv)
                        for (const Vector2f &p : {t.t0, t.t1, t.t2})
                            uv.insert(uv.end(), {p.x, p.y});
                    if (has_t) {
                        tg.insert(tg.end(), {t.tan0.x, t.tan0.y, t.tan0.z, t.tangentW0});
                        tg.insert(tg.end(), {t.tan1.x, t.tan1.y, t.tan1.z, t.tangentW1});
                        tg.insert(tg.end(), {t.tan2.x, t.tan2.y, t.tan2.z, t.tangentW2});
                    }
                }
                prr_detail::check(prr_scene_add_mesh_attr(
                    h_, v.data(), has_n ? nrm.data() : nullptr, has_uv ? uv.data() : nullptr,
                    has_t ? tg.data() : nullptr, (int64_t) n, mid, nullptr));
            } else if (auto *s = dynamic_cast<Sphere *>(o)) {
                const float c[3] = {s->center.x, s->center.y, s->center.z};
                prr_detail::check(prr_scene_add_sphere(h_, c, s->radius, mid, nullptr));
            } else {
                throw std::runtime_error("unsupported object type");
            }
        }
        const float bg[3] = {backgroundColor.x, backgroundColor.y, backgroundColor.z};
        prr_detail::check(prr_scene_set_background(h_, bg));
        if (!envMap.empty())
            prr_detail::check(prr_scene_set_env(h_, envMap.rgb.data(), envMap.width, envMap.height));
        prr_camera c{};
        const Vector3f *vs[3] = {&camera.eye, &camera.target, &camera.up};
        float *ds[3] = {c.eye, c.target, c.up};
        for (int k = 0; k < 3; k++) {
            ds[k][0] = vs[k]->x;
            ds[k][1] = vs[k]->y;
            ds[k][2] = vs[k]->z;
        }
        c.fovv = camera.fovv;
        c.fovh = camera.fovh;
        c.aperture = camera.aperture;
        c.focus_distance = camera.focusDistance;
        if (camera.width > 0)
            prr_detail::check(prr_scene_set_camera(h_, &c, camera.width, camera.height));
        prr_detail::check(prr_scene_build(h_, nullptr));
    }

    // Scene::intersect (one-ray batch)
    Intersection intersect(const Ray &ray) const {
        const float o[3] = {ray.origin.x, ray.origin.y, ray.origin.z};
        const float d[3] = {ray.direction.x, ray.direction.y, ray.direction.z};
        prr_detail::DeviceArray<float> dO(3), dD(3), dT(1), dG(6);
        prr_detail::DeviceArray<int32_t> dObj(1), dPrim(1);
        dO.put(o);
        dD.put(d);
        prr_detail::check(prr_scene_intersect(h_, dO.p, dD.p, 1, dObj.p, dPrim.p, dT.p, dG.p, nullptr));
        int32_t obj, prim;
        float t, g[6];
        dObj.get(&obj);
        dPrim.get(&prim);
        dT.get(&t);
        dG.get(g);
        Intersection in;
        in.happened = obj >= 0;
        if (in.happened) {
            in.object = obj;
            in.primitive = prim;
            in.tnear = t;
            in.coords = Vector3f(g[0], g[1], g[2]);
            in.normal = Vector3f(g[3], g[4], g[5]);
        }
        return in;
    }

    // Scene::intersectP (one-ray batch)
    bool intersectP(const Ray &ray, float tMax = std::numeric_limits<float>::infinity()) const {
        const float o[3] = {ray.origin.x, ray.origin.y, ray.origin.z};
        const float d[3] = {ray.direction.x, ray.direction.y, ray.direction.z};
        prr_detail::DeviceArray<float> dO(3), dD(3), dM(1);
        prr_detail::DeviceArray<uint8_t> dH(1);
        dO.put(o);
        dD.put(d);
        dM.put(&tMax);
        prr_detail::check(prr_scene_occluded(h_, dO.p, dD.p, dM.p, 1, dH.p, nullptr));
        uint8_t hit;
        dH.get(&hit);
        return hit != 0;
    }

    prr_scene *handle() const { return h_; }

  private:
    prr_scene *h_ = nullptr;
};

class Integrator {
  public:
    float directClamp = 0.f;
    float indirectClamp = 10.0f;
    Integrator(const Scene &scene_, int maxDepth_, float rrThreshold_)
        : scene(scene_), maxDepth(maxDepth_), rrThreshold(rrThreshold_) {}

    // Integrator::castRay (Integrator.cpp:104-263) for one ray; successive
    // calls draw from streams (seed, 0, 0), (seed, 1, 0), ...
    Vector3f castRay(const Ray &ray) const {
        const float o[3] = {ray.origin.x, ray.origin.y, ray.origin.z};
        const float d[3] = {ray.direction.x, ray.direction.y, ray.direction.z};
        prr_detail::DeviceArray<float> dO(3), dD(3), out(3);
        dO.put(o);
        dD.put(d);
        prr_detail::check(prr_cast_rays(scene.handle(), dO.p, dD.p, 1, seed_ + calls_++ * 0x9E3779B97F4A7C15ull,
                                        maxDepth, indirectClamp, out.p, nullptr));
        float r[3];
        out.get(r);
        return Vector3f(r[0], r[1], r[2]);
    }

    // castRay for camera sample `sample` of pixel (i, j): the path the
    // renderer traces for it (the ray itself is generated from the scene's
    // camera and the (seed, pixel, sample) stream).
    Vector3f castSample(int i, int j, int sample, uint64_t seed = 1) const {
        prr_detail::DeviceArray<int32_t> a(1), b(1), c(1);
        prr_detail::DeviceArray<float> out(3);
        a.put(&i);
        b.put(&j);
        c.put(&sample);
        prr_detail::check(prr_cast_samples(scene.handle(), a.p, b.p, c.p, 1, seed, maxDepth,
                                           indirectClamp, out.p, nullptr));
        float r[3];
        out.get(r);
        return Vector3f(r[0], r[1], r[2]);
    }
    const Scene &scene;
    int maxDepth;
    float rrThreshold; // stored, unused: as in the reference (Integrator.cpp:250-256)

  private:
    uint64_t seed_ = 1;
    mutable uint64_t calls_ = 0;
};

namespace tonemap {
enum class ToneMapper { Raw = PRR_TONEMAP_RAW, Standard = PRR_TONEMAP_STANDARD,
                        AgX = PRR_TONEMAP_AGX, PBRNeutral = PRR_TONEMAP_PBR_NEUTRAL,
                        ACES = PRR_TONEMAP_ACES };
} // namespace tonemap

struct RenderSettings {
    int width = 1280;
    int height = 1720;
    int minSPP = 64;
    int maxSPP = 64;
    float russianRoulette = 0.95f;
    int maxDepth = 30;
    float varianceThreshold = 0.05f;
    float exposure = 0.18f;
    tonemap::ToneMapper toneMapper = tonemap::ToneMapper::AgX;
    // additions of this implementation
    uint64_t seed = 1;
    int mode = PRR_RENDER_WAVEFRONT;
};

class Renderer {
  public:
    // Renderer::Render (Renderer.cpp:24-212): render, tone map, write PPMs.
    void Render(const Scene &scene, const Integrator &integrator, const RenderSettings &s) {
        prr_render_settings rs{};
        rs.width = s.width;
        rs.height = s.height;
        rs.min_spp = s.minSPP;
        rs.max_spp = s.maxSPP;
        rs.max_depth = integrator.maxDepth;
        rs.variance_threshold = s.varianceThreshold;
        rs.indirect_clamp = integrator.indirectClamp;
        rs.mode = s.mode;
        rs.seed = s.seed;
        const size_t n = (size_t) s.width * s.height;
        prr_detail::DeviceArray<float> rgb(n * 3);
        prr_detail::DeviceArray<int32_t> spp(n);
        prr_detail::check(prr_render(scene.handle(), &rs, rgb.p, spp.p, nullptr, nullptr));
        framebuffer_.resize(n * 3);
        rgb.get(framebuffer_.data());
        sampleCount_.resize(n);
        spp.get(sampleCount_.data());
        write(rgb, s.exposure, (int) s.toneMapper, s.width, s.height, "output");
        if (s.toneMapper != tonemap::ToneMapper::Raw)
            write(rgb, s.exposure, PRR_TONEMAP_RAW, s.width, s.height, "output_raw");
        // adaptive-sampling visualisation (Renderer.cpp:193-211)
        std::vector<uint8_t> vis(n * 3);
        prr_detail::check(
            prr_sample_count_image(sampleCount_.data(), (int64_t) n, s.maxSPP, vis.data()));
        prr_detail::check(prr_write_image("sample_count.ppm", vis.data(), s.width, s.height));
        prr_detail::check(prr_write_image("sample_count.png", vis.data(), s.width, s.height));
    }
    const std::vector<float> &framebuffer() const { return framebuffer_; }
    const std::vector<int32_t> &sampleCount() const { return sampleCount_; }

  private:
    // Renderer.cpp:163-185: tone map, then <base>.ppm and <base>.png
    static void write(const prr_detail::DeviceArray<float> &rgb, float exposure, int mapper, int w,
                      int h, const char *base) {
        const size_t n = (size_t) w * h;
        prr_detail::DeviceArray<uint8_t> u8(n * 3);
        prr_detail::check(prr_tonemap(mapper, exposure, rgb.p, (int64_t) n, nullptr, u8.p, nullptr));
        std::vector<uint8_t> buf(n * 3);
        u8.get(buf.data());
        prr_detail::check(prr_write_image((std::string(base) + ".ppm").c_str(), buf.data(), w, h));
        prr_detail::check(prr_write_image((std::string(base) + ".png").c_str(), buf.data(), w, h));
    }
    std::vector<float> framebuffer_;
    std::vector<int32_t> sampleCount_;
};
