// Test infrastructure only (the oracle): a C ABI over the reference renderer's
// own C++ code, compiled in place from the reference sources by
// oracle/Makefile. Tests and the CPU-baseline leg of bench.py load the
// resulting oracle/_ref/libprr_ref*.so with ctypes; nothing in the product
// links it.
//
// What it wraps (reference file:line):
//   MeshTriangle(tris, bounds, mat)      Triangle.hpp:116-124 -> BVHAccel(ptrs, 4)
//   BVHAccel::Intersect / IntersectP     BVH.cpp:311-415 / :421-473
//   Scene::Add / buildBVH / intersect    Scene.hpp:15-41, Scene.cpp:15-35
//   Camera::create / init / generateRay  Camera.hpp:23-56, :75-95
//   Integrator::castRay                  Integrator.cpp:104-263
//   Renderer per-pixel sample loop       Renderer.cpp:63-99 (restated below: the
//                                        reference keeps the linear framebuffer
//                                        local to Render and only writes 8-bit files)
//   EnvMap::load / sample / importance*  EnvMap.hpp:35-169
//   PhotonMap::emit / trace / build      Photon.cpp:96-188 (emit restated so that
//                                        each photon draws from its own RNG stream)
//   PhotonGrid / estimateIrradiance      Photon.cpp:24-94
//   tonemap::apply + exposure            ToneMapping.hpp:267-279, Renderer.cpp:149-171
//
// Random numbers: prelude.hpp renames the reference's thread-local SplitMix64
// (global.hpp:35-50) and routes every call site to get_random_float() below,
// a SplitMix64 whose state is set per path from (seed, stream, index).

#include <algorithm>
#include <array>
#include <atomic>
#include <cassert>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <limits>
#include <numeric>
#include <queue>
#include <random>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>
#include <omp.h>

#include "GLTFLoader.hpp"

// Private members needed by the oracle: BVHAccel's flattened nodes (to diff
// the device tree node for node) and PhotonMap::trace (to key each photon's RNG
// stream by its index).
#define private public
#include "Camera.hpp"
#include "EnvMap.hpp"
#include "Integrator.hpp"
#include "Material.hpp"
#include "Renderer.hpp"
#include "Scene.hpp"
#include "Sphere.hpp"
#include "ToneMapping.hpp"
#include "Triangle.hpp"
#undef private

#include "stb_image_write.h"

// ---------------------------------------------------------------------------
// Counter-keyed SplitMix64 stream (the replacement for global.hpp:35-50).
// path state = mix(mix(seed ^ K0) ^ (stream << 32 | index)); each draw adds
// the golden gamma and returns the top 24 bits of the finalised value, the
// same output form as the reference generator.
// ---------------------------------------------------------------------------
static inline uint64_t ref_mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

static inline uint64_t ref_path_state(uint64_t seed, uint32_t stream, uint32_t index) {
    return ref_mix64(ref_mix64(seed ^ 0x6A09E667F3BCC909ULL) ^
                     (((uint64_t) stream << 32) | (uint64_t) index));
}

static thread_local uint64_t g_rng_state = 0;
static thread_local uint64_t g_rng_draws = 0;

float get_random_float() {
    uint64_t z = (g_rng_state += 0x9E3779B97F4A7C15ULL);
    z = ref_mix64(z);
    g_rng_draws++;
    return (z >> 40) * 0x1p-24f;
}

static inline void ref_set_path(uint64_t seed, uint32_t stream, uint32_t index) {
    g_rng_state = ref_path_state(seed, stream, index);
    g_rng_draws = 0;
}

extern "C" {

void prr_ref_rng_stream(uint64_t seed, uint32_t stream, uint32_t index, int n, float *out) {
    ref_set_path(seed, stream, index);
    for (int i = 0; i < n; i++)
        out[i] = get_random_float();
}

int prr_ref_max_threads(void) {
    return omp_get_max_threads();
}

// ---------------------------------------------------------------------------
// Single mesh: MeshTriangle + its BVHAccel(maxPrimsInNode = 4).
// ---------------------------------------------------------------------------
struct RefMesh {
    DiffuseMaterial mat;
    MeshTriangle *mesh = nullptr;
};

static Bounds3 vertex_bounds(const float *v, int64_t ntri) {
    // Same bounds the OBJ constructor computes (Triangle.cpp:12-30).
    Vector3f minVert(std::numeric_limits<float>::infinity());
    Vector3f maxVert(-std::numeric_limits<float>::infinity());
    for (int64_t i = 0; i < ntri * 3; i++) {
        Vector3f p(v[i * 3 + 0], v[i * 3 + 1], v[i * 3 + 2]);
        minVert = Vector3f(std::min(minVert.x, p.x), std::min(minVert.y, p.y),
                           std::min(minVert.z, p.z));
        maxVert = Vector3f(std::max(maxVert.x, p.x), std::max(maxVert.y, p.y),
                           std::max(maxVert.z, p.z));
    }
    return Bounds3(minVert, maxVert);
}

static std::vector<Triangle> make_tris(const float *v, int64_t ntri, Material *m) {
    std::vector<Triangle> tris;
    tris.reserve(ntri);
    for (int64_t i = 0; i < ntri; i++) {
        const float *p = v + i * 9;
        tris.emplace_back(Vector3f(p[0], p[1], p[2]), Vector3f(p[3], p[4], p[5]),
                          Vector3f(p[6], p[7], p[8]), m);
    }
    return tris;
}

void *prr_ref_mesh_new(const float *verts, int64_t ntri) {
    RefMesh *rm = new RefMesh();
    rm->mesh = new MeshTriangle(make_tris(verts, ntri, &rm->mat), vertex_bounds(verts, ntri),
                                &rm->mat);
    return rm;
}

void prr_ref_mesh_free(void *h) {
    RefMesh *rm = (RefMesh *) h;
    if (!rm)
        return;
    delete rm->mesh->bvh;
    delete rm->mesh;
    delete rm;
}

static int64_t export_bvh(const BVHAccel *bvh, const Object *first_prim, size_t prim_size,
                          float *bounds, uint32_t *first_child, uint32_t *meta, float *areas,
                          int32_t *ordered) {
    int64_t n = (int64_t) bvh->nodes.size();
    for (int64_t i = 0; i < n; i++) {
        const BVHNode &nd = bvh->nodes[i];
        if (bounds)
            for (int k = 0; k < 6; k++)
                bounds[i * 6 + k] = nd.bounds[k];
        if (first_child)
            first_child[i] = nd.first_child;
        if (meta)
            meta[i] = nd.meta;
        if (areas)
            areas[i] = bvh->nodeAreas[i];
    }
    if (ordered)
        for (size_t i = 0; i < bvh->orderedPrims.size(); i++)
            ordered[i] = (int32_t) (((const char *) bvh->orderedPrims[i] -
                                     (const char *) first_prim) /
                                    (ptrdiff_t) prim_size);
    return n;
}

int64_t prr_ref_mesh_nodes(void *h, float *bounds, uint32_t *first_child, uint32_t *meta,
                           float *areas, int32_t *ordered) {
    RefMesh *rm = (RefMesh *) h;
    return export_bvh(rm->mesh->bvh, &rm->mesh->triangles[0], sizeof(Triangle), bounds,
                      first_child, meta, areas, ordered);
}

float prr_ref_mesh_area(void *h, float *bvh_total_area) {
    RefMesh *rm = (RefMesh *) h;
    if (bvh_total_area)
        *bvh_total_area = rm->mesh->bvh->totalArea;
    return rm->mesh->area;
}

// Closest hit through BVHAccel::Intersect on the mesh BVH (the config-2
// micro-path). id = index of the hit triangle in input order, -1 on a miss.
void prr_ref_mesh_intersect(void *h, const float *o, const float *d, int64_t n, int32_t *id,
                            float *t, float *u, float *v, int nthreads) {
    RefMesh *rm = (RefMesh *) h;
    const Triangle *base = &rm->mesh->triangles[0];
    if (nthreads > 0)
        omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t i = 0; i < n; i++) {
        Ray ray(Vector3f(o[i * 3], o[i * 3 + 1], o[i * 3 + 2]),
                Vector3f(d[i * 3], d[i * 3 + 1], d[i * 3 + 2]));
        Intersection in = rm->mesh->bvh->Intersect(ray);
        if (in.happened) {
            id[i] = (int32_t) ((const Triangle *) in.obj - base);
            t[i] = (float) in.tnear;
            if (u || v) {
                // finalize() keeps only the interpolated uv; recompute the
                // barycentrics of the winning triangle with its own hitTest.
                Triangle::TriHit hh = ((const Triangle *) in.obj)->hitTest(ray);
                if (u)
                    u[i] = hh.u;
                if (v)
                    v[i] = hh.v;
            }
        } else {
            id[i] = -1;
            t[i] = std::numeric_limits<float>::infinity();
            if (u)
                u[i] = 0.f;
            if (v)
                v[i] = 0.f;
        }
    }
}

void prr_ref_mesh_occluded(void *h, const float *o, const float *d, const float *tmax, int64_t n,
                           uint8_t *hit, int nthreads) {
    RefMesh *rm = (RefMesh *) h;
    if (nthreads > 0)
        omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t i = 0; i < n; i++) {
        Ray ray(Vector3f(o[i * 3], o[i * 3 + 1], o[i * 3 + 2]),
                Vector3f(d[i * 3], d[i * 3 + 1], d[i * 3 + 2]));
        hit[i] = rm->mesh->bvh->IntersectP(ray, tmax[i]) ? 1 : 0;
    }
}

// ---------------------------------------------------------------------------
// Scene: materials, meshes, spheres, env map, camera.
// ---------------------------------------------------------------------------
enum { REF_MAT_DIFFUSE = 0, REF_MAT_EMISSIVE = 1, REF_MAT_MIRROR = 2, REF_MAT_GLASS = 3 };

struct RefScene {
    Scene scene;
    std::vector<Material *> materials;
    std::vector<Object *> objects;
    std::vector<int> object_kind; // 0 mesh, 1 sphere
    int width = 0, height = 0;
};

void *prr_ref_scene_new(void) {
    return new RefScene();
}

void prr_ref_scene_free(void *h) {
    RefScene *rs = (RefScene *) h;
    if (!rs)
        return;
    for (size_t i = 0; i < rs->objects.size(); i++) {
        if (rs->object_kind[i] == 0) {
            MeshTriangle *m = (MeshTriangle *) rs->objects[i];
            delete m->bvh;
            delete m;
        } else {
            delete (Sphere *) rs->objects[i];
        }
    }
    for (auto *m : rs->materials)
        delete m;
    delete rs->scene.bvh;
    delete rs;
}

// params: baseColor[3], roughness, metallic, ior, emission[3]
int prr_ref_scene_add_material(void *h, int type, const float *p) {
    RefScene *rs = (RefScene *) h;
    Material *m = nullptr;
    switch (type) {
    case REF_MAT_DIFFUSE:
        m = new DiffuseMaterial();
        break;
    case REF_MAT_EMISSIVE:
        m = new EmissiveMaterial();
        break;
    case REF_MAT_MIRROR:
        m = new MirrorMaterial();
        break;
    case REF_MAT_GLASS:
        m = new GlassMaterial();
        break;
    default:
        return -1;
    }
    m->baseColor = Vector3f(p[0], p[1], p[2]);
    m->roughness = p[3];
    m->metallic = p[4];
    m->ior = p[5];
    m->m_emission = Vector3f(p[6], p[7], p[8]);
    rs->materials.push_back(m);
    return (int) rs->materials.size() - 1;
}

int prr_ref_scene_add_mesh(void *h, const float *verts, int64_t ntri, int mat) {
    RefScene *rs = (RefScene *) h;
    Material *m = rs->materials.at(mat);
    MeshTriangle *mesh = new MeshTriangle(make_tris(verts, ntri, m), vertex_bounds(verts, ntri), m);
    rs->scene.Add(mesh);
    rs->objects.push_back(mesh);
    rs->object_kind.push_back(0);
    return (int) rs->objects.size() - 1;
}

// A MeshTriangle whose triangles carry per-corner data set the way
// GLTFLoader::load does (GLTFLoader.cpp:236-262): normalized corner normals
// and face normal normalize(n0 + n1 + n2), uvs, tangents with handedness.
int prr_ref_scene_add_mesh_attr(void *h, const float *verts, const float *nrm, const float *uv,
                                const float *tan, int64_t ntri, int mat) {
    RefScene *rs = (RefScene *) h;
    Material *m = rs->materials.at(mat);
    std::vector<Triangle> tris = make_tris(verts, ntri, m);
    for (int64_t i = 0; i < ntri; i++) {
        Triangle &tri = tris[i];
        if (nrm) {
            const float *n = nrm + i * 9;
            tri.n0 = normalize(Vector3f(n[0], n[1], n[2]));
            tri.n1 = normalize(Vector3f(n[3], n[4], n[5]));
            tri.n2 = normalize(Vector3f(n[6], n[7], n[8]));
            tri.hasSmoothNormals = true;
            tri.normal = normalize(tri.n0 + tri.n1 + tri.n2);
        }
        if (uv) {
            const float *t = uv + i * 6;
            tri.t0 = Vector2f(t[0], t[1]);
            tri.t1 = Vector2f(t[2], t[3]);
            tri.t2 = Vector2f(t[4], t[5]);
        }
        if (tan) {
            const float *t = tan + i * 12;
            tri.tan0 = Vector3f(t[0], t[1], t[2]);
            tri.tan1 = Vector3f(t[4], t[5], t[6]);
            tri.tan2 = Vector3f(t[8], t[9], t[10]);
            tri.tangentW0 = t[3];
            tri.tangentW1 = t[7];
            tri.tangentW2 = t[11];
            tri.hasTangents = true;
        }
    }
    MeshTriangle *mesh = new MeshTriangle(std::move(tris), vertex_bounds(verts, ntri), m);
    rs->scene.Add(mesh);
    rs->objects.push_back(mesh);
    rs->object_kind.push_back(0);
    return (int) rs->objects.size() - 1;
}

// Material textures (Material.hpp:45-48): slot 0 base colour, 1 metallic-
// roughness, 2 normal, 3 emissive.
int prr_ref_scene_set_texture(void *h, int mat, int slot, const uint8_t *texels, int w, int hgt,
                              int channels) {
    RefScene *rs = (RefScene *) h;
    Material *m = rs->materials.at(mat);
    Texture *t = slot == 0   ? &m->baseColorTex
                 : slot == 1 ? &m->metallicRoughnessTex
                 : slot == 2 ? &m->normalTex
                 : slot == 3 ? &m->emissiveTex
                             : nullptr;
    if (!t)
        return -1;
    t->data.assign(texels, texels + (size_t) w * hgt * channels);
    t->width = w;
    t->height = hgt;
    t->channels = channels;
    return 0;
}

// GLTFLoader::load(path, type) + Scene::Add of every mesh it returns (the
// reference's own ingest, main scene files' usage).
int prr_ref_scene_add_gltf(void *h, const char *path, int type) {
    RefScene *rs = (RefScene *) h;
    std::vector<MeshTriangle *> meshes = GLTFLoader::load(path, (MaterialType) type);
    for (MeshTriangle *m : meshes) {
        rs->scene.Add(m);
        rs->objects.push_back(m);
        rs->object_kind.push_back(0);
        rs->materials.push_back(m->m);
    }
    return (int) meshes.size();
}

// MeshTriangle(filename, offset, m) + Scene::Add (Triangle.cpp:4-32): the OBJ
// file read by the reference's own loader. Returns the object index.
int prr_ref_scene_add_obj(void *h, const char *path, const float *offset, int mat) {
    RefScene *rs = (RefScene *) h;
    MeshTriangle *m = new MeshTriangle(std::string(path), Vector3f(offset[0], offset[1], offset[2]),
                                       rs->materials.at(mat));
    rs->scene.Add(m);
    rs->objects.push_back(m);
    rs->object_kind.push_back(0);
    return (int) rs->objects.size() - 1;
}

// A mesh object's triangles as the reference holds them: v0 v1 v2, n0 n1 n2,
// t0 t1 t2, tan0..2 with handedness; attr bit 1 = smooth normals, 4 = tangents.
int64_t prr_ref_scene_export_mesh(void *h, int obj, int *attr, float *verts, float *normals,
                                  float *uvs, float *tangents) {
    RefScene *rs = (RefScene *) h;
    MeshTriangle *mt = dynamic_cast<MeshTriangle *>(rs->objects.at(obj));
    if (!mt)
        return -1;
    int a = 0;
    const int64_t n = (int64_t) mt->triangles.size();
    for (int64_t i = 0; i < n; i++) {
        const Triangle &t = mt->triangles[i];
        a |= (t.hasSmoothNormals ? 1 : 0) | (t.hasTangents ? 4 : 0);
        const Vector3f *p[3] = {&t.v0, &t.v1, &t.v2};
        const Vector3f *nn[3] = {&t.n0, &t.n1, &t.n2};
        const Vector2f *uv[3] = {&t.t0, &t.t1, &t.t2};
        const Vector3f *tg[3] = {&t.tan0, &t.tan1, &t.tan2};
        const float tw[3] = {t.tangentW0, t.tangentW1, t.tangentW2};
        for (int q = 0; q < 3; q++) {
            if (verts) {
                verts[i * 9 + q * 3] = p[q]->x;
                verts[i * 9 + q * 3 + 1] = p[q]->y;
                verts[i * 9 + q * 3 + 2] = p[q]->z;
            }
            if (normals) {
                normals[i * 9 + q * 3] = nn[q]->x;
                normals[i * 9 + q * 3 + 1] = nn[q]->y;
                normals[i * 9 + q * 3 + 2] = nn[q]->z;
            }
            if (uvs) {
                uvs[i * 6 + q * 2] = uv[q]->x;
                uvs[i * 6 + q * 2 + 1] = uv[q]->y;
            }
            if (tangents) {
                tangents[i * 12 + q * 4] = tg[q]->x;
                tangents[i * 12 + q * 4 + 1] = tg[q]->y;
                tangents[i * 12 + q * 4 + 2] = tg[q]->z;
                tangents[i * 12 + q * 4 + 3] = tw[q];
            }
        }
    }
    if (attr)
        *attr = a;
    return n;
}

// The material of a mesh object: kind (0 diffuse, 1 emissive, 2 mirror, 3
// glass), params[9], and per texture slot (base colour, metallic-roughness,
// normal, emissive) its width, height, channels and byte count (zeros when
// empty; a 16-bit emissive image keeps 2 bytes per sample).
int prr_ref_scene_export_material(void *h, int obj, int *kind, float *params, int *tex_dims) {
    RefScene *rs = (RefScene *) h;
    MeshTriangle *mt = dynamic_cast<MeshTriangle *>(rs->objects.at(obj));
    if (!mt)
        return -1;
    const Material *m = mt->m;
    *kind = dynamic_cast<const EmissiveMaterial *>(m) ? 1
            : dynamic_cast<const MirrorMaterial *>(m) ? 2
            : dynamic_cast<const GlassMaterial *>(m)  ? 3
                                                      : 0;
    const float p[9] = {m->baseColor.x, m->baseColor.y, m->baseColor.z, m->roughness,
                        m->metallic,    m->ior,         m->m_emission.x, m->m_emission.y,
                        m->m_emission.z};
    std::memcpy(params, p, sizeof(p));
    const Texture *t[4] = {&m->baseColorTex, &m->metallicRoughnessTex, &m->normalTex,
                           &m->emissiveTex};
    for (int k = 0; k < 4; k++) {
        const bool e = t[k]->empty();
        tex_dims[k * 4] = e ? 0 : t[k]->width;
        tex_dims[k * 4 + 1] = e ? 0 : t[k]->height;
        tex_dims[k * 4 + 2] = e ? 0 : t[k]->channels;
        tex_dims[k * 4 + 3] = e ? 0 : (int) t[k]->data.size();
    }
    return 0;
}

int prr_ref_scene_export_texture(void *h, int obj, int slot, uint8_t *texels) {
    RefScene *rs = (RefScene *) h;
    MeshTriangle *mt = dynamic_cast<MeshTriangle *>(rs->objects.at(obj));
    if (!mt || slot < 0 || slot > 3)
        return -1;
    const Material *m = mt->m;
    const Texture *t[4] = {&m->baseColorTex, &m->metallicRoughnessTex, &m->normalTex,
                           &m->emissiveTex};
    std::memcpy(texels, t[slot]->data.data(), t[slot]->data.size());
    return 0;
}

int prr_ref_scene_add_sphere(void *h, const float *c, float r, int mat) {
    RefScene *rs = (RefScene *) h;
    Sphere *s = new Sphere(Vector3f(c[0], c[1], c[2]), r, rs->materials.at(mat));
    rs->scene.Add(s);
    rs->objects.push_back(s);
    rs->object_kind.push_back(1);
    return (int) rs->objects.size() - 1;
}

void prr_ref_scene_set_background(void *h, const float *rgb) {
    RefScene *rs = (RefScene *) h;
    rs->scene.backgroundColor = Vector3f(rgb[0], rgb[1], rgb[2]);
}

// EnvMap can only be filled through load(path) (buildCDF is private,
// EnvMap.hpp:189). Write the pixels as Radiance .hdr with the vendored stb
// writer, then load them back through the reference's own loader.
int prr_ref_scene_set_env(void *h, const float *rgb, int w, int hgt, const char *tmp_path) {
    RefScene *rs = (RefScene *) h;
    if (!stbi_write_hdr(tmp_path, w, hgt, 3, rgb))
        return -1;
    return rs->scene.envMap.load(tmp_path) ? 0 : -2;
}

int prr_ref_scene_env_export(void *h, float *pixels, float *cdf, float *marginal, float *total) {
    RefScene *rs = (RefScene *) h;
    const EnvMap &e = rs->scene.envMap;
    if (!e.loaded)
        return -1;
    int64_t n = (int64_t) e.width * e.height;
    if (pixels)
        for (int64_t i = 0; i < n; i++) {
            pixels[i * 3 + 0] = e.pixels[i].x;
            pixels[i * 3 + 1] = e.pixels[i].y;
            pixels[i * 3 + 2] = e.pixels[i].z;
        }
    if (cdf)
        std::memcpy(cdf, e.cdf.data(), sizeof(float) * n);
    if (marginal)
        std::memcpy(marginal, e.marginalCdf.data(), sizeof(float) * e.height);
    if (total)
        *total = e.totalLuminance;
    return 0;
}

// EnvMap lookups for unit parity: sample(dir) -> rgb, importanceSamplePdf(dir).
void prr_ref_env_eval(void *h, const float *dirs, int64_t n, float *rgb, float *pdf) {
    RefScene *rs = (RefScene *) h;
    const EnvMap &e = rs->scene.envMap;
    for (int64_t i = 0; i < n; i++) {
        Vector3f d(dirs[i * 3], dirs[i * 3 + 1], dirs[i * 3 + 2]);
        Vector3f c = e.sample(d);
        rgb[i * 3 + 0] = c.x;
        rgb[i * 3 + 1] = c.y;
        rgb[i * 3 + 2] = c.z;
        pdf[i] = e.importanceSamplePdf(d);
    }
}

// EnvMap::importanceSample with the stream (seed, i, 0) per sample.
void prr_ref_env_importance(void *h, uint64_t seed, int64_t n, float *dirs, float *pdf) {
    RefScene *rs = (RefScene *) h;
    const EnvMap &e = rs->scene.envMap;
    for (int64_t i = 0; i < n; i++) {
        ref_set_path(seed, (uint32_t) i, 0u);
        float p;
        Vector3f d = e.importanceSample(p);
        dirs[i * 3 + 0] = d.x;
        dirs[i * 3 + 1] = d.y;
        dirs[i * 3 + 2] = d.z;
        pdf[i] = p;
    }
}

void prr_ref_scene_set_camera(void *h, const float *eye, const float *target, const float *up,
                              float fovv, float fovh, float aperture, float focus, int W, int H) {
    RefScene *rs = (RefScene *) h;
    Camera c = Camera::create(Vector3f(eye[0], eye[1], eye[2]),
                              Vector3f(target[0], target[1], target[2]),
                              Vector3f(up[0], up[1], up[2]), fovv, fovh);
    c.aperture = aperture;
    c.focusDistance = focus;
    rs->scene.camera = c;
    rs->scene.camera.init(W, H);
    rs->width = W;
    rs->height = H;
}

void prr_ref_scene_build(void *h) {
    RefScene *rs = (RefScene *) h;
    rs->scene.buildBVH();
}

// The reference Scene object itself, for code that consumes reference scenes
// (the libprr bridge test in bridge.cpp).
void *prr_ref_scene_object(void *h, int *width, int *height) {
    RefScene *rs = (RefScene *) h;
    *width = rs->width;
    *height = rs->height;
    return &rs->scene;
}

int64_t prr_ref_scene_tlas_nodes(void *h, float *bounds, uint32_t *first_child, uint32_t *meta,
                                 float *areas, int32_t *ordered) {
    RefScene *rs = (RefScene *) h;
    const BVHAccel *bvh = rs->scene.bvh;
    int64_t n = export_bvh(bvh, nullptr, 1, bounds, first_child, meta, areas, nullptr);
    if (ordered)
        for (size_t i = 0; i < bvh->orderedPrims.size(); i++) {
            int idx = -1;
            for (size_t k = 0; k < rs->objects.size(); k++)
                if (rs->objects[k] == bvh->orderedPrims[i])
                    idx = (int) k;
            ordered[i] = idx;
        }
    return n;
}

int64_t prr_ref_scene_object_nodes(void *h, int obj, float *bounds, uint32_t *first_child,
                                   uint32_t *meta, float *areas, int32_t *ordered) {
    RefScene *rs = (RefScene *) h;
    if (rs->object_kind.at(obj) != 0)
        return -1;
    MeshTriangle *m = (MeshTriangle *) rs->objects[obj];
    return export_bvh(m->bvh, &m->triangles[0], sizeof(Triangle), bounds, first_child, meta,
                      areas, ordered);
}

float prr_ref_scene_emit_area(void *h) {
    return ((RefScene *) h)->scene.totalEmitArea;
}

// Map an Intersection back to (object index, triangle index in that mesh).
static void locate_hit(const RefScene *rs, const Intersection &in, int32_t *obj, int32_t *prim) {
    *obj = -1;
    *prim = -1;
    for (size_t k = 0; k < rs->objects.size(); k++) {
        if (rs->object_kind[k] == 1) {
            if (in.obj == rs->objects[k]) {
                *obj = (int32_t) k;
                *prim = 0;
                return;
            }
        } else {
            const MeshTriangle *m = (const MeshTriangle *) rs->objects[k];
            const Triangle *b = &m->triangles[0];
            const Triangle *e = b + m->triangles.size();
            const Triangle *t = (const Triangle *) in.obj;
            if (t >= b && t < e) {
                *obj = (int32_t) k;
                *prim = (int32_t) (t - b);
                return;
            }
        }
    }
}

// Scene::intersect (two-level: scene BVH over objects, mesh BVHs below).
// geo[i*6..] = hit coords and normal.
void prr_ref_scene_intersect(void *h, const float *o, const float *d, int64_t n, int32_t *obj,
                             int32_t *prim, float *t, float *geo, int nthreads) {
    RefScene *rs = (RefScene *) h;
    if (nthreads > 0)
        omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < n; i++) {
        Ray ray(Vector3f(o[i * 3], o[i * 3 + 1], o[i * 3 + 2]),
                Vector3f(d[i * 3], d[i * 3 + 1], d[i * 3 + 2]));
        Intersection in = rs->scene.intersect(ray);
        if (in.happened) {
            locate_hit(rs, in, &obj[i], &prim[i]);
            t[i] = (float) in.tnear;
            if (geo) {
                geo[i * 6 + 0] = in.coords.x;
                geo[i * 6 + 1] = in.coords.y;
                geo[i * 6 + 2] = in.coords.z;
                geo[i * 6 + 3] = in.normal.x;
                geo[i * 6 + 4] = in.normal.y;
                geo[i * 6 + 5] = in.normal.z;
            }
        } else {
            obj[i] = -1;
            prim[i] = -1;
            t[i] = std::numeric_limits<float>::infinity();
        }
    }
}

void prr_ref_scene_occluded(void *h, const float *o, const float *d, const float *tmax, int64_t n,
                            uint8_t *hit, int nthreads) {
    RefScene *rs = (RefScene *) h;
    if (nthreads > 0)
        omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < n; i++) {
        Ray ray(Vector3f(o[i * 3], o[i * 3 + 1], o[i * 3 + 2]),
                Vector3f(d[i * 3], d[i * 3 + 1], d[i * 3 + 2]));
        hit[i] = rs->scene.intersectP(ray, tmax[i]) ? 1 : 0;
    }
}

// Scene::sampleLight with stream (seed, i, 0) per sample: coords, normal, pdf.
void prr_ref_scene_sample_light(void *h, uint64_t seed, int64_t n, float *pos, float *nrm,
                                float *pdf) {
    RefScene *rs = (RefScene *) h;
    for (int64_t i = 0; i < n; i++) {
        ref_set_path(seed, (uint32_t) i, 0u);
        Intersection li;
        float p = 0.f;
        rs->scene.sampleLight(li, p);
        pos[i * 3 + 0] = li.coords.x;
        pos[i * 3 + 1] = li.coords.y;
        pos[i * 3 + 2] = li.coords.z;
        nrm[i * 3 + 0] = li.normal.x;
        nrm[i * 3 + 1] = li.normal.y;
        nrm[i * 3 + 2] = li.normal.z;
        pdf[i] = p;
    }
}

// ---------------------------------------------------------------------------
// Rendering: the Renderer.cpp:63-99 per-pixel loop, restated so the linear
// framebuffer is returned. Pixel m = i + j*W draws from stream (seed, m, n)
// for its n-th sample. Window [x0,x1) x [y0,y1); out is (y1-y0)*(x1-x0)*3.
// min_spp == max_spp gives the fixed-spp mode; otherwise the Welford
// confidence-interval stop of Renderer.cpp:88-95 applies.
// ---------------------------------------------------------------------------
void prr_ref_render(void *h, int max_depth, int min_spp, int max_spp, float threshold,
                    uint64_t seed, int x0, int y0, int x1, int y1, float *out_rgb,
                    int32_t *out_spp, int nthreads) {
    RefScene *rs = (RefScene *) h;
    const int W = rs->width, H = rs->height;
    Integrator integrator(rs->scene, max_depth, 0.8f);
    const int ww = x1 - x0, wh = y1 - y0;
    if (nthreads > 0)
        omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t q = 0; q < (int64_t) ww * wh; q++) {
        int i = x0 + (int) (q % ww);
        int j = y0 + (int) (q / ww);
        int m = i + j * W;
        Welford wR, wG, wB;
        Vector3f acc(0.f);
        int n = 0;
        while (n < max_spp) {
            ref_set_path(seed, (uint32_t) m, (uint32_t) n);
            float xOffset = get_random_float();
            float yOffset = get_random_float();
            Ray ray = rs->scene.camera.generateRay(i, j, W, H, xOffset, yOffset);
            Vector3f s = integrator.castRay(ray);
            if (std::isnan(s.x) || std::isnan(s.y) || std::isnan(s.z))
                s = Vector3f(0.f);
            acc += s;
            n++;
            wR.update(s.x);
            wG.update(s.y);
            wB.update(s.z);
            if (n >= min_spp) {
                if (wR.ci() < threshold && wG.ci() < threshold && wB.ci() < threshold)
                    break;
            }
        }
        acc = acc / (float) n;
        out_rgb[q * 3 + 0] = acc.x;
        out_rgb[q * 3 + 1] = acc.y;
        out_rgb[q * 3 + 2] = acc.z;
        if (out_spp)
            out_spp[q] = n;
    }
}

// One path per (pixel, sample) pair: the radiance castRay returns and the
// number of random numbers the path drew (for lockstep checks).
void prr_ref_cast_samples(void *h, int max_depth, uint64_t seed, const int32_t *px,
                          const int32_t *py, const int32_t *sample, int64_t n, float *out_rgb,
                          int32_t *out_draws, int nthreads) {
    RefScene *rs = (RefScene *) h;
    const int W = rs->width, H = rs->height;
    Integrator integrator(rs->scene, max_depth, 0.8f);
    if (nthreads > 0)
        omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t k = 0; k < n; k++) {
        int i = px[k], j = py[k];
        ref_set_path(seed, (uint32_t) (i + j * W), (uint32_t) sample[k]);
        float xOffset = get_random_float();
        float yOffset = get_random_float();
        Ray ray = rs->scene.camera.generateRay(i, j, W, H, xOffset, yOffset);
        Vector3f s = integrator.castRay(ray);
        if (std::isnan(s.x) || std::isnan(s.y) || std::isnan(s.z))
            s = Vector3f(0.f);
        out_rgb[k * 3 + 0] = s.x;
        out_rgb[k * 3 + 1] = s.y;
        out_rgb[k * 3 + 2] = s.z;
        if (out_draws)
            out_draws[k] = (int32_t) g_rng_draws;
    }
}

// Camera::generateRay for (pixel, offsets): origin and direction.
void prr_ref_camera_rays(void *h, const int32_t *px, const int32_t *py, const float *xo,
                         const float *yo, int64_t n, float *o, float *d) {
    RefScene *rs = (RefScene *) h;
    for (int64_t k = 0; k < n; k++) {
        Ray r = rs->scene.camera.generateRay(px[k], py[k], rs->width, rs->height, xo[k], yo[k]);
        o[k * 3 + 0] = r.origin.x;
        o[k * 3 + 1] = r.origin.y;
        o[k * 3 + 2] = r.origin.z;
        d[k * 3 + 0] = r.direction.x;
        d[k * 3 + 1] = r.direction.y;
        d[k * 3 + 2] = r.direction.z;
    }
}

// ---------------------------------------------------------------------------
// Display transform: exposure + sanitise (Renderer.cpp:149-161), operator
// (ToneMapping.hpp:267-279), 8-bit quantise (Renderer.cpp:169-171).
// mapper: 0 Raw, 1 Standard, 2 AgX, 3 PBRNeutral.
// ---------------------------------------------------------------------------
void prr_ref_tonemap(int mapper, float exposure, const float *in_rgb, int64_t n, float *out_rgb,
                     uint8_t *out_u8) {
    for (int64_t i = 0; i < n; i++) {
        Vector3f c = Vector3f(in_rgb[i * 3], in_rgb[i * 3 + 1], in_rgb[i * 3 + 2]) * exposure;
        if (!std::isfinite(c.x))
            c.x = 0.f;
        if (!std::isfinite(c.y))
            c.y = 0.f;
        if (!std::isfinite(c.z))
            c.z = 0.f;
        c.x = std::max(0.f, c.x);
        c.y = std::max(0.f, c.y);
        c.z = std::max(0.f, c.z);
        Vector3f co = tonemap::apply((tonemap::ToneMapper) mapper, c);
        if (out_rgb) {
            out_rgb[i * 3 + 0] = co.x;
            out_rgb[i * 3 + 1] = co.y;
            out_rgb[i * 3 + 2] = co.z;
        }
        if (out_u8) {
            out_u8[i * 3 + 0] = (unsigned char) (std::clamp(co.x, 0.f, 1.f) * 255.f + 0.5f);
            out_u8[i * 3 + 1] = (unsigned char) (std::clamp(co.y, 0.f, 1.f) * 255.f + 0.5f);
            out_u8[i * 3 + 2] = (unsigned char) (std::clamp(co.z, 0.f, 1.f) * 255.f + 0.5f);
        }
    }
}

// ---------------------------------------------------------------------------
// Caustic photons. The emit loop of Photon.cpp:156-188 is restated so photon i
// draws from stream (seed, i, 0xFFFFFFFF); each photon's stored records are
// kept in trace order and concatenated in photon order, so the output order
// is canonical (photon index, then depth). Returns the number of photons
// stored; with out == nullptr only counts. Record layout (11 floats + 2 ints):
// position[3], direction[3], power[3], and in the int arrays photon index and
// the running record index within that photon.
// ---------------------------------------------------------------------------
struct RefPhotons {
    std::vector<Photon> photons;
    std::vector<int32_t> owner;
};

void *prr_ref_photon_emit(void *h, int64_t num_photons, uint64_t seed, int max_depth,
                          int nthreads) {
    RefScene *rs = (RefScene *) h;
    PhotonMap pm;
    pm.maxDepth = max_depth;
    std::vector<std::vector<Photon>> per(num_photons);
    if (nthreads > 0)
        omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 100)
    for (int64_t i = 0; i < num_photons; i++) {
        ref_set_path(seed, (uint32_t) i, 0xFFFFFFFFu);
        Intersection lightPoint;
        float light_pdf;
        rs->scene.sampleLight(lightPoint, light_pdf);
        float area = 1.0f / light_pdf;
        Vector3f dir = sampleCosineHemisphere(lightPoint.normal);
        Vector3f power = lightPoint.material->m_emission * area / num_photons;
        Photon p;
        p.position = lightPoint.coords + lightPoint.normal * EPSILON;
        p.direction = dir;
        p.power = power;
        p.is_caustic = false;
        pm.trace(p, 0, per[i], rs->scene);
    }
    RefPhotons *out = new RefPhotons();
    for (int64_t i = 0; i < num_photons; i++)
        for (auto &p : per[i]) {
            out->photons.push_back(p);
            out->owner.push_back((int32_t) i);
        }
    return out;
}

int64_t prr_ref_photon_export(void *ph, float *rec, int32_t *owner) {
    RefPhotons *p = (RefPhotons *) ph;
    int64_t n = (int64_t) p->photons.size();
    if (rec)
        for (int64_t i = 0; i < n; i++) {
            const Photon &q = p->photons[i];
            float *r = rec + i * 9;
            r[0] = q.position.x;
            r[1] = q.position.y;
            r[2] = q.position.z;
            r[3] = q.direction.x;
            r[4] = q.direction.y;
            r[5] = q.direction.z;
            r[6] = q.power.x;
            r[7] = q.power.y;
            r[8] = q.power.z;
        }
    if (owner)
        std::memcpy(owner, p->owner.data(), sizeof(int32_t) * n);
    return n;
}

void prr_ref_photon_free(void *ph) {
    delete (RefPhotons *) ph;
}

// PhotonGrid::build + PhotonMap::estimateIrradiance on a given photon array
// (rec = n x 9 floats as above), radius r, at nq query points.
void prr_ref_photon_estimate(const float *rec, int64_t n, float radius, const float *q,
                             int64_t nq, float *out_rgb, int32_t *grid_res, int nthreads) {
    PhotonMap pm;
    pm.photon_radius = radius;
    pm.caustic_map.resize(n);
    for (int64_t i = 0; i < n; i++) {
        const float *r = rec + i * 9;
        pm.caustic_map[i].position = Vector3f(r[0], r[1], r[2]);
        pm.caustic_map[i].direction = Vector3f(r[3], r[4], r[5]);
        pm.caustic_map[i].power = Vector3f(r[6], r[7], r[8]);
        pm.caustic_map[i].is_caustic = true;
    }
    pm.build();
    if (grid_res)
        *grid_res = pm.caustic_grid.resolution;
    if (nthreads > 0)
        omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t k = 0; k < nq; k++) {
        Vector3f e = pm.estimateIrradiance(Vector3f(q[k * 3], q[k * 3 + 1], q[k * 3 + 2]),
                                           Vector3f(0, 1, 0));
        out_rgb[k * 3 + 0] = e.x;
        out_rgb[k * 3 + 1] = e.y;
        out_rgb[k * 3 + 2] = e.z;
    }
}

// ---------------------------------------------------------------------------
// k-nearest-capped estimate and the caustic render at camera hits. Neither
// exists in the reference (castRay never gathers photons; estimateIrradiance
// is fixed-radius), so these restate the library's definition with the
// reference's own pieces:
//   candidates   PhotonGrid::query(pos, radius) on a grid built by
//                PhotonGrid::build (Photon.cpp:24-81) from the given array;
//   <= k inside  PhotonMap::estimateIrradiance itself (Photon.cpp:82-94);
//   > k inside   brute force over the candidates: the k smallest
//                (distance, photon index) pairs, distance as the query
//                computes it ((p - x).norm()), their powers added in the
//                order the query returns them (as estimateIrradiance adds),
//                divided by pi r_k^2 written as estimateIrradiance writes
//                pi r^2, r_k the k-th smallest distance.
// The photon index travels in the direction field (unused by the estimate).
// ---------------------------------------------------------------------------
struct KnnMap {
    PhotonMap pm;
    std::vector<Vector3f> power; // in photon order
};

static KnnMap *knn_map_new(const float *rec, int64_t n, float radius) {
    KnnMap *m = new KnnMap();
    m->pm.photon_radius = radius;
    m->pm.caustic_map.resize(n);
    m->power.resize(n);
    for (int64_t i = 0; i < n; i++) {
        const float *r = rec + i * 9;
        m->pm.caustic_map[i].position = Vector3f(r[0], r[1], r[2]);
        m->pm.caustic_map[i].direction = Vector3f((float) i, 0.f, 0.f);
        m->pm.caustic_map[i].power = Vector3f(r[6], r[7], r[8]);
        m->pm.caustic_map[i].is_caustic = true;
        m->power[i] = Vector3f(r[6], r[7], r[8]);
    }
    m->pm.build();
    return m;
}

static Vector3f knn_estimate(const KnnMap &m, const Vector3f &pos, int k, int32_t *inside) {
    thread_local std::vector<const Photon *> near;
    thread_local std::vector<std::pair<float, int32_t>> cand;
    m.pm.caustic_grid.query(pos, m.pm.photon_radius, near);
    if (inside)
        *inside = (int32_t) near.size();
    if (k <= 0 || (int) near.size() <= k)
        return m.pm.estimateIrradiance(pos, Vector3f(0, 1, 0));
    cand.clear();
    for (const Photon *p : near)
        cand.emplace_back((p->position - pos).norm(), (int32_t) p->direction.x);
    std::vector<std::pair<float, int32_t>> sorted(cand);
    std::sort(sorted.begin(), sorted.end());
    const std::pair<float, int32_t> kth = sorted[k - 1];
    const float rk = kth.first;
    Vector3f e = {};
    for (size_t q = 0; q < near.size(); q++)
        if (cand[q] <= kth)
            e += near[q]->power;
    float area = M_PI * rk * rk;
    return e / area;
}

// Irradiance at nq points: fixed radius (k = 0) or capped at the k nearest;
// out_inside (optional) gets the number of photons inside the radius.
void prr_ref_photon_estimate_knn(const float *rec, int64_t n, float radius, int k, const float *q,
                                 int64_t nq, float *out_rgb, int32_t *out_inside, int nthreads) {
    KnnMap *m = knn_map_new(rec, n, radius);
    if (nthreads > 0)
        omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t j = 0; j < nq; j++) {
        const Vector3f e = knn_estimate(*m, Vector3f(q[j * 3], q[j * 3 + 1], q[j * 3 + 2]), k,
                                        out_inside ? out_inside + j : nullptr);
        out_rgb[j * 3 + 0] = e.x;
        out_rgb[j * 3 + 1] = e.y;
        out_rgb[j * 3 + 2] = e.z;
    }
    delete m;
}

// The caustic radiance of a camera sample: the camera ray of Renderer.cpp:75-77
// follows castRay's delta chain (Integrator.cpp:143-169: the material's own
// sample, the pdf cut, beta *= f / pdf, the offset origin, the baseColor tint on
// transmission) for at most max_depth hits; at the first non-delta, non-emissive
// hit the estimate is beta * baseColor / pi * E(hit point), with baseColor from
// the diffuse material's buildShadingData (Material.cpp:3-26). A miss, an
// emitter or the depth limit contributes zero. Pixel m = i + j*W, sample n draws
// stream (seed, m, sample_offset + n); the pixel value is the mean of its spp
// samples added in sample order.
void prr_ref_caustic_render(void *h, const float *rec, int64_t n, float radius, int k,
                            int max_depth, int spp, uint64_t seed, int sample_offset, int x0,
                            int y0, int x1, int y1, float *out_rgb, int nthreads) {
    RefScene *rs = (RefScene *) h;
    const int W = rs->width, H = rs->height;
    KnnMap *m = knn_map_new(rec, n, radius);
    const int ww = x1 - x0, wh = y1 - y0;
    if (nthreads > 0)
        omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t qp = 0; qp < (int64_t) ww * wh; qp++) {
        const int i = x0 + (int) (qp % ww), j = y0 + (int) (qp / ww);
        const int mpix = i + j * W;
        Vector3f acc(0.f);
        for (int s = 0; s < spp; s++) {
            ref_set_path(seed, (uint32_t) mpix, (uint32_t) (sample_offset + s));
            const float xOffset = get_random_float();
            const float yOffset = get_random_float();
            Ray ray = rs->scene.camera.generateRay(i, j, W, H, xOffset, yOffset);
            Vector3f beta(1.f), c(0.f);
            for (int d = 0; d < max_depth; d++) {
                Intersection inter = rs->scene.intersect(ray);
                if (!inter.happened)
                    break;
                Material *mat = inter.material;
                if (mat->isEmissive())
                    break;
                const Vector3f geoNormal = inter.normal;
                if (mat->isDelta()) {
                    ShadingData sd = inter.hasTangent
                                         ? mat->buildShadingData(inter.tcoords, geoNormal,
                                                                 normalize(inter.tangent),
                                                                 inter.tangentHandedness)
                                         : mat->buildShadingData(inter.tcoords, geoNormal);
                    BSDFSample bsdf = mat->sample(-ray.direction, sd);
                    if (bsdf.pdf < 1e-6f)
                        break;
                    beta = beta * bsdf.f / bsdf.pdf;
                    const bool trans = dotProduct(bsdf.wi, geoNormal) < 0.f;
                    const Vector3f offset = trans ? -geoNormal : geoNormal;
                    ray = Ray(inter.coords + offset * EPSILON, bsdf.wi);
                    if (trans)
                        beta = beta * sd.baseColor;
                    continue;
                }
                DiffuseMaterial *dm = static_cast<DiffuseMaterial *>(mat);
                const Vector3f sn = dotProduct(ray.direction, geoNormal) < 0.f ? geoNormal
                                                                              : -geoNormal;
                ShadingData sd = inter.hasTangent
                                     ? dm->buildShadingData(inter.tcoords, sn,
                                                            normalize(inter.tangent),
                                                            inter.tangentHandedness)
                                     : dm->buildShadingData(inter.tcoords, sn);
                const Vector3f e = knn_estimate(*m, inter.coords, k, nullptr);
                c = beta * (sd.baseColor / (float) M_PI) * e;
                break;
            }
            acc += c;
        }
        acc = acc / (float) spp;
        out_rgb[qp * 3 + 0] = acc.x;
        out_rgb[qp * 3 + 1] = acc.y;
        out_rgb[qp * 3 + 2] = acc.z;
    }
    delete m;
}

// ---- participating media (Volume.hpp, Volume.cpp; unused by castRay)

// Medium::dust() (0) or Medium::fog() (1): sigma_a, sigma_s, sigma_t, g.
void prr_ref_medium_preset(int which, float *out) {
    const Medium m = which == 0 ? Medium::dust() : Medium::fog();
    out[0] = m.sigma_a;
    out[1] = m.sigma_s;
    out[2] = m.sigma_t;
    out[3] = m.g;
}

void prr_ref_medium_intersect(int bounded, const float *lo, const float *hi, const float *o,
                              const float *d, int64_t n, float *t_enter, float *t_exit,
                              uint8_t *hit) {
    Medium m;
    m.bounded = bounded != 0;
    m.bounds.pMin = Vector3f(lo[0], lo[1], lo[2]);
    m.bounds.pMax = Vector3f(hi[0], hi[1], hi[2]);
    for (int64_t i = 0; i < n; i++) {
        const Ray r(Vector3f(o[i * 3], o[i * 3 + 1], o[i * 3 + 2]),
                    Vector3f(d[i * 3], d[i * 3 + 1], d[i * 3 + 2]));
        float te = 0.f, tx = 0.f;
        const bool h = m.intersect(r, te, tx);
        hit[i] = h ? 1 : 0;
        t_enter[i] = h ? te : 0.f;
        t_exit[i] = h ? tx : 0.f;
    }
}

void prr_ref_phase_hg(const float *c, int64_t n, float g, float *out) {
    for (int64_t i = 0; i < n; i++)
        out[i] = phaseHG(c[i], g);
}

// samplePhaseHG(wo[i], g), item i drawing from stream (seed, i, 0).
void prr_ref_phase_hg_sample(const float *wo, int64_t n, float g, uint64_t seed, float *out) {
    for (int64_t i = 0; i < n; i++) {
        ref_set_path(seed, (uint32_t) i, 0u);
        const Vector3f w = samplePhaseHG(Vector3f(wo[i * 3], wo[i * 3 + 1], wo[i * 3 + 2]), g);
        out[i * 3] = w.x;
        out[i * 3 + 1] = w.y;
        out[i * 3 + 2] = w.z;
    }
}

} // extern "C"
