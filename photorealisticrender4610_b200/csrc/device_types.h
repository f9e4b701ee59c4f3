// Device-resident scene layout shared by the host builder and the kernels.
//
// BVH nodes. The reference flattens its SAH tree into 32-byte nodes and, at
// every interior step, reads both children from two unrelated addresses
// (left = idx+1, right = first_child; BVH.cpp:263-280, :370-373). Here each
// interior node of that same tree becomes one 64-byte record holding the two
// CHILD boxes, so one interior step is one aligned 64-byte fetch (two 32-byte
// sectors) instead of two scattered 32-byte ones. Leaves need no record: a
// child reference with the top bit set points straight at the leaf's first
// triangle and carries the leaf's primitive count.
//
// The slab test reads the same float bounds and does the same operations in
// the same order as BVHAccel::nodeIntersect (BVH.hpp:115-124), so entry
// distances, traversal order and tie-breaks are those of the reference tree.
#pragma once
#include <cstdint>

#ifdef __CUDACC__
#define PRR_HD __host__ __device__
#else
#define PRR_HD
#endif

namespace prr {

constexpr uint32_t kLeafBit = 0x80000000u;

// Mesh-BVH leaf references carry their primitive count: a mesh BVH is built
// with maxPrimsInNode 4 (Triangle.hpp:173-179), so count-1 fits in the low two
// bits and the first triangle in the 29 above. Scene-BVH leaves hold exactly
// one object (maxPrimsInNode 1, Scene.cpp:17) and store its index directly.
constexpr int64_t kMaxTriangles = int64_t(1) << 29;
PRR_HD inline uint32_t mesh_leaf_ref(uint32_t first, uint32_t count) {
    return kLeafBit | (first << 2) | (count - 1u);
}
PRR_HD inline uint32_t leaf_first(uint32_t ref) { return (ref & ~kLeafBit) >> 2; }
PRR_HD inline uint32_t leaf_count(uint32_t ref) { return (ref & 3u) + 1u; }

// One interior node: boxes of its left (reference idx+1) and right
// (reference first_child) children, interleaved [minX,maxX,minY,maxY,minZ,maxZ]
// like BVHNode::bounds, plus the child references.
struct alignas(64) WNode {
    float lb[6];        // left child bounds
    float rb[6];        // right child bounds
    uint32_t left;      // interior: WNode index; leaf: mesh_leaf_ref / kLeafBit | object
    uint32_t right;
    uint32_t axis;      // split axis of this node (IntersectP near-child choice, BVH.cpp:384-391)
    float left_area;    // nodeAreas[idx+1] (light-sampling descent, BVH.cpp:488-496)
};
static_assert(sizeof(WNode) == 64, "WNode must be 64 bytes");

// One triangle in leaf order (orderedPrims order): v0, e1 = v1-v0, e2 = v2-v0
// exactly as Triangle's constructor computes them (Triangle.hpp:27-31). The
// intersection test reads 36 bytes: the first eight floats as one 32-byte
// record (one memory sector), e2.z from a parallel float array (a sector there
// covers eight neighbouring triangles, so a leaf's four usually share one).
// The input id and the area live in a third array (TriMeta), read once per
// hit or only by light sampling.
struct alignas(32) Tri {
    float v0x, v0y, v0z, e1x;
    float e1y, e1z, e2x, e2y;
};
static_assert(sizeof(Tri) == 32, "Tri must be 32 bytes");

struct TriMeta {
    int32_t id;         // index of the triangle in its mesh's input order
    float area;         // Triangle::area (Triangle.hpp:31)
};

enum ObjectKind : int32_t { kObjMesh = 0, kObjSphere = 1 };
enum MaterialKind : int32_t { kMatDiffuse = 0, kMatEmissive = 1, kMatMirror = 2, kMatGlass = 3 };

// Scene-level primitive (an entry of Scene::objects).
struct alignas(16) DevObject {
    int32_t kind;
    int32_t material;
    uint32_t root;      // mesh: root reference into nodes/tris
    int32_t tri_base;   // mesh: first triangle (global index)
    float root_box[6];  // own bounds (IntersectP tests the root box first)
    float area;         // MeshTriangle::area or Sphere::area
    float bvh_area;     // mesh: BVHAccel::totalArea (root->area)
    float cx, cy, cz, radius, radius2;
    int32_t ntri;
    int32_t depth;      // max leaf depth of the mesh BVH (stack bound)
    int32_t attr;       // mesh: kAttr* bits of the per-corner data it carries
    int32_t attr_base;  // mesh: its first record in DevScene::attr
    int32_t pad[2];
};

// Per-corner mesh data of Triangle (Triangle.hpp:17-23), one record of
// kAttrFloats floats per triangle of an attributed mesh, leaf order:
// n0 n1 n2 (normalized), t0 t1 t2, tan0 tan1 tan2, w0 w1 w2, pad.
enum : int32_t { kAttrNormals = 1, kAttrUV = 2, kAttrTangents = 4 };
constexpr int kAttrFloats = 28;

// A material texture (TextureUtils.hpp:9-18): 8-bit texels, row-major.
struct DevTexture {
    const uint8_t *data;
    int32_t width, height, channels, pad;
};

struct alignas(16) DevMaterial {
    int32_t kind;
    float base[3];
    float roughness, metallic, ior;
    float emission[3];
    int32_t has_emission; // Material::hasEmission: |m_emission| > EPSILON
    // textures (index into DevScene::textures, -1 none): baseColorTex,
    // metallicRoughnessTex, normalTex, emissiveTex (Material.hpp:45-48)
    int32_t tex_base, tex_mr, tex_normal, tex_emissive;
};

struct DevCamera {
    float eye[3], forward[3], right[3], up[3];
    float focal_px;     // (W*0.5) / tan(halfFovH) (Camera.hpp:76)
    float aperture, focus_distance;
    int32_t width, height;
};

struct DevEnv {
    const float4 *pixels; // rgb + pad, row-major
    const float *cdf;     // width*height conditional CDFs
    const float *marginal;// height
    // guide tables of the CDF searches: (height + 1) rows of guide_n + 1
    // indices, the marginal's first; entry k of a table = lower_bound(cdf, k /
    // guide_n); a table whose first entry is -1 is searched whole (its CDF is
    // not non-decreasing). guide_n = 0: no tables.
    const int32_t *guide;
    int32_t guide_n;
    int32_t width, height;
    float total;          // totalLuminance
    int32_t loaded;
};

struct DevScene {
    const WNode *nodes;
    const Tri *tris;
    const float *tri_e2z;      // e2.z of each triangle (completes Tri)
    const TriMeta *tri_meta;   // input id and area of each triangle
    const float *verts;   // original v0,v1,v2 per triangle, leaf order (sampling, fp64 re-solve)
    const float *normals; // Triangle::normal per triangle, leaf order
    const DevObject *objects;
    const DevMaterial *materials;
    const float *attr;            // per-corner records of attributed meshes
    const DevTexture *textures;
    int32_t n_textures;
    const int32_t *emissives; // Scene::emissives, in object order
    int32_t n_objects, n_materials, n_emissives;
    int32_t has_emissive_kind; // some material is of the emissive kind (hit-emission MIS
                               // then needs the previous hit point)
    float total_emit_area;
    uint32_t tlas_root;
    float tlas_box[6];
    int32_t tlas_depth;
    int32_t blas_depth;   // max over meshes
    float background[3];
    DevCamera camera;
    DevEnv env;
    // bounds of the node and triangle arrays and the scene's status words,
    // read only by the checked build (compiled with -DPRR_CHECKED)
    uint32_t n_nodes, n_tris;
    uint32_t *check;
};

} // namespace prr
