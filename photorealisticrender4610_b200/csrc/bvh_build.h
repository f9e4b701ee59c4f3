// Host SAH builder: restates BVHAccel's construction (BVH.cpp:13-280) so the
// tree, its flattened node order and its primitive order are identical to the
// reference's, then hands the result to the device-layout packer.
#pragma once
#include <cstdint>
#include <vector>

namespace prr {

struct PrimBox {
    float mn[3], mx[3];
};

// The reference's flattened tree (BVHNode array + nodeAreas + orderedPrims).
struct FlatBVH {
    std::vector<float> bounds;          // 6 per node: minX,maxX,minY,maxY,minZ,maxZ
    std::vector<uint32_t> first_child;  // leaf: prim offset; interior: right child index
    std::vector<uint32_t> meta;         // [31:24] split axis, [23:0] prim count
    std::vector<float> area;            // nodeAreas
    std::vector<int32_t> ordered;       // orderedPrims as input indices
    int max_depth = 0;                  // deepest node (root = 0)
    float total_area = 0.f;             // root->area
    size_t size() const { return meta.size(); }
};

// prims[i]: getBounds() of primitive i; areas[i]: getArea(). max_prims is
// clamped to 255 like the reference (BVH.cpp:14). threads <= 0 -> hardware.
FlatBVH build_sah(const std::vector<PrimBox> &prims, const std::vector<float> &areas,
                  int max_prims, int threads = 0);

// Triangle::getBounds (Triangle.hpp:183-185) and Triangle::area
// (Triangle.hpp:27-31) for a triangle soup of n x 9 floats.
void triangle_prims(const float *verts, int64_t n, std::vector<PrimBox> &prims,
                    std::vector<float> &areas);

} // namespace prr
