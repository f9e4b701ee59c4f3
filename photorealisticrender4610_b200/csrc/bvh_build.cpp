// Host SAH builder. Restates BVHAccel::recursiveBuild / flatten
// (BVH.cpp:66-280) operation for operation so the tree is the reference's:
//   - per node: bounds and centroid bounds of its prims (BVH.cpp:77-86)
//   - leaf at 1 prim, or at count <= maxPrimsInNode (BVH.cpp:89-109)
//   - split axis = longest centroid extent (BVH.cpp:112-113)
//   - degenerate centroids: median split, order untouched (BVH.cpp:118-131)
//   - count > 4: 12-bucket binned SAH over all 3 axes, cost
//     1 + (nL*AL + nR*AR)/AP in float, first strict minimum wins; stable
//     partition at lo + (best+1)*span/12 (BVH.cpp:131-241)
//   - count <= 4: std::nth_element at the median (BVH.cpp:241-250), restated
//     from libstdc++'s introselect for the 2..4 elements that reach it
//   - depth-first, left-first flatten; interior first_child = right child
// Subtrees are independent once their prim range is fixed, so large ranges
// are built on separate threads. Every subtree over prims [s, e) owns node
// slots [slot, slot + 2(e-s) - 1), which makes the slot of every node a pure
// function of the tree; flatten then renumbers depth-first exactly as the
// reference does.
#include "bvh_build.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <thread>

namespace prr {
namespace {

// std::min / std::max exactly as libstdc++ defines them.
inline float smin(float a, float b) { return (b < a) ? b : a; }
inline float smax(float a, float b) { return (a < b) ? b : a; }

struct Box {
    float mn[3], mx[3];
};

inline Box empty_box() {
    // Bounds3() stores +-DBL_MAX narrowed to float, i.e. +-inf (Bounds3.hpp:15-20).
    const float inf = std::numeric_limits<float>::infinity();
    return Box{{inf, inf, inf}, {-inf, -inf, -inf}};
}
inline void grow(Box &a, const Box &b) {
    for (int k = 0; k < 3; k++) {
        a.mn[k] = smin(a.mn[k], b.mn[k]);
        a.mx[k] = smax(a.mx[k], b.mx[k]);
    }
}
inline void grow_pt(Box &a, const float *p) {
    for (int k = 0; k < 3; k++) {
        a.mn[k] = smin(a.mn[k], p[k]);
        a.mx[k] = smax(a.mx[k], p[k]);
    }
}
// Bounds3::SurfaceArea evaluates in float (Bounds3.hpp:43-47).
inline float surface_area(const Box &b) {
    float dx = b.mx[0] - b.mn[0], dy = b.mx[1] - b.mn[1], dz = b.mx[2] - b.mn[2];
    return 2 * (dx * dy + dx * dz + dy * dz);
}
inline int max_extent(const Box &b) {
    float dx = b.mx[0] - b.mn[0], dy = b.mx[1] - b.mn[1], dz = b.mx[2] - b.mn[2];
    if (dx > dy && dx > dz)
        return 0;
    if (dy > dz)
        return 1;
    return 2;
}

struct Slot {
    Box box;
    int64_t child[2];
    int axis;
    int64_t off, cnt;
    float area;
};

struct Builder {
    const PrimBox *prims;
    const float *areas;
    int max_prims;
    std::vector<int32_t> work;
    std::vector<float> cent; // 3 per prim, precomputed Bounds3::Centroid
    std::vector<Slot> slots;
    std::vector<int32_t> tmp;

    float key(int32_t p, int axis) const { return cent[(size_t) p * 3 + axis]; }

    // libstdc++ nth_element for 2..4 elements: one median-of-three Hoare step
    // when there are 4, then insertion sort.
    void nth_small(int32_t *first, int32_t *nth, int32_t *last, int axis) {
        auto less = [&](int32_t a, int32_t b) { return key(a, axis) < key(b, axis); };
        if (first == last || nth == last)
            return;
        while (last - first > 3) {
            int32_t *mid = first + (last - first) / 2;
            int32_t *a = first + 1, *b = mid, *c = last - 1;
            if (less(*a, *b)) {
                if (less(*b, *c))
                    std::swap(*first, *b);
                else if (less(*a, *c))
                    std::swap(*first, *c);
                else
                    std::swap(*first, *a);
            } else if (less(*a, *c))
                std::swap(*first, *a);
            else if (less(*b, *c))
                std::swap(*first, *c);
            else
                std::swap(*first, *b);
            int32_t *lo = first + 1, *hi = last;
            for (;;) {
                while (less(*lo, *first))
                    ++lo;
                --hi;
                while (less(*first, *hi))
                    --hi;
                if (!(lo < hi))
                    break;
                std::swap(*lo, *hi);
                ++lo;
            }
            if (lo <= nth)
                first = lo;
            else
                last = lo;
        }
        for (int32_t *i = first + 1; i < last; ++i) {
            int32_t val = *i;
            if (less(val, *first)) {
                std::memmove(first + 1, first, (size_t) (i - first) * sizeof(int32_t));
                *first = val;
            } else {
                int32_t *j = i;
                while (less(val, *(j - 1))) {
                    *j = *(j - 1);
                    --j;
                }
                *j = val;
            }
        }
    }

    void build(int64_t start, int64_t end, int64_t slot, int spawn_depth) {
        Slot &node = slots[slot];
        node.child[0] = node.child[1] = -1;
        node.axis = 0;
        node.off = node.cnt = 0;
        const int64_t count = end - start;

        Box bounds = empty_box(), cb = empty_box();
        for (int64_t i = start; i < end; i++) {
            const PrimBox &pb = prims[work[i]];
            Box b{{pb.mn[0], pb.mn[1], pb.mn[2]}, {pb.mx[0], pb.mx[1], pb.mx[2]}};
            grow(bounds, b);
            grow_pt(cb, &cent[(size_t) work[i] * 3]);
        }
        node.box = bounds;

        if (count == 1) {
            node.off = start;
            node.cnt = 1;
            node.area = areas[work[start]];
            return;
        }
        if (count <= max_prims) {
            node.off = start;
            node.cnt = count;
            node.area = 0.f;
            for (int64_t i = start; i < end; i++)
                node.area += areas[work[i]];
            return;
        }

        const int axis = max_extent(cb);
        node.axis = axis;
        int64_t mid = (start + end) / 2;

        if (cb.mx[axis] == cb.mn[axis]) {
            // all centroids coincide on the longest axis: median split
        } else if (count > 4) {
            constexpr int NB = 12;
            float best_cost = std::numeric_limits<float>::infinity();
            int best_axis = axis, best_split = NB / 2;
            const float parent_area = surface_area(bounds);
            for (int a = 0; a < 3; a++) {
                const float lo = cb.mn[a], hi = cb.mx[a];
                if (lo == hi)
                    continue;
                int bc[NB] = {0};
                Box bb[NB];
                for (int k = 0; k < NB; k++)
                    bb[k] = empty_box();
                const float span = hi - lo;
                for (int64_t i = start; i < end; i++) {
                    const int32_t p = work[i];
                    int b = (int) (NB * (key(p, a) - lo) / span);
                    b = std::clamp(b, 0, NB - 1);
                    bc[b]++;
                    const PrimBox &pb = prims[p];
                    Box pbx{{pb.mn[0], pb.mn[1], pb.mn[2]}, {pb.mx[0], pb.mx[1], pb.mx[2]}};
                    grow(bb[b], pbx);
                }
                float la[NB - 1], ra[NB - 1];
                int lc[NB - 1], rc[NB - 1];
                Box acc = empty_box();
                int n = 0;
                for (int k = 0; k < NB - 1; k++) {
                    grow(acc, bb[k]);
                    n += bc[k];
                    la[k] = surface_area(acc);
                    lc[k] = n;
                }
                acc = empty_box();
                n = 0;
                for (int k = NB - 2; k >= 0; k--) {
                    grow(acc, bb[k + 1]);
                    n += bc[k + 1];
                    ra[k] = surface_area(acc);
                    rc[k] = n;
                }
                for (int k = 0; k < NB - 1; k++) {
                    if (lc[k] == 0 || rc[k] == 0)
                        continue;
                    float cost = 1.f + (lc[k] * la[k] + rc[k] * ra[k]) / parent_area;
                    if (cost < best_cost) {
                        best_cost = cost;
                        best_axis = a;
                        best_split = k;
                    }
                }
            }
            const float lo = cb.mn[best_axis];
            const float span = cb.mx[best_axis] - lo;
            const float edge = lo + (best_split + 1) * span / NB;
            int64_t nl = 0;
            for (int64_t i = start; i < end; i++)
                nl += key(work[i], best_axis) < edge;
            if (nl > 0 && nl < count) {
                int64_t wl = start, wr = start + nl;
                for (int64_t i = start; i < end; i++) {
                    const int32_t p = work[i];
                    if (key(p, best_axis) < edge)
                        tmp[wl++] = p;
                    else
                        tmp[wr++] = p;
                }
                std::memcpy(&work[start], &tmp[start], sizeof(int32_t) * count);
                mid = start + nl;
            }
        } else {
            nth_small(&work[start], &work[mid], &work[end], axis);
        }

        const int64_t ls = slot + 1, rs = slot + 2 * (mid - start);
        if (spawn_depth > 0 && count > 16384) {
            std::thread t([&, start, mid, ls, spawn_depth] { build(start, mid, ls, spawn_depth - 1); });
            build(mid, end, rs, spawn_depth - 1);
            t.join();
        } else {
            build(start, mid, ls, 0);
            build(mid, end, rs, 0);
        }
        Slot &n2 = slots[slot];
        n2.child[0] = ls;
        n2.child[1] = rs;
        n2.area = slots[ls].area + slots[rs].area;
    }
};

struct Flattener {
    const Builder &B;
    FlatBVH &out;
    uint32_t flatten(int64_t slot, uint32_t &offset, int depth) {
        const Slot &s = B.slots[slot];
        const uint32_t my = offset++;
        out.max_depth = std::max(out.max_depth, depth);
        float *b = &out.bounds[(size_t) my * 6];
        b[0] = s.box.mn[0];
        b[1] = s.box.mx[0];
        b[2] = s.box.mn[1];
        b[3] = s.box.mx[1];
        b[4] = s.box.mn[2];
        b[5] = s.box.mx[2];
        out.area[my] = s.area;
        if (s.cnt > 0) {
            out.first_child[my] = (uint32_t) s.off;
            out.meta[my] = (uint32_t) s.cnt & 0x00FFFFFFu;
        } else {
            out.meta[my] = (uint32_t) s.axis << 24;
            flatten(s.child[0], offset, depth + 1);
            out.first_child[my] = flatten(s.child[1], offset, depth + 1);
        }
        return my;
    }
};

} // namespace

FlatBVH build_sah(const std::vector<PrimBox> &prims, const std::vector<float> &areas,
                  int max_prims, int threads) {
    FlatBVH out;
    const int64_t n = (int64_t) prims.size();
    if (n == 0)
        return out;
    Builder B;
    B.prims = prims.data();
    B.areas = areas.data();
    B.max_prims = std::min(255, max_prims);
    B.work.resize(n);
    for (int64_t i = 0; i < n; i++)
        B.work[i] = (int32_t) i;
    B.cent.resize((size_t) n * 3);
    for (int64_t i = 0; i < n; i++)
        for (int k = 0; k < 3; k++)
            B.cent[(size_t) i * 3 + k] = prims[i].mn[k] * 0.5f + prims[i].mx[k] * 0.5f;
    B.slots.resize((size_t) 2 * n);
    B.tmp.resize(n);
    if (threads <= 0)
        threads = (int) std::max(1u, std::thread::hardware_concurrency());
    int spawn = 0;
    while ((1 << spawn) < threads * 4 && spawn < 12)
        spawn++;
    B.build(0, n, 0, threads > 1 ? spawn : 0);

    // count reachable nodes, then flatten depth-first
    size_t nodes = 0;
    {
        std::vector<int64_t> st{0};
        while (!st.empty()) {
            int64_t s = st.back();
            st.pop_back();
            nodes++;
            if (B.slots[s].cnt == 0) {
                st.push_back(B.slots[s].child[0]);
                st.push_back(B.slots[s].child[1]);
            }
        }
    }
    out.bounds.resize(nodes * 6);
    out.first_child.resize(nodes);
    out.meta.resize(nodes);
    out.area.resize(nodes);
    uint32_t off = 0;
    Flattener F{B, out};
    F.flatten(0, off, 0);
    out.ordered = std::move(B.work);
    out.total_area = out.area[0];
    return out;
}

void triangle_prims(const float *v, int64_t n, std::vector<PrimBox> &prims,
                    std::vector<float> &areas) {
    prims.resize(n);
    areas.resize(n);
    for (int64_t i = 0; i < n; i++) {
        const float *p = v + i * 9;
        PrimBox &b = prims[i];
        for (int k = 0; k < 3; k++) {
            // Union(Bounds3(v0, v1), v2): fmin/fmax then std::min/max
            b.mn[k] = smin(std::fmin(p[k], p[3 + k]), p[6 + k]);
            b.mx[k] = smax(std::fmax(p[k], p[3 + k]), p[6 + k]);
        }
        float e1x = p[3] - p[0], e1y = p[4] - p[1], e1z = p[5] - p[2];
        float e2x = p[6] - p[0], e2y = p[7] - p[1], e2z = p[8] - p[2];
        float cx = e1y * e2z - e1z * e2y, cy = e1z * e2x - e1x * e2z, cz = e1x * e2y - e1y * e2x;
        areas[i] = std::sqrt(cx * cx + cy * cy + cz * cz) * 0.5f;
    }
}

} // namespace prr

extern "C" int64_t prr_bvh_build(const float *prim_bounds, const float *prim_areas, int64_t n,
                                 int max_prims_in_node, float *bounds, uint32_t *first_child,
                                 uint32_t *meta, float *areas, int32_t *ordered,
                                 int32_t *max_depth) {
    if (n < 0 || (n > 0 && (!prim_bounds || !prim_areas)) || max_prims_in_node < 1)
        return -1;
    std::vector<prr::PrimBox> pb((size_t) n);
    for (int64_t i = 0; i < n; i++)
        for (int k = 0; k < 3; k++) {
            pb[i].mn[k] = prim_bounds[i * 6 + k];
            pb[i].mx[k] = prim_bounds[i * 6 + 3 + k];
        }
    std::vector<float> pa(prim_areas, prim_areas + n);
    prr::FlatBVH f = prr::build_sah(pb, pa, max_prims_in_node, 0);
    const size_t nn = f.size();
    if (bounds)
        std::memcpy(bounds, f.bounds.data(), nn * 6 * sizeof(float));
    if (first_child)
        std::memcpy(first_child, f.first_child.data(), nn * sizeof(uint32_t));
    if (meta)
        std::memcpy(meta, f.meta.data(), nn * sizeof(uint32_t));
    if (areas)
        std::memcpy(areas, f.area.data(), nn * sizeof(float));
    if (ordered)
        std::memcpy(ordered, f.ordered.data(), f.ordered.size() * sizeof(int32_t));
    if (max_depth)
        *max_depth = f.max_depth;
    return (int64_t) nn;
}
