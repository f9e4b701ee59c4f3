// Two-level scene traversal as resumable per-lane state machines, for
// persistent kernels whose lanes take new rays as soon as theirs finish.
// Each call to step() does one unit of work -- one interior node, one
// triangle, one sphere, or entering a mesh -- in exactly the order of the
// recursive walks in trace.cuh (scene_closest / scene_occluded, which restate
// BVH.cpp:311-473 over MeshTriangle and Sphere leaves), so results are
// identical; only the scheduling of rays onto lanes changes.
#pragma once
#include "trace.cuh"

namespace prr {

// Closest hit: Scene::intersect -> scene BVH, general path; each mesh leaf is
// searched from +inf on its own (BVH.cpp:359-369).
struct ClosestWalk {
    RayD r;
    RayPre p;
    float closest;
    int hit_obj, hit_tri;
    uint32_t tref;
    int tsp;
    bool in_mesh;
    int cur_obj;
    uint32_t bref, tri, ntri;
    float bbest;
    int bhit;
    int bsp;

    __device__ __forceinline__ void start(const DevScene &S, const RayD &ray) {
        r = ray;
        p = precompute(ray);
        closest = kInf;
        hit_obj = hit_tri = -1;
        tref = S.tlas_root;
        tsp = 0;
        in_mesh = false;
        ntri = 0;
    }

    // pops the scene-level stack; true when the walk is over
    __device__ __forceinline__ bool scene_pop(const StackCol<uint2> &tc) {
        while (tsp > 0) {
            --tsp;
            const uint2 e = tc.get(tsp);
            if (__uint_as_float(e.y) < closest) {
                tref = e.x;
                return false;
            }
        }
        return true;
    }

    __device__ __forceinline__ void set_mesh_ref(uint32_t ref) {
        if (ref & kLeafBit) {
            tri = leaf_first(ref);
            ntri = leaf_count(ref);
        } else {
            bref = ref;
            ntri = 0;
        }
    }

    __device__ __forceinline__ bool step(const DevScene &S, const StackCol<uint2> &tc,
                                         const StackCol<uint2> &bc) {
        if (in_mesh) {
            bool pop = false;
            if (ntri > 0) {
                const TriV T = load_tri(S, tri);
                float t, u, v;
                if (tri_hit(T, r, t, u, v) && t < bbest) {
                    bbest = t;
                    bhit = (int) tri;
                }
                tri++;
                ntri--;
                pop = ntri == 0;
            } else {
                const NodeV n = load_node(S, bref);
                const float tl = slab(n.a.x, n.a.y, n.a.z, n.a.w, n.b.x, n.b.y, p);
                const float tr = slab(n.b.z, n.b.w, n.c.x, n.c.y, n.c.z, n.c.w, p);
                if (tl <= tr) {
                    if (tl < bbest) {
                        if (tr < bbest)
                            bc.put(bsp++, make_uint2(n.link.y, __float_as_uint(tr)));
                        set_mesh_ref(n.link.x);
                        return false;
                    }
                } else {
                    if (tr < bbest) {
                        if (tl < bbest)
                            bc.put(bsp++, make_uint2(n.link.x, __float_as_uint(tl)));
                        set_mesh_ref(n.link.y);
                        return false;
                    }
                }
                pop = true;
            }
            if (!pop)
                return false;
            while (bsp > 0) {
                --bsp;
                const uint2 e = bc.get(bsp);
                if (__uint_as_float(e.y) < bbest) {
                    set_mesh_ref(e.x);
                    return false;
                }
            }
            // mesh finished: MeshTriangle::getIntersection's answer
            if (bhit >= 0 && bbest < closest) {
                closest = bbest;
                hit_obj = cur_obj;
                hit_tri = bhit;
            }
            in_mesh = false;
            return scene_pop(tc);
        }
        if (!(tref & kLeafBit)) {
            const NodeV n = load_node(S, tref);
            const float tl = slab(n.a.x, n.a.y, n.a.z, n.a.w, n.b.x, n.b.y, p);
            const float tr = slab(n.b.z, n.b.w, n.c.x, n.c.y, n.c.z, n.c.w, p);
            if (tl <= tr) {
                if (tl < closest) {
                    if (tr < closest)
                        tc.put(tsp++, make_uint2(n.link.y, __float_as_uint(tr)));
                    tref = n.link.x;
                    return false;
                }
            } else {
                if (tr < closest) {
                    if (tl < closest)
                        tc.put(tsp++, make_uint2(n.link.x, __float_as_uint(tl)));
                    tref = n.link.y;
                    return false;
                }
            }
            return scene_pop(tc);
        }
        const int k = (int) (tref & ~kLeafBit);
        const DevObject &o = S.objects[k];
        if (o.kind == kObjMesh) {
            in_mesh = true;
            cur_obj = k;
            bbest = kInf;
            bhit = -1;
            bsp = 0;
            set_mesh_ref(o.root);
            return false;
        }
        float t;
        if (sphere_hit(o, r, t) && t < closest) {
            closest = t;
            hit_obj = k;
            hit_tri = -1;
        }
        return scene_pop(tc);
    }
};

// Any hit: Scene::intersectP -> scene BVH IntersectP over MeshTriangle /
// Sphere intersectT (BVH.cpp:421-473, Triangle.hpp:141-147, Object.hpp:24-29).
struct AnyWalk {
    RayD r;
    RayPair p;
    float tmax;
    uint32_t tref;
    int tsp;
    bool in_mesh;
    uint32_t bref, tri, ntri;
    int bsp;
    bool occluded;

    // false when the scene's root box already misses
    __device__ __forceinline__ bool start(const DevScene &S, const RayD &ray, float t_max) {
        r = ray;
        p = precompute_pair(ray);
        tmax = t_max;
        tref = S.tlas_root;
        tsp = 0;
        in_mesh = false;
        ntri = 0;
        occluded = false;
        return S.n_objects > 0 && slab6(S.tlas_box, p) < tmax;
    }

    __device__ __forceinline__ void set_mesh_ref(uint32_t ref) {
        if (ref & kLeafBit) {
            tri = leaf_first(ref);
            ntri = leaf_count(ref);
        } else {
            bref = ref;
            ntri = 0;
        }
    }

    __device__ __forceinline__ bool scene_pop(const StackCol<uint32_t> &tc) {
        if (tsp == 0)
            return true;
        --tsp;
        tref = tc.get(tsp);
        return false;
    }

    // one unit of work; true when the walk is over (result in `occluded`)
    __device__ __forceinline__ bool step(const DevScene &S, const StackCol<uint32_t> &tc,
                                         const StackCol<uint32_t> &bc) {
        if (in_mesh) {
            if (ntri > 0) {
                const TriV T = load_tri(S, tri);
                if (tri_occludes(T, r, tmax)) {
                    // MeshTriangle::intersectT answers 1e-3; the scene-level
                    // caller then needs 1e-3 < tMax
                    in_mesh = false;
                    if (1e-3f < tmax) {
                        occluded = true;
                        return true;
                    }
                    return scene_pop(tc);
                }
                tri++;
                ntri--;
                if (ntri > 0)
                    return false;
            } else {
                const NodeV n = load_node(S, bref);
                const float tl = slab(n.a.x, n.a.y, n.a.z, n.a.w, n.b.x, n.b.y, p);
                const float tr = slab(n.b.z, n.b.w, n.c.x, n.c.y, n.c.z, n.c.w, p);
                const uint32_t axis = n.link.z;
                const bool neg = axis == 0 ? p.nx : (axis == 1 ? p.ny : p.nz);
                const uint32_t near_ref = neg ? n.link.y : n.link.x;
                const uint32_t far_ref = neg ? n.link.x : n.link.y;
                const float tnear = neg ? tr : tl;
                const float tfar = neg ? tl : tr;
                if (tfar < tmax)
                    bc.put(bsp++, far_ref);
                if (tnear < tmax) {
                    set_mesh_ref(near_ref);
                    return false;
                }
            }
            if (bsp > 0) {
                --bsp;
                set_mesh_ref(bc.get(bsp));
                return false;
            }
            in_mesh = false;
            return scene_pop(tc);
        }
        if (!(tref & kLeafBit)) {
            const NodeV n = load_node(S, tref);
            const float tl = slab(n.a.x, n.a.y, n.a.z, n.a.w, n.b.x, n.b.y, p);
            const float tr = slab(n.b.z, n.b.w, n.c.x, n.c.y, n.c.z, n.c.w, p);
            const uint32_t axis = n.link.z;
            const bool neg = axis == 0 ? p.nx : (axis == 1 ? p.ny : p.nz);
            const uint32_t near_ref = neg ? n.link.y : n.link.x;
            const uint32_t far_ref = neg ? n.link.x : n.link.y;
            const float tnear = neg ? tr : tl;
            const float tfar = neg ? tl : tr;
            if (tfar < tmax)
                tc.put(tsp++, far_ref);
            if (tnear < tmax) {
                tref = near_ref;
                return false;
            }
            return scene_pop(tc);
        }
        const DevObject &o = S.objects[tref & ~kLeafBit];
        if (o.kind == kObjMesh) {
            // the mesh's own IntersectP first tests its root box
            if (slab6(o.root_box, p) < tmax) {
                in_mesh = true;
                bsp = 0;
                set_mesh_ref(o.root);
                return false;
            }
            return scene_pop(tc);
        }
        float t;
        if (sphere_hit(o, r, t) && t < tmax && t >= 0.f) {
            occluded = true;
            return true;
        }
        return scene_pop(tc);
    }
};

} // namespace prr
