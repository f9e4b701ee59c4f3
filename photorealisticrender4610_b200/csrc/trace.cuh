// Device ray traversal: the reference's closest-hit and any-hit BVH walks
// (BVH.cpp:311-473) with Möller-Trumbore (Triangle.hpp:46-92) and the
// analytic sphere (Sphere.hpp:22-44), over the 64-byte child-pair nodes of
// device_types.h.
//
// Bit-exactness. Everything here is compiled with --fmad=false and IEEE
// division/sqrt, and every expression keeps the reference's operation order,
// so each slab distance, determinant and t is the float the reference's
// IEEE build computes. The traversal order (near child first on
// tLeft <= tRight, cull on tBox < closestT at push and at pop) is the
// reference's, so ties resolve to the same triangle.
//
// Stacks live in shared memory, one column per thread ([depth][block]
// layout), so a warp's pushes and pops hit distinct banks.
//
// Checked build (-DPRR_CHECKED): every node and triangle fetch is tested
// against the array's length and every stack push against the column's
// depth. A failed test records an error code (first one wins), the offending
// value and a count in the scene's status words and keeps the access in
// bounds (an out-of-range node reads as two empty boxes, a triangle as a
// degenerate one that never hits, an overflowing push is dropped), so the
// kernel runs to its end and the host reads the status (prr_check_status).
// Nothing traps and nothing waits. In the normal build the tests compile to
// nothing.
#pragma once
#include <cuda_runtime.h>

#include "device_types.h"

namespace prr {

#define kInf (__int_as_float(0x7f800000))

// Error codes of the checked build's status words.
enum : uint32_t { kCheckNode = 1, kCheckTri = 2, kCheckStack = 3, kCheckQueue = 4 };

// status[0] = first error code, status[1] = its value, status[2] = errors seen
__device__ __forceinline__ void check_fail(uint32_t *status, uint32_t code, uint32_t value) {
    if (!status)
        return;
    if (atomicCAS(status, 0u, code) == 0u)
        atomicExch(status + 1, value);
    atomicAdd(status + 2, 1u);
}

// What a checked fetch tests against.
struct TraceBounds {
    uint32_t n_nodes, n_tris;
    uint32_t *check;
};

__device__ __forceinline__ TraceBounds bounds_of(const DevScene &S) {
    return TraceBounds{S.n_nodes, S.n_tris, S.check};
}

struct RayD {
    float ox, oy, oz;
    float dx, dy, dz;
};

// BVHAccel::precompute (BVH.cpp:290-299)
struct RayPre {
    float ox, oy, oz;
    float ix, iy, iz;
    bool nx, ny, nz; // octant: direction negative on that axis
};

__device__ __forceinline__ RayPre precompute(const RayD &r) {
    RayPre p;
    p.ox = r.ox;
    p.oy = r.oy;
    p.oz = r.oz;
    p.ix = (r.dx != 0.f) ? (1.f / r.dx) : kInf;
    p.iy = (r.dy != 0.f) ? (1.f / r.dy) : kInf;
    p.iz = (r.dz != 0.f) ? (1.f / r.dz) : kInf;
    p.nx = r.dx < 0.f;
    p.ny = r.dy < 0.f;
    p.nz = r.dz < 0.f;
    return p;
}

// Three-input max and min (sm_100's max.f32 / min.f32 with three sources).
// Like fmaxf/fminf they ignore a NaN input (the result is the max or min of
// the others), so fmax3(a, b, c) == fmaxf(fmaxf(a, b), c) and likewise for
// fmin3, in one instruction instead of two.
__device__ __forceinline__ float fmax3(float a, float b, float c) {
    float d;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}

__device__ __forceinline__ float fmin3(float a, float b, float c) {
    float d;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}

// BVHAccel::nodeIntersect (BVH.hpp:115-124) on bounds
// [minX,maxX,minY,maxY,minZ,maxZ]. The reference folds the three axes into
// tMin = 0 and tMax = +inf one at a time with std::max(tMin, t0) and
// std::min(tMax, t1); fmaxf/fminf agree with those for every input, NaN
// included (the running bound is never NaN, and both return it when the new
// term is NaN), and so do the three-input forms over the same terms.
__device__ __forceinline__ float slab(float x0, float x1, float y0, float y1, float z0, float z1,
                                      const RayPre &p) {
    const float t0x = ((p.nx ? x1 : x0) - p.ox) * p.ix;
    const float t1x = ((p.nx ? x0 : x1) - p.ox) * p.ix;
    const float t0y = ((p.ny ? y1 : y0) - p.oy) * p.iy;
    const float t1y = ((p.ny ? y0 : y1) - p.oy) * p.iy;
    const float t0z = ((p.nz ? z1 : z0) - p.oz) * p.iz;
    const float t1z = ((p.nz ? z0 : z1) - p.oz) * p.iz;
    const float tmin = fmax3(fmaxf(0.f, t0x), t0y, t0z);
    const float tmax = fmin3(fminf(kInf, t1x), t1y, t1z);
    return tmin <= tmax ? tmin : kInf;
}

// The same precomputation with the origin and the reciprocal direction held
// twice per axis, as the register pairs of sm_100's packed float2 arithmetic:
// one packed subtract and one packed multiply give an axis's distances to both
// of its planes. Used by the query-set kernels and by the any-hit walk of the
// wavefront's shadow stage, which have the registers for the pairs (in the
// closest-hit walk of the extend stage the six extra registers cost a
// resident block per SM, more than the packed arithmetic saves).
struct RayPair {
    float2 o2x, o2y, o2z; // (o, o) per axis
    float2 i2x, i2y, i2z; // (1/d, 1/d) per axis
    bool nx, ny, nz;      // octant: direction negative on that axis
};

__device__ __forceinline__ RayPair precompute_pair(const RayD &r) {
    const RayPre q = precompute(r);
    RayPair p;
    p.o2x = make_float2(q.ox, q.ox);
    p.o2y = make_float2(q.oy, q.oy);
    p.o2z = make_float2(q.oz, q.oz);
    p.i2x = make_float2(q.ix, q.ix);
    p.i2y = make_float2(q.iy, q.iy);
    p.i2z = make_float2(q.iz, q.iz);
    p.nx = q.nx;
    p.ny = q.ny;
    p.nz = q.nz;
    return p;
}

// (a.x - b.x, a.y - b.y), each rounded to nearest like the scalar subtract.
__device__ __forceinline__ float2 fsub2(float2 a, float2 b) {
    float2 d;
    asm("{\n\t.reg .b64 a2, b2, d2;\n\t"
        "mov.b64 a2, {%2, %3};\n\t"
        "mov.b64 b2, {%4, %5};\n\t"
        "sub.rn.f32x2 d2, a2, b2;\n\t"
        "mov.b64 {%0, %1}, d2;\n\t}"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}

// slab() on the packed form: per axis (t at the min plane, t at the max
// plane) as (plane - o) * inv, each lane the float the scalar form computes;
// the octant then picks which of the two enters, as the reference picks the
// plane before subtracting.
__device__ __forceinline__ float slab(float x0, float x1, float y0, float y1, float z0, float z1,
                                      const RayPair &p) {
    const float2 tx = __fmul2_rn(fsub2(make_float2(x0, x1), p.o2x), p.i2x);
    const float2 ty = __fmul2_rn(fsub2(make_float2(y0, y1), p.o2y), p.i2y);
    const float2 tz = __fmul2_rn(fsub2(make_float2(z0, z1), p.o2z), p.i2z);
    const float t0x = p.nx ? tx.y : tx.x, t1x = p.nx ? tx.x : tx.y;
    const float t0y = p.ny ? ty.y : ty.x, t1y = p.ny ? ty.x : ty.y;
    const float t0z = p.nz ? tz.y : tz.x, t1z = p.nz ? tz.x : tz.y;
    const float tmin = fmax3(fmaxf(0.f, t0x), t0y, t0z);
    const float tmax = fmin3(fminf(kInf, t1x), t1y, t1z);
    return tmin <= tmax ? tmin : kInf;
}

__device__ __forceinline__ float slab6(const float *b, const RayPre &p) {
    return slab(b[0], b[1], b[2], b[3], b[4], b[5], p);
}

__device__ __forceinline__ float slab6(const float *b, const RayPair &p) {
    return slab(b[0], b[1], b[2], b[3], b[4], b[5], p);
}

struct NodeV {
    float4 a, b, c;
    uint4 link;
};

// 32 bytes from 32-byte aligned read-only global memory in one load
// instruction (sm_100's 256-bit vector load): half a node, or a whole Tri
// record. Builds with -DPRR_LDG128 use two 128-bit loads instead.
__device__ __forceinline__ void ldg256(const void *p, float4 &lo, float4 &hi) {
#ifdef PRR_LDG128
    lo = __ldg(reinterpret_cast<const float4 *>(p));
    hi = __ldg(reinterpret_cast<const float4 *>(p) + 1);
#else
    asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=f"(lo.x), "=f"(lo.y), "=f"(lo.z), "=f"(lo.w), "=f"(hi.x), "=f"(hi.y), "=f"(hi.z),
          "=f"(hi.w)
        : "l"(p));
#endif
}

__device__ __forceinline__ NodeV load_node(const WNode *nodes, uint32_t idx) {
    const WNode *q = nodes + idx;
    NodeV n;
    float4 l;
    ldg256(q, n.a, n.b);
    ldg256(reinterpret_cast<const float4 *>(q) + 2, n.c, l);
    n.link = make_uint4(__float_as_uint(l.x), __float_as_uint(l.y), __float_as_uint(l.z),
                        __float_as_uint(l.w));
    return n;
}

struct TriV {
    float4 p, q, r;
};

__device__ __forceinline__ TriV load_tri(const Tri *tris, const float *e2z, uint32_t idx) {
    TriV v;
    ldg256(tris + idx, v.p, v.q);
    v.r = make_float4(__ldg(e2z + idx), 0.f, 0.f, 0.f);
    return v;
}

// Checked forms: the plain fetch unless the build is checked and the index is
// out of range.
__device__ __forceinline__ NodeV load_node(const WNode *nodes, uint32_t idx,
                                           const TraceBounds &B) {
#ifdef PRR_CHECKED
    if (idx >= B.n_nodes) {
        check_fail(B.check, kCheckNode, idx);
        NodeV n; // two empty boxes: no slab test enters them
        n.a = make_float4(kInf, -kInf, kInf, -kInf);
        n.b = make_float4(kInf, -kInf, kInf, -kInf);
        n.c = make_float4(kInf, -kInf, kInf, -kInf);
        n.link = make_uint4(0u, 0u, 0u, 0u);
        return n;
    }
#endif
    return load_node(nodes, idx);
}

__device__ __forceinline__ TriV load_tri(const Tri *tris, const float *e2z, uint32_t idx,
                                         const TraceBounds &B) {
#ifdef PRR_CHECKED
    if (idx >= B.n_tris) {
        check_fail(B.check, kCheckTri, idx);
        TriV v; // all zero: det = 0 fails the parallel test
        v.p = v.q = v.r = make_float4(0.f, 0.f, 0.f, 0.f);
        return v;
    }
#endif
    return load_tri(tris, e2z, idx);
}

__device__ __forceinline__ NodeV load_node(const DevScene &S, uint32_t idx) {
    return load_node(S.nodes, idx, bounds_of(S));
}

__device__ __forceinline__ TriV load_tri(const DevScene &S, uint32_t idx) {
    return load_tri(S.tris, S.tri_e2z, idx, bounds_of(S));
}

// Triangle::hitTest (Triangle.hpp:46-64), evaluated without early exits. The
// miss tests are kept in their negated form so NaNs fall through exactly as
// the reference's `if (cond) return miss` chain lets them.
__device__ __forceinline__ bool tri_hit(const TriV &T, const RayD &r, float &t, float &u,
                                        float &v) {
    const float v0x = T.p.x, v0y = T.p.y, v0z = T.p.z;
    const float e1x = T.p.w, e1y = T.q.x, e1z = T.q.y;
    const float e2x = T.q.z, e2y = T.q.w, e2z = T.r.x;
    // P = d x e2
    const float px = r.dy * e2z - r.dz * e2y;
    const float py = r.dz * e2x - r.dx * e2z;
    const float pz = r.dx * e2y - r.dy * e2x;
    const float det = px * e1x + py * e1y + pz * e1z;
    const float inv = 1.f / det;
    const float tx = r.ox - v0x, ty = r.oy - v0y, tz = r.oz - v0z;
    u = (px * tx + py * ty + pz * tz) * inv;
    // Q = T x e1
    const float qx = ty * e1z - tz * e1y;
    const float qy = tz * e1x - tx * e1z;
    const float qz = tx * e1y - ty * e1x;
    v = (qx * r.dx + qy * r.dy + qz * r.dz) * inv;
    t = (qx * e2x + qy * e2y + qz * e2z) * inv;
    return !(fabsf(det) < 1e-6f) && !(u < 0.f) && !(v < 0.f || u + v > 1.f) && !(t <= 1e-3f);
}

// Triangle::intersectT (Triangle.hpp:75-92) followed by the caller's
// `t >= 0 && t < tMax` check (BVH.cpp:395-398).
__device__ __forceinline__ bool tri_occludes(const TriV &T, const RayD &r, float tmax) {
    const float v0x = T.p.x, v0y = T.p.y, v0z = T.p.z;
    const float e1x = T.p.w, e1y = T.q.x, e1z = T.q.y;
    const float e2x = T.q.z, e2y = T.q.w, e2z = T.r.x;
    const float px = r.dy * e2z - r.dz * e2y;
    const float py = r.dz * e2x - r.dx * e2z;
    const float pz = r.dx * e2y - r.dy * e2x;
    const float det = px * e1x + py * e1y + pz * e1z;
    const float inv = 1.f / det;
    const float tx = r.ox - v0x, ty = r.oy - v0y, tz = r.oz - v0z;
    const float u = (px * tx + py * ty + pz * tz) * inv;
    const float qx = ty * e1z - tz * e1y;
    const float qy = tz * e1x - tx * e1z;
    const float qz = tx * e1y - ty * e1x;
    const float v = (qx * r.dx + qy * r.dy + qz * r.dz) * inv;
    const float t = (qx * e2x + qy * e2y + qz * e2z) * inv;
    return !(fabsf(det) < 1e-6f) && !(u < 0.f || u > 1.f) && !(v < 0.f || u + v > 1.f) &&
           (t > 1e-3f && t < tmax);
}

// Per-thread stack with a bounded shared-memory part: entries [0, cap) in the
// thread's shared-memory column (entry k at sm[k * blockDim.x]), deeper
// entries in a global buffer laid out [entry - cap][grid thread], so a warp's
// spills are coalesced. A walk pushes at most once per tree level, so tree
// depth + 1 entries in the two parts together always suffice; the global part
// is only reached deep in unbalanced subtrees and stays in L1/L2. Its address
// is formed only on that cold path, so the stack costs two registers. `cap`
// is a launch parameter: fewer shared entries leave more of the SM's L1 for
// node and triangle fetches and let more blocks be resident.
template <class E> struct StackCol {
    E *sm;
    E *gl;
    int cap;
    int total = 1 << 30;     // entries in both parts (tested by the checked build)
    uint32_t *check = nullptr;
    __device__ __forceinline__ E *spill_at(int k) const {
        return gl + (size_t) (k - cap) * (gridDim.x * blockDim.x) + blockIdx.x * blockDim.x +
               threadIdx.x;
    }
    __device__ __forceinline__ void put(int k, E v) const {
#ifdef PRR_CHECKED
        if (k >= total || k < 0) {
            check_fail(check, kCheckStack, (uint32_t) k);
            return;
        }
#endif
        if (k < cap)
            sm[k * blockDim.x] = v;
        else
            *spill_at(k) = v;
    }
    __device__ __forceinline__ E get(int k) const {
#ifdef PRR_CHECKED
        if (k >= total || k < 0) {
            check_fail(check, kCheckStack, (uint32_t) k);
            return E{};
        }
#endif
        return k < cap ? sm[k * blockDim.x] : *spill_at(k);
    }
};

// Per-thread stack column in shared memory.
struct SmemStack {
    uint2 *base; // &smem[tid]; entry k at base[k * stride]
    int stride;
    int sp;
    int cap = 1 << 30;         // entries in the column (tested by the checked build)
    uint32_t *check = nullptr; // where the checked build reports
    __device__ __forceinline__ void push(uint32_t ref, float t) {
#ifdef PRR_CHECKED
        if (sp >= cap) {
            check_fail(check, kCheckStack, (uint32_t) sp);
            return;
        }
#endif
        base[sp * stride] = make_uint2(ref, __float_as_uint(t));
        sp++;
    }
    __device__ __forceinline__ uint2 pop() {
        --sp;
        return base[sp * stride];
    }
};

// BVHAccel::Intersect, triangle fast path (BVH.cpp:311-415) on one mesh BVH.
// best_t enters as +inf (every mesh-level search starts fresh, BVH.cpp:331).
// Returns the winning triangle's global leaf-order index, or -1.
__device__ __forceinline__ int blas_closest(const WNode *__restrict__ nodes,
                                            const Tri *__restrict__ tris,
                                            const float *__restrict__ e2z, uint32_t root,
                                            const RayD &r, const RayPre &p, SmemStack &st,
                                            float &best_t, float &best_u, float &best_v,
                                            const TraceBounds &B) {
    const int sp0 = st.sp;
    uint32_t ref = root;
    int hit = -1;
    for (;;) {
        if (!(ref & kLeafBit)) {
            const NodeV n = load_node(nodes, ref, B);
            const float tl = slab(n.a.x, n.a.y, n.a.z, n.a.w, n.b.x, n.b.y, p);
            const float tr = slab(n.b.z, n.b.w, n.c.x, n.c.y, n.c.z, n.c.w, p);
            if (tl <= tr) {
                if (tl < best_t) {
                    if (tr < best_t)
                        st.push(n.link.y, tr);
                    ref = n.link.x;
                    continue;
                }
            } else {
                if (tr < best_t) {
                    if (tl < best_t)
                        st.push(n.link.x, tl);
                    ref = n.link.y;
                    continue;
                }
            }
        } else {
            const uint32_t first = leaf_first(ref);
            const uint32_t cnt = leaf_count(ref);
            for (uint32_t i = 0; i < cnt; i++) {
                const TriV T = load_tri(tris, e2z, first + i, B);
                float t, u, v;
                if (tri_hit(T, r, t, u, v) && t < best_t) {
                    best_t = t;
                    best_u = u;
                    best_v = v;
                    hit = (int) (first + i);
                }
            }
        }
        // pop the next entry whose box is still nearer than the closest hit
        for (;;) {
            if (st.sp == sp0)
                return hit;
            const uint2 e = st.pop();
            if (__uint_as_float(e.y) < best_t) {
                ref = e.x;
                break;
            }
        }
    }
}

// BVHAccel::IntersectP (BVH.cpp:421-473) on one mesh BVH whose root box is
// root_box: true when a triangle occludes within tmax. Child boxes are tested
// where the reference tests them (far child at push, near child at the top of
// the next iteration), so exactly the same subtrees are entered.
__device__ __forceinline__ bool blas_occluded(const WNode *__restrict__ nodes,
                                              const Tri *__restrict__ tris,
                                              const float *__restrict__ e2z, uint32_t root,
                                              const float *root_box, const RayD &r,
                                              const RayPre &p, SmemStack &st, float tmax,
                                              const TraceBounds &B) {
    if (!(slab6(root_box, p) < tmax))
        return false;
    const int sp0 = st.sp;
    uint32_t ref = root;
    for (;;) {
        if (!(ref & kLeafBit)) {
            const NodeV n = load_node(nodes, ref, B);
            const float tl = slab(n.a.x, n.a.y, n.a.z, n.a.w, n.b.x, n.b.y, p);
            const float tr = slab(n.b.z, n.b.w, n.c.x, n.c.y, n.c.z, n.c.w, p);
            const uint32_t axis = n.link.z;
            const bool neg = axis == 0 ? p.nx : (axis == 1 ? p.ny : p.nz);
            // octant 0 -> near = left
            const uint32_t near_ref = neg ? n.link.y : n.link.x;
            const uint32_t far_ref = neg ? n.link.x : n.link.y;
            const float tnear = neg ? tr : tl;
            const float tfar = neg ? tl : tr;
            if (tfar < tmax)
                st.push(far_ref, 0.f);
            if (tnear < tmax) {
                ref = near_ref;
                continue;
            }
        } else {
            const uint32_t first = leaf_first(ref);
            const uint32_t cnt = leaf_count(ref);
            for (uint32_t i = 0; i < cnt; i++) {
                const TriV T = load_tri(tris, e2z, first + i, B);
                if (tri_occludes(T, r, tmax)) {
                    st.sp = sp0;
                    return true;
                }
            }
        }
        if (st.sp == sp0)
            return false;
        ref = st.pop().x;
    }
}

// Sphere::getIntersection (Sphere.hpp:22-44) with solveQuadratic
// (global.hpp:19-33). The reference calls the double sqrt there and mixes
// -0.5 (a double) into both roots, so those steps run in double and round to
// float exactly where the reference's assignments do.
__device__ __forceinline__ bool sphere_hit(const DevObject &s, const RayD &r, float &t_out) {
    const float Lx = r.ox - s.cx, Ly = r.oy - s.cy, Lz = r.oz - s.cz;
    const float a = r.dx * r.dx + r.dy * r.dy + r.dz * r.dz;
    const float b = 2 * (r.dx * Lx + r.dy * Ly + r.dz * Lz);
    const float c = (Lx * Lx + Ly * Ly + Lz * Lz) - s.radius2;
    const float discr = b * b - 4 * a * c;
    float x0, x1;
    if (discr < 0)
        return false;
    else if (discr == 0) {
        x0 = x1 = (float) (-0.5 * (double) b / (double) a);
    } else {
        const double sq = sqrt((double) discr);
        const float q = (b > 0) ? (float) (-0.5 * ((double) b + sq))
                                : (float) (-0.5 * ((double) b - sq));
        x0 = q / a;
        x1 = c / q;
    }
    if (x0 > x1) {
        float tmp = x0;
        x0 = x1;
        x1 = tmp;
    }
    float t0 = x0;
    if (t0 < 0)
        t0 = x1;
    if (t0 < 0)
        return false;
    t_out = t0;
    return true;
}

struct SceneHit {
    int obj;      // object index, -1 on a miss
    int tri;      // global leaf-order triangle index (meshes), -1 for spheres
    float t, u, v;
};

// Scene::intersect -> BVHAccel::Intersect, general path (BVH.cpp:359-369):
// every scene-BVH leaf object is intersected on its own (meshes start their
// own search at +inf) and replaces the winner when tnear < closestT.
__device__ __forceinline__ SceneHit scene_closest(const DevScene &S, const RayD &r,
                                                  const RayPre &p, SmemStack &tst,
                                                  SmemStack &bst) {
    SceneHit h;
    h.obj = -1;
    h.tri = -1;
    h.t = kInf;
    h.u = h.v = 0.f;
    if (S.n_objects == 0)
        return h;
    float closest = kInf;
    const int sp0 = tst.sp;
    uint32_t ref = S.tlas_root;
    for (;;) {
        if (!(ref & kLeafBit)) {
            const NodeV n = load_node(S, ref);
            const float tl = slab(n.a.x, n.a.y, n.a.z, n.a.w, n.b.x, n.b.y, p);
            const float tr = slab(n.b.z, n.b.w, n.c.x, n.c.y, n.c.z, n.c.w, p);
            if (tl <= tr) {
                if (tl < closest) {
                    if (tr < closest)
                        tst.push(n.link.y, tr);
                    ref = n.link.x;
                    continue;
                }
            } else {
                if (tr < closest) {
                    if (tl < closest)
                        tst.push(n.link.x, tl);
                    ref = n.link.y;
                    continue;
                }
            }
        } else {
            const int k = (int) (ref & ~kLeafBit);
            const DevObject &o = S.objects[k];
            if (o.kind == kObjMesh) {
                float t = kInf, u = 0.f, v = 0.f;
                const int tri = blas_closest(S.nodes, S.tris, S.tri_e2z, o.root, r, p, bst, t, u, v,
                                             bounds_of(S));
                if (tri >= 0 && t < closest) {
                    closest = t;
                    h.obj = k;
                    h.tri = tri;
                    h.t = t;
                    h.u = u;
                    h.v = v;
                }
            } else {
                float t;
                if (sphere_hit(o, r, t) && t < closest) {
                    closest = t;
                    h.obj = k;
                    h.tri = -1;
                    h.t = t;
                }
            }
        }
        for (;;) {
            if (tst.sp == sp0)
                return h;
            const uint2 e = tst.pop();
            if (__uint_as_float(e.y) < closest) {
                ref = e.x;
                break;
            }
        }
    }
}

// Scene::intersectP -> BVHAccel::IntersectP over objects (BVH.cpp:421-473):
// MeshTriangle::intersectT answers 1e-3 when its own IntersectP finds an
// occluder (Triangle.hpp:141-147) and Sphere falls back to
// Object::intersectT (Object.hpp:24-29); the caller then requires
// t >= 0 && t < tMax.
__device__ __forceinline__ bool scene_occluded(const DevScene &S, const RayD &r,
                                               const RayPre &p, SmemStack &tst, SmemStack &bst,
                                               float tmax) {
    if (S.n_objects == 0)
        return false;
    if (!(slab6(S.tlas_box, p) < tmax))
        return false;
    const int sp0 = tst.sp;
    uint32_t ref = S.tlas_root;
    for (;;) {
        if (!(ref & kLeafBit)) {
            const NodeV n = load_node(S, ref);
            const float tl = slab(n.a.x, n.a.y, n.a.z, n.a.w, n.b.x, n.b.y, p);
            const float tr = slab(n.b.z, n.b.w, n.c.x, n.c.y, n.c.z, n.c.w, p);
            const uint32_t axis = n.link.z;
            const bool neg = axis == 0 ? p.nx : (axis == 1 ? p.ny : p.nz);
            const uint32_t near_ref = neg ? n.link.y : n.link.x;
            const uint32_t far_ref = neg ? n.link.x : n.link.y;
            const float tnear = neg ? tr : tl;
            const float tfar = neg ? tl : tr;
            if (tfar < tmax)
                tst.push(far_ref, 0.f);
            if (tnear < tmax) {
                ref = near_ref;
                continue;
            }
        } else {
            const DevObject &o = S.objects[ref & ~kLeafBit];
            bool occ;
            if (o.kind == kObjMesh) {
                occ = blas_occluded(S.nodes, S.tris, S.tri_e2z, o.root, o.root_box, r, p, bst, tmax,
                                    bounds_of(S)) &&
                      (1e-3f < tmax);
            } else {
                float t;
                occ = sphere_hit(o, r, t) && t < tmax && t >= 0.f;
            }
            if (occ) {
                tst.sp = sp0;
                return true;
            }
        }
        if (tst.sp == sp0)
            return false;
        ref = tst.pop().x;
    }
}

} // namespace prr
