// Batch ray-query kernels: mesh closest hit / any hit (the BVHAccel::Intersect
// and IntersectP micro-path, BVH.cpp:311-473) and scene-level closest hit /
// any hit (Scene::intersect / intersectP, Scene.cpp:29-35).
//
// One thread traces one ray. Stacks are columns of a dynamic shared-memory
// array sized from the tree depth measured at build time, so the stack bound is
// proven rather than guessed (a push only happens at an interior node and at
// most one entry per tree level is outstanding).
//
// Two launch shapes: a plain grid (one ray per thread) and a persistent grid
// sized to the SM count in which each warp pulls 32-ray batches from a global
// counter; the autotuner picks per scene.
#include "prr_internal.h"
#include "trace.cuh"

#include <algorithm>

namespace prr {

namespace {

__device__ __forceinline__ RayD load_ray(const float *__restrict__ O, const float *__restrict__ D,
                                         int64_t i) {
    RayD r;
    r.ox = __ldg(O + i * 3 + 0);
    r.oy = __ldg(O + i * 3 + 1);
    r.oz = __ldg(O + i * 3 + 2);
    r.dx = __ldg(D + i * 3 + 0);
    r.dy = __ldg(D + i * 3 + 1);
    r.dz = __ldg(D + i * 3 + 2);
    return r;
}

// Möller-Trumbore in fp64 on the input vertices: the winner's t re-solved for
// the 1e-6-relative check, once per ray.
__device__ double tri_t64(const float *__restrict__ v, const RayD &r) {
    const double v0x = v[0], v0y = v[1], v0z = v[2];
    const double e1x = (double) v[3] - v0x, e1y = (double) v[4] - v0y, e1z = (double) v[5] - v0z;
    const double e2x = (double) v[6] - v0x, e2y = (double) v[7] - v0y, e2z = (double) v[8] - v0z;
    const double ox = r.ox, oy = r.oy, oz = r.oz, dx = r.dx, dy = r.dy, dz = r.dz;
    const double tx = ox - v0x, ty = oy - v0y, tz = oz - v0z;
    const double px = dy * e2z - dz * e2y, py = dz * e2x - dx * e2z, pz = dx * e2y - dy * e2x;
    const double qx = ty * e1z - tz * e1y, qy = tz * e1x - tx * e1z, qz = tx * e1y - ty * e1x;
    const double det = px * e1x + py * e1y + pz * e1z;
    return (qx * e2x + qy * e2y + qz * e2z) / det;
}

struct MeshArgs {
    const WNode *nodes;
    const Tri *tris;
    const float *e2z;
    const TriMeta *meta;
    const float *verts;
    uint32_t root;
    const float *O, *D;
    int64_t n;
    int32_t *out_id;
    float *out_t;
    double *out_t64;
    unsigned long long *counter;
    int stack_stride;
    int stack_cap;        // entries of a thread's stack column
    TraceBounds B;        // array bounds and status words (checked build)
    const uint32_t *perm; // trace order -> input index (nullptr: input order)
};

// Push onto this thread's stack column; the checked build tests the depth.
#ifdef PRR_CHECKED
#define PRR_COL_PUSH(val)                                                                          \
    do {                                                                                           \
        if (sp < a.stack_cap) {                                                                    \
            col[sp * stride] = (val);                                                              \
            sp++;                                                                                  \
        } else {                                                                                   \
            check_fail(a.B.check, kCheckStack, (uint32_t) sp);                                     \
        }                                                                                          \
    } while (0)
#else
#define PRR_COL_PUSH(val)                                                                          \
    do {                                                                                           \
        col[sp * stride] = (val);                                                                  \
        sp++;                                                                                      \
    } while (0)
#endif

// Input index of the ray traced in position i.
__device__ __forceinline__ int64_t ray_at(const MeshArgs &a, int64_t i) {
    return a.perm ? (int64_t) __ldg(a.perm + i) : i;
}

__device__ __forceinline__ void mesh_closest_one(const MeshArgs &a, SmemStack &st, int64_t i) {
    const RayD r = load_ray(a.O, a.D, i);
    const RayPre p = precompute(r);
    float t = kInf, u = 0.f, v = 0.f;
    const int hit = blas_closest(a.nodes, a.tris, a.e2z, a.root, r, p, st, t, u, v, a.B);
    a.out_id[i] = hit >= 0 ? __ldg(&a.meta[hit].id) : -1;
    a.out_t[i] = t;
    if (a.out_t64)
        a.out_t64[i] = hit >= 0 ? tri_t64(a.verts + (size_t) hit * 9, r) : __longlong_as_double(0x7ff8000000000000LL);
}

__global__ void k_mesh_closest(MeshArgs a) {
    extern __shared__ uint2 smem[];
    SmemStack st{smem + threadIdx.x, (int) blockDim.x, 0, a.stack_cap, a.B.check};
    const int64_t stride = (int64_t) gridDim.x * blockDim.x;
    for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride)
        mesh_closest_one(a, st, ray_at(a, i));
}

// Persistent: each warp takes the next 32 rays from the counter until none
// are left. The counter is zeroed on the stream before the launch.
__global__ void k_mesh_closest_persistent(MeshArgs a) {
    extern __shared__ uint2 smem[];
    SmemStack st{smem + threadIdx.x, (int) blockDim.x, 0, a.stack_cap, a.B.check};
    const int lane = threadIdx.x & 31;
    for (;;) {
        unsigned long long base = 0;
        if (lane == 0)
            base = atomicAdd(a.counter, 32ull);
        base = __shfl_sync(0xffffffffu, base, 0);
        if ((int64_t) base >= a.n)
            break;
        const int64_t i = (int64_t) base + lane;
        if (i < a.n)
            mesh_closest_one(a, st, ray_at(a, i));
    }
}

// Persistent with per-lane refill. Each loop iteration performs ONE step of
// the lane's ray: one interior node (two child slab tests, BVH.cpp:368-397),
// or one triangle of the current leaf (BVH.cpp:343-357), followed when needed
// by the pop of BVH.cpp:400-407. A lane whose ray is done stays idle until
// `refill` lanes of its warp are idle; then the warp takes that many new rays
// with one atomic and the idle lanes start them. Rays finishing at different
// depths therefore no longer hold their warp hostage, and every ray still
// visits exactly the nodes and triangles, in exactly the order, of the
// reference walk.
__global__ void k_mesh_closest_refill(MeshArgs a, int refill) {
    extern __shared__ uint2 smem[];
    uint2 *col = smem + threadIdx.x;
    const int stride = blockDim.x;
    const int lane = threadIdx.x & 31;
    const unsigned full = 0xffffffffu;
    int64_t idx = -1;
    RayD r{};
    RayPair p{};
    float best = kInf;
    int hit = -1;
    uint32_t ref = 0, tri = 0, ntri = 0;
    int sp = 0;
    bool more = true; // warp-uniform: the ray counter is not exhausted
    for (;;) {
        const bool idle = idx < 0;
        const unsigned im = __ballot_sync(full, idle);
        if (!more && im == full)
            break;
        if (more && __popc(im) >= refill) {
            const int cnt = __popc(im);
            unsigned long long base = 0;
            if (lane == 0)
                base = atomicAdd(a.counter, (unsigned long long) cnt);
            base = __shfl_sync(full, base, 0);
            if ((int64_t) (base + cnt) >= a.n)
                more = false;
            if (idle) {
                const int64_t ni = (int64_t) base + __popc(im & ((1u << lane) - 1u));
                if (ni < a.n) {
                    idx = ray_at(a, ni);
                    r = load_ray(a.O, a.D, idx);
                    p = precompute_pair(r);
                    best = kInf;
                    hit = -1;
                    sp = 0;
                    if (a.root & kLeafBit) {
                        tri = leaf_first(a.root);
                        ntri = leaf_count(a.root);
                    } else {
                        ref = a.root;
                        ntri = 0;
                    }
                }
            }
        }
        if (idx < 0)
            continue;
        bool pop = false;
        if (ntri > 0) {
            const TriV T = load_tri(a.tris, a.e2z, tri, a.B);
            float t, u, v;
            if (tri_hit(T, r, t, u, v) && t < best) {
                best = t;
                hit = (int) tri;
            }
            tri++;
            ntri--;
            pop = ntri == 0;
        } else {
            const NodeV n = load_node(a.nodes, ref, a.B);
            const float tl = slab(n.a.x, n.a.y, n.a.z, n.a.w, n.b.x, n.b.y, p);
            const float tr = slab(n.b.z, n.b.w, n.c.x, n.c.y, n.c.z, n.c.w, p);
            uint32_t next = 0;
            bool down = false;
            if (tl <= tr) {
                if (tl < best) {
                    if (tr < best) {
                        PRR_COL_PUSH(make_uint2(n.link.y, __float_as_uint(tr)));
                    }
                    next = n.link.x;
                    down = true;
                }
            } else {
                if (tr < best) {
                    if (tl < best) {
                        PRR_COL_PUSH(make_uint2(n.link.x, __float_as_uint(tl)));
                    }
                    next = n.link.y;
                    down = true;
                }
            }
            if (down) {
                if (next & kLeafBit) {
                    tri = leaf_first(next);
                    ntri = leaf_count(next);
                } else {
                    ref = next;
                }
            } else {
                pop = true;
            }
        }
        if (pop) {
            bool found = false;
            uint32_t next = 0;
            while (sp > 0) {
                --sp;
                const uint2 e = col[sp * stride];
                if (__uint_as_float(e.y) < best) {
                    next = e.x;
                    found = true;
                    break;
                }
            }
            if (found) {
                if (next & kLeafBit) {
                    tri = leaf_first(next);
                    ntri = leaf_count(next);
                } else {
                    ref = next;
                }
            } else {
                a.out_id[idx] = hit >= 0 ? __ldg(&a.meta[hit].id) : -1;
                a.out_t[idx] = best;
                if (a.out_t64)
                    a.out_t64[idx] = hit >= 0 ? tri_t64(a.verts + (size_t) hit * 9, r)
                                              : __longlong_as_double(0x7ff8000000000000LL);
                idx = -1;
            }
        }
    }
}

// Persistent closest hit with postponed leaves (phased): a lane that reaches a
// leaf parks it and keeps walking interior nodes until it reaches a second
// leaf; each warp step is then either a node step for every lane that can
// walk or a triangle step for every lane holding a parked leaf (chosen when
// at least `tri_min` lanes hold one), so the two kinds of work no longer
// split a warp. Exactness: leaves are still taken in the reference's DFS
// order, and a parked leaf is re-tested against the closest hit at the time
// its triangles are tested (the box entry < closest test the reference makes
// when it reaches that leaf); the interior nodes walked meanwhile with an
// older closest hit only add leaves that this re-test then drops, since a
// box contains the boxes below it and the slab entry distance is monotone in
// the box.
constexpr uint32_t kNoRef = 0xFFFFFFFFu;

__global__ void k_mesh_closest_phased(MeshArgs a, int refill, int tri_min) {
    extern __shared__ uint2 smem[];
    uint2 *col = smem + threadIdx.x;
    const int stride = blockDim.x;
    const int lane = threadIdx.x & 31;
    const unsigned full = 0xffffffffu;
    int64_t idx = -1;
    RayD r{};
    RayPair p{};
    float best = kInf;
    int hit = -1;
    uint32_t ref = kNoRef; // walk position: interior node, leaf waiting for the slot, or none
    float ref_t = 0.f;     // box entry distance of ref
    uint32_t ptri = 0;     // parked leaf: next triangle, triangles left, box entry
    int pcnt = 0;
    float pt = 0.f;
    int sp = 0;
    bool more = true; // warp-uniform: the ray counter is not exhausted
    for (;;) {
        const bool idle = idx < 0;
        const unsigned im = __ballot_sync(full, idle);
        if (!more && im == full)
            break;
        if (more && __popc(im) >= refill) {
            const int cnt = __popc(im);
            unsigned long long base = 0;
            if (lane == 0)
                base = atomicAdd(a.counter, (unsigned long long) cnt);
            base = __shfl_sync(full, base, 0);
            if ((int64_t) (base + cnt) >= a.n)
                more = false;
            if (idle) {
                const int64_t ni = (int64_t) base + __popc(im & ((1u << lane) - 1u));
                if (ni < a.n) {
                    idx = ray_at(a, ni);
                    r = load_ray(a.O, a.D, idx);
                    p = precompute_pair(r);
                    best = kInf;
                    hit = -1;
                    sp = 0;
                    ref = a.root;
                    ref_t = -kInf; // the root is entered without a box test
                    pcnt = 0;
                }
            }
        }
        const bool act = idx >= 0;
        const bool leaf_wait = ref != kNoRef && (ref & kLeafBit);
        const bool tw = act && pcnt > 0;
        const bool nw = act && !(leaf_wait && pcnt > 0) && !(ref == kNoRef && sp == 0);
        const unsigned tm = __ballot_sync(full, tw);
        const unsigned nm = __ballot_sync(full, nw);
        if (tm != 0 && (nm == 0 || __popc(tm) >= tri_min)) {
            if (tw) {
                if (pt < best) {
                    pt = -kInf; // the leaf passed; its other triangles follow unconditionally
                    const TriV T = load_tri(a.tris, a.e2z, ptri, a.B);
                    float t, u, v;
                    if (tri_hit(T, r, t, u, v) && t < best) {
                        best = t;
                        hit = (int) ptri;
                    }
                    ptri++;
                    pcnt--;
                } else {
                    pcnt = 0;
                }
            }
        } else if (nw) {
            if (ref != kNoRef && !(ref & kLeafBit)) {
                const NodeV n = load_node(a.nodes, ref, a.B);
                const float tl = slab(n.a.x, n.a.y, n.a.z, n.a.w, n.b.x, n.b.y, p);
                const float tr = slab(n.b.z, n.b.w, n.c.x, n.c.y, n.c.z, n.c.w, p);
                uint32_t next = kNoRef;
                float next_t = 0.f;
                if (tl <= tr) {
                    if (tl < best) {
                        if (tr < best) {
                            PRR_COL_PUSH(make_uint2(n.link.y, __float_as_uint(tr)));
                        }
                        next = n.link.x;
                        next_t = tl;
                    }
                } else {
                    if (tr < best) {
                        if (tl < best) {
                            PRR_COL_PUSH(make_uint2(n.link.x, __float_as_uint(tl)));
                        }
                        next = n.link.y;
                        next_t = tr;
                    }
                }
                ref = next;
                ref_t = next_t;
            }
            if (ref != kNoRef && (ref & kLeafBit) && pcnt == 0) {
                ptri = leaf_first(ref);
                pcnt = (int) leaf_count(ref);
                pt = ref_t;
                ref = kNoRef;
            }
            while (ref == kNoRef && sp > 0) {
                --sp;
                const uint2 e = col[sp * stride];
                if (__uint_as_float(e.y) < best) {
                    ref = e.x;
                    ref_t = __uint_as_float(e.y);
                }
            }
        }
        if (act && ref == kNoRef && sp == 0 && pcnt == 0) {
            a.out_id[idx] = hit >= 0 ? __ldg(&a.meta[hit].id) : -1;
            a.out_t[idx] = best;
            if (a.out_t64)
                a.out_t64[idx] = hit >= 0 ? tri_t64(a.verts + (size_t) hit * 9, r)
                                          : __longlong_as_double(0x7ff8000000000000LL);
            idx = -1;
        }
    }
}

__global__ void k_mesh_occluded(const WNode *nodes, const Tri *tris, const float *e2z,
                                uint32_t root,
                                DevObject obj, const float *O, const float *D,
                                const float *__restrict__ tmax, int64_t n, uint8_t *out,
                                TraceBounds B, int stack_cap) {
    extern __shared__ uint2 smem[];
    SmemStack st{smem + threadIdx.x, (int) blockDim.x, 0, stack_cap, B.check};
    const int64_t stride = (int64_t) gridDim.x * blockDim.x;
    for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const RayD r = load_ray(O, D, i);
        const RayPre p = precompute(r);
        out[i] = blas_occluded(nodes, tris, e2z, root, obj.root_box, r, p, st, __ldg(tmax + i), B)
                     ? 1
                     : 0;
    }
}

__global__ void k_scene_closest(DevScene S, const float *O, const float *D, int64_t n,
                                int32_t *out_obj, int32_t *out_prim, float *out_t, float *geo,
                                int tlas_cap) {
    extern __shared__ uint2 smem[];
    SmemStack tst{smem + threadIdx.x, (int) blockDim.x, 0, S.tlas_depth + 1, S.check};
    SmemStack bst{smem + (size_t) tlas_cap * blockDim.x + threadIdx.x, (int) blockDim.x, 0,
                  S.blas_depth + 1, S.check};
    const int64_t stride = (int64_t) gridDim.x * blockDim.x;
    for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const RayD r = load_ray(O, D, i);
        const RayPre p = precompute(r);
        const SceneHit h = scene_closest(S, r, p, tst, bst);
        out_obj[i] = h.obj;
        out_t[i] = h.t;
        if (h.obj < 0) {
            out_prim[i] = -1;
            continue;
        }
        const DevObject &o = S.objects[h.obj];
        // hit coords (Triangle.cpp:37 / Sphere.hpp:37): origin + direction * t
        const float cx = r.ox + r.dx * h.t, cy = r.oy + r.dy * h.t, cz = r.oz + r.dz * h.t;
        float nx, ny, nz;
        if (o.kind == kObjMesh) {
            out_prim[i] = __ldg(&S.tri_meta[h.tri].id);
            nx = S.normals[(size_t) h.tri * 3 + 0];
            ny = S.normals[(size_t) h.tri * 3 + 1];
            nz = S.normals[(size_t) h.tri * 3 + 2];
            if (o.attr & kAttrNormals) {
                // Triangle::finalize (Triangle.cpp:44-47): normalize(n0*w0 + n1*u + n2*v)
                float t, u, v;
                tri_hit(load_tri(S, (uint32_t) h.tri), r, t, u, v);
                const float w0 = 1.f - u - v;
                const float *R = S.attr + (size_t) (o.attr_base + (h.tri - o.tri_base)) * kAttrFloats;
                float x = R[0] * w0 + R[3] * u + R[6] * v;
                float y = R[1] * w0 + R[4] * u + R[7] * v;
                float z = R[2] * w0 + R[5] * u + R[8] * v;
                const float m2 = x * x + y * y + z * z;
                if (m2 > 0) {
                    const float inv = 1 / sqrtf(m2);
                    x = x * inv;
                    y = y * inv;
                    z = z * inv;
                }
                nx = x;
                ny = y;
                nz = z;
            }
        } else {
            out_prim[i] = 0;
            // normalize(coords - center) (Vector.hpp:103-111)
            float x = cx - o.cx, y = cy - o.cy, z = cz - o.cz;
            float m2 = x * x + y * y + z * z;
            if (m2 > 0) {
                float inv = 1 / sqrtf(m2);
                x = x * inv;
                y = y * inv;
                z = z * inv;
            }
            nx = x;
            ny = y;
            nz = z;
        }
        if (geo) {
            geo[i * 6 + 0] = cx;
            geo[i * 6 + 1] = cy;
            geo[i * 6 + 2] = cz;
            geo[i * 6 + 3] = nx;
            geo[i * 6 + 4] = ny;
            geo[i * 6 + 5] = nz;
        }
    }
}

__global__ void k_scene_occluded(DevScene S, const float *O, const float *D,
                                 const float *__restrict__ tmax, int64_t n, uint8_t *out,
                                 int tlas_cap) {
    extern __shared__ uint2 smem[];
    SmemStack tst{smem + threadIdx.x, (int) blockDim.x, 0, S.tlas_depth + 1, S.check};
    SmemStack bst{smem + (size_t) tlas_cap * blockDim.x + threadIdx.x, (int) blockDim.x, 0,
                  S.blas_depth + 1, S.check};
    const int64_t stride = (int64_t) gridDim.x * blockDim.x;
    for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const RayD r = load_ray(O, D, i);
        const RayPre p = precompute(r);
        out[i] = scene_occluded(S, r, p, tst, bst, __ldg(tmax + i)) ? 1 : 0;
    }
}

// ---------------------------------------------------------------- ray order
// Coherence reordering before a closest-hit batch. Each ray gets a 30-bit key
// from where it enters the mesh's root box (its origin if it starts inside)
// and its normalised direction, each quantised to 5 bits per axis; the
// buckets are the key's top `bits` bits. A counting pass, an exclusive scan
// and a scatter with one atomic per ray give a permutation grouped by bucket
// (the order inside a bucket is whatever the atomics give: it does not matter,
// because every ray's result is written at its own input index and the walk
// of one ray does not depend on any other). Rays that miss the root box get
// the last bucket.

// bit k of v (k < 5) to bit 6k, for a 6-way interleave
__device__ __forceinline__ uint32_t spread6(uint32_t v) {
    uint32_t r = 0;
#pragma unroll
    for (int b = 0; b < 5; b++)
        r |= ((v >> b) & 1u) << (6 * b);
    return r;
}

// bit k of v (k < 5) to bit 3k, for a 3-way interleave
__device__ __forceinline__ uint32_t spread3(uint32_t v) {
    uint32_t r = 0;
#pragma unroll
    for (int b = 0; b < 5; b++)
        r |= ((v >> b) & 1u) << (3 * b);
    return r;
}

__device__ __forceinline__ uint32_t quant5(float u) {
    const float q = u * 32.f;
    return q <= 0.f ? 0u : (q >= 31.f ? 31u : (uint32_t) q);
}

struct RayKeyArgs {
    const float *O, *D;
    int64_t n;
    float box[6]; // root box [minX,maxX,minY,maxY,minZ,maxZ]
    int mode;     // 1 entry and direction interleaved, 2 direction-major, 3 entry-major,
                  // 4 entry and exit point interleaved, 5 entry-major then exit
    int shift;    // key >> shift = bucket
    uint32_t *bucket;
    uint32_t *count;
};

__global__ void k_ray_buckets(RayKeyArgs a) {
    const int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n)
        return;
    const RayD r = load_ray(a.O, a.D, i);
    const RayPre p = precompute(r);
    const float t = slab(a.box[0], a.box[1], a.box[2], a.box[3], a.box[4], a.box[5], p);
    uint32_t key = (1u << 30) - 1u;
    if (t < kInf) {
        const float ex = (r.ox + r.dx * t - a.box[0]) / (a.box[1] - a.box[0]);
        const float ey = (r.oy + r.dy * t - a.box[2]) / (a.box[3] - a.box[2]);
        const float ez = (r.oz + r.dz * t - a.box[4]) / (a.box[5] - a.box[4]);
        const float inv = rsqrtf(r.dx * r.dx + r.dy * r.dy + r.dz * r.dz);
        const uint32_t qx = quant5(ex), qy = quant5(ey), qz = quant5(ez);
        const uint32_t dx = quant5(0.5f + 0.5f * r.dx * inv);
        const uint32_t dy = quant5(0.5f + 0.5f * r.dy * inv);
        const uint32_t dz = quant5(0.5f + 0.5f * r.dz * inv);
        const uint32_t e3 = spread3(qx) << 2 | spread3(qy) << 1 | spread3(qz);
        const uint32_t d3 = spread3(dx) << 2 | spread3(dy) << 1 | spread3(dz);
        if (a.mode == 2) {
            key = d3 << 15 | e3;
        } else if (a.mode == 3) {
            key = e3 << 15 | d3;
        } else if (a.mode >= 4) {
            // where the ray leaves the box: the nearest far slab
            const float fx = ((p.nx ? a.box[0] : a.box[1]) - p.ox) * p.ix;
            const float fy = ((p.ny ? a.box[2] : a.box[3]) - p.oy) * p.iy;
            const float fz = ((p.nz ? a.box[4] : a.box[5]) - p.oz) * p.iz;
            const float tx = fminf(fx, fminf(fy, fz));
            const uint32_t xx = quant5((r.ox + r.dx * tx - a.box[0]) / (a.box[1] - a.box[0]));
            const uint32_t xy = quant5((r.oy + r.dy * tx - a.box[2]) / (a.box[3] - a.box[2]));
            const uint32_t xz = quant5((r.oz + r.dz * tx - a.box[4]) / (a.box[5] - a.box[4]));
            if (a.mode == 4)
                key = spread6(qx) << 5 | spread6(qy) << 4 | spread6(qz) << 3 | spread6(xx) << 2 |
                      spread6(xy) << 1 | spread6(xz);
            else
                key = e3 << 15 | spread3(xx) << 2 | spread3(xy) << 1 | spread3(xz);
        } else {
            key = spread6(qx) << 5 | spread6(qy) << 4 | spread6(qz) << 3 | spread6(dx) << 2 |
                  spread6(dy) << 1 | spread6(dz);
        }
    }
    const uint32_t b = key >> a.shift;
    a.bucket[i] = b;
    atomicAdd(a.count + b, 1u);
}

// Exclusive scan of count[0, m) in place, in tiles of 4096 (1024 threads x 4):
// tile sums first, then the sums' scan, then the tiles.
constexpr int kScanTile = 4096;

__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t *sh,
                                                         uint32_t *total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o)
            x += y;
    }
    if (lane == 31)
        sh[warp] = x;
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
        uint32_t w = lane < nw ? sh[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o)
                w += y;
        }
        if (lane < nw)
            sh[lane] = w;
    }
    __syncthreads();
    const uint32_t before = (warp > 0 ? sh[warp - 1] : 0u) + x - v;
    if (total)
        *total = sh[(blockDim.x >> 5) - 1];
    __syncthreads();
    return before;
}

__global__ void k_scan_tile_sums(const uint32_t *count, int64_t m, uint32_t *sums) {
    __shared__ uint32_t sh[32];
    const int64_t base = (int64_t) blockIdx.x * kScanTile + (int64_t) threadIdx.x * 4;
    uint32_t v = 0;
    for (int k = 0; k < 4; k++)
        if (base + k < m)
            v += count[base + k];
    uint32_t total = 0;
    block_exclusive_scan(v, sh, &total);
    if (threadIdx.x == 0)
        sums[blockIdx.x] = total;
}

// one block: exclusive scan of the tile sums (at most 1024 tiles)
__global__ void k_scan_sums(uint32_t *sums, int tiles) {
    __shared__ uint32_t sh[32];
    const uint32_t v = (int) threadIdx.x < tiles ? sums[threadIdx.x] : 0u;
    const uint32_t e = block_exclusive_scan(v, sh, nullptr);
    if ((int) threadIdx.x < tiles)
        sums[threadIdx.x] = e;
}

__global__ void k_scan_tiles(uint32_t *count, int64_t m, const uint32_t *sums) {
    __shared__ uint32_t sh[32];
    const int64_t base = (int64_t) blockIdx.x * kScanTile + (int64_t) threadIdx.x * 4;
    uint32_t c[4], v = 0;
    for (int k = 0; k < 4; k++) {
        c[k] = base + k < m ? count[base + k] : 0u;
        v += c[k];
    }
    uint32_t run = sums[blockIdx.x] + block_exclusive_scan(v, sh, nullptr);
    for (int k = 0; k < 4; k++)
        if (base + k < m) {
            count[base + k] = run;
            run += c[k];
        }
}

__global__ void k_ray_scatter(const uint32_t *bucket, int64_t n, uint32_t *offset,
                              uint32_t *perm) {
    const int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const uint32_t pos = atomicAdd(offset + bucket[i], 1u);
    perm[pos] = (uint32_t) i;
}

// Bucket bits for n rays: about 8 rays per bucket, 2^8 .. 2^22 buckets (the
// scan handles at most 1024 tiles of 4096).
int ray_bucket_bits(int64_t n) {
    int b = 0;
    while (b < 30 && (int64_t(1) << b) < n)
        b++;
    return std::max(8, std::min(22, b - 3));
}

// Device bytes of the reordering scratch for n rays.
size_t ray_order_bytes(int64_t n) {
    const int64_t m = int64_t(1) << ray_bucket_bits(n);
    const int64_t tiles = (m + kScanTile - 1) / kScanTile;
    return (size_t) (2 * n + m + tiles) * sizeof(uint32_t);
}

// Fills perm[0, n) with the coherence order of the rays (scratch from
// ray_order_bytes(n), which starts with perm).
int ray_order(const float *o, const float *d, int64_t n, const float box[6], int mode,
              void *scratch, cudaStream_t st) {
    const int bits = ray_bucket_bits(n);
    const int64_t m = int64_t(1) << bits;
    const int64_t tiles = (m + kScanTile - 1) / kScanTile;
    uint32_t *perm = (uint32_t *) scratch;
    uint32_t *bucket = perm + n;
    uint32_t *count = bucket + n;
    uint32_t *sums = count + m;
    RayKeyArgs a;
    a.O = o;
    a.D = d;
    a.n = n;
    for (int k = 0; k < 6; k++)
        a.box[k] = box[k];
    a.mode = mode;
    a.shift = 30 - bits;
    a.bucket = bucket;
    a.count = count;
    PRR_CUDA_TRY(cudaMemsetAsync(count, 0, (size_t) m * sizeof(uint32_t), st));
    const unsigned g = (unsigned) ((n + 255) / 256);
    k_ray_buckets<<<g, 256, 0, st>>>(a);
    k_scan_tile_sums<<<(unsigned) tiles, 1024, 0, st>>>(count, m, sums);
    k_scan_sums<<<1, 1024, 0, st>>>(sums, (int) tiles);
    k_scan_tiles<<<(unsigned) tiles, 1024, 0, st>>>(count, m, sums);
    k_ray_scatter<<<g, 256, 0, st>>>(bucket, n, count, perm);
    PRR_CUDA_TRY(cudaGetLastError());
    return PRR_OK;
}

TraceBounds host_bounds(const DevScene &S) {
    return TraceBounds{S.n_nodes, S.n_tris, S.check};
}

int stack_cap(int depth) {
    // entries outstanding <= deepest leaf depth; keep one spare slot
    return std::max(1, depth + 1);
}

int grid_for(int64_t n, int block) {
    const int64_t g = (n + block - 1) / block;
    const int64_t cap = (int64_t) device_sm_count() * 64;
    return (int) std::max<int64_t>(1, std::min(g, cap));
}

int set_smem(const void *fn, size_t bytes) {
    // The stack columns live in shared memory: ask for the largest carveout so
    // the resident-block count the occupancy query reports is what launches.
    cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout,
                         cudaSharedmemCarveoutMaxShared);
    if (bytes > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int) bytes);
        if (e != cudaSuccess)
            return fail(PRR_ERR_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
    }
    return PRR_OK;
}

} // namespace

int device_sm_count() {
    static int sms = [] {
        int dev = 0, v = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0)
            v = 148;
        return v;
    }();
    return sms;
}

namespace {

// The traversal launch of launch_mesh_closest.
int trace_mesh_closest(MeshArgs &a, int mode, int block, size_t smem, unsigned *counter,
                       const prr_trace_config *cfg, int64_t n, cudaStream_t st) {
    if (mode > 0) {
        if (!counter)
            return fail(PRR_ERR_INVALID_ARGUMENT, "persistent launch needs a counter");
        const void *fn = mode == 1   ? (const void *) k_mesh_closest_persistent
                         : mode == 2 ? (const void *) k_mesh_closest_refill
                                     : (const void *) k_mesh_closest_phased;
        if (int rc = set_smem(fn, smem))
            return rc;
        int bps = cfg->blocks_per_sm > 0 ? cfg->blocks_per_sm : 0;
        if (bps == 0) {
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, fn, block, smem);
            bps = std::max(1, bps);
        }
        PRR_CUDA_TRY(cudaMemsetAsync(counter, 0, sizeof(unsigned long long), st));
        if (mode == 1) {
            k_mesh_closest_persistent<<<device_sm_count() * bps, block, smem, st>>>(a);
        } else if (mode == 2) {
            const int refill = cfg->batch > 0 ? std::min(cfg->batch, 32) : 8;
            k_mesh_closest_refill<<<device_sm_count() * bps, block, smem, st>>>(a, refill);
        } else {
            const int refill = cfg->batch > 0 ? std::min(cfg->batch, 32) : 8;
            const int tri_min = cfg->leaf_batch > 0 ? std::min(cfg->leaf_batch, 32) : 16;
            k_mesh_closest_phased<<<device_sm_count() * bps, block, smem, st>>>(a, refill,
                                                                              tri_min);
        }
    } else {
        if (int rc = set_smem((const void *) k_mesh_closest, smem))
            return rc;
        k_mesh_closest<<<grid_for(n, block), block, smem, st>>>(a);
    }
    PRR_CUDA_TRY(cudaGetLastError());
    return PRR_OK;
}

} // namespace

int launch_mesh_closest(const Scene &s, int object, const float *o, const float *d, int64_t n,
                        int32_t *id, float *t, double *t64, unsigned *counter,
                        const prr_trace_config *cfg, cudaStream_t st) {
    if (n == 0)
        return PRR_OK;
    const HostObject &obj = s.objects[object];
    MeshArgs a;
    a.nodes = s.dev.nodes;
    a.tris = s.dev.tris;
    a.e2z = s.dev.tri_e2z;
    a.meta = s.dev.tri_meta;
    a.verts = s.dev.verts;
    a.root = obj.root;
    a.O = o;
    a.D = d;
    a.n = n;
    a.out_id = id;
    a.out_t = t;
    a.out_t64 = t64;
    a.counter = (unsigned long long *) counter;
    a.perm = nullptr;
    const int block = (cfg && cfg->block_size > 0) ? cfg->block_size : 128;
    if (block % 32 != 0 || block > 1024)
        return fail(PRR_ERR_INVALID_ARGUMENT, "block_size must be a multiple of 32 <= 1024");
    const int cap = stack_cap(obj.bvh.max_depth);
    a.stack_stride = block;
    a.stack_cap = cap;
    a.B = host_bounds(s.dev);
    const size_t smem = (size_t) cap * block * sizeof(uint2);
    if (smem > 227 * 1024)
        return fail(PRR_ERR_UNSUPPORTED, "BVH too deep for the shared-memory stack");
    const int mode = cfg ? cfg->persistent : 0;
    if (mode < 0 || mode > 3)
        return fail(PRR_ERR_INVALID_ARGUMENT, "persistent must be 0, 1, 2 or 3");
    const int sort = cfg ? cfg->sort_rays : 0;
    if (sort < 0 || sort > 5)
        return fail(PRR_ERR_INVALID_ARGUMENT, "sort_rays must be 0 to 5");
    // reordering scratch from the library's stream-ordered pool, released on
    // the stream after the traversal (concurrent calls get their own)
    void *order = nullptr;
    if (sort > 0 && n < (int64_t(1) << 31)) {
        cudaMemPool_t pool;
        PRR_CUDA_TRY(library_pool(&pool));
        PRR_CUDA_TRY(cudaMallocFromPoolAsync(&order, ray_order_bytes(n), pool, st));
        float box[6];
        for (int k = 0; k < 6; k++)
            box[k] = obj.bvh.bounds[k];
        if (int rc = ray_order(o, d, n, box, sort, order, st)) {
            cudaFreeAsync(order, st);
            return rc;
        }
        a.perm = (const uint32_t *) order;
    }
    const int rc = trace_mesh_closest(a, mode, block, smem, counter, cfg, n, st);
    if (order)
        cudaFreeAsync(order, st);
    return rc;
}

int launch_mesh_occluded(const Scene &s, int object, const float *o, const float *d,
                         const float *tmax, int64_t n, uint8_t *hit, cudaStream_t st) {
    if (n == 0)
        return PRR_OK;
    const HostObject &obj = s.objects[object];
    DevObject dobj{};
    for (int k = 0; k < 6; k++)
        dobj.root_box[k] = obj.bvh.bounds[k];
    const int block = 128;
    const size_t smem = (size_t) stack_cap(obj.bvh.max_depth) * block * sizeof(uint2);
    if (smem > 227 * 1024)
        return fail(PRR_ERR_UNSUPPORTED, "BVH too deep for the shared-memory stack");
    if (int rc = set_smem((const void *) k_mesh_occluded, smem))
        return rc;
    k_mesh_occluded<<<grid_for(n, block), block, smem, st>>>(s.dev.nodes, s.dev.tris,
                                                             s.dev.tri_e2z, obj.root,
                                                             dobj, o, d, tmax, n, hit,
                                                             host_bounds(s.dev),
                                                             stack_cap(obj.bvh.max_depth));
    PRR_CUDA_TRY(cudaGetLastError());
    return PRR_OK;
}

int launch_scene_closest(const Scene &s, const float *o, const float *d, int64_t n,
                         int32_t *obj, int32_t *prim, float *t, float *geo, cudaStream_t st) {
    if (n == 0)
        return PRR_OK;
    const int block = 128;
    const int tcap = stack_cap(s.dev.tlas_depth), bcap = stack_cap(s.dev.blas_depth);
    const size_t smem = (size_t) (tcap + bcap) * block * sizeof(uint2);
    if (smem > 227 * 1024)
        return fail(PRR_ERR_UNSUPPORTED, "BVH too deep for the shared-memory stack");
    if (int rc = set_smem((const void *) k_scene_closest, smem))
        return rc;
    k_scene_closest<<<grid_for(n, block), block, smem, st>>>(s.dev, o, d, n, obj, prim, t, geo,
                                                             tcap);
    PRR_CUDA_TRY(cudaGetLastError());
    return PRR_OK;
}

int launch_scene_occluded(const Scene &s, const float *o, const float *d, const float *tmax,
                          int64_t n, uint8_t *hit, cudaStream_t st) {
    if (n == 0)
        return PRR_OK;
    const int block = 128;
    const int tcap = stack_cap(s.dev.tlas_depth), bcap = stack_cap(s.dev.blas_depth);
    const size_t smem = (size_t) (tcap + bcap) * block * sizeof(uint2);
    if (smem > 227 * 1024)
        return fail(PRR_ERR_UNSUPPORTED, "BVH too deep for the shared-memory stack");
    if (int rc = set_smem((const void *) k_scene_occluded, smem))
        return rc;
    k_scene_occluded<<<grid_for(n, block), block, smem, st>>>(s.dev, o, d, tmax, n, hit, tcap);
    PRR_CUDA_TRY(cudaGetLastError());
    return PRR_OK;
}

} // namespace prr
