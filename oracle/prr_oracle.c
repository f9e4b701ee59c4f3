/*
 * prr_oracle.c -- test infrastructure only (the oracle): a plain-C CPU
 * restatement of the reference renderer's closest-hit path and the numeric
 * kernels beside it. See prr_oracle.h. Built with -ffp-contract=off so every
 * float operation rounds like the reference's IEEE build.
 */
#include "prr_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define PRR_PI 3.141592653589793f /* global.hpp:10 */

typedef struct {
    float x, y, z;
} v3;

static inline v3 mk(float x, float y, float z) {
    v3 r = {x, y, z};
    return r;
}
static inline v3 sub(v3 a, v3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 add(v3 a, v3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline float dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3 cross(v3 a, v3 b) {
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline float at(v3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
/* std::min / std::max as libstdc++ defines them: min(a,b) = b<a ? b : a. */
static inline float smin(float a, float b) { return (b < a) ? b : a; }
static inline float smax(float a, float b) { return (a < b) ? b : a; }

/* ------------------------------------------------------------------------ */
/* RNG: counter-keyed SplitMix64 in the output form of global.hpp:35-50.     */
/* ------------------------------------------------------------------------ */
static inline uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

uint64_t prr_oracle_path_state(uint64_t seed, uint32_t stream, uint32_t index) {
    return mix64(mix64(seed ^ 0x6A09E667F3BCC909ULL) ^ (((uint64_t) stream << 32) | index));
}

float prr_oracle_rand(uint64_t *state) {
    uint64_t z = (*state += 0x9E3779B97F4A7C15ULL);
    z = mix64(z);
    return (float) (z >> 40) * 0x1p-24f;
}

void prr_oracle_rng_stream(uint64_t seed, uint32_t stream, uint32_t index, int n, float *out) {
    uint64_t s = prr_oracle_path_state(seed, stream, index);
    for (int i = 0; i < n; i++)
        out[i] = prr_oracle_rand(&s);
}

/* ------------------------------------------------------------------------ */
/* Bounds3 (Bounds3.hpp:13-126)                                              */
/* ------------------------------------------------------------------------ */
typedef struct {
    v3 mn, mx;
} box;

static inline box box_empty(void) {
    /* Bounds3() stores +-DBL_MAX converted to float: +-inf (Bounds3.hpp:15-20). */
    box b = {mk(INFINITY, INFINITY, INFINITY), mk(-INFINITY, -INFINITY, -INFINITY)};
    return b;
}
static inline box box_union(box a, box b) {
    box r;
    r.mn = mk(smin(a.mn.x, b.mn.x), smin(a.mn.y, b.mn.y), smin(a.mn.z, b.mn.z));
    r.mx = mk(smax(a.mx.x, b.mx.x), smax(a.mx.y, b.mx.y), smax(a.mx.z, b.mx.z));
    return r;
}
static inline box box_union_pt(box a, v3 p) {
    box r;
    r.mn = mk(smin(a.mn.x, p.x), smin(a.mn.y, p.y), smin(a.mn.z, p.z));
    r.mx = mk(smax(a.mx.x, p.x), smax(a.mx.y, p.y), smax(a.mx.z, p.z));
    return r;
}
static inline v3 box_centroid(box b) {
    /* 0.5 * pMin + 0.5 * pMax with the float friend operator* (Bounds3.hpp:48). */
    return mk(b.mn.x * 0.5f + b.mx.x * 0.5f, b.mn.y * 0.5f + b.mx.y * 0.5f,
              b.mn.z * 0.5f + b.mx.z * 0.5f);
}
static inline float box_area(box b) {
    /* SurfaceArea (Bounds3.hpp:43-47): float arithmetic, returned as double. */
    v3 d = sub(b.mx, b.mn);
    return 2 * (d.x * d.y + d.x * d.z + d.y * d.z);
}
static inline int box_max_extent(box b) {
    v3 d = sub(b.mx, b.mn);
    if (d.x > d.y && d.x > d.z)
        return 0;
    else if (d.y > d.z)
        return 1;
    return 2;
}

/* ------------------------------------------------------------------------ */
/* SAH build (BVH.cpp:66-256) and DFS flatten (BVH.cpp:263-280)               */
/* ------------------------------------------------------------------------ */
typedef struct {
    box bounds;
    int64_t child[2];
    int split_axis;
    int64_t prim_offset;
    int64_t prim_count;
    float area;
} bnode;

typedef struct {
    const box *pb; /* prim bounds */
    const float *pa;
    int max_prims;
    int32_t *work;
    bnode *pool;
    int64_t npool;
    box *tmp_bounds;
    v3 *tmp_cent;
    int32_t *tmp_idx;
} builder;

static inline float cent_key(const builder *B, int32_t prim, int axis) {
    return at(box_centroid(B->pb[prim]), axis);
}

/* libstdc++ std::nth_element (introselect) as the reference build sees it: it
 * is only reached with 2..4 prims (BVH.cpp:241-250), where introselect is a
 * single median-of-three partition step for n == 4 followed by insertion sort. */
static void nth_small(builder *B, int32_t *first, int32_t *nth, int32_t *last, int axis) {
#define KEY(p) cent_key(B, *(p), axis)
#define LESS(a, b) (KEY(a) < KEY(b))
#define SWAP(a, b)                                                                               \
    do {                                                                                         \
        int32_t t__ = *(a);                                                                      \
        *(a) = *(b);                                                                             \
        *(b) = t__;                                                                              \
    } while (0)
    if (first == last || nth == last)
        return;
    while (last - first > 3) {
        int32_t *mid = first + (last - first) / 2;
        int32_t *a = first + 1, *b = mid, *c = last - 1;
        if (LESS(a, b)) {
            if (LESS(b, c))
                SWAP(first, b);
            else if (LESS(a, c))
                SWAP(first, c);
            else
                SWAP(first, a);
        } else if (LESS(a, c))
            SWAP(first, a);
        else if (LESS(b, c))
            SWAP(first, c);
        else
            SWAP(first, b);
        int32_t *lo = first + 1, *hi = last;
        for (;;) {
            while (LESS(lo, first))
                ++lo;
            --hi;
            while (LESS(first, hi))
                --hi;
            if (!(lo < hi))
                break;
            SWAP(lo, hi);
            ++lo;
        }
        if (lo <= nth)
            first = lo;
        else
            last = lo;
    }
    /* insertion sort */
    for (int32_t *i = first + 1; i < last; ++i) {
        int32_t val = *i;
        float kv = cent_key(B, val, axis);
        if (kv < KEY(first)) {
            memmove(first + 1, first, (size_t) (i - first) * sizeof(int32_t));
            *first = val;
        } else {
            int32_t *j = i;
            while (kv < KEY(j - 1)) {
                *j = *(j - 1);
                --j;
            }
            *j = val;
        }
    }
#undef KEY
#undef LESS
#undef SWAP
}

static int64_t build_rec(builder *B, int64_t start, int64_t end) {
    int64_t me = B->npool++;
    bnode *node = &B->pool[me];
    memset(node, 0, sizeof(*node));
    node->child[0] = node->child[1] = -1;
    const int64_t count = end - start;

    box bounds = box_empty(), cb = box_empty();
    box *pbs = B->tmp_bounds + start; /* per-range caches, as BVH.cpp:77-86 */
    v3 *pcs = B->tmp_cent + start;
    for (int64_t i = 0; i < count; i++) {
        pbs[i] = B->pb[B->work[start + i]];
        pcs[i] = box_centroid(pbs[i]);
        bounds = box_union(bounds, pbs[i]);
        cb = box_union_pt(cb, pcs[i]);
    }
    node->bounds = bounds;

    if (count == 1) {
        node->prim_offset = start;
        node->prim_count = 1;
        node->area = B->pa[B->work[start]];
        return me;
    }
    if (count <= B->max_prims) {
        node->prim_offset = start;
        node->prim_count = count;
        node->area = 0.f;
        for (int64_t i = start; i < end; i++)
            node->area += B->pa[B->work[i]];
        return me;
    }

    const int axis = box_max_extent(cb);
    node->split_axis = axis;
    int64_t mid = (start + end) / 2;

    if (at(cb.mx, axis) == at(cb.mn, axis)) {
        /* degenerate centroids: median split, no reordering (BVH.cpp:120-133) */
    } else if (count > 4) {
        enum { NB = 12 };
        float best_cost = INFINITY;
        int best_axis = axis, best_split = NB / 2;
        const float parent_area = box_area(bounds);
        for (int a = 0; a < 3; a++) {
            float lo = at(cb.mn, a), hi = at(cb.mx, a);
            if (lo == hi)
                continue;
            int bc[NB];
            box bb[NB];
            for (int k = 0; k < NB; k++) {
                bc[k] = 0;
                bb[k] = box_empty();
            }
            const float span = hi - lo;
            for (int64_t i = 0; i < count; i++) {
                int b = (int) (NB * (at(pcs[i], a) - lo) / span);
                b = b < 0 ? 0 : (b > NB - 1 ? NB - 1 : b);
                bc[b]++;
                bb[b] = box_union(bb[b], pbs[i]);
            }
            float la[NB - 1], ra[NB - 1];
            int lc[NB - 1], rc[NB - 1];
            box bl = box_empty();
            int cl = 0;
            for (int k = 0; k < NB - 1; k++) {
                bl = box_union(bl, bb[k]);
                cl += bc[k];
                la[k] = box_area(bl);
                lc[k] = cl;
            }
            box br = box_empty();
            int cr = 0;
            for (int k = NB - 2; k >= 0; k--) {
                br = box_union(br, bb[k + 1]);
                cr += bc[k + 1];
                ra[k] = box_area(br);
                rc[k] = cr;
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
        float lo = at(cb.mn, best_axis);
        float span = at(cb.mx, best_axis) - lo;
        float edge = lo + (best_split + 1) * span / NB;
        /* stable partition (BVH.cpp:217-240) */
        int64_t nl = 0;
        for (int64_t i = 0; i < count; i++)
            if (at(pcs[i], best_axis) < edge)
                nl++;
        if (nl > 0 && nl < count) {
            int32_t *tmp = B->tmp_idx + start;
            int64_t wl = 0, wr = nl;
            for (int64_t i = 0; i < count; i++) {
                if (at(pcs[i], best_axis) < edge)
                    tmp[wl++] = B->work[start + i];
                else
                    tmp[wr++] = B->work[start + i];
            }
            memcpy(B->work + start, tmp, sizeof(int32_t) * count);
            mid = start + nl;
        }
    } else {
        nth_small(B, B->work + start, B->work + mid, B->work + end, axis);
    }

    int64_t c0 = build_rec(B, start, mid);
    int64_t c1 = build_rec(B, mid, end);
    node = &B->pool[me];
    node->child[0] = c0;
    node->child[1] = c1;
    node->area = B->pool[c0].area + B->pool[c1].area;
    return me;
}

static uint32_t flatten_rec(const builder *B, int64_t bn, uint32_t *offset, float *nb,
                            uint32_t *fc, uint32_t *meta, float *na) {
    const bnode *node = &B->pool[bn];
    uint32_t my = (*offset)++;
    float *b = nb + (size_t) my * 6;
    b[0] = node->bounds.mn.x;
    b[1] = node->bounds.mx.x;
    b[2] = node->bounds.mn.y;
    b[3] = node->bounds.mx.y;
    b[4] = node->bounds.mn.z;
    b[5] = node->bounds.mx.z;
    na[my] = node->area;
    if (node->prim_count > 0) {
        fc[my] = (uint32_t) node->prim_offset;
        meta[my] = (uint32_t) node->prim_count & 0x00FFFFFFu;
    } else {
        meta[my] = (uint32_t) node->split_axis << 24;
        flatten_rec(B, node->child[0], offset, nb, fc, meta, na);
        fc[my] = flatten_rec(B, node->child[1], offset, nb, fc, meta, na);
    }
    return my;
}

int64_t prr_oracle_bvh_build(const float *prim_bounds, const float *prim_area, int64_t n,
                             int max_prims, float *node_bounds, uint32_t *first_child,
                             uint32_t *meta, float *node_area, int32_t *ordered) {
    if (n <= 0)
        return 0;
    builder B;
    memset(&B, 0, sizeof(B));
    box *pb = (box *) malloc(sizeof(box) * n);
    for (int64_t i = 0; i < n; i++) {
        const float *p = prim_bounds + i * 6;
        pb[i].mn = mk(p[0], p[1], p[2]);
        pb[i].mx = mk(p[3], p[4], p[5]);
    }
    B.pb = pb;
    B.pa = prim_area;
    B.max_prims = max_prims < 255 ? max_prims : 255;
    B.work = (int32_t *) malloc(sizeof(int32_t) * n);
    for (int64_t i = 0; i < n; i++)
        B.work[i] = (int32_t) i;
    B.pool = (bnode *) malloc(sizeof(bnode) * (2 * n));
    B.tmp_bounds = (box *) malloc(sizeof(box) * n);
    B.tmp_cent = (v3 *) malloc(sizeof(v3) * n);
    B.tmp_idx = (int32_t *) malloc(sizeof(int32_t) * n);
    build_rec(&B, 0, n);
    uint32_t off = 0;
    flatten_rec(&B, 0, &off, node_bounds, first_child, meta, node_area);
    if (ordered)
        memcpy(ordered, B.work, sizeof(int32_t) * n);
    int64_t nn = B.npool;
    free(pb);
    free(B.work);
    free(B.pool);
    free(B.tmp_bounds);
    free(B.tmp_cent);
    free(B.tmp_idx);
    return nn;
}

void prr_oracle_triangle_prims(const float *verts, int64_t n, float *prim_bounds, float *area) {
    for (int64_t i = 0; i < n; i++) {
        const float *p = verts + i * 9;
        v3 v0 = mk(p[0], p[1], p[2]), v1 = mk(p[3], p[4], p[5]), v2 = mk(p[6], p[7], p[8]);
        /* Union(Bounds3(v0, v1), v2) (Triangle.hpp:183-185) */
        box b;
        b.mn = mk(fminf(v0.x, v1.x), fminf(v0.y, v1.y), fminf(v0.z, v1.z));
        b.mx = mk(fmaxf(v0.x, v1.x), fmaxf(v0.y, v1.y), fmaxf(v0.z, v1.z));
        b = box_union_pt(b, v2);
        float *o = prim_bounds + i * 6;
        o[0] = b.mn.x;
        o[1] = b.mn.y;
        o[2] = b.mn.z;
        o[3] = b.mx.x;
        o[4] = b.mx.y;
        o[5] = b.mx.z;
        /* area = |e1 x e2| * 0.5 (Triangle.hpp:30-36) */
        v3 c = cross(sub(v1, v0), sub(v2, v0));
        area[i] = sqrtf(c.x * c.x + c.y * c.y + c.z * c.z) * 0.5f;
    }
}

/* ------------------------------------------------------------------------ */
/* Mesh closest hit / any hit                                                */
/* ------------------------------------------------------------------------ */
typedef struct {
    v3 v0, e1, e2;
    int32_t id;
} otri;

struct prr_oracle_mesh {
    int64_t nnodes, ntri;
    float *nb;
    uint32_t *fc, *meta;
    float *na;
    int32_t *ordered;
    otri *tris; /* in orderedPrims order */
    const float *src;
    float *verts;
};

prr_oracle_mesh *prr_oracle_mesh_new(const float *verts, int64_t ntri) {
    prr_oracle_mesh *m = (prr_oracle_mesh *) calloc(1, sizeof(*m));
    m->ntri = ntri;
    float *pb = (float *) malloc(sizeof(float) * 6 * ntri);
    float *pa = (float *) malloc(sizeof(float) * ntri);
    prr_oracle_triangle_prims(verts, ntri, pb, pa);
    m->nb = (float *) malloc(sizeof(float) * 6 * (2 * ntri));
    m->fc = (uint32_t *) malloc(sizeof(uint32_t) * (2 * ntri));
    m->meta = (uint32_t *) malloc(sizeof(uint32_t) * (2 * ntri));
    m->na = (float *) malloc(sizeof(float) * (2 * ntri));
    m->ordered = (int32_t *) malloc(sizeof(int32_t) * ntri);
    m->nnodes = prr_oracle_bvh_build(pb, pa, ntri, 4, m->nb, m->fc, m->meta, m->na, m->ordered);
    free(pb);
    free(pa);
    m->verts = (float *) malloc(sizeof(float) * 9 * ntri);
    memcpy(m->verts, verts, sizeof(float) * 9 * ntri);
    m->tris = (otri *) malloc(sizeof(otri) * ntri);
    for (int64_t k = 0; k < ntri; k++) {
        int32_t id = m->ordered[k];
        const float *p = verts + (int64_t) id * 9;
        v3 v0 = mk(p[0], p[1], p[2]), v1 = mk(p[3], p[4], p[5]), v2 = mk(p[6], p[7], p[8]);
        m->tris[k].v0 = v0;
        m->tris[k].e1 = sub(v1, v0); /* Triangle.hpp:29-30 */
        m->tris[k].e2 = sub(v2, v0);
        m->tris[k].id = id;
    }
    return m;
}

void prr_oracle_mesh_free(prr_oracle_mesh *m) {
    if (!m)
        return;
    free(m->nb);
    free(m->fc);
    free(m->meta);
    free(m->na);
    free(m->ordered);
    free(m->tris);
    free(m->verts);
    free(m);
}

int64_t prr_oracle_mesh_nodes(const prr_oracle_mesh *m, float *bounds, uint32_t *first_child,
                              uint32_t *meta, float *areas, int32_t *ordered) {
    if (bounds)
        memcpy(bounds, m->nb, sizeof(float) * 6 * m->nnodes);
    if (first_child)
        memcpy(first_child, m->fc, sizeof(uint32_t) * m->nnodes);
    if (meta)
        memcpy(meta, m->meta, sizeof(uint32_t) * m->nnodes);
    if (areas)
        memcpy(areas, m->na, sizeof(float) * m->nnodes);
    if (ordered)
        memcpy(ordered, m->ordered, sizeof(int32_t) * m->ntri);
    return m->nnodes;
}

typedef struct {
    float org[3], inv[3];
    int oct[3];
} rdata;

static inline rdata precompute(v3 o, v3 d) {
    /* BVH.cpp:290-299 */
    rdata r;
    for (int a = 0; a < 3; a++) {
        float dd = at(d, a);
        r.org[a] = at(o, a);
        r.inv[a] = (dd != 0.f) ? (1.f / dd) : INFINITY;
        r.oct[a] = (dd < 0.f) ? 1 : 0;
    }
    return r;
}

static inline float node_isect(const float *b, const rdata *r) {
    /* BVH.hpp:115-124 */
    float tmin = 0.f, tmax = INFINITY;
    for (int a = 0; a < 3; a++) {
        float t0 = (b[a * 2 + r->oct[a]] - r->org[a]) * r->inv[a];
        float t1 = (b[a * 2 + 1 - r->oct[a]] - r->org[a]) * r->inv[a];
        tmin = smax(tmin, t0);
        tmax = smin(tmax, t1);
    }
    return tmin <= tmax ? tmin : INFINITY;
}

/* Triangle::hitTest (Triangle.hpp:46-64): returns t or a negative miss. */
static inline int tri_hit(const otri *tr, v3 o, v3 d, float *t, float *u, float *v) {
    v3 P = cross(d, tr->e2);
    float det = dot(P, tr->e1);
    if (fabsf(det) < 1e-6f)
        return 0;
    float inv = 1.f / det;
    v3 T = sub(o, tr->v0);
    float uu = dot(P, T) * inv;
    if (uu < 0.f)
        return 0;
    v3 Q = cross(T, tr->e1);
    float vv = dot(Q, d) * inv;
    if (vv < 0.f || uu + vv > 1.f)
        return 0;
    float tt = dot(Q, tr->e2) * inv;
    if (tt <= 1e-3f)
        return 0;
    *t = tt;
    *u = uu;
    *v = vv;
    return 1;
}

/* Triangle::intersectT (Triangle.hpp:75-92) */
static inline float tri_hit_t(const otri *tr, v3 o, v3 d, float tmax) {
    v3 P = cross(d, tr->e2);
    float det = dot(P, tr->e1);
    if (fabsf(det) < 1e-6f)
        return -1.f;
    float inv = 1.f / det;
    v3 T = sub(o, tr->v0);
    float uu = dot(P, T) * inv;
    if (uu < 0.f || uu > 1.f)
        return -1.f;
    v3 Q = cross(T, tr->e1);
    float vv = dot(Q, d) * inv;
    if (vv < 0.f || uu + vv > 1.f)
        return -1.f;
    float tt = dot(Q, tr->e2) * inv;
    return (tt > 1e-3f && tt < tmax) ? tt : -1.f;
}

/* Möller-Trumbore in fp64 on the input vertices: the t reference for the
 * 1e-6 relative bar. */
static double tri_t64(const float *p, v3 of, v3 df) {
    double v0[3] = {p[0], p[1], p[2]}, v1[3] = {p[3], p[4], p[5]}, v2[3] = {p[6], p[7], p[8]};
    double o[3] = {of.x, of.y, of.z}, d[3] = {df.x, df.y, df.z};
    double e1[3], e2[3], T[3], P[3], Q[3];
    for (int k = 0; k < 3; k++) {
        e1[k] = v1[k] - v0[k];
        e2[k] = v2[k] - v0[k];
        T[k] = o[k] - v0[k];
    }
    P[0] = d[1] * e2[2] - d[2] * e2[1];
    P[1] = d[2] * e2[0] - d[0] * e2[2];
    P[2] = d[0] * e2[1] - d[1] * e2[0];
    Q[0] = T[1] * e1[2] - T[2] * e1[1];
    Q[1] = T[2] * e1[0] - T[0] * e1[2];
    Q[2] = T[0] * e1[1] - T[1] * e1[0];
    double det = P[0] * e1[0] + P[1] * e1[1] + P[2] * e1[2];
    return (Q[0] * e2[0] + Q[1] * e2[1] + Q[2] * e2[2]) / det;
}

/* BVHAccel::Intersect, triangle fast path (BVH.cpp:311-415). */
static int32_t closest(const prr_oracle_mesh *m, v3 o, v3 d, float *tout, int32_t *nvis,
                       int32_t *ntest) {
    if (m->nnodes == 0) {
        *tout = INFINITY;
        return -1;
    }
    rdata rd = precompute(o, d);
    uint32_t st_idx[64];
    float st_t[64];
    int sp = 0;
    uint32_t ni = 0;
    float closest_t = INFINITY;
    int64_t hit = -1;
    int32_t vis = 0, tst = 0;
    for (;;) {
        uint32_t meta = m->meta[ni];
        uint32_t cnt = meta & 0x00FFFFFFu;
        if (cnt > 0) {
            for (uint32_t i = 0; i < cnt; i++) {
                const otri *tr = &m->tris[m->fc[ni] + i];
                float t, u, v;
                tst++;
                if (tri_hit(tr, o, d, &t, &u, &v) && t < closest_t) {
                    closest_t = t;
                    hit = m->fc[ni] + i;
                }
            }
        } else {
            vis++;
            uint32_t left = ni + 1, right = m->fc[ni];
            float tl = node_isect(m->nb + (size_t) left * 6, &rd);
            float tr = node_isect(m->nb + (size_t) right * 6, &rd);
            if (tl <= tr) {
                if (tl < closest_t) {
                    if (tr < closest_t) {
                        st_idx[sp] = right;
                        st_t[sp++] = tr;
                    }
                    ni = left;
                    continue;
                }
            } else {
                if (tr < closest_t) {
                    if (tl < closest_t) {
                        st_idx[sp] = left;
                        st_t[sp++] = tl;
                    }
                    ni = right;
                    continue;
                }
            }
        }
        for (;;) {
            if (sp == 0)
                goto done;
            ni = st_idx[--sp];
            if (st_t[sp] < closest_t)
                break;
        }
    }
done:
    *tout = closest_t;
    if (nvis)
        *nvis = vis;
    if (ntest)
        *ntest = tst;
    return hit < 0 ? -1 : m->tris[hit].id;
}

void prr_oracle_mesh_intersect(const prr_oracle_mesh *m, const float *o, const float *d,
                               int64_t n, int32_t *id, float *t, double *t64, int32_t *visits,
                               int32_t *tests, int nthreads) {
#pragma omp parallel for schedule(dynamic, 1024) num_threads(nthreads > 0 ? nthreads : 1)
    for (int64_t i = 0; i < n; i++) {
        v3 oo = mk(o[i * 3], o[i * 3 + 1], o[i * 3 + 2]);
        v3 dd = mk(d[i * 3], d[i * 3 + 1], d[i * 3 + 2]);
        float tt;
        int32_t nv = 0, nt = 0;
        int32_t h = closest(m, oo, dd, &tt, &nv, &nt);
        id[i] = h;
        t[i] = tt;
        if (t64)
            t64[i] = h < 0 ? NAN : tri_t64(m->verts + (int64_t) h * 9, oo, dd);
        if (visits)
            visits[i] = nv;
        if (tests)
            tests[i] = nt;
    }
}

/* BVHAccel::IntersectP (BVH.cpp:421-473) over Triangle::intersectT. */
static int occluded(const prr_oracle_mesh *m, v3 o, v3 d, float tmax) {
    if (m->nnodes == 0)
        return 0;
    rdata rd = precompute(o, d);
    uint32_t st[64];
    int sp = 0;
    uint32_t ni = 0;
    for (;;) {
        float tb = node_isect(m->nb + (size_t) ni * 6, &rd);
        if (tb < tmax) {
            uint32_t cnt = m->meta[ni] & 0x00FFFFFFu;
            if (cnt > 0) {
                for (uint32_t i = 0; i < cnt; i++) {
                    float t = tri_hit_t(&m->tris[m->fc[ni] + i], o, d, tmax);
                    if (t >= 0.f && t < tmax)
                        return 1;
                }
            } else {
                uint32_t left = ni + 1, right = m->fc[ni];
                uint32_t axis = m->meta[ni] >> 24;
                uint32_t nearc, farc;
                if (rd.oct[axis] == 0) {
                    nearc = left;
                    farc = right;
                } else {
                    nearc = right;
                    farc = left;
                }
                if (node_isect(m->nb + (size_t) farc * 6, &rd) < tmax)
                    st[sp++] = farc;
                ni = nearc;
                continue;
            }
        }
        if (sp == 0)
            break;
        ni = st[--sp];
    }
    return 0;
}

void prr_oracle_mesh_occluded(const prr_oracle_mesh *m, const float *o, const float *d,
                              const float *tmax, int64_t n, uint8_t *hit, int nthreads) {
#pragma omp parallel for schedule(dynamic, 1024) num_threads(nthreads > 0 ? nthreads : 1)
    for (int64_t i = 0; i < n; i++) {
        v3 oo = mk(o[i * 3], o[i * 3 + 1], o[i * 3 + 2]);
        v3 dd = mk(d[i * 3], d[i * 3 + 1], d[i * 3 + 2]);
        hit[i] = (uint8_t) occluded(m, oo, dd, tmax[i]);
    }
}

/* ------------------------------------------------------------------------ */
/* Display transform                                                         */
/* ------------------------------------------------------------------------ */
static inline float clampf(float x, float lo, float hi) {
    /* std::clamp(v, lo, hi) = v < lo ? lo : (hi < v ? hi : v) */
    return x < lo ? lo : (hi < x ? hi : x);
}

static inline float srgb_oetf(float x) { /* ToneMapping.hpp:45-48 */
    x = clampf(x, 0.f, 1.f);
    return x < 0.0031308f ? 12.92f * x : 1.055f * powf(x, 1.f / 2.4f) - 0.055f;
}

typedef struct {
    float contrast, toe_a, slope, w, shoulder_max, output_max;
} allenwp;
static const float CROSSOVER = 0.1841865f;

static allenwp allenwp_params(float contrast, float high_clip_in, float output_max) {
    /* ToneMapping.hpp:125-147 */
    allenwp p;
    p.contrast = contrast;
    p.output_max = output_max;
    float high_clip = smax(high_clip_in, output_max);
    p.toe_a = ((1.f / CROSSOVER) - 1.f) * powf(CROSSOVER, contrast);
    float denom = powf(CROSSOVER, contrast) + p.toe_a;
    p.slope = (contrast * powf(CROSSOVER, contrast - 1.f) * p.toe_a) / (denom * denom);
    p.shoulder_max = output_max - CROSSOVER;
    p.w = high_clip - CROSSOVER;
    p.w = p.w * p.w;
    p.w = p.w / p.shoulder_max;
    p.w = p.w * p.slope;
    return p;
}

static float allenwp_curve(float x, const allenwp *p) { /* ToneMapping.hpp:151-166 */
    x = smax(x, 0.f);
    if (x < CROSSOVER) {
        float t = powf(x, p->contrast);
        return t / (t + p->toe_a);
    }
    float s = x - CROSSOVER;
    float slope_s = p->slope * s;
    s = slope_s * (1.f + s / p->w) / (1.f + (slope_s / p->shoulder_max));
    s += CROSSOVER;
    return s;
}

static v3 mat3mul(const float m[3][3], v3 v) {
    return mk(m[0][0] * v.x + m[0][1] * v.y + m[0][2] * v.z,
              m[1][0] * v.x + m[1][1] * v.y + m[1][2] * v.z,
              m[2][0] * v.x + m[2][1] * v.y + m[2][2] * v.z);
}

static v3 agx(v3 c) { /* ToneMapping.hpp:172-214 */
    static const float inset[3][3] = {{0.544814746488245f, 0.373787398372697f, 0.0813978551390581f},
                                      {0.140416948464053f, 0.754137554567394f, 0.105445496968552f},
                                      {0.0888104196149096f, 0.178871756420858f, 0.732317823964232f}};
    static const float outset[3][3] = {
        {1.96488741169489f, -0.855988495690215f, -0.108898916004672f},
        {-0.299313364904742f, 1.32639796461980f, -0.0270845997150571f},
        {-0.164352742528393f, -0.238183969428088f, 1.40253671195648f}};
    allenwp p = allenwp_params(1.25f, 16.0f, 1.0f);
    c.x = smax(c.x, 0.f);
    c.y = smax(c.y, 0.f);
    c.z = smax(c.z, 0.f);
    c = mat3mul(inset, c);
    c = mk(allenwp_curve(c.x, &p), allenwp_curve(c.y, &p), allenwp_curve(c.z, &p));
    c.x = smin(1.0f, c.x);
    c.y = smin(1.0f, c.y);
    c.z = smin(1.0f, c.z);
    c = mat3mul(outset, c);
    c = mk(clampf(c.x, 0.f, 1.f), clampf(c.y, 0.f, 1.f), clampf(c.z, 0.f, 1.f));
    return mk(srgb_oetf(c.x), srgb_oetf(c.y), srgb_oetf(c.z));
}

static v3 pbr_neutral(v3 c) { /* ToneMapping.hpp:234-262 */
    const float start = 0.8f - 0.04f;
    const float desat = 0.15f;
    float x = smin(c.x, smin(c.y, c.z));
    float offset = x < 0.08f ? x - 6.25f * x * x : 0.04f;
    c.x -= offset;
    c.y -= offset;
    c.z -= offset;
    float peak = smax(c.x, smax(c.y, c.z));
    if (peak < start)
        return mk(srgb_oetf(c.x), srgb_oetf(c.y), srgb_oetf(c.z));
    float d = 1.f - start;
    float new_peak = 1.f - d * d / (peak + d - start);
    float scale = new_peak / peak;
    c.x *= scale;
    c.y *= scale;
    c.z *= scale;
    float g = 1.f - 1.f / (desat * (peak - new_peak) + 1.f);
    c.x = c.x * (1.f - g) + new_peak * g;
    c.y = c.y * (1.f - g) + new_peak * g;
    c.z = c.z * (1.f - g) + new_peak * g;
    return mk(srgb_oetf(c.x), srgb_oetf(c.y), srgb_oetf(c.z));
}

/* ACES filmic fit of K. Narkowicz (2015), "ACES Filmic Tone Mapping Curve":
 * f(x) = x(2.51x + 0.03) / (x(2.43x + 0.59) + 0.14), clamped, then the sRGB
 * OETF. The reference has no ACES operator; this one is new. */
static float aces1(float x) {
    float n = x * (2.51f * x + 0.03f);
    float dd = x * (2.43f * x + 0.59f) + 0.14f;
    return clampf(n / dd, 0.f, 1.f);
}

void prr_oracle_tonemap(int mapper, float exposure, const float *in, int64_t n, float *out,
                        uint8_t *out_u8) {
    for (int64_t i = 0; i < n; i++) {
        /* Renderer.cpp:149-161 */
        v3 c = mk(in[i * 3] * exposure, in[i * 3 + 1] * exposure, in[i * 3 + 2] * exposure);
        if (!isfinite(c.x))
            c.x = 0.f;
        if (!isfinite(c.y))
            c.y = 0.f;
        if (!isfinite(c.z))
            c.z = 0.f;
        c.x = smax(0.f, c.x);
        c.y = smax(0.f, c.y);
        c.z = smax(0.f, c.z);
        v3 r;
        switch (mapper) {
        case 0:
            r = mk(clampf(c.x, 0.f, 1.f), clampf(c.y, 0.f, 1.f), clampf(c.z, 0.f, 1.f));
            break;
        case 1:
            r = mk(srgb_oetf(c.x), srgb_oetf(c.y), srgb_oetf(c.z));
            break;
        case 2:
            r = agx(c);
            break;
        case 3:
            r = pbr_neutral(c);
            break;
        default:
            r = mk(srgb_oetf(aces1(c.x)), srgb_oetf(aces1(c.y)), srgb_oetf(aces1(c.z)));
            break;
        }
        if (out) {
            out[i * 3] = r.x;
            out[i * 3 + 1] = r.y;
            out[i * 3 + 2] = r.z;
        }
        if (out_u8) { /* Renderer.cpp:169-171 */
            out_u8[i * 3] = (uint8_t) (clampf(r.x, 0.f, 1.f) * 255.f + 0.5f);
            out_u8[i * 3 + 1] = (uint8_t) (clampf(r.y, 0.f, 1.f) * 255.f + 0.5f);
            out_u8[i * 3 + 2] = (uint8_t) (clampf(r.z, 0.f, 1.f) * 255.f + 0.5f);
        }
    }
}

/* ------------------------------------------------------------------------ */
/* EnvMap::buildCDF (EnvMap.hpp:189-224)                                      */
/* ------------------------------------------------------------------------ */
void prr_oracle_env_cdf(const float *rgb, int w, int h, float *cdf, float *marginal,
                        float *total_out) {
    float *row_sums = (float *) malloc(sizeof(float) * h);
    for (int row = 0; row < h; row++) {
        float theta = (row + 0.5f) / (float) h * PRR_PI;
        float sin_t = sinf(theta);
        float row_sum = 0.f;
        for (int col = 0; col < w; col++) {
            const float *p = rgb + ((int64_t) row * w + col) * 3;
            float lum = (0.2126f * p[0] + 0.7152f * p[1] + 0.0722f * p[2]) * sin_t;
            row_sum += lum;
            cdf[(int64_t) row * w + col] = row_sum;
        }
        if (row_sum > 0.f)
            for (int col = 0; col < w; col++)
                cdf[(int64_t) row * w + col] /= row_sum;
        row_sums[row] = row_sum;
    }
    float total = 0.f;
    for (int row = 0; row < h; row++) {
        total += row_sums[row];
        marginal[row] = total;
    }
    *total_out = total;
    if (total > 0.f)
        for (int row = 0; row < h; row++)
            marginal[row] /= total;
    free(row_sums);
}

/* ------------------------------------------------------------------------ */
/* Photon grid + fixed-radius irradiance (Photon.cpp:24-94), and the          */
/* k-nearest-capped variant: with more than k photons inside the radius, the  */
/* k smallest (distance, photon index) pairs, their powers added in the walk  */
/* order of the query, over pi r_k^2 (r_k the k-th smallest distance).        */
/* ------------------------------------------------------------------------ */
typedef struct {
    float d;
    int64_t i;
} knn_cand;

static int knn_cmp(const void *a, const void *b) {
    const knn_cand *x = (const knn_cand *) a, *y = (const knn_cand *) b;
    if (x->d != y->d)
        return x->d < y->d ? -1 : 1;
    return x->i < y->i ? -1 : (x->i > y->i);
}

/* pi r^2 as estimateIrradiance writes it (Photon.cpp:87): float throughout, as
 * the reference redefines M_PI as a float literal (global.hpp:9-10) */
static float disc_area(float r) {
    return PRR_PI * r * r;
}

void prr_oracle_photon_estimate_knn(const float *rec, int64_t n, float radius, int k,
                                    const float *q, int64_t nq, float *out, int32_t *inside,
                                    int32_t *grid_res) {
    if (n <= 0) {
        memset(out, 0, sizeof(float) * 3 * nq);
        if (inside)
            memset(inside, 0, sizeof(int32_t) * nq);
        return;
    }
    v3 bmin = mk(rec[0], rec[1], rec[2]), bmax = bmin;
    for (int64_t i = 0; i < n; i++) {
        const float *p = rec + i * 9;
        bmin.x = smin(bmin.x, p[0]);
        bmin.y = smin(bmin.y, p[1]);
        bmin.z = smin(bmin.z, p[2]);
        bmax.x = smax(bmax.x, p[0]);
        bmax.y = smax(bmax.y, p[1]);
        bmax.z = smax(bmax.z, p[2]);
    }
    bmin = sub(bmin, mk(0.01f, 0.01f, 0.01f));
    bmax = add(bmax, mk(0.01f, 0.01f, 0.01f));
    v3 ext = sub(bmax, bmin);
    int res = (int) (sqrtf(ext.x * ext.x + ext.y * ext.y + ext.z * ext.z) / radius);
    res = res > 200 ? 200 : res;
    res = res < 10 ? 10 : res;
    if (grid_res)
        *grid_res = res;
    v3 cs = mk(ext.x / (float) res, ext.y / (float) res, ext.z / (float) res);
    int64_t ncell = (int64_t) res * res * res;
    int32_t *cell = (int32_t *) malloc(sizeof(int32_t) * n);
    int64_t *start = (int64_t *) calloc(ncell + 1, sizeof(int64_t));
    for (int64_t i = 0; i < n; i++) {
        const float *p = rec + i * 9;
        /* worldToCell goes through a Vector3f of ints (Photon.cpp:8-12) */
        int cx = (int) (float) (int) ((p[0] - bmin.x) / cs.x);
        int cy = (int) (float) (int) ((p[1] - bmin.y) / cs.y);
        int cz = (int) (float) (int) ((p[2] - bmin.z) / cs.z);
        cell[i] = cx + cy * res + cz * res * res;
        start[cell[i] + 1]++;
    }
    for (int64_t c = 0; c < ncell; c++)
        start[c + 1] += start[c];
    int64_t *fill = (int64_t *) malloc(sizeof(int64_t) * ncell);
    memcpy(fill, start, sizeof(int64_t) * ncell);
    int64_t *order = (int64_t *) malloc(sizeof(int64_t) * n);
    for (int64_t i = 0; i < n; i++)
        order[fill[cell[i]]++] = i;
    const float area = disc_area(radius);
#pragma omp parallel
    {
        int64_t cap = 1024, sorted_cap = 0;
        knn_cand *cand = (knn_cand *) malloc(sizeof(knn_cand) * cap);
        knn_cand *sorted = NULL;
#pragma omp for schedule(dynamic, 256)
        for (int64_t j = 0; j < nq; j++) {
            v3 pos = mk(q[j * 3], q[j * 3 + 1], q[j * 3 + 2]);
            int x0 = (int) ((pos.x - radius - bmin.x) / cs.x);
            int y0 = (int) ((pos.y - radius - bmin.y) / cs.y);
            int z0 = (int) ((pos.z - radius - bmin.z) / cs.z);
            int x1 = (int) ((pos.x + radius - bmin.x) / cs.x);
            int y1 = (int) ((pos.y + radius - bmin.y) / cs.y);
            int z1 = (int) ((pos.z + radius - bmin.z) / cs.z);
            x0 = x0 > 0 ? x0 : 0;
            x1 = x1 < res - 1 ? x1 : res - 1;
            y0 = y0 > 0 ? y0 : 0;
            y1 = y1 < res - 1 ? y1 : res - 1;
            z0 = z0 > 0 ? z0 : 0;
            z1 = z1 < res - 1 ? z1 : res - 1;
            v3 e = mk(0.f, 0.f, 0.f);
            int64_t found = 0;
            for (int cx = x0; cx <= x1; cx++)
                for (int cy = y0; cy <= y1; cy++)
                    for (int cz = z0; cz <= z1; cz++) {
                        int64_t c = (int64_t) cx + (int64_t) cy * res + (int64_t) cz * res * res;
                        for (int64_t s = start[c]; s < start[c + 1]; s++) {
                            const float *p = rec + order[s] * 9;
                            v3 dd = sub(mk(p[0], p[1], p[2]), pos);
                            float dist = sqrtf(dd.x * dd.x + dd.y * dd.y + dd.z * dd.z);
                            if (dist <= radius) {
                                e = add(e, mk(p[6], p[7], p[8]));
                                if (found == cap) {
                                    cap *= 2;
                                    cand = (knn_cand *) realloc(cand, sizeof(knn_cand) * cap);
                                }
                                cand[found].d = dist;
                                cand[found].i = order[s];
                                found++;
                            }
                        }
                    }
            if (inside)
                inside[j] = (int32_t) found;
            float a = area;
            if (found == 0) {
                e = mk(0.f, 0.f, 0.f);
            } else if (k > 0 && found > k) {
                /* cand holds the candidates in walk order; the k-th smallest
                 * pair by a sorted copy, then the walk-order sum of the pairs
                 * at or below it */
                if (sorted_cap < found) {
                    sorted_cap = found;
                    sorted = (knn_cand *) realloc(sorted, sizeof(knn_cand) * sorted_cap);
                }
                memcpy(sorted, cand, sizeof(knn_cand) * (size_t) found);
                qsort(sorted, (size_t) found, sizeof(knn_cand), knn_cmp);
                const knn_cand kth = sorted[k - 1];
                e = mk(0.f, 0.f, 0.f);
                for (int64_t t = 0; t < found; t++)
                    if (knn_cmp(&cand[t], &kth) <= 0) {
                        const float *p = rec + cand[t].i * 9;
                        e = add(e, mk(p[6], p[7], p[8]));
                    }
                a = disc_area(kth.d);
            }
            out[j * 3] = e.x / a;
            out[j * 3 + 1] = e.y / a;
            out[j * 3 + 2] = e.z / a;
        }
        free(cand);
        free(sorted);
    }
    free(cell);
    free(start);
    free(fill);
    free(order);
}

void prr_oracle_photon_estimate(const float *rec, int64_t n, float radius, const float *q,
                                int64_t nq, float *out, int32_t *grid_res) {
    prr_oracle_photon_estimate_knn(rec, n, radius, 0, q, nq, out, NULL, grid_res);
}
