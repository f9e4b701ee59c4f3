// Wavefront integrator: Integrator::castRay (Integrator.cpp:104-263) cut into
// stages that run over queues of paths instead of one path per thread.
//
// A pass traces samples [base, base + k) of every pixel of the window at once
// (P = k * pixels paths). Per bounce:
//   extend   closest hit of every queued ray; the path is appended to the
//            miss, delta (mirror/glass) or surface (diffuse/emissive) queue of
//            its hit -- the sort by material, made with warp-aggregated appends
//   miss     background / env contributions, path ends
//   delta    specular chain step (Integrator.cpp:143-169)
//   surface  NEE towards emitters and the environment (shadow rays queued with
//            their would-be contributions), BSDF sample, next ray queued
//   shadow   any-hit of the queued shadow rays; visible contributions added
// The pending part of a non-delta bounce -- the MIS terms for an env miss or
// an emitter hit, beta *= f/pdf, Russian roulette (Integrator.cpp:205-256) --
// runs at the start of the stage that sees the next hit, so every path makes
// the same random draws and the same additions to L in the same order as
// castRay. At the end of a pass each pixel adds its k results in sample order,
// so the film is the plain renderer's, bit for bit.
//
// Every kernel reads its queue length from device memory, so a pass is one
// fixed launch sequence; it is captured once in a CUDA graph and replayed.
#include "integrator.cuh"
#include "prr_internal.h"
#include "trace_step.cuh"

#include <algorithm>
#include <cstring>

namespace prr {
namespace {

enum : int { kFlagSpecular = 1, kFlagPending = 2, kFlagEndAfterShadow = 4 };
enum : int {
    kCntRay0 = 0, kCntRay1 = 1, kCntMiss = 2, kCntDelta = 3, kCntSurf = 4, kCntShadow = 5,
    kCntExtend = 6, kCntShadowJobs = 7, kCntRays = 8, kCntShadowRays = 10, kCntShadowFetch = 12,
    kCntActive = 13, kCntSlots = 16
};

// One request of a multi-request step (the render server): its scene, camera
// and window, the samples this step traces, and where its paths and pixels
// start in the step's arrays.
struct WfReq {
    const DevScene *scene;
    DevCamera camera;
    int W, x0, y0, ww, npix;     // image width, window, window pixels
    int s0, nspp;                // samples [s0, s0 + nspp) of every window pixel
    int max_depth;
    float clamp;
    uint64_t seed;
    int64_t path_base, pix_base; // first path / first pixel of this request in the step
    float3 *film;                // running per-pixel sums, window order
    unsigned long long rays[2];  // closest, shadow rays traced (added by the kernels)
};

struct Wf {
    int P, npix, spp_pass;
    int W, x0, y0, ww;
    int max_depth;
    float clamp;
    uint64_t seed;
    int tlas_cap, blas_cap; // stack entries a walk may need (tree depth + 1)
    int blas_sm;            // mesh-stack entries kept in shared memory
    void *spill;            // global part of the mesh stacks ([entry][grid thread])
    // path state
    uint64_t *rng;
    float4 *ro, *rd;     // current ray
    float4 *beta;        // xyz
    float4 *L;           // xyz
    int *bounce, *flags;
    float4 *pend;        // pending BSDF: f/pdf xyz, pdf
    float4 *prev;        // pending BSDF: hit point it left from
    int4 *hit;           // obj, tri, t bits
    float4 *slo, *sld, *slc; // light shadow ray: origin+tmax, dir+valid, contribution
    float4 *seo, *sed, *sec; // env shadow ray
    float4 *result;      // final L per path
    float3 *film;        // per pixel running sum
    // queues
    int *qray[2], *qmiss, *qdelta, *qsurf, *qshadow, *qjob;
    uint8_t *vis;        // per shadow job (2 per path): 1 when nothing occludes
    unsigned *cnt;       // kCntSlots counters (64-bit ray totals at kCntRays, kCntShadowRays)
    int *pass_base;      // first sample of the current pass (advanced by the film kernel)
    int sample_offset;
    // ordered queues: stages tag paths instead of appending them, and a stable
    // partition builds the next queues in path (= pixel) order
    int ordered;
    uint8_t *tag;        // per path: bucket of the pending partition, 0xFF none
    unsigned *tile;      // per partition tile: 8 bucket counts, then offsets
    // adaptive sampling (min_spp < max_spp): each pass traces the next
    // spp_pass samples of the pixels still active; the film stage replays the
    // reference's per-sample Welford stop (Renderer.cpp:74-95) on them
    int adaptive, min_spp, max_spp;
    float threshold;
    int *act, *act_next; // active pixels (window-local indices), in pixel order
    uint8_t *ptag;       // per active slot: 0 = stays active, 0xFF = done
    float4 *wel0, *wel1; // per pixel: (n, mean r, g, b), (M2 r, g, b, -)
    // multi-request steps: the request table and each path's request
    WfReq *reqs;
    int n_reqs;
    int *req;
    // traversal counts (kStat* slots), filled only by the counting variants of
    // the extend and shadow stages
    unsigned long long *stats;
    uint32_t *check; // status words of the checked build (nullptr: not reported)
};

// q[slot] = v for an appended queue entry; the checked build tests the slot
// against the queue's capacity (and drops and reports an entry beyond it).
__device__ __forceinline__ void queue_put(const Wf &w, int *q, int slot, int64_t cap, int v) {
#ifdef PRR_CHECKED
    if (slot < 0 || (int64_t) slot >= cap) {
        check_fail(w.check, kCheckQueue, (uint32_t) slot);
        return;
    }
#endif
    (void) w;
    (void) cap;
    q[slot] = v;
}

// A queue's length as a stage reads it. The checked build tests it against
// the queue's capacity (and reports and clamps a longer one).
__device__ __forceinline__ int queue_len(const Wf &w, unsigned n, int64_t cap) {
#ifdef PRR_CHECKED
    if ((int64_t) n > cap) {
        if (blockIdx.x == 0 && threadIdx.x == 0)
            check_fail(w.check, kCheckQueue, n);
        return (int) cap;
    }
#endif
    (void) w;
    (void) cap;
    return (int) n;
}

// Slots of Wf::stats: traversal work of closest-hit (extend) and shadow rays
// (interior nodes of either BVH level, triangle tests, object leaves: mesh
// entries and sphere tests) and the extend results by class.
enum : int {
    kStatClosestNodes = 0, kStatClosestTris = 1, kStatClosestObjects = 2,
    kStatShadowNodes = 3, kStatShadowTris = 4, kStatShadowObjects = 5,
    kStatMiss = 6, kStatDelta = 7, kStatSurface = 8, kStatSlots = 9
};
static_assert(kStatSlots == kWfStatSlots, "counter slots of prr_render_counts");

// Adds a lane's counts to the stats slots [slot, slot + n), one atomic per
// slot per warp.
template <int N>
__device__ __forceinline__ void flush_stats(unsigned long long *stats, int slot,
                                            const unsigned (&c)[N]) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < N; k++) {
        unsigned long long v = c[k];
        for (int off = 16; off > 0; off >>= 1)
            v += __shfl_down_sync(0xffffffffu, v, off);
        if (lane == 0 && v)
            atomicAdd(stats + slot + k, v);
    }
}

// Per-path scene, clamp and depth: the kernel's own for a render, the path's
// request's for a server step.
template <bool MULTI>
__device__ __forceinline__ const DevScene &scene_of(const DevScene &S0, const Wf &w, int p) {
    if constexpr (MULTI)
        return *w.reqs[w.req[p]].scene;
    else
        return S0;
}
template <bool MULTI> __device__ __forceinline__ float clamp_of(const Wf &w, int p) {
    if constexpr (MULTI)
        return w.reqs[w.req[p]].clamp;
    else
        return w.clamp;
}
template <bool MULTI> __device__ __forceinline__ int depth_of(const Wf &w, int p) {
    if constexpr (MULTI)
        return w.reqs[w.req[p]].max_depth;
    else
        return w.max_depth;
}
// the request whose [base, base + count) range holds index x (bases ascending)
__device__ __forceinline__ int find_req(const WfReq *reqs, int n, int64_t x, bool pixels) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        const int64_t b = pixels ? reqs[mid].pix_base : reqs[mid].path_base;
        if (b <= x)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}
// Adds one to a per-request ray counter for every lane of `mask` whose
// predicate holds, one atomic per request present in the warp.
__device__ __forceinline__ void count_req_rays(const Wf &w, unsigned mask, bool pred, int r,
                                               int which) {
    const unsigned m = __ballot_sync(mask, pred);
    if (!pred)
        return;
    const unsigned same = __match_any_sync(m, r);
    if ((threadIdx.x & 31) == __ffs(same) - 1)
        atomicAdd(&w.reqs[r].rays[which], (unsigned long long) __popc(same));
}

__device__ __forceinline__ uint8_t dir_octant(V3 d) {
    return (uint8_t) ((d.x < 0.f) | ((d.y < 0.f) << 1) | ((d.z < 0.f) << 2));
}

__device__ __forceinline__ int warp_append(unsigned *counter, bool pred) {
    const unsigned active = __activemask();
    const unsigned mask = __ballot_sync(active, pred);
    if (!mask)
        return -1;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(mask) - 1;
    unsigned base = 0;
    if (lane == leader)
        base = atomicAdd(counter, (unsigned) __popc(mask));
    base = __shfl_sync(active, base, leader);
    return pred ? (int) (base + __popc(mask & ((1u << lane) - 1u))) : -1;
}

__device__ __forceinline__ V3 ld3(const float4 *a, int i) {
    const float4 v = a[i];
    return v3(v.x, v.y, v.z);
}
__device__ __forceinline__ void st3(float4 *a, int i, V3 v, float w = 0.f) {
    a[i] = make_float4(v.x, v.y, v.z, w);
}

__device__ __forceinline__ void finish(const Wf &w, int p, V3 L) {
    if (!finite3(L))
        L = v3(0.f);
    w.result[p] = make_float4(L.x, L.y, L.z, 0.f);
}

// ---- generate: camera rays for every (pixel, sample) of the pass
template <bool MULTI> __global__ void k_wf_generate(DevScene S, Wf w) {
    const int base = MULTI ? 0 : *w.pass_base;
    const int stride = gridDim.x * blockDim.x;
    // fixed spp: every pixel; adaptive: the active ones (their count is on
    // the device, set by the previous pass); server step: every request's
    // window times its samples of this step, request after request
    const int nq = w.adaptive ? (int) w.cnt[kCntActive] : w.npix;
    const int P = (w.adaptive && !MULTI) ? nq * w.spp_pass : w.P;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < P; p += stride) {
        int i, j;
        uint32_t m, sample;
        uint64_t seed;
        const DevCamera *cam;
        if constexpr (MULTI) {
            const int r = find_req(w.reqs, w.n_reqs, p, false);
            const WfReq &R = w.reqs[r];
            const int64_t o = p - R.path_base;
            const int q = (int) (o % R.npix);
            i = R.x0 + q % R.ww;
            j = R.y0 + q / R.ww;
            m = (uint32_t) i + (uint32_t) j * (uint32_t) R.W;
            sample = (uint32_t) (R.s0 + o / R.npix);
            seed = R.seed;
            cam = &R.camera;
            w.req[p] = r;
        } else {
            const int q = w.adaptive ? w.act[p % nq] : p % w.npix;
            i = w.x0 + q % w.ww;
            j = w.y0 + q / w.ww;
            m = (uint32_t) i + (uint32_t) j * (uint32_t) w.W;
            sample = (uint32_t) (w.sample_offset + base + p / nq);
            seed = w.seed;
            cam = &S.camera;
        }
        Rng rng{path_state(seed, m, sample)};
        const float xo = rng.next();
        const float yo = rng.next();
        const Ray3 r = generate_ray(*cam, i, j, xo, yo, rng);
        w.rng[p] = rng.s;
        st3(w.ro, p, r.o);
        st3(w.rd, p, r.d);
        st3(w.beta, p, v3(1.f));
        st3(w.L, p, v3(0.f));
        w.bounce[p] = 0;
        w.flags[p] = 0;
        w.qray[0][p] = p;
        w.tag[p] = 0xFF;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        w.cnt[kCntRay0] = (unsigned) P;
        w.cnt[kCntRay1] = 0;
    }
}

// ---- per bounce: rotate the ray queues, clear the stage queues
__global__ void k_wf_begin(Wf w, int it) {
    // bounce `it` reads ray queue it&1 (filled by the previous bounce, or by
    // generate) and its shading stages append to queue (it+1)&1
    const int in = it & 1;
    if (threadIdx.x == 0) {
        w.cnt[kCntRay0 + (in ^ 1)] = 0;
        w.cnt[kCntMiss] = w.cnt[kCntDelta] = w.cnt[kCntSurf] = w.cnt[kCntShadow] = 0;
        w.cnt[kCntExtend] = w.cnt[kCntShadowJobs] = w.cnt[kCntShadowFetch] = 0;
        unsigned long long *tot = reinterpret_cast<unsigned long long *>(w.cnt + kCntRays);
        *tot += w.cnt[kCntRay0 + in];
    }
}

// ---- extend: closest hit of the queued rays, then sort by material class.
// Persistent: a lane whose ray is finished takes the next queued ray once
// `refill` lanes of its warp are idle (one atomic per refill).
// The scene-level stack of this thread (all in shared memory) and its mesh-level
// stack (blas_sm entries in shared memory, the rest in the spill buffer).
template <class E>
__device__ __forceinline__ void make_stacks(const Wf &w, E *smem, StackCol<E> &tc,
                                            StackCol<E> &bc) {
    tc = StackCol<E>{smem + threadIdx.x, nullptr, w.tlas_cap, w.tlas_cap, w.check};
    bc = StackCol<E>{smem + (size_t) w.tlas_cap * blockDim.x + threadIdx.x, (E *) w.spill,
                     w.blas_sm, w.blas_cap, w.check};
}

template <bool MULTI>
__device__ __forceinline__ const DevScene &lane_scene(const DevScene &S0, const DevScene *ls) {
    if constexpr (MULTI)
        return *ls;
    else
        return S0;
}

template <bool MULTI, bool STATS>
__device__ __forceinline__ void wf_extend(const DevScene &S0, const Wf &w, int it, int refill) {
    extern __shared__ uint2 smem[];
    StackCol<uint2> tc, bc;
    make_stacks(w, smem, tc, bc);
    const int *qin = w.qray[it & 1];
    const int n = queue_len(w, w.cnt[kCntRay0 + (it & 1)], w.P);
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    int p = -1;
    // this lane's ray's scene (server steps; a valid scene before the first ray)
    const DevScene *ls = MULTI ? w.reqs[0].scene : nullptr;
    ClosestWalk cw;
    unsigned cnt_[6] = {0, 0, 0, 0, 0, 0}; // nodes, tris, objects, miss, delta, surface
    bool more = n > 0;
    if (!more)
        return;
    for (;;) {
        const bool idle = p < 0;
        const unsigned im = __ballot_sync(full, idle);
        if (!more && im == full) {
            if constexpr (STATS) {
                const unsigned a[3] = {cnt_[0], cnt_[1], cnt_[2]};
                const unsigned b[3] = {cnt_[3], cnt_[4], cnt_[5]};
                flush_stats(w.stats, kStatClosestNodes, a);
                flush_stats(w.stats, kStatMiss, b);
            }
            break;
        }
        if (more && __popc(im) >= refill) {
            const int cnt = __popc(im);
            unsigned base = 0;
            if (lane == 0)
                base = atomicAdd(w.cnt + kCntExtend, (unsigned) cnt);
            base = __shfl_sync(full, base, 0);
            if ((int) (base + cnt) >= n)
                more = false;
            const int k = (int) base + __popc(im & ((1u << lane) - 1u));
            const bool take = idle && k < n;
            int r = 0;
            if (take) {
                p = qin[k];
                if constexpr (MULTI) {
                    r = w.req[p];
                    ls = w.reqs[r].scene;
                }
                const float4 o = w.ro[p], d = w.rd[p];
                cw.start(lane_scene<MULTI>(S0, ls), RayD{o.x, o.y, o.z, d.x, d.y, d.z});
            }
            if constexpr (MULTI)
                count_req_rays(w, full, take, r, 0);
        }
        bool done = false;
        const DevScene &S = lane_scene<MULTI>(S0, ls);
        if (p >= 0) {
            if constexpr (STATS) {
                if (S.n_objects > 0)
                    cnt_[cw.in_mesh ? (cw.ntri > 0 ? 1 : 0) : ((cw.tref & kLeafBit) ? 2 : 0)]++;
            }
            done = S.n_objects == 0 || cw.step(S, tc, bc);
        }
        int cls = -1;
        if (done) {
            w.hit[p] = make_int4(cw.hit_obj, cw.hit_tri, __float_as_int(cw.closest), 0);
            if (cw.hit_obj < 0) {
                cls = 0;
            } else {
                const int kind = S.materials[S.objects[cw.hit_obj].material].kind;
                cls = (kind == kMatMirror || kind == kMatGlass) ? 1 : 2;
            }
            if constexpr (STATS)
                cnt_[3 + cls]++;
        }
        if (w.ordered) {
            if (cls >= 0)
                w.tag[p] = (uint8_t) cls;
        } else {
            const int a = warp_append(w.cnt + kCntMiss, cls == 0);
            const int b = warp_append(w.cnt + kCntDelta, cls == 1);
            const int c = warp_append(w.cnt + kCntSurf, cls == 2);
            if (cls == 0)
                queue_put(w, w.qmiss, a, w.P, p);
            else if (cls == 1)
                queue_put(w, w.qdelta, b, w.P, p);
            else if (cls == 2)
                queue_put(w, w.qsurf, c, w.P, p);
        }
        if (done)
            p = -1;
    }
}

// Hit record -> Inter (Triangle::finalize / Sphere::getIntersection fields).
__device__ __forceinline__ Inter load_inter(const DevScene &S, const Wf &w, int p) {
    const int4 h = w.hit[p];
    Inter in;
    in.hit = h.x >= 0;
    in.a = no_attr();
    if (!in.hit) {
        in.mat = -1;
        in.p = in.n = v3(0.f);
        return in;
    }
    const float t = __int_as_float(h.z);
    const V3 o = ld3(w.ro, p), d = ld3(w.rd, p);
    const DevObject &ob = S.objects[h.x];
    in.mat = ob.material;
    if (ob.kind == kObjMesh) {
        in.p = o + t * d;
        in.n = v3(S.normals[(size_t) h.y * 3], S.normals[(size_t) h.y * 3 + 1],
                  S.normals[(size_t) h.y * 3 + 2]);
        finalize_attr(S, ob, h.y, RayD{o.x, o.y, o.z, d.x, d.y, d.z}, in.n, in.a);
    } else {
        in.p = o + d * t;
        in.n = normalize(in.p - v3(ob.cx, ob.cy, ob.cz));
    }
    return in;
}

// The tail of a non-delta bounce (Integrator.cpp:205-256) for the hit of the
// ray it spawned, then the head of the next loop iteration. Returns false
// when the path has ended (its result is written). `it` and `specular` are
// the loop variables of the iteration that now processes `in`.
__device__ __forceinline__ bool enter_iteration(const DevScene &S, const Wf &w, int p,
                                                const Inter &in, Rng &rng, V3 &beta, V3 &L,
                                                int &it, bool &specular, float clamp,
                                                int max_depth) {
    const int k = w.bounce[p];
    const int fl = w.flags[p];
    const V3 bg = v3(S.background[0], S.background[1], S.background[2]);
    if (fl & kFlagPending) {
        const float4 pe = w.pend[p];
        const V3 scale = v3(pe.x, pe.y, pe.z);
        const float bpdf = pe.w;
        const V3 wi = ld3(w.rd, p);
        const bool indirect = k > 0;
        if (!in.hit) {
            V3 c;
            if (S.env.loaded) {
                const V3 el = env_lookup(S.env, wi);
                const float ep = env_pdf(S.env, wi);
                c = beta * scale * mis(bpdf, ep) * el;
            } else {
                c = beta * scale * bg;
            }
            L = L + (indirect ? clamp_indirect(c, clamp) : c);
            return false;
        }
        const DevMaterial &hm = S.materials[in.mat];
        if (hm.kind == kMatEmissive) {
            const V3 hp = ld3(w.prev, p);
            const float cos_l = smax(0.f, dot(-wi, normalized(in.n)));
            const V3 dd = in.p - hp;
            const float hd2 = dot(dd, dd);
            const float pdf_area = S.total_emit_area > 0.f ? 1.f / S.total_emit_area : 0.f;
            const float pdf_sa = pdf_area * hd2 / smax(cos_l, 1e-4f);
            const V3 c = beta * scale * mis(bpdf, pdf_sa) *
                         v3(hm.emission[0], hm.emission[1], hm.emission[2]);
            L = L + (indirect ? clamp_indirect(c, clamp) : c);
            return false;
        }
        beta = beta * scale;
        if (!finite3(beta))
            return false;
        if (k >= 3) {
            const float mc = max3(beta);
            const float q = smax(0.05f, 1.f - mc);
            if (rng.next() < q)
                return false;
            beta = beta * (1.f / (1.f - q));
        }
        it = k + 1;
        specular = false;
    } else if (fl & kFlagSpecular) {
        it = k + 1;
        specular = true;
    } else {
        it = 0;
        specular = false;
    }
    if (it >= max_depth)
        return false;
    if (it == 0 || specular) {
        const V3 d = ld3(w.rd, p);
        if (!in.hit) {
            const V3 b = S.env.loaded ? env_lookup(S.env, d) : bg;
            const V3 c = beta * b;
            L = L + ((it > 0) ? clamp_indirect(c, clamp) : c);
        } else if (S.materials[in.mat].kind == kMatEmissive) {
            const DevMaterial &hm = S.materials[in.mat];
            const V3 c = beta * v3(hm.emission[0], hm.emission[1], hm.emission[2]);
            L = L + ((it > 0) ? clamp_indirect(c, clamp) : c);
        }
    }
    return in.hit;
}

// ---- miss: the path leaves the scene
template <bool MULTI> __global__ void k_wf_miss(DevScene S0, Wf w) {
    const int n = queue_len(w, w.cnt[kCntMiss], w.P);
    const int stride = gridDim.x * blockDim.x;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += stride) {
        const int p = w.qmiss[k];
        const DevScene &S = scene_of<MULTI>(S0, w, p);
        Rng rng{w.rng[p]};
        V3 beta = ld3(w.beta, p), L = ld3(w.L, p);
        Inter in;
        in.hit = false;
        in.mat = -1;
        in.a = no_attr();
        int it;
        bool spec;
        enter_iteration(S, w, p, in, rng, beta, L, it, spec, clamp_of<MULTI>(w, p),
                        depth_of<MULTI>(w, p));
        finish(w, p, L);
    }
}

// ---- delta: one step of the specular chain
template <bool MULTI> __global__ void k_wf_delta(DevScene S0, Wf w, int it_next) {
    const int n = queue_len(w, w.cnt[kCntDelta], w.P);
    int *qout = w.qray[it_next & 1];
    const int stride = gridDim.x * blockDim.x;
    for (int base = blockIdx.x * blockDim.x; base < n; base += stride) {
        const int k = base + threadIdx.x;
        bool cont = false;
        int p = 0;
        if (k < n) {
            p = w.qdelta[k];
            const DevScene &S = scene_of<MULTI>(S0, w, p);
            const int max_depth = depth_of<MULTI>(w, p);
            Rng rng{w.rng[p]};
            V3 beta = ld3(w.beta, p), L = ld3(w.L, p);
            const Inter in = load_inter(S, w, p);
            int it;
            bool spec;
            if (!enter_iteration(S, w, p, in, rng, beta, L, it, spec, clamp_of<MULTI>(w, p),
                                 max_depth)) {
                finish(w, p, L);
            } else {
                const DevMaterial &m = S.materials[in.mat];
                const V3 cd = ld3(w.rd, p);
                const Shading sd = build_shading(S, m, in.n, in.a);
                const BSDFSample bs = delta_sample(m, sd, -cd, rng);
                if (bs.pdf < 1e-6f) {
                    finish(w, p, L);
                } else {
                    beta = beta * bs.f / bs.pdf;
                    const bool trans = dot(bs.wi, in.n) < 0.f;
                    const V3 off = trans ? -in.n : in.n;
                    if (trans)
                        beta = beta * sd.base;
                    // the next ray is only looked at if the loop runs again
                    if (it + 1 >= max_depth) {
                        finish(w, p, L);
                    } else {
                        st3(w.ro, p, in.p + off * PRR_EPS);
                        st3(w.rd, p, bs.wi);
                        st3(w.beta, p, beta);
                        st3(w.L, p, L);
                        w.bounce[p] = it;
                        w.flags[p] = kFlagSpecular;
                        w.rng[p] = rng.s;
                        cont = true;
                    }
                }
            }
        }
        if (w.ordered) {
            if (cont)
                w.tag[p] = dir_octant(ld3(w.rd, p));
        } else {
            const int slot = warp_append(w.cnt + kCntRay0 + (it_next & 1), cont);
            if (cont)
                queue_put(w, qout, slot, w.P, p);
        }
    }
}

// ---- surface: NEE + BSDF sampling of a non-delta bounce
// 64 registers (8 blocks of 128 per SM): this stage waits on scattered path
// state and scene data, so resident warps matter more than a few spills.
template <bool MULTI>
__global__ void __launch_bounds__(128, 8) k_wf_surface(DevScene S0, Wf w, int it_next) {
    const int n = queue_len(w, w.cnt[kCntSurf], w.P);
    int *qout = w.qray[it_next & 1];
    const int stride = gridDim.x * blockDim.x;
    for (int base = blockIdx.x * blockDim.x; base < n; base += stride) {
        const int k = base + threadIdx.x;
        bool cont = false, shadow = false, jl = false, je = false;
        uint8_t oct = 0;
        int p = 0;
        if (k < n) {
            p = w.qsurf[k];
            const DevScene &S = scene_of<MULTI>(S0, w, p);
            Rng rng{w.rng[p]};
            V3 beta = ld3(w.beta, p), L = ld3(w.L, p);
            const V3 L0 = L;
            const Inter in = load_inter(S, w, p);
            int it;
            bool spec;
            if (!enter_iteration(S, w, p, in, rng, beta, L, it, spec, clamp_of<MULTI>(w, p),
                                 depth_of<MULTI>(w, p))) {
                finish(w, p, L);
            } else {
                const DevMaterial &m = S.materials[in.mat];
                const V3 cd = ld3(w.rd, p);
                const V3 hp = in.p;
                const V3 sn = dot(cd, in.n) < 0.f ? in.n : -in.n;
                const Shading sd = build_shading(S, m, sn, in.a);
                const V3 wo = -cd;
                const bool indirect = it > 0;
                // NEE towards emitters: the contribution is formed now and
                // added by the shadow stage if the light is visible
                float4 lo = make_float4(0.f, 0.f, 0.f, 0.f), ld = lo, lc = lo;
                if (S.total_emit_area > 0.f) {
                    const LightPoint lp = sample_light(S, rng);
                    const float pdf_area = 1.0f / S.total_emit_area;
                    const V3 to = lp.p - hp;
                    const float dist2 = dot(to, to);
                    const float dist = sqrtf(dist2);
                    const V3 wi = to / dist;
                    const float cos_l = smax(0.f, dot(-wi, normalized(lp.n)));
                    if (cos_l > 0.f) {
                        const float pdf_sa = pdf_area * dist2 / cos_l;
                        V3 f;
                        float bp;
                        mat_eval_pdf(m, sd, wi, wo, &f, &bp);
                        const DevMaterial &lm = S.materials[lp.material];
                        V3 c = mis(pdf_sa, bp) * v3(lm.emission[0], lm.emission[1], lm.emission[2]) *
                               f / pdf_sa;
                        c = beta * c;
                        if (!(c.x == 0.f && c.y == 0.f && c.z == 0.f)) {
                            const V3 o = hp + wi * PRR_EPS;
                            lo = make_float4(o.x, o.y, o.z, dist - 2.f * PRR_EPS);
                            ld = make_float4(wi.x, wi.y, wi.z, 1.f);
                            lc = make_float4(c.x, c.y, c.z, indirect ? 1.f : 0.f);
                            shadow = true;
                        }
                    }
                }
                float4 eo = make_float4(0.f, 0.f, 0.f, 0.f), ed = eo, ec = eo;
                if (S.env.loaded) {
                    float pdf;
                    const V3 dir = env_importance(S.env, rng, pdf);
                    if (!(pdf < 1e-6f)) {
                        const V3 em = env_lookup(S.env, dir);
                        V3 f;
                        float bp;
                        mat_eval_pdf(m, sd, dir, wo, &f, &bp);
                        V3 c = mis(pdf, bp) * em * f / (pdf + 1e-6f);
                        c = beta * c;
                        if (!(c.x == 0.f && c.y == 0.f && c.z == 0.f)) {
                            const V3 o = hp + dir * PRR_EPS;
                            eo = make_float4(o.x, o.y, o.z, kInf);
                            ed = make_float4(dir.x, dir.y, dir.z, 1.f);
                            ec = make_float4(c.x, c.y, c.z, indirect ? 1.f : 0.f);
                            shadow = true;
                        }
                    }
                }
                if (shadow) {
                    // a ray's direction carries its flag (w = 0: none); its
                    // origin and contribution are read only when set
                    w.sld[p] = ld;
                    w.sed[p] = ed;
                    if (ld.w != 0.f) {
                        w.slo[p] = lo;
                        w.slc[p] = lc;
                    }
                    if (ed.w != 0.f) {
                        w.seo[p] = eo;
                        w.sec[p] = ec;
                    }
                    jl = ld.w != 0.f;
                    je = ed.w != 0.f;
                }
                BSDFSample bs;
                if (m.kind == kMatDiffuse)
                    bs = diffuse_sample(m, sd, wo, rng);
                else
                    bs.pdf = 0.f;
                if (bs.pdf < 1e-6f) {
                    if (shadow) {
                        st3(w.L, p, L);
                        w.flags[p] = kFlagEndAfterShadow;
                    } else {
                        finish(w, p, L);
                    }
                } else {
                    const V3 scale = bs.f / bs.pdf;
                    const V3 off = dot(bs.wi, sd.f.N) >= 0.f ? sd.f.N : -sd.f.N;
                    st3(w.ro, p, hp + off * PRR_EPS);
                    st3(w.rd, p, bs.wi);
                    oct = dir_octant(bs.wi);
                    st3(w.pend, p, scale, bs.pdf);
                    if (S.has_emissive_kind) // read only on an emissive hit
                        st3(w.prev, p, hp);
                    st3(w.beta, p, beta);
                    if (__float_as_uint(L.x) != __float_as_uint(L0.x) ||
                        __float_as_uint(L.y) != __float_as_uint(L0.y) ||
                        __float_as_uint(L.z) != __float_as_uint(L0.z))
                        st3(w.L, p, L); // changed only by emission at this hit
                    w.bounce[p] = it;
                    w.flags[p] = kFlagPending;
                    cont = true;
                }
                w.rng[p] = rng.s;
            }
        }
        if (w.ordered) {
            if (cont)
                w.tag[p] = oct;
        } else {
            const int slot = warp_append(w.cnt + kCntRay0 + (it_next & 1), cont);
            if (cont)
                queue_put(w, qout, slot, w.P, p);
        }
        const int sslot = warp_append(w.cnt + kCntShadow, shadow);
        if (shadow)
            queue_put(w, w.qshadow, sslot, w.P, p);
        const int j0 = warp_append(w.cnt + kCntShadowJobs, jl);
        if (jl)
            queue_put(w, w.qjob, j0, 2 * (int64_t) w.P, p * 2);
        const int j1 = warp_append(w.cnt + kCntShadowJobs, je);
        if (je)
            queue_put(w, w.qjob, j1, 2 * (int64_t) w.P, p * 2 + 1);
    }
}

// ---- shadow: visibility of every queued NEE ray (persistent, per-lane refill)
template <bool MULTI, bool STATS>
__device__ __forceinline__ void wf_shadow(const DevScene &S0, const Wf &w, int refill) {
    extern __shared__ uint32_t smem32[];
    StackCol<uint32_t> tc, bc;
    make_stacks(w, smem32, tc, bc);
    const int n = queue_len(w, w.cnt[kCntShadowJobs], 2 * (int64_t) w.P);
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    int job = -1;
    // this lane's ray's scene (server steps; a valid scene before the first ray)
    const DevScene *ls = MULTI ? w.reqs[0].scene : nullptr;
    AnyWalk aw;
    bool more = n > 0;
    unsigned rays = 0;
    unsigned cnt_[3] = {0, 0, 0}; // nodes, tris, objects
    for (;;) {
        const bool idle = job < 0;
        const unsigned im = __ballot_sync(full, idle);
        if (!more && im == full)
            break;
        if (more && __popc(im) >= refill) {
            const int cnt = __popc(im);
            unsigned base = 0;
            if (lane == 0)
                base = atomicAdd(w.cnt + kCntShadowFetch, (unsigned) cnt);
            base = __shfl_sync(full, base, 0);
            if ((int) (base + cnt) >= n)
                more = false;
            const int k = (int) base + __popc(im & ((1u << lane) - 1u));
            const bool take = idle && k < n;
            int r = 0;
            if (take) {
                job = w.qjob[k];
                const int p = job >> 1;
                if constexpr (MULTI) {
                    r = w.req[p];
                    ls = w.reqs[r].scene;
                }
                const float4 o = (job & 1) ? w.seo[p] : w.slo[p];
                const float4 d = (job & 1) ? w.sed[p] : w.sld[p];
                rays++;
                if (!aw.start(lane_scene<MULTI>(S0, ls), RayD{o.x, o.y, o.z, d.x, d.y, d.z}, o.w)) {
                    w.vis[job] = 1;
                    job = -1;
                }
            }
            if constexpr (MULTI)
                count_req_rays(w, full, take, r, 1);
        }
        const DevScene &S = lane_scene<MULTI>(S0, ls);
        if constexpr (STATS) {
            if (job >= 0)
                cnt_[aw.in_mesh ? (aw.ntri > 0 ? 1 : 0) : ((aw.tref & kLeafBit) ? 2 : 0)]++;
        }
        if (job >= 0 && aw.step(S, tc, bc)) {
            w.vis[job] = aw.occluded ? 0 : 1;
            job = -1;
        }
    }
    if constexpr (STATS)
        flush_stats(w.stats, kStatShadowNodes, cnt_);
    for (int off = 16; off > 0; off >>= 1)
        rays += __shfl_down_sync(full, rays, off);
    if (lane == 0 && rays)
        atomicAdd(reinterpret_cast<unsigned long long *>(w.cnt + kCntShadowRays),
                  (unsigned long long) rays);
}

// The traversal stages held to 48 registers (no spills): 10 resident blocks of
// 128 (or 21 of 64) instead of 9 at the 54-56 they take otherwise; the
// museum-like frame 216.6 -> 213.5 ms.
template <bool MULTI, bool STATS = false>
__global__ void __maxnreg__(48) k_wf_extend(DevScene S, Wf w, int it, int refill) {
    wf_extend<MULTI, STATS>(S, w, it, refill);
}
// The server's extend stage (paths of several requests; the request index
// selects scene and camera), held to 48 registers like the others: 10
// resident blocks of 128 instead of 8 at the 64 it takes otherwise (16 bytes
// of spills).
__global__ void __maxnreg__(48) k_wf_extend_multi(DevScene S, Wf w, int it, int refill) {
    wf_extend<true, false>(S, w, it, refill);
}
template <bool MULTI, bool STATS = false>
__global__ void __maxnreg__(48) k_wf_shadow(DevScene S, Wf w, int refill) {
    wf_shadow<MULTI, STATS>(S, w, refill);
}

// ---- add the visible NEE contributions, light first, then env, as castRay
template <bool MULTI> __global__ void k_wf_shadow_resolve(Wf w) {
    const int n = queue_len(w, w.cnt[kCntShadow], w.P);
    const int stride = gridDim.x * blockDim.x;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += stride) {
        const int p = w.qshadow[k];
        V3 L = ld3(w.L, p);
        for (int r = 0; r < 2; r++) {
            const float4 d = r == 0 ? w.sld[p] : w.sed[p];
            if (d.w == 0.f || !w.vis[p * 2 + r])
                continue;
            const float4 c = r == 0 ? w.slc[p] : w.sec[p];
            const V3 cv = v3(c.x, c.y, c.z);
            L = L + (c.w != 0.f ? clamp_indirect(cv, clamp_of<MULTI>(w, p)) : cv);
        }
        if (w.flags[p] & kFlagEndAfterShadow)
            finish(w, p, L);
        else
            st3(w.L, p, L);
    }
}

// ---- film: add the pass's samples per pixel in sample order
// ---- ordered queues: a stable partition of the per-path tags into bucket
// queues, in path order within each bucket. A tile is 4096 paths: 256
// threads x 16 tags read as one 16-byte vector. Tiles are counted, the tile
// counts scanned per bucket, then each tile writes its paths to their buckets
// in order and clears their tags for the next partition. The tag array is
// padded with 0xFF to whole tiles.
constexpr int kPartThreads = 256;
constexpr int kPartTile = kPartThreads * 16;

struct PartSpec {
    uint8_t *tag;       // the tags, padded with 0xFF to whole tiles
    const int *map;     // item k is written as map[k] (nullptr: k itself)
    int *q[8];          // bucket b's queue; concatenated: all in q[0], bucket order
    int nb;             // buckets (<= 8)
    int concat;
    int count_slot[8];  // counter slot receiving bucket b's size (-1: none)
    int total_slot;     // counter slot receiving the total (-1: none)
};

// How many of the 16 tag bytes in v equal b.
__device__ __forceinline__ unsigned count_tag(const uint4 &v, unsigned b) {
    const unsigned bb = b * 0x01010101u;
    return (__popc(__vcmpeq4(v.x, bb)) + __popc(__vcmpeq4(v.y, bb)) +
            __popc(__vcmpeq4(v.z, bb)) + __popc(__vcmpeq4(v.w, bb))) >> 3;
}

__global__ void __launch_bounds__(kPartThreads) k_part_count(Wf w, PartSpec ps) {
    const int nb = ps.nb;
    __shared__ unsigned c[8];
    if (threadIdx.x < 8)
        c[threadIdx.x] = 0;
    __syncthreads();
    const uint4 v = reinterpret_cast<const uint4 *>(ps.tag)[blockIdx.x * kPartThreads + threadIdx.x];
#pragma unroll
    for (int b = 0; b < 8; b++)
        if (b < nb) {
            const unsigned r = __reduce_add_sync(0xffffffffu, count_tag(v, b));
            if ((threadIdx.x & 31) == 0 && r)
                atomicAdd(&c[b], r);
        }
    __syncthreads();
    if (threadIdx.x < 8)
        w.tile[blockIdx.x * 8 + threadIdx.x] = c[threadIdx.x];
}

// Exclusive scan over the tiles, all buckets at once: one block, one tile per
// thread per round. Tile counts become the tiles' first output slots.
__global__ void __launch_bounds__(1024) k_part_scan(Wf w, int ntiles, PartSpec ps) {
    __shared__ unsigned wsum[32][8];
    __shared__ unsigned carry[8];
    __shared__ unsigned total[8];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (threadIdx.x < 8)
        carry[threadIdx.x] = 0;
    __syncthreads();
    for (int r0 = 0; r0 < ntiles; r0 += 1024) {
        const int t = r0 + threadIdx.x;
        unsigned v[8];
        if (t < ntiles) {
            const uint4 a = reinterpret_cast<const uint4 *>(w.tile)[t * 2];
            const uint4 b = reinterpret_cast<const uint4 *>(w.tile)[t * 2 + 1];
            v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
            v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
        } else {
#pragma unroll
            for (int k = 0; k < 8; k++)
                v[k] = 0;
        }
        unsigned x[8];
#pragma unroll
        for (int k = 0; k < 8; k++) {
            x[k] = v[k];
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned y = __shfl_up_sync(0xffffffffu, x[k], o);
                if (lane >= o)
                    x[k] += y;
            }
            if (lane == 31)
                wsum[wid][k] = x[k];
        }
        __syncthreads();
        // warp 0 scans the 32 warp sums of each bucket
        if (wid == 0) {
#pragma unroll
            for (int k = 0; k < 8; k++) {
                const unsigned s0 = wsum[lane][k];
                unsigned z = s0;
                for (int o = 1; o < 32; o <<= 1) {
                    const unsigned y = __shfl_up_sync(0xffffffffu, z, o);
                    if (lane >= o)
                        z += y;
                }
                wsum[lane][k] = z - s0; // exclusive
                if (lane == 31) {
                    // round total folded into the running carry after use
                    total[k] = z;
                }
            }
        }
        __syncthreads();
        if (t < ntiles) {
            unsigned o[8];
#pragma unroll
            for (int k = 0; k < 8; k++)
                o[k] = carry[k] + wsum[wid][k] + x[k] - v[k];
            reinterpret_cast<uint4 *>(w.tile)[t * 2] = make_uint4(o[0], o[1], o[2], o[3]);
            reinterpret_cast<uint4 *>(w.tile)[t * 2 + 1] = make_uint4(o[4], o[5], o[6], o[7]);
        }
        __syncthreads();
        if (threadIdx.x < 8)
            carry[threadIdx.x] += total[threadIdx.x];
        __syncthreads();
    }
    // bucket bases (concatenated queues) and counts
    if (threadIdx.x == 0) {
        unsigned base = 0;
#pragma unroll
        for (int k = 0; k < 8; k++)
            if (k < ps.nb) {
                total[k] = base; // reuse: first slot of bucket k
                if (ps.count_slot[k] >= 0)
                    w.cnt[ps.count_slot[k]] = carry[k];
                base += carry[k];
            }
        if (ps.total_slot >= 0)
            w.cnt[ps.total_slot] = base;
    }
    __syncthreads();
    if (ps.concat)
        for (int i = threadIdx.x; i < ntiles * 8; i += 1024) {
            const int k = i & 7;
            if (k < ps.nb)
                w.tile[i] += total[k];
        }
}

__global__ void __launch_bounds__(kPartThreads) k_part_scatter(Wf w, PartSpec ps) {
    __shared__ unsigned wsum[kPartThreads / 32][8];
    __shared__ unsigned base[8][kPartThreads];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint4 *tv = reinterpret_cast<uint4 *>(ps.tag) + blockIdx.x * kPartThreads + threadIdx.x;
    const uint4 v = *tv;
    unsigned c[8], x[8];
#pragma unroll
    for (int k = 0; k < 8; k++) {
        c[k] = k < ps.nb ? count_tag(v, k) : 0u;
        x[k] = c[k];
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned y = __shfl_up_sync(0xffffffffu, x[k], o);
            if (lane >= o)
                x[k] += y;
        }
        if (lane == 31)
            wsum[wid][k] = x[k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 8; k++) {
        unsigned before = 0;
        for (int u = 0; u < wid; u++)
            before += wsum[u][k];
        base[k][threadIdx.x] = (k < ps.nb ? w.tile[blockIdx.x * 8 + k] : 0u) + before + x[k] - c[k];
    }
    const uint32_t words[4] = {v.x, v.y, v.z, v.w};
    const int first = (blockIdx.x * kPartThreads + threadIdx.x) * 16;
#pragma unroll
    for (int i = 0; i < 16; i++) {
        const unsigned t = (words[i >> 2] >> ((i & 3) * 8)) & 0xFFu;
        if (t < (unsigned) ps.nb) {
            int *q = ps.q[0];
            if (!ps.concat) {
#pragma unroll
                for (int k = 1; k < 8; k++)
                    if (t == (unsigned) k)
                        q = ps.q[k];
            }
            q[base[t][threadIdx.x]++] = ps.map ? ps.map[first + i] : first + i;
        }
    }
    *tv = make_uint4(0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu);
}

// ---- adaptive film: each active pixel takes this pass's samples in sample
// order -- running sum, per-channel Welford update, and the stop test after
// every sample once min_spp samples are in (Renderer.cpp:74-95). Samples
// traced past a pixel's stop are dropped, as the reference never draws them.
__global__ void k_wf_film_adaptive(Wf w) {
    const int na = (int) w.cnt[kCntActive];
    const int stride = gridDim.x * blockDim.x;
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < na; a += stride) {
        const int q = w.act[a];
        const float4 s0 = w.wel0[q], s1 = w.wel1[q];
        Welford wr{(int) s0.x, s0.y, s1.x}, wg{(int) s0.x, s0.z, s1.y}, wb{(int) s0.x, s0.w, s1.z};
        float3 f = w.film[q];
        bool done = false;
        for (int k = 0; k < w.spp_pass && !done; k++) {
            float4 r = w.result[(size_t) k * na + a];
            if (isnan(r.x) || isnan(r.y) || isnan(r.z))
                r = make_float4(0.f, 0.f, 0.f, 0.f);
            f.x += r.x;
            f.y += r.y;
            f.z += r.z;
            wr.update(r.x);
            wg.update(r.y);
            wb.update(r.z);
            done = wr.n >= w.min_spp && wr.ci() < w.threshold && wg.ci() < w.threshold &&
                   wb.ci() < w.threshold;
        }
        w.film[q] = f;
        w.wel0[q] = make_float4((float) wr.n, wr.mean, wg.mean, wb.mean);
        w.wel1[q] = make_float4(wr.M2, wg.M2, wb.M2, 0.f);
        w.ptag[a] = (done || wr.n >= w.max_spp) ? 0xFF : 0;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0)
        *w.pass_base += w.spp_pass;
}

__global__ void k_wf_copy_active(Wf w) {
    const int na = (int) w.cnt[kCntActive];
    const int stride = gridDim.x * blockDim.x;
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < na; a += stride)
        w.act[a] = w.act_next[a];
}

__global__ void k_wf_adaptive_init(Wf w) {
    const int stride = gridDim.x * blockDim.x;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < w.npix; q += stride) {
        w.act[q] = q;
        w.wel0[q] = make_float4(0.f, 0.f, 0.f, 0.f);
        w.wel1[q] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0)
        w.cnt[kCntActive] = (unsigned) w.npix;
}

// mean = sum / n per pixel (Renderer.cpp:98-99)
__global__ void k_wf_resolve_adaptive(const float3 *film, const float4 *wel0, int npix, float *out,
                                      int32_t *spp) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= npix)
        return;
    const float3 f = film[q];
    const int n = (int) wel0[q].x;
    out[(size_t) q * 3 + 0] = f.x / (float) n;
    out[(size_t) q * 3 + 1] = f.y / (float) n;
    out[(size_t) q * 3 + 2] = f.z / (float) n;
    if (spp)
        spp[q] = n;
}

// ---- server step film: every request's window pixels take this step's
// samples in sample order (the same sums as a render of the request alone)
__global__ void k_wf_film_multi(Wf w, int64_t total_pixels) {
    const int64_t stride = (int64_t) gridDim.x * blockDim.x;
    for (int64_t t = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; t < total_pixels;
         t += stride) {
        const int r = find_req(w.reqs, w.n_reqs, t, true);
        const WfReq &R = w.reqs[r];
        const int q = (int) (t - R.pix_base);
        float3 f = R.film[q];
        for (int s = 0; s < R.nspp; s++) {
            const float4 v = w.result[R.path_base + (int64_t) s * R.npix + q];
            if (!(isnan(v.x) || isnan(v.y) || isnan(v.z))) {
                f.x += v.x;
                f.y += v.y;
                f.z += v.z;
            }
        }
        R.film[q] = f;
    }
}

__global__ void k_wf_film(Wf w) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < w.npix) {
        float3 f = w.film[q];
        for (int s = 0; s < w.spp_pass; s++) {
            const float4 r = w.result[(size_t) s * w.npix + q];
            // a NaN sample is zeroed before accumulation (Renderer.cpp:78-83)
            if (!(isnan(r.x) || isnan(r.y) || isnan(r.z))) {
                f.x += r.x;
                f.y += r.y;
                f.z += r.z;
            }
        }
        w.film[q] = f;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0)
        *w.pass_base += w.spp_pass;
}

__global__ void k_wf_resolve(const float3 *film, int npix, int n, float *out, int32_t *spp) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= npix)
        return;
    const float3 f = film[q];
    out[(size_t) q * 3 + 0] = f.x / (float) n;
    out[(size_t) q * 3 + 1] = f.y / (float) n;
    out[(size_t) q * 3 + 2] = f.z / (float) n;
    if (spp)
        spp[q] = n;
}

__global__ void k_wf_rays_out(const unsigned *cnt, unsigned long long *out) {
    out[0] = *reinterpret_cast<const unsigned long long *>(cnt + kCntRays);
    out[1] = *reinterpret_cast<const unsigned long long *>(cnt + kCntShadowRays);
}

uint32_t float_bits(float f) {
    uint32_t u;
    std::memcpy(&u, &f, sizeof(u));
    return u;
}

template <class T> T *carve(char *&p, size_t n) {
    T *r = reinterpret_cast<T *>(p);
    p += (n * sizeof(T) + 255) & ~size_t(255);
    return r;
}

} // namespace

struct WavefrontPlan {
    // one captured pass per (scene, window, spp_pass, depth, block shape)
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint64_t key = 0;
    ~WavefrontPlan() {
        if (exec)
            cudaGraphExecDestroy(exec);
        if (graph)
            cudaGraphDestroy(graph);
    }
};

namespace {

// Bytes of the path-state layout for P paths and npix film pixels.
size_t wf_bytes(size_t P, int npix) {
    const int ntiles = (int) ((P + kPartTile - 1) / kPartTile);
    const int ptiles = (npix + kPartTile - 1) / kPartTile;
    return 256 * 48 + P * (8 + 16 * 16 + 4 * 2 + 4 * 9 + 2 + 4) + (size_t) ntiles * kPartTile +
           (size_t) npix * (16 + 8 + 32) + (size_t) ptiles * kPartTile +
           (size_t) std::max(ntiles, ptiles) * 32 + 4096;
}

// Carves the per-path arrays, queues, counters and partition buffers of P
// paths and npix pixels out of `buf` (grown as needed).
int wf_layout(DevBuf &buf, Wf &w, size_t P, int npix) {
    const int ntiles = (int) ((P + kPartTile - 1) / kPartTile);
    const int ptiles = (npix + kPartTile - 1) / kPartTile;
    const size_t bytes = wf_bytes(P, npix);
    PRR_CUDA_TRY(buf.ensure(bytes));
    char *cur = (char *) buf.ptr;
    w.rng = carve<uint64_t>(cur, P);
    w.ro = carve<float4>(cur, P);
    w.rd = carve<float4>(cur, P);
    w.beta = carve<float4>(cur, P);
    w.L = carve<float4>(cur, P);
    w.pend = carve<float4>(cur, P);
    w.prev = carve<float4>(cur, P);
    w.hit = carve<int4>(cur, P);
    w.slo = carve<float4>(cur, P);
    w.sld = carve<float4>(cur, P);
    w.slc = carve<float4>(cur, P);
    w.seo = carve<float4>(cur, P);
    w.sed = carve<float4>(cur, P);
    w.sec = carve<float4>(cur, P);
    w.result = carve<float4>(cur, P);
    w.bounce = carve<int>(cur, P);
    w.flags = carve<int>(cur, P);
    w.req = carve<int>(cur, P);
    w.qray[0] = carve<int>(cur, P);
    w.qray[1] = carve<int>(cur, P);
    w.qmiss = carve<int>(cur, P);
    w.qdelta = carve<int>(cur, P);
    w.qsurf = carve<int>(cur, P);
    w.qshadow = carve<int>(cur, P);
    w.qjob = carve<int>(cur, 2 * P);
    w.vis = carve<uint8_t>(cur, 2 * P);
    w.film = carve<float3>(cur, (size_t) npix);
    w.cnt = carve<unsigned>(cur, kCntSlots);
    w.pass_base = carve<int>(cur, 4);
    w.tag = carve<uint8_t>(cur, (size_t) ntiles * kPartTile);
    w.tile = carve<unsigned>(cur, (size_t) std::max(ntiles, ptiles) * 8);
    w.act = carve<int>(cur, (size_t) npix);
    w.act_next = carve<int>(cur, (size_t) npix);
    w.ptag = carve<uint8_t>(cur, (size_t) ptiles * kPartTile);
    w.wel0 = carve<float4>(cur, (size_t) npix);
    w.wel1 = carve<float4>(cur, (size_t) npix);
    if ((size_t) (cur - (char *) buf.ptr) > bytes)
        return fail(PRR_ERR_INTERNAL, "wavefront buffer layout overflow");
    return PRR_OK;
}

// Launch shape of one bounce: traversal grids, stack split, spill buffer.
struct WfShape {
    int block, refill, g_ext, g_sh, g_shade, g_gen, ntiles, ptiles;
    size_t smem_ext, smem_sh;
    void (*ext)(DevScene, Wf, int, int);
    void (*sh)(DevScene, Wf, int);
};

template <bool MULTI>
int wf_shape(Wf &w, DevBuf &spill, int block_req, int stack_req, int refill_req, WfShape &L) {
    const int sms = device_sm_count();
    L.block = block_req > 0 ? block_req : 128;
    // Stacks: the scene-level one wholly in shared memory, the mesh one up to
    // stack_req entries (0: all of it) within 96 KB per block; its deeper
    // entries go to the global spill buffer.
    const int max_sm_entries = (96 * 1024) / (L.block * (int) sizeof(uint2));
    if (w.tlas_cap + 1 > max_sm_entries)
        return fail(PRR_ERR_UNSUPPORTED, "scene BVH too deep for the shared-memory stack");
    w.blas_sm = stack_req > 0 ? std::min(stack_req, w.blas_cap) : w.blas_cap;
    w.blas_sm = std::max(1, std::min(w.blas_sm, max_sm_entries - w.tlas_cap));
    L.smem_ext = (size_t) (w.tlas_cap + w.blas_sm) * L.block * sizeof(uint2);
    L.smem_sh = (size_t) (w.tlas_cap + w.blas_sm) * L.block * sizeof(uint32_t);
    L.ext = MULTI ? k_wf_extend_multi : k_wf_extend<false>;
    L.sh = k_wf_shadow<MULTI>;
    if constexpr (!MULTI) {
        if (w.stats) { // the counting variants (a separate, untimed render)
            L.ext = k_wf_extend<false, true>;
            L.sh = k_wf_shadow<false, true>;
        }
    }
    if (L.smem_ext > 48 * 1024)
        PRR_CUDA_TRY(cudaFuncSetAttribute((const void *) L.ext,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int) L.smem_ext));
    if (L.smem_sh > 48 * 1024)
        PRR_CUDA_TRY(cudaFuncSetAttribute((const void *) L.sh,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int) L.smem_sh));
    // Deep stacks want the largest shared-memory split; shallow ones keep the
    // default, since every change of split between consecutive kernels drains
    // the SM (which dominates frames made of many short launches).
    const int carve_pref = L.smem_ext > 16 * 1024 ? (int) cudaSharedmemCarveoutMaxShared
                                                  : (int) cudaSharedmemCarveoutDefault;
    cudaFuncSetAttribute((const void *) L.ext, cudaFuncAttributePreferredSharedMemoryCarveout,
                         carve_pref);
    cudaFuncSetAttribute((const void *) L.sh, cudaFuncAttributePreferredSharedMemoryCarveout,
                         carve_pref);
    L.refill = refill_req > 0 ? std::min(refill_req, 32) : 8;
    int occ_ext = 1, occ_sh = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_ext, (const void *) L.ext, L.block,
                                                  L.smem_ext);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_sh, (const void *) L.sh, L.block,
                                                  L.smem_sh);
    L.g_ext = sms * std::max(1, occ_ext);
    L.g_sh = sms * std::max(1, occ_sh);
    const size_t spill_entries = (size_t) (w.blas_cap - w.blas_sm);
    const size_t spill_bytes =
        spill_entries * std::max((size_t) L.g_ext * L.block * sizeof(uint2),
                                 (size_t) L.g_sh * L.block * sizeof(uint32_t));
    PRR_CUDA_TRY(spill.ensure(spill_bytes));
    w.spill = spill.ptr;
    L.g_shade = sms * 8;
    L.g_gen = (int) std::min<int64_t>(((int64_t) w.P + 255) / 256, (int64_t) sms * 16);
    L.ntiles = (int) (((size_t) w.P + kPartTile - 1) / kPartTile);
    L.ptiles = (w.npix + kPartTile - 1) / kPartTile;
    return PRR_OK;
}

// The stable partitions of the ordered queues.
struct WfParts {
    PartSpec cls, ray[2], act;
};
WfParts wf_parts(const Wf &w) {
    WfParts P;
    // hit classes -> miss / delta / surface queues
    P.cls = PartSpec{};
    P.cls.tag = w.tag;
    P.cls.q[0] = w.qmiss;
    P.cls.q[1] = w.qdelta;
    P.cls.q[2] = w.qsurf;
    P.cls.nb = 3;
    P.cls.concat = 0;
    P.cls.count_slot[0] = kCntMiss;
    P.cls.count_slot[1] = kCntDelta;
    P.cls.count_slot[2] = kCntSurf;
    P.cls.total_slot = -1;
    // next rays -> the ray queue, direction octant major
    for (int r = 0; r < 2; r++) {
        P.ray[r] = PartSpec{};
        P.ray[r].tag = w.tag;
        P.ray[r].q[0] = w.qray[r];
        P.ray[r].nb = 8;
        P.ray[r].concat = 1;
        for (int b = 0; b < 8; b++)
            P.ray[r].count_slot[b] = -1;
        P.ray[r].total_slot = kCntRay0 + r;
    }
    // adaptive: the pixels still active -> the next pass's active list
    P.act = PartSpec{};
    P.act.tag = w.ptag;
    P.act.map = w.act;
    P.act.q[0] = w.act_next;
    P.act.nb = 1;
    P.act.concat = 1;
    P.act.count_slot[0] = -1;
    P.act.total_slot = kCntActive;
    return P;
}

void wf_partition(const Wf &w, const PartSpec &ps, int nt, cudaStream_t cs) {
    k_part_count<<<nt, kPartThreads, 0, cs>>>(w, ps);
    k_part_scan<<<1, 1024, 0, cs>>>(w, nt, ps);
    k_part_scatter<<<nt, kPartThreads, 0, cs>>>(w, ps);
}

// generate + every bounce of one pass (no film stage)
template <bool MULTI>
int wf_enqueue_bounces(const DevScene &S, const Wf &w, const WfShape &L, const WfParts &parts,
                       cudaStream_t cs) {
    k_wf_generate<MULTI><<<L.g_gen, 256, 0, cs>>>(S, w);
    for (int it = 0; it <= w.max_depth; it++) {
        k_wf_begin<<<1, 32, 0, cs>>>(w, it);
        L.ext<<<L.g_ext, L.block, L.smem_ext, cs>>>(S, w, it, L.refill);
        if (w.ordered)
            wf_partition(w, parts.cls, L.ntiles, cs);
        k_wf_miss<MULTI><<<L.g_shade, 128, 0, cs>>>(S, w);
        k_wf_delta<MULTI><<<L.g_shade, 128, 0, cs>>>(S, w, it + 1);
        k_wf_surface<MULTI><<<L.g_shade, 128, 0, cs>>>(S, w, it + 1);
        L.sh<<<L.g_sh, L.block, L.smem_sh, cs>>>(S, w, L.refill);
        k_wf_shadow_resolve<MULTI><<<L.g_shade, 128, 0, cs>>>(w);
        if (w.ordered)
            wf_partition(w, parts.ray[(it + 1) & 1], L.ntiles, cs);
    }
    PRR_CUDA_TRY(cudaGetLastError());
    return PRR_OK;
}

} // namespace

int render_wavefront(Scene &s, const prr_render_settings &rs, float *out_rgb, int32_t *out_spp,
                     unsigned long long *out_rays, cudaStream_t st) {
    const DevScene &S = s.dev;
    Wf w{};
    w.W = s.width;
    w.x0 = rs.x0;
    w.y0 = rs.y0;
    w.ww = rs.x1 - rs.x0;
    const int wh = rs.y1 - rs.y0;
    w.npix = w.ww * wh;
    w.max_depth = rs.max_depth;
    w.clamp = rs.indirect_clamp;
    w.seed = rs.seed;
    w.sample_offset = rs.sample_offset;
    w.tlas_cap = S.tlas_depth + 1;
    w.blas_cap = S.blas_depth + 1;
    // paths per pass: whole samples of the window, about 8M paths in flight
    const int64_t target = s.wf_paths > 0 ? s.wf_paths : (int64_t) 1 << 23;
    int spp_pass = (int) std::max<int64_t>(1, target / std::max(1, w.npix));
    spp_pass = std::min(spp_pass, rs.max_spp);
    while (rs.max_spp % spp_pass)
        spp_pass--;
    w.spp_pass = spp_pass;
    w.P = spp_pass * w.npix;
    if (int rc = wf_layout(s.d_wavefront, w, (size_t) w.P, w.npix))
        return rc;
    w.ordered = s.wf_ordered ? 1 : 0;
    w.adaptive = rs.min_spp < rs.max_spp ? 1 : 0;
    w.min_spp = rs.min_spp;
    w.max_spp = rs.max_spp;
    w.threshold = rs.variance_threshold;
    w.stats = s.wf_stats;
    w.check = S.check;
    WfShape L;
    if (int rc = wf_shape<false>(w, s.d_wf_spill, s.wf_block, s.wf_stack, s.wf_refill, L))
        return rc;
    const WfParts parts = wf_parts(w);

    PRR_CUDA_TRY(cudaMemsetAsync(w.film, 0, (size_t) w.npix * sizeof(float3), st));
    PRR_CUDA_TRY(cudaMemsetAsync(w.tag, 0xFF, (size_t) L.ntiles * kPartTile, st));
    PRR_CUDA_TRY(cudaMemsetAsync(w.cnt, 0, kCntSlots * sizeof(unsigned), st));
    PRR_CUDA_TRY(cudaMemsetAsync(w.pass_base, 0, sizeof(int), st));
    if (w.adaptive) { // after the counters are cleared: it sets the active count
        PRR_CUDA_TRY(cudaMemsetAsync(w.ptag, 0xFF, (size_t) L.ptiles * kPartTile, st));
        k_wf_adaptive_init<<<(w.npix + 255) / 256, 256, 0, st>>>(w);
    }

    // one pass: the bounces, then the film stage
    auto enqueue_pass = [&](cudaStream_t cs) -> int {
        if (int rc = wf_enqueue_bounces<false>(S, w, L, parts, cs))
            return rc;
        if (w.adaptive) {
            k_wf_film_adaptive<<<(w.npix + 255) / 256, 256, 0, cs>>>(w);
            wf_partition(w, parts.act, L.ptiles, cs);
            k_wf_copy_active<<<(w.npix + 255) / 256, 256, 0, cs>>>(w);
        } else {
            k_wf_film<<<(w.npix + 255) / 256, 256, 0, cs>>>(w);
        }
        PRR_CUDA_TRY(cudaGetLastError());
        return PRR_OK;
    };
    const int passes = rs.max_spp / spp_pass;
    uint64_t key = (uint64_t) (uintptr_t) s.d_wavefront.ptr;
    key = mix64(key ^ ((uint64_t) w.P << 20) ^ ((uint64_t) w.max_depth << 8) ^
                (uint64_t) L.block ^ ((uint64_t) L.refill << 50));
    key = mix64(key ^ (uint64_t) (uintptr_t) w.spill ^ ((uint64_t) w.blas_sm << 32) ^
                ((uint64_t) w.ordered << 60));
    key = mix64(key ^ ((uint64_t) w.adaptive << 7) ^ ((uint64_t) w.min_spp << 24) ^
                ((uint64_t) float_bits(w.threshold) << 28) ^ (uint64_t) w.max_spp);
    key = mix64(key ^ ((uint64_t) (uint32_t) w.x0 << 32 | (uint32_t) w.y0) ^
                ((uint64_t) (uint32_t) w.ww << 16) ^ rs.seed ^ ((uint64_t) rs.sample_offset << 40) ^
                (uint64_t) float_bits(w.clamp));
    if (!s.wf_plan)
        s.wf_plan = std::make_shared<WavefrontPlan>();
    WavefrontPlan &plan = *s.wf_plan;
    if (s.wf_graphs && passes > 1 && !w.stats) {
        if (plan.key != key || !plan.exec) {
            if (plan.exec) {
                cudaGraphExecDestroy(plan.exec);
                plan.exec = nullptr;
            }
            if (plan.graph) {
                cudaGraphDestroy(plan.graph);
                plan.graph = nullptr;
            }
            cudaStream_t cap;
            PRR_CUDA_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
            PRR_CUDA_TRY(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
            int rc = enqueue_pass(cap);
            cudaGraph_t g = nullptr;
            cudaError_t e = cudaStreamEndCapture(cap, &g);
            cudaStreamDestroy(cap);
            if (rc)
                return rc;
            if (e != cudaSuccess)
                return fail(PRR_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
            plan.graph = g;
            PRR_CUDA_TRY(cudaGraphInstantiate(&plan.exec, g, 0));
            plan.key = key;
        }
        for (int k = 0; k < passes; k++)
            PRR_CUDA_TRY(cudaGraphLaunch(plan.exec, st));
    } else {
        for (int k = 0; k < passes; k++)
            if (int rc = enqueue_pass(st))
                return rc;
    }
    if (w.adaptive)
        k_wf_resolve_adaptive<<<(w.npix + 255) / 256, 256, 0, st>>>(w.film, w.wel0, w.npix,
                                                                    out_rgb, out_spp);
    else
        k_wf_resolve<<<(w.npix + 255) / 256, 256, 0, st>>>(w.film, w.npix, rs.max_spp, out_rgb,
                                                            out_spp);
    PRR_CUDA_TRY(cudaGetLastError());
    if (out_rays) {
        k_wf_rays_out<<<1, 1, 0, st>>>(w.cnt, out_rays);
        PRR_CUDA_TRY(cudaGetLastError());
    }
    // generate + per bounce (begin, extend, miss, delta, surface, shadow,
    // shadow_resolve, and two 3-kernel partitions when ordered) + film
    const int64_t per_pass = 2 + (int64_t) (w.max_depth + 1) * (7 + (w.ordered ? 6 : 0)) +
                             (w.adaptive ? 4 : 0);
    s.last_launches = per_pass * passes + 1 + (w.adaptive ? 1 : 0) + (out_rays ? 1 : 0);
    return PRR_OK;
}

int wavefront_step_multi(WfMultiState &ms, const WfStepReq *reqs, int n,
                         int64_t paths_per_launch, int tlas_cap, int blas_cap,
                         unsigned long long *rays_host, cudaStream_t st, int64_t *launches) {
    if (n <= 0)
        return PRR_OK;
    // the request table of the whole step in pinned memory, one copy up
    const size_t table_bytes = (size_t) n * sizeof(WfReq);
    if (table_bytes > ms.h_cap) {
        if (ms.h_table)
            cudaFreeHost(ms.h_table);
        ms.h_table = nullptr;
        ms.h_cap = std::max(table_bytes, 2 * ms.h_cap);
        PRR_CUDA_TRY(cudaMallocHost(&ms.h_table, ms.h_cap));
    }
    PRR_CUDA_TRY(ms.reqs.ensure(ms.h_cap));
    WfReq *table = static_cast<WfReq *>(ms.h_table);
    // launch groups: consecutive requests of at most paths_per_launch paths
    // (a request alone may exceed it); bases count from each group's start
    struct Group {
        int a, b, max_depth;
        int64_t P, npix;
    };
    std::vector<Group> groups;
    Group g{0, 0, 1, 0, 0};
    for (int k = 0; k < n; k++) {
        const WfStepReq &q = reqs[k];
        const int64_t paths = (int64_t) q.ww * q.wh * q.nspp;
        if (k > g.a && g.P + paths > paths_per_launch) {
            groups.push_back(g);
            g = Group{k, k, 1, 0, 0};
        }
        WfReq &t = table[k];
        std::memset(&t, 0, sizeof(t));
        t.scene = q.scene;
        t.camera = q.camera;
        t.W = q.camera.width;
        t.x0 = q.x0;
        t.y0 = q.y0;
        t.ww = q.ww;
        t.npix = q.ww * q.wh;
        t.s0 = q.s0;
        t.nspp = q.nspp;
        t.max_depth = q.max_depth;
        t.clamp = q.clamp;
        t.seed = q.seed;
        t.path_base = g.P;
        t.pix_base = g.npix;
        t.film = q.film;
        g.P += paths;
        g.npix += t.npix;
        g.max_depth = std::max(g.max_depth, q.max_depth);
        g.b = k + 1;
    }
    groups.push_back(g);
    int64_t maxP = 0;
    for (const Group &x : groups)
        maxP = std::max(maxP, x.P);
    if (maxP >= ((int64_t) 1 << 31))
        return fail(PRR_ERR_INVALID_ARGUMENT, "server step too large");
    PRR_CUDA_TRY(cudaMemcpyAsync(ms.reqs.ptr, table, table_bytes, cudaMemcpyHostToDevice, st));
    int64_t nl = 0;
    for (const Group &x : groups) {
        Wf w{};
        w.P = (int) x.P;
        w.npix = 0; // no per-render film or active list in a server step
        w.max_depth = x.max_depth;
        w.ordered = 1;
        w.reqs = ms.reqs.as<WfReq>() + x.a;
        w.n_reqs = x.b - x.a;
        w.tlas_cap = tlas_cap;
        w.blas_cap = blas_cap;
        if (int rc = wf_layout(ms.state, w, (size_t) maxP, 1))
            return rc;
        WfShape L;
        if (int rc = wf_shape<true>(w, ms.spill, 128, 8, 8, L))
            return rc;
        const WfParts parts = wf_parts(w);
        PRR_CUDA_TRY(cudaMemsetAsync(w.tag, 0xFF, (size_t) L.ntiles * kPartTile, st));
        PRR_CUDA_TRY(cudaMemsetAsync(w.cnt, 0, kCntSlots * sizeof(unsigned), st));
        if (int rc = wf_enqueue_bounces<true>(DevScene{}, w, L, parts, st))
            return rc;
        k_wf_film_multi<<<(int) std::min<int64_t>((x.npix + 255) / 256,
                                                  (int64_t) device_sm_count() * 16),
                          256, 0, st>>>(w, x.npix);
        PRR_CUDA_TRY(cudaGetLastError());
        // generate + per bounce (begin, extend, 3-kernel partition, miss,
        // delta, surface, shadow, shadow_resolve, 3-kernel partition) + film
        nl += 1 + (int64_t) (w.max_depth + 1) * 13 + 1;
    }
    // the rays each request traced: one strided copy out of the table
    if (rays_host)
        PRR_CUDA_TRY(cudaMemcpy2DAsync(rays_host, 2 * sizeof(unsigned long long),
                                       &ms.reqs.as<WfReq>()[0].rays, sizeof(WfReq),
                                       2 * sizeof(unsigned long long), n,
                                       cudaMemcpyDeviceToHost, st));
    if (launches)
        *launches = nl;
    return PRR_OK;
}

} // namespace prr
