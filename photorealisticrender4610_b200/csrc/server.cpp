// Render server: continuous batching of render requests on one GPU.
//
// Requests (scene, window, spp, depth, seed, output buffer) are queued by
// prr_server_submit and admitted in arrival order by a worker thread as long
// as (a) fewer than max_active requests are running and (b) the device bytes
// of the resident scenes plus every admitted request stay within the budget.
// Every step renders the next sample chunk of EVERY running request, so
// requests that arrive while others are on the GPU join at the next step and
// overlap with them; a request leaves as soon as its last chunk is done,
// freeing its slot and memory for the queue. A step runs either on the
// wavefront integrator (k_wavefront.cu: the paths of all running requests,
// up to paths_per_launch per group, share one set of ordered ray queues, so
// each bounce is one traversal launch for all of them) or as one megakernel
// launch over (request, 16x8 tile) items (k_serve.cu).
//
// On wavefront steps a request's film adds its samples one by one in sample
// order, as a render of the request does, so its image does not depend on how
// many samples each step takes: the scheduler splits each step's paths among
// the running requests freely. On megakernel steps the film adds chunk sums,
// and a request's chunk size depends only on the request (samples_per_step /
// its pixel count). Either way its image is the same alone as in any mix.
#include "prr_internal.h"
#include "serve.h"

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <thread>
#include <unordered_map>

namespace prr {
namespace {

double now_s() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

struct Req {
    uint64_t id = 0;
    int scene = 0;
    prr_render_settings rs{};
    float *out = nullptr;
    bool out_on_device = false;
    int status = PRR_REQUEST_QUEUED;
    int error = PRR_OK;
    double t_submit = 0, t_admit = 0, t_done = 0;
    int next = 0, chunk = 1, npix = 0, ww = 0, wh = 0;
    int64_t credit = 0; // wavefront steps: paths earned towards the next samples
    DevCamera camera{};
    size_t bytes = 0;
    void *film = nullptr, *result = nullptr; // device blocks from the server's pool
    size_t film_cap = 0, result_cap = 0;
    unsigned long long rays = 0;
};

struct Server {
    prr_server_config cfg{};
    int device = 0;
    std::vector<Scene *> scenes;
    std::vector<size_t> scene_bytes;
    DevBuf d_scenes; // DevScene per scene
    int tlas_cap = 1, blas_cap = 1;

    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Req *> queue;
    std::vector<Req *> active;
    std::unordered_map<uint64_t, std::unique_ptr<Req>> reqs;
    uint64_t next_id = 1;
    size_t used = 0;
    bool stop = false;
    std::thread worker;
    cudaStream_t st = nullptr;
    int64_t admissions = 0;

    // step tables
    std::vector<ServeItem> h_items;
    std::vector<ServeReq> h_reqs;
    ServeItem *p_items = nullptr; // pinned
    ServeReq *p_reqs = nullptr;   // pinned
    size_t cap_items = 0, cap_reqs = 0;
    DevBuf d_items, d_reqs;
    // wavefront steps
    WfMultiState wf;
    std::vector<WfStepReq> wf_reqs;
    std::vector<int> chunks;
    std::vector<size_t> order, stepped;
    unsigned long long *p_rays = nullptr; // pinned, 2 per active request
    size_t cap_rays = 0;

    // Device blocks of finished requests kept for later admissions: freeing
    // and allocating device memory between steps would stall the worker.
    std::multimap<size_t, void *> pool;
    size_t pooled = 0;
    static constexpr size_t kPoolCap = (size_t) 2 << 30;

    // stats
    int64_t submitted = 0, completed = 0, failed = 0, samples = 0, steps = 0, launches = 0;
    unsigned long long rays = 0;
    double busy = 0, admit_time = 0, complete_time = 0;

    ~Server() {
        if (p_items)
            cudaFreeHost(p_items);
        if (p_reqs)
            cudaFreeHost(p_reqs);
        if (p_rays)
            cudaFreeHost(p_rays);
        for (auto &b : pool)
            cudaFree(b.second);
        if (st)
            cudaStreamDestroy(st);
    }
};

// A block of at least n bytes: a pooled one up to twice that size, else a
// new allocation (after giving the pool back when the device is full).
cudaError_t pool_get(Server &S, size_t n, void **out, size_t *cap) {
    auto it = S.pool.lower_bound(n);
    if (it != S.pool.end() && it->first <= 2 * n) {
        *out = it->second;
        *cap = it->first;
        S.pooled -= it->first;
        S.pool.erase(it);
        return cudaSuccess;
    }
    cudaError_t e = cudaMalloc(out, n);
    if (e == cudaErrorMemoryAllocation && !S.pool.empty()) {
        cudaGetLastError();
        for (auto &b : S.pool)
            cudaFree(b.second);
        S.pool.clear();
        S.pooled = 0;
        e = cudaMalloc(out, n);
    }
    *cap = e == cudaSuccess ? n : 0;
    return e;
}

// Work on a returned block is ordered on the server's stream like all later
// uses, so it can go straight back into the pool.
void pool_put(Server &S, void *&p, size_t &cap) {
    if (!p)
        return;
    S.pool.emplace(cap, p);
    S.pooled += cap;
    p = nullptr;
    cap = 0;
    while (S.pooled > Server::kPoolCap) {
        auto big = std::prev(S.pool.end());
        S.pooled -= big->first;
        cudaFree(big->second);
        S.pool.erase(big);
    }
}

void finish_locked(Server &S, Req *r, int status, int error) {
    r->status = status;
    r->error = error;
    r->t_done = now_s();
    pool_put(S, r->film, r->film_cap);
    pool_put(S, r->result, r->result_cap);
    S.used -= r->bytes;
    if (status == PRR_REQUEST_DONE)
        S.completed++;
    else if (status == PRR_REQUEST_FAILED)
        S.failed++;
    S.cv_done.notify_all();
}

// Admit queued requests in arrival order while a slot and budget are free.
void admit_locked(Server &S) {
    const double t0 = now_s();
    while (!S.queue.empty() && (int) S.active.size() < S.cfg.max_active) {
        Req *r = S.queue.front();
        if (S.used + r->bytes > (size_t) S.cfg.device_budget_bytes)
            break; // keep arrival order: wait for memory instead of skipping ahead
        S.queue.pop_front();
        S.used += r->bytes;
        S.admissions++;
        bool fail_alloc = S.cfg.fail_every_nth_admission > 0 &&
                          S.admissions % S.cfg.fail_every_nth_admission == 0;
        cudaError_t e = fail_alloc ? cudaErrorMemoryAllocation
                                   : pool_get(S, (size_t) r->npix * sizeof(float3), &r->film,
                                              &r->film_cap);
        if (e == cudaSuccess)
            e = cudaMemsetAsync(r->film, 0, (size_t) r->npix * sizeof(float3), S.st);
        if (e == cudaSuccess && !r->out_on_device)
            e = pool_get(S, (size_t) r->npix * 3 * sizeof(float), &r->result, &r->result_cap);
        if (e != cudaSuccess) {
            cudaGetLastError();
            finish_locked(S, r, PRR_REQUEST_FAILED, PRR_ERR_OUT_OF_MEMORY);
            continue;
        }
        r->status = PRR_REQUEST_RUNNING;
        r->t_admit = now_s();
        S.active.push_back(r);
    }
    S.admit_time += now_s() - t0;
}

int ensure_tables(Server &S, size_t items, size_t reqs) {
    if (items > S.cap_items) {
        if (S.p_items)
            cudaFreeHost(S.p_items);
        S.cap_items = std::max(items, S.cap_items * 2);
        PRR_CUDA_TRY(cudaMallocHost(&S.p_items, S.cap_items * sizeof(ServeItem)));
        PRR_CUDA_TRY(S.d_items.alloc(S.cap_items * sizeof(ServeItem)));
    }
    if (reqs > S.cap_reqs) {
        if (S.p_reqs)
            cudaFreeHost(S.p_reqs);
        S.cap_reqs = std::max(reqs, S.cap_reqs * 2);
        PRR_CUDA_TRY(cudaMallocHost(&S.p_reqs, S.cap_reqs * sizeof(ServeReq)));
        PRR_CUDA_TRY(S.d_reqs.alloc(S.cap_reqs * sizeof(ServeReq)));
    }
    return PRR_OK;
}

// One wavefront step over every running request: groups of requests (in
// admission order) of at most paths_per_launch paths each, one after another
// on the server's stream, then one wait for the stream.
int run_step_wavefront(Server &S) {
    const DevScene *d_scenes = S.d_scenes.as<DevScene>();
    const size_t n = S.active.size();
    if (2 * n > S.cap_rays) {
        if (S.p_rays)
            cudaFreeHost(S.p_rays);
        S.p_rays = nullptr;
        S.cap_rays = std::max(2 * n, 2 * S.cap_rays);
        PRR_CUDA_TRY(cudaMallocHost(&S.p_rays, S.cap_rays * sizeof(unsigned long long)));
    }
    // This step's samples per request (the image does not depend on them).
    // A quarter of the step's paths is shared equally as credit: a request
    // takes whole samples of its window once its credit pays for them, so a
    // large window progresses every few steps without crowding the step. The
    // rest goes to the requests with the least work left, so short requests
    // leave in one step.
    const int64_t budget = S.cfg.paths_per_launch;
    const int64_t fair = std::max<int64_t>(1, budget / (4 * (int64_t) n));
    S.chunks.assign(n, 0);
    S.order.resize(n);
    int64_t left = budget;
    for (size_t q = 0; q < n; q++) {
        Req *r = S.active[q];
        const int64_t rem = r->rs.max_spp - r->next;
        r->credit = std::min(r->credit + fair, rem * r->npix);
        const int64_t c = r->credit / r->npix;
        S.chunks[q] = (int) c;
        r->credit -= c * r->npix;
        left -= c * r->npix;
        S.order[q] = q;
    }
    std::sort(S.order.begin(), S.order.end(), [&](size_t a, size_t b) {
        const Req *ra = S.active[a], *rb = S.active[b];
        return (int64_t) (ra->rs.max_spp - ra->next) * ra->npix <
               (int64_t) (rb->rs.max_spp - rb->next) * rb->npix;
    });
    bool any = false;
    for (size_t i = 0; i < n; i++) {
        const size_t q = S.order[i];
        const Req *r = S.active[q];
        const int64_t more = std::min<int64_t>(r->rs.max_spp - r->next - S.chunks[q],
                                               std::max<int64_t>(0, left) / r->npix);
        if (more > 0) {
            S.chunks[q] += (int) more;
            left -= more * r->npix;
        }
        any = any || S.chunks[q] > 0;
    }
    if (!any) // every window is larger than the step: one sample of the shortest
        S.chunks[S.order[0]] = 1;
    // the table holds the requests that take samples this step
    S.wf_reqs.clear();
    S.stepped.clear();
    for (size_t q = 0; q < n; q++) {
        if (S.chunks[q] == 0)
            continue;
        const Req *r = S.active[q];
        WfStepReq d;
        d.scene = d_scenes + r->scene;
        d.camera = r->camera;
        d.x0 = r->rs.x0;
        d.y0 = r->rs.y0;
        d.ww = r->ww;
        d.wh = r->wh;
        d.s0 = r->rs.sample_offset + r->next;
        d.nspp = S.chunks[q];
        d.max_depth = r->rs.max_depth;
        d.clamp = r->rs.indirect_clamp;
        d.seed = r->rs.seed;
        d.film = static_cast<float3 *>(r->film);
        S.wf_reqs.push_back(d);
        S.stepped.push_back(q);
    }
    const double t0 = now_s();
    int64_t launches = 0;
    if (int rc = wavefront_step_multi(S.wf, S.wf_reqs.data(), (int) S.wf_reqs.size(),
                                      S.cfg.paths_per_launch, S.tlas_cap, S.blas_cap, S.p_rays,
                                      S.st, &launches))
        return rc;
    PRR_CUDA_TRY(cudaStreamSynchronize(S.st));
    S.busy += now_s() - t0;
    S.steps++;
    S.launches += launches;
    for (size_t k = 0; k < S.stepped.size(); k++) {
        Req *r = S.active[S.stepped[k]];
        const int c = S.chunks[S.stepped[k]];
        S.samples += (int64_t) c * r->npix;
        r->next += c;
        const unsigned long long rays = S.p_rays[2 * k] + S.p_rays[2 * k + 1];
        r->rays += rays;
        S.rays += rays;
    }
    return PRR_OK;
}

// One step over every running request; returns a status for the whole step.
int run_step(Server &S) {
    if (S.cfg.integrator == PRR_SERVER_WAVEFRONT)
        return run_step_wavefront(S);
    const DevScene *d_scenes = S.d_scenes.as<DevScene>();
    size_t n_items = 0;
    for (Req *r : S.active)
        n_items += (size_t) serve_tiles(r->ww, r->wh);
    if (int rc = ensure_tables(S, std::max<size_t>(n_items, 1), std::max<size_t>(S.active.size(), 1)))
        return rc;
    size_t k = 0;
    for (size_t q = 0; q < S.active.size(); q++) {
        Req *r = S.active[q];
        ServeReq &d = S.p_reqs[q];
        d.scene = d_scenes + r->scene;
        d.camera = r->camera;
        d.x0 = r->rs.x0;
        d.y0 = r->rs.y0;
        d.ww = r->ww;
        d.wh = r->wh;
        d.s0 = r->rs.sample_offset + r->next;
        d.s1 = r->rs.sample_offset + std::min(r->next + r->chunk, r->rs.max_spp);
        d.max_depth = r->rs.max_depth;
        d.clamp = r->rs.indirect_clamp;
        d.seed = r->rs.seed;
        d.film = static_cast<float3 *>(r->film);
        d.rays = 0;
        const int tiles = serve_tiles(r->ww, r->wh);
        for (int t = 0; t < tiles; t++)
            S.p_items[k++] = ServeItem{(int) q, t};
    }
    PRR_CUDA_TRY(cudaMemcpyAsync(S.d_items.ptr, S.p_items, n_items * sizeof(ServeItem),
                                 cudaMemcpyHostToDevice, S.st));
    PRR_CUDA_TRY(cudaMemcpyAsync(S.d_reqs.ptr, S.p_reqs, S.active.size() * sizeof(ServeReq),
                                 cudaMemcpyHostToDevice, S.st));
    const double t0 = now_s();
    if (int rc = serve_launch_step(S.d_items.as<ServeItem>(), (int) n_items,
                                   S.d_reqs.as<ServeReq>(), S.tlas_cap, S.blas_cap, S.st))
        return rc;
    PRR_CUDA_TRY(cudaMemcpyAsync(S.p_reqs, S.d_reqs.ptr, S.active.size() * sizeof(ServeReq),
                                 cudaMemcpyDeviceToHost, S.st));
    PRR_CUDA_TRY(cudaStreamSynchronize(S.st));
    S.busy += now_s() - t0;
    S.steps++;
    S.launches += n_items > 0 ? 1 : 0;
    for (size_t q = 0; q < S.active.size(); q++) {
        Req *r = S.active[q];
        const int s1 = std::min(r->next + r->chunk, r->rs.max_spp);
        S.samples += (int64_t) (s1 - r->next) * r->npix;
        r->next = s1;
        r->rays += S.p_reqs[q].rays;
        S.rays += S.p_reqs[q].rays;
    }
    return PRR_OK;
}

// Resolve finished requests into their outputs.
int complete(Server &S, std::vector<Req *> &done) {
    const double t0 = now_s();
    for (Req *r : done) {
        float *target = r->out_on_device ? r->out : static_cast<float *>(r->result);
        if (int rc = serve_resolve(static_cast<const float3 *>(r->film), r->npix, r->rs.max_spp,
                                   target, S.st))
            return rc;
        S.launches++;
        if (!r->out_on_device)
            PRR_CUDA_TRY(cudaMemcpyAsync(r->out, r->result, (size_t) r->npix * 3 * sizeof(float),
                                         cudaMemcpyDeviceToHost, S.st));
    }
    PRR_CUDA_TRY(cudaStreamSynchronize(S.st));
    S.complete_time += now_s() - t0;
    return PRR_OK;
}

void worker_main(Server *Sp) {
    Server &S = *Sp;
    cudaSetDevice(S.device);
    std::unique_lock<std::mutex> lk(S.mu);
    for (;;) {
        S.cv_work.wait(lk, [&] { return S.stop || !S.queue.empty() || !S.active.empty(); });
        if (S.stop && S.active.empty())
            break;
        admit_locked(S);
        if (S.active.empty())
            continue;
        lk.unlock();
        int rc = run_step(S);
        std::vector<Req *> done;
        if (rc == PRR_OK) {
            for (Req *r : S.active)
                if (r->next >= r->rs.max_spp)
                    done.push_back(r);
            if (!done.empty())
                rc = complete(S, done);
        }
        lk.lock();
        if (rc != PRR_OK) {
            // a failed step fails every request it carried; the server goes on
            for (Req *r : S.active)
                finish_locked(S, r, PRR_REQUEST_FAILED, rc);
            S.active.clear();
            cudaGetLastError();
            continue;
        }
        for (Req *r : done) {
            finish_locked(S, r, r->status == PRR_REQUEST_CANCELLED ? PRR_REQUEST_CANCELLED
                                                                   : PRR_REQUEST_DONE,
                          PRR_OK);
            S.active.erase(std::find(S.active.begin(), S.active.end(), r));
        }
        // cancelled while running: drop at the step boundary
        for (size_t q = 0; q < S.active.size();) {
            Req *r = S.active[q];
            if (r->status == PRR_REQUEST_CANCELLED) {
                finish_locked(S, r, PRR_REQUEST_CANCELLED, PRR_OK);
                S.active.erase(S.active.begin() + q);
            } else {
                q++;
            }
        }
    }
}

Server *SV(prr_server *s) { return reinterpret_cast<Server *>(s); }

void fill_info(const Req &r, prr_request_info *info) {
    info->status = r.status;
    info->error = r.error;
    info->submit_s = r.t_submit;
    info->admit_s = r.t_admit;
    info->done_s = r.t_done;
    info->samples = (int64_t) r.next * r.npix;
    info->rays = r.rays;
}

} // namespace
} // namespace prr

using namespace prr;

extern "C" {

int prr_server_create(const prr_server_config *config, prr_server **out) {
    if (!out)
        return fail(PRR_ERR_INVALID_ARGUMENT, "out is NULL");
    auto *S = new Server();
    if (config)
        S->cfg = *config;
    if (S->cfg.device_budget_bytes <= 0)
        S->cfg.device_budget_bytes = (int64_t) 120 << 30;
    if (S->cfg.max_active <= 0)
        S->cfg.max_active = 64;
    if (S->cfg.samples_per_step <= 0)
        S->cfg.samples_per_step = (int64_t) 1 << 20;
    if (S->cfg.integrator != PRR_SERVER_WAVEFRONT && S->cfg.integrator != PRR_SERVER_MEGAKERNEL) {
        delete S;
        return fail(PRR_ERR_INVALID_ARGUMENT, "unknown server integrator");
    }
    if (S->cfg.paths_per_launch <= 0)
        S->cfg.paths_per_launch = (int64_t) 1 << 24;
    S->cfg.paths_per_launch = std::min<int64_t>(S->cfg.paths_per_launch, (int64_t) 1 << 30);
    cudaError_t e = cudaGetDevice(&S->device);
    if (e == cudaSuccess)
        e = cudaStreamCreateWithFlags(&S->st, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete S;
        return fail(PRR_ERR_CUDA, std::string("server stream: ") + cudaGetErrorString(e));
    }
    S->worker = std::thread(worker_main, S);
    *out = reinterpret_cast<prr_server *>(S);
    return PRR_OK;
}

int prr_server_destroy(prr_server *server) {
    if (!server)
        return PRR_OK;
    Server &S = *SV(server);
    {
        std::lock_guard<std::mutex> g(S.mu);
        S.stop = true;
        for (Req *r : S.queue)
            finish_locked(S, r, PRR_REQUEST_CANCELLED, PRR_OK);
        S.queue.clear();
    }
    S.cv_work.notify_all();
    if (S.worker.joinable())
        S.worker.join();
    delete &S;
    return PRR_OK;
}

int prr_server_add_scene(prr_server *server, prr_scene *scene, int *out_id) {
    if (!server || !scene)
        return fail(PRR_ERR_INVALID_ARGUMENT, "server and scene are required");
    Server &S = *SV(server);
    Scene &sc = *reinterpret_cast<Scene *>(scene);
    if (!sc.built || !sc.camera_set)
        return fail(PRR_ERR_NOT_BUILT, "scene must be built and have a camera");
    std::lock_guard<std::mutex> g(S.mu);
    if (!S.active.empty() || !S.queue.empty())
        return fail(PRR_ERR_INVALID_ARGUMENT, "add scenes before submitting requests");
    if (S.used + sc.device_bytes > (size_t) S.cfg.device_budget_bytes)
        return fail(PRR_ERR_BUDGET, "scene does not fit in the device budget");
    S.scenes.push_back(&sc);
    S.scene_bytes.push_back(sc.device_bytes);
    S.used += sc.device_bytes;
    S.tlas_cap = std::max(S.tlas_cap, sc.dev.tlas_depth + 1);
    S.blas_cap = std::max(S.blas_cap, sc.dev.blas_depth + 1);
    std::vector<DevScene> all;
    for (Scene *p : S.scenes)
        all.push_back(p->dev);
    PRR_CUDA_TRY(S.d_scenes.alloc(all.size() * sizeof(DevScene)));
    PRR_CUDA_TRY(cudaMemcpy(S.d_scenes.ptr, all.data(), all.size() * sizeof(DevScene),
                            cudaMemcpyHostToDevice));
    if (out_id)
        *out_id = (int) S.scenes.size() - 1;
    return PRR_OK;
}

int prr_server_submit(prr_server *server, const prr_request *request, uint64_t *out_id) {
    if (!server || !request || !request->out_rgb)
        return fail(PRR_ERR_INVALID_ARGUMENT, "server, request and out_rgb are required");
    Server &S = *SV(server);
    std::unique_ptr<Req> r(new Req());
    r->t_submit = now_s();
    if (request->scene < 0 || request->scene >= (int) S.scenes.size())
        return fail(PRR_ERR_INVALID_ARGUMENT, "unknown scene id");
    r->scene = request->scene;
    r->rs = request->settings;
    r->rs.mode = PRR_RENDER_PLAIN;
    if (r->rs.min_spp != r->rs.max_spp)
        return fail(PRR_ERR_UNSUPPORTED, "served requests use fixed spp");
    // the request may ask for its own resolution of the scene's camera
    const Scene &sc = *S.scenes[r->scene];
    if (r->rs.width <= 0 || r->rs.height <= 0 || r->rs.width > 16384 || r->rs.height > 16384)
        return fail(PRR_ERR_INVALID_ARGUMENT, "bad request resolution");
    if (r->rs.x1 <= 0 || r->rs.y1 <= 0) {
        r->rs.x0 = r->rs.y0 = 0;
        r->rs.x1 = r->rs.width;
        r->rs.y1 = r->rs.height;
    }
    if (r->rs.x0 < 0 || r->rs.y0 < 0 || r->rs.x1 > r->rs.width || r->rs.y1 > r->rs.height ||
        r->rs.x0 >= r->rs.x1 || r->rs.y0 >= r->rs.y1 || r->rs.max_spp < 1 || r->rs.max_depth < 1 ||
        r->rs.max_depth > 1024 || r->rs.sample_offset < 0)
        return fail(PRR_ERR_INVALID_ARGUMENT, "bad request settings");
    r->camera = make_camera(sc.camera, r->rs.width, r->rs.height);
    r->out = request->out_rgb;
    cudaPointerAttributes pa{};
    if (cudaPointerGetAttributes(&pa, r->out) == cudaSuccess)
        r->out_on_device = pa.type == cudaMemoryTypeDevice || pa.type == cudaMemoryTypeManaged;
    cudaGetLastError();
    r->ww = r->rs.x1 - r->rs.x0;
    r->wh = r->rs.y1 - r->rs.y0;
    r->npix = r->ww * r->wh;
    // megakernel steps: a chunk that depends only on the request (its film
    // adds chunk sums); wavefront steps choose samples per step (below)
    r->chunk = (int) std::max<int64_t>(1, std::min<int64_t>(r->rs.max_spp,
                                                            S.cfg.samples_per_step / r->npix));
    r->bytes = (size_t) r->npix * sizeof(float3) + (r->out_on_device ? 0 : (size_t) r->npix * 12);
    std::lock_guard<std::mutex> g(S.mu);
    if (S.stop)
        return fail(PRR_ERR_INVALID_ARGUMENT, "server is shutting down");
    size_t scenes_total = 0;
    for (size_t b : S.scene_bytes)
        scenes_total += b;
    if (scenes_total + r->bytes > (size_t) S.cfg.device_budget_bytes)
        return fail(PRR_ERR_BUDGET, "request can never fit in the device budget");
    r->id = S.next_id++;
    if (out_id)
        *out_id = r->id;
    S.queue.push_back(r.get());
    S.reqs.emplace(r->id, std::move(r));
    S.submitted++;
    S.cv_work.notify_one();
    return PRR_OK;
}

int prr_server_cancel(prr_server *server, uint64_t id) {
    if (!server)
        return fail(PRR_ERR_INVALID_ARGUMENT, "server is NULL");
    Server &S = *SV(server);
    std::lock_guard<std::mutex> g(S.mu);
    auto it = S.reqs.find(id);
    if (it == S.reqs.end())
        return fail(PRR_ERR_INVALID_ARGUMENT, "unknown request id");
    Req *r = it->second.get();
    if (r->status == PRR_REQUEST_QUEUED) {
        S.queue.erase(std::find(S.queue.begin(), S.queue.end(), r));
        finish_locked(S, r, PRR_REQUEST_CANCELLED, PRR_OK);
    } else if (r->status == PRR_REQUEST_RUNNING) {
        r->status = PRR_REQUEST_CANCELLED; // dropped at the next step boundary
    }
    return PRR_OK;
}

int prr_server_poll(prr_server *server, uint64_t id, prr_request_info *info) {
    if (!server || !info)
        return fail(PRR_ERR_INVALID_ARGUMENT, "server and info are required");
    Server &S = *SV(server);
    std::lock_guard<std::mutex> g(S.mu);
    auto it = S.reqs.find(id);
    if (it == S.reqs.end())
        return fail(PRR_ERR_INVALID_ARGUMENT, "unknown request id");
    fill_info(*it->second, info);
    return PRR_OK;
}

int prr_server_wait(prr_server *server, uint64_t id, double timeout_s, prr_request_info *info) {
    if (!server)
        return fail(PRR_ERR_INVALID_ARGUMENT, "server is NULL");
    Server &S = *SV(server);
    std::unique_lock<std::mutex> lk(S.mu);
    auto it = S.reqs.find(id);
    if (it == S.reqs.end())
        return fail(PRR_ERR_INVALID_ARGUMENT, "unknown request id");
    Req *r = it->second.get();
    auto finished = [&] {
        return r->status == PRR_REQUEST_DONE || r->status == PRR_REQUEST_FAILED ||
               (r->status == PRR_REQUEST_CANCELLED && r->t_done > 0);
    };
    if (timeout_s < 0)
        S.cv_done.wait(lk, finished);
    else if (!S.cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), finished)) {
        if (info)
            fill_info(*r, info);
        return fail(PRR_ERR_TIMEOUT, "request not finished within the timeout");
    }
    if (info)
        fill_info(*r, info);
    return PRR_OK;
}

int prr_server_stats_get(prr_server *server, prr_server_stats *out) {
    if (!server || !out)
        return fail(PRR_ERR_INVALID_ARGUMENT, "server and out are required");
    Server &S = *SV(server);
    std::lock_guard<std::mutex> g(S.mu);
    out->submitted = S.submitted;
    out->completed = S.completed;
    out->failed = S.failed;
    out->active = (int64_t) S.active.size();
    out->queued = (int64_t) S.queue.size();
    out->samples = S.samples;
    out->rays = S.rays;
    out->steps = S.steps;
    out->busy_s = S.busy;
    out->admit_s = S.admit_time;
    out->complete_s = S.complete_time;
    out->bytes_in_use = (int64_t) S.used;
    out->now_s = now_s();
    out->launches = S.launches;
    return PRR_OK;
}

} // extern "C"
