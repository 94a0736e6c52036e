// Continuous-batching request loop over scenes of one lattice.
//
// A request is a scene (domain, parameters, initial density) plus a number
// of steps. Two threads share the work:
//   * the caller's thread runs naga_server_tick: it enqueues
//     `steps_per_tick` steps of every active scene (one batch, one CUDA
//     graph launch per step, a CUDA event after each), waits for them,
//     retires the requests that have their steps (probe trace copied to the
//     host) and adds the scenes that finished set-up to the batch;
//   * the server's set-up thread admits queued requests in FIFO order --
//     their set-up (kNN, RPIM and stencil weight solves, initial state) runs
//     on each scene's own stream, overlapping the batch's steps on the
//     device -- and frees retired scenes, so the tick never waits on host
//     set-up or on a device-synchronising free.
// Admission takes a request when its device memory fits the budget, a slot
// is free and, with a per-step latency target, when the batch's step time
// with it -- estimated from the measured time per node-step -- stays within
// the target (an empty batch always admits one request). Each active scene
// keeps its populations, stencils and tables resident on the device from
// admission to retirement.
//
// No reference counterpart: NAGA steps one engine at a time
// (fluids/nonlocal_lattice_boltzmann/simulation_engine.cuh:76).
#include "common.cuh"
#include "scene_dev.hpp"

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

using namespace naga;

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

struct Request {
    int64_t id = 0;
    int state = 0;  // 0 queued (or in set-up), 1 active, 2 done, 3 failed
    int64_t steps = 0;
    int64_t base_steps = 0;  // scene step count at admission
    naga_scene_desc desc{};
    std::vector<float> points, normals, sigma, probes, drho;
    naga_scene* scene = nullptr;
    int64_t est_bytes = 0;
    std::vector<float> result;  // [steps][n_probes]
    std::string error;
    int64_t nodes = 0;
    Clock::time_point t_submit, t_admit;
};

}  // namespace

struct naga_server {
    naga_server_config cfg{};
    int device = 0;
    naga_batch* batch = nullptr;
    std::map<int64_t, std::unique_ptr<Request>> reqs;  // guarded by mu
    std::deque<int64_t> queue;                         // guarded by mu
    std::vector<Request*> ready;                       // set up, not yet in the batch (mu)
    std::vector<naga_scene*> to_free;                  // retired scenes the set-up thread frees (mu)
    std::vector<Request*> active;                      // tick thread only
    int active_count = 0;                              // mu: size of `active`
    int64_t bytes_in_use = 0, peak_bytes = 0;          // mu
    int64_t active_nodes = 0, pending_nodes = 0;       // mu: in the batch / set up or setting up
    int setting_up = 0;                                // mu
    double ms_per_node_step = 0;                       // mu: measured batch step time per node
    int64_t next_id = 1;                               // mu
    int64_t ticks = 0, steps = 0, node_updates = 0;
    double busy_ms = 0;
    double prepare_ms = 0, admit_ms = 0, wait_ms = 0, retire_ms = 0;
    std::vector<float> step_ms;     // per-step latency samples (CUDA events)
    std::vector<double> request_ms; // submit -> finished, per completed request (mu)
    std::vector<double> queue_ms;   // submit -> admitted (set-up done), per admitted request (mu)
    std::vector<cudaEvent_t> ev;    // steps_per_tick + 1 events on the batch stream
    int64_t done = 0, failed = 0;   // mu
    std::mutex mu;
    // held around the batch's graph capture (tick thread) and around the
    // set-up thread's frees: cudaFree synchronises the device, which a
    // stream capture in progress must not see
    std::mutex capture_mu;
    std::condition_variable cv;
    bool stop = false;
    std::thread worker;
};

namespace {

void fail_request(naga_server* s, Request& r, const std::string& why) {
    r.state = 3;
    r.error = why;
    s->failed++;
}

// set-up of one queued request on the set-up thread (the batch keeps
// stepping on its own stream meanwhile)
int setup_scene(Request& r) {
    naga_scene_desc d = r.desc;
    d.points = r.points.data();
    d.normals = r.normals.empty() ? nullptr : r.normals.data();
    d.sigma = r.sigma.empty() ? nullptr : r.sigma.data();
    d.probes = r.probes.empty() ? nullptr : r.probes.data();
    int rc = naga_scene_create(&d, &r.scene);
    if (rc) return rc;
    rc = naga_scene_set_density(r.scene, r.drho.empty() ? nullptr : r.drho.data());
    if (rc == NAGA_OK) rc = naga_scene_sync(r.scene);
    if (rc) {
        naga_scene_destroy(r.scene);
        r.scene = nullptr;
        return rc;
    }
    r.base_steps = naga_scene_step_count(r.scene);
    // the inputs live on the device now
    r.points = {};
    r.drho = {};
    return NAGA_OK;
}

// whether the queue's front request may start set-up now (mu held)
bool may_admit(const naga_server* s, const Request& r) {
    const int slots = s->active_count + (int)s->ready.size() + s->setting_up;
    if (s->cfg.max_active > 0 && slots >= s->cfg.max_active) return false;
    if (s->bytes_in_use + r.est_bytes > s->cfg.memory_budget) return false;
    // with a latency target, a scene joins a non-empty batch only once a
    // step has been measured and the estimate with it stays on target
    const int64_t nodes = s->active_nodes + s->pending_nodes;
    if (s->cfg.target_step_ms > 0 && nodes > 0 &&
        (s->ms_per_node_step <= 0 || (double)(nodes + r.nodes) * s->ms_per_node_step > s->cfg.target_step_ms))
        return false;
    return true;
}

void setup_thread(naga_server* s) {
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        // retired scenes first: their memory may let the next request in
        if (!s->to_free.empty()) {
            std::vector<naga_scene*> f;
            f.swap(s->to_free);
            lk.unlock();
            {
                std::lock_guard<std::mutex> cl(s->capture_mu);
                for (naga_scene* sc : f) naga_scene_destroy(sc);
            }
            lk.lock();
            s->cv.notify_all();
            continue;
        }
        if (s->stop) return;
        // requests that can never fit fail instead of blocking the queue
        while (!s->queue.empty() && s->reqs[s->queue.front()]->est_bytes > s->cfg.memory_budget) {
            Request& r = *s->reqs[s->queue.front()];
            s->queue.pop_front();
            fail_request(s, r, "request needs more device memory than the server budget");
        }
        if (s->queue.empty() || !may_admit(s, *s->reqs[s->queue.front()])) {
            s->cv.wait(lk);
            continue;
        }
        Request& r = *s->reqs[s->queue.front()];
        s->queue.pop_front();
        s->bytes_in_use += r.est_bytes;
        s->peak_bytes = std::max(s->peak_bytes, s->bytes_in_use);
        s->pending_nodes += r.nodes;
        s->setting_up++;
        lk.unlock();
        const auto t0 = Clock::now();
        const int rc = setup_scene(r);
        const std::string err = rc ? naga_last_error() : std::string();
        const auto t1 = Clock::now();
        lk.lock();
        s->setting_up--;
        s->admit_ms += ms_between(t0, t1);
        if (rc == NAGA_ENOMEM && !s->stop) {
            // the device is fuller than the budget assumed: back to the
            // front of the queue until a retirement frees memory
            s->bytes_in_use -= r.est_bytes;
            s->pending_nodes -= r.nodes;
            s->queue.push_front(r.id);
            s->cv.wait(lk);
            continue;
        }
        if (rc) {
            s->bytes_in_use -= r.est_bytes;
            s->pending_nodes -= r.nodes;
            fail_request(s, r, err);
            continue;
        }
        r.t_admit = t1;
        s->queue_ms.push_back(ms_between(r.t_submit, t1));
        s->ready.push_back(&r);
    }
}

double percentile(std::vector<double> v, double p) {
    if (v.empty()) return 0.0;
    const size_t k = (size_t)std::min<double>((double)v.size() - 1, std::max(0.0, p * ((double)v.size() - 1)));
    std::nth_element(v.begin(), v.begin() + (ptrdiff_t)k, v.end());
    return v[k];
}

}  // namespace

// Device bytes a scene will hold (engine.cu allocation plan) plus the
// transient set-up scratch, used for admission before the scene exists.
extern "C" int64_t naga_scene_estimate_bytes(const naga_scene_desc* d) {
    if (!d || (d->dim != 2 && d->dim != 3)) return -1;
    const int64_t N = d->n_bulk + d->n_layer + d->n_boundary + d->n_ghost;
    const int64_t QP = d->dim == 2 ? D2Q9::QP : D3Q27::QP;
    const int64_t rec = 16;  // float4 stencil records (plus 8-B filter records below)
    int64_t b = N * (7 * QP * 4 + 16 + 1 + (int64_t)d->k * (rec + 8 + 4) + 4 * d->dim);
    b += (int64_t)d->n_boundary * d->k_boundary * 8 + (int64_t)d->n_probes * d->k_probe * 8;
    b += ((N + 127) / 128) * 2 * QP * 8 + (int64_t)std::max(1, d->probe_capacity) * std::max(1, d->n_probes) * 4;
    // PML field rows of the layer and the per-node mean vectors
    b += d->n_layer * QP * 4 + (d->n_bulk + d->n_layer + 1) * 32;
    if (d->n_layer > 0) b += (d->n_bulk + d->n_layer) * (int64_t)d->k * 16;  // PML gather records
    if (d->dim == 2) b += N * (int64_t)d->k * 12;                           // compact stencil triplets
    if (d->dim == 3 && d->k == kHaloK)                                      // RK stage halo blobs
        b += (d->n_bulk + d->n_layer + 31) / 32 * (int64_t)kHaloBlobBytes;
    // set-up scratch: kNN sort + distances, nearest-neighbour means
    b += N * (16 + 12 + (int64_t)d->k * 4 + 8);
    return b;
}

extern "C" int naga_server_create(const naga_server_config* cfg, naga_server** out) {
    if (!cfg || !out) return set_error(NAGA_EINVAL, "naga_server_create: null argument");
    if ((cfg->dim != 2 && cfg->dim != 3) || cfg->steps_per_tick < 1 || cfg->memory_budget <= 0 || cfg->max_active < 0 ||
        (cfg->step_priority != 0 && cfg->step_priority != 1) || !(cfg->target_step_ms >= 0))
        return set_error(NAGA_EINVAL, "naga_server_create: invalid configuration");
    auto s = std::make_unique<naga_server>();
    s->cfg = *cfg;
    NAGA_CUDA_TRY(cudaGetDevice(&s->device));
    int rc = naga_batch_create_with_priority(cfg->dim, cfg->step_priority, &s->batch);
    if (rc) return rc;
    s->ev.assign((size_t)cfg->steps_per_tick + 1, nullptr);
    for (auto& e : s->ev) NAGA_CUDA_TRY(cudaEventCreate(&e));
    s->worker = std::thread(setup_thread, s.get());
    *out = s.release();
    return NAGA_OK;
}

extern "C" int naga_server_destroy(naga_server* s) {
    if (!s) return NAGA_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv.notify_all();
    if (s->worker.joinable()) s->worker.join();
    if (s->batch) naga_batch_sync(s->batch);
    for (naga_scene* sc : s->to_free) naga_scene_destroy(sc);
    for (auto& kv : s->reqs)
        if (kv.second->scene) {
            naga_batch_remove(s->batch, kv.second->scene);
            naga_scene_destroy(kv.second->scene);
        }
    s->reqs.clear();
    naga_batch_destroy(s->batch);
    for (auto& e : s->ev)
        if (e) cudaEventDestroy(e);
    delete s;
    return NAGA_OK;
}

extern "C" int naga_server_submit(naga_server* s, const naga_scene_desc* d, const float* drho, int64_t steps,
                                  int64_t* id) {
    if (!s || !d || !id) return set_error(NAGA_EINVAL, "naga_server_submit: null argument");
    if (d->dim != s->cfg.dim) return set_error(NAGA_EINVAL, "naga_server_submit: lattice differs from the server's");
    if (steps < 1) return set_error(NAGA_EINVAL, "naga_server_submit: steps must be >= 1");
    const int64_t N = d->n_bulk + d->n_layer + d->n_boundary + d->n_ghost;
    if (N <= 0 || !d->points) return set_error(NAGA_EINVAL, "naga_server_submit: empty domain");
    auto r = std::make_unique<Request>();
    r->steps = steps;
    r->desc = *d;
    r->nodes = N;
    const int D = d->dim;
    r->points.assign(d->points, d->points + N * D);
    if (d->n_boundary && d->normals) r->normals.assign(d->normals, d->normals + d->n_boundary * D);
    if (d->n_layer && d->sigma) r->sigma.assign(d->sigma, d->sigma + d->n_layer);
    if (d->n_probes && d->probes) r->probes.assign(d->probes, d->probes + (int64_t)d->n_probes * D);
    if (drho) r->drho.assign(drho, drho + N);
    // the probe ring holds the whole request plus one tick of overshoot
    r->desc.probe_capacity = (int)std::min<int64_t>(steps + s->cfg.steps_per_tick, 1 << 30);
    r->est_bytes = naga_scene_estimate_bytes(&r->desc);
    r->t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        r->id = s->next_id++;
        *id = r->id;
        s->queue.push_back(r->id);
        s->reqs[r->id] = std::move(r);
    }
    s->cv.notify_all();
    return NAGA_OK;
}

extern "C" int naga_server_tick(naga_server* s, int* n_active, int* n_queued) {
    if (!s) return set_error(NAGA_EINVAL, "naga_server_tick: null server");
    const int spt = s->cfg.steps_per_tick;
    cudaStream_t bst = (cudaStream_t)naga_batch_stream(s->batch);
    int rc;
    // 1. steps of the active scenes, one event after each step
    const bool stepping = !s->active.empty();
    if (stepping) {
        // membership changes (rebuild, first-time shape tuning, graph
        // capture) happen here, outside the timed steps
        const auto t0 = Clock::now();
        {
            std::lock_guard<std::mutex> cl(s->capture_mu);
            rc = naga_batch_prepare(s->batch);
        }
        if (rc) return rc;
        s->prepare_ms += ms_between(t0, Clock::now());
        NAGA_CUDA_TRY(cudaEventRecord(s->ev[0], bst));
        for (int t = 0; t < spt; ++t) {
            if ((rc = naga_batch_step(s->batch, 1))) return rc;
            NAGA_CUDA_TRY(cudaEventRecord(s->ev[t + 1], bst));
        }
        const auto t1 = Clock::now();
        NAGA_CUDA_TRY(cudaEventSynchronize(s->ev[spt]));
        s->wait_ms += ms_between(t1, Clock::now());
        float total = 0;
        for (int t = 0; t < spt; ++t) {
            float ms = 0;
            NAGA_CUDA_TRY(cudaEventElapsedTime(&ms, s->ev[t], s->ev[t + 1]));
            s->step_ms.push_back(ms);
            total += ms;
        }
        s->busy_ms += total;
        s->ticks++;
        s->steps += spt;
        int64_t nodes = 0;
        for (const Request* r : s->active) nodes += r->nodes;
        s->node_updates += nodes * spt;
        // time per node-step of this batch: the admission estimate
        {
            std::lock_guard<std::mutex> lk(s->mu);
            const double m = total / spt / (double)std::max<int64_t>(nodes, 1);
            s->ms_per_node_step = s->ms_per_node_step > 0 ? 0.5 * (s->ms_per_node_step + m) : m;
        }
        if (s->cfg.target_step_ms > 0) s->cv.notify_all();
    }
    // 2. retire finished requests; their scenes go to the set-up thread to
    // be freed. Then the scenes that finished set-up join the batch.
    const auto t_retire = Clock::now();
    struct Finished {
        Request* r;
        std::vector<float> result;
        int rc;
        std::string error;
    };
    std::vector<Request*> still;
    std::vector<Finished> fin;
    for (Request* r : s->active) {
        const int64_t done = naga_scene_step_count(r->scene) - r->base_steps;
        if (done < r->steps) {
            still.push_back(r);
            continue;
        }
        Finished f{r, {}, NAGA_OK, {}};
        const int np = r->desc.n_probes;
        f.result.assign((size_t)r->steps * std::max(np, 0), 0.f);
        if (np > 0 && (f.rc = naga_scene_read_probes(r->scene, r->base_steps, r->steps, f.result.data())))
            f.error = naga_last_error();
        naga_batch_remove(s->batch, r->scene);
        fin.push_back(std::move(f));
    }
    std::vector<Request*> joining;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        const auto now = Clock::now();
        for (Finished& f : fin) {
            Request& r = *f.r;
            if (f.rc) {
                r.state = 3;
                r.error = f.error;
                s->failed++;
            } else {
                r.state = 2;
                r.result = std::move(f.result);
                s->done++;
                s->request_ms.push_back(ms_between(r.t_submit, now));
            }
            // freed by the set-up thread; the batch's next prepare (before
            // any further step) no longer references it
            s->to_free.push_back(r.scene);
            r.scene = nullptr;
            s->active_nodes -= r.nodes;
            s->bytes_in_use -= r.est_bytes;
        }
        joining.swap(s->ready);
        for (Request* r : joining) {
            r->state = 1;
            s->pending_nodes -= r->nodes;
            s->active_nodes += r->nodes;
        }
        s->active_count = (int)(still.size() + joining.size());
    }
    s->active.swap(still);
    for (Request* r : joining) {
        if ((rc = naga_batch_add(s->batch, r->scene))) return rc;
        s->active.push_back(r);
    }
    if (!fin.empty() || !joining.empty()) s->cv.notify_all();
    s->retire_ms += ms_between(t_retire, Clock::now());
    if (n_active) *n_active = (int)s->active.size();
    if (n_queued) {
        std::lock_guard<std::mutex> lk(s->mu);
        *n_queued = (int)s->queue.size() + s->setting_up + (int)s->ready.size();
    }
    return NAGA_OK;
}

extern "C" int naga_server_request_state(naga_server* s, int64_t id, int* state, int64_t* steps_done) {
    if (!s) return set_error(NAGA_EINVAL, "naga_server_request_state: null server");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return set_error(NAGA_EINVAL, "naga_server_request_state: unknown request");
    Request& r = *it->second;
    if (state) *state = r.state;
    if (steps_done)
        *steps_done = r.state == 2 ? r.steps
                                   : (r.state == 1 && r.scene ? naga_scene_step_count(r.scene) - r.base_steps : 0);
    if (r.state == 3) set_error(NAGA_EINVAL, r.error);
    return NAGA_OK;
}

extern "C" int naga_server_result(naga_server* s, int64_t id, float* probes) {
    if (!s) return set_error(NAGA_EINVAL, "naga_server_result: null server");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return set_error(NAGA_EINVAL, "naga_server_result: unknown request");
    Request& r = *it->second;
    if (r.state == 3) return set_error(NAGA_EINVAL, "naga_server_result: request failed: " + r.error);
    if (r.state != 2) return set_error(NAGA_EINVAL, "naga_server_result: request not finished");
    if (probes && !r.result.empty()) std::copy(r.result.begin(), r.result.end(), probes);
    s->reqs.erase(it);
    return NAGA_OK;
}

extern "C" int naga_server_read_stats(naga_server* s, naga_server_stats* out) {
    if (!s || !out) return set_error(NAGA_EINVAL, "naga_server_read_stats: null argument");
    naga_server_stats st{};
    st.ticks = s->ticks;
    st.steps = s->steps;
    st.node_updates = s->node_updates;
    st.busy_ms = s->busy_ms;
    st.active = (int)s->active.size();
    st.prepare_ms = s->prepare_ms;
    st.wait_ms = s->wait_ms;
    st.retire_ms = s->retire_ms;
    if (!s->step_ms.empty()) {
        std::vector<double> v(s->step_ms.begin(), s->step_ms.end());
        st.p50_step_ms = percentile(v, 0.50);
        st.p99_step_ms = percentile(v, 0.99);
    }
    std::lock_guard<std::mutex> lk(s->mu);
    st.bytes_in_use = s->bytes_in_use;
    st.peak_bytes = s->peak_bytes;
    st.queued = (int)s->queue.size() + s->setting_up + (int)s->ready.size();
    st.done = s->done;
    st.failed = s->failed;
    st.admit_ms = s->admit_ms;
    st.p50_request_ms = percentile(s->request_ms, 0.50);
    st.p99_request_ms = percentile(s->request_ms, 0.99);
    st.p50_queue_ms = percentile(s->queue_ms, 0.50);
    st.admitted = (int64_t)s->queue_ms.size();
    *out = st;
    return NAGA_OK;
}
