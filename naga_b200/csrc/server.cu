// Continuous-batching request loop over scenes of one lattice.
//
// A request is a scene (domain, parameters, initial density) plus a number
// of steps. Requests wait in a FIFO queue; each tick the server
//   1. enqueues `steps_per_tick` steps of every active scene (one batch,
//      one CUDA graph, asynchronous),
//   2. while those steps run, admits queued requests whose device memory fits
//      the budget and the slot limit: their set-up (kNN, RPIM and stencil
//      weights) runs on the scene's own stream, overlapping the batch,
//   3. waits for the batch, retires requests that have their steps (probe
//      trace copied to the host, scene freed), and adds the admitted scenes
//      to the batch for the next tick.
// Each active scene keeps its populations, stencils and tables resident on
// the device from admission to retirement. Per-step latency of the batch is
// measured with CUDA events on the batch stream.
//
// No reference counterpart: NAGA steps one engine at a time
// (fluids/nonlocal_lattice_boltzmann/simulation_engine.cuh:76).
#include "common.cuh"
#include "scene_dev.hpp"

#include <algorithm>
#include <chrono>
#include <deque>
#include <map>
#include <memory>
#include <string>
#include <vector>

using namespace naga;

namespace {

struct Request {
    int64_t id = 0;
    int state = 0;  // 0 queued, 1 active, 2 done, 3 failed
    int64_t steps = 0;
    int64_t base_steps = 0;  // scene step count at admission
    naga_scene_desc desc{};
    std::vector<float> points, normals, sigma, probes, drho;
    naga_scene* scene = nullptr;
    int64_t est_bytes = 0;
    std::vector<float> result;  // [steps][n_probes]
    std::string error;
    int64_t nodes = 0;
};

}  // namespace

struct naga_server {
    naga_server_config cfg{};
    naga_batch* batch = nullptr;
    std::deque<int64_t> queue;
    std::map<int64_t, std::unique_ptr<Request>> reqs;
    std::vector<int64_t> active;
    int64_t next_id = 1;
    int64_t bytes_in_use = 0, peak_bytes = 0;
    int64_t ticks = 0, steps = 0, node_updates = 0;
    double busy_ms = 0;
    double last_tick_ms = 0;     // device time of the previous tick's steps
    double prepare_ms = 0, admit_ms = 0, wait_ms = 0, retire_ms = 0;  // host wall time per tick phase
    std::vector<float> step_ms;  // per-step latency samples
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int64_t done = 0, failed = 0;
};

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
    // set-up scratch: kNN sort + distances, nearest-neighbour means
    b += N * (16 + 12 + (int64_t)d->k * 4 + 8);
    return b;
}

extern "C" int naga_server_create(const naga_server_config* cfg, naga_server** out) {
    if (!cfg || !out) return set_error(NAGA_EINVAL, "naga_server_create: null argument");
    if ((cfg->dim != 2 && cfg->dim != 3) || cfg->steps_per_tick < 1 || cfg->memory_budget <= 0 || cfg->max_active < 0 ||
        (cfg->step_priority != 0 && cfg->step_priority != 1))
        return set_error(NAGA_EINVAL, "naga_server_create: invalid configuration");
    auto s = std::make_unique<naga_server>();
    s->cfg = *cfg;
    int rc = naga_batch_create_with_priority(cfg->dim, cfg->step_priority, &s->batch);
    if (rc) return rc;
    NAGA_CUDA_TRY(cudaEventCreate(&s->ev0));
    NAGA_CUDA_TRY(cudaEventCreate(&s->ev1));
    *out = s.release();
    return NAGA_OK;
}

extern "C" int naga_server_destroy(naga_server* s) {
    if (!s) return NAGA_OK;
    if (s->batch) naga_batch_sync(s->batch);
    for (auto& kv : s->reqs)
        if (kv.second->scene) {
            naga_batch_remove(s->batch, kv.second->scene);
            naga_scene_destroy(kv.second->scene);
        }
    naga_batch_destroy(s->batch);
    if (s->ev0) cudaEventDestroy(s->ev0);
    if (s->ev1) cudaEventDestroy(s->ev1);
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
    r->id = s->next_id++;
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
    *id = r->id;
    s->queue.push_back(r->id);
    s->reqs[r->id] = std::move(r);
    return NAGA_OK;
}

namespace {

void fail_request(naga_server* s, Request& r, const std::string& why) {
    r.state = 3;
    r.error = why;
    s->failed++;
}

// set-up of one queued request (runs while the batch steps on its stream)
int admit(naga_server* s, Request& r) {
    naga_scene_desc d = r.desc;
    d.points = r.points.data();
    d.normals = r.normals.empty() ? nullptr : r.normals.data();
    d.sigma = r.sigma.empty() ? nullptr : r.sigma.data();
    d.probes = r.probes.empty() ? nullptr : r.probes.data();
    int rc = naga_scene_create(&d, &r.scene);
    if (rc) return rc;
    rc = naga_scene_set_density(r.scene, r.drho.empty() ? nullptr : r.drho.data());
    if (rc) {
        naga_scene_destroy(r.scene);
        r.scene = nullptr;
        return rc;
    }
    r.base_steps = naga_scene_step_count(r.scene);
    // inputs are on the device now
    r.points.clear();
    r.points.shrink_to_fit();
    r.drho.clear();
    r.drho.shrink_to_fit();
    return NAGA_OK;
}

}  // namespace

extern "C" int naga_server_tick(naga_server* s, int* n_active, int* n_queued) {
    if (!s) return set_error(NAGA_EINVAL, "naga_server_tick: null server");
    const int spt = s->cfg.steps_per_tick;
    // 1. steps of the active scenes, asynchronous on the batch stream
    const bool stepping = !s->active.empty();
    cudaStream_t bst = (cudaStream_t)naga_batch_stream(s->batch);
    int rc;
    using clock = std::chrono::steady_clock;
    auto since = [](clock::time_point t0) {
        return std::chrono::duration<double, std::milli>(clock::now() - t0).count();
    };
    if (stepping) {
        // membership changes (rebuild, first-time shape tuning, graph
        // capture) happen here, outside the timed window of the steps
        const auto t_prep = clock::now();
        if ((rc = naga_batch_prepare(s->batch))) return rc;
        s->prepare_ms += since(t_prep);
        NAGA_CUDA_TRY(cudaEventRecord(s->ev0, bst));
        if ((rc = naga_batch_step(s->batch, spt))) return rc;
        NAGA_CUDA_TRY(cudaEventRecord(s->ev1, bst));
    }
    // 2. admissions, overlapping the batch on the device. Set-up (kNN,
    // stencil and weight solves) runs on the host thread while the batch
    // steps; once this tick's set-up time exceeds the device time of the
    // previous tick's steps the rest waits, so a burst of arrivals does not
    // stall the running scenes (at least one request is admitted per tick).
    std::vector<int64_t> admitted;
    const auto t_admit = clock::now();
    const double admit_budget_ms = std::max(5.0, s->last_tick_ms);
    while (!s->queue.empty()) {
        if (!admitted.empty() && stepping && since(t_admit) > admit_budget_ms) break;
        Request& r = *s->reqs[s->queue.front()];
        const int slots_used = (int)(s->active.size() + admitted.size());
        if (s->cfg.max_active > 0 && slots_used >= s->cfg.max_active) break;
        if (r.est_bytes > s->cfg.memory_budget) {
            // can never fit: fail it rather than block the queue
            s->queue.pop_front();
            fail_request(s, r, "request needs more device memory than the server budget");
            continue;
        }
        if (s->bytes_in_use + r.est_bytes > s->cfg.memory_budget) break;
        s->queue.pop_front();
        rc = admit(s, r);
        if (rc == NAGA_ENOMEM) {
            // the device is fuller than the budget assumed: retry later
            s->queue.push_front(r.id);
            break;
        }
        if (rc) {
            fail_request(s, r, naga_last_error());
            continue;
        }
        s->bytes_in_use += r.est_bytes;
        s->peak_bytes = std::max(s->peak_bytes, s->bytes_in_use);
        r.state = 1;
        admitted.push_back(r.id);
    }
    s->admit_ms += since(t_admit);
    // 3. retire finished requests, then grow the batch
    if (stepping) {
        const auto t_wait = clock::now();
        NAGA_CUDA_TRY(cudaEventSynchronize(s->ev1));
        s->wait_ms += since(t_wait);
        float ms = 0;
        NAGA_CUDA_TRY(cudaEventElapsedTime(&ms, s->ev0, s->ev1));
        s->busy_ms += ms;
        s->last_tick_ms = ms;
        for (int t = 0; t < spt; ++t) s->step_ms.push_back(ms / spt);
        s->ticks++;
        s->steps += spt;
        for (int64_t id : s->active) s->node_updates += s->reqs[id]->nodes * spt;
    }
    const auto t_retire = clock::now();
    std::vector<int64_t> still;
    for (int64_t id : s->active) {
        Request& r = *s->reqs[id];
        const int64_t done = naga_scene_step_count(r.scene) - r.base_steps;
        if (done < r.steps) {
            still.push_back(id);
            continue;
        }
        const int np = r.desc.n_probes;
        r.result.assign((size_t)r.steps * std::max(np, 0), 0.f);
        if (np > 0 && (rc = naga_scene_read_probes(r.scene, r.base_steps, r.steps, r.result.data())))
            fail_request(s, r, naga_last_error());
        else {
            r.state = 2;
            s->done++;
        }
        naga_batch_remove(s->batch, r.scene);
        naga_scene_destroy(r.scene);
        r.scene = nullptr;
        s->bytes_in_use -= r.est_bytes;
    }
    s->active.swap(still);
    for (int64_t id : admitted) {
        if ((rc = naga_batch_add(s->batch, s->reqs[id]->scene))) return rc;
        s->active.push_back(id);
    }
    s->retire_ms += since(t_retire);
    if (n_active) *n_active = (int)s->active.size();
    if (n_queued) *n_queued = (int)s->queue.size();
    return NAGA_OK;
}

extern "C" int naga_server_request_state(naga_server* s, int64_t id, int* state, int64_t* steps_done) {
    if (!s) return set_error(NAGA_EINVAL, "naga_server_request_state: null server");
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return set_error(NAGA_EINVAL, "naga_server_request_state: unknown request");
    Request& r = *it->second;
    if (state) *state = r.state;
    if (steps_done) *steps_done = r.state == 2 ? r.steps : (r.scene ? naga_scene_step_count(r.scene) - r.base_steps : 0);
    if (r.state == 3) set_error(NAGA_EINVAL, r.error);
    return NAGA_OK;
}

extern "C" int naga_server_result(naga_server* s, int64_t id, float* probes) {
    if (!s) return set_error(NAGA_EINVAL, "naga_server_result: null server");
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
    st.bytes_in_use = s->bytes_in_use;
    st.peak_bytes = s->peak_bytes;
    st.active = (int)s->active.size();
    st.queued = (int)s->queue.size();
    st.done = s->done;
    st.failed = s->failed;
    st.prepare_ms = s->prepare_ms;
    st.admit_ms = s->admit_ms;
    st.wait_ms = s->wait_ms;
    st.retire_ms = s->retire_ms;
    if (!s->step_ms.empty()) {
        std::vector<float> v = s->step_ms;
        auto pct = [&](double p) {
            size_t k = (size_t)std::min<double>(v.size() - 1, std::max(0.0, p * (v.size() - 1)));
            std::nth_element(v.begin(), v.begin() + k, v.end());
            return (double)v[k];
        };
        st.p50_step_ms = pct(0.50);
        st.p99_step_ms = pct(0.99);
    }
    *out = st;
    return NAGA_OK;
}
