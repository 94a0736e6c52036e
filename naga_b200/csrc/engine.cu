// Scenes and batches: device memory, the set-up pipeline (kNN, stencil and
// RPIM weights on the GPU), work tables, CUDA-graph replay of the step, and
// the C ABI around them.
//
// Reference: fluids/nonlocal_lattice_boltzmann/simulation_engine.cuh:40-121
// (public engine) and detail/simulation_engine.cuh:94-339 (parameters and
// init_domain), simulation_observers/density_observer.cuh:62-113 (probes).
#include "common.cuh"
#include "scene_dev.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <type_traits>
#include <vector>

namespace naga {

int sm_count() {
    static int cached[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) dev = 0;
    if (!cached[dev]) {
        int v = 0;
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
        cached[dev] = v > 0 ? v : 148;
    }
    return cached[dev];
}

// ------------------------------------------------------------- profiling
namespace {
struct ProfState {
    bool on = false;
    std::mutex mu;
    struct Rec {
        int id;
        cudaEvent_t a, b;
    };
    std::vector<Rec> pending;
    std::vector<int64_t> launches;
    std::vector<double> ms;
    cudaEvent_t cur_a = nullptr;
} g_prof;

void prof_drain() {
    for (auto& r : g_prof.pending) {
        cudaEventSynchronize(r.b);
        float t = 0;
        cudaEventElapsedTime(&t, r.a, r.b);
        if ((size_t)r.id >= g_prof.ms.size()) {
            g_prof.ms.resize(r.id + 1, 0.0);
            g_prof.launches.resize(r.id + 1, 0);
        }
        g_prof.ms[r.id] += t;
        g_prof.launches[r.id] += 1;
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    g_prof.pending.clear();
}
}  // namespace

bool prof_on() { return g_prof.on; }
void prof_begin(int, cudaStream_t st) {
    cudaEventCreate(&g_prof.cur_a);
    cudaEventRecord(g_prof.cur_a, st);
}
void prof_end(int id, cudaStream_t st) {
    cudaEvent_t b;
    cudaEventCreate(&b);
    cudaEventRecord(b, st);
    std::lock_guard<std::mutex> lk(g_prof.mu);
    g_prof.pending.push_back({id, g_prof.cur_a, b});
    if (g_prof.pending.size() > 4096) prof_drain();
}

}  // namespace naga

using namespace naga;

// ================================================================ objects
struct naga_batch;

struct naga_scene {
    int dim = 0, Q = 0, QP = 0;
    naga_scene_desc desc{};
    int64_t N = 0, nb = 0, nl = 0, nbd = 0, ng = 0, nbl = 0, nd = 0;
    cudaStream_t stream = nullptr;
    SceneDev dev{};
    std::vector<void*> allocs;
    int64_t bytes = 0;
    std::vector<WorkItem> items_all, items_all_mt, items_fluid, items_edge, items_pml;  // scene slot 0
    WorkItem* d_lists = nullptr;  // the five lists above back to back on the device (batch rebuilds copy them)
    int64_t n_list[5] = {};
    naga_batch* owner = nullptr;                               // user batch, if any
    naga_batch* solo = nullptr;                                // private batch for naga_scene_step
    int64_t steps = 0;                                         // host mirror of the device counter
    int* src_slot = nullptr;                                   // density sources (see SceneDev)
    float* src_vals = nullptr;
    int64_t src_vals_cap = 0;
    std::vector<int64_t> src_nodes;
    std::vector<float> probe_xyz;
    float* d_pts = nullptr;  // node coordinates on the device (probe tables)

    template <class T>
    int alloc(T** p, int64_t count) {
        size_t b = sizeof(T) * (size_t)std::max<int64_t>(count, 1);
        cudaError_t e = cudaMalloc((void**)p, b);
        if (e != cudaSuccess) {
            *p = nullptr;
            cudaGetLastError();
            return set_error(e == cudaErrorMemoryAllocation ? NAGA_ENOMEM : NAGA_ECUDA,
                             std::string("naga_scene_create: cudaMalloc: ") + cudaGetErrorString(e));
        }
        allocs.push_back((void*)*p);
        bytes += (int64_t)b;
        return NAGA_OK;
    }
};

// one scene's item list copied into a batch list, with the scene slot set
struct ListCopy {
    const WorkItem* src;
    int64_t dst;
    uint32_t n, scene;
};

struct naga_batch {
    int dim = 0;
    bool is_solo = false;
    std::vector<naga_scene*> members;
    bool dirty = true;
    cudaStream_t stream = nullptr;
    SceneDev* d_scenes = nullptr;
    WorkItem *d_all = nullptr, *d_all_mt = nullptr, *d_fluid = nullptr, *d_edge = nullptr, *d_pml = nullptr;
    int n_all = 0, n_all_mt = 0, n_fluid = 0, n_edge = 0, n_pml = 0;
    int k = 0, kb = 0;  // common stencil sizes of the members (0 if they differ)
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    // grow-only device tables (a membership change rewrites them in place on
    // the batch stream; they are reallocated only when they must grow)
    WorkItem* d_items = nullptr;  // the five item lists back to back
    int64_t items_cap = 0;
    int scenes_cap = 0;
    ListCopy* d_copies = nullptr;
    int copies_cap = 0;
    void* h_stage = nullptr;  // page-locked staging of the scene and copy tables
    size_t stage_cap = 0;

    void free_graph() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
    }
    void free_tables() {
        free_graph();
        if (d_scenes) cudaFree(d_scenes);
        if (d_items) cudaFree(d_items);
        if (d_copies) cudaFree(d_copies);
        if (h_stage) cudaFreeHost(h_stage);
        d_scenes = nullptr;
        d_items = nullptr;
        d_copies = nullptr;
        h_stage = nullptr;
        d_all = d_all_mt = d_fluid = d_edge = d_pml = nullptr;
        items_cap = stage_cap = 0;
        scenes_cap = copies_cap = 0;
    }
};

__global__ void concat_items_kernel(const ListCopy* __restrict__ copies, WorkItem* __restrict__ dst) {
    const ListCopy c = copies[blockIdx.y];
    for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < c.n; w += gridDim.x * blockDim.x) {
        WorkItem it = c.src[w];
        it.scene = c.scene;
        dst[c.dst + w] = it;
    }
}

// boundary interpolation records (weight, source index bits) in pass order
// from the RPIM support indices / weights [nq][kk], and the flag of every
// node some boundary node interpolates from (idempotent stores)
__global__ void boundary_records_kernel(const uint32_t* __restrict__ idx, const double* __restrict__ w, int64_t nq,
                                        int kk, int npb, float2* __restrict__ rec, uint8_t* __restrict__ is_src) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nq * kk) return;
    const int64_t q = e / kk;
    const int t = (int)(e - q * kk);
    const uint32_t j = idx[e];
    rec[pass_record(q, t, kk, nq, nq, npb)] = make_float2((float)w[e], __uint_as_float(j));
    is_src[j] = 1;
}

// the largest layer-support count of each PML item's nodes (the count of
// node i rides in the bits of PV[2 i].w): the item's PML tile only needs
// that many records per node
__global__ void pml_item_kmax_kernel(const WorkItem* __restrict__ items, int n, const float4* __restrict__ PV,
                                     uint32_t* __restrict__ kmax) {
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= n) return;
    uint32_t m = 0;
    for (uint32_t i = items[w].begin; i < items[w].end; ++i) m = max(m, __float_as_uint(PV[2 * (int64_t)i].w));
    kmax[w] = m;
}

// flag[w] = 1 when a node of item w has a stencil support in the layer
// [nb, nb + nl) (idx: node-major [n][k] kNN indices)
__global__ void layer_touch_kernel(const uint32_t* __restrict__ idx, int k, const WorkItem* __restrict__ items,
                                   int nitems, int64_t nb, int64_t nl, uint8_t* __restrict__ flag) {
    const int w = blockIdx.x;
    if (w >= nitems) return;
    const WorkItem it = items[w];
    const int64_t n = (int64_t)(it.end - it.begin) * k;
    int touch = 0;
    for (int64_t e = threadIdx.x; e < n && !touch; e += blockDim.x) {
        const int64_t j = idx[(int64_t)it.begin * k + e];
        touch = j >= nb && j < nb + nl;
    }
    touch = __syncthreads_or(touch);
    if (threadIdx.x == 0) flag[w] = (uint8_t)touch;
}

namespace {

cudaStream_t active_stream(naga_scene* s) { return s->owner ? s->owner->stream : s->stream; }

int check_device() {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        cudaGetLastError();
        return set_error(NAGA_ENODEVICE, "no CUDA device available");
    }
    return NAGA_OK;
}

void make_items(int64_t begin, int64_t end, std::vector<WorkItem>& out, int size = 128) {
    out.clear();
    uint32_t local = 0;
    for (int64_t b = begin; b < end; b += size)
        out.push_back({0u, (uint32_t)b, (uint32_t)std::min<int64_t>(end, b + size), local++});
}

// slot of population a in a node row (paired order, see common.cuh)
int slot_of(int dim, int a) { return dim == 2 ? D2Q9::pos(a) : D3Q27::pos(a); }

float lattice_cs_f() { return 0.57735026918962576450914878050196f; }

// set_problem_parameters (detail/simulation_engine.cuh:94-124) in FP32, and
// the relaxation rates of the collision models
void set_parameters(naga_scene* s) {
    const naga_scene_desc& d = s->desc;
    SceneDev& D = s->dev;
    const float c = (float)d.speed_of_sound;
    const float ratio = lattice_cs_f() / c;
    const float dt_lat = (float)d.time_step / ratio;
    const float nu_lat = (float)d.viscosity / ratio;
    D.dt_lat = dt_lat;
    D.inv_dt = 1.f / dt_lat;
    D.rho0 = (float)d.rho0;
    if (s->dim == 3) {
        D.om_ab = 1.f / (3.f * nu_lat + .5f) / dt_lat;
        const float fixed[6] = {1.5f, 1.83f, 1.4f, 1.61f, 1.98f, 1.74f};
        for (int t = 0; t < 6; ++t) {
            float unit_nu = (1.f / fixed[t] - .5f) / 3.f;
            D.om_fix[t] = 1.f / (3.f * unit_nu + .5f) / dt_lat;
        }
    } else {
        D.om_ab = 1.f / (3.f * nu_lat + .5f * dt_lat);
        for (int t = 0; t < 6; ++t) D.om_fix[t] = 0.f;
    }
    D.rk_a[0] = dt_lat * 0.25f;
    D.rk_a[1] = dt_lat * (float)(1.0 / 3.0);
    D.rk_a[2] = dt_lat * 0.5f;
    D.rk_a[3] = dt_lat;
    D.half_dt = dt_lat / 2.f;
}

// RPIM interpolation tables at nq host query points from the first nsrc
// nodes (kNN + weight solves on the device): the boundary form writes
// pass-ordered (weight, index) records and flags the sources in dsrc; the
// probe form writes [kk][nq] index and weight tables
int rpim_tables(naga_scene* s, const float* pts, const float* qry_host, int64_t nq, int64_t nsrc, int kk,
                uint32_t** idx_out, float** w_out, float2** rec_out, uint8_t* dsrc) {
    const naga_scene_desc& d = s->desc;
    const int D = s->dim;
    const int npb = nodes_per_pass(D);
    cudaStream_t st = s->stream;
    uint32_t* didx = nullptr;
    float* dd2 = nullptr;
    float* dq = nullptr;
    double* dqd = nullptr;
    double* dw = nullptr;
    NAGA_CUDA_TRY(cudaMallocAsync(&didx, sizeof(uint32_t) * nq * kk, st));
    NAGA_CUDA_TRY(cudaMallocAsync(&dd2, sizeof(float) * nq * kk, st));
    NAGA_CUDA_TRY(cudaMallocAsync(&dq, sizeof(float) * nq * D, st));
    NAGA_CUDA_TRY(cudaMallocAsync(&dqd, sizeof(double) * nq * D, st));
    NAGA_CUDA_TRY(cudaMallocAsync(&dw, sizeof(double) * nq * kk, st));
    std::vector<double> qd(nq * D);
    for (int64_t t = 0; t < nq * D; ++t) qd[t] = qry_host[t];
    NAGA_CUDA_TRY(cudaMemcpyAsync(dq, qry_host, sizeof(float) * nq * D, cudaMemcpyHostToDevice, st));
    NAGA_CUDA_TRY(cudaMemcpyAsync(dqd, qd.data(), sizeof(double) * nq * D, cudaMemcpyHostToDevice, st));
    int r = knn_device(pts, nsrc, dq, nq, D, kk, didx, dd2, st);
    if (!r) r = rbf_weights_device(pts, nsrc, D, didx, kk, dqd, nq, 1, d.nodal_spacing, d.shape,
                                   d.weight_precision, dw, st);
    if (!r && rec_out) {
        // boundary: records and source flags built on the device
        r = s->alloc(rec_out, nq * kk);
        if (!r) {
            const int64_t ne = nq * kk;
            boundary_records_kernel<<<(unsigned)((ne + 255) / 256), 256, 0, st>>>(didx, dw, nq, kk, npb, *rec_out,
                                                                                  dsrc);
            cudaError_t e = cudaGetLastError();
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) r = set_error(NAGA_ECUDA, std::string("boundary records: ") + cudaGetErrorString(e));
        }
        cudaFreeAsync(didx, st);
        cudaFreeAsync(dd2, st);
        cudaFreeAsync(dq, st);
        cudaFreeAsync(dqd, st);
        cudaFreeAsync(dw, st);
        return r;
    }
    std::vector<uint32_t> hi(nq * kk);
    std::vector<double> hw(nq * kk);
    if (!r) {
        cudaError_t e1 = cudaMemcpyAsync(hi.data(), didx, sizeof(uint32_t) * nq * kk, cudaMemcpyDeviceToHost, st);
        cudaError_t e2 = cudaMemcpyAsync(hw.data(), dw, sizeof(double) * nq * kk, cudaMemcpyDeviceToHost, st);
        cudaError_t e3 = cudaStreamSynchronize(st);
        if (e1 || e2 || e3) r = set_error(NAGA_ECUDA, "naga_scene_create: copy of interpolation tables failed");
    }
    cudaFreeAsync(didx, st);
    cudaFreeAsync(dd2, st);
    cudaFreeAsync(dq, st);
    cudaFreeAsync(dqd, st);
    cudaFreeAsync(dw, st);
    if (r) return r;
    {
        // probes: [k][nq] indices and weights
        std::vector<uint32_t> ti(nq * kk);
        std::vector<float> tw(nq * kk);
        for (int64_t q = 0; q < nq; ++q)
            for (int t = 0; t < kk; ++t) {
                ti[(int64_t)t * nq + q] = hi[q * kk + t];
                tw[(int64_t)t * nq + q] = (float)hw[q * kk + t];
            }
        if ((r = s->alloc(idx_out, nq * kk))) return r;
        if ((r = s->alloc(w_out, nq * kk))) return r;
        NAGA_CUDA_TRY(cudaMemcpyAsync(*idx_out, ti.data(), sizeof(uint32_t) * nq * kk, cudaMemcpyHostToDevice, st));
        NAGA_CUDA_TRY(cudaMemcpyAsync(*w_out, tw.data(), sizeof(float) * nq * kk, cudaMemcpyHostToDevice, st));
        NAGA_CUDA_TRY(cudaStreamSynchronize(st));
    }
    return NAGA_OK;
}

int scene_setup(naga_scene* s) {
    const naga_scene_desc& d = s->desc;
    const int D = s->dim, QP = s->QP;
    const int64_t N = s->N;
    cudaStream_t st = s->stream;
    SceneDev& V = s->dev;
    V.N = N;
    V.nb = s->nb;
    V.nl = s->nl;
    V.nbd = s->nbd;
    V.ng = s->ng;
    V.nbl = s->nbl;
    V.k = d.k;
    V.kb = d.k_boundary;
    V.kp = d.k_probe;
    V.np = d.n_probes;
    V.pml_shift = d.pml_indexing == 0 ? (int)s->nb : 0;
    V.probe_cap = std::max(1, d.probe_capacity);
    set_parameters(s);

    float* pts = nullptr;
    int rc;
    if ((rc = s->alloc(&pts, N * D))) return rc;
    s->d_pts = pts;
    NAGA_CUDA_TRY(cudaMemcpyAsync(pts, d.points, sizeof(float) * N * D, cudaMemcpyHostToDevice, st));
    NAGA_CUDA_TRY(cudaStreamSynchronize(st));
    float* nrm = nullptr;
    float* sig = nullptr;
    if ((rc = s->alloc(&nrm, s->nbd * D))) return rc;
    if ((rc = s->alloc(&sig, s->nl))) return rc;
    if (s->nbd) NAGA_CUDA_TRY(cudaMemcpyAsync(nrm, d.normals, sizeof(float) * s->nbd * D, cudaMemcpyHostToDevice, st));
    if (s->nl) NAGA_CUDA_TRY(cudaMemcpyAsync(sig, d.sigma, sizeof(float) * s->nl, cudaMemcpyHostToDevice, st));
    V.normals = nrm;
    V.sigma = sig;

    // state buffers
    // (the RK stage buffers G1, G2 hold rows of the gathered chunks only)
    const int QS = D == 2 ? D2Q9::QS : D3Q27::QS;
    float* bufs[7];
    for (int b = 0; b < 7; ++b) {
        const int64_t row = (b == 1 || b == 2) ? QS : QP;
        if ((rc = s->alloc(&bufs[b], N * row))) return rc;
        NAGA_CUDA_TRY(cudaMemsetAsync(bufs[b], 0, sizeof(float) * N * row, st));
    }
    V.G = bufs[0];
    V.G1 = bufs[1];
    V.G2 = bufs[2];
    V.S1 = bufs[3];
    V.S1P = bufs[4];
    V.Q1a = bufs[5];
    V.Q1b = bufs[6];
    float4* M = nullptr;
    if ((rc = s->alloc(&M, N))) return rc;
    NAGA_CUDA_TRY(cudaMemsetAsync(M, 0, sizeof(float4) * N, st));
    V.M = M;

    // divergence stencil + filter weights over the domain [0, nd)
    const int k = d.k;
    const int npb = nodes_per_pass(D);
    StencilOut out{};
    out.filter_sigma = d.nodal_spacing / 2.5;
    out.split = s->nbl;
    out.n_total = N;
    out.npb = npb;
    uint32_t* knn_idx = nullptr;
    if ((rc = s->alloc(&knn_idx, s->nd * k))) return rc;
    float4* W = nullptr;
    if ((rc = s->alloc(&W, (int64_t)k * N))) return rc;
    NAGA_CUDA_TRY(cudaMemsetAsync(W, 0, sizeof(float4) * k * N, st));
    out.Wf = W;
    V.stW = W;
    V.stF = nullptr;
    {
        // (weight, index) records of the selective filter, pass order
        float2* F = nullptr;
        if ((rc = s->alloc(&F, (int64_t)k * N))) return rc;
        NAGA_CUDA_TRY(cudaMemsetAsync(F, 0, sizeof(float2) * k * N, st));
        out.Ff = F;
        V.stF = F;
    }
    rc = divergence_build_device(pts, s->nd, D, k, d.shape, d.weight_precision, knn_idx, out, st);
    if (rc) return rc;
    // PML: field rows of the layer nodes and the per-node mean vectors
    float* phi = nullptr;
    float4* pv = nullptr;
    if (s->nl > 0) {
        if ((rc = s->alloc(&phi, s->nl * QS))) return rc;
        NAGA_CUDA_TRY(cudaMemsetAsync(phi, 0, sizeof(float) * s->nl * QS, st));
    }
    if ((rc = s->alloc(&pv, 2 * std::max<int64_t>(s->nbl, 1)))) return rc;
    NAGA_CUDA_TRY(cudaMemsetAsync(pv, 0, sizeof(float4) * 2 * std::max<int64_t>(s->nbl, 1), st));
    if (s->nl > 0 && (rc = pml_vectors_device(D, W, V.sigma, s->nb, s->nl, s->nbl, N, k, pv, st))) return rc;
    float4* stp = nullptr;
    if (s->nl > 0) {
        if ((rc = s->alloc(&stp, (int64_t)k * s->nbl))) return rc;
        if ((rc = pml_table_device(D, W, s->nb, s->nl, s->nbl, N, k, stp, st))) return rc;
    }
    V.PHI = phi;
    V.PV = pv;
    V.stP = stp;
    float* str = nullptr;
    if (D == 2) {
        if ((rc = s->alloc(&str, 3 * (int64_t)k * N))) return rc;
        if ((rc = compact_records_device(W, (int64_t)k * N, str, st))) return rc;
    }
    V.stR = str;
    // halo blobs of the D3Q27 RK stages (one per bulk/layer pass)
    float4* sth = nullptr;
    if (D == 3 && k == kHaloK && npb == 32 && s->nbl > 0) {
        const int64_t n_pass = (s->nbl + npb - 1) / npb;
        if ((rc = s->alloc(&sth, n_pass * (kHaloBlobBytes / 16)))) return rc;
        if ((rc = halo_build_device(W, s->nbl, k, npb, sth, st))) return rc;
    }
    V.stH = sth;

    // boundary interpolation: kNN among bulk + layer, RPIM at the boundary
    // node with the nodal spacing (detail/simulation_engine.cuh:223-258)
    uint8_t* dsrc = nullptr;
    if ((rc = s->alloc(&dsrc, N))) return rc;
    NAGA_CUDA_TRY(cudaMemsetAsync(dsrc, 0, N, st));
    auto rpim = [&](const float* qry_host, int64_t nq, int64_t nsrc, int kk, uint32_t** idx_out, float** w_out,
                    float2** rec_out) -> int {
        return rpim_tables(s, pts, qry_host, nq, nsrc, kk, idx_out, w_out, rec_out, dsrc);
    };
    float2* btab = nullptr;
    if (s->nbd > 0) {
        if ((rc = rpim(d.points + s->nbl * D, s->nbd, s->nbl, d.k_boundary, nullptr, nullptr, &btab))) return rc;
    }
    V.btab = btab;
    uint32_t* pidx = nullptr;
    float* pw = nullptr;
    if (d.n_probes > 0) {
        // probes: kNN among all points (density_observer.cuh:62-97)
        if ((rc = rpim(d.probes, d.n_probes, N, d.k_probe, &pidx, &pw, nullptr))) return rc;
    }
    V.pidx = pidx;
    V.pw = pw;
    V.is_src = dsrc;

    float* ring = nullptr;
    if ((rc = s->alloc(&ring, (int64_t)V.probe_cap * std::max(1, d.n_probes)))) return rc;
    NAGA_CUDA_TRY(cudaMemsetAsync(ring, 0, sizeof(float) * V.probe_cap * std::max(1, d.n_probes), st));
    V.probe_ring = ring;

    make_items(0, N, s->items_all);
    // pass-sized items follow the pass order of the tables: [0, nbl), [nbl, N)
    make_items(0, s->nbl, s->items_all_mt, npb);
    {
        std::vector<WorkItem> rest;
        make_items(s->nbl, N, rest, npb);
        for (WorkItem it : rest) {
            it.local = (uint32_t)s->items_all_mt.size();
            s->items_all_mt.push_back(it);
        }
    }
    make_items(0, s->nbl, s->items_fluid, npb);
    make_items(s->nbl, s->nbl + s->nbd, s->items_edge, npb);
    // bulk/layer items with at least one stencil support in the layer
    s->items_pml.clear();
    if (s->nl > 0 && !s->items_fluid.empty()) {
        const int nf = (int)s->items_fluid.size();
        WorkItem* ditems = nullptr;
        uint8_t* dflag = nullptr;
        NAGA_CUDA_TRY(cudaMallocAsync(&ditems, sizeof(WorkItem) * nf, st));
        NAGA_CUDA_TRY(cudaMallocAsync(&dflag, nf, st));
        std::vector<uint8_t> flag(nf, 0);
        cudaError_t e = cudaMemcpyAsync(ditems, s->items_fluid.data(), sizeof(WorkItem) * nf, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) {
            layer_touch_kernel<<<nf, 256, 0, st>>>(knn_idx, k, ditems, nf, s->nb, s->nl, dflag);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(flag.data(), dflag, nf, cudaMemcpyDeviceToHost, st);
        cudaFreeAsync(ditems, st);
        cudaFreeAsync(dflag, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return set_error(NAGA_ECUDA, std::string("layer items: ") + cudaGetErrorString(e));
        for (int w = 0; w < nf; ++w)
            if (flag[w]) s->items_pml.push_back(s->items_fluid[w]);
        // each PML item carries its nodes' largest layer-support count in
        // `local` (its tile is that many records per node)
        const int np = (int)s->items_pml.size();
        if (np > 0) {
            WorkItem* dpi = nullptr;
            uint32_t* dk = nullptr;
            std::vector<uint32_t> km(np, 0);
            e = cudaMallocAsync(&dpi, sizeof(WorkItem) * np, st);
            if (e == cudaSuccess) e = cudaMallocAsync(&dk, sizeof(uint32_t) * np, st);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(dpi, s->items_pml.data(), sizeof(WorkItem) * np, cudaMemcpyHostToDevice, st);
            if (e == cudaSuccess) {
                pml_item_kmax_kernel<<<(np + 255) / 256, 256, 0, st>>>(dpi, np, pv, dk);
                e = cudaGetLastError();
            }
            if (e == cudaSuccess) e = cudaMemcpyAsync(km.data(), dk, sizeof(uint32_t) * np, cudaMemcpyDeviceToHost, st);
            if (dpi) cudaFreeAsync(dpi, st);
            if (dk) cudaFreeAsync(dk, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) return set_error(NAGA_ECUDA, std::string("PML items: ") + cudaGetErrorString(e));
            for (int w = 0; w < np; ++w) s->items_pml[w].local = std::min<uint32_t>(km[w], (uint32_t)k);
        }
    }
    V.n_all_items = (int)s->items_all.size();
    {
        const std::vector<WorkItem>* lists[5] = {&s->items_all, &s->items_all_mt, &s->items_fluid, &s->items_edge,
                                                 &s->items_pml};
        std::vector<WorkItem> packed;
        for (int l = 0; l < 5; ++l) {
            s->n_list[l] = (int64_t)lists[l]->size();
            packed.insert(packed.end(), lists[l]->begin(), lists[l]->end());
        }
        if ((rc = s->alloc(&s->d_lists, (int64_t)packed.size()))) return rc;
        if (!packed.empty())
            NAGA_CUDA_TRY(cudaMemcpyAsync(s->d_lists, packed.data(), sizeof(WorkItem) * packed.size(),
                                          cudaMemcpyHostToDevice, st));
        NAGA_CUDA_TRY(cudaStreamSynchronize(st));
    }
    double* partials = nullptr;
    if ((rc = s->alloc(&partials, (int64_t)V.n_all_items * 2 * QP))) return rc;
    NAGA_CUDA_TRY(cudaMemsetAsync(partials, 0, sizeof(double) * V.n_all_items * 2 * QP, st));
    V.partials = partials;
    float* means = nullptr;
    if ((rc = s->alloc(&means, 2 * QP))) return rc;
    NAGA_CUDA_TRY(cudaMemsetAsync(means, 0, sizeof(float) * 2 * QP, st));
    V.means = means;
    unsigned long long* step = nullptr;
    if ((rc = s->alloc(&step, 1))) return rc;
    NAGA_CUDA_TRY(cudaMemsetAsync(step, 0, sizeof(unsigned long long), st));
    V.step = step;
    NAGA_CUDA_TRY(cudaStreamSynchronize(st));
    return NAGA_OK;
}

int batch_rebuild(naga_batch* b) {
    b->free_graph();
    const int ns = (int)b->members.size();
    b->k = ns == 0 ? 0 : b->members[0]->desc.k;
    b->kb = ns == 0 ? 0 : b->members[0]->desc.k_boundary;
    int64_t n[5] = {}, base[6] = {};
    for (naga_scene* s : b->members) {
        if (s->desc.k != b->k) b->k = 0;
        if (s->desc.k_boundary != b->kb) b->kb = 0;
        for (int l = 0; l < 5; ++l) n[l] += s->n_list[l];
    }
    for (int l = 0; l < 5; ++l) base[l + 1] = base[l] + n[l];
    for (int l = 0; l < 5; ++l)
        if (n[l] > 0x7fffffff) return set_error(NAGA_EINVAL, "batch: more than 2^31 - 1 work items in one list");
    // grow the device tables (cudaFree waits for the device, so only here)
    auto grow = [&](auto** p, auto& cap, int64_t need) -> int {
        if (need <= (int64_t)cap && *p) return NAGA_OK;
        if (*p) cudaFree(*p);
        *p = nullptr;
        const int64_t c = std::max<int64_t>(need + need / 4, 16);
        using T = typename std::remove_pointer<typename std::remove_reference<decltype(*p)>::type>::type;
        cudaError_t e = cudaMalloc((void**)p, sizeof(T) * (size_t)c);
        if (e != cudaSuccess) {
            cudaGetLastError();
            cap = 0;
            return set_error(e == cudaErrorMemoryAllocation ? NAGA_ENOMEM : NAGA_ECUDA,
                             std::string("batch tables: ") + cudaGetErrorString(e));
        }
        cap = (std::remove_reference_t<decltype(cap)>)c;
        return NAGA_OK;
    };
    std::vector<ListCopy> copies;
    int64_t dst[5];
    for (int l = 0; l < 5; ++l) dst[l] = base[l];
    for (int t = 0; t < ns; ++t) {
        naga_scene* s = b->members[t];
        int64_t at = 0;
        for (int l = 0; l < 5; ++l) {
            if (s->n_list[l] > 0) copies.push_back({s->d_lists + at, dst[l], (uint32_t)s->n_list[l], (uint32_t)t});
            at += s->n_list[l];
            dst[l] += s->n_list[l];
        }
    }
    int rc;
    if ((rc = grow(&b->d_items, b->items_cap, std::max<int64_t>(base[5], 1)))) return rc;
    if ((rc = grow(&b->d_scenes, b->scenes_cap, std::max(ns, 1)))) return rc;
    if ((rc = grow(&b->d_copies, b->copies_cap, std::max<int64_t>((int64_t)copies.size(), 1)))) return rc;
    const size_t sb = sizeof(SceneDev) * ns, cb = sizeof(ListCopy) * copies.size();
    if (sb + cb > b->stage_cap) {
        if (b->h_stage) cudaFreeHost(b->h_stage);
        b->h_stage = nullptr;
        b->stage_cap = 0;
        NAGA_CUDA_TRY(cudaMallocHost(&b->h_stage, (sb + cb) * 5 / 4 + 256));
        b->stage_cap = (sb + cb) * 5 / 4 + 256;
    }
    char* stage = (char*)b->h_stage;
    for (int t = 0; t < ns; ++t) std::memcpy(stage + sizeof(SceneDev) * t, &b->members[t]->dev, sizeof(SceneDev));
    if (cb) std::memcpy(stage + sb, copies.data(), cb);
    if (sb) NAGA_CUDA_TRY(cudaMemcpyAsync(b->d_scenes, stage, sb, cudaMemcpyHostToDevice, b->stream));
    if (cb) NAGA_CUDA_TRY(cudaMemcpyAsync(b->d_copies, stage + sb, cb, cudaMemcpyHostToDevice, b->stream));
    uint32_t most = 1;
    for (const ListCopy& c : copies) most = std::max(most, c.n);
    const unsigned gx = (unsigned)std::min<uint32_t>((most + 255) / 256, 256);
    for (size_t c0 = 0; c0 < copies.size(); c0 += 65535) {
        const unsigned gy = (unsigned)std::min<size_t>(copies.size() - c0, 65535);
        concat_items_kernel<<<dim3(gx, gy), 256, 0, b->stream>>>(b->d_copies + c0, b->d_items);
        NAGA_CUDA_TRY(cudaGetLastError());
    }
    // the staging buffer is reused by the next rebuild
    NAGA_CUDA_TRY(cudaStreamSynchronize(b->stream));
    b->d_all = b->d_items + base[0];
    b->d_all_mt = b->d_items + base[1];
    b->d_fluid = b->d_items + base[2];
    b->d_edge = b->d_items + base[3];
    b->d_pml = b->d_items + base[4];
    b->n_all = (int)n[0];
    b->n_all_mt = (int)n[1];
    b->n_fluid = (int)n[2];
    b->n_edge = (int)n[3];
    b->n_pml = (int)n[4];
    b->dirty = false;
    return NAGA_OK;
}

StepLaunch launch_of(naga_batch* b) {
    StepLaunch P;
    P.scenes = b->d_scenes;
    P.nscenes = (int)b->members.size();
    P.all = b->d_all;
    P.n_all = b->n_all;
    P.all_mt = b->d_all_mt;
    P.n_all_mt = b->n_all_mt;
    P.fluid = b->d_fluid;
    P.n_fluid = b->n_fluid;
    P.edge = b->d_edge;
    P.n_edge = b->n_edge;
    P.pml = b->d_pml;
    P.n_pml = b->n_pml;
    return P;
}

// rebuilds the batch's item lists after a membership change, tunes the
// launch shape of a new batch shape and captures the step graph, so that
// the next batch_step only launches
int batch_prepare(naga_batch* b) {
    if (b->members.empty()) return NAGA_OK;
    int rc;
    if (b->dirty && (rc = batch_rebuild(b))) return rc;
    StepLaunch P = launch_of(b);
    if (!b->exec && (rc = tune_step_shapes(b->dim, b->k, b->kb, P, b->stream))) return rc;
    if (!b->exec && !prof_on()) {
        NAGA_CUDA_TRY(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        rc = enqueue_step(b->dim, b->k, b->kb, P, b->stream);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(b->stream, &g);
        if (rc) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (e != cudaSuccess) return set_error(NAGA_ECUDA, std::string("graph capture: ") + cudaGetErrorString(e));
        b->graph = g;
        NAGA_CUDA_TRY(cudaGraphInstantiate(&b->exec, g, 0));
    }
    return NAGA_OK;
}

int batch_step(naga_batch* b, int nsteps) {
    if (nsteps < 0) return set_error(NAGA_EINVAL, "step: negative step count");
    if (b->members.empty() || nsteps == 0) return NAGA_OK;
    int rc;
    if ((rc = batch_prepare(b))) return rc;
    StepLaunch P = launch_of(b);
    if (prof_on()) {
        for (int n = 0; n < nsteps; ++n)
            if ((rc = enqueue_step(b->dim, b->k, b->kb, P, b->stream))) return rc;
    } else {
        for (int n = 0; n < nsteps; ++n) NAGA_CUDA_TRY(cudaGraphLaunch(b->exec, b->stream));
    }
    for (auto* s : b->members) s->steps += nsteps;
    return NAGA_OK;
}

}  // namespace

// ================================================================== C ABI
extern "C" int naga_scene_create(const naga_scene_desc* d, naga_scene** out) {
    if (!d || !out) return set_error(NAGA_EINVAL, "naga_scene_create: null argument");
    *out = nullptr;
    if (d->dim != 2 && d->dim != 3) return set_error(NAGA_EINVAL, "naga_scene_create: dim must be 2 or 3");
    if (d->n_bulk < 0 || d->n_layer < 0 || d->n_boundary < 0 || d->n_ghost < 0)
        return set_error(NAGA_EINVAL, "naga_scene_create: negative node count");
    const int64_t N = d->n_bulk + d->n_layer + d->n_boundary + d->n_ghost;
    const int nsys_k = d->k + d->dim + 1, nsys_b = d->k_boundary + d->dim + 1, nsys_p = d->k_probe + d->dim + 1;
    if (d->k < d->dim + 2 || nsys_k > 64 || d->k_boundary < d->dim + 1 || nsys_b > 64 || d->k_probe < d->dim + 1 ||
        nsys_p > 64)
        return set_error(NAGA_EINVAL, "naga_scene_create: stencil sizes must satisfy dim + 2 <= k <= 64 - dim - 1");
    if (N - d->n_ghost < d->k || d->n_bulk + d->n_layer < d->k_boundary || N < d->k_probe)
        return set_error(NAGA_EINVAL, "naga_scene_create: fewer nodes than the stencil size");
    if (N > (int64_t)0x7fffffff) return set_error(NAGA_EINVAL, "naga_scene_create: more than 2^31 - 1 nodes");
    if (!d->points || (d->n_boundary > 0 && !d->normals) || (d->n_layer > 0 && !d->sigma) ||
        (d->n_probes > 0 && !d->probes) || d->n_probes < 0)
        return set_error(NAGA_EINVAL, "naga_scene_create: missing input array");
    {
        // non-finite inputs would reach the kNN as coordinates or as queries
        auto finite = [](const float* v, int64_t m) {
            for (int64_t t = 0; t < m; ++t)
                if (!std::isfinite(v[t])) return false;
            return true;
        };
        if (!finite(d->points, N * d->dim) || (d->n_boundary > 0 && !finite(d->normals, d->n_boundary * d->dim)) ||
            (d->n_layer > 0 && !finite(d->sigma, d->n_layer)) ||
            (d->n_probes > 0 && !finite(d->probes, (int64_t)d->n_probes * d->dim)))
            return set_error(NAGA_EINVAL,
                             "naga_scene_create: non-finite point coordinates, normals, absorption or probe positions");
    }
    if (!(d->nodal_spacing > 0) || !(d->time_step > 0) || !(d->speed_of_sound > 0) || !(d->rho0 > 0) ||
        !(d->viscosity >= 0))
        return set_error(NAGA_EINVAL, "naga_scene_create: physical parameters must be positive");
    if (d->shape != 0 && d->shape != 1) return set_error(NAGA_EINVAL, "naga_scene_create: unknown RBF shape");
    if (d->pml_indexing != 0 && d->pml_indexing != 1)
        return set_error(NAGA_EINVAL, "naga_scene_create: pml_indexing must be 0 or 1");
    if (d->weight_precision != 0 && d->weight_precision != 1)
        return set_error(NAGA_EINVAL, "naga_scene_create: weight_precision must be 0 or 1");
    int rc;
    if ((rc = check_device())) return rc;
    auto s = std::make_unique<naga_scene>();
    s->dim = d->dim;
    s->Q = d->dim == 2 ? D2Q9::Q : D3Q27::Q;
    s->QP = d->dim == 2 ? D2Q9::QP : D3Q27::QP;
    s->desc = *d;
    s->N = N;
    s->nb = d->n_bulk;
    s->nl = d->n_layer;
    s->nbd = d->n_boundary;
    s->ng = d->n_ghost;
    s->nbl = s->nb + s->nl;
    s->nd = N - s->ng;
    s->desc.points = nullptr;
    s->desc.normals = nullptr;
    s->desc.sigma = nullptr;
    s->desc.probes = nullptr;
    if (d->n_probes > 0) s->probe_xyz.assign(d->probes, d->probes + (size_t)d->n_probes * d->dim);
    NAGA_CUDA_TRY(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    naga_scene_desc full = *d;
    s->desc = full;
    rc = scene_setup(s.get());
    s->desc.points = s->desc.normals = s->desc.sigma = s->desc.probes = nullptr;
    if (rc) {
        naga_scene_destroy(s.release());
        return rc;
    }
    *out = s.release();
    return NAGA_OK;
}

extern "C" int naga_scene_destroy(naga_scene* s) {
    if (!s) return NAGA_OK;
    if (s->owner) naga_batch_remove(s->owner, s);
    if (s->solo) naga_batch_destroy(s->solo);
    if (s->stream) cudaStreamSynchronize(s->stream);
    for (void* p : s->allocs) cudaFree(p);
    if (s->src_slot) cudaFree(s->src_slot);
    if (s->src_vals) cudaFree(s->src_vals);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return NAGA_OK;
}

extern "C" void* naga_scene_stream(naga_scene* s) { return s ? (void*)active_stream(s) : nullptr; }

extern "C" int naga_scene_set_density(naga_scene* s, const float* drho) {
    if (!s) return set_error(NAGA_EINVAL, "naga_scene_set_density: null scene");
    cudaStream_t st = active_stream(s);
    const int QP = s->QP;
    SceneDev& V = s->dev;
    // upload the N densities into the collision scratch S1 (N QP floats; the
    // next step's node-local kernel rewrites all of it before any read) and
    // expand them to population rows on the device: no allocation, and the
    // work is ordered on the scene's stream behind any steps still queued
    float* d = nullptr;
    if (drho) {
        d = V.S1;
        NAGA_CUDA_TRY(cudaMemcpyAsync(d, drho, sizeof(float) * s->N, cudaMemcpyHostToDevice, st));
    }
    int rc = density_rows_device(s->dim, d, s->N, V.G, st);
    if (rc) return rc;
    NAGA_CUDA_TRY(cudaMemsetAsync(V.M, 0, sizeof(float4) * s->N, st));
    NAGA_CUDA_TRY(cudaMemsetAsync(V.Q1a, 0, sizeof(float) * s->N * QP, st));
    NAGA_CUDA_TRY(cudaMemsetAsync(V.Q1b, 0, sizeof(float) * s->N * QP, st));
    NAGA_CUDA_TRY(cudaMemsetAsync(V.step, 0, sizeof(unsigned long long), st));
    NAGA_CUDA_TRY(cudaMemsetAsync(V.probe_ring, 0, sizeof(float) * V.probe_cap * std::max(1, V.np), st));
    NAGA_CUDA_TRY(cudaStreamSynchronize(st));
    s->steps = 0;
    return NAGA_OK;
}

extern "C" int naga_scene_set_initial_condition(naga_scene* s, const float* drho) {
    return naga_scene_set_density(s, drho);
}

extern "C" int naga_scene_set_params(naga_scene* s, double viscosity, double rho0, double time_step,
                                     double speed_of_sound) {
    if (!s) return set_error(NAGA_EINVAL, "naga_scene_set_params: null scene");
    if (!(viscosity >= 0) || !(rho0 > 0) || !(time_step > 0) || !(speed_of_sound > 0))
        return set_error(NAGA_EINVAL, "naga_scene_set_params: physical parameters must be positive");
    NAGA_CUDA_TRY(cudaStreamSynchronize(active_stream(s)));
    s->desc.viscosity = viscosity;
    s->desc.rho0 = rho0;
    s->desc.time_step = time_step;
    s->desc.speed_of_sound = speed_of_sound;
    set_parameters(s);
    // the batches holding the scene re-upload its parameters before stepping
    if (s->owner) s->owner->dirty = true;
    if (s->solo) s->solo->dirty = true;
    return NAGA_OK;
}

extern "C" int naga_scene_init_domain(naga_scene* s, const naga_scene_desc* d) {
    if (!s || !d) return set_error(NAGA_EINVAL, "naga_scene_init_domain: null argument");
    if (s->owner) return set_error(NAGA_EINVAL, "naga_scene_init_domain: remove the scene from its batch first");
    naga_scene* fresh = nullptr;
    int rc = naga_scene_create(d, &fresh);
    if (rc) return rc;  // the scene keeps its previous domain
    NAGA_CUDA_TRY(cudaStreamSynchronize(active_stream(s)));
    // the handle takes the new scene; the old contents are released
    std::swap(*s, *fresh);
    return naga_scene_destroy(fresh);
}

namespace {
// frees one of the scene's device allocations now
void release(naga_scene* s, void* p) {
    if (!p) return;
    auto it = std::find(s->allocs.begin(), s->allocs.end(), p);
    if (it == s->allocs.end()) return;
    s->allocs.erase(it);
    cudaFree(p);
}
}  // namespace

extern "C" int naga_scene_add_probe(naga_scene* s, const float* xyz, int* index) {
    if (!s || !xyz) return set_error(NAGA_EINVAL, "naga_scene_add_probe: null argument");
    if (!s->d_pts) return set_error(NAGA_EINVAL, "naga_scene_add_probe: scene has no domain");
    for (int d = 0; d < s->dim; ++d)
        if (!std::isfinite(xyz[d])) return set_error(NAGA_EINVAL, "naga_scene_add_probe: non-finite probe position");
    cudaStream_t st = active_stream(s);
    NAGA_CUDA_TRY(cudaStreamSynchronize(st));
    const int D = s->dim;
    const int np_old = s->dev.np, np = np_old + 1;
    s->probe_xyz.insert(s->probe_xyz.end(), xyz, xyz + D);
    uint32_t* pidx = nullptr;
    float* pw = nullptr;
    int rc = rpim_tables(s, s->d_pts, s->probe_xyz.data(), np, s->N, s->desc.k_probe, &pidx, &pw, nullptr, nullptr);
    float* ring = nullptr;
    const int64_t cap = s->dev.probe_cap;
    if (!rc) rc = s->alloc(&ring, cap * np);
    if (rc) {
        s->probe_xyz.resize((size_t)np_old * D);
        release(s, pidx);
        release(s, pw);
        return rc;
    }
    // the ring gains a column: earlier samples of the old probes are kept,
    // the new probe's read as zero before it was added
    NAGA_CUDA_TRY(cudaMemsetAsync(ring, 0, sizeof(float) * cap * np, st));
    if (np_old > 0)
        NAGA_CUDA_TRY(cudaMemcpy2DAsync(ring, sizeof(float) * np, s->dev.probe_ring, sizeof(float) * np_old,
                                        sizeof(float) * np_old, cap, cudaMemcpyDeviceToDevice, st));
    NAGA_CUDA_TRY(cudaStreamSynchronize(st));
    release(s, const_cast<uint32_t*>(s->dev.pidx));
    release(s, const_cast<float*>(s->dev.pw));
    release(s, s->dev.probe_ring);
    s->dev.pidx = pidx;
    s->dev.pw = pw;
    s->dev.probe_ring = ring;
    s->dev.np = np;
    s->desc.n_probes = np;
    if (s->owner) s->owner->dirty = true;
    if (s->solo) s->solo->dirty = true;
    if (index) *index = np - 1;
    return NAGA_OK;
}

extern "C" int naga_scene_step(naga_scene* s, int nsteps) {
    if (!s) return set_error(NAGA_EINVAL, "naga_scene_step: null scene");
    if (s->owner) return set_error(NAGA_EINVAL, "naga_scene_step: scene belongs to a batch; step the batch");
    if (!s->solo) {
        s->solo = new naga_batch();
        s->solo->dim = s->dim;
        s->solo->is_solo = true;
        s->solo->stream = s->stream;
        s->solo->members.push_back(s);
    }
    return batch_step(s->solo, nsteps);
}

extern "C" int naga_scene_sync(naga_scene* s) {
    if (!s) return set_error(NAGA_EINVAL, "naga_scene_sync: null scene");
    NAGA_CUDA_TRY(cudaStreamSynchronize(active_stream(s)));
    return tile_timeout_check(active_stream(s));
}

extern "C" int64_t naga_scene_step_count(const naga_scene* s) { return s ? s->steps : -1; }

extern "C" int naga_scene_read_probes(naga_scene* s, int64_t first, int64_t count, float* out) {
    if (!s || (!out && count > 0)) return set_error(NAGA_EINVAL, "naga_scene_read_probes: null argument");
    const int np = s->dev.np, cap = s->dev.probe_cap;
    if (first < 0 || count < 0 || first + count > s->steps || first < s->steps - cap)
        return set_error(NAGA_EINVAL, "naga_scene_read_probes: requested steps are not in the probe ring");
    if (np == 0 || count == 0) return NAGA_OK;
    // the requested steps occupy at most two runs of the ring
    cudaStream_t st = active_stream(s);
    const int64_t a = first % cap, n1 = std::min<int64_t>(count, cap - a);
    NAGA_CUDA_TRY(cudaMemcpyAsync(out, s->dev.probe_ring + a * np, sizeof(float) * n1 * np, cudaMemcpyDeviceToHost, st));
    if (count > n1)
        NAGA_CUDA_TRY(cudaMemcpyAsync(out + n1 * np, s->dev.probe_ring, sizeof(float) * (count - n1) * np,
                                      cudaMemcpyDeviceToHost, st));
    NAGA_CUDA_TRY(cudaStreamSynchronize(st));
    return NAGA_OK;
}

extern "C" int naga_scene_read_probes_async(naga_scene* s, int64_t first, int64_t count, float* out) {
    if (!s || (!out && count > 0)) return set_error(NAGA_EINVAL, "naga_scene_read_probes_async: null argument");
    const int np = s->dev.np, cap = s->dev.probe_cap;
    if (first < 0 || count < 0 || count > cap || first + count > s->steps || first < s->steps - cap)
        return set_error(NAGA_EINVAL, "naga_scene_read_probes_async: requested steps are not in the probe ring");
    if (np == 0 || count == 0) return NAGA_OK;
    cudaStream_t st = active_stream(s);
    const int64_t a = first % cap, n1 = std::min<int64_t>(count, cap - a);
    NAGA_CUDA_TRY(cudaMemcpyAsync(out, s->dev.probe_ring + a * np, sizeof(float) * n1 * np, cudaMemcpyDeviceToHost, st));
    if (count > n1)
        NAGA_CUDA_TRY(cudaMemcpyAsync(out + n1 * np, s->dev.probe_ring, sizeof(float) * (count - n1) * np,
                                      cudaMemcpyDeviceToHost, st));
    return NAGA_OK;
}

// --------------------------------------------------------- density sources
extern "C" int naga_scene_set_density_source(naga_scene* s, const int64_t* nodes, int64_t n_nodes,
                                             const float* values, int64_t first_step, int64_t n_steps) {
    if (!s) return set_error(NAGA_EINVAL, "naga_scene_set_density_source: null scene");
    if (n_nodes < 0 || n_steps < 0 || first_step < 0 || (n_nodes > 0 && (!nodes || (n_steps > 0 && !values))))
        return set_error(NAGA_EINVAL, "naga_scene_set_density_source: invalid arguments");
    cudaStream_t st = active_stream(s);
    NAGA_CUDA_TRY(cudaStreamSynchronize(st));
    if (n_nodes == 0 || n_steps == 0) {
        if (s->src_slot) cudaFree(s->src_slot);
        if (s->src_vals) cudaFree(s->src_vals);
        s->src_slot = nullptr;
        s->src_vals = nullptr;
        s->src_nodes.clear();
        s->src_vals_cap = 0;
    } else {
        const bool same_nodes = s->src_slot && (int64_t)s->src_nodes.size() == n_nodes &&
                                std::equal(nodes, nodes + n_nodes, s->src_nodes.begin());
        if (!same_nodes) {
            std::vector<int> slot((size_t)s->N, -1);
            for (int64_t t = 0; t < n_nodes; ++t) {
                if (nodes[t] < 0 || nodes[t] >= s->N)
                    return set_error(NAGA_EINVAL, "naga_scene_set_density_source: node index out of range");
                if (slot[nodes[t]] >= 0)
                    return set_error(NAGA_EINVAL, "naga_scene_set_density_source: node listed twice");
                slot[nodes[t]] = (int)t;
            }
            if (!s->src_slot) NAGA_CUDA_TRY(cudaMalloc(&s->src_slot, sizeof(int) * (size_t)s->N));
            NAGA_CUDA_TRY(cudaMemcpyAsync(s->src_slot, slot.data(), sizeof(int) * slot.size(), cudaMemcpyHostToDevice, st));
            s->src_nodes.assign(nodes, nodes + n_nodes);
        }
        const int64_t nv = n_nodes * n_steps;
        if (nv > s->src_vals_cap) {
            if (s->src_vals) cudaFree(s->src_vals);
            s->src_vals = nullptr;
            NAGA_CUDA_TRY(cudaMalloc(&s->src_vals, sizeof(float) * (size_t)nv));
            s->src_vals_cap = nv;
        }
        NAGA_CUDA_TRY(cudaMemcpyAsync(s->src_vals, values, sizeof(float) * (size_t)nv, cudaMemcpyHostToDevice, st));
        NAGA_CUDA_TRY(cudaStreamSynchronize(st));
    }
    const bool on = s->src_slot != nullptr;
    const bool relink = s->dev.src_slot != s->src_slot || s->dev.src_vals != s->src_vals ||
                        s->dev.src_n != (on ? n_nodes : 0) || s->dev.src_first != (on ? first_step : 0) ||
                        s->dev.src_steps != (on ? n_steps : 0);
    s->dev.src_slot = s->src_slot;
    s->dev.src_vals = s->src_vals;
    s->dev.src_n = on ? n_nodes : 0;
    s->dev.src_first = on ? first_step : 0;
    s->dev.src_steps = on ? n_steps : 0;
    // the batches hold device copies of the scene description
    if (relink) {
        if (s->owner) s->owner->dirty = true;
        if (s->solo) s->solo->dirty = true;
    }
    return NAGA_OK;
}

// ------------------------------------------------------------- snapshots
// Dynamic state of a scene, enough to resume stepping bit for bit in a scene
// created from the same description: populations, macros, both PML
// integral buffers, the device step counter (its parity selects the Q1
// buffer), the host step count and the probe ring. Tables are not included:
// they are rebuilt from the description.
namespace {
constexpr int32_t kSnapshotVersion = 2;
struct SnapshotHeader {
    char magic[8];  // "NAGASNP1"
    // 2: D2Q9 rows with the pairs first and the rest population in the
    // third chunk (1 had the rest population first)
    int32_t version, dim, qp, n_probes;
    int64_t n, probe_cap, steps;
    uint64_t device_step;
    int64_t payload;  // bytes after the header
};
int64_t snapshot_payload(const naga_scene* s) {
    const int64_t rows = s->N * s->QP * (int64_t)sizeof(float);
    return 3 * rows + s->N * (int64_t)sizeof(float4) +
           (int64_t)s->dev.probe_cap * std::max(1, s->dev.np) * (int64_t)sizeof(float);
}
}  // namespace

extern "C" int64_t naga_scene_snapshot_bytes(const naga_scene* s) {
    return s ? (int64_t)sizeof(SnapshotHeader) + snapshot_payload(s) : -1;
}

extern "C" int naga_scene_save(naga_scene* s, void* buf, int64_t cap) {
    if (!s || !buf) return set_error(NAGA_EINVAL, "naga_scene_save: null argument");
    const int64_t need = naga_scene_snapshot_bytes(s);
    if (cap < need) return set_error(NAGA_EINVAL, "naga_scene_save: buffer smaller than naga_scene_snapshot_bytes");
    cudaStream_t st = active_stream(s);
    NAGA_CUDA_TRY(cudaStreamSynchronize(st));
    SnapshotHeader h{};
    std::memcpy(h.magic, "NAGASNP1", 8);
    h.version = kSnapshotVersion;
    h.dim = s->dim;
    h.qp = s->QP;
    h.n_probes = s->dev.np;
    h.n = s->N;
    h.probe_cap = s->dev.probe_cap;
    h.steps = s->steps;
    h.payload = snapshot_payload(s);
    NAGA_CUDA_TRY(cudaMemcpyAsync(&h.device_step, s->dev.step, sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
    char* p = static_cast<char*>(buf) + sizeof(SnapshotHeader);
    const size_t rows = sizeof(float) * (size_t)s->N * s->QP;
    NAGA_CUDA_TRY(cudaMemcpyAsync(p, s->dev.G, rows, cudaMemcpyDeviceToHost, st));
    NAGA_CUDA_TRY(cudaMemcpyAsync(p + rows, s->dev.Q1a, rows, cudaMemcpyDeviceToHost, st));
    NAGA_CUDA_TRY(cudaMemcpyAsync(p + 2 * rows, s->dev.Q1b, rows, cudaMemcpyDeviceToHost, st));
    NAGA_CUDA_TRY(cudaMemcpyAsync(p + 3 * rows, s->dev.M, sizeof(float4) * s->N, cudaMemcpyDeviceToHost, st));
    NAGA_CUDA_TRY(cudaMemcpyAsync(p + 3 * rows + sizeof(float4) * s->N, s->dev.probe_ring,
                                  sizeof(float) * (size_t)s->dev.probe_cap * std::max(1, s->dev.np),
                                  cudaMemcpyDeviceToHost, st));
    NAGA_CUDA_TRY(cudaStreamSynchronize(st));
    std::memcpy(buf, &h, sizeof h);
    return NAGA_OK;
}

extern "C" int naga_scene_load(naga_scene* s, const void* buf, int64_t size) {
    if (!s || !buf) return set_error(NAGA_EINVAL, "naga_scene_load: null argument");
    if (size < (int64_t)sizeof(SnapshotHeader)) return set_error(NAGA_EINVAL, "naga_scene_load: truncated snapshot");
    SnapshotHeader h;
    std::memcpy(&h, buf, sizeof h);
    if (std::memcmp(h.magic, "NAGASNP1", 8) != 0 || h.version != kSnapshotVersion)
        return set_error(NAGA_EINVAL, "naga_scene_load: not a snapshot of this format");
    if (h.dim != s->dim || h.qp != s->QP || h.n != s->N || h.n_probes != s->dev.np || h.probe_cap != s->dev.probe_cap ||
        h.payload != snapshot_payload(s))
        return set_error(NAGA_EINVAL, "naga_scene_load: snapshot is of a scene with another shape");
    if (size < (int64_t)sizeof h + h.payload) return set_error(NAGA_EINVAL, "naga_scene_load: truncated snapshot");
    cudaStream_t st = active_stream(s);
    NAGA_CUDA_TRY(cudaStreamSynchronize(st));
    const char* p = static_cast<const char*>(buf) + sizeof h;
    const size_t rows = sizeof(float) * (size_t)s->N * s->QP;
    NAGA_CUDA_TRY(cudaMemcpyAsync(s->dev.G, p, rows, cudaMemcpyHostToDevice, st));
    NAGA_CUDA_TRY(cudaMemcpyAsync(s->dev.Q1a, p + rows, rows, cudaMemcpyHostToDevice, st));
    NAGA_CUDA_TRY(cudaMemcpyAsync(s->dev.Q1b, p + 2 * rows, rows, cudaMemcpyHostToDevice, st));
    NAGA_CUDA_TRY(cudaMemcpyAsync(s->dev.M, p + 3 * rows, sizeof(float4) * s->N, cudaMemcpyHostToDevice, st));
    NAGA_CUDA_TRY(cudaMemcpyAsync(s->dev.probe_ring, p + 3 * rows + sizeof(float4) * s->N,
                                  sizeof(float) * (size_t)s->dev.probe_cap * std::max(1, s->dev.np),
                                  cudaMemcpyHostToDevice, st));
    NAGA_CUDA_TRY(cudaMemcpyAsync(s->dev.step, &h.device_step, sizeof(uint64_t), cudaMemcpyHostToDevice, st));
    NAGA_CUDA_TRY(cudaStreamSynchronize(st));
    s->steps = h.steps;
    return NAGA_OK;
}

extern "C" int naga_scene_read_state(naga_scene* s, float* g, float* drho) {
    if (!s) return set_error(NAGA_EINVAL, "naga_scene_read_state: null scene");
    NAGA_CUDA_TRY(cudaStreamSynchronize(active_stream(s)));
    const int Q = s->Q, QP = s->QP;
    std::vector<float> buf((size_t)s->N * QP);
    NAGA_CUDA_TRY(cudaMemcpy(buf.data(), s->dev.G, sizeof(float) * buf.size(), cudaMemcpyDeviceToHost));
    for (int64_t i = 0; i < s->N; ++i) {
        double r = 0;
        for (int a = 0; a < Q; ++a) {
            float v = buf[(size_t)i * QP + slot_of(s->dim, a)];
            if (g) g[i * Q + a] = v;
            r += v;
        }
        if (drho) drho[i] = (float)(r * s->desc.rho0);
    }
    return NAGA_OK;
}

extern "C" int naga_lattice(int dim, int* q, float* weights, int* velocities) {
    if (dim != 2 && dim != 3) return set_error(NAGA_EINVAL, "naga_lattice: dim must be 2 or 3");
    const int Q = dim == 2 ? D2Q9::Q : D3Q27::Q;
    if (q) *q = Q;
    for (int a = 0; a < Q; ++a) {
        if (weights) weights[a] = dim == 2 ? LatticeTables<D2Q9>::w(a) : LatticeTables<D3Q27>::w(a);
        if (velocities) {
            if (dim == 2) {
                velocities[a * 2] = LatticeTables<D2Q9>::cx(a);
                velocities[a * 2 + 1] = LatticeTables<D2Q9>::cy(a);
            } else {
                velocities[a * 3] = LatticeTables<D3Q27>::cx(a);
                velocities[a * 3 + 1] = LatticeTables<D3Q27>::cy(a);
                velocities[a * 3 + 2] = LatticeTables<D3Q27>::cz(a);
            }
        }
    }
    return NAGA_OK;
}

extern "C" int naga_scene_read_macros(naga_scene* s, float* density, float* velocity) {
    if (!s) return set_error(NAGA_EINVAL, "naga_scene_read_macros: null scene");
    NAGA_CUDA_TRY(cudaStreamSynchronize(active_stream(s)));
    std::vector<float4> m((size_t)s->N);
    NAGA_CUDA_TRY(cudaMemcpy(m.data(), s->dev.M, sizeof(float4) * m.size(), cudaMemcpyDeviceToHost));
    // NAGA stores the macros dimensional: rho rho0 and u c / c_s
    // (detail/simulation_engine.cuh:53-82)
    const double rho0 = s->desc.rho0;
    const double uscale = s->desc.speed_of_sound / (double)lattice_cs_f();
    const int D = s->dim;
    for (int64_t i = 0; i < s->N; ++i) {
        const float4 v = m[(size_t)i];
        if (density) density[i] = (float)((1.0 + (double)v.x) * rho0);
        if (velocity) {
            // the bounce-back of the step resets the boundary nodes' stored
            // velocity to 0 (detail/simulation_engine.cuh:874-877)
            const bool wall = i >= s->nbl && i < s->nbl + s->nbd;
            const float u[3] = {v.y, v.z, v.w};
            for (int d = 0; d < D; ++d) velocity[i * D + d] = wall ? 0.f : (float)((double)u[d] * uscale);
        }
    }
    return NAGA_OK;
}

extern "C" int naga_scene_write_state(naga_scene* s, const float* g) {
    if (!s || !g) return set_error(NAGA_EINVAL, "naga_scene_write_state: null argument");
    NAGA_CUDA_TRY(cudaStreamSynchronize(active_stream(s)));
    const int Q = s->Q, QP = s->QP;
    std::vector<float> buf((size_t)s->N * QP, 0.f);
    for (int64_t i = 0; i < s->N; ++i)
        for (int a = 0; a < Q; ++a) buf[(size_t)i * QP + slot_of(s->dim, a)] = g[i * Q + a];
    cudaStream_t st = active_stream(s);
    NAGA_CUDA_TRY(cudaMemcpyAsync(s->dev.G, buf.data(), sizeof(float) * buf.size(), cudaMemcpyHostToDevice, st));
    NAGA_CUDA_TRY(cudaStreamSynchronize(st));
    return NAGA_OK;
}

extern "C" int naga_scene_read_tables(naga_scene* s, uint32_t* idx, float* W, float* fw, uint32_t* bidx, float* bw,
                                      uint32_t* pidx, float* pw) {
    if (!s) return set_error(NAGA_EINVAL, "naga_scene_read_tables: null scene");
    NAGA_CUDA_TRY(cudaStreamSynchronize(active_stream(s)));
    const int k = s->desc.k, D = s->dim, npb = nodes_per_pass(D);
    const int64_t N = s->N;
    // the device tables are in pass order; the outputs are node-major
    if (idx || W) {
        std::vector<float4> wv((size_t)k * N);
        NAGA_CUDA_TRY(cudaMemcpy(wv.data(), s->dev.stW, sizeof(float4) * wv.size(), cudaMemcpyDeviceToHost));
        for (int64_t i = 0; i < N; ++i)
            for (int t = 0; t < k; ++t) {
                const size_t e = (size_t)i * k + t;
                const float4 r = wv[pass_record(i, t, k, s->nbl, N, npb)];
                if (W) {
                    W[e * D + 0] = r.x;
                    W[e * D + 1] = r.y;
                    if (D == 3) W[e * D + 2] = r.z;
                }
                if (idx) std::memcpy(&idx[e], &r.w, 4);
            }
    }
    if (fw) {
        std::vector<float2> fv((size_t)k * N);
        NAGA_CUDA_TRY(cudaMemcpy(fv.data(), s->dev.stF, sizeof(float2) * fv.size(), cudaMemcpyDeviceToHost));
        for (int64_t i = 0; i < N; ++i)
            for (int t = 0; t < k; ++t) fw[(size_t)i * k + t] = fv[pass_record(i, t, k, s->nbl, N, npb)].x;
    }
    if ((bidx || bw) && s->nbd > 0) {
        const int kb = s->desc.k_boundary;
        const size_t n = (size_t)s->nbd * kb;
        std::vector<float2> bv(n);
        NAGA_CUDA_TRY(cudaMemcpy(bv.data(), s->dev.btab, sizeof(float2) * n, cudaMemcpyDeviceToHost));
        for (int64_t q = 0; q < s->nbd; ++q)
            for (int t = 0; t < kb; ++t) {
                const size_t e = (size_t)q * kb + t;
                const float2 r = bv[pass_record(q, t, kb, s->nbd, s->nbd, npb)];
                if (bw) bw[e] = r.x;
                if (bidx) std::memcpy(&bidx[e], &r.y, 4);
            }
    }
    auto tr = [&](const void* dsrc_i, const float* dsrc_w, int64_t nq, int kk, uint32_t* oi, float* ow) -> int {
        if (nq == 0) return NAGA_OK;
        std::vector<uint32_t> ti((size_t)nq * kk);
        std::vector<float> tw((size_t)nq * kk);
        NAGA_CUDA_TRY(cudaMemcpy(ti.data(), dsrc_i, sizeof(uint32_t) * ti.size(), cudaMemcpyDeviceToHost));
        NAGA_CUDA_TRY(cudaMemcpy(tw.data(), dsrc_w, sizeof(float) * tw.size(), cudaMemcpyDeviceToHost));
        for (int64_t q = 0; q < nq; ++q)
            for (int t = 0; t < kk; ++t) {
                if (oi) oi[q * kk + t] = ti[(size_t)t * nq + q];
                if (ow) ow[q * kk + t] = tw[(size_t)t * nq + q];
            }
        return NAGA_OK;
    };
    int rc;
    if ((pidx || pw) && (rc = tr(s->dev.pidx, s->dev.pw, s->dev.np, s->desc.k_probe, pidx, pw))) return rc;
    return NAGA_OK;
}

extern "C" int64_t naga_scene_device_bytes(const naga_scene* s) { return s ? s->bytes : 0; }

extern "C" int naga_scene_size(const naga_scene* s, int64_t* n, int* q) {
    if (!s) return set_error(NAGA_EINVAL, "naga_scene_size: null scene");
    if (n) *n = s->N;
    if (q) *q = s->Q;
    return NAGA_OK;
}

// --------------------------------------------------------------- batches
extern "C" int naga_batch_create_with_priority(int dim, int priority, naga_batch** out) {
    if (!out || (dim != 2 && dim != 3) || (priority != 0 && priority != 1))
        return set_error(NAGA_EINVAL, "naga_batch_create: bad argument");
    int rc;
    if ((rc = check_device())) return rc;
    auto b = new naga_batch();
    b->dim = dim;
    int lo = 0, hi = 0;
    cudaDeviceGetStreamPriorityRange(&lo, &hi);
    cudaError_t e = cudaStreamCreateWithPriority(&b->stream, cudaStreamNonBlocking, priority ? hi : lo);
    if (e != cudaSuccess) {
        delete b;
        return set_error(NAGA_ECUDA, std::string("naga_batch_create: ") + cudaGetErrorString(e));
    }
    *out = b;
    return NAGA_OK;
}

extern "C" int naga_batch_create(int dim, naga_batch** out) { return naga_batch_create_with_priority(dim, 0, out); }

extern "C" int naga_batch_destroy(naga_batch* b) {
    if (!b) return NAGA_OK;
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (!b->is_solo)
        for (auto* s : b->members) s->owner = nullptr;
    b->free_tables();
    if (b->stream && !b->is_solo) cudaStreamDestroy(b->stream);
    delete b;
    return NAGA_OK;
}

extern "C" int naga_batch_add(naga_batch* b, naga_scene* s) {
    if (!b || !s) return set_error(NAGA_EINVAL, "naga_batch_add: null argument");
    if (b->is_solo) return set_error(NAGA_EINVAL, "naga_batch_add: not a user batch");
    if (s->dim != b->dim) return set_error(NAGA_EINVAL, "naga_batch_add: lattice of the scene differs from the batch");
    if (s->owner) return set_error(NAGA_EINVAL, "naga_batch_add: scene already belongs to a batch");
    NAGA_CUDA_TRY(cudaStreamSynchronize(s->stream));
    NAGA_CUDA_TRY(cudaStreamSynchronize(b->stream));
    s->owner = b;
    b->members.push_back(s);
    b->dirty = true;
    return NAGA_OK;
}

extern "C" int naga_batch_remove(naga_batch* b, naga_scene* s) {
    if (!b || !s) return set_error(NAGA_EINVAL, "naga_batch_remove: null argument");
    auto it = std::find(b->members.begin(), b->members.end(), s);
    if (it == b->members.end()) return set_error(NAGA_EINVAL, "naga_batch_remove: scene is not a member");
    NAGA_CUDA_TRY(cudaStreamSynchronize(b->stream));
    b->members.erase(it);
    s->owner = nullptr;
    b->dirty = true;
    return NAGA_OK;
}

extern "C" int naga_batch_size(const naga_batch* b) { return b ? (int)b->members.size() : 0; }
extern "C" void* naga_batch_stream(naga_batch* b) { return b ? (void*)b->stream : nullptr; }

extern "C" int naga_batch_prepare(naga_batch* b) {
    if (!b) return set_error(NAGA_EINVAL, "naga_batch_prepare: null batch");
    return batch_prepare(b);
}

extern "C" int naga_batch_step(naga_batch* b, int nsteps) {
    if (!b) return set_error(NAGA_EINVAL, "naga_batch_step: null batch");
    return batch_step(b, nsteps);
}

extern "C" int naga_batch_sync(naga_batch* b) {
    if (!b) return set_error(NAGA_EINVAL, "naga_batch_sync: null batch");
    NAGA_CUDA_TRY(cudaStreamSynchronize(b->stream));
    return tile_timeout_check(b->stream);
}

extern "C" int64_t naga_tuning_report(char* buf, int64_t cap) {
    const std::string r = tuning_report();
    if (buf && cap > 0) {
        const int64_t n = std::min<int64_t>(cap - 1, (int64_t)r.size());
        std::memcpy(buf, r.data(), (size_t)n);
        buf[n] = 0;
    }
    return (int64_t)r.size();
}

extern "C" int naga_selftest_wait_timeout(int polls) {
    int rc;
    if ((rc = check_device())) return rc;
    return wait_selftest(polls, 0);
}

// --------------------------------------------------------------- profiling
extern "C" int naga_profile_enable(int on) {
    std::lock_guard<std::mutex> lk(g_prof.mu);
    prof_drain();
    g_prof.on = on != 0;
    return NAGA_OK;
}

extern "C" int naga_profile_reset(void) {
    std::lock_guard<std::mutex> lk(g_prof.mu);
    prof_drain();
    g_prof.ms.assign(g_prof.ms.size(), 0.0);
    g_prof.launches.assign(g_prof.launches.size(), 0);
    return NAGA_OK;
}

extern "C" int naga_profile_read(int* count, const char** names, int64_t* launches, double* ms) {
    if (!count) return set_error(NAGA_EINVAL, "naga_profile_read: null count");
    std::lock_guard<std::mutex> lk(g_prof.mu);
    prof_drain();
    const int n = std::min(*count, kernel_count());
    for (int i = 0; i < n; ++i) {
        if (names) names[i] = kernel_name(i);
        if (launches) launches[i] = i < (int)g_prof.launches.size() ? g_prof.launches[i] : 0;
        if (ms) ms[i] = i < (int)g_prof.ms.size() ? g_prof.ms[i] : 0.0;
    }
    *count = kernel_count();
    return NAGA_OK;
}
