// Device-resident description of one scene, as the step kernels see it.
//
// HBM layout of a scene with N nodes (order: bulk [0, nb), layer
// [nb, nb + nl), boundary [nbl, nbl + nbd), ghost [.., N)):
//   populations   centred g = f - w, populations in paired slot order
//                 (common.cuh). G: node-major rows of QP floats (QP = 28
//                 for D3Q27, 12 for D2Q9); RK stage buffers G1, G2: rows of
//                 the gathered chunks (QS floats: 28, 8); collision scratch
//                 S1, S1P: D3Q27 rows of QP floats, D2Q9 rows of the 8
//                 moving populations followed by the N rest populations
//                 (s1_ld in step.cu)
//   Q1a, Q1b      PML trapezoid integrals, rows of QP floats, ping-pong
//                 by step parity
//   PHI           rows of the layer nodes' PML field -2 sigma Q1 + sigma^2 Q2
//   PV            per bulk/layer node: sum_s W_s sigma_j and sum_s W_s
//                 sigma_j^2 over its layer supports (two float4)
//   M             float4 per node: (rho - 1, ux, uy, uz) in lattice units
//   stencil       [N][k] float4 records in pass order (below): D3Q27 (Wx,
//                 Wy, Wz, index bits); D2Q9 (Wx, Wy, filter weight, index
//                 bits)
//   filter        D3Q27: [N][k] float2 (weight, index bits), pass order
//   boundary      [nbd][kb] float2 (weight, index bits), pass order;
//                 probes [kp][np] indices + weights
// Pass order: the nodes are cut into passes of npb consecutive nodes
// (npb = nodes_per_pass), separately over [0, nbl) and [nbl, N) (boundary
// tables: over [0, nbd)). A pass's records form one contiguous block (one
// bulk copy into shared memory) and are neighbour-major inside it: record
// (node b + r, neighbour s) of the pass [b, b + nn) sits at b k + s nn + r,
// so the nodes a warp gathers for read consecutive records of the tile.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

namespace naga {

struct SceneDev {
    int64_t N, nb, nl, nbd, ng, nbl;
    int k, kb, kp, np;
    int pml_shift;  // index offset of the layer's Q reads (n_bulk as NAGA, or 0)
    int probe_cap;
    int n_all_items;
    int _pad0;
    // lattice-unit parameters, FP32 as the reference computes them
    float dt_lat;     // lattice time step
    float om_ab;      // viscosity-dependent relaxation rate
    float om_fix[6];  // D3Q27 fixed higher-order rates (1.5, 1.83, 1.4, 1.61, 1.98, 1.74)
    float inv_dt;     // 1 / dt_lat
    float rho0;
    float rk_a[4];                 // Horner RK4 stage factors dt/4, dt/3, dt/2, dt
    float half_dt;                 // dt_lat / 2 of the PML trapezoid rule
    float _pad1;
    // state
    float* G;
    float* G1;
    float* G2;
    float* S1;
    float* S1P;
    float* Q1a;
    float* Q1b;
    float* PHI;  // [nl][QP] PML field -2 sigma Q1 + sigma^2 Q2 of each layer node
    float4* M;
    // tables
    const float4* stW;
    const float4* stH;  // D3Q27, k = kHaloK: halo blobs of the bulk/layer passes (below), else null
    const float4* stP;  // PML gather records, pass order (Wx, Wy, Wz or 0, PHI row bits)
    const float* stR;   // D2Q9: the stencil records compacted to (Wx, Wy, index bits), pass order
    const float4* PV;  // [nbl][2]: (V1, V2) = sum over layer supports of W_s sigma_j, W_s sigma_j^2
    const float2* stF;
    const float* sigma;
    const float* normals;
    const float2* btab;
    const uint32_t* pidx;
    const float* pw;
    const uint8_t* is_src;
    // outputs / bookkeeping
    // density sources: src_slot[i] = column of node i in src_vals (-1:
    // none); src_vals [src_steps][src_n], row r for step src_first + r,
    // FLT_MAX = no term that step.
    // Null src_slot: the scene has no sources.
    const int* src_slot;
    const float* src_vals;
    int64_t src_n, src_first, src_steps;  // rows apply to steps [src_first, src_first + src_steps)
    float* probe_ring;
    double* partials;  // [2 QP][n_all_items]: column t (slot order) of every item's sums
    float* means;      // [2 QP], slot order
    unsigned long long* step;
};

// position of record (node i, neighbour t) in pass order; the passes of
// [0, split) and [split, n) are cut separately
__host__ __device__ inline int64_t pass_record(int64_t i, int t, int k, int64_t split, int64_t n, int npb) {
    const int64_t base = i < split ? 0 : split;
    const int64_t end = i < split ? split : n;
    const int64_t b = base + (i - base) / npb * npb;
    const int64_t nn = end - b < npb ? end - b : npb;
    return b * k + (int64_t)t * nn + (i - b);
}

// Halo blobs of the D3Q27 RK stages at k = kHaloK: one per bulk/layer pass
// (the passes of [0, nbl), in order), kHaloBlobBytes each:
//   u32 [4 + kHaloCap]   row count m, three zero pads, the pass's m distinct
//                        neighbour rows in ascending order (zero after m)
//   float4 [npb k]       the pass's stencil records in tile order, with the
//                        row's position in that list in place of the node
//                        index; zero after the pass's nn k records
// A pass with m > kHaloCap keeps the node indices in its records and its
// stages gather the rows from global memory.
constexpr int kHaloK = 32;
constexpr int kHaloCap = 272;
constexpr int kHaloListBytes = (4 + kHaloCap) * 4;
constexpr int kHaloBlobBytes = kHaloListBytes + 32 * kHaloK * 16;
static_assert(kHaloListBytes % 16 == 0 && kHaloBlobBytes % 16 == 0, "bulk-copy sizes");

struct WorkItem {
    uint32_t scene;
    uint32_t begin;
    uint32_t end;
    uint32_t local;  // index of the item among its scene's items of the same range kind
};

}  // namespace naga

namespace naga {

// Output targets of the divergence-stencil build; any pointer may be null.
struct StencilOut {
    double* W64;          // [n][k][D], FP64
    double* delta;        // [n]
    float* W32;           // [n][k][D], FP32 (the C++ facade's divergence_operator<float, D>)
    float* delta32;       // [n]
    float4* Wf;           // scene records [n][k]: (Wx, Wy, Wz | filter weight, index bits)
    float2* Ff;           // D == 3 filter records [n][k] (weight, index bits)
    double filter_sigma;  // Gaussian sigma of the selective filter (h / 2.5)
    // pass order of Wf / Ff: passes of npb nodes over [0, split) and
    // [split, n_total); npb = 0 keeps node-major order
    int64_t split, n_total;
    int npb;
};

// One step's launch parameters for a batch of scenes.
struct StepLaunch {
    const SceneDev* scenes;
    int nscenes;
    const WorkItem* all;  // 128-node items (thread-per-node kernels)
    int n_all;
    const WorkItem* all_mt;  // pass-sized items of all nodes (multi-thread kernels)
    int n_all_mt;
    const WorkItem* fluid;
    int n_fluid;
    const WorkItem* edge;  // pass-sized items of the boundary nodes
    int n_edge;
    const WorkItem* pml;  // bulk/layer items whose stencils reach the layer
    int n_pml;
};

// k, kb: the batch's common stencil sizes (0 if the members differ)
int enqueue_step(int dim, int k, int kb, const StepLaunch& P, cudaStream_t st);
// nodes of one pass of the multi-thread-per-node kernels
int nodes_per_pass(int dim);
const char* kernel_name(int id);
int kernel_count();
// NAGA_ETIMEOUT (and clears the flag) if a step kernel gave up waiting for a
// table copy since the last check; synchronises `st`
int tile_timeout_check(cudaStream_t st);
// a bounded wait that nothing completes, then tile_timeout_check (expects
// NAGA_ETIMEOUT): the failure path of the step kernels' tile pipeline
int wait_selftest(int polls, cudaStream_t st);
// G rows of the rest state plus a density perturbation (device drho [n],
// or null for the rest state)
int density_rows_device(int dim, const float* drho, int64_t n, float* G, cudaStream_t st);
// chooses the gather kernels' resident blocks per SM for this batch shape
// (once per shape; must not run during stream capture)
int tune_step_shapes(int dim, int k, int kb, const StepLaunch& P, cudaStream_t st);
// the tuner's measurements, one line per tuned shape
std::string tuning_report();
// D2Q9: (Wx, Wy, index) triplets of the pass-ordered stencil records
int compact_records_device(const float4* stW, int64_t count, float* stR, cudaStream_t st);
// the PML gather records of a scene (stW in pass order)
int pml_table_device(int dim, const float4* stW, int64_t nb, int64_t nl, int64_t nbl, int64_t n, int k, float4* stP,
                     cudaStream_t st);
// the halo blobs of a D3Q27 scene with k = kHaloK (stW in pass order,
// npb-node passes over [0, nbl)); stH holds ceil(nbl / npb) blobs
int halo_build_device(const float4* stW, int64_t nbl, int k, int npb, float4* stH, cudaStream_t st);
// the per-node PML vectors PV of a scene (stW in pass order)
int pml_vectors_device(int dim, const float4* stW, const float* sigma, int64_t nb, int64_t nl, int64_t nbl, int64_t n,
                       int k, float4* PV, cudaStream_t st);
void prof_begin(int id, cudaStream_t st);
void prof_end(int id, cudaStream_t st);
bool prof_on();
int knn_device(const float* src, int64_t n, const float* qry, int64_t nq, int dim, int k, uint32_t* idx,
               float* d2, cudaStream_t st);
int rbf_weights_device(const float* src, int64_t nsrc, int dim, const uint32_t* support, int k, const double* qry,
                       int64_t ngroups, int group, double spacing, int shape, int precision, double* weights,
                       cudaStream_t st);
int divergence_build_device(const float* pts, int64_t n, int dim, int k, int shape, int precision, uint32_t* idx,
                            StencilOut out, cudaStream_t st);
int batched_inverse(const double* A, double* Ainv, int n, int64_t batch, int* info, bool refined, int max_iter,
                    double tol, cudaStream_t st);

}  // namespace naga
