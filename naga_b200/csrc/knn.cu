// Exact k-nearest-neighbour search for point clouds on the GPU.
//
// Contract: for every query, the k source points that are smallest under the
// lexicographic order (dist^2, index), with dist^2 the FP32 value of NAGA's
// euclidean_squared (distance_functions.hpp:138-161). NAGA's own search
// (segmentation/nearest_neighbors.cuh:181-440) visits cells in a randomised
// order, breaks ties by visit order and stops one ring after k points are
// found; this search is exact instead, so results are reproducible and
// bit-identical to any exact implementation of the same order.
//
// Layout: each cloud is binned on a uniform grid (about two points per
// cell); the points are counting-sorted by cell into float4 records
// (x, y, z, local index). One warp serves one query: it walks Chebyshev
// shells of cells around the query's cell, gathering the shell's points
// from contiguous row segments (cells along x are adjacent in the sorted
// array), and keeps the k best candidates spread over the warp's lanes
// (entry e in lane e % 32, register e / 32). The walk stops once the k-th
// candidate is strictly closer than the nearest face of the searched block
// that does not already touch the edge of the grid.
#include "common.cuh"
#include "scene_dev.hpp"

#include <cstring>

#include <cub/device/device_scan.cuh>
#include <cuda.h>

#include <cmath>
#include <mutex>
#include <string>
#include <vector>

namespace naga {

namespace {

struct CloudGrid {
    double lo[3];
    double w;
    int dims[3];
    int _pad;
    int64_t cell_base;  // first cell of this cloud in the global cell array
    int64_t pt_base;    // first point of this cloud (in the input arrays)
    int64_t n;          // points in the cloud
};

__device__ __forceinline__ int find_cloud(const int64_t* offsets, int nclouds, int64_t p) {
    int lo = 0, hi = nclouds - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (offsets[mid] <= p)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// order-preserving float <-> int encoding for atomic min / max
__device__ __forceinline__ int f2ord(float f) {
    int i = __float_as_int(f);
    return i >= 0 ? i : i ^ 0x7fffffff;
}
__host__ __device__ inline float ord2f(int i) {
#ifdef __CUDA_ARCH__
    return __int_as_float(i >= 0 ? i : i ^ 0x7fffffff);
#else
    int j = i >= 0 ? i : i ^ 0x7fffffff;
    float f;
    std::memcpy(&f, &j, 4);
    return f;
#endif
}

template <int D>
__global__ void bbox_kernel(const float* pts, const int64_t* offsets, int nclouds, int64_t total,
                            int* bbox /* [nclouds][2][3] ordered ints */) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < total;
         p += (int64_t)gridDim.x * blockDim.x) {
        int c = find_cloud(offsets, nclouds, p);
#pragma unroll
        for (int d = 0; d < D; ++d) {
            int v = f2ord(pts[p * D + d]);
            atomicMin(&bbox[c * 6 + d], v);
            atomicMax(&bbox[c * 6 + 3 + d], v);
        }
    }
}

template <int D>
__device__ __forceinline__ void cell_of(const CloudGrid& g, const float* x, int* c) {
#pragma unroll
    for (int d = 0; d < D; ++d) {
        double v = floor(((double)x[d] - g.lo[d]) / g.w);
        long long iv = (long long)v;
        c[d] = (int)min(max(iv, 0LL), (long long)g.dims[d] - 1);
    }
}

template <int D>
__device__ __forceinline__ int64_t cell_id(const CloudGrid& g, const int* c) {
    int64_t id = c[0];
    if (D > 1) id += (int64_t)g.dims[0] * c[1];
    if (D > 2) id += (int64_t)g.dims[0] * g.dims[1] * c[2];
    return id;
}

template <int D>
__global__ void count_kernel(const float* pts, const int64_t* offsets, int nclouds, int64_t total,
                             const CloudGrid* grids, unsigned* counts) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < total;
         p += (int64_t)gridDim.x * blockDim.x) {
        int cl = find_cloud(offsets, nclouds, p);
        CloudGrid g = grids[cl];
        int c[3];
        cell_of<D>(g, pts + p * D, c);
        atomicAdd(&counts[g.cell_base + cell_id<D>(g, c)], 1u);
    }
}

template <int D>
__global__ void scatter_kernel(const float* pts, const int64_t* offsets, int nclouds, int64_t total,
                               const CloudGrid* grids, const unsigned* start, unsigned* fill,
                               float4* sorted) {
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < total;
         p += (int64_t)gridDim.x * blockDim.x) {
        int cl = find_cloud(offsets, nclouds, p);
        CloudGrid g = grids[cl];
        int c[3];
        cell_of<D>(g, pts + p * D, c);
        int64_t cid = g.cell_base + cell_id<D>(g, c);
        unsigned pos = start[cid] + atomicAdd(&fill[cid], 1u);
        float4 r;
        r.x = pts[p * D + 0];
        r.y = D > 1 ? pts[p * D + 1] : 0.f;
        r.z = D > 2 ? pts[p * D + 2] : 0.f;
        r.w = __uint_as_float((unsigned)(p - g.pt_base));
        sorted[pos] = r;
    }
}

struct Cand {
    float d2;
    unsigned idx;
};

__device__ __forceinline__ bool cand_less(float ad, unsigned ai, float bd, unsigned bi) {
    return ad < bd || (ad == bd && ai < bi);
}

// Warp-per-query exact search. R = list registers per lane (k <= 32 R).
template <int D, int R>
__global__ void __launch_bounds__(256) query_kernel(const float* qry, int64_t nq, const int64_t* q_offsets,
                                                    int q_nclouds, const CloudGrid* grids,
                                                    const unsigned* cell_start, const float4* sorted,
                                                    int k, uint32_t* out_idx, float* out_d2) {
    const int lane = lane_id();
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t q = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; q < nq; q += warps) {
        const int cl = q_offsets ? find_cloud(q_offsets, q_nclouds, q) : 0;
        const CloudGrid g = grids[cl];
        float x[3] = {0.f, 0.f, 0.f};
#pragma unroll
        for (int d = 0; d < D; ++d) x[d] = qry[q * D + d];
        int c0[3] = {0, 0, 0};
        cell_of<D>(g, x, c0);

        float ld[R];
        unsigned li[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            ld[r] = INFINITY;
            li[r] = 0xffffffffu;
        }
        const int kl = (k - 1) & 31, kr = (k - 1) >> 5;

        for (int rad = 0;; ++rad) {
            // rows of the shell: (2 rad + 1)^(D-1) rows along x, each giving at
            // most two segments (the full row, or its two end cells)
            int side = 2 * rad + 1;
            int nrows = (D == 2) ? side : side * side;
            int nseg = 2 * nrows;
            for (int s0 = 0; s0 < nseg; s0 += 32) {
                int sid = s0 + lane;
                unsigned sb = 0, se = 0;
                if (sid < nseg) {
                    int row = sid >> 1, half = sid & 1;
                    int dy = (row % side) - rad;
                    int dz = (D == 3) ? (row / side) - rad : 0;
                    int cy = c0[1] + dy, cz = c0[2] + dz;
                    bool full = (dy == -rad || dy == rad) || (D == 3 && (dz == -rad || dz == rad));
                    bool row_ok = cy >= 0 && cy < g.dims[1] && (D < 3 || (cz >= 0 && cz < g.dims[2]));
                    int xa, xb;
                    if (full) {
                        xa = half ? 1 : c0[0] - rad;
                        xb = half ? 0 : c0[0] + rad;
                    } else {
                        xa = xb = half ? c0[0] + rad : c0[0] - rad;
                    }
                    xa = max(xa, 0);
                    xb = min(xb, g.dims[0] - 1);
                    if (row_ok && xa <= xb) {
                        int ca[3] = {xa, cy, cz}, cb[3] = {xb, cy, cz};
                        int64_t ia = g.cell_base + cell_id<D>(g, ca);
                        int64_t ib = g.cell_base + cell_id<D>(g, cb);
                        sb = cell_start[ia];
                        se = cell_start[ib + 1];
                    }
                }
                unsigned len = se - sb;
                // inclusive scan of segment lengths across the warp
                unsigned incl = len;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    unsigned t = __shfl_up_sync(kFull, incl, o);
                    if (lane >= o) incl += t;
                }
                unsigned excl = incl - len;
                unsigned total = __shfl_sync(kFull, incl, 31);
                for (unsigned base = 0; base < total; base += 32) {
                    unsigned t = base + lane;
                    float cd = INFINITY;
                    unsigned ci = 0xffffffffu;
                    // find the segment holding item t: largest lane j with excl_j <= t
                    int j = 0;
#pragma unroll
                    for (int step = 16; step > 0; step >>= 1) {
                        unsigned e = __shfl_sync(kFull, excl, j + step);
                        if (j + step < 32 && e <= t) j += step;
                    }
                    unsigned sbj = __shfl_sync(kFull, sb, j);
                    unsigned exj = __shfl_sync(kFull, excl, j);
                    if (t < total) {
                        float4 p = sorted[sbj + (t - exj)];
                        float pv[3] = {p.x, p.y, p.z};
                        cd = dist2_ref<D>(x, pv);
                        ci = __float_as_uint(p.w);
                    }
                    float kd = __shfl_sync(kFull, ld[kr], kl);
                    unsigned ki = __shfl_sync(kFull, li[kr], kl);
                    unsigned mask = __ballot_sync(kFull, cand_less(cd, ci, kd, ki));
                    while (mask) {
                        int b = __ffs(mask) - 1;
                        mask &= mask - 1;
                        float bd = __shfl_sync(kFull, cd, b);
                        unsigned bi = __shfl_sync(kFull, ci, b);
                        kd = __shfl_sync(kFull, ld[kr], kl);
                        ki = __shfl_sync(kFull, li[kr], kl);
                        if (!cand_less(bd, bi, kd, ki)) continue;
                        int pos = 0;
#pragma unroll
                        for (int r = 0; r < R; ++r)
                            pos += __popc(__ballot_sync(kFull, cand_less(ld[r], li[r], bd, bi)));
                        // shift entries >= pos up by one and drop the last
                        float carry_d = INFINITY;
                        unsigned carry_i = 0xffffffffu;
#pragma unroll
                        for (int r = 0; r < R; ++r) {
                            float upd = __shfl_up_sync(kFull, ld[r], 1);
                            unsigned upi = __shfl_up_sync(kFull, li[r], 1);
                            float topd = __shfl_sync(kFull, ld[r], 31);
                            unsigned topi = __shfl_sync(kFull, li[r], 31);
                            float prevd = lane == 0 ? carry_d : upd;
                            unsigned previ = lane == 0 ? carry_i : upi;
                            int e = 32 * r + lane;
                            if (e == pos) {
                                ld[r] = bd;
                                li[r] = bi;
                            } else if (e > pos) {
                                ld[r] = prevd;
                                li[r] = previ;
                            }
                            carry_d = topd;
                            carry_i = topi;
                        }
                    }
                }
            }
            // stopping test after the full shell
            double bound = INFINITY;
            bool covered = true;
#pragma unroll
            for (int d = 0; d < D; ++d) {
                if (c0[d] - rad > 0) {
                    covered = false;
                    bound = fmin(bound, (double)x[d] - (g.lo[d] + (double)(c0[d] - rad) * g.w));
                }
                if (c0[d] + rad < g.dims[d] - 1) {
                    covered = false;
                    bound = fmin(bound, (g.lo[d] + (double)(c0[d] + rad + 1) * g.w) - (double)x[d]);
                }
            }
            if (covered) break;
            float kd = __shfl_sync(kFull, ld[kr], kl);
            if (kd < INFINITY && bound > 0 && (double)kd < bound * bound * (1.0 - 1e-5)) break;
        }
#pragma unroll
        for (int r = 0; r < R; ++r) {
            int e = 32 * r + lane;
            if (e < k) {
                out_idx[q * k + e] = li[r];
                out_d2[q * k + e] = ld[r];
            }
        }
    }
}

template <int D>
int knn_run(const float* src, const int64_t* h_src_off, int nclouds, const float* qry, int64_t nq,
            const int64_t* h_q_off, int k, uint32_t* idx, float* d2, cudaStream_t st) {
    const int64_t total = h_src_off[nclouds];
    int64_t* d_off = nullptr;
    int64_t* d_qoff = nullptr;
    int* d_bbox = nullptr;
    CloudGrid* d_grids = nullptr;
    unsigned *d_counts = nullptr, *d_start = nullptr, *d_fill = nullptr;
    float4* d_sorted = nullptr;
    void* d_tmp = nullptr;
    int rc = NAGA_OK;
    std::vector<int> hb(6 * nclouds);
    std::vector<CloudGrid> grids(nclouds);
    int64_t ncell = 0;
    size_t tmp_bytes = 0;
    auto fail = [&](cudaError_t e, const char* what) {
        rc = set_error(NAGA_ECUDA, std::string("naga_knn: ") + what + ": " + cudaGetErrorString(e));
    };
    cudaError_t e;
#define KTRY(x, what)          \
    if ((e = (x)) != cudaSuccess) { \
        fail(e, what);         \
        goto done;             \
    }
    KTRY(cudaMallocAsync(&d_off, sizeof(int64_t) * (nclouds + 1), st), "alloc");
    KTRY(cudaMemcpyAsync(d_off, h_src_off, sizeof(int64_t) * (nclouds + 1), cudaMemcpyHostToDevice, st), "copy");
    if (h_q_off) {
        KTRY(cudaMallocAsync(&d_qoff, sizeof(int64_t) * (nclouds + 1), st), "alloc");
        KTRY(cudaMemcpyAsync(d_qoff, h_q_off, sizeof(int64_t) * (nclouds + 1), cudaMemcpyHostToDevice, st), "copy");
    }
    for (int c = 0; c < nclouds; ++c)
        for (int d = 0; d < 3; ++d) {
            hb[c * 6 + d] = 0x7fffffff;
            hb[c * 6 + 3 + d] = (int)0x80000000;
        }
    KTRY(cudaMallocAsync(&d_bbox, sizeof(int) * 6 * nclouds, st), "alloc");
    KTRY(cudaMemcpyAsync(d_bbox, hb.data(), sizeof(int) * 6 * nclouds, cudaMemcpyHostToDevice, st), "copy");
    if (total > 0) {
        int blocks = (int)std::min<int64_t>((total + 255) / 256, 4 * 148 * 8);
        bbox_kernel<D><<<blocks, 256, 0, st>>>(src, d_off, nclouds, total, d_bbox);
        KTRY(cudaGetLastError(), "bbox kernel");
    }
    KTRY(cudaMemcpyAsync(hb.data(), d_bbox, sizeof(int) * 6 * nclouds, cudaMemcpyDeviceToHost, st), "copy");
    KTRY(cudaStreamSynchronize(st), "sync");
    for (int c = 0; c < nclouds; ++c) {
        CloudGrid& g = grids[c];
        int64_t n = h_src_off[c + 1] - h_src_off[c];
        double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0}, vol = 1;
        for (int d = 0; d < D; ++d) {
            lo[d] = n > 0 ? (double)ord2f(hb[c * 6 + d]) : 0.0;
            hi[d] = n > 0 ? (double)ord2f(hb[c * 6 + 3 + d]) : 1.0;
            // a NaN or infinite coordinate always lands in a bound (the
            // ordered-integer min / max puts NaN at one end)
            if (!std::isfinite(lo[d]) || !std::isfinite(hi[d])) {
                rc = set_error(NAGA_EINVAL, "naga_knn: non-finite point coordinates in cloud " + std::to_string(c));
                goto done;
            }
            if (hi[d] - lo[d] < 1e-6) hi[d] = lo[d] + 1e-6;
            vol *= hi[d] - lo[d];
        }
        double w = std::pow(2.0 * vol / (double)std::max<int64_t>(n, 1), 1.0 / D);
        int64_t cells = 1;
        for (int d = 0; d < 3; ++d) {
            g.lo[d] = lo[d];
            int64_t dd = d < D ? std::max<int64_t>(1, (int64_t)std::ceil((hi[d] - lo[d]) / w)) : 1;
            dd = std::min<int64_t>(dd, 1 << 20);
            g.dims[d] = (int)dd;
            cells *= dd;
        }
        g.w = w;
        g.cell_base = ncell;
        g.pt_base = h_src_off[c];
        g.n = n;
        ncell += cells;
    }
    KTRY(cudaMallocAsync(&d_grids, sizeof(CloudGrid) * nclouds, st), "alloc");
    KTRY(cudaMemcpyAsync(d_grids, grids.data(), sizeof(CloudGrid) * nclouds, cudaMemcpyHostToDevice, st), "copy");
    KTRY(cudaMallocAsync(&d_counts, sizeof(unsigned) * (ncell + 1), st), "alloc");
    KTRY(cudaMallocAsync(&d_start, sizeof(unsigned) * (ncell + 1), st), "alloc");
    KTRY(cudaMallocAsync(&d_fill, sizeof(unsigned) * (ncell + 1), st), "alloc");
    KTRY(cudaMemsetAsync(d_counts, 0, sizeof(unsigned) * (ncell + 1), st), "memset");
    KTRY(cudaMemsetAsync(d_fill, 0, sizeof(unsigned) * (ncell + 1), st), "memset");
    KTRY(cudaMallocAsync(&d_sorted, sizeof(float4) * std::max<int64_t>(total, 1), st), "alloc");
    if (total > 0) {
        int blocks = (int)std::min<int64_t>((total + 255) / 256, 4 * 148 * 8);
        count_kernel<D><<<blocks, 256, 0, st>>>(src, d_off, nclouds, total, d_grids, d_counts);
        KTRY(cudaGetLastError(), "count kernel");
    }
    KTRY(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, d_counts, d_start, ncell + 1, st), "scan size");
    KTRY(cudaMallocAsync(&d_tmp, tmp_bytes, st), "alloc");
    KTRY(cub::DeviceScan::ExclusiveSum(d_tmp, tmp_bytes, d_counts, d_start, ncell + 1, st), "scan");
    if (total > 0) {
        int blocks = (int)std::min<int64_t>((total + 255) / 256, 4 * 148 * 8);
        scatter_kernel<D><<<blocks, 256, 0, st>>>(src, d_off, nclouds, total, d_grids, d_start, d_fill,
                                                  d_sorted);
        KTRY(cudaGetLastError(), "scatter kernel");
    }
    if (nq > 0) {
        int64_t warps_needed = nq;
        int blocks = (int)std::min<int64_t>((warps_needed + 7) / 8, (int64_t)sm_count() * 16);
        if (k <= 32)
            query_kernel<D, 1><<<blocks, 256, 0, st>>>(qry, nq, d_qoff, nclouds, d_grids, d_start, d_sorted, k,
                                                       idx, d2);
        else
            query_kernel<D, 2><<<blocks, 256, 0, st>>>(qry, nq, d_qoff, nclouds, d_grids, d_start, d_sorted, k,
                                                       idx, d2);
        KTRY(cudaGetLastError(), "query kernel");
    }
done:
#undef KTRY
    cudaFreeAsync(d_off, st);
    if (d_qoff) cudaFreeAsync(d_qoff, st);
    cudaFreeAsync(d_bbox, st);
    if (d_grids) cudaFreeAsync(d_grids, st);
    if (d_counts) cudaFreeAsync(d_counts, st);
    if (d_start) cudaFreeAsync(d_start, st);
    if (d_fill) cudaFreeAsync(d_fill, st);
    if (d_sorted) cudaFreeAsync(d_sorted, st);
    if (d_tmp) cudaFreeAsync(d_tmp, st);
    return rc;
}

}  // namespace

// internal entry used by the scene set-up (src and queries on the device)
int knn_device(const float* src, int64_t n, const float* qry, int64_t nq, int dim, int k, uint32_t* idx,
               float* d2, cudaStream_t st) {
    if (dim != 2 && dim != 3) return set_error(NAGA_EINVAL, "naga_knn: dim must be 2 or 3");
    if (k < 1 || k > 64) return set_error(NAGA_EINVAL, "naga_knn: k must be in [1, 64]");
    if (n < 0 || nq < 0 || n > (int64_t)0xfffffffe) return set_error(NAGA_EINVAL, "naga_knn: bad sizes");
    int64_t off[2] = {0, n};
    return dim == 2 ? knn_run<2>(src, off, 1, qry, nq, nullptr, k, idx, d2, st)
                    : knn_run<3>(src, off, 1, qry, nq, nullptr, k, idx, d2, st);
}

// ----------------------------------------------- allocation-free variant
// Some callers cannot call cudaMalloc once they are running: processes that
// hand all free device memory to their own caching allocator at start-up
// and run on a fixed budget, and latency-critical serving paths, where
// cudaMalloc / cudaFree may synchronise the device and stall every other
// stream. naga_knn_noalloc serves them: its scratch (cell grid, counting
// sort, sorted point records) lives in one file-scope device array that every
// GPU loading this library holds until the process exits. The array's
// host-side name is only a stand-in; its device address is looked up once
// per device with cudaGetSymbolAddress.
namespace {

constexpr int64_t kNoAllocMaxPoints = 65536;  // largest source cloud
constexpr int64_t kNoAllocMaxCells = 65536;   // cap on the cell grid

struct NoAllocScratch {
    int bbox[8];
    int64_t offsets[2];
    CloudGrid grid;
    unsigned counts[kNoAllocMaxCells + 1];
    unsigned start[kNoAllocMaxCells + 1];
    unsigned fill[kNoAllocMaxCells + 1];
    float4 sorted[kNoAllocMaxPoints];
};

static __device__ __align__(256) unsigned char g_knn_scratch[sizeof(NoAllocScratch)];

// Unique id of the calling thread's current context (cuCtxGetId through the
// runtime's driver entry points, so the library needs no libcuda link);
// false when it cannot be had (no current context, an older driver).
bool current_context_id(unsigned long long* id) {
    using GetCurrent = CUresult (*)(CUcontext*);
    using GetId = CUresult (*)(CUcontext, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", (void**)&get_current, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            get_current = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", (void**)&get_id, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            get_id = nullptr;
    });
    CUcontext ctx = nullptr;
    if (!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || !ctx) return false;
    return get_id(ctx, id) == CUDA_SUCCESS;
}

// device address of g_knn_scratch in the current context: looked up once
// per device and context, and again when the device's context changed (a
// cudaDeviceReset or a host framework resetting the primary context loads
// the module anew, and the array may move); without a context id the
// lookup is made on every call
int noalloc_scratch(NoAllocScratch** out) {
    static std::mutex mu;
    static void* addr[64] = {nullptr};
    static unsigned long long ctx_of[64] = {0};
    int dev = 0;
    NAGA_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return set_error(NAGA_EINVAL, "naga_knn_noalloc: device ordinal above 63");
    unsigned long long ctx = 0;
    const bool known = current_context_id(&ctx);
    std::lock_guard<std::mutex> lk(mu);
    if (!known || !addr[dev] || ctx_of[dev] != ctx) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_knn_scratch);
        if (e != cudaSuccess)
            return set_error(NAGA_ECUDA, std::string("naga_knn_noalloc: cudaGetSymbolAddress: ") +
                                             cudaGetErrorString(e));
        addr[dev] = known ? p : nullptr;
        ctx_of[dev] = ctx;
        *out = reinterpret_cast<NoAllocScratch*>(p);
        return NAGA_OK;
    }
    *out = reinterpret_cast<NoAllocScratch*>(addr[dev]);
    return NAGA_OK;
}

// resets what must start at zero and the bounding box of a new call
__global__ void noalloc_init_kernel(NoAllocScratch* s, int64_t n) {
    const int64_t t0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    for (int64_t t = t0; t <= kNoAllocMaxCells; t += (int64_t)gridDim.x * blockDim.x) {
        s->counts[t] = 0u;
        s->fill[t] = 0u;
    }
    if (t0 < 3) {
        s->bbox[t0] = 0x7fffffff;
        s->bbox[3 + t0] = (int)0x80000000;
    }
    if (t0 == 0) {
        s->offsets[0] = 0;
        s->offsets[1] = n;
    }
}

__global__ void noalloc_set_grid_kernel(NoAllocScratch* s, CloudGrid g) { s->grid = g; }

// exclusive scan of counts[0, m) into start[0, m) by one block
__global__ void noalloc_scan_kernel(NoAllocScratch* s, int m) {
    __shared__ unsigned part[1024];
    const int t = threadIdx.x;
    const int per = (m + blockDim.x - 1) / blockDim.x;
    const int b = t * per, e = min(m, b + per);
    unsigned acc = 0;
    for (int i = b; i < e; ++i) acc += s->counts[i];
    part[t] = acc;
    __syncthreads();
    for (int o = 1; o < (int)blockDim.x; o <<= 1) {
        unsigned v = t >= o ? part[t - o] : 0u;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    unsigned run = part[t] - acc;
    for (int i = b; i < e; ++i) {
        s->start[i] = run;
        run += s->counts[i];
    }
}

template <int D>
int knn_noalloc_run(const float* src, int64_t n, const float* qry, int64_t nq, int k, uint32_t* idx, float* d2,
                    cudaStream_t st) {
    NoAllocScratch* scr = nullptr;
    int rc = noalloc_scratch(&scr);
    if (rc) return rc;
    noalloc_init_kernel<<<64, 256, 0, st>>>(scr, n);
    NAGA_CUDA_TRY(cudaGetLastError());
    if (n > 0) {
        const int blocks = (int)std::min<int64_t>((n + 255) / 256, 4 * 148 * 8);
        bbox_kernel<D><<<blocks, 256, 0, st>>>(src, scr->offsets, 1, n, scr->bbox);
        NAGA_CUDA_TRY(cudaGetLastError());
    }
    int hb[6];
    NAGA_CUDA_TRY(cudaMemcpyAsync(hb, scr->bbox, sizeof(hb), cudaMemcpyDeviceToHost, st));
    NAGA_CUDA_TRY(cudaStreamSynchronize(st));
    CloudGrid g{};
    double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0}, vol = 1;
    for (int d = 0; d < D; ++d) {
        lo[d] = n > 0 ? (double)ord2f(hb[d]) : 0.0;
        hi[d] = n > 0 ? (double)ord2f(hb[3 + d]) : 1.0;
        if (!std::isfinite(lo[d]) || !std::isfinite(hi[d]))
            return set_error(NAGA_EINVAL, "naga_knn_noalloc: non-finite point coordinates");
        if (hi[d] - lo[d] < 1e-6) hi[d] = lo[d] + 1e-6;
        vol *= hi[d] - lo[d];
    }
    double w = std::pow(2.0 * vol / (double)std::max<int64_t>(n, 1), 1.0 / D);
    int64_t cells = 0;
    for (;;) {
        cells = 1;
        for (int d = 0; d < 3; ++d) {
            const int64_t dd = d < D ? std::max<int64_t>(1, (int64_t)std::ceil((hi[d] - lo[d]) / w)) : 1;
            g.dims[d] = (int)std::min<int64_t>(dd, 1 << 20);
            cells *= g.dims[d];
        }
        if (cells <= kNoAllocMaxCells) break;
        w *= 1.25;  // coarser cells: the search stays exact, only slower
    }
    for (int d = 0; d < 3; ++d) g.lo[d] = lo[d];
    g.w = w;
    g.cell_base = 0;
    g.pt_base = 0;
    g.n = n;
    noalloc_set_grid_kernel<<<1, 1, 0, st>>>(scr, g);
    if (n > 0) {
        const int blocks = (int)std::min<int64_t>((n + 255) / 256, 4 * 148 * 8);
        count_kernel<D><<<blocks, 256, 0, st>>>(src, scr->offsets, 1, n, &scr->grid, scr->counts);
        noalloc_scan_kernel<<<1, 1024, 0, st>>>(scr, (int)cells + 1);
        scatter_kernel<D><<<blocks, 256, 0, st>>>(src, scr->offsets, 1, n, &scr->grid, scr->start, scr->fill,
                                                  scr->sorted);
    } else {
        noalloc_scan_kernel<<<1, 1024, 0, st>>>(scr, (int)cells + 1);
    }
    NAGA_CUDA_TRY(cudaGetLastError());
    if (nq > 0) {
        const int blocks = (int)std::min<int64_t>((nq + 7) / 8, (int64_t)sm_count() * 16);
        if (k <= 32)
            query_kernel<D, 1><<<blocks, 256, 0, st>>>(qry, nq, nullptr, 1, &scr->grid, scr->start, scr->sorted, k,
                                                       idx, d2);
        else
            query_kernel<D, 2><<<blocks, 256, 0, st>>>(qry, nq, nullptr, 1, &scr->grid, scr->start, scr->sorted, k,
                                                       idx, d2);
        NAGA_CUDA_TRY(cudaGetLastError());
    }
    return NAGA_OK;
}

}  // namespace

}  // namespace naga

using namespace naga;

extern "C" int naga_knn_noalloc(const float* src, int64_t n, const float* qry, int64_t nq, int dim, int k,
                                uint32_t* idx, float* d2, void* stream) {
    if (dim != 2 && dim != 3) return set_error(NAGA_EINVAL, "naga_knn_noalloc: dim must be 2 or 3");
    if (k < 1 || k > 64) return set_error(NAGA_EINVAL, "naga_knn_noalloc: k must be in [1, 64]");
    if (n < 0 || nq < 0) return set_error(NAGA_EINVAL, "naga_knn_noalloc: negative size");
    if (n > kNoAllocMaxPoints)
        return set_error(NAGA_EINVAL, "naga_knn_noalloc: " + std::to_string(n) +
                                          " source points exceed the fixed scratch of 65536 points; use naga_knn");
    if ((n > 0 && !src) || (nq > 0 && (!qry || !idx || !d2)))
        return set_error(NAGA_EINVAL, "naga_knn_noalloc: null pointer");
    cudaStream_t st = (cudaStream_t)stream;
    return dim == 2 ? knn_noalloc_run<2>(src, n, qry, nq, k, idx, d2, st)
                    : knn_noalloc_run<3>(src, n, qry, nq, k, idx, d2, st);
}

extern "C" int naga_knn(const float* src, int64_t n, const float* qry, int64_t nq, int dim, int k,
                        uint32_t* idx, float* d2, void* stream) {
    if ((n > 0 && !src) || (nq > 0 && (!qry || !idx || !d2)))
        return set_error(NAGA_EINVAL, "naga_knn: null pointer");
    return knn_device(src, n, qry, nq, dim, k, idx, d2, (cudaStream_t)stream);
}

extern "C" int naga_knn_clouds(const float* pts, const int64_t* offsets, int n_clouds, int dim, int k,
                               uint32_t* idx, float* d2, void* stream) {
    if (!offsets || n_clouds < 1) return set_error(NAGA_EINVAL, "naga_knn_clouds: bad offsets");
    if (dim != 2 && dim != 3) return set_error(NAGA_EINVAL, "naga_knn_clouds: dim must be 2 or 3");
    if (k < 1 || k > 64) return set_error(NAGA_EINVAL, "naga_knn_clouds: k must be in [1, 64]");
    for (int c = 0; c < n_clouds; ++c)
        if (offsets[c + 1] < offsets[c]) return set_error(NAGA_EINVAL, "naga_knn_clouds: offsets decrease");
    if (offsets[0] != 0) return set_error(NAGA_EINVAL, "naga_knn_clouds: offsets[0] must be 0");
    int64_t total = offsets[n_clouds];
    if (total > 0 && (!pts || !idx || !d2)) return set_error(NAGA_EINVAL, "naga_knn_clouds: null pointer");
    cudaStream_t st = (cudaStream_t)stream;
    return dim == 2 ? knn_run<2>(pts, offsets, n_clouds, pts, total, offsets, k, idx, d2, st)
                    : knn_run<3>(pts, offsets, n_clouds, pts, total, offsets, k, idx, d2, st);
}
