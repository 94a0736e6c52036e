// The standalone meshless primitives of NAGA's C++ API that the step does
// not call directly, on the device:
//   * nd_cubic_segmentation (segmentation/nd_cubic_segmentation.cuh:227-303,
//     376-392): the uniform partition of a point cloud NAGA's ring search
//     walks, as its shape and, per partition, the point indices;
//   * radial_point_method<T>::compute_weights with T = float and
//     ::interpolate (interpolation/radial_point_method.cuh:118-280);
//   * divergence_operator<T, D>::apply with a centring offset
//     (nonlocal_calculus/divergence.cuh:377-488), FP32 and FP64.
// The step's own kernels (step.cu) keep their fused forms; these entry points
// serve callers of the primitives (the C++ facade's classes of the same
// names).
#include "common.cuh"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

namespace naga {

int rbf_weights_device(const float* src, int64_t nsrc, int dim, const uint32_t* support, int k, const double* qry,
                       int64_t ngroups, int group, double spacing, int shape, int precision, double* weights,
                       cudaStream_t st);

namespace {

// ------------------------------------------------------------ segmentation
// order-preserving float <-> int encoding for atomic min / max
__device__ __forceinline__ int ord_of(float f) {
    const int i = __float_as_int(f);
    return i >= 0 ? i : i ^ 0x7fffffff;
}
float float_of(int i) {
    const int j = i >= 0 ? i : i ^ 0x7fffffff;
    float f;
    std::memcpy(&f, &j, 4);
    return f;
}

template <int D>
__global__ void seg_bounds_kernel(const float* __restrict__ pts, int64_t n, int* __restrict__ bounds) {
    int lo[D], hi[D];
#pragma unroll
    for (int d = 0; d < D; ++d) {
        lo[d] = 0x7fffffff;
        hi[d] = (int)0x80000000;
    }
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
#pragma unroll
        for (int d = 0; d < D; ++d) {
            const int v = ord_of(pts[i * D + d]);
            lo[d] = min(lo[d], v);
            hi[d] = max(hi[d], v);
        }
#pragma unroll
    for (int d = 0; d < D; ++d) {
        for (int o = 16; o > 0; o >>= 1) {
            lo[d] = min(lo[d], __shfl_xor_sync(kFull, lo[d], o));
            hi[d] = max(hi[d], __shfl_xor_sync(kFull, hi[d], o));
        }
        if ((threadIdx.x & 31) == 0) {
            atomicMin(&bounds[d], lo[d]);
            atomicMax(&bounds[3 + d], hi[d]);
        }
    }
}

struct SegGrid {
    float lo[3], hi[3], w;
    uint32_t shape[3];
};

// get_partition_index (nd_cubic_segmentation.cuh:376-392): below the lower
// bound -> 0, at or above the upper bound -> shape - 1, else floor((x - lo) /
// w) in FP32 with IEEE division, clamped to shape - 1 (rounding can reach
// shape just below the upper bound)
template <int D>
__global__ void seg_cell_kernel(const float* __restrict__ pts, int64_t n, SegGrid g, uint32_t* __restrict__ cell,
                                uint32_t* __restrict__ iota, uint32_t* __restrict__ sizes) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        uint32_t lin = 0, mul = 1;
#pragma unroll
        for (int d = 0; d < D; ++d) {
            const float x = pts[i * D + d];
            uint32_t c;
            if (x < g.lo[d])
                c = 0;
            else if (x >= g.hi[d])
                c = g.shape[d] - 1;
            else
                c = min((uint32_t)floorf(__fdiv_rn(x - g.lo[d], g.w)), g.shape[d] - 1);
            lin += c * mul;
            mul *= g.shape[d];
        }
        cell[i] = lin;
        iota[i] = (uint32_t)i;
        atomicAdd(&sizes[lin], 1u);
    }
}

int seg_grid_from_bounds(int dim, int64_t n, int approx, const int* hb, SegGrid& g, int64_t& cells) {
    // nd_cubic_segmentation.cuh:245-286 in FP32: a thin axis is widened to
    // 1e-3, width = (approx / n * volume)^(1 / D), shape = ceil(extent /
    // width), upper bound moved to lower + shape * width
    const float tol = 1e-3f;
    float vol = 1.0f;
    for (int d = 0; d < dim; ++d) {
        g.lo[d] = float_of(hb[d]);
        g.hi[d] = float_of(hb[3 + d]);
        if (!std::isfinite(g.lo[d]) || !std::isfinite(g.hi[d]))
            return set_error(NAGA_EINVAL, "naga_segmentation: non-finite point coordinates");
        if (g.hi[d] - g.lo[d] < tol) g.hi[d] = g.lo[d] + tol;
        vol *= g.hi[d] - g.lo[d];
    }
    g.w = std::pow((float)approx / (float)n * vol, 1.0f / (float)dim);
    cells = 1;
    for (int d = 0; d < 3; ++d) {
        if (d < dim) {
            const float s = std::ceil((g.hi[d] - g.lo[d]) / g.w);
            if (!(s >= 1.0f) || s > 4.0e9f) return set_error(NAGA_EINVAL, "naga_segmentation: partition grid too large");
            g.shape[d] = (uint32_t)s;
            g.hi[d] = g.lo[d] + (float)g.shape[d] * g.w;
        } else {
            g.lo[d] = g.hi[d] = 0.f;
            g.shape[d] = 1;
        }
        cells *= g.shape[d];
    }
    if (cells > (int64_t)UINT32_MAX) return set_error(NAGA_EINVAL, "naga_segmentation: partition grid too large");
    return NAGA_OK;
}

// ---------------------------------------------------------- RPIM, FP32 I/O
__global__ void widen_kernel(const float* __restrict__ in, double* __restrict__ out, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (double)in[i];
}
__global__ void narrow_kernel(const double* __restrict__ in, float* __restrict__ out, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (float)in[i];
}

// destination(c, q) = sum_s w(s, q) (field(c, support(s, q / group)) - offset)
// + offset, summed over s in order in FP32 (radial_point_method.cuh:204-218,
// 243-257); one thread per (component, query)
__global__ void rbf_interpolate_kernel(const float* __restrict__ w, const uint32_t* __restrict__ support,
                                       int64_t nq, int group, int k, const float* __restrict__ field,
                                       int n_fields, float offset, float* __restrict__ out) {
    const int64_t total = nq * n_fields;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t q = t / n_fields;
        const int c = (int)(t - q * n_fields);
        const uint32_t* sup = support + (q / group) * k;
        const float* wq = w + q * k;
        float sum = 0.f;
        for (int s = 0; s < k; ++s) sum = fmaf(wq[s], field[(int64_t)sup[s] * n_fields + c] - offset, sum);
        out[t] = sum + offset;
    }
}

// ----------------------------------------------------- divergence apply
// result_i = sum_s t_s with t_s = sum_d W(d, s, i) (F_d(idx(s, i)) - offset)
// accumulated over d in order, and the t_s reduced by NAGA's pairwise tree
// (divergence.cuh:452-468: stride 1, 2, 4, ..., slot 2 s j gains slot 2 s j
// + s when that exists). One warp per node, supports s and s + 32 in each
// lane.
template <class T, int D>
__global__ void divergence_apply_kernel(const T* __restrict__ W, const uint32_t* __restrict__ idx, int64_t n,
                                        int k, const T* __restrict__ field, T offset, T* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
        T v[2] = {T(0), T(0)};
#pragma unroll
        for (int r = 0; r < 2; ++r) {
            const int s = lane + 32 * r;
            if (s < k) {
                const uint32_t j = idx[i * k + s];
                T t = T(0);
#pragma unroll
                for (int d = 0; d < D; ++d) t = fma(W[(i * k + s) * D + d], field[(int64_t)j * D + d] - offset, t);
                v[r] = t;
            }
        }
        // pairwise tree over the k slots: slots 0..31 in v[0] of lanes
        // 0..31, slots 32..63 in v[1]
        for (int st = 1; st < k; st *= 2) {
            if (st < 32) {
#pragma unroll
                for (int r = 0; r < 2; ++r) {
                    const T up = __shfl_down_sync(kFull, v[r], st);
                    const int s = lane + 32 * r;
                    if ((s % (2 * st)) == 0 && s + st < k) v[r] += up;
                }
            } else {  // st == 32: slot 0 gains slot 32
                if (lane == 0 && 32 < k) v[0] += v[1];
            }
        }
        if (lane == 0) out[i] = v[0];
    }
}

}  // namespace
}  // namespace naga

using namespace naga;

extern "C" int naga_segmentation_shape(const float* pts, int64_t n, int dim, int approx_partition_size,
                                       float* lower, float* upper, float* width, int64_t* shape, void* stream) {
    if (dim != 2 && dim != 3) return set_error(NAGA_EINVAL, "naga_segmentation_shape: dim must be 2 or 3");
    if (n < 1 || n > (int64_t)UINT32_MAX || approx_partition_size < 1 || !pts)
        return set_error(NAGA_EINVAL, "naga_segmentation_shape: need n >= 1 points and a partition size >= 1");
    cudaStream_t st = (cudaStream_t)stream;
    int* d_b = nullptr;
    int hb[6];
    for (int d = 0; d < 3; ++d) {
        hb[d] = 0x7fffffff;
        hb[3 + d] = (int)0x80000000;
    }
    NAGA_CUDA_TRY(cudaMallocAsync(&d_b, sizeof hb, st));
    NAGA_CUDA_TRY(cudaMemcpyAsync(d_b, hb, sizeof hb, cudaMemcpyHostToDevice, st));
    const int blocks = (int)std::min<int64_t>((n + 255) / 256, (int64_t)sm_count() * 8);
    if (dim == 2)
        seg_bounds_kernel<2><<<blocks, 256, 0, st>>>(pts, n, d_b);
    else
        seg_bounds_kernel<3><<<blocks, 256, 0, st>>>(pts, n, d_b);
    NAGA_CUDA_TRY(cudaGetLastError());
    NAGA_CUDA_TRY(cudaMemcpyAsync(hb, d_b, sizeof hb, cudaMemcpyDeviceToHost, st));
    NAGA_CUDA_TRY(cudaFreeAsync(d_b, st));
    NAGA_CUDA_TRY(cudaStreamSynchronize(st));
    SegGrid g{};
    int64_t cells = 0;
    int rc = seg_grid_from_bounds(dim, n, approx_partition_size, hb, g, cells);
    if (rc) return rc;
    for (int d = 0; d < dim; ++d) {
        if (lower) lower[d] = g.lo[d];
        if (upper) upper[d] = g.hi[d];
        if (shape) shape[d] = g.shape[d];
    }
    if (width) *width = g.w;
    return NAGA_OK;
}

extern "C" int naga_segmentation_build(const float* pts, int64_t n, int dim, const float* lower,
                                       const float* upper, float width, const int64_t* shape, uint32_t* sizes,
                                       uint32_t* offsets, uint32_t* indices, void* stream) {
    if (dim != 2 && dim != 3) return set_error(NAGA_EINVAL, "naga_segmentation_build: dim must be 2 or 3");
    if (n < 1 || n > (int64_t)UINT32_MAX || !pts || !lower || !upper || !shape || !sizes || !offsets || !indices ||
        !(width > 0))
        return set_error(NAGA_EINVAL, "naga_segmentation_build: invalid argument");
    SegGrid g{};
    int64_t cells = 1;
    for (int d = 0; d < 3; ++d) {
        const bool used = d < dim;
        g.lo[d] = used ? lower[d] : 0.f;
        g.hi[d] = used ? upper[d] : 0.f;
        const int64_t s = used ? shape[d] : 1;
        if (s < 1 || s > (int64_t)UINT32_MAX) return set_error(NAGA_EINVAL, "naga_segmentation_build: bad shape");
        g.shape[d] = (uint32_t)s;
        cells *= s;
        if (cells > (int64_t)UINT32_MAX) return set_error(NAGA_EINVAL, "naga_segmentation_build: bad shape");
    }
    g.w = width;
    cudaStream_t st = (cudaStream_t)stream;
    uint32_t *cell = nullptr, *cell_sorted = nullptr, *iota = nullptr;
    void* tmp = nullptr;
    size_t tmp_scan = 0, tmp_sort = 0;
    int bits = 1;
    while (bits < 32 && (((int64_t)1 << bits) < cells)) ++bits;
    NAGA_CUDA_TRY(cudaMallocAsync(&cell, sizeof(uint32_t) * n, st));
    NAGA_CUDA_TRY(cudaMallocAsync(&cell_sorted, sizeof(uint32_t) * n, st));
    NAGA_CUDA_TRY(cudaMallocAsync(&iota, sizeof(uint32_t) * n, st));
    NAGA_CUDA_TRY(cudaMemsetAsync(sizes, 0, sizeof(uint32_t) * cells, st));
    const int blocks = (int)std::min<int64_t>((n + 255) / 256, (int64_t)sm_count() * 8);
    if (dim == 2)
        seg_cell_kernel<2><<<blocks, 256, 0, st>>>(pts, n, g, cell, iota, sizes);
    else
        seg_cell_kernel<3><<<blocks, 256, 0, st>>>(pts, n, g, cell, iota, sizes);
    NAGA_CUDA_TRY(cudaGetLastError());
    // offsets: exclusive prefix sums of the sizes (nd_cubic_segmentation
    // .inl compute_index_offsets); indices: grouped by partition with a
    // stable sort on the partition index, so each partition lists its
    // points in ascending index order (NAGA's order there is that of its
    // atomic increments, which no two runs need share)
    NAGA_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tmp_scan, sizes, offsets, cells, st));
    NAGA_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tmp_sort, cell, cell_sorted, iota, indices, n, 0, bits,
                                                  st));
    NAGA_CUDA_TRY(cudaMallocAsync(&tmp, std::max(tmp_scan, tmp_sort), st));
    NAGA_CUDA_TRY(cub::DeviceScan::ExclusiveSum(tmp, tmp_scan, sizes, offsets, cells, st));
    NAGA_CUDA_TRY(cub::DeviceRadixSort::SortPairs(tmp, tmp_sort, cell, cell_sorted, iota, indices, n, 0, bits, st));
    NAGA_CUDA_TRY(cudaFreeAsync(tmp, st));
    NAGA_CUDA_TRY(cudaFreeAsync(cell, st));
    NAGA_CUDA_TRY(cudaFreeAsync(cell_sorted, st));
    NAGA_CUDA_TRY(cudaFreeAsync(iota, st));
    return NAGA_OK;
}

extern "C" int naga_rbf_weights_f32(const float* src, int64_t n, int dim, const uint32_t* support, int k,
                                    const float* qry, int64_t ngroups, int group, float spacing, int shape,
                                    int precision, float* weights, void* stream) {
    if (ngroups < 0 || group < 1) return set_error(NAGA_EINVAL, "naga_rbf_weights_f32: bad group size");
    if (ngroups == 0) return NAGA_OK;
    if (!src || !support || !qry || !weights) return set_error(NAGA_EINVAL, "naga_rbf_weights_f32: null pointer");
    if (dim != 2 && dim != 3) return set_error(NAGA_EINVAL, "naga_rbf_weights_f32: dim must be 2 or 3");
    if (k < 1 || k > 64) return set_error(NAGA_EINVAL, "naga_rbf_weights_f32: k out of range");
    cudaStream_t st = (cudaStream_t)stream;
    const int64_t nq = ngroups * group;
    double *q64 = nullptr, *w64 = nullptr;
    NAGA_CUDA_TRY(cudaMallocAsync(&q64, sizeof(double) * nq * dim, st));
    NAGA_CUDA_TRY(cudaMallocAsync(&w64, sizeof(double) * nq * k, st));
    const int b1 = (int)std::min<int64_t>((nq * dim + 255) / 256, (int64_t)sm_count() * 8);
    widen_kernel<<<b1, 256, 0, st>>>(qry, q64, nq * dim);
    NAGA_CUDA_TRY(cudaGetLastError());
    int rc = rbf_weights_device(src, n, dim, support, k, q64, ngroups, group, (double)spacing, shape, precision,
                                w64, st);
    if (rc == NAGA_OK) {
        const int b2 = (int)std::min<int64_t>((nq * k + 255) / 256, (int64_t)sm_count() * 8);
        narrow_kernel<<<b2, 256, 0, st>>>(w64, weights, nq * k);
        if (cudaGetLastError() != cudaSuccess) rc = set_error(NAGA_ECUDA, "naga_rbf_weights_f32: narrow kernel");
    }
    cudaFreeAsync(q64, st);
    cudaFreeAsync(w64, st);
    return rc;
}

extern "C" int naga_rbf_interpolate(const float* weights, const uint32_t* support, int64_t nq, int group, int k,
                                    const float* field, int64_t n_src, int n_fields, float centering_offset,
                                    float* out, void* stream) {
    (void)n_src;
    if (nq < 0 || group < 1 || k < 1 || n_fields < 1)
        return set_error(NAGA_EINVAL, "naga_rbf_interpolate: bad sizes");
    if (nq == 0) return NAGA_OK;
    if (!weights || !support || !field || !out) return set_error(NAGA_EINVAL, "naga_rbf_interpolate: null pointer");
    cudaStream_t st = (cudaStream_t)stream;
    const int blocks = (int)std::min<int64_t>((nq * n_fields + 255) / 256, (int64_t)sm_count() * 8);
    rbf_interpolate_kernel<<<blocks, 256, 0, st>>>(weights, support, nq, group, k, field, n_fields,
                                                   centering_offset, out);
    NAGA_CUDA_TRY(cudaGetLastError());
    return NAGA_OK;
}

namespace {
template <class T>
int divergence_apply_any(const T* W, const uint32_t* idx, int64_t n, int dim, int k, const T* field, T offset,
                         T* result, void* stream, const char* name) {
    if (n < 0 || k < 1 || k > 64 || (dim != 2 && dim != 3))
        return set_error(NAGA_EINVAL, std::string(name) + ": bad sizes");
    if (n == 0) return NAGA_OK;
    if (!W || !idx || !field || !result) return set_error(NAGA_EINVAL, std::string(name) + ": null pointer");
    cudaStream_t st = (cudaStream_t)stream;
    const int blocks = (int)std::min<int64_t>((n + 7) / 8, (int64_t)sm_count() * 16);
    if (dim == 2)
        divergence_apply_kernel<T, 2><<<blocks, 256, 0, st>>>(W, idx, n, k, field, offset, result);
    else
        divergence_apply_kernel<T, 3><<<blocks, 256, 0, st>>>(W, idx, n, k, field, offset, result);
    NAGA_CUDA_TRY(cudaGetLastError());
    return NAGA_OK;
}
}  // namespace

extern "C" int naga_divergence_apply(const float* W, const uint32_t* idx, int64_t n, int dim, int k,
                                     const float* field, float centering_offset, float* result, void* stream) {
    return divergence_apply_any<float>(W, idx, n, dim, k, field, centering_offset, result, stream,
                                       "naga_divergence_apply");
}

extern "C" int naga_divergence_apply_f64(const double* W, const uint32_t* idx, int64_t n, int dim, int k,
                                         const double* field, double centering_offset, double* result,
                                         void* stream) {
    return divergence_apply_any<double>(W, idx, n, dim, k, field, centering_offset, result, stream,
                                        "naga_divergence_apply_f64");
}
