// Batched inverse of small dense matrices: one warp per matrix, the matrix
// and its factors in shared memory.
//
// Replaces linalg::batched_matrix_inverse (linalg/batched_matrix_inverse.cuh:
// 325-397), which hands slices of the batch to cuBLAS getrfBatched +
// getriBatched on an executor thread per device (:121-282).
#include "warp_lu.cuh"
#include "scene_dev.hpp"

#include <algorithm>

namespace naga {

namespace {

size_t smem_limit() {
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    return v > 0 ? (size_t)v : 48 * 1024;
}

__global__ void inverse_f64_kernel(const double* __restrict__ A, double* __restrict__ Ainv, int n, int64_t batch,
                                   int* __restrict__ info, int warps_per_block) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int w = threadIdx.x >> 5, lane = lane_id();
    const size_t per_warp = (size_t)16 * n * n + 16 * ((n + 3) / 4);
    double* LU = reinterpret_cast<double*>(smem + per_warp * w);
    double* X = LU + n * n;
    int* piv = reinterpret_cast<int*>(X + n * n);
    const int64_t nw = (int64_t)gridDim.x * warps_per_block;
    for (int64_t b = (int64_t)blockIdx.x * warps_per_block + w; b < batch; b += nw) {
        const double* a = A + b * (int64_t)n * n;
        for (int e = lane; e < n * n; e += 32) LU[e] = a[e];
        __syncwarp();
        int inf = warp_lu(LU, n, piv);
        warp_lu_inverse(LU, n, piv, X);
        double* o = Ainv + b * (int64_t)n * n;
        for (int e = lane; e < n * n; e += 32) o[e] = X[(e % n) * n + e / n];
        if (info && lane == 0) info[b] = inf;
        __syncwarp();
    }
}

// FP32 LU, FP64 residual refinement of every column of the inverse.
__global__ void inverse_f32r_kernel(const double* __restrict__ A, double* __restrict__ Ainv, int n, int64_t batch,
                                    int max_iter, double tol, int* __restrict__ info, int warps_per_block) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int w = threadIdx.x >> 5, lane = lane_id();
    const size_t per_warp = (size_t)24 * n * n + 16 * ((n + 3) / 4);
    double* Ad = reinterpret_cast<double*>(smem + per_warp * w);
    double* X = Ad + n * n;
    float* LUf = reinterpret_cast<float*>(X + n * n);
    float* R = LUf + n * n;
    int* piv = reinterpret_cast<int*>(R + n * n);
    const int64_t nw = (int64_t)gridDim.x * warps_per_block;
    for (int64_t b = (int64_t)blockIdx.x * warps_per_block + w; b < batch; b += nw) {
        const double* a = A + b * (int64_t)n * n;
        for (int e = lane; e < n * n; e += 32) {
            double v = a[e];
            Ad[e] = v;
            LUf[e] = (float)v;
        }
        __syncwarp();
        int inf = warp_lu(LUf, n, piv);
        warp_lu_inverse(LUf, n, piv, R);
        for (int e = lane; e < n * n; e += 32) X[e] = (double)R[e];
        __syncwarp();
        // per column: last correction, the one before, and whether it is done
        double dlast[2] = {INFINITY, INFINITY}, dprev[2] = {INFINITY, INFINITY}, xlast[2] = {0, 0};
        bool cdone[2] = {lane >= n, lane + 32 >= n};
        bool done = false;
        for (int it = 0; it < max_iter && !done && inf == 0; ++it) {
            // residual R = I - A X, column c by lane c
            for (int c = lane; c < n; c += 32)
                for (int i = 0; i < n; ++i) {
                    double r = (i == c) ? 1.0 : 0.0;
                    for (int j = 0; j < n; ++j) r -= Ad[i + n * j] * X[j * n + c];
                    R[i * n + c] = (float)r;
                }
            __syncwarp();
            // correction D = LU^-1 R (in place), X += D
            for (int c = lane, t = 0; c < n; c += 32, ++t) {
                if (cdone[t]) continue;
                for (int j = 0; j < n; ++j) {
                    const int p = piv[j];
                    if (p != j) {
                        float tmp = R[j * n + c];
                        R[j * n + c] = R[p * n + c];
                        R[p * n + c] = tmp;
                    }
                }
                for (int j = 0; j < n; ++j) {
                    const float xj = R[j * n + c];
                    for (int i = j + 1; i < n; ++i) R[i * n + c] -= LUf[i + n * j] * xj;
                }
                for (int j = n - 1; j >= 0; --j) {
                    const float xj = R[j * n + c] / LUf[j + n * j];
                    R[j * n + c] = xj;
                    for (int i = 0; i < j; ++i) R[i * n + c] -= LUf[i + n * j] * xj;
                }
                double dmax = 0, xmax = 0;
                for (int i = 0; i < n; ++i) {
                    double x = X[i * n + c] + (double)R[i * n + c];
                    X[i * n + c] = x;
                    dmax = fmax(dmax, fabs((double)R[i * n + c]));
                    xmax = fmax(xmax, fabs(x));
                }
                dprev[t] = dlast[t];
                dlast[t] = dmax;
                xlast[t] = xmax;
                // done when below the tolerance or no longer contracting
                cdone[t] = dmax <= tol * xmax || dmax > 0.5 * dprev[t];
            }
            done = __all_sync(kFull, cdone[0] && cdone[1]);
            __syncwarp();
        }
        // converged: last correction within the tolerance, or within 1e-10
        // of the column when refinement stagnated at the FP64 residual floor
        bool conv = true;
        for (int t = 0; t < 2; ++t)
            if (lane + 32 * t < n)
                conv = conv && (dlast[t] <= tol * xlast[t] || dlast[t] <= 1e-10 * xlast[t]);
        done = __all_sync(kFull, conv);
        double* o = Ainv + b * (int64_t)n * n;
        for (int e = lane; e < n * n; e += 32) o[e] = X[(e % n) * n + e / n];
        if (info && lane == 0) info[b] = inf != 0 ? inf : (done ? 0 : -1);
        __syncwarp();
    }
}

}  // namespace

int batched_inverse(const double* A, double* Ainv, int n, int64_t batch, int* info, bool refined, int max_iter,
                    double tol, cudaStream_t st) {
    if (n < 1 || n > 64) return set_error(NAGA_EINVAL, "batched inverse: n must be in [1, 64]");
    if (batch < 0) return set_error(NAGA_EINVAL, "batched inverse: negative batch");
    if (batch == 0) return NAGA_OK;
    if (!A || !Ainv) return set_error(NAGA_EINVAL, "batched inverse: null pointer");
    const size_t per_warp = (refined ? (size_t)24 : (size_t)16) * n * n + 16 * ((n + 3) / 4);
    const size_t lim = smem_limit();
    int wpb = (int)std::min<size_t>(8, lim / per_warp);
    if (wpb < 1) return set_error(NAGA_EINVAL, "batched inverse: matrix too large for shared memory");
    const size_t smem = per_warp * wpb;
    const int64_t blocks_needed = (batch + wpb - 1) / wpb;
    const int blocks = (int)std::min<int64_t>(blocks_needed, (int64_t)sm_count() * 32);
    if (!refined) {
        NAGA_CUDA_TRY(cudaFuncSetAttribute(inverse_f64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        inverse_f64_kernel<<<blocks, 32 * wpb, smem, st>>>(A, Ainv, n, batch, info, wpb);
    } else {
        NAGA_CUDA_TRY(cudaFuncSetAttribute(inverse_f32r_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        inverse_f32r_kernel<<<blocks, 32 * wpb, smem, st>>>(A, Ainv, n, batch, max_iter, tol, info, wpb);
    }
    NAGA_CUDA_TRY(cudaGetLastError());
    return NAGA_OK;
}

}  // namespace naga

extern "C" int naga_batched_inverse_f64(const double* A, double* A_inv, int n, int64_t batch, int* info,
                                        void* stream) {
    return naga::batched_inverse(A, A_inv, n, batch, info, false, 0, 0.0, (cudaStream_t)stream);
}

extern "C" int naga_batched_inverse_f32r(const double* A, double* A_inv, int n, int64_t batch, int max_iter,
                                         double rel_tol, int* info, void* stream) {
    if (max_iter < 0 || !(rel_tol >= 0)) return naga::set_error(NAGA_EINVAL, "naga_batched_inverse_f32r: bad tolerance");
    return naga::batched_inverse(A, A_inv, n, batch, info, true, max_iter, rel_tol, (cudaStream_t)stream);
}
