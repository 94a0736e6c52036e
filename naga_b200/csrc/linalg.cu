// Batched inverse of small dense matrices, one warp per matrix: FP64
// Gauss-Jordan in registers for the stencil system sizes (19, 20, 35, 36),
// FP64 LU in shared memory for any other n <= 64, and FP32 LU with FP64
// residual refinement.
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

// Register-resident Gauss-Jordan inverse for the stencil system sizes
// (n = k + D + 1: 19 / 20 for k = 16, 35 / 36 for k = 32). Lane l holds rows
// l and l + 32 in registers. Each elimination step publishes the scaled pivot
// row in shared memory and every lane updates its rows from it, so the n^3
// multiply-adds are independent register FMAs rather than a chain of
// shared-memory read-modify-writes.
//
// Pivoting is virtual: every row carries its getrf position (the row order
// after the swaps so far). The pivot of step k is the first row, in that
// order, of maximal |a| among positions >= k. That is getrf's choice, so the
// pivot sequence and info match the LU kernel. With B = P A the matrix in
// pivot order, the in-place sweep (pivot row scaled by p = 1 / a_kk, a_kk
// replaced by p; every other row i: a_ij -= a_ik a_kj, a_ik = -a_ik p) leaves
// row k of B^-1 in the row pivoted at step k. Since A^-1 = B^-1 P, the store
// un-permutes: A^-1(k, r_m) = B^-1(k, m), with r_m the row pivoted at step m.
//
// Register columns rotate by one each step: at step k register j holds column
// (k + j) mod n, so the pivot column is always register 0 and the new inverse
// column enters at register n - 1; after n steps the order is the identity
// again. The step loop therefore indexes no register by k.
//
// Measured alternatives, all slower or equal (10^6 systems of 36 x 36 on
// B200, 18.6 ms for this form): per-row scales instead of rescaling the pivot
// row (19.6 ms), the next pivot searched while the current step's columns
// update (19.6-19.9 ms), a vote-and-shuffle fast path for a unique maximum
// (19.3 ms), the step loop fully unrolled without rotation (25.3 ms at 228
// registers).
constexpr int kGjWarps = 2;

template <int N>
__global__ void __launch_bounds__(32 * kGjWarps, (N > 32 ? 5 : 8))
    inverse_gj_kernel(const double* __restrict__ A, double* __restrict__ Ainv, int64_t batch,
                      int* __restrict__ info) {
    constexpr int S = (N + 31) / 32;
    constexpr int NP = (N + 1) & ~1;
    // per warp: the published pivot row (double-buffered by step parity) and
    // the physical row pivoted at each step
    __shared__ __align__(16) double prow[kGjWarps][2][NP];
    __shared__ int rowk[kGjWarps][N];
    const int w = threadIdx.x >> 5, lane = lane_id();
    const int64_t nw = (int64_t)gridDim.x * kGjWarps;
    for (int64_t b = (int64_t)blockIdx.x * kGjWarps + w; b < batch; b += nw) {
        const double* ai = A + b * (int64_t)(N * N);
        double a[S][N];
        int pos[S];
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const int r = lane + 32 * s;
            pos[s] = r < N ? r : N;  // N marks a padding row
#pragma unroll
            for (int c = 0; c < N; ++c) a[s][c] = r < N ? ai[r + N * c] : 0.0;
        }
        int inf = 0;
#pragma unroll 1
        for (int k = 0; k < N; ++k) {
            // pivot: max |a| over positions >= k, ties to the lowest position.
            // |a| >= 0, so its bits order like unsigned integers.
            unsigned hi = 0, lo = 0;
            int bp = N;
#pragma unroll
            for (int s = 0; s < S; ++s) {
                const unsigned long long v = (unsigned long long)__double_as_longlong(fabs(a[s][0]));
                const unsigned h = (unsigned)(v >> 32), l = (unsigned)v;
                const bool better = h > hi || (h == hi && (l > lo || (l == lo && pos[s] < bp)));
                if (pos[s] >= k && pos[s] < N && better) {
                    hi = h;
                    lo = l;
                    bp = pos[s];
                }
            }
            const unsigned mh = __reduce_max_sync(kFull, hi);
            const unsigned ml = __reduce_max_sync(kFull, hi == mh ? lo : 0u);
            const int bpos = __reduce_min_sync(kFull, (hi == mh && lo == ml) ? bp : N);
            const bool zero = (mh | ml) == 0u;
            if (zero && !inf) inf = k + 1;
            bool piv[S];
#pragma unroll
            for (int s = 0; s < S; ++s) {
                piv[s] = pos[s] == bpos;
                pos[s] = pos[s] == k ? bpos : (piv[s] ? k : pos[s]);
            }
            // the pivot row's owner scales it and publishes it rotated:
            // pr[m] = a_r(m + 1) p for m < N - 1, pr[N - 1] = p
            double* pr = prow[w][k & 1];
#pragma unroll
            for (int s = 0; s < S; ++s)
                if (piv[s]) {
                    rowk[w][k] = lane + 32 * s;
                    const double p = zero ? 0.0 : 1.0 / a[s][0];
                    a[s][0] = p;
#pragma unroll
                    for (int j = 1; j < N; ++j) a[s][j] *= p;
#pragma unroll
                    for (int m = 0; m + 1 < N; m += 2)
                        *reinterpret_cast<double2*>(pr + m) = make_double2(a[s][m + 1], m + 2 < N ? a[s][m + 2] : p);
                    if (N & 1) pr[N - 1] = p;
                }
            __syncwarp();
            // every row: a_i(m) = a_i(m + 1) - f_i pr[m] (rotated), the new
            // column -f_i p; the pivot row (f = 0) only rotates, keeping p
            double f[S], l[S];
#pragma unroll
            for (int s = 0; s < S; ++s) {
                f[s] = piv[s] ? 0.0 : a[s][0];
                l[s] = piv[s] ? a[s][0] : 0.0;
            }
#pragma unroll
            for (int m = 0; m < N; m += 2) {
                const double2 q = *reinterpret_cast<const double2*>(pr + m);
#pragma unroll
                for (int s = 0; s < S; ++s) {
                    a[s][m] = fma(-f[s], q.x, m + 1 < N ? a[s][m + 1] : l[s]);
                    if (m + 1 < N) a[s][m + 1] = fma(-f[s], q.y, m + 2 < N ? a[s][m + 2] : l[s]);
                }
            }
        }
        __syncwarp();
        double* o = Ainv + b * (int64_t)(N * N);
#pragma unroll
        for (int s = 0; s < S; ++s)
            if (lane + 32 * s < N)
#pragma unroll
                for (int j = 0; j < N; ++j) o[pos[s] + N * rowk[w][j]] = a[s][j];
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

template <int N>
int launch_gj(const double* A, double* Ainv, int64_t batch, int* info, cudaStream_t st) {
    static int per_sm = 0;
    if (per_sm < 1) {
        NAGA_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, inverse_gj_kernel<N>, 32 * kGjWarps, 0));
        per_sm = std::max(per_sm, 1);
    }
    const int64_t need = (batch + kGjWarps - 1) / kGjWarps;
    const int blocks = (int)std::min<int64_t>(need, (int64_t)sm_count() * per_sm);
    inverse_gj_kernel<N><<<blocks, 32 * kGjWarps, 0, st>>>(A, Ainv, batch, info);
    NAGA_CUDA_TRY(cudaGetLastError());
    return NAGA_OK;
}

}  // namespace

int batched_inverse(const double* A, double* Ainv, int n, int64_t batch, int* info, bool refined, int max_iter,
                    double tol, cudaStream_t st) {
    if (n < 1 || n > 64) return set_error(NAGA_EINVAL, "batched inverse: n must be in [1, 64]");
    if (batch < 0) return set_error(NAGA_EINVAL, "batched inverse: negative batch");
    if (batch == 0) return NAGA_OK;
    if (!A || !Ainv) return set_error(NAGA_EINVAL, "batched inverse: null pointer");
    if (!refined) switch (n) {
            case 19: return launch_gj<19>(A, Ainv, batch, info, st);
            case 20: return launch_gj<20>(A, Ainv, batch, info, st);
            case 35: return launch_gj<35>(A, Ainv, batch, info, st);
            case 36: return launch_gj<36>(A, Ainv, batch, info, st);
            default: break;
        }
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
