// Warp-cooperative dense LU factorisation and solves for small systems
// (n <= 64) held in shared memory, one warp per system.
//
// Pivoting follows LAPACK getrf: at column j the pivot is the first row of
// maximal |a| among rows j..n-1 (the semantics of the cuBLAS getrfBatched
// call NAGA makes at linalg/detail/batched_matrix_inverse.cuh:46-72).
// Matrices are column-major with leading dimension n: a(i, j) = A[i + n j].
#pragma once
#include "common.cuh"

namespace naga {

// In-place LU of the n x n matrix A. piv[j] receives the row swapped with j.
// Returns 0, or j + 1 for the first column whose pivot is exactly zero
// (that column is then left unreduced, as LAPACK does).
template <class T>
__device__ int warp_lu(T* A, int n, int* piv) {
    const int lane = lane_id();
    int info = 0;
    for (int j = 0; j < n; ++j) {
        T best = T(-1);
        int bi = n;
        for (int i = j + lane; i < n; i += 32) {
            T v = fabs(A[i + n * j]);
            if (v > best) {
                best = v;
                bi = i;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            T ov = __shfl_xor_sync(kFull, best, o);
            int oi = __shfl_xor_sync(kFull, bi, o);
            if (ov > best || (ov == best && oi < bi)) {
                best = ov;
                bi = oi;
            }
        }
        // NaN is never a candidate (v > best fails), so the order is total
        // and the lanes agree; lane 0's choice is broadcast anyway, and a
        // column with no candidate (all NaN) pivots on its own row
        bi = __shfl_sync(kFull, bi, 0);
        const int p = bi < n ? bi : j;
        if (lane == 0) piv[j] = p;
        const T pv = A[p + n * j];
        if (pv == T(0)) {
            if (!info) info = j + 1;
            __syncwarp();
            continue;
        }
        if (p != j)
            for (int c = lane; c < n; c += 32) {
                T t = A[j + n * c];
                A[j + n * c] = A[p + n * c];
                A[p + n * c] = t;
            }
        __syncwarp();
        const T inv = T(1) / A[j + n * j];
        for (int i = j + 1 + lane; i < n; i += 32) A[i + n * j] *= inv;
        __syncwarp();
        for (int i = j + 1 + lane; i < n; i += 32) {
            const T l = A[i + n * j];
            for (int c = j + 1; c < n; ++c) A[i + n * c] -= l * A[j + n * c];
        }
        __syncwarp();
    }
    return info;
}

// Solve A x = b for one right-hand side distributed over the warp: entry e
// of x lives in lane e % 32, register e / 32 (x0 for e < 32, x1 otherwise).
template <class T>
__device__ __forceinline__ T warp_get(T x0, T x1, int e) {
    return __shfl_sync(kFull, e < 32 ? x0 : x1, e & 31);
}

template <class T, class TL>
__device__ void warp_lu_solve_reg(const TL* LU, int n, const int* piv, T& x0, T& x1) {
    const int lane = lane_id();
    for (int j = 0; j < n; ++j) {
        const int p = piv[j];
        if (p != j) {
            T vj = warp_get(x0, x1, j), vp = warp_get(x0, x1, p);
            if (lane == (j & 31)) {
                if (j < 32) x0 = vp; else x1 = vp;
            }
            if (lane == (p & 31)) {
                if (p < 32) x0 = vj; else x1 = vj;
            }
        }
    }
    for (int j = 0; j < n; ++j) {
        const T xj = warp_get(x0, x1, j);
        if (lane > j && lane < n) x0 -= (T)LU[lane + n * j] * xj;
        if (lane + 32 > j && lane + 32 < n) x1 -= (T)LU[lane + 32 + n * j] * xj;
    }
    for (int j = n - 1; j >= 0; --j) {
        T xj = warp_get(x0, x1, j) / (T)LU[j + n * j];
        if (lane == (j & 31)) {
            if (j < 32) x0 = xj; else x1 = xj;
        }
        if (lane < j) x0 -= (T)LU[lane + n * j] * xj;
        if (lane + 32 < j) x1 -= (T)LU[lane + 32 + n * j] * xj;
    }
}

// Inverse from the factors: lane c computes column c of A^-1 (columns c,
// c + 32, ...). X is row-major in shared memory (x(i, c) = X[i n + c]) so
// the lanes' accesses are consecutive.
template <class T>
__device__ void warp_lu_inverse(const T* LU, int n, const int* piv, T* X) {
    const int lane = lane_id();
    for (int c = lane; c < n; c += 32) {
        for (int i = 0; i < n; ++i) X[i * n + c] = (i == c) ? T(1) : T(0);
        for (int j = 0; j < n; ++j) {
            const int p = piv[j];
            if (p != j) {
                T t = X[j * n + c];
                X[j * n + c] = X[p * n + c];
                X[p * n + c] = t;
            }
        }
        for (int j = 0; j < n; ++j) {
            const T xj = X[j * n + c];
            if (xj != T(0))
                for (int i = j + 1; i < n; ++i) X[i * n + c] -= LU[i + n * j] * xj;
        }
        for (int j = n - 1; j >= 0; --j) {
            const T xj = X[j * n + c] / LU[j + n * j];
            X[j * n + c] = xj;
            for (int i = 0; i < j; ++i) X[i * n + c] -= LU[i + n * j] * xj;
        }
    }
    __syncwarp();
}

}  // namespace naga
