// Device-side helpers shared by the kernels of libnaga_b200.so (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "naga_internal.hpp"

#define NAGA_CUDA_TRY(expr)                                                              \
    do {                                                                                 \
        cudaError_t _e = (expr);                                                         \
        if (_e != cudaSuccess)                                                           \
            return ::naga::set_error(NAGA_ECUDA, std::string(#expr) + ": " +            \
                                                     cudaGetErrorString(_e));           \
    } while (0)

namespace naga {

constexpr int kWarp = 32;
constexpr unsigned kFull = 0xffffffffu;

// number of streaming multiprocessors of the current device (cached)
int sm_count();

// ------------------------------------------------------------------ lattices
// Velocity sets, weights, bounce-back maps and collision matrices of the two
// lattices NAGA defines (fluids/nonlocal_lattice_boltzmann/detail/
// d3q27_lattice.cuh:45-98,380-387 and d2q9_lattice.cuh:44-82,142-155). The
// numeric tables are part of the collision model and are identical to the
// reference's.
// Node rows in HBM hold the populations in a "paired" order: every
// direction is followed by its opposite, so a float4 chunk holds two
// opposite pairs (c and -c share |c . W| in the streaming gather, and
// bounce-back swaps within a chunk). D3Q27 starts with the rest population
// and one pad; D2Q9 puts its four pairs in the first two chunks and the rest
// population (zero streaming rate) with three pads in the third, so its RK
// stages and PML gather never touch the third chunk. row(slot) is the
// population stored in a slot (-1: pad), pos(a) the slot of population a.
struct D2Q9 {
    static constexpr int D = 2, Q = 9, QP = 12;  // QP: padded row (3 x float4)
    static constexpr int NGATHER = 2;             // chunks with a nonzero streaming rate
    // rows of the RK stage buffers and the PML field: only the gathered
    // chunks, 32 B (one sector per neighbour gather instead of 1.5 at 48 B)
    static constexpr int QS = 4 * NGATHER;
    static constexpr __host__ __device__ int row(int slot) {
        constexpr int t[12] = {1, 5, 2, 6, 3, 7, 4, 8, 0, -1, -1, -1};
        return t[slot];
    }
    static constexpr __host__ __device__ int pos(int a) {
        constexpr int t[9] = {8, 0, 2, 4, 6, 1, 3, 5, 7};
        return t[a];
    }
};
struct D3Q27 {
    static constexpr int D = 3, Q = 27, QP = 28;  // QP: padded row (7 x float4)
    static constexpr int NGATHER = 7;              // chunk 0 holds the rest population and a pair
    static constexpr int QS = QP;                  // stage and PML field rows: the full row
    static constexpr __host__ __device__ int row(int slot) {
        constexpr int t[28] = {0,  -1, 1,  2,  3,  4,  5,  6,  7,  10, 8,  9,  11, 14,
                               12, 13, 15, 18, 16, 17, 19, 26, 20, 25, 21, 24, 22, 23};
        return t[slot];
    }
    static constexpr __host__ __device__ int pos(int a) {
        constexpr int t[27] = {0,  2,  3,  4,  5,  6,  7,  8,  10, 11, 9,  12, 14, 15,
                               13, 16, 18, 19, 17, 20, 22, 24, 26, 27, 25, 23, 21};
        return t[a];
    }
};

template <class L>
struct LatticeTables;

template <>
struct LatticeTables<D2Q9> {
    // rest, nw, w, sw, s, se, e, ne, n
    static constexpr __host__ __device__ int cx(int a) {
        constexpr int t[9] = {0, -1, -1, -1, 0, 1, 1, 1, 0};
        return t[a];
    }
    static constexpr __host__ __device__ int cy(int a) {
        constexpr int t[9] = {0, 1, 0, -1, -1, -1, 0, 1, 1};
        return t[a];
    }
    static constexpr __host__ __device__ int cz(int a) {
        constexpr int t[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        return t[a];
    }
    static constexpr __host__ __device__ float w(int a) {
        constexpr float t[9] = {4.f / 9.f,  1.f / 36.f, 1.f / 9.f,  1.f / 36.f, 1.f / 9.f,
                                   1.f / 36.f, 1.f / 9.f,  1.f / 36.f, 1.f / 9.f};
        return t[a];
    }
    static constexpr __host__ __device__ int bb(int a) {
        constexpr int t[9] = {0, 5, 6, 7, 8, 1, 2, 3, 4};
        return t[a];
    }
    static constexpr __host__ __device__ int K(int l, int j) {
        constexpr int t[9][9] = {{1, 0, 0, -4, 0, 0, 0, 0, 4},   {1, -1, 1, 2, 0, 1, -1, 1, 1},
                                    {1, -1, 0, -1, 1, 0, 0, -2, -2}, {1, -1, -1, 2, 0, -1, 1, 1, 1},
                                    {1, 0, -1, -1, -1, 0, -2, 0, -2}, {1, 1, -1, 2, 0, 1, 1, -1, 1},
                                    {1, 1, 0, -1, 1, 0, 0, 2, -2},   {1, 1, 1, 2, 0, -1, -1, -1, 1},
                                    {1, 0, 1, -1, -1, 0, 2, 0, -2}};
        return t[l][j];
    }
};

template <>
struct LatticeTables<D3Q27> {
    static constexpr __host__ __device__ int cx(int a) {
        constexpr int t[27] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1,
                                   -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1};
        return t[a];
    }
    static constexpr __host__ __device__ int cy(int a) {
        constexpr int t[27] = {0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0,
                                   0, 1, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, -1};
        return t[a];
    }
    static constexpr __host__ __device__ int cz(int a) {
        constexpr int t[27] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1,
                                   -1, 1, 1, -1, -1, 1, 1, 1, 1, -1, -1, -1, -1};
        return t[a];
    }
    static constexpr __host__ __device__ float w(int a) {
        constexpr float t[27] = {
        8.f / 27.f,  2.f / 27.f,  2.f / 27.f,  2.f / 27.f,  2.f / 27.f,  2.f / 27.f,  2.f / 27.f,
        1.f / 54.f,  1.f / 54.f,  1.f / 54.f,  1.f / 54.f,  1.f / 54.f,  1.f / 54.f,  1.f / 54.f,
        1.f / 54.f,  1.f / 54.f,  1.f / 54.f,  1.f / 54.f,  1.f / 54.f,  1.f / 216.f, 1.f / 216.f,
        1.f / 216.f, 1.f / 216.f, 1.f / 216.f, 1.f / 216.f, 1.f / 216.f, 1.f / 216.f};
        return t[a];
    }
    static constexpr __host__ __device__ int bb(int a) {
        constexpr int t[27] = {0,  2,  1,  4,  3,  6,  5,  10, 9,  8,  7,  14, 13, 12,
                                   11, 18, 17, 16, 15, 26, 25, 24, 23, 22, 21, 20, 19};
        return t[a];
    }
    static constexpr __host__ __device__ int K(int l, int j) {
        constexpr int t[27][27] = {
        {1, 0, 0, 0, 0, 0, 0, 0, 0, -2, 0, 0, 0, 0, 0, 0, 0, 4, 0, 0, 0, 0, 0, 0, 0, 0, -8},
        {1, 1, 0, 0, 0, 0, 0, 1, 1, -1, -4, 0, 0, 0, 0, 0, 0, 0, -4, 0, 0, 0, 0, 4, 0, 0, 4},
        {1, -1, 0, 0, 0, 0, 0, 1, 1, -1, 4, 0, 0, 0, 0, 0, 0, 0, -4, 0, 0, 0, 0, -4, 0, 0, 4},
        {1, 0, 1, 0, 0, 0, 0, -1, 1, -1, 0, -4, 0, 0, 0, 0, 0, 0, 2, -2, 0, 0, 0, 0, 4, 0, 4},
        {1, 0, -1, 0, 0, 0, 0, -1, 1, -1, 0, 4, 0, 0, 0, 0, 0, 0, 2, -2, 0, 0, 0, 0, -4, 0, 4},
        {1, 0, 0, 1, 0, 0, 0, 0, -2, -1, 0, 0, -4, 0, 0, 0, 0, 0, 2, 2, 0, 0, 0, 0, 0, 4, 4},
        {1, 0, 0, -1, 0, 0, 0, 0, -2, -1, 0, 0, 4, 0, 0, 0, 0, 0, 2, 2, 0, 0, 0, 0, 0, -4, 4},
        {1, 1, 1, 0, 1, 0, 0, 0, 2, 0, -1, -1, 0, 1, 1, 0, 0, -1, 1, 1, 0, 0, -2, -2, -2, 0, -2},
        {1, -1, 1, 0, -1, 0, 0, 0, 2, 0, 1, -1, 0, -1, 1, 0, 0, -1, 1, 1, 0, 0, 2, 2, -2, 0, -2},
        {1, 1, -1, 0, -1, 0, 0, 0, 2, 0, -1, 1, 0, 1, -1, 0, 0, -1, 1, 1, 0, 0, 2, -2, 2, 0, -2},
        {1, -1, -1, 0, 1, 0, 0, 0, 2, 0, 1, 1, 0, -1, -1, 0, 0, -1, 1, 1, 0, 0, -2, 2, 2, 0, -2},
        {1, 1, 0, 1, 0, 1, 0, 1, -1, 0, -1, 0, -1, -1, 0, 1, 0, -1, 1, -1, 0, -2, 0, -2, 0, -2, -2},
        {1, -1, 0, 1, 0, -1, 0, 1, -1, 0, 1, 0, -1, 1, 0, 1, 0, -1, 1, -1, 0, 2, 0, 2, 0, -2, -2},
        {1, 1, 0, -1, 0, -1, 0, 1, -1, 0, -1, 0, 1, -1, 0, -1, 0, -1, 1, -1, 0, 2, 0, -2, 0, 2, -2},
        {1, -1, 0, -1, 0, 1, 0, 1, -1, 0, 1, 0, 1, 1, 0, -1, 0, -1, 1, -1, 0, -2, 0, 2, 0, 2, -2},
        {1, 0, 1, 1, 0, 0, 1, -1, -1, 0, 0, -1, -1, 0, -1, -1, 0, -1, -2, 0, -2, 0, 0, 0, -2, -2, -2},
        {1, 0, -1, 1, 0, 0, -1, -1, -1, 0, 0, 1, -1, 0, 1, -1, 0, -1, -2, 0, 2, 0, 0, 0, 2, -2, -2},
        {1, 0, 1, -1, 0, 0, -1, -1, -1, 0, 0, -1, 1, 0, -1, 1, 0, -1, -2, 0, 2, 0, 0, 0, -2, 2, -2},
        {1, 0, -1, -1, 0, 0, 1, -1, -1, 0, 0, 1, 1, 0, 1, 1, 0, -1, -2, 0, -2, 0, 0, 0, 2, 2, -2},
        {1, 1, 1, 1, 1, 1, 1, 0, 0, 1, 2, 2, 2, 0, 0, 0, 1, 1, 0, 0, 1, 1, 1, 1, 1, 1, 1},
        {1, -1, 1, 1, -1, -1, 1, 0, 0, 1, -2, 2, 2, 0, 0, 0, -1, 1, 0, 0, 1, -1, -1, -1, 1, 1, 1},
        {1, 1, -1, 1, -1, 1, -1, 0, 0, 1, 2, -2, 2, 0, 0, 0, -1, 1, 0, 0, -1, 1, -1, 1, -1, 1, 1},
        {1, -1, -1, 1, 1, -1, -1, 0, 0, 1, -2, -2, 2, 0, 0, 0, 1, 1, 0, 0, -1, -1, 1, -1, -1, 1, 1},
        {1, 1, 1, -1, 1, -1, -1, 0, 0, 1, 2, 2, -2, 0, 0, 0, -1, 1, 0, 0, -1, -1, 1, 1, 1, -1, 1},
        {1, -1, 1, -1, -1, 1, -1, 0, 0, 1, -2, 2, -2, 0, 0, 0, 1, 1, 0, 0, -1, 1, -1, -1, 1, -1, 1},
        {1, 1, -1, -1, -1, -1, 1, 0, 0, 1, 2, -2, -2, 0, 0, 0, 1, 1, 0, 0, 1, -1, -1, 1, -1, -1, 1},
        {1, -1, -1, -1, 1, 1, 1, 0, 0, 1, -2, -2, -2, 0, 0, 0, -1, 1, 0, 0, 1, 1, 1, -1, -1, -1, 1},
    };
        return t[l][j];
    }
};

// --------------------------------------------------------------- warp utils
__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}

// Squared distance exactly as NAGA's loopless euclidean_squared
// (distance_functions.hpp:138-161): highest dimension added last, rounded
// multiplies and adds (no FMA contraction) so host and device agree bit for
// bit.
template <int D>
__device__ __forceinline__ float dist2_ref(const float* a, const float* b) {
    float dx = __fsub_rn(a[0], b[0]);
    float s = __fmul_rn(dx, dx);
#pragma unroll
    for (int d = 1; d < D; ++d) {
        float t = __fsub_rn(a[d], b[d]);
        s = __fadd_rn(__fmul_rn(t, t), s);
    }
    return s;
}

}  // namespace naga
