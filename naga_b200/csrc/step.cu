// The time step of NAGA's nonlocal lattice-Boltzmann engine on sm_100a.
//
// Reference: fluids/nonlocal_lattice_boltzmann/detail/simulation_engine.cuh
// step_forward :1325-1375, issued there as ~1000 launches (27 populations x
// separate divergence gathers, reductions and axpy passes). Here one step is
// a fixed sequence of fused kernels over work items (<= 128 consecutive nodes
// of one scene), so one launch covers every scene of a batch:
//
//   macro_pml     all nodes   rho, u; PML trapezoid integrals Q1, Q2, the
//                             local absorption term and the layer field rows
//                             phi; central-moment collision; per-item layer
//                             sums of Q1, Q2
//   scene_tail    per scene   layer means of Q1, Q2 (fixed-order sums); RPIM
//                             probe of rho at the start of the step; step
//                             counter
//   pml_gather    layer-adjacent bulk+layer nodes: the two PML divergence
//                             gathers div(-2 c sigma (Q1 - <Q1>)) and
//                             div(c sigma^2 (Q2 - <Q2>))
//   edge_collide  boundary    RPIM boundary interpolation (+ collision)
//   filter        all nodes   selective Gaussian filter; bounce-back
//   rk(1..4)      bulk+layer  streaming gather + RK4 stage update
//   edge_interp   boundary    RPIM boundary interpolation of the result
//
// Arithmetic is FP32 on centred populations g = f - w and rho - 1: the
// reference keeps f itself in FP32 (T = float), which quantises a 1e-4
// acoustic perturbation of f ~ w to ~1e-3 relative; g keeps full relative
// precision. Where the collision formulas subtract the O(1) equilibrium
// parts of the moments, those parts are cancelled analytically and only the
// small remainders enter the FP32 arithmetic.
//
// Gathers run TPN threads per node (8 for D3Q27, 4 for D2Q9): thread c owns
// float4 chunk c of the node's row, so one warp-wide load of neighbour rows
// touches 4 (8) rows instead of 32, and each thread holds two opposite
// population pairs of its chunk.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <type_traits>
#include <utility>

#include <cub/block/block_radix_sort.cuh>
#include <cub/block/block_scan.cuh>

#include "common.cuh"
#include "scene_dev.hpp"

namespace naga {

namespace {

constexpr int kBlock = 128;    // thread-per-node kernels
constexpr int kBlockMT = 256;  // multi-thread-per-node kernels

template <class L>
struct Lat : LatticeTables<L> {
    static constexpr int D = L::D, Q = L::Q, QP = L::QP;
};

template <class L>
struct MT {
    static constexpr int TPN = L::D == 3 ? 8 : 4;  // threads per node
    static constexpr int NCH = L::QP / 4;          // float4 chunks per row
    static constexpr int NPB = kBlockMT / TPN;     // nodes per block pass
};

// Thread shapes of the pipelined gather kernels: TPN threads per node,
// thread c owning float4 chunk c, passes of MT<L>::NPB nodes (the tables'
// pass order), blocks of NPB * TPN threads. D2Q9 runs without an idle lane:
// its RK stages and PML gather touch only the two pair chunks that carry a
// direction (L::NGATHER), its filter and boundary kernels the three chunks
// of the row (256-scene batch: 1725 -> 2053 MNUPS over four threads per
// node). D3Q27 keeps eight threads for its seven chunks: at seven, nodes
// straddle warps and every 128-B row is requested by two warps (RK stage
// 80 -> 107 us, step 458 -> 361 MNUPS).
template <class L, int TPN_>
struct Shape {
    static constexpr int TPN = TPN_;
    static constexpr int NCH = L::QP / 4;
    static constexpr int NPB = MT<L>::NPB;
    static constexpr int BLOCK = NPB * TPN;
};
template <class L>
using MTR = Shape<L, L::D == 3 ? 8 : L::NGATHER>;  // RK stages, PML gather
template <class L>
using MTF = Shape<L, L::D == 3 ? 8 : L::QP / 4>;   // boundary kernels
// the filter: D2Q9 at two threads per node, thread 0 also filtering the
// rest population (a scalar of the same row), so no lane works on pads
template <class L>
using MTFF = Shape<L, L::D == 3 ? 8 : L::NGATHER>;
// blocks per SM of the filter for the RK stages' tuned bps: the same threads
// per SM (its blocks are the RK stages' size)
template <class L>
constexpr int filter_bps(int bps) {
    return (bps * MTR<L>::BLOCK + MTFF<L>::BLOCK - 1) / MTFF<L>::BLOCK;
}

// blocks per SM of the MTF-shaped kernels for the RK stages' tuned bps: the
// same threads per SM
template <class L>
constexpr int other_bps(int bps) {
    return (bps * MTR<L>::BLOCK + MTF<L>::BLOCK - 1) / MTF<L>::BLOCK;
}

// direction of the first population of each slot pair of a row
// ((0, pad) and (pad, pad) pairs have zero direction)
__constant__ float c_pdir3[14][3] = {{0, 0, 0},  {1, 0, 0},  {0, 1, 0},   {0, 0, 1},  {1, 1, 0},
                                     {-1, 1, 0}, {1, 0, 1},  {-1, 0, 1},  {0, 1, 1},  {0, -1, 1},
                                     {1, 1, 1},  {-1, 1, 1}, {1, -1, 1},  {-1, -1, 1}};
__constant__ float c_pdir2[6][3] = {{-1, 1, 0}, {-1, 0, 0}, {-1, -1, 0}, {0, -1, 0}, {0, 0, 0}, {0, 0, 0}};

template <class L>
__device__ __forceinline__ void pair_dirs(int c, float* d0, float* d1) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        d0[d] = L::D == 3 ? c_pdir3[2 * c][d] : c_pdir2[2 * c][d];
        d1[d] = L::D == 3 ? c_pdir3[2 * c + 1][d] : c_pdir2[2 * c + 1][d];
    }
}

// lattice speed of sound as the reference spells it (lattices.cuh:46-49)
__device__ __forceinline__ float cs_f() { return 0.57735026918962576450914878050196f; }

// full row (QP floats) of node i, slot order
template <class L>
__device__ __forceinline__ void load_row(const float* base, int64_t i, float* v) {
    const float4* p = reinterpret_cast<const float4*>(base + i * L::QP);
#pragma unroll
    for (int c = 0; c < L::QP / 4; ++c) {
        float4 t = p[c];
        v[4 * c + 0] = t.x;
        v[4 * c + 1] = t.y;
        v[4 * c + 2] = t.z;
        v[4 * c + 3] = t.w;
    }
}
template <class L>
__device__ __forceinline__ void store_row(float* base, int64_t i, const float* v) {
    float4* p = reinterpret_cast<float4*>(base + i * L::QP);
#pragma unroll
    for (int c = 0; c < L::QP / 4; ++c) p[c] = make_float4(v[4 * c], v[4 * c + 1], v[4 * c + 2], v[4 * c + 3]);
}
__device__ __forceinline__ float4 ld4(const float* base, int64_t i, int qp, int c) {
    return __ldg(reinterpret_cast<const float4*>(base + i * qp) + c);
}

// The collision scratch S1, S1P of a scene of n nodes. D3Q27: node-major
// rows of QP floats like G. D2Q9: rows of the eight moving populations
// (32 B: one sector per neighbour gather instead of two for a 48-B row),
// the rest population of node i at 8 n + i. Chunk c of node i as a float4;
// D2Q9's chunk 2 carries the rest population in x (its other lanes zero).
template <class L>
__device__ __forceinline__ float4 s1_ld(const float* base, int64_t n, int64_t i, int c) {
    if constexpr (L::D == 2) {
        if (c >= L::NGATHER) return make_float4(base[L::QS * n + i], 0.f, 0.f, 0.f);
        return reinterpret_cast<const float4*>(base + i * L::QS)[c];
    } else {
        return reinterpret_cast<const float4*>(base + i * L::QP)[c];
    }
}
template <class L>
__device__ __forceinline__ void s1_st(float* base, int64_t n, int64_t i, int c, const float4& v) {
    if constexpr (L::D == 2) {
        if (c >= L::NGATHER)
            base[L::QS * n + i] = v.x;
        else
            reinterpret_cast<float4*>(base + i * L::QS)[c] = v;
    } else {
        reinterpret_cast<float4*>(base + i * L::QP)[c] = v;
    }
}
// the whole row (slot order, QP floats of which the pads are not stored)
template <class L>
__device__ __forceinline__ void s1_store_row(float* base, int64_t n, int64_t i, const float* v) {
    if constexpr (L::D == 2) {
        float4* p = reinterpret_cast<float4*>(base + i * L::QS);
#pragma unroll
        for (int c = 0; c < L::NGATHER; ++c) p[c] = make_float4(v[4 * c], v[4 * c + 1], v[4 * c + 2], v[4 * c + 3]);
        base[L::QS * n + i] = v[L::QS];
    } else {
        store_row<L>(base, i, v);
    }
}
// neighbour-row gathers cached in L2 only (.cg): the rows of a pass's
// neighbours are re-read by other passes long after L1 would have evicted
// them, and allocating them in L1 costs more than it saves (D3Q27 RK gather:
// 85 -> 80 us per 250k-node launch)
__device__ __forceinline__ float4 ld4cg(const float* base, int64_t i, int qp, int c) {
    const float4* a = reinterpret_cast<const float4*>(base + i * qp) + c;
    float4 v;
    asm volatile("ld.global.cg.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "l"(a));
    return v;
}
// the gather load of a lattice: D3Q27 rows (112 B) bypass L1; D2Q9 rows
// (48 B, 4.6x more nodes per line) keep the L1 reuse (measured both ways)
template <class L>
__device__ __forceinline__ float4 ld4g(const float* base, int64_t i, int c) {
    if constexpr (L::D == 3)
        return ld4cg(base, i, L::QP, c);
    else
        return __ldg(reinterpret_cast<const float4*>(base + i * L::QP) + c);
}
// the same gather load on a stage or PML field row (L::QS floats)
template <class L>
__device__ __forceinline__ float4 ld4s(const float* base, int64_t i, int c) {
    if constexpr (L::D == 3)
        return ld4cg(base, i, L::QS, c);
    else
        return __ldg(reinterpret_cast<const float4*>(base + i * L::QS) + c);
}
// the gather load of chunk c of a collision scratch row (s1_ld's layout)
template <class L>
__device__ __forceinline__ float4 s1_ldg(const float* base, int64_t n, int64_t j, int c) {
    if constexpr (L::D == 2) {
        if (c >= L::NGATHER) return make_float4(__ldg(base + L::QS * n + j), 0.f, 0.f, 0.f);
        return __ldg(reinterpret_cast<const float4*>(base + j * L::QS) + c);
    } else {
        return ld4g<L>(base, j, c);
    }
}
__device__ __forceinline__ float4 ld4rw(const float* base, int64_t i, int qp, int c) {
    return reinterpret_cast<const float4*>(base + i * qp)[c];
}
__device__ __forceinline__ void st4(float* base, int64_t i, int qp, int c, float4 v) {
    reinterpret_cast<float4*>(base + i * qp)[c] = v;
}

// rho - 1 and u (lattice units) from centred populations (reference order);
// sums in population order as detail/simulation_engine.cuh:53-82
template <class L>
__device__ __forceinline__ void macros(const float* g, float& drho, float* u) {
    using T = Lat<L>;
    drho = 0.f;
    float m[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int a = 0; a < L::Q; ++a) {
        drho += g[a];
        if (T::cx(a)) m[0] += T::cx(a) > 0 ? g[a] : -g[a];
        if (T::cy(a)) m[1] += T::cy(a) > 0 ? g[a] : -g[a];
        if (L::D == 3 && T::cz(a)) m[2] += T::cz(a) > 0 ? g[a] : -g[a];
    }
    const float rho = 1.f + drho;
#pragma unroll
    const float rrho = 1.f / rho;
    for (int d = 0; d < L::D; ++d) u[d] = m[d] * rrho;
}

// centred equilibrium feq - w of detail/equilibrium_distribution.cuh:41-64:
// w rho (1 + u.c / cs^2 + (u.c)^2 / (2 cs^4) - u.u) - w
template <class L>
__device__ __forceinline__ float feq_c(int a, float drho, const float* u) {
    using T = Lat<L>;
    const float cs = cs_f();
    const float cs2 = cs * cs, cs4 = cs2 * cs2;
    float uu = u[0] * u[0] + u[1] * u[1];
    float uc = (float)T::cx(a) * u[0] + (float)T::cy(a) * u[1];
    if (L::D == 3) {
        uu += u[2] * u[2];
        uc += (float)T::cz(a) * u[2];
    }
    const float w = T::w(a);
    // 1 / cs^2 and 1 / (2 cs^4) are compile-time constants: multiplications
    // instead of 2 x 27 IEEE divisions per feq evaluation (rounding differs
    // from dividing by at most an ulp of each term)
    constexpr float r_cs2 = (float)(1.0 / ((double)0.57735026918962576451f * 0.57735026918962576451f));
    constexpr float r_2cs4 = 0.5f * r_cs2 * r_cs2;
    (void)cs4;
    return w * drho + w * (1.f + drho) * (uc * r_cs2 + (uc * uc) * r_2cs4 - uu);
}

// ------------------------------------------------------------- collision
// D3Q27 central-moment collision (detail/d3q27_lattice.cuh:125-378) on
// centred populations. Central moments K_mnp of f = w + g split into the
// weight part, a product of 1-D moments M_0 = 1, M_1 = -u, M_2 = 1/3 + u^2
// (the D3Q27 weights factorise per axis), and the g part. Every moment is
// carried as K = C + s, with C its value at u = 0 (non-zero only for the
// even moments) and s small; terms of the k formulas without a velocity
// factor use s (and rho - 1), where the reference's C contributions cancel
// exactly, all other terms use K.
__device__ __forceinline__ void mom1(int m, float u, float& a, float& x) {
    a = (m == 0) ? 1.f : (m == 1 ? 0.f : 1.f * (1.f / 3.f));
    x = (m == 0) ? 0.f : (m == 1 ? -u : u * u);
}

__device__ void collide_d3q27(const float* g, float drho, const float* u, const SceneDev& S, float* delta) {
    using T = Lat<D3Q27>;
    // central moments of g by successive 1-D transforms along x, y, z
    float Tx[3][3][3];  // [m][cy+1][cz+1]
#pragma unroll
    for (int m = 0; m < 3; ++m)
#pragma unroll
        for (int y = 0; y < 3; ++y)
#pragma unroll
            for (int z = 0; z < 3; ++z) Tx[m][y][z] = 0.f;
#pragma unroll
    for (int a = 0; a < 27; ++a) {
        const float ax = (float)T::cx(a) - u[0];
        const int y = T::cy(a) + 1, z = T::cz(a) + 1;
        Tx[0][y][z] += g[a];
        Tx[1][y][z] += g[a] * ax;
        Tx[2][y][z] += g[a] * (ax * ax);
    }
    float U[3][3][3];  // [m][n][cz+1]
#pragma unroll
    for (int m = 0; m < 3; ++m)
#pragma unroll
        for (int z = 0; z < 3; ++z) {
            float s0 = 0.f, s1 = 0.f, s2 = 0.f;
#pragma unroll
            for (int y = 0; y < 3; ++y) {
                const float ay = (float)(y - 1) - u[1];
                const float t = Tx[m][y][z];
                s0 += t;
                s1 += t * ay;
                s2 += t * (ay * ay);
            }
            U[m][0][z] = s0;
            U[m][1][z] = s1;
            U[m][2][z] = s2;
        }
    float Kg[3][3][3];
#pragma unroll
    for (int m = 0; m < 3; ++m)
#pragma unroll
        for (int n = 0; n < 3; ++n) {
            float s0 = 0.f, s1 = 0.f, s2 = 0.f;
#pragma unroll
            for (int z = 0; z < 3; ++z) {
                const float az = (float)(z - 1) - u[2];
                const float t = U[m][n][z];
                s0 += t;
                s1 += t * az;
                s2 += t * (az * az);
            }
            Kg[m][n][0] = s0;
            Kg[m][n][1] = s1;
            Kg[m][n][2] = s2;
        }
    // small parts s_mnp = (Kw(u) - C) + Kg and full values K = C + s
    float sK[3][3][3], K[3][3][3];
#pragma unroll
    for (int m = 0; m < 3; ++m)
#pragma unroll
        for (int n = 0; n < 3; ++n)
#pragma unroll
            for (int p = 0; p < 3; ++p) {
                float a0, x0, a1, x1, a2, x2;
                mom1(m, u[0], a0, x0);
                mom1(n, u[1], a1, x1);
                mom1(p, u[2], a2, x2);
                const float e = x0 * ((a1 + x1) * (a2 + x2)) + a0 * (x1 * (a2 + x2) + a1 * x2);
                sK[m][n][p] = e + Kg[m][n][p];
                K[m][n][p] = a0 * a1 * a2 + sK[m][n][p];
            }
    const float rho = 1.f + drho;
    const float v0 = u[0], v1 = u[1], v2 = u[2];
    const float v0sq = v0 * v0, v1sq = v1 * v1, v2sq = v2 * v2;
    // odd moments (C = 0): one value
    const float Kxy = K[1][1][0], Kxz = K[1][0][1], Kyz = K[0][1][1];
    const float Kxxy = K[2][1][0], Kxxz = K[2][0][1], Kxyy = K[1][2][0];
    const float Kyyz = K[0][2][1], Kxzz = K[1][0][2], Kyzz = K[0][1][2];
    const float Kxyz = K[1][1][1], Kxyzz = K[1][1][2], Kxxyz = K[2][1][1], Kxyyz = K[1][2][1];
    const float Kxxyzz = K[2][1][2], Kxyyzz = K[1][2][2], Kxxyyz = K[2][2][1];
    // even moments: full (u terms) and small (constant terms)
    const float Kxx = K[2][0][0], Kyy = K[0][2][0], Kzz = K[0][0][2];
    const float Kxxyy = K[2][2][0], Kxxzz = K[2][0][2], Kyyzz = K[0][2][2], Kxxyyzz = K[2][2][2];
    const float sxx = sK[2][0][0], syy = sK[0][2][0], szz = sK[0][0][2];
    const float sxxyy = sK[2][2][0], sxxzz = sK[2][0][2], syyzz = sK[0][2][2], sxxyyzz = sK[2][2][2];
    (void)Kxxyyzz;

    float k[27];
    k[0] = k[1] = k[2] = k[3] = 0.f;
    float om = S.om_ab;
    k[4] = om * (-Kxy * (1.f / 12.f));
    k[5] = om * (-Kxz * (1.f / 12.f));
    k[6] = om * (-Kyz * (1.f / 12.f));
    k[7] = om * (-(sxx - syy) * (1.f / 12.f));
    k[8] = om * (-(sxx + syy - 2.f * szz) * (1.f / 36.f));
    k[9] = om * (-(sxx + syy + szz - drho) * (1.f / 18.f));
    om = S.om_fix[0];
    k[10] = om * (-(6.f * Kxy * v1 + 3.f * Kxyy + 6.f * Kxz * v2 + 3.f * Kxzz + 3.f * Kyy * v0 + 3.f * Kzz * v0 -
                    2.f * rho * v0) * (1.f / 72.f));
    k[11] = om * (-(3.f * Kxx * v1 + 3.f * Kxxy + 6.f * Kxy * v0 + 6.f * Kyz * v2 + 3.f * Kyzz + 3.f * Kzz * v1 -
                    2.f * rho * v1) * (1.f / 72.f));
    k[12] = om * (-(3.f * Kxx * v2 + 3.f * Kxxz + 6.f * Kxz * v0 + 3.f * Kyy * v2 + 3.f * Kyyz + 6.f * Kyz * v1 -
                    2.f * rho * v2) * (1.f / 72.f));
    om = S.om_fix[1];
    k[13] = om * (-(2.f * Kxy * v1 + Kxyy - 2.f * Kxz * v2 - Kxzz + Kyy * v0 - Kzz * v0) / 8.f);
    k[14] = om * (-(Kxx * v1 + Kxxy + 2.f * Kxy * v0 - 2.f * Kyz * v2 - Kyzz - Kzz * v1) / 8.f);
    k[15] = om * (-(Kxx * v2 + Kxxz + 2.f * Kxz * v0 - Kyy * v2 - Kyyz - 2.f * Kyz * v1) / 8.f);
    om = S.om_fix[2];
    k[16] = om * (-(Kxy * v2 + Kxyz + Kxz * v1 + Kyz * v0) / 8.f);
    om = S.om_fix[3];
    k[17] = om * (-(3.f * Kxx * v1sq + 3.f * Kxx * v2sq - 4.f * sxx + 6.f * Kxxy * v1 + 3.f * sxxyy +
                    6.f * Kxxz * v2 + 3.f * sxxzz + 12.f * Kxy * v0 * v1 + 6.f * Kxyy * v0 +
                    12.f * Kxz * v0 * v2 + 6.f * Kxzz * v0 + 3.f * Kyy * v0sq + 3.f * Kyy * v2sq - 4.f * syy +
                    6.f * Kyyz * v2 + 3.f * syyzz + 12.f * Kyz * v1 * v2 + 6.f * Kyzz * v1 + 3.f * Kzz * v0sq +
                    3.f * Kzz * v1sq - 4.f * szz - 2.f * rho * v0sq - 2.f * rho * v1sq - 2.f * rho * v2sq +
                    3.f * drho) * (1.f / 36.f));
    om = S.om_fix[4];
    k[18] = om * (-(3.f * Kxx * v1sq + 3.f * Kxx * v2sq - 4.f * sxx + 6.f * Kxxy * v1 + 3.f * sxxyy +
                    6.f * Kxxz * v2 + 3.f * sxxzz + 12.f * Kxy * v0 * v1 + 6.f * Kxyy * v0 +
                    12.f * Kxz * v0 * v2 + 6.f * Kxzz * v0 + 3.f * Kyy * v0sq - 6.f * Kyy * v2sq + 2.f * syy -
                    12.f * Kyyz * v2 - 6.f * syyzz - 24.f * Kyz * v1 * v2 - 12.f * Kyzz * v1 + 3.f * Kzz * v0sq -
                    6.f * Kzz * v1sq + 2.f * szz - 2.f * rho * v0sq + rho * v1sq + rho * v2sq) * (1.f / 72.f));
    k[19] = om * (-(3.f * Kxx * v1sq - 3.f * Kxx * v2sq + 6.f * Kxxy * v1 + 3.f * sxxyy - 6.f * Kxxz * v2 -
                    3.f * sxxzz + 12.f * Kxy * v0 * v1 + 6.f * Kxyy * v0 - 12.f * Kxz * v0 * v2 -
                    6.f * Kxzz * v0 + 3.f * Kyy * v0sq - 2.f * syy - 3.f * Kzz * v0sq + 2.f * szz - rho * v1sq +
                    rho * v2sq) * (1.f / 24.f));
    om = S.om_fix[4];
    k[20] = om * (-(3.f * Kxx * v1 * v2 + 3.f * Kxxy * v2 + 3.f * Kxxyz + 3.f * Kxxz * v1 + 6.f * Kxy * v0 * v2 +
                    6.f * Kxyz * v0 + 6.f * Kxz * v0 * v1 + 3.f * Kyz * v0sq - 2.f * Kyz - rho * v1 * v2) * (1.f / 24.f));
    k[21] = om * (-(6.f * Kxy * v1 * v2 + 3.f * Kxyy * v2 + 3.f * Kxyyz + 6.f * Kxyz * v1 + 3.f * Kxz * v1sq -
                    2.f * Kxz + 3.f * Kyy * v0 * v2 + 3.f * Kyyz * v0 + 6.f * Kyz * v0 * v1 - rho * v0 * v2) * (1.f / 24.f));
    k[22] = om * (-(3.f * Kxy * v2sq - 2.f * Kxy + 6.f * Kxyz * v2 + 3.f * Kxyzz + 6.f * Kxz * v1 * v2 +
                    3.f * Kxzz * v1 + 6.f * Kyz * v0 * v2 + 3.f * Kyzz * v0 + 3.f * Kzz * v0 * v1 - rho * v0 * v1) /
                  24.f);
    om = S.om_fix[5];
    k[23] = om * (-(6.f * Kxy * v1 * v2sq - 4.f * Kxy * v1 + 3.f * Kxyy * v2sq - 2.f * Kxyy + 6.f * Kxyyz * v2 +
                    3.f * Kxyyzz + 12.f * Kxyz * v1 * v2 + 6.f * Kxyzz * v1 + 6.f * Kxz * v1sq * v2 -
                    4.f * Kxz * v2 + 3.f * Kxzz * v1sq - 2.f * Kxzz + 3.f * Kyy * v0 * v2sq - 2.f * Kyy * v0 +
                    6.f * K[0][2][1] * v0 * v2 + 3.f * Kyyzz * v0 + 12.f * Kyz * v0 * v1 * v2 +
                    6.f * Kyzz * v0 * v1 + 3.f * Kzz * v0 * v1sq - 2.f * Kzz * v0 - rho * v0 * v1sq -
                    rho * v0 * v2sq + rho * v0) * (1.f / 24.f));
    k[24] = om * (-(3.f * Kxx * v1 * v2sq - 2.f * Kxx * v1 + 3.f * Kxxy * v2sq - 2.f * Kxxy + 6.f * Kxxyz * v2 +
                    3.f * Kxxyzz + 6.f * Kxxz * v1 * v2 + 3.f * Kxxzz * v1 + 6.f * Kxy * v0 * v2sq -
                    4.f * Kxy * v0 + 12.f * Kxyz * v0 * v2 + 6.f * Kxyzz * v0 + 12.f * Kxz * v0 * v1 * v2 +
                    6.f * Kxzz * v0 * v1 + 6.f * Kyz * v0sq * v2 - 4.f * Kyz * v2 + 3.f * Kyzz * v0sq -
                    2.f * Kyzz + 3.f * Kzz * v0sq * v1 - 2.f * Kzz * v1 - rho * v0sq * v1 - rho * v1 * v2sq +
                    rho * v1) * (1.f / 24.f));
    k[25] = om * (-(3.f * Kxx * v1sq * v2 - 2.f * Kxx * v2 + 6.f * Kxxy * v1 * v2 + 3.f * Kxxyy * v2 +
                    3.f * Kxxyyz + 6.f * Kxxyz * v1 + 3.f * Kxxz * v1sq - 2.f * Kxxz + 12.f * Kxy * v0 * v1 * v2 +
                    6.f * Kxyy * v0 * v2 + 6.f * Kxyyz * v0 + 12.f * Kxyz * v0 * v1 + 6.f * Kxz * v0 * v1sq -
                    4.f * Kxz * v0 + 3.f * Kyy * v0sq * v2 - 2.f * Kyy * v2 + 3.f * Kyyz * v0sq - 2.f * Kyyz +
                    6.f * Kyz * v0sq * v1 - 4.f * Kyz * v1 - rho * v0sq * v2 - rho * v1sq * v2 + rho * v2) * (1.f / 24.f));
    k[26] = om * (-(27.f * Kxx * v1sq * v2sq - 18.f * Kxx * v1sq - 18.f * Kxx * v2sq + 12.f * sxx +
                    54.f * Kxxy * v1 * v2sq - 36.f * Kxxy * v1 + 27.f * Kxxyy * v2sq - 18.f * sxxyy +
                    54.f * Kxxyyz * v2 + 27.f * sxxyyzz + 108.f * Kxxyz * v1 * v2 + 54.f * Kxxyzz * v1 +
                    54.f * Kxxz * v1sq * v2 - 36.f * Kxxz * v2 + 27.f * Kxxzz * v1sq - 18.f * sxxzz +
                    108.f * Kxy * v0 * v1 * v2sq - 72.f * Kxy * v0 * v1 + 54.f * Kxyy * v0 * v2sq -
                    36.f * Kxyy * v0 + 108.f * Kxyyz * v0 * v2 + 54.f * Kxyyzz * v0 + 216.f * Kxyz * v0 * v1 * v2 +
                    108.f * Kxyzz * v0 * v1 + 108.f * Kxz * v0 * v1sq * v2 - 72.f * Kxz * v0 * v2 +
                    54.f * Kxzz * v0 * v1sq - 36.f * Kxzz * v0 + 27.f * Kyy * v0sq * v2sq - 18.f * Kyy * v0sq -
                    18.f * Kyy * v2sq + 12.f * syy + 54.f * Kyyz * v0sq * v2 - 36.f * Kyyz * v2 +
                    27.f * Kyyzz * v0sq - 18.f * syyzz + 108.f * Kyz * v0sq * v1 * v2 - 72.f * Kyz * v1 * v2 +
                    54.f * Kyzz * v0sq * v1 - 36.f * Kyzz * v1 + 27.f * Kzz * v0sq * v1sq - 18.f * Kzz * v0sq -
                    18.f * Kzz * v1sq + 12.f * szz - 9.f * rho * v0sq * v1sq - 9.f * rho * v0sq * v2sq +
                    9.f * rho * v0sq - 9.f * rho * v1sq * v2sq + 9.f * rho * v1sq + 9.f * rho * v2sq -
                    7.f * drho) * (1.f / 216.f));
    // df = K k dt (detail/simulation_engine.cuh:518-527)
#pragma unroll
    for (int l = 0; l < 27; ++l) {
        float s = 0.f;
#pragma unroll
        for (int j = 4; j < 27; ++j)
            if (T::K(l, j) != 0) s += (float)T::K(l, j) * k[j];
        delta[l] = s * S.dt_lat;
    }
}

// D2Q9 collision (detail/d2q9_lattice.cuh:120-299) with f = w + g. Terms
// without a velocity factor are written in g and rho - 1 (their w parts
// cancel exactly); u-weighted sums of f use the exact weight sums.
__device__ void collide_d2q9(const float* g, float drho, const float* u, const SceneDev& S, float* delta) {
    enum { R = 0, NW = 1, W = 2, SW = 3, Sd = 4, SE = 5, E = 6, NE = 7, N = 8 };
    const float rho = 1.f + drho;
    const float u0 = u[0], u1 = u[1];
    const float om = S.om_ab, idt = S.inv_dt;
    float k[9];
    k[0] = k[1] = k[2] = 0.f;
    k[3] = idt * (rho * (u0 * u0 + u1 * u1) - g[E] - g[N] - g[Sd] - g[W] -
                  2.f * (g[SE] + g[SW] + g[NE] + g[NW] - drho * (1.f / 3.f))) * (1.f / 12.f);
    k[4] = om * (g[N] + g[Sd] - g[E] - g[W] + rho * (u0 * u0 - u1 * u1)) / 4.f;
    k[5] = om * (g[NE] + g[SW] - g[NW] - g[SE] + rho * (u0 * u1)) / 4.f;
    {
        float t1 = (g[SE] + g[SW] - g[NE] - g[NW] - 2.f * u0 * u0 * u1 * rho +
                    u1 * (1.f * (1.f / 3.f) + (drho - g[N] - g[Sd] - g[R]))) / 4.f;
        float t2 = u0 / 2.f * (g[NE] - g[NW] - g[SE] + g[SW]);
        float t3 = -u1 / 2.f * (-3.f * k[3] - k[4]) - 2.f * u0 * k[5];
        k[6] = -idt * (t1 + t2) + t3;
    }
    {
        float t1 = (g[SW] + g[NW] - g[SE] - g[NE] - 2.f * u0 * u1 * u1 * rho +
                    u0 * (1.f * (1.f / 3.f) + (drho - g[W] - g[E] - g[R]))) / 4.f;
        float t2 = u1 / 2.f * (g[NE] + g[SW] - g[SE] - g[NW]);
        float t3 = -u0 / 2.f * (-3.f * k[3] + k[4]) - 2.f * u1 * k[5];
        k[7] = -idt * (t1 + t2) + t3;
    }
    {
        float t1 = drho * (1.f / 9.f) - g[NE] - g[NW] - g[SE] - g[SW];
        float t2 = 2.f * (u0 * (g[NE] - g[NW] + g[SE] - g[SW]) + u1 * (g[NE] + g[NW] - g[SE] - g[SW]));
        float t3 = 4.f * u0 * u1 * (g[NW] - g[NE] + g[SE] - g[SW]);
        float t4 = -u0 * u0 * (1.f * (1.f / 3.f) + (g[N] + g[NE] + g[NW] + g[Sd] + g[SE] + g[SW]));
        float t5 = u1 * u1 * (3.f * u0 * u0 * rho - (1.f * (1.f / 3.f) + (g[E] + g[NE] + g[NW] + g[SE] + g[SW] + g[W])));
        float t6 = -2.f * k[3] - 2.f * u0 * k[7] - 2.f * u1 * k[6] + 4.f * u0 * u1 * k[5] -
                   (3.f / 2.f * k[3] - k[4] / 2.f) * (u0 * u0 + u1 * u1);
        k[8] = idt * (1.f / 4.f * (t1 + t2 + t3 + t4 + t5)) + t6;
    }
    using T = Lat<D2Q9>;
#pragma unroll
    for (int l = 0; l < 9; ++l) {
        float s = 0.f;
#pragma unroll
        for (int j = 3; j < 9; ++j)
            if (T::K(l, j) != 0) s += (float)T::K(l, j) * k[j];
        delta[l] = s * S.dt_lat;
    }
}

template <class L>
__device__ __forceinline__ void collide(const float* g, float drho, const float* u, const SceneDev& S, float* delta) {
    if constexpr (L::D == 3)
        collide_d3q27(g, drho, u, S, delta);
    else
        collide_d2q9(g, drho, u, S, delta);
}

// ------------------------------------------------------------- kernels
// SceneDev of the current item into shared memory (warp 0 copies words)
// Programmatic dependent launch between the step's kernels: a kernel lets
// the next one be scheduled once all its blocks have finished their work
// (earlier, the waiting blocks of later kernels took SM slots from the
// running one), and the next kernel's blocks run their prologue -- shared-memory set-up and the first
// bulk copy of table records, which no kernel of the step writes -- before
// waiting for the previous kernel's completion and memory (griddepcontrol.
// wait) ahead of their first read of step data. Without a programmatic
// dependency (a plain launch) the wait returns at once.
__device__ __forceinline__ void pdl_allow_next() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait_prev() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

__device__ __forceinline__ void load_scene(SceneDev& dst, const SceneDev* src) {
    if (threadIdx.x < 32) {
        const int* a = reinterpret_cast<const int*>(src);
        int* b = reinterpret_cast<int*>(&dst);
        for (int t = threadIdx.x; t < (int)(sizeof(SceneDev) / 4); t += 32) b[t] = a[t];
    }
}

#define NAGA_FOR_ITEMS(items, nitems)                           \
    __shared__ SceneDev S;                                      \
    pdl_wait_prev();                                            \
    for (int w_ = blockIdx.x; w_ < (nitems); w_ += gridDim.x) { \
        const WorkItem it = (items)[w_];                        \
        __syncthreads();                                        \
        load_scene(S, scenes + it.scene);                       \
        __syncthreads();

#define NAGA_END_ITEMS \
    }                      \
    pdl_allow_next();

// Node-local part of the step, one thread per node (all nodes):
// rho, u (stored for the probes and the next step); the PML trapezoid
// integrals Q1 = (f~ + f~_prev) dt / 2, Q2 = (Q1 + Q1_prev) dt / 2 with
// f~ = feq - w (pml_absorption.inl:531-631); the local absorption term
// -sigma (3 f~ + 3 sigma Q1 + sigma^2 Q2) on layer nodes; the collision
// increment K k dt (simulation_engine.cuh:469-531). Writes
//   bulk/layer: S1 = g + local + collision, and S1P = g + local on nodes the
//               boundary interpolation reads;
//   boundary:   S1 = collision (the interpolated part is added later);
//   ghost:      S1 = g + collision.
// The item's rows of G and Q1_prev are staged in shared memory by coalesced
// loads of the whole block before the (register-heavy) per-node work.
// D3Q27 runs 4 blocks/SM (its collision needs the registers; tighter bounds
// spill and were slower); D2Q9 fits 8 (one resident wave of the item grid;
// at 7, 72 registers without spills, the 256-scene batch's kernel took 0.45
// ms against 0.34)
template <class L>
__global__ void __launch_bounds__(kBlock, (L::D == 3 ? 4 : 8)) k_macro_pml(const WorkItem* __restrict__ items, int nitems,
                                                         const SceneDev* __restrict__ scenes) {
    constexpr int Q = L::Q, QP = L::QP;
    // rows of the item's nodes: G and Q1_prev in, then the layer terms
    // (Q1, Q2 of layer nodes, zero elsewhere) for the item's column sums
    __shared__ float4 rowG[kBlock * QP / 4], rowQ[kBlock * QP / 4];
    __shared__ double red[2][2 * QP];
    NAGA_FOR_ITEMS(items, nitems)
    const unsigned long long step = *S.step;
    const int par = (int)(step & 1ull);
    float* Q1cur = par ? S.Q1b : S.Q1a;
    const float* Q1prev = par ? S.Q1a : S.Q1b;
    const int nn = (int)(it.end - it.begin);
    const int64_t i = (int64_t)it.begin + threadIdx.x;
    const bool active = (int)threadIdx.x < nn;
    const bool layer = active && i >= S.nb && i < S.nb + S.nl;
    // node i carries NAGA's PML field of layer node i + pml_shift
    const int64_t jf = i + S.pml_shift;
    const bool field = active && jf >= S.nb && jf < S.nb + S.nl;
    // per-node inputs issued before the row staging so their latency overlaps it
    const float4 mp = active ? S.M[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    const float sg = layer ? __ldg(S.sigma + (i - S.nb)) : 0.f;
    const float sf = field ? __ldg(S.sigma + (jf - S.nb)) : 0.f;
    const bool src = active && i < S.nbl && S.is_src[i];
    {
        // copied with cp.async (16 B a thread and copy, no register staging),
        // all of the thread's copies in flight at once
        const float4* g4 = reinterpret_cast<const float4*>(S.G + (int64_t)it.begin * QP);
        const float4* q4 = reinterpret_cast<const float4*>(Q1prev + (int64_t)it.begin * QP);
        constexpr int NQ = QP / 4;  // float4 per row: the block moves kBlock * NQ of each
        const int ne = nn * NQ;
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            const int e = (int)threadIdx.x + q * kBlock;
            if (e < ne) {
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(
                                 (uint32_t)__cvta_generic_to_shared(rowG + e)),
                             "l"(g4 + e)
                             : "memory");
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(
                                 (uint32_t)__cvta_generic_to_shared(rowQ + e)),
                             "l"(q4 + e)
                             : "memory");
            }
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
        asm volatile("cp.async.wait_group 0;" ::: "memory");
    }
    __syncthreads();
    float* myG = reinterpret_cast<float*>(rowG) + threadIdx.x * QP;
    float* myQ = reinterpret_cast<float*>(rowQ) + threadIdx.x * QP;
    if (active) {
        float g[Q];
#pragma unroll
        for (int a = 0; a < Q; ++a) g[a] = myG[L::pos(a)];
        float drho, u[3] = {0.f, 0.f, 0.f};
        macros<L>(g, drho, u);
        // density source of this step (after the probes sampled the macros):
        // f_a += (s / rho0) w_a, and the reference's density statement
        // rho <- (rho + (rho + s)) / 2 applied once, u unchanged
        // (detail/simulation_engine.cuh:1057-1107 without its race)
        if (S.src_slot) {
            const int sl = S.src_slot[i];
            const int64_t row = (int64_t)step - S.src_first;
            if (sl >= 0 && row >= 0 && row < S.src_steps) {
                const float sv = S.src_vals[row * S.src_n + sl];
                if (sv != FLT_MAX) {
                    const float ds = sv / S.rho0;
#pragma unroll
                    for (int a = 0; a < Q; ++a) g[a] = fmaf(ds, LatticeTables<L>::w(a), g[a]);
                    drho += 0.5f * ds;
                }
            }
        }
        const float up[3] = {mp.y, mp.z, mp.w};
        S.M[i] = make_float4(drho, u[0], u[1], L::D == 3 ? u[2] : 0.f);
        float dcol[Q];
        collide<L>(g, drho, u, S, dcol);
        float q1[QP], out[QP], phi[QP];
#pragma unroll
        for (int t = 0; t < QP; ++t) q1[t] = out[t] = phi[t] = 0.f;
#pragma unroll
        for (int a = 0; a < Q; ++a) {
            const int t = L::pos(a);
            const float ft = feq_c<L>(a, drho, u);
            const float ftp = feq_c<L>(a, mp.x, up);
            q1[t] = (ft + ftp) * S.dt_lat / 2.f;
            const float q2 = (q1[t] + myQ[t]) * S.dt_lat / 2.f;
            phi[t] = -2.f * sf * q1[t] + sf * sf * q2;
            myG[t] = layer ? q1[t] : 0.f;
            myQ[t] = layer ? q2 : 0.f;
            out[t] = layer ? g[a] - sg * (3.f * ft + 3.f * sg * q1[t] + sg * sg * q2) : g[a];
        }
        store_row<L>(Q1cur, i, q1);
        if (field) {
            // the field row holds the gathered chunks (L::QS floats)
            float4* pr = reinterpret_cast<float4*>(S.PHI + (jf - S.nb) * L::QS);
#pragma unroll
            for (int c = 0; c < L::QS / 4; ++c)
                pr[c] = make_float4(phi[4 * c], phi[4 * c + 1], phi[4 * c + 2], phi[4 * c + 3]);
        }
        if (src) s1_store_row<L>(S.S1P, S.N, i, out);
        const bool boundary = i >= S.nbl && i < S.nbl + S.nbd;
#pragma unroll
        for (int a = 0; a < Q; ++a) {
            const int t = L::pos(a);
            out[t] = boundary ? dcol[a] : out[t] + dcol[a];
        }
        s1_store_row<L>(S.S1, S.N, i, out);
    } else {
#pragma unroll
        for (int t = 0; t < QP; ++t) myG[t] = myQ[t] = 0.f;
    }
    // per-item layer sums of Q1 and Q2 in FP64, fixed order: column t of
    // the rows, two halves of the item summed in node order, then added
    const bool touches = (int64_t)it.end > S.nb && (int64_t)it.begin < S.nb + S.nl;
    __syncthreads();
    if (touches && threadIdx.x < 4 * QP) {
        const int col = threadIdx.x % (2 * QP), half = threadIdx.x / (2 * QP);
        const float* base = col < QP ? reinterpret_cast<const float*>(rowG) : reinterpret_cast<const float*>(rowQ);
        const int t = col < QP ? col : col - QP;
        const int r0 = half * (kBlock / 2), r1 = min(nn, r0 + kBlock / 2);
        double v = 0.0;
        for (int r = r0; r < r1; ++r) v += (double)base[r * QP + t];
        red[half][col] = v;
    }
    __syncthreads();
    if (threadIdx.x < 2 * QP)
        S.partials[(int64_t)threadIdx.x * S.n_all_items + it.local] =
            touches ? red[0][threadIdx.x] + red[1][threadIdx.x] : 0.0;
    NAGA_END_ITEMS
}

// Per-scene tail of the node-local pass, one launch for all scenes:
// blocks (scene, t < 2 QP) reduce the layer means of Q1 and Q2 (the
// reductions of pml_absorption.inl:776-836; item partials summed in item
// order strided over the block, then a fixed tree); block (scene, 2 QP)
// samples the probe densities rho - rho0 from the RPIM probe weights
// (simulation_observers/density_observer.cuh:99-113) into the ring slot of
// the current step and then advances the scene's step counter (no later
// kernel of the step reads it).
template <int QP>
__global__ void __launch_bounds__(256) k_scene_tail(const SceneDev* __restrict__ scenes) {
    __shared__ double red[256];
    pdl_wait_prev();
    const SceneDev& S = scenes[blockIdx.x];
    const int t = blockIdx.y;
    if (t < 2 * QP) {
        // the thread's partials in item order, loads issued eight at a time
        // ahead of their adds (same order of additions); column t is
        // contiguous, so the block's loads are coalesced
        double acc = 0.0;
        const double* col = S.partials + (int64_t)t * S.n_all_items;
        const int bs = (int)blockDim.x;
        int it = threadIdx.x;
        for (; it + 7 * bs < S.n_all_items; it += 8 * bs) {
            double v[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) v[u] = col[it + u * bs];
#pragma unroll
            for (int u = 0; u < 8; ++u) acc += v[u];
        }
        for (; it < S.n_all_items; it += bs) acc += col[it];
        red[threadIdx.x] = acc;
        __syncthreads();
        for (int o = blockDim.x / 2; o >= 32; o >>= 1) {
            if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
            __syncthreads();
        }
        // the last five levels of the same tree in warp 0 (lane l < o adds
        // lane l + o, as the shared-memory levels do)
        if (threadIdx.x < 32) {
            double v = red[threadIdx.x];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(kFull, v, o);
            if (threadIdx.x == 0) S.means[t] = S.nl > 0 ? (float)v / (float)S.nl : 0.f;
        }
        return;
    }
    const unsigned long long step = *S.step;
    const int slot = (int)(step % (unsigned long long)S.probe_cap);
    for (int p = threadIdx.x >> 5; p < S.np; p += blockDim.x >> 5) {
        float v = 0.f;
        for (int s = lane_id(); s < S.kp; s += 32) {
            const uint32_t j = S.pidx[(int64_t)s * S.np + p];
            float dr = S.M[j].x;
            // the probes see the density before this step's source term
            if (S.src_slot) {
                const int sl = S.src_slot[j];
                const int64_t row = (int64_t)step - S.src_first;
                if (sl >= 0 && row >= 0 && row < S.src_steps) {
                    const float sv = S.src_vals[row * S.src_n + sl];
                    if (sv != FLT_MAX) dr -= 0.5f * (sv / S.rho0);
                }
            }
            v += S.pw[(int64_t)s * S.np + p] * dr;
        }
        v = warp_sum(v);
        if (lane_id() == 0) S.probe_ring[(int64_t)slot * S.np + p] = v * S.rho0;
    }
    __syncthreads();
    if (threadIdx.x == 0) *S.step = step + 1ull;
}

// Multi-thread-per-node kernels: one work item = one pass of <= NPB
// consecutive nodes; thread c of node slot ns owns float4 chunk c of node
// i = begin + ns. The pass's table records (one contiguous block, see
// scene_dev.hpp) are double-buffered in shared memory: while the block
// gathers for item w, one thread has already started the bulk copy
// (cp.async.bulk, completion on an mbarrier) of item w + gridDim.x's
// records, so the neighbour loop waits only on the neighbour rows. Inside a
// tile, record (s, ns) sits at s * nn + ns: a warp's four (eight) nodes read
// consecutive records, free of bank conflicts.
struct TileSrc {
    const void* p;
    uint32_t bytes;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// one bulk copy global -> shared, completing on `bar` (16-byte aligned
// addresses, size a multiple of 16: checked by the caller)
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// bounded wait for the phase of `bar` with the given parity; false if the
// copy did not complete within `polls` polls. A failed poll suspends the
// thread for a hardware-defined time (about 4 us measured on B200 when
// nothing completes the phase), so the step kernels' kTileWaitPolls give up
// after about a second; naga_selftest_wait_timeout runs this same wait and
// the tests time it. A clock-checked variant cost the gather kernels ~3 %.
constexpr int kTileWaitPolls = 1 << 18;
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int polls = kTileWaitPolls) {
    for (int it = 0; it < polls; ++it) {
        uint32_t ok;
        asm volatile(
            "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
            : "=r"(ok)
            : "r"(smem_u32(bar)), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

// a plain arrive (release) on a count-1 barrier: completes its phase
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

}  // namespace

// set (never cleared by the kernels) when a tile wait ran out: the step
// kernels then return early and the host reports NAGA_ETIMEOUT
__device__ unsigned int g_tile_timeout;

namespace {

template <class T>
__device__ __forceinline__ void copy_tile(T* tile, TileSrc src) {
    const T* g = static_cast<const T*>(src.p);
    const int count = (int)(src.bytes / sizeof(T));
    for (int e = threadIdx.x; e < count; e += blockDim.x) tile[e] = __ldg(g + e);
}

// two tile buffers of CAP records: static shared memory for the unrolled
// stencil sizes, dynamic shared memory for any other size
template <class T, int CAP>
__device__ __forceinline__ T* static_tiles() {
    __shared__ __align__(128) T t[2 * CAP];
    return t;
}
template <class T>
__device__ __forceinline__ T* dynamic_tiles() {
    extern __shared__ __align__(128) unsigned char dyn_smem[];
    return reinterpret_cast<T*>(dyn_smem);
}
template <class T, int NPB, int K>
__device__ __forceinline__ T* tile_pair() {
    if constexpr (K > 0)
        return static_tiles<T, NPB * K>();
    else
        return dynamic_tiles<T>();
}
// records per tile buffer (the generic kernels take stencils of up to 64)
template <int NPB, int K>
constexpr int tile_cap() {
    return NPB * (K > 0 ? K : 64);
}

// Item loop of the gather kernels. SRC(scene, item) names the item's table
// block (TileSrc); inside the loop, `S` is the item's scene, `it` the item
// and `tile` its records. One block barrier an item: right after it, the
// next item's table block (bulk copy) and scene (shared slot) go into the
// previous item's buffers, and every thread waits for that block at the end
// of the current item, so the next barrier also checks the waits. An item
// whose table block cannot be bulk-copied (empty, or larger than a tile
// buffer) completes its buffer's phase with a plain arrive, which also
// publishes the block's mode; the block then copies what fits of it after
// the barrier.
#define NAGA_PIPE_BEGIN(T, CAP, SRC)                                                                   \
    __shared__ SceneDev pipe_S_[2];                                                                    \
    __shared__ __align__(8) uint64_t pipe_bar_[2];                                                     \
    __shared__ int pipe_mode_[2]; /* 0 bulk-copied, 1 copied after the barrier, 2 empty */             \
    T* const pipe_buf_ = tile_pair<T, G::NPB, K_>();                                                   \
    if (threadIdx.x == 0) {                                                                            \
        mbar_init(&pipe_bar_[0]);                                                                      \
        mbar_init(&pipe_bar_[1]);                                                                      \
        mbar_init_fence();                                                                             \
    }                                                                                                  \
    __syncthreads();                                                                                   \
    auto pipe_issue_ = [&](const WorkItem& itn, int b) {                                               \
        const TileSrc ts = SRC(scenes[itn.scene], itn);                                                \
        const bool bulk = ts.bytes > 0 && ts.bytes % 16 == 0 && ((uintptr_t)ts.p & 15) == 0 &&         \
                          ts.bytes <= (uint32_t)(CAP * sizeof(T));                                     \
        pipe_mode_[b] = bulk ? 0 : (ts.bytes > 0 ? 1 : 2);                                             \
        if (bulk)                                                                                      \
            bulk_load(pipe_buf_ + b * (CAP), ts.p, ts.bytes, &pipe_bar_[b]);                           \
        else                                                                                           \
            mbar_arrive(&pipe_bar_[b]);                                                                \
    };                                                                                                 \
    uint32_t pipe_par_ = 0;                                                                            \
    bool pipe_ok_ = true;                                                                              \
    auto pipe_wait_ = [&](int b) {                                                                     \
        if (!pipe_ok_) return;                                                                         \
        pipe_ok_ = mbar_wait(&pipe_bar_[b], (pipe_par_ >> b) & 1u);                                    \
        if (pipe_ok_) pipe_par_ ^= 1u << b;                                                            \
    };                                                                                                 \
    WorkItem pipe_it_ = (int)blockIdx.x < nitems ? items[blockIdx.x] : WorkItem{0u, 0u, 0u, 0u};       \
    if ((int)blockIdx.x < nitems) {                                                                    \
        if (threadIdx.x == 0) pipe_issue_(pipe_it_, 0);                                                \
        load_scene(pipe_S_[0], scenes + pipe_it_.scene);                                               \
    }                                                                                                  \
    pdl_wait_prev();                                                                                   \
    if ((int)blockIdx.x < nitems) pipe_wait_(0);                                                       \
    int pipe_t_ = 0;                                                                                   \
    for (int w_ = blockIdx.x; w_ < nitems; w_ += gridDim.x, ++pipe_t_) {                               \
        const int b_ = pipe_t_ & 1;                                                                    \
        const WorkItem it = pipe_it_;                                                                  \
        const bool more_ = w_ + (int)gridDim.x < nitems;                                               \
        if (__syncthreads_or(!pipe_ok_)) {                                                             \
            if (threadIdx.x == 0) {                                                                    \
                atomicOr(&g_tile_timeout, 1u);                                                         \
                mbar_wait(&pipe_bar_[b_], (pipe_par_ >> b_) & 1u); /* the copy still in flight */      \
            }                                                                                          \
            return;                                                                                    \
        }                                                                                              \
        if (more_) {                                                                                   \
            pipe_it_ = items[w_ + gridDim.x];                                                          \
            if (threadIdx.x == 0) pipe_issue_(pipe_it_, b_ ^ 1);                                       \
            load_scene(pipe_S_[b_ ^ 1], scenes + pipe_it_.scene);                                      \
        }                                                                                              \
        const SceneDev& S = pipe_S_[b_];                                                               \
        T* const tile = pipe_buf_ + b_ * (CAP);                                                        \
        if (pipe_mode_[b_] == 1) {                                                                     \
            TileSrc ts_ = SRC(S, it);                                                                  \
            if (ts_.bytes > (uint32_t)((CAP) * sizeof(T))) ts_.bytes = (uint32_t)((CAP) * sizeof(T));  \
            copy_tile(tile, ts_);                                                                      \
            __syncthreads();                                                                           \
        }                                                                                              \
        {

#define NAGA_PIPE_END                   \
        }                               \
        if (more_) pipe_wait_(b_ ^ 1);  \
    }                                   \
    pdl_allow_next();

// table blocks of the gather kernels
struct StencilSrc {  // divergence stencil (Wx, Wy, Wz | filter weight, index)
    __device__ TileSrc operator()(const SceneDev& sc, const WorkItem& w) const {
        const int k = sc.k;
        return {sc.stW + (int64_t)w.begin * k, (uint32_t)((w.end - w.begin) * k * sizeof(float4))};
    }
};
struct CompactSrc {  // D2Q9 stencil triplets (Wx, Wy, index)
    __device__ TileSrc operator()(const SceneDev& sc, const WorkItem& w) const {
        const int k = sc.k;
        return {sc.stR + (int64_t)w.begin * k * 3, (uint32_t)((w.end - w.begin) * k * 3 * sizeof(float))};
    }
};
struct PmlSrc {  // PML gather records (see pml_table_kernel): the first
                 // w.local (the item's largest layer-support count) per node
    __device__ TileSrc operator()(const SceneDev& sc, const WorkItem& w) const {
        const int k = sc.k;
        const uint32_t kl = w.local < (uint32_t)k ? w.local : (uint32_t)k;
        return {sc.stP + (int64_t)w.begin * k, (uint32_t)((w.end - w.begin) * kl * sizeof(float4))};
    }
};
struct FilterSrc {  // filter records of the item's bulk/layer nodes
    __device__ TileSrc operator()(const SceneDev& sc, const WorkItem& w) const {
        const int k = sc.k;
        const int64_t nf = (int64_t)w.begin < sc.nbl ? (int64_t)w.end - w.begin : 0;
        return {sc.stF + (int64_t)w.begin * k, (uint32_t)(nf * k * sizeof(float2))};
    }
};
struct EdgeSrc {  // boundary interpolation records
    __device__ TileSrc operator()(const SceneDev& sc, const WorkItem& w) const {
        const int kb = sc.kb;
        return {sc.btab + ((int64_t)w.begin - sc.nbl) * kb, (uint32_t)((w.end - w.begin) * kb * sizeof(float2))};
    }
};

// The RK stage gather of a thread's chunk, sum_s over the stencil of
// ((d0 . W_s) v.x, -(d0 . W_s) v.y, (d1 . W_s) v.z, -(d1 . W_s) v.w) for the
// chunk's two opposite pairs (d0, -d0), (d1, -d1), records (Wx, Wy, Wz | -)
// and neighbour values v. The sums run as two packed FP32 pairs (one
// fma.rn.f32x2 each per term): (sum p0 v.x, sum p0 v.y) and (sum p1 v.z,
// sum p1 v.w), the second of each pair negated at the end -- the same
// rounding as accumulating -p0 v.y term by term. Shared by every RK stage
// kernel so that all of them round alike.
struct RkAcc {
    float2 xy = make_float2(0.f, 0.f), zw = make_float2(0.f, 0.f);
    __device__ __forceinline__ float4 rate_sum() const { return make_float4(xy.x, -xy.y, zw.x, -zw.y); }
};
template <class L>
__device__ __forceinline__ void rk_term(const float4& rec, const float* d0, const float* d1, const float4& v,
                                        RkAcc& r) {
    const float wz = L::D == 3 ? rec.z : 0.f;
    const float p0 = d0[0] * rec.x + d0[1] * rec.y + d0[2] * wz;
    const float p1 = d1[0] * rec.x + d1[1] * rec.y + d1[2] * wz;
    r.xy = __ffma2_rn(make_float2(p0, p0), make_float2(v.x, v.y), r.xy);
    r.zw = __ffma2_rn(make_float2(p1, p1), make_float2(v.z, v.w), r.zw);
}

// PML divergence gathers of pml_absorption.inl:770-855 on bulk/layer nodes
// whose stencils reach into the layer. NAGA adds div(-2 c sigma (Q1 - <Q1>))
// + div(c sigma^2 (Q2 - <Q2>)), with sigma of the support node j and Q read
// at node j - pml_shift (its field maps index Q by the layer position,
// pml_absorption.inl:438-448). By linearity this is
//   sum_s (c . W_s) phi_j  +  c . (2 <Q1> V1 - <Q2> V2),
// phi_j = -2 sigma_j Q1 + sigma_j^2 Q2 (one row per layer node, written by
// the macro kernel) and V1 = sum_s W_s sigma_j, V2 = sum_s W_s sigma_j^2
// over the node's layer supports (set-up). Adds to S1 and, on
// interpolation sources, S1P.
template <class L, int K>
__global__ void __launch_bounds__(MTR<L>::BLOCK) k_pml_gather(const WorkItem* __restrict__ items, int nitems,
                                                              const SceneDev* __restrict__ scenes) {
    using G = MTR<L>;  // like the RK stages: only the L::NGATHER chunks carry a term
    constexpr int QP = L::QP, K_ = K;
    const int c = threadIdx.x % G::TPN, ns = threadIdx.x / G::TPN;
    float d0[3], d1[3];
    pair_dirs<L>(c < G::NCH ? c : 0, d0, d1);
    NAGA_PIPE_BEGIN(float4, (tile_cap<G::NPB, K>()), PmlSrc{})
    const int k = K > 0 ? K : S.k;
    const int nn = (int)(it.end - it.begin);
    const int64_t i = (int64_t)it.begin + ns;
    // chunks past NGATHER carry no direction (their term is zero)
    if (ns < nn && c < L::NGATHER) {
        float4 dv = make_float4(0.f, 0.f, 0.f, 0.f);
        // the node's layer supports lead its records (in stencil order), their
        // count riding in V1.w, then zero-weight records on a valid row.
        // D3Q27 runs each node over its own supports; D2Q9 runs every node of
        // the pass to the pass's largest count (the tile's records per node,
        // it.local) so that its warps (16 nodes) do not diverge -- the zero
        // terms leave the sums unchanged (256-scene batch: 0.245 -> 0.214 ms;
        // in D3Q27, 4 nodes a warp, the extra row loads cost more: 70 -> 89 us)
        const float4 v1 = __ldg(S.PV + 2 * i), v2 = __ldg(S.PV + 2 * i + 1);
        const int kn = min(L::D == 2 ? (int)it.local : (int)__float_as_uint(v1.w), k);
#pragma unroll 8
        for (int s = 0; s < kn; ++s) {
            const float4 rec = tile[s * nn + ns];
            const uint32_t jl = __float_as_uint(rec.w);
            const float wz = L::D == 3 ? rec.z : 0.f;
            const float4 v = ld4s<L>(S.PHI, jl, c);
            const float p0 = d0[0] * rec.x + d0[1] * rec.y + d0[2] * wz;
            const float p1 = d1[0] * rec.x + d1[1] * rec.y + d1[2] * wz;
            dv.x = fmaf(p0, v.x, dv.x);
            dv.y = fmaf(-p0, v.y, dv.y);
            dv.z = fmaf(p1, v.z, dv.z);
            dv.w = fmaf(-p1, v.w, dv.w);
        }
        const float4 m1 = *reinterpret_cast<const float4*>(S.means + 4 * c);
        const float4 m2 = *reinterpret_cast<const float4*>(S.means + QP + 4 * c);
        const float e1 = d0[0] * v1.x + d0[1] * v1.y + d0[2] * v1.z;
        const float e2 = d0[0] * v2.x + d0[1] * v2.y + d0[2] * v2.z;
        const float f1 = d1[0] * v1.x + d1[1] * v1.y + d1[2] * v1.z;
        const float f2 = d1[0] * v2.x + d1[1] * v2.y + d1[2] * v2.z;
        dv.x += 2.f * m1.x * e1 - m2.x * e2;
        dv.y -= 2.f * m1.y * e1 - m2.y * e2;
        dv.z += 2.f * m1.z * f1 - m2.z * f2;
        dv.w -= 2.f * m1.w * f1 - m2.w * f2;
        const float4 o = s1_ld<L>(S.S1, S.N, i, c);
        s1_st<L>(S.S1, S.N, i, c, make_float4(o.x + dv.x, o.y + dv.y, o.z + dv.z, o.w + dv.w));
        if (S.is_src[i]) {
            const float4 q = s1_ld<L>(S.S1P, S.N, i, c);
            s1_st<L>(S.S1P, S.N, i, c, make_float4(q.x + dv.x, q.y + dv.y, q.z + dv.z, q.w + dv.w));
        }
    }
    NAGA_PIPE_END
}

// boundary: s1 = interp(s1 of bulk + layer, before collision) + collision
// (simulation_engine.cuh:434-467 then :469-531); S1 holds the collision
// sum_s w_s row_s[c] over the kb records (weight, index) of node slot ns:
// loads issued 16 at a time before their products, so one item's gather
// (these kernels run about one item per block) waits on two batches of
// loads, not kb dependent steps. The boundary kernels' launch bound of 5
// blocks/SM leaves registers for the batch while every boundary item of
// the benchmark scene stays resident in one wave (measured: 17.4 -> 13.8
// and 15.4 -> 13.5 us; a bound of 2 allows 117 registers but needs three
// waves)
// (S1ROWS: rows in the collision scratch layout, see s1_ld; else rows of
// QP floats)
template <class L, int KB, bool S1ROWS>
__device__ __forceinline__ float4 edge_sum(const float2* tile, int kb, int nn, int ns, const float* rows, int64_t n,
                                           int c) {
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
    constexpr int B = 16;
    for (int s0 = 0; s0 < kb; s0 += B) {
        float4 v[B];
        float w[B];
#pragma unroll
        for (int u = 0; u < B; ++u) {
            if (KB > 0 || s0 + u < kb) {
                const float2 r = tile[(s0 + u) * nn + ns];
                w[u] = r.x;
                v[u] = S1ROWS ? s1_ldg<L>(rows, n, __float_as_uint(r.y), c) : ld4g<L>(rows, __float_as_uint(r.y), c);
            }
        }
#pragma unroll
        for (int u = 0; u < B; ++u) {
            if (KB > 0 || s0 + u < kb) {
                acc.x = fmaf(w[u], v[u].x, acc.x);
                acc.y = fmaf(w[u], v[u].y, acc.y);
                acc.z = fmaf(w[u], v[u].z, acc.z);
                acc.w = fmaf(w[u], v[u].w, acc.w);
            }
        }
    }
    return acc;
}

template <class L, int KB>
__global__ void __launch_bounds__(MTF<L>::BLOCK, 5) k_edge_collide(const WorkItem* __restrict__ items, int nitems,
                                                           const SceneDev* __restrict__ scenes) {
    using G = MTF<L>;
    constexpr int QP = L::QP, K_ = KB;
    const int c = threadIdx.x % G::TPN, ns = threadIdx.x / G::TPN;
    NAGA_PIPE_BEGIN(float2, (tile_cap<G::NPB, KB>()), EdgeSrc{})
    const int kb = KB > 0 ? KB : S.kb;
    const int nn = (int)(it.end - it.begin);
    const int64_t i = (int64_t)it.begin + ns;
    if (ns < nn && c < G::NCH) {
        const float4 acc = edge_sum<L, KB, true>(tile, kb, nn, ns, S.S1P, S.N, c);
        const float4 d = s1_ld<L>(S.S1, S.N, i, c);
        s1_st<L>(S.S1, S.N, i, c, make_float4(acc.x + d.x, acc.y + d.y, acc.z + d.z, acc.w + d.w));
    }
    NAGA_PIPE_END
}

// bulk + layer: f = s1 + 0.75 sum_s w_s (s1_s - s1) (simulation_engine.cuh:
// 1233-1323); boundary: bounce-back f_a <- f_bb(a) where c_a . n > 0
// (:789-944), a swap within each opposite pair; ghost: copy
// DRY (the launch-shape tuner's trials): the same gathers and arithmetic,
// the result written into the interpolation-source scratch S1P (dead between
// steps: the next step's node-local kernel rewrites it) instead of the state.
// Launch bounds: D3Q27 6 blocks/SM (40 registers; at 4, 64 registers, 68 ->
// 70 us); D2Q9 8 (64 registers instead of 40 at 12, so a thread keeps more
// gather loads in flight at the 7 blocks/SM the tuner runs it at: 256-scene
// batch filter 0.61 -> 0.48 ms)
template <class L, int K, bool DRY = false>
__global__ void __launch_bounds__(MTFF<L>::BLOCK, (L::D == 3 ? 6 : 8)) k_filter(const WorkItem* __restrict__ items, int nitems,
                                                           const SceneDev* __restrict__ scenes) {
    using G = MTFF<L>;
    // D2Q9: slot of the rest population (chunk NGATHER, first float)
    constexpr int REST = 4 * L::NGATHER;
    constexpr int QP = L::QP, K_ = K;
    // (weight, index) filter records, 8 B each
    using T = float2;
    using Src = FilterSrc;
    const int c = threadIdx.x % G::TPN, ns = threadIdx.x / G::TPN;
    float d0[3], d1[3];
    pair_dirs<L>(c < G::NCH ? c : 0, d0, d1);
    NAGA_PIPE_BEGIN(T, (tile_cap<G::NPB, K>()), Src{})
    const int k = K > 0 ? K : S.k;
    const int nn = (int)(it.end - it.begin);
    const int64_t i = (int64_t)it.begin + ns;
    if (ns < nn && c < G::NCH) {
        const float4 f = s1_ld<L>(S.S1, S.N, i, c);
        // D2Q9 thread 0 also carries the rest population (s1_ld's chunk 2)
        const bool rest = L::D == 2 && c == 0;
        const float fr = rest ? s1_ld<L>(S.S1, S.N, i, L::NGATHER).x : 0.f;
        float outr = fr;
        float4 out;
        if (i < S.nbl) {
            float4 sum = make_float4(0.f, 0.f, 0.f, 0.f);
            float sumr = 0.f;
#pragma unroll 8
            for (int s = 0; s < k; ++s) {
                const float2 r = tile[s * nn + ns];
                const uint32_t j = __float_as_uint(r.y);
                const float4 v = s1_ldg<L>(S.S1, S.N, j, c);
                sum.x = fmaf(r.x, v.x - f.x, sum.x);
                sum.y = fmaf(r.x, v.y - f.y, sum.y);
                sum.z = fmaf(r.x, v.z - f.z, sum.z);
                sum.w = fmaf(r.x, v.w - f.w, sum.w);
                if (rest) sumr = fmaf(r.x, s1_ldg<L>(S.S1, S.N, j, L::NGATHER).x - fr, sumr);
            }
            out = make_float4(fmaf(0.75f, sum.x, f.x), fmaf(0.75f, sum.y, f.y), fmaf(0.75f, sum.z, f.z),
                              fmaf(0.75f, sum.w, f.w));
            outr = fmaf(0.75f, sumr, fr);
        } else if (i - S.nbl < S.nbd) {
            const int64_t b = i - S.nbl;
            float n[3] = {0.f, 0.f, 0.f};
#pragma unroll
            for (int d = 0; d < L::D; ++d) n[d] = __ldg(S.normals + b * L::D + d);
            const float cn0 = d0[0] * n[0] + d0[1] * n[1] + d0[2] * n[2];
            const float cn1 = d1[0] * n[0] + d1[1] * n[1] + d1[2] * n[2];
            // element 2m carries direction d_m, element 2m+1 carries -d_m
            out.x = cn0 > 0.f ? f.y : f.x;
            out.y = -cn0 > 0.f ? f.x : f.y;
            out.z = cn1 > 0.f ? f.w : f.z;
            out.w = -cn1 > 0.f ? f.z : f.w;
        } else {
            out = f;
        }
        float* const Gout = DRY ? S.S1P : S.G;
        st4(Gout, i, QP, c, out);
        // the rest population: filtered on bulk and layer nodes, kept on
        // boundary (zero velocity: no bounce-back partner) and ghost nodes;
        // the row's pads stay zero
        if (rest) Gout[i * QP + REST] = outr;
        if constexpr (DRY) {
        } else if constexpr (L::D == 2) {
            // the gathered chunks of every row also go to G2, the compact
            // (32-B) rows RK stage 1 gathers from; boundary and ghost rows
            // keep their values through the stages, so G1 carries them too
            if (c < L::NGATHER) {
                st4(S.G2, i, L::QS, c, out);
                if (i >= S.nbl) st4(S.G1, i, L::QS, c, out);
            }
        } else if (i >= S.nbl) {
            // boundary and ghost rows keep their values through the RK
            // stages: the stage buffers carry them so the gathers read
            // every support from one array
            st4(S.G1, i, L::QS, c, out);
            st4(S.G2, i, L::QS, c, out);
        }
    }
    NAGA_PIPE_END
}

// RK4 stage STAGE (detail/rk4_solver.cuh:48-171) with the streaming rates
// rate_a(i) = -sum_s (c_a . W_s) g_a(j_s) (pde_right_hand_side.cuh:82-176,
// divergence.cuh:377-488). The rates are linear in g and independent of t
// (the right-hand side's field map is f - w; its finalize does nothing), so
// NAGA's classic RK4 -- k1 = A g, k2 = A(g + dt/2 k1), k3 = A(g + dt/2 k2),
// k4 = A(g + dt k3), g' = g + dt/6 (k1 + 2 k2 + 2 k3 + k4) -- is the
// polynomial g' = (1 + hA + (hA)^2/2 + (hA)^3/6 + (hA)^4/24) g, evaluated
// here in Horner form g' = g + hA(g + h/2 A(g + h/3 A(g + h/4 A g))): the
// same four gathers without the df/dt accumulator array (equal up to FP32
// rounding). Boundary and ghost nodes keep zero rates, so
// their stage values equal the step's start values, which the filter kernel
// also wrote into the stage buffers G1 and G2.
// TPN_ threads per node: with fewer threads than gathered chunks a thread
// serves chunks c, c + TPN_, ... (the tuner picks TPN_ per batch shape; the
// arithmetic of a chunk, and so the result, does not depend on it)
template <class L, int K, int STAGE, int TPN_ = MTR<L>::TPN>
__global__ void __launch_bounds__(MT<L>::NPB * TPN_) k_rk(const WorkItem* __restrict__ items, int nitems,
                                                          const SceneDev* __restrict__ scenes) {
    using G = Shape<L, TPN_>;
    // D3Q27 tiles hold (Wx, Wy, Wz, index) records; D2Q9 tiles the
    // (Wx, Wy, index) triplets, three floats per record
    constexpr bool D2 = L::D == 2;
    using T = typename std::conditional<D2, float, float4>::type;
    constexpr int QP = L::QP, K_ = D2 ? 3 * K : K;
    using Src = typename std::conditional<D2, CompactSrc, StencilSrc>::type;
    const int c0 = threadIdx.x % G::TPN, ns = threadIdx.x / G::TPN;
    NAGA_PIPE_BEGIN(T, ((D2 ? 3 : 1) * tile_cap<G::NPB, K>()), Src{})
    const int k = K > 0 ? K : S.k;
    const int nn = (int)(it.end - it.begin);
    const int64_t i = (int64_t)it.begin + ns;
    // chunks past NGATHER (D2Q9's rest population and pads) have zero rate:
    // their stage values equal g, G keeps them and no gather reads them
    // from the stage buffers
    if (ns < nn) {
#pragma unroll 1
    for (int c = c0; c < L::NGATHER; c += G::TPN) {
        float d0[3], d1[3];
        pair_dirs<L>(c, d0, d1);
        // Horner stages: G1 = g + dt/4 A g, G2 = g + dt/3 A G1, G1 = g + dt/2 A G2,
        // G = g + dt A G1
        // (D2Q9's stage 1 gathers the filter's compact copy of G in G2;
        // every stage buffer row holds L::QS floats, G rows L::QP)
        const float* src = (STAGE == 1) ? (D2 ? S.G2 : S.G) : (STAGE == 2) ? S.G1 : (STAGE == 3) ? S.G2 : S.G1;
        float* dst = (STAGE == 1) ? S.G1 : (STAGE == 2) ? S.G2 : (STAGE == 3) ? S.G1 : S.G;
        constexpr int QSRC = (STAGE == 1 && !D2) ? QP : L::QS;
        constexpr int QDST = STAGE == 4 ? QP : L::QS;
        const float a = S.rk_a[STAGE - 1];
        const float4 f0 = ld4(S.G, i, QP, c);
        RkAcc acc;
#pragma unroll 16
        for (int s = 0; s < k; ++s) {
            float4 rec;
            if constexpr (D2) {
                const float* t3 = reinterpret_cast<const float*>(tile) + 3 * (s * nn + ns);
                rec = make_float4(t3[0], t3[1], 0.f, t3[2]);
            } else {
                rec = reinterpret_cast<const float4*>(tile)[s * nn + ns];
            }
            const uint32_t j = __float_as_uint(rec.w);
            const float4 v = QSRC == QP ? ld4g<L>(src, j, c) : ld4s<L>(src, j, c);
            rk_term<L>(rec, d0, d1, v, acc);
        }
        // rate = -r; stage value = g + a rate
        const float4 r = acc.rate_sum();
        st4(dst, i, QDST, c, make_float4(fmaf(-a, r.x, f0.x), fmaf(-a, r.y, f0.y), fmaf(-a, r.z, f0.z),
                                        fmaf(-a, r.w, f0.w)));
    }
    }
    NAGA_PIPE_END
}

// threads-per-node candidates of the RK stages: the default first (one
// chunk per thread), then a shape without idle lanes (D3Q27: 7) and one with
// two chunks per thread (D3Q27: 4, D2Q9: 1)
template <class L>
struct RkShapes;
template <>
struct RkShapes<D3Q27> {
    static constexpr int n = 3;
    static constexpr int tpn[3] = {8, 7, 4};
};
template <>
struct RkShapes<D2Q9> {
    static constexpr int n = 2;
    static constexpr int tpn[2] = {2, 1};
};

// Shape code of the halo RK stages in the tuner's threads-per-node slot
constexpr int kRkHalo = 100;
// dynamic shared memory of k_rk_halo: three blob buffers (the pass being
// computed and two in flight) and two halo row buffers (the pass being
// computed and the next), two blocks per SM
constexpr int kHaloRowChunks = D3Q27::NGATHER;
constexpr size_t kHaloSmem = 3 * (size_t)kHaloBlobBytes + 2 * (size_t)kHaloCap * kHaloRowChunks * 16;

__device__ __forceinline__ void cp_async16(void* sdst, const void* gsrc) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(sdst)), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// RK stage STAGE of D3Q27 at k = kHaloK with the neighbour rows of each pass
// read from shared memory. A pass of 32 nodes references 1024 neighbour
// rows but only ~190 distinct ones on the benchmark grid (set-up lists them
// in the pass's halo blob, see SceneDev::stH); gathering each (node,
// neighbour, chunk) value from L2 moves ~5x the rows a pass needs and is
// bound by L2 latency. Here each block streams its passes through a
// pipeline: the halo blob (records with list positions, and the list) is
// bulk-copied two passes ahead; one pass ahead, the listed rows' gathered
// chunks are copied into shared memory with cp.async (16 B per thread, the
// 7 chunks of a row by 7 consecutive threads); the stage then reads its
// operands from shared memory, eight threads per node as in k_rk, so each
// quarter warp reads one row's 112 contiguous bytes (no bank conflicts).
// The arithmetic is k_rk's (rk_term, same order), so results are bit-equal
// to every other RK stage shape. A pass whose list overflowed (more than
// kHaloCap rows) gathers from global memory like k_rk.
template <int STAGE>
__global__ void __launch_bounds__(256, 2) k_rk_halo(const WorkItem* __restrict__ items, int nitems,
                                                    const SceneDev* __restrict__ scenes) {
    using L = D3Q27;
    constexpr int K = kHaloK, TPN = 8, NPB = MT<L>::NPB, NCH = kHaloRowChunks, QP = L::QP;
    constexpr int NB = 3, NH = 2, BLOB = kHaloBlobBytes;
    static_assert(NPB * TPN == 256 && NPB == 32, "one 32-node pass per 256-thread block");
    extern __shared__ __align__(128) unsigned char dyn_smem[];
    unsigned char* const blobs = dyn_smem;
    float4* const halo = reinterpret_cast<float4*>(dyn_smem + NB * BLOB);
    __shared__ __align__(8) uint64_t bar[NB];
    // the scenes of the pass being computed and of the next one (pass t uses
    // S2[t % 2]), so the next pass's scene loads without a barrier
    __shared__ SceneDev S2[2];
    const int c = threadIdx.x % TPN, ns = threadIdx.x / TPN;
    if (threadIdx.x == 0) {
        for (int b = 0; b < NB; ++b) mbar_init(&bar[b]);
        mbar_init_fence();
    }
    __syncthreads();
    // this block's passes: items blockIdx.x + t gridDim.x, t < T. The items
    // of passes t + 1 and t + 2 are held in registers and pass t + 3's is
    // loaded one iteration before its use, and the scene fields the copies
    // need are re-read only when the scene changes, so no dependent global
    // load stalls a pass
    const int T = (int)blockIdx.x < nitems ? (nitems - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
    auto item_of = [&](int t) {
        return t < T ? items[(int)blockIdx.x + t * (int)gridDim.x] : WorkItem{0u, 0u, 0u, 0u};
    };
    int issued = 0, waited = 0;  // blob copies (thread 0 issues; every thread waits)
    uint32_t par = 0;
    bool ok = true;
    uint32_t blob_scene = 0xFFFFFFFFu;  // thread 0: the scene whose blobs blob_base points at
    const float4* blob_base = nullptr;
    auto issue_blob = [&](const WorkItem& w, int t) {
        if (w.scene != blob_scene) {
            blob_scene = w.scene;
            blob_base = scenes[w.scene].stH;
        }
        // bulk/layer pass w.begin / NPB of its scene (the passes start at
        // multiples of NPB)
        bulk_load(blobs + (t % NB) * BLOB, blob_base + (int64_t)(w.begin / NPB) * (BLOB / 16), BLOB, &bar[t % NB]);
        ++issued;
    };
    auto wait_blob = [&](int t) {
        if (!ok) return;
        const int b = t % NB;
        ok = mbar_wait(&bar[b], (par >> b) & 1u);
        if (ok) {
            par ^= 1u << b;
            ++waited;
        }
    };
    // the listed rows of pass t (stage source rows of its scene) into halo
    // buffer t % NH
    uint32_t row_scene = 0xFFFFFFFFu;
    const float* row_src = nullptr;
    uint32_t row_n = 0;
    auto issue_rows = [&](const WorkItem& w, int t) {
        const uint32_t* list = reinterpret_cast<const uint32_t*>(blobs + (t % NB) * BLOB);
        const uint32_t m = list[0];
        if (m > (uint32_t)kHaloCap) return;
        if (w.scene != row_scene) {
            const SceneDev& sc = scenes[w.scene];
            row_scene = w.scene;
            row_src = STAGE == 1 ? sc.G : STAGE == 3 ? sc.G2 : sc.G1;
            row_n = (uint32_t)sc.N;
        }
        // thread (row r, chunk ch): rows r = threadIdx / 8 + 32 q, the
        // eighth lane of each row idle
        float4* hb = halo + (t % NH) * kHaloCap * NCH + c;
        if (c < NCH)
            for (int row = ns; row < (int)m; row += NPB) {
                const uint32_t j = list[4 + row];
                if (j < row_n) cp_async16(hb + row * NCH, row_src + (int64_t)j * QP + 4 * c);
            }
    };
    WorkItem w0 = item_of(0), w1 = item_of(1), w2 = item_of(2);
    // the tables do not depend on the previous kernel: the first blobs are
    // in flight before the wait for it
    if (threadIdx.x == 0) {
        if (T > 0) issue_blob(w0, 0);
        if (T > 1) issue_blob(w1, 1);
    }
    uint32_t scene_even = 0xFFFFFFFFu, scene_odd = 0xFFFFFFFFu;  // the scenes in S2[0], S2[1]
    if (T > 0) {
        scene_even = w0.scene;
        load_scene(S2[0], scenes + w0.scene);
    }
    pdl_wait_prev();
    if (T > 0) {
        wait_blob(0);
        if (ok) issue_rows(w0, 0);
    }
    cp_async_commit();
    float d0[3], d1[3];
    pair_dirs<L>(c < NCH ? c : 0, d0, d1);
    // one barrier a pass: after it, this pass's rows are in shared memory and
    // every thread is done with pass t - 1, whose blob, halo and scene
    // buffers the copies for passes t + 1 and t + 2 then reuse
    for (int t = 0; t < T; ++t) {
        const WorkItem w3 = item_of(t + 3);
        cp_async_wait<0>();  // this pass's rows (this thread's copies)
        if (__syncthreads_or(!ok)) {
            if (threadIdx.x == 0) atomicOr(&g_tile_timeout, 1u);
            break;
        }
        if (threadIdx.x == 0 && t + 2 < T) issue_blob(w2, t + 2);
        if (t + 1 < T) {
            wait_blob(t + 1);
            if (ok) issue_rows(w1, t + 1);
            uint32_t& held = ((t + 1) & 1) ? scene_odd : scene_even;
            if (w1.scene != held) {
                held = w1.scene;
                load_scene(S2[(t + 1) & 1], scenes + w1.scene);
            }
        }
        cp_async_commit();
        const SceneDev& S = S2[t & 1];
        const unsigned char* blob = blobs + (t % NB) * BLOB;
        const uint32_t m = reinterpret_cast<const uint32_t*>(blob)[0];
        const float4* tile = reinterpret_cast<const float4*>(blob + kHaloListBytes);
        const int nn = (int)(w0.end - w0.begin);
        const int64_t i = (int64_t)w0.begin + ns;
        if (ns < nn && c < NCH) {
            // stage buffers as in k_rk: G1 = g + dt/4 A g, G2 = g + dt/3 A G1,
            // G1 = g + dt/2 A G2, G = g + dt A G1
            const float* src = STAGE == 1 ? S.G : STAGE == 3 ? S.G2 : S.G1;
            float* dst = (STAGE == 1 || STAGE == 3) ? S.G1 : STAGE == 2 ? S.G2 : S.G;
            const float a = S.rk_a[STAGE - 1];
            const float4 f0 = ld4(S.G, i, QP, c);
            RkAcc acc;
            if (m <= (uint32_t)kHaloCap) {
                const float4* hb = halo + (t % NH) * kHaloCap * NCH + c;
                if (nn == NPB) {
                    // a full pass: records at a fixed stride
#pragma unroll 16
                    for (int s = 0; s < K; ++s) {
                        const float4 rec = tile[s * NPB + ns];
                        rk_term<L>(rec, d0, d1, hb[__float_as_uint(rec.w) * NCH], acc);
                    }
                } else {
#pragma unroll 4
                    for (int s = 0; s < K; ++s) {
                        const float4 rec = tile[s * nn + ns];
                        rk_term<L>(rec, d0, d1, hb[__float_as_uint(rec.w) * NCH], acc);
                    }
                }
            } else {
                // (rare: kept short so it does not raise the register count)
#pragma unroll 4
                for (int s = 0; s < K; ++s) {
                    const float4 rec = tile[s * nn + ns];
                    rk_term<L>(rec, d0, d1, ld4g<L>(src, __float_as_uint(rec.w), c), acc);
                }
            }
            const float4 r = acc.rate_sum();
            st4(dst, i, STAGE == 4 ? QP : L::QS, c,
                make_float4(fmaf(-a, r.x, f0.x), fmaf(-a, r.y, f0.y), fmaf(-a, r.z, f0.z), fmaf(-a, r.w, f0.w)));
        }
        w0 = w1;
        w1 = w2;
        w2 = w3;
    }
    cp_async_wait<0>();
    // a block that gave up waits (bounded) for the blob copies it still has
    // in flight before it exits
    if (threadIdx.x == 0)
        for (int t = waited; t < issued; ++t) {
            const int b = t % NB;
            if (mbar_wait(&bar[b], (par >> b) & 1u)) par ^= 1u << b;
        }
    pdl_allow_next();
}

// boundary: f = interp(f of bulk + layer) (simulation_engine.cuh:1370)
template <class L, int KB>
__global__ void __launch_bounds__(MTF<L>::BLOCK, 5) k_edge_interp(const WorkItem* __restrict__ items, int nitems,
                                                          const SceneDev* __restrict__ scenes) {
    using G = MTF<L>;
    constexpr int QP = L::QP, K_ = KB;
    const int c = threadIdx.x % G::TPN, ns = threadIdx.x / G::TPN;
    NAGA_PIPE_BEGIN(float2, (tile_cap<G::NPB, KB>()), EdgeSrc{})
    const int kb = KB > 0 ? KB : S.kb;
    const int nn = (int)(it.end - it.begin);
    const int64_t i = (int64_t)it.begin + ns;
    if (ns < nn && c < G::NCH) {
        const float4 acc = edge_sum<L, KB, false>(tile, kb, nn, ns, S.G, S.N, c);
        st4(S.G, i, QP, c, acc);
    }
    NAGA_PIPE_END
}

}  // namespace

// ------------------------------------------------------------- launches
enum {
    K_MACRO = 0,
    K_TAIL,
    K_PML,
    K_EDGE_COLLIDE,
    K_FILTER,
    K_RK1,
    K_RK2,
    K_RK3,
    K_RK4,
    K_EDGE_INTERP,
    K_COUNT
};

const char* kernel_name(int id) {
    static const char* names[K_COUNT] = {"macro_pml",    "means_probe", "pml_gather", "edge_collide",
                                         "filter",       "rk_stage1",   "rk_stage2",  "rk_stage3",
                                         "rk_stage4",    "edge_interp"};
    return (id >= 0 && id < K_COUNT) ? names[id] : "?";
}
int kernel_count() { return K_COUNT; }

namespace {
// V1 = sum_s W_s sigma_j, V2 = sum_s W_s sigma_j^2 over the layer supports j
// of each bulk/layer node, in support order (the mean part of the PML
// gather, see k_pml_gather)
__global__ void pml_vectors_kernel(const float4* __restrict__ stW, const float* __restrict__ sigma, int64_t nb,
                                   int64_t nl, int64_t nbl, int64_t n, int k, int npb, int dim,
                                   float4* __restrict__ PV) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nbl) return;
    float4 v1 = make_float4(0.f, 0.f, 0.f, 0.f), v2 = v1;
    uint32_t cnt = 0;
    for (int s = 0; s < k; ++s) {
        const float4 r = stW[pass_record(i, s, k, nbl, n, npb)];
        const int64_t jl = (int64_t)__float_as_uint(r.w) - nb;
        if (jl < 0 || jl >= nl) continue;
        const float sg = sigma[jl], sg2 = sg * sg;
        v1.x = fmaf(r.x, sg, v1.x);
        v1.y = fmaf(r.y, sg, v1.y);
        v2.x = fmaf(r.x, sg2, v2.x);
        v2.y = fmaf(r.y, sg2, v2.y);
        if (dim == 3) {  // D2Q9 records carry the filter weight in z
            v1.z = fmaf(r.z, sg, v1.z);
            v2.z = fmaf(r.z, sg2, v2.z);
        }
        ++cnt;
    }
    v1.w = __uint_as_float(cnt);  // count of layer supports (pml_table_kernel puts them first)
    PV[2 * i] = v1;
    PV[2 * i + 1] = v2;
}
}  // namespace

namespace {
// PML gather records in the stencil's pass order: the node's supports in
// the layer first, in stencil order, as (Wx, Wy, Wz or 0, PHI row j - nb);
// then zero-weight records on the last such row (never read by the gather,
// whose trip count is the node's layer-support count, but valid rows)
__global__ void pml_table_kernel(const float4* __restrict__ stW, int64_t nb, int64_t nl, int64_t nbl, int64_t n,
                                 int k, int npb, int dim, float4* __restrict__ stP) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nbl || nl <= 0) return;
    int o = 0;
    uint32_t last = 0;
    for (int s = 0; s < k; ++s) {
        const float4 r = stW[pass_record(i, s, k, nbl, n, npb)];
        const int64_t jl = (int64_t)__float_as_uint(r.w) - nb;
        if (jl < 0 || jl >= nl) continue;
        last = (uint32_t)jl;
        stP[pass_record(i, o++, k, nbl, n, npb)] = make_float4(r.x, r.y, dim == 3 ? r.z : 0.f, __uint_as_float(last));
    }
    for (; o < k; ++o) stP[pass_record(i, o, k, nbl, n, npb)] = make_float4(0.f, 0.f, 0.f, __uint_as_float(last));
}
}  // namespace

namespace {
__global__ void compact_records_kernel(const float4* __restrict__ stW, int64_t count, float* __restrict__ stR) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= count) return;
    const float4 r = stW[e];
    stR[3 * e] = r.x;
    stR[3 * e + 1] = r.y;
    stR[3 * e + 2] = r.w;
}
}  // namespace

int compact_records_device(const float4* stW, int64_t count, float* stR, cudaStream_t st) {
    if (count <= 0) return NAGA_OK;
    compact_records_kernel<<<(unsigned)((count + 255) / 256), 256, 0, st>>>(stW, count, stR);
    NAGA_CUDA_TRY(cudaGetLastError());
    return NAGA_OK;
}

namespace {
// One block per bulk/layer pass: the pass's nn k neighbour indices (at most
// 1024) are sorted, their distinct values listed, and each record's index
// replaced by its position in the list (binary search), or kept when the
// list would exceed kHaloCap (layout at SceneDev::stH)
__global__ void __launch_bounds__(256) halo_build_kernel(const float4* __restrict__ stW, int64_t nbl, int npb,
                                                         float4* __restrict__ stH) {
    constexpr int K = kHaloK, PER = 4, CAP = 256 * PER;
    static_assert(32 * K <= CAP, "a pass's records fit the block's keys");
    using Sort = cub::BlockRadixSort<uint32_t, 256, PER>;
    using Scan = cub::BlockScan<int, 256>;
    __shared__ union {
        typename Sort::TempStorage sort;
        typename Scan::TempStorage scan;
    } tmp;
    __shared__ uint32_t sorted[CAP];
    __shared__ uint32_t uniq[CAP];
    const int64_t b = (int64_t)blockIdx.x * npb;
    const int nn = (int)(nbl - b < npb ? nbl - b : npb);
    const int total = nn * K;
    const float4* rec = stW + b * K;
    uint32_t keys[PER];
#pragma unroll
    for (int q = 0; q < PER; ++q) {
        const int e = threadIdx.x * PER + q;
        keys[q] = e < total ? __float_as_uint(rec[e].w) : 0xFFFFFFFFu;
    }
    Sort(tmp.sort).Sort(keys);
#pragma unroll
    for (int q = 0; q < PER; ++q) sorted[threadIdx.x * PER + q] = keys[q];
    __syncthreads();
    int flag[PER], pos[PER], m = 0;
#pragma unroll
    for (int q = 0; q < PER; ++q) {
        const int e = threadIdx.x * PER + q;
        flag[q] = e < total && (e == 0 || sorted[e] != sorted[e - 1]);
    }
    Scan(tmp.scan).ExclusiveSum(flag, pos, m);
#pragma unroll
    for (int q = 0; q < PER; ++q)
        if (flag[q]) uniq[pos[q]] = sorted[threadIdx.x * PER + q];
    __syncthreads();
    uint32_t* list = reinterpret_cast<uint32_t*>(stH + (int64_t)blockIdx.x * (kHaloBlobBytes / 16));
    float4* out = stH + (int64_t)blockIdx.x * (kHaloBlobBytes / 16) + kHaloListBytes / 16;
    const bool local = m <= kHaloCap;
    for (int e = threadIdx.x; e < 4 + kHaloCap; e += blockDim.x)
        list[e] = e == 0 ? (uint32_t)m : (e >= 4 && local && e - 4 < m ? uniq[e - 4] : 0u);
    for (int e = threadIdx.x; e < 32 * K; e += blockDim.x) {
        float4 r = make_float4(0.f, 0.f, 0.f, 0.f);
        if (e < total) {
            r = rec[e];
            if (local) {
                const uint32_t j = __float_as_uint(r.w);
                int lo = 0, hi = m - 1;  // j is in the list
                while (lo < hi) {
                    const int mid = (lo + hi) >> 1;
                    if (uniq[mid] < j)
                        lo = mid + 1;
                    else
                        hi = mid;
                }
                r.w = __uint_as_float((uint32_t)lo);
            }
        }
        out[e] = r;
    }
}
}  // namespace

int halo_build_device(const float4* stW, int64_t nbl, int k, int npb, float4* stH, cudaStream_t st) {
    if (k != kHaloK || npb != 32) return set_error(NAGA_EINVAL, "halo blobs: need k = 32 and 32-node passes");
    if (nbl <= 0) return NAGA_OK;
    const int64_t n_pass = (nbl + npb - 1) / npb;
    halo_build_kernel<<<(unsigned)n_pass, 256, 0, st>>>(stW, nbl, npb, stH);
    NAGA_CUDA_TRY(cudaGetLastError());
    return NAGA_OK;
}

int pml_table_device(int dim, const float4* stW, int64_t nb, int64_t nl, int64_t nbl, int64_t n, int k, float4* stP,
                     cudaStream_t st) {
    if (nbl <= 0 || nl <= 0) return NAGA_OK;
    pml_table_kernel<<<(unsigned)((nbl + 255) / 256), 256, 0, st>>>(stW, nb, nl, nbl, n, k, nodes_per_pass(dim), dim,
                                                                    stP);
    NAGA_CUDA_TRY(cudaGetLastError());
    return NAGA_OK;
}

int pml_vectors_device(int dim, const float4* stW, const float* sigma, int64_t nb, int64_t nl, int64_t nbl, int64_t n,
                       int k, float4* PV, cudaStream_t st) {
    if (nbl <= 0) return NAGA_OK;
    const int npb = nodes_per_pass(dim);
    pml_vectors_kernel<<<(unsigned)((nbl + 255) / 256), 256, 0, st>>>(stW, sigma, nb, nl, nbl, n, k, npb, dim, PV);
    NAGA_CUDA_TRY(cudaGetLastError());
    return NAGA_OK;
}

namespace {
// rest state plus a density perturbation: g = f - w = w drho (u = 0)
template <class L>
__global__ void density_rows_kernel(const float* __restrict__ drho, int64_t n, float* __restrict__ G) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float d = drho ? drho[i] : 0.f;
    float v[L::QP];
#pragma unroll
    for (int t = 0; t < L::QP; ++t) v[t] = L::row(t) < 0 ? 0.f : LatticeTables<L>::w(L::row(t)) * d;
    store_row<L>(G, i, v);
}
}  // namespace

int density_rows_device(int dim, const float* drho, int64_t n, float* G, cudaStream_t st) {
    const unsigned blocks = (unsigned)((n + 255) / 256);
    if (blocks == 0) return NAGA_OK;
    if (dim == 2)
        density_rows_kernel<D2Q9><<<blocks, 256, 0, st>>>(drho, n, G);
    else
        density_rows_kernel<D3Q27><<<blocks, 256, 0, st>>>(drho, n, G);
    NAGA_CUDA_TRY(cudaGetLastError());
    return NAGA_OK;
}

namespace {
// one wait on a barrier whose phase nothing completes: it gives up after
// limit_ns and raises the flag the step kernels raise
__global__ void k_wait_selftest(int polls) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar);
        mbar_init_fence();
    }
    __syncthreads();
    if (threadIdx.x == 0 && !mbar_wait(&bar, 0u, polls)) atomicOr(&g_tile_timeout, 1u);
}
}  // namespace

int wait_selftest(int polls, cudaStream_t st) {
    if (polls < 0 || polls > kTileWaitPolls) return set_error(NAGA_EINVAL, "wait self-test: polls out of range");
    k_wait_selftest<<<1, 32, 0, st>>>(polls > 0 ? polls : kTileWaitPolls);
    NAGA_CUDA_TRY(cudaGetLastError());
    return tile_timeout_check(st);
}

int tile_timeout_check(cudaStream_t st) {
    unsigned int flag = 0;
    NAGA_CUDA_TRY(cudaMemcpyFromSymbolAsync(&flag, g_tile_timeout, sizeof(flag), 0, cudaMemcpyDeviceToHost, st));
    NAGA_CUDA_TRY(cudaStreamSynchronize(st));
    if (!flag) return NAGA_OK;
    const unsigned int zero = 0;
    NAGA_CUDA_TRY(cudaMemcpyToSymbolAsync(g_tile_timeout, &zero, sizeof(zero), 0, cudaMemcpyHostToDevice, st));
    NAGA_CUDA_TRY(cudaStreamSynchronize(st));
    return set_error(NAGA_ETIMEOUT, "step kernel: a table copy into shared memory did not complete in time");
}
int nodes_per_pass(int dim) { return dim == 2 ? MT<D2Q9>::NPB : MT<D3Q27>::NPB; }

// dynamic shared memory of the generic (K == 0) variants: two buffers of
// NPB x 64 records
template <class L, int K, class T>
size_t tile_bytes() {
    return K > 0 ? 0 : 2 * (size_t)MT<L>::NPB * 64 * sizeof(T);
}
// opts a kernel into `bytes` of dynamic shared memory when its static plus
// dynamic shared memory exceeds the 48 KB a launch gets without opting in
template <class Kern>
int allow_smem(Kern kern, size_t bytes) {
    if (bytes == 0) return NAGA_OK;
    cudaFuncAttributes fa{};
    NAGA_CUDA_TRY(cudaFuncGetAttributes(&fa, kern));
    if (fa.sharedSizeBytes + bytes > 48 * 1024)
        NAGA_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    return NAGA_OK;
}

// resident blocks per SM of a kernel at its launch shape (occupancy
// calculator). The answer depends on the shared-memory carveout set on the
// kernel, so it is cached per kernel, shared memory and applied shape bps
template <class Kern>
int resident_blocks(Kern kern, int block, size_t smem, int bps) {
    static std::mutex mu;
    static std::map<std::tuple<const void*, size_t, int>, int> cache;
    const auto key = std::make_tuple(reinterpret_cast<const void*>(kern), smem, bps);
    std::lock_guard<std::mutex> lk(mu);
    auto f = cache.find(key);
    if (f != cache.end()) return f->second;
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, block, smem) != cudaSuccess || n < 1) n = 1;
    cache[key] = n;
    return n;
}

// ------------------------------------------------------------ launch shapes
// The gather kernels share the SM's unified L1 / shared-memory storage
// between their tile buffers and the L1 cache that absorbs the neighbour-row
// re-reads: more resident blocks hide more latency but leave less L1. The
// number of resident blocks per SM (bps) is set through the shared-memory
// carveout and chosen per (lattice, k, kb, batch size) by tune_step_shapes;
// bps = 0 keeps the driver's default carveout and the occupancy maximum.
struct ShapeKey {
    int dim, k, kb, bucket;
    bool operator<(const ShapeKey& o) const {
        return std::tie(dim, k, kb, bucket) < std::tie(o.dim, o.k, o.kb, o.bucket);
    }
};
// the tuned launch shape of a batch shape: resident blocks per SM of the
// gather kernels (0: default carveout) and threads per node of the RK
// stages (0: the default, one chunk per thread)
struct TunedShape {
    int bps = 0, tpn = 0;
    int fbps = 0;  // the filter's resident blocks per SM (0: default carveout)
    int pbps = 0;  // the PML gather's
};
std::mutex g_shape_mu;
std::map<ShapeKey, TunedShape> g_shape;
std::string g_tune_log;

int smem_per_sm() {
    static int v = 0;
    if (!v) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess || v <= 0)
            v = 228 * 1024;
    }
    return v;
}

// carveout (percent of the maximum shared memory) that holds bps blocks of
// the kernel; bps = 0 restores the default preference
template <class Kern>
int set_blocks_per_sm(Kern kern, size_t dyn_smem, int bps) {
    int pct = -1;  // cudaSharedmemCarveoutDefault
    if (bps > 0) {
        cudaFuncAttributes fa{};
        NAGA_CUDA_TRY(cudaFuncGetAttributes(&fa, kern));
        const double need = (double)bps * (double)(fa.sharedSizeBytes + dyn_smem + 1024);
        pct = (int)std::ceil(100.0 * need / smem_per_sm());
        pct = pct < 1 ? 1 : (pct > 100 ? 100 : pct);
    }
    NAGA_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, pct));
    return NAGA_OK;
}

ShapeKey shape_key(int dim, int k, int kb, int n_items) {
    int b = 0;
    while ((1 << (b + 1)) <= n_items) ++b;
    return {dim, k, kb, b};
}

TunedShape tuned_shape(const ShapeKey& key) {
    std::lock_guard<std::mutex> lk(g_shape_mu);
    auto f = g_shape.find(key);
    return f == g_shape.end() ? TunedShape{} : f->second;
}

// fn(kernel, block, dynamic shared memory) with RK stage STAGE's
// instantiation for the shape code tpn: threads per node (the unrolled
// stencil sizes have every RkShapes candidate; the generic K == 0 kernels
// only the default) or kRkHalo (D3Q27 at k = kHaloK)
template <class L, int K, int STAGE, class Fn>
int rk_dispatch(int tpn, Fn&& fn) {
    constexpr size_t s4 = K > 0 ? 0 : 2 * (size_t)MT<L>::NPB * 64 * sizeof(float4);
    constexpr int NPB = MT<L>::NPB;
    if constexpr (K > 0) {
        if constexpr (L::D == 3) {
            if constexpr (K == kHaloK)
                if (tpn == kRkHalo) return fn(k_rk_halo<STAGE>, 256, kHaloSmem);
            if (tpn == 7) return fn(k_rk<L, K, STAGE, 7>, NPB * 7, s4);
            if (tpn == 4) return fn(k_rk<L, K, STAGE, 4>, NPB * 4, s4);
        } else {
            if (tpn == 1) return fn(k_rk<L, K, STAGE, 1>, NPB * 1, s4);
        }
    }
    return fn(k_rk<L, K, STAGE, MTR<L>::TPN>, NPB * MTR<L>::TPN, s4);
}
// resident blocks per SM the RK stages of shape code tpn run at for the
// tuned bps (the halo stages always at their two)
inline int rk_bps(int tpn, int bps) { return tpn == kRkHalo ? 2 : bps; }
// the halo shape is offered for D3Q27 at k = kHaloK
template <class L, int K>
constexpr bool has_halo() {
    return L::D == 3 && K == kHaloK;
}
// a shape code as the tuner's log names it
template <class L>
std::string shape_name(int tpn) {
    return tpn == kRkHalo ? std::string("halo") : std::to_string(tpn ? tpn : MTR<L>::TPN);
}
template <class L, int K, class Fn>
int rk_each_stage(int tpn, Fn&& fn) {
    int rc;
    if ((rc = rk_dispatch<L, K, 1>(tpn, fn)) || (rc = rk_dispatch<L, K, 2>(tpn, fn)) ||
        (rc = rk_dispatch<L, K, 3>(tpn, fn)) || (rc = rk_dispatch<L, K, 4>(tpn, fn)))
        return rc;
    return NAGA_OK;
}

template <class L, int K, int KB>
struct AppliedShape {
    static int bps, tpn, fbps, pbps;  // shape currently set on the instantiation's kernels (-2: unknown)
};
template <class L, int K, int KB>
int AppliedShape<L, K, KB>::pbps = -2;
template <class L, int K, int KB>
int AppliedShape<L, K, KB>::bps = -2;
template <class L, int K, int KB>
int AppliedShape<L, K, KB>::tpn = -2;
template <class L, int K, int KB>
int AppliedShape<L, K, KB>::fbps = -2;

// carveout of every gather kernel of an instantiation (set only when the
// shape changes)
template <class L, int K, int KB>
int apply_shape(const TunedShape& sh) {
    int& applied = AppliedShape<L, K, KB>::bps;
    int& applied_tpn = AppliedShape<L, K, KB>::tpn;
    int& applied_fbps = AppliedShape<L, K, KB>::fbps;
    std::lock_guard<std::mutex> lk(g_shape_mu);
    const int bps = sh.bps;
    int& applied_pbps = AppliedShape<L, K, KB>::pbps;
    if (applied == bps && applied_tpn == sh.tpn && applied_fbps == sh.fbps && applied_pbps == sh.pbps) return NAGA_OK;
    using TF = float2;  // filter records
    const size_t s4 = tile_bytes<L, K, float4>(), s2 = tile_bytes<L, K, TF>(), sb = tile_bytes<L, KB, float2>();
    int rc;
    const int bo = other_bps<L>(bps);
    if ((rc = set_blocks_per_sm(k_pml_gather<L, K>, s4, sh.pbps)) ||
        (rc = rk_each_stage<L, K>(sh.tpn, [&](auto kern, int, size_t sm) {
             return set_blocks_per_sm(kern, sm, rk_bps(sh.tpn, bps));
         })) ||
        (rc = set_blocks_per_sm(k_filter<L, K>, s2, sh.fbps)) ||
        (rc = set_blocks_per_sm(k_edge_collide<L, KB>, sb, bo)) ||
        (rc = set_blocks_per_sm(k_edge_interp<L, KB>, sb, bo)))
        return rc;
    applied = bps;
    applied_tpn = sh.tpn;
    applied_fbps = sh.fbps;
    applied_pbps = sh.pbps;
    return NAGA_OK;
}

// programmatic dependent launch of the step's kernels (see pdl_wait_prev);
// NAGA_PDL=0 in the environment launches them plainly
bool pdl_on() {
    static const bool on = [] {
        const char* e = std::getenv("NAGA_PDL");
        return !(e && e[0] == '0');
    }();
    return on;
}
template <class... KArgs, class... Args>
cudaError_t launch_step_kernel(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                               Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = pdl_on() ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kern, args...);
}

template <class L, int K, int KB>
int enqueue_step_k(const StepLaunch& P, cudaStream_t st) {
    const int cap = sm_count() * 8;
    using TF = float2;  // filter records
    const size_t s4 = tile_bytes<L, K, float4>(), s2 = tile_bytes<L, K, TF>(), sb = tile_bytes<L, KB, float2>();
    int rc;
    const TunedShape sh = tuned_shape(shape_key(L::D, K, KB, P.n_fluid));
    if ((rc = allow_smem(k_pml_gather<L, K>, s4)) ||
        (rc = rk_each_stage<L, K>(sh.tpn, [&](auto kern, int, size_t sm) { return allow_smem(kern, sm); })) ||
        (rc = allow_smem(k_filter<L, K>, s2)) || (rc = allow_smem(k_edge_collide<L, KB>, sb)) ||
        (rc = allow_smem(k_edge_interp<L, KB>, sb)))
        return rc;
    auto grid = [&](int n) { return n < cap ? n : cap; };
    // the pipelined gather kernels loop over their items: one wave of
    // resident blocks, bps per SM when the tuned shape fixes it
    const int sms = sm_count();
    const int bps = sh.bps;
    if ((rc = apply_shape<L, K, KB>(sh))) return rc;
    const int bo = other_bps<L>(bps);
    // the RK stages and the PML gather at their block size and bps, the
    // filter and boundary kernels at theirs and bo
    auto pgrid_b = [&](auto kern, size_t smem, int n, int block, int b) {
        int r = resident_blocks(kern, block, smem, b);
        if (b > 0 && b < r) r = b;
        const int g = r * sms;
        return n < g ? n : g;
    };
    constexpr int RB = MTR<L>::BLOCK, FB = MTF<L>::BLOCK, FFB = MTFF<L>::BLOCK;
    auto pgrid = [&](auto kern, size_t smem, int n) { return pgrid_b(kern, smem, n, FB, bo); };
    const bool prof = prof_on();
    cudaError_t lerr = cudaSuccess;
    auto keep = [&](cudaError_t e) {
        if (lerr == cudaSuccess) lerr = e;
    };
#define LAUNCH(id, n, ...)                      \
    if ((n) > 0) {                              \
        if (prof) prof_begin(id, st);           \
        __VA_ARGS__;                            \
        if (prof) prof_end(id, st);             \
    }
    LAUNCH(K_MACRO, P.n_all, keep(launch_step_kernel(k_macro_pml<L>, grid(P.n_all), kBlock, 0, st, P.all, P.n_all, P.scenes)));
    LAUNCH(K_TAIL, P.nscenes, keep(launch_step_kernel(k_scene_tail<L::QP>, dim3(P.nscenes, 2 * L::QP + 1), 256, 0, st, P.scenes)));
    LAUNCH(K_PML, P.n_pml, keep(launch_step_kernel(k_pml_gather<L, K>, pgrid_b(k_pml_gather<L, K>, s4, P.n_pml, RB, sh.pbps), RB, s4, st, P.pml, P.n_pml, P.scenes)));
    LAUNCH(K_EDGE_COLLIDE, P.n_edge,
           keep(launch_step_kernel(k_edge_collide<L, KB>, pgrid(k_edge_collide<L, KB>, sb, P.n_edge), FB, sb, st, P.edge, P.n_edge, P.scenes)));
    LAUNCH(K_FILTER, P.n_all_mt,
           keep(launch_step_kernel(k_filter<L, K>, pgrid_b(k_filter<L, K>, s2, P.n_all_mt, FFB, sh.fbps), FFB, s2, st, P.all_mt, P.n_all_mt, P.scenes)));
    // the RK stages at the tuned threads per node
    auto rk_launch = [&](auto kern, int blk, size_t sm) {
        keep(launch_step_kernel(kern, pgrid_b(kern, sm, P.n_fluid, blk, rk_bps(sh.tpn, bps)), blk, sm, st, P.fluid,
                                P.n_fluid, P.scenes));
        return NAGA_OK;
    };
    LAUNCH(K_RK1, P.n_fluid, (rk_dispatch<L, K, 1>(sh.tpn, rk_launch)));
    LAUNCH(K_RK2, P.n_fluid, (rk_dispatch<L, K, 2>(sh.tpn, rk_launch)));
    LAUNCH(K_RK3, P.n_fluid, (rk_dispatch<L, K, 3>(sh.tpn, rk_launch)));
    LAUNCH(K_RK4, P.n_fluid, (rk_dispatch<L, K, 4>(sh.tpn, rk_launch)));
    LAUNCH(K_EDGE_INTERP, P.n_edge,
           keep(launch_step_kernel(k_edge_interp<L, KB>, pgrid(k_edge_interp<L, KB>, sb, P.n_edge), FB, sb, st, P.edge, P.n_edge, P.scenes)));
#undef LAUNCH
    NAGA_CUDA_TRY(lerr);
    NAGA_CUDA_TRY(cudaGetLastError());
    return NAGA_OK;
}

// Launch-shape tuner: times RK stage 1 (it reads G or its compact copy and
// overwrites only the stage scratch G1, so it can run between steps) on the
// batch's own items for each candidate shape -- threads per node of the RK
// stages (RkShapes: the default first) times resident blocks per SM (the
// default carveout 0, then 2 .. max), then the halo stages (D3Q27, k = 32)
// -- and keeps the fastest; a shape other than the default (default threads
// per node, default carveout) must beat the best default-shape time by 3%
// when it fixes a carveout, since that binds the other gather kernels too,
// and by 1% otherwise. NAGA_GATHER_BPS=<n> and NAGA_GATHER_TPN=<t> fix the
// choice instead (bps 0: default carveout; tpn 0 or unlisted: the default;
// tpn "halo": the halo stages).
template <class L, int K, int KB>
int tune_k(const StepLaunch& P, cudaStream_t st) {
    if (P.n_fluid <= 0) return NAGA_OK;
    const ShapeKey key = shape_key(L::D, K, KB, P.n_fluid);
    {
        std::lock_guard<std::mutex> lk(g_shape_mu);
        if (g_shape.count(key)) return NAGA_OK;
    }
    const size_t s4 = tile_bytes<L, K, float4>();
    int rc = NAGA_OK;
    char line[200];
    const char* env_bps = std::getenv("NAGA_GATHER_BPS");
    const char* env_tpn = std::getenv("NAGA_GATHER_TPN");
    if (env_bps || env_tpn) {
        TunedShape sh;
        sh.bps = env_bps ? std::max(0, std::atoi(env_bps)) : 0;
        sh.fbps = filter_bps<L>(sh.bps);
        sh.pbps = sh.bps;
        const int t = env_tpn ? std::atoi(env_tpn) : 0;
        for (int c = 0; c < RkShapes<L>::n; ++c)
            if (RkShapes<L>::tpn[c] == t && (K > 0 || c == 0)) sh.tpn = c == 0 ? 0 : t;
        if (env_tpn && std::string(env_tpn) == "halo" && has_halo<L, K>()) sh.tpn = kRkHalo;
        std::lock_guard<std::mutex> lk(g_shape_mu);
        g_shape[key] = sh;
        std::snprintf(line, sizeof line,
                      "dim %d k %d kb %d items 2^%d: tpn %s bps %d filter bps %d (NAGA_GATHER_BPS / _TPN)\n",
                      key.dim, key.k, key.kb, key.bucket, shape_name<L>(sh.tpn).c_str(), sh.bps, sh.fbps);
        g_tune_log += line;
        return NAGA_OK;
    }
    const int sms = sm_count();
    cudaEvent_t e0, e1;
    NAGA_CUDA_TRY(cudaEventCreate(&e0));
    NAGA_CUDA_TRY(cudaEventCreate(&e1));
    cudaError_t terr = cudaSuccess;  // the error of a failed trial
    TunedShape best;
    float best_ms = -1.f, best_default_ms = -1.f;
    std::string log;
    // candidates: the RkShapes thread shapes, then the halo stages (timed at
    // their own two blocks per SM only; NAGA_RK_HALO=0 leaves them out)
    const char* env_halo = std::getenv("NAGA_RK_HALO");
    const bool try_halo = has_halo<L, K>() && !(env_halo && env_halo[0] == '0');
    const int ncand = (K > 0 ? RkShapes<L>::n : 1) + (try_halo ? 1 : 0);
    for (int ci = 0; ci < ncand && rc == NAGA_OK; ++ci) {
        const bool halo = try_halo && ci == ncand - 1;
        const int tpn = halo ? kRkHalo : ci == 0 ? 0 : RkShapes<L>::tpn[ci];
        rc = rk_dispatch<L, K, 1>(tpn, [&](auto kern, int blk, size_t sm) -> int {
            int r;
            if ((r = allow_smem(kern, sm)) || (r = set_blocks_per_sm(kern, sm, 0))) return r;
            int maxr = 0;
            NAGA_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&maxr, kern, blk, sm));
            maxr = std::max(maxr, halo ? rk_bps(tpn, 0) : 1);
            std::snprintf(line, sizeof line, " | tpn %s", shape_name<L>(tpn).c_str());
            log += line;
            for (int bps = halo ? rk_bps(tpn, 0) : 0; bps <= maxr; bps = bps == 0 ? 2 : bps + 1) {
                if ((r = set_blocks_per_sm(kern, sm, bps))) return r;
                const int g = std::min(P.n_fluid, (bps > 0 ? bps : maxr) * sms);
                // one untimed and one timed launch; launches shorter than
                // ~0.4 ms are timed again over enough repetitions to span ~2 ms
                auto timed = [&](int reps, float* ms) -> bool {
                    cudaEventRecord(e0, st);
                    for (int q = 0; q < reps; ++q) kern<<<g, blk, sm, st>>>(P.fluid, P.n_fluid, P.scenes);
                    cudaEventRecord(e1, st);
                    terr = cudaEventSynchronize(e1);
                    if (terr == cudaSuccess) terr = cudaGetLastError();
                    if (terr != cudaSuccess) return false;
                    cudaEventElapsedTime(ms, e0, e1);
                    *ms /= reps;
                    return true;
                };
                kern<<<g, blk, sm, st>>>(P.fluid, P.n_fluid, P.scenes);
                float ms = 0.f, ms2 = 0.f;
                bool ok = timed(1, &ms);
                if (ok && ms < 0.4f) ok = timed(std::min(8, std::max(2, (int)(2.f / std::max(ms, 1e-3f)))), &ms);
                // twice, the faster kept: other streams' work (a server's
                // scene set-up) can slow a single trial
                const int reps2 = ms < 0.4f ? std::min(8, std::max(2, (int)(2.f / std::max(ms, 1e-3f)))) : 1;
                if (ok && timed(reps2, &ms2)) ms = std::min(ms, ms2);
                if (!ok)
                    return set_error(NAGA_ECUDA,
                                     std::string("launch-shape tuning: a trial launch failed: ") + cudaGetErrorString(terr));
                std::snprintf(line, sizeof line, " %d:%.1fus", bps, ms * 1000.f);
                log += line;
                const bool is_default = tpn == 0 && bps == 0;
                if (is_default) best_default_ms = ms;
                const bool hopeless = tpn != 0 && bps == 0 && best_ms > 0.f && ms > 1.25f * best_ms;
                if (best_ms < 0.f || ms < best_ms) {
                    // the halo stages keep their own carveout; the other
                    // gather kernels stay at the default
                    best.bps = halo ? 0 : bps;
                    best.tpn = tpn;
                    best_ms = ms;
                }
                // a thread shape 25% behind at the default carveout is not
                // tried at the others (keeps the tuning of a large batch short)
                if (hopeless) {
                    log += " (skipped)";
                    break;
                }
            }
            // the trials changed this kernel's carveout
            return set_blocks_per_sm(kern, sm, 0);
        });
    }
    // a non-default shape must beat the default: by 3% when it fixes a
    // carveout (which binds the other gather kernels too), by 1% otherwise
    const float margin = best.bps != 0 ? 0.97f : 0.99f;
    if (best_default_ms > 0.f && (best.bps != 0 || best.tpn != 0) && best_ms > margin * best_default_ms) best = {};
    // resident blocks per SM of the filter, timed on its dry variant (same
    // gathers, result into dead scratch), and of the PML gather, which only
    // adds into the collision scratch (dead between steps), over the batch's
    // items: the default carveout, then 2 .. max; a fixed carveout must win
    // by 3%
    auto tune_bps = [&](auto kern, size_t smem, int block, const WorkItem* list, int n, const char* name,
                        int* out) {
        if (rc != NAGA_OK || n <= 0) return;
        float kbest = -1.f, kdefault = -1.f;
        int kb = 0, maxr = 0;
        if ((rc = allow_smem(kern, smem)) || (rc = set_blocks_per_sm(kern, smem, 0))) return;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&maxr, kern, block, smem) != cudaSuccess) {
            rc = set_error(NAGA_ECUDA, "launch-shape tuning: occupancy query failed");
            return;
        }
        maxr = std::max(maxr, 1);
        log += " | ";
        log += name;
        for (int bps = 0; bps <= maxr; bps = bps == 0 ? 2 : bps + 1) {
            if ((rc = set_blocks_per_sm(kern, smem, bps))) return;
            const int g = std::min(n, (bps > 0 ? bps : maxr) * sms);
            auto timed = [&](int reps, float* ms) -> bool {
                cudaEventRecord(e0, st);
                for (int q = 0; q < reps; ++q) kern<<<g, block, smem, st>>>(list, n, P.scenes);
                cudaEventRecord(e1, st);
                terr = cudaEventSynchronize(e1);
                if (terr == cudaSuccess) terr = cudaGetLastError();
                if (terr != cudaSuccess) return false;
                cudaEventElapsedTime(ms, e0, e1);
                *ms /= reps;
                return true;
            };
            kern<<<g, block, smem, st>>>(list, n, P.scenes);
            float ms = 0.f, ms2 = 0.f;
            bool ok = timed(1, &ms);
            const int reps2 = ms < 0.4f ? std::min(8, std::max(2, (int)(2.f / std::max(ms, 1e-3f)))) : 1;
            if (ok && timed(reps2, &ms2)) ms = std::min(ms, ms2);
            if (!ok) {
                rc = set_error(NAGA_ECUDA,
                               std::string("launch-shape tuning: a trial launch failed: ") + cudaGetErrorString(terr));
                return;
            }
            std::snprintf(line, sizeof line, " %d:%.1fus", bps, ms * 1000.f);
            log += line;
            if (bps == 0) kdefault = ms;
            if (kbest < 0.f || ms < kbest) {
                kbest = ms;
                kb = bps;
            }
        }
        if (kb != 0 && kbest > 0.97f * kdefault) kb = 0;
        *out = kb;
        rc = set_blocks_per_sm(kern, smem, 0);
    };
    tune_bps(k_filter<L, K, true>, tile_bytes<L, K, float2>(), MTFF<L>::BLOCK, P.all_mt, P.n_all_mt, "filter",
             &best.fbps);
    tune_bps(k_pml_gather<L, K>, s4, MTR<L>::BLOCK, P.pml, P.n_pml, "pml", &best.pbps);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    AppliedShape<L, K, KB>::bps = -2;  // the trials changed rk stage 1's carveouts
    AppliedShape<L, K, KB>::tpn = -2;
    AppliedShape<L, K, KB>::fbps = -2;
    AppliedShape<L, K, KB>::pbps = -2;
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(g_shape_mu);
    g_shape[key] = best;
    std::snprintf(line, sizeof line, "dim %d k %d kb %d items 2^%d: tpn %s bps %d filter bps %d pml bps %d of",
                  key.dim, key.k, key.kb, key.bucket, shape_name<L>(best.tpn).c_str(), best.bps, best.fbps,
                  best.pbps);
    g_tune_log += line + log + "\n";
    return NAGA_OK;
}

int tune_step_shapes(int dim, int k, int kb, const StepLaunch& P, cudaStream_t st) {
    if (dim == 2) return k == 16 && kb == 16 ? tune_k<D2Q9, 16, 16>(P, st) : tune_k<D2Q9, 0, 0>(P, st);
    if (k == 32 && kb == 32) return tune_k<D3Q27, 32, 32>(P, st);
    if (k == 16 && kb == 16) return tune_k<D3Q27, 16, 16>(P, st);
    return tune_k<D3Q27, 0, 0>(P, st);
}

std::string tuning_report() {
    std::lock_guard<std::mutex> lk(g_shape_mu);
    return g_tune_log;
}

// k, kb: the batch's common stencil sizes (0 if the members differ); the
// common sizes get fully unrolled gathers with fixed-size tiles
int enqueue_step(int dim, int k, int kb, const StepLaunch& P, cudaStream_t st) {
    if (dim == 2) {
        // unrolled variants whose two tile buffers fit static shared memory
        if (k == 16 && kb == 16) return enqueue_step_k<D2Q9, 16, 16>(P, st);
        return enqueue_step_k<D2Q9, 0, 0>(P, st);
    }
    if (k == 32 && kb == 32) return enqueue_step_k<D3Q27, 32, 32>(P, st);
    if (k == 16 && kb == 16) return enqueue_step_k<D3Q27, 16, 16>(P, st);
    return enqueue_step_k<D3Q27, 0, 0>(P, st);
}

}  // namespace naga
