// The time step of NAGA's nonlocal lattice-Boltzmann engine on sm_100a.
//
// Reference: fluids/nonlocal_lattice_boltzmann/detail/simulation_engine.cuh
// step_forward :1325-1375, issued there as ~1000 launches (27 populations x
// separate divergence gathers, reductions and axpy passes). Here one step is
// a fixed sequence of fused kernels over work items (<= 128 consecutive nodes
// of one scene), so one launch covers every scene of a batch:
//
//   macro_pml     all nodes   rho, u; PML trapezoid integrals Q1, Q2;
//                             per-item layer sums of Q1, Q2
//   pml_means     per scene   layer means of Q1, Q2 (fixed-order sums)
//   probe         per scene   RPIM probe of rho at the start of the step
//   pml_collide   bulk+layer  f - sigma(3f~ + 3 sigma Q1 + sigma^2 Q2) + PML
//                             divergence gathers + central-moment collision
//   edge_collide  boundary    RPIM boundary interpolation + collision
//   filter        all nodes   selective Gaussian filter; bounce-back
//   rk(1..4)      bulk+layer  streaming gather + RK4 stage update
//   edge_interp   boundary    RPIM boundary interpolation of the result
//   step_end      per scene   step counter
//
// Arithmetic is FP32 on centred populations g = f - w and rho - 1: the
// reference keeps f itself in FP32 (T = float), which quantises a 1e-4
// acoustic perturbation of f ~ w to ~1e-3 relative; g keeps full relative
// precision. Where the collision formulas subtract the O(1) equilibrium
// parts of the moments, those parts are cancelled analytically and only the
// small remainders enter the FP32 arithmetic.
#include "common.cuh"
#include "scene_dev.hpp"

namespace naga {

namespace {

constexpr int kBlock = 128;

template <class L>
struct Lat : LatticeTables<L> {
    using T = LatticeTables<L>;
    static constexpr int D = L::D, Q = L::Q, QP = L::QP;
};

// lattice speed of sound as the reference spells it (lattices.cuh:46-49)
__device__ __forceinline__ float cs_f() { return 0.57735026918962576450914878050196f; }

template <class L>
__device__ __forceinline__ void load_row(const float* base, int64_t i, float* v) {
    const float4* p = reinterpret_cast<const float4*>(base + i * L::QP);
#pragma unroll
    for (int c = 0; c < L::QP / 4; ++c) {
        float4 t = __ldg(p + c);
        v[4 * c + 0] = t.x;
        v[4 * c + 1] = t.y;
        v[4 * c + 2] = t.z;
        v[4 * c + 3] = t.w;
    }
}
template <class L>
__device__ __forceinline__ void load_row_rw(const float* base, int64_t i, float* v) {
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
    for (int c = 0; c < L::QP / 4; ++c) {
        float4 t;
        t.x = v[4 * c + 0];
        t.y = (4 * c + 1 < L::Q) ? v[4 * c + 1] : 0.f;
        t.z = (4 * c + 2 < L::Q) ? v[4 * c + 2] : 0.f;
        t.w = (4 * c + 3 < L::Q) ? v[4 * c + 3] : 0.f;
        p[c] = t;
    }
}

// rho - 1 and u (lattice units) from centred populations; sums in
// population order as detail/simulation_engine.cuh:53-82
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
    for (int d = 0; d < L::D; ++d) u[d] = m[d] / rho;
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
    return w * drho + w * (1.f + drho) * (uc / cs2 + (uc * uc) / (2.f * cs4) - uu);
}

// c_a . W for a population a
template <class L>
__device__ __forceinline__ float proj(int a, float wx, float wy, float wz) {
    using T = Lat<L>;
    float p = 0.f;
    if (T::cx(a)) p = T::cx(a) > 0 ? wx : -wx;
    if (T::cy(a)) p = T::cy(a) > 0 ? p + wy : p - wy;
    if (L::D == 3 && T::cz(a)) p = T::cz(a) > 0 ? p + wz : p - wz;
    return p;
}

// stencil record s of node i: weights and support index
template <class L>
__device__ __forceinline__ void stencil(const SceneDev& S, int s, int64_t i, float& wx, float& wy, float& wz,
                                        uint32_t& j) {
    if (L::D == 3) {
        float4 r = __ldg(reinterpret_cast<const float4*>(S.stW) + (int64_t)s * S.N + i);
        wx = r.x;
        wy = r.y;
        wz = r.z;
        j = __float_as_uint(r.w);
    } else {
        float2 r = __ldg(reinterpret_cast<const float2*>(S.stW) + (int64_t)s * S.N + i);
        wx = r.x;
        wy = r.y;
        wz = 0.f;
        j = __ldg(S.stI + (int64_t)s * S.N + i);
    }
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
    a = (m == 0) ? 1.f : (m == 1 ? 0.f : 1.f / 3.f);
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
    k[4] = om * (-Kxy / 12.f);
    k[5] = om * (-Kxz / 12.f);
    k[6] = om * (-Kyz / 12.f);
    k[7] = om * (-(sxx - syy) / 12.f);
    k[8] = om * (-(sxx + syy - 2.f * szz) / 36.f);
    k[9] = om * (-(sxx + syy + szz - drho) / 18.f);
    om = S.om_fix[0];
    k[10] = om * (-(6.f * Kxy * v1 + 3.f * Kxyy + 6.f * Kxz * v2 + 3.f * Kxzz + 3.f * Kyy * v0 + 3.f * Kzz * v0 -
                    2.f * rho * v0) / 72.f);
    k[11] = om * (-(3.f * Kxx * v1 + 3.f * Kxxy + 6.f * Kxy * v0 + 6.f * Kyz * v2 + 3.f * Kyzz + 3.f * Kzz * v1 -
                    2.f * rho * v1) / 72.f);
    k[12] = om * (-(3.f * Kxx * v2 + 3.f * Kxxz + 6.f * Kxz * v0 + 3.f * Kyy * v2 + 3.f * Kyyz + 6.f * Kyz * v1 -
                    2.f * rho * v2) / 72.f);
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
                    3.f * drho) / 36.f);
    om = S.om_fix[4];
    k[18] = om * (-(3.f * Kxx * v1sq + 3.f * Kxx * v2sq - 4.f * sxx + 6.f * Kxxy * v1 + 3.f * sxxyy +
                    6.f * Kxxz * v2 + 3.f * sxxzz + 12.f * Kxy * v0 * v1 + 6.f * Kxyy * v0 +
                    12.f * Kxz * v0 * v2 + 6.f * Kxzz * v0 + 3.f * Kyy * v0sq - 6.f * Kyy * v2sq + 2.f * syy -
                    12.f * Kyyz * v2 - 6.f * syyzz - 24.f * Kyz * v1 * v2 - 12.f * Kyzz * v1 + 3.f * Kzz * v0sq -
                    6.f * Kzz * v1sq + 2.f * szz - 2.f * rho * v0sq + rho * v1sq + rho * v2sq) / 72.f);
    k[19] = om * (-(3.f * Kxx * v1sq - 3.f * Kxx * v2sq + 6.f * Kxxy * v1 + 3.f * sxxyy - 6.f * Kxxz * v2 -
                    3.f * sxxzz + 12.f * Kxy * v0 * v1 + 6.f * Kxyy * v0 - 12.f * Kxz * v0 * v2 -
                    6.f * Kxzz * v0 + 3.f * Kyy * v0sq - 2.f * syy - 3.f * Kzz * v0sq + 2.f * szz - rho * v1sq +
                    rho * v2sq) / 24.f);
    om = S.om_fix[4];
    k[20] = om * (-(3.f * Kxx * v1 * v2 + 3.f * Kxxy * v2 + 3.f * Kxxyz + 3.f * Kxxz * v1 + 6.f * Kxy * v0 * v2 +
                    6.f * Kxyz * v0 + 6.f * Kxz * v0 * v1 + 3.f * Kyz * v0sq - 2.f * Kyz - rho * v1 * v2) / 24.f);
    k[21] = om * (-(6.f * Kxy * v1 * v2 + 3.f * Kxyy * v2 + 3.f * Kxyyz + 6.f * Kxyz * v1 + 3.f * Kxz * v1sq -
                    2.f * Kxz + 3.f * Kyy * v0 * v2 + 3.f * Kyyz * v0 + 6.f * Kyz * v0 * v1 - rho * v0 * v2) / 24.f);
    k[22] = om * (-(3.f * Kxy * v2sq - 2.f * Kxy + 6.f * Kxyz * v2 + 3.f * Kxyzz + 6.f * Kxz * v1 * v2 +
                    3.f * Kxzz * v1 + 6.f * Kyz * v0 * v2 + 3.f * Kyzz * v0 + 3.f * Kzz * v0 * v1 - rho * v0 * v1) /
                  24.f);
    om = S.om_fix[5];
    k[23] = om * (-(6.f * Kxy * v1 * v2sq - 4.f * Kxy * v1 + 3.f * Kxyy * v2sq - 2.f * Kxyy + 6.f * Kxyyz * v2 +
                    3.f * Kxyyzz + 12.f * Kxyz * v1 * v2 + 6.f * Kxyzz * v1 + 6.f * Kxz * v1sq * v2 -
                    4.f * Kxz * v2 + 3.f * Kxzz * v1sq - 2.f * Kxzz + 3.f * Kyy * v0 * v2sq - 2.f * Kyy * v0 +
                    6.f * K[0][2][1] * v0 * v2 + 3.f * Kyyzz * v0 + 12.f * Kyz * v0 * v1 * v2 +
                    6.f * Kyzz * v0 * v1 + 3.f * Kzz * v0 * v1sq - 2.f * Kzz * v0 - rho * v0 * v1sq -
                    rho * v0 * v2sq + rho * v0) / 24.f);
    k[24] = om * (-(3.f * Kxx * v1 * v2sq - 2.f * Kxx * v1 + 3.f * Kxxy * v2sq - 2.f * Kxxy + 6.f * Kxxyz * v2 +
                    3.f * Kxxyzz + 6.f * Kxxz * v1 * v2 + 3.f * Kxxzz * v1 + 6.f * Kxy * v0 * v2sq -
                    4.f * Kxy * v0 + 12.f * Kxyz * v0 * v2 + 6.f * Kxyzz * v0 + 12.f * Kxz * v0 * v1 * v2 +
                    6.f * Kxzz * v0 * v1 + 6.f * Kyz * v0sq * v2 - 4.f * Kyz * v2 + 3.f * Kyzz * v0sq -
                    2.f * Kyzz + 3.f * Kzz * v0sq * v1 - 2.f * Kzz * v1 - rho * v0sq * v1 - rho * v1 * v2sq +
                    rho * v1) / 24.f);
    k[25] = om * (-(3.f * Kxx * v1sq * v2 - 2.f * Kxx * v2 + 6.f * Kxxy * v1 * v2 + 3.f * Kxxyy * v2 +
                    3.f * Kxxyyz + 6.f * Kxxyz * v1 + 3.f * Kxxz * v1sq - 2.f * Kxxz + 12.f * Kxy * v0 * v1 * v2 +
                    6.f * Kxyy * v0 * v2 + 6.f * Kxyyz * v0 + 12.f * Kxyz * v0 * v1 + 6.f * Kxz * v0 * v1sq -
                    4.f * Kxz * v0 + 3.f * Kyy * v0sq * v2 - 2.f * Kyy * v2 + 3.f * Kyyz * v0sq - 2.f * Kyyz +
                    6.f * Kyz * v0sq * v1 - 4.f * Kyz * v1 - rho * v0sq * v2 - rho * v1sq * v2 + rho * v2) / 24.f);
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
                    7.f * drho) / 216.f);
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
                  2.f * (g[SE] + g[SW] + g[NE] + g[NW] - drho / 3.f)) / 12.f;
    k[4] = om * (g[N] + g[Sd] - g[E] - g[W] + rho * (u0 * u0 - u1 * u1)) / 4.f;
    k[5] = om * (g[NE] + g[SW] - g[NW] - g[SE] + rho * (u0 * u1)) / 4.f;
    {
        float t1 = (g[SE] + g[SW] - g[NE] - g[NW] - 2.f * u0 * u0 * u1 * rho +
                    u1 * (1.f / 3.f + (drho - g[N] - g[Sd] - g[R]))) / 4.f;
        float t2 = u0 / 2.f * (g[NE] - g[NW] - g[SE] + g[SW]);
        float t3 = -u1 / 2.f * (-3.f * k[3] - k[4]) - 2.f * u0 * k[5];
        k[6] = -idt * (t1 + t2) + t3;
    }
    {
        float t1 = (g[SW] + g[NW] - g[SE] - g[NE] - 2.f * u0 * u1 * u1 * rho +
                    u0 * (1.f / 3.f + (drho - g[W] - g[E] - g[R]))) / 4.f;
        float t2 = u1 / 2.f * (g[NE] + g[SW] - g[SE] - g[NW]);
        float t3 = -u0 / 2.f * (-3.f * k[3] + k[4]) - 2.f * u1 * k[5];
        k[7] = -idt * (t1 + t2) + t3;
    }
    {
        float t1 = drho / 9.f - g[NE] - g[NW] - g[SE] - g[SW];
        float t2 = 2.f * (u0 * (g[NE] - g[NW] + g[SE] - g[SW]) + u1 * (g[NE] + g[NW] - g[SE] - g[SW]));
        float t3 = 4.f * u0 * u1 * (g[NW] - g[NE] + g[SE] - g[SW]);
        float t4 = -u0 * u0 * (1.f / 3.f + (g[N] + g[NE] + g[NW] + g[Sd] + g[SE] + g[SW]));
        float t5 = u1 * u1 * (3.f * u0 * u0 * rho - (1.f / 3.f + (g[E] + g[NE] + g[NW] + g[SE] + g[SW] + g[W])));
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
#define NAGA_FOR_ITEMS(items, nitems)                                       \
    __shared__ SceneDev S;                                                  \
    for (int w_ = blockIdx.x; w_ < (nitems); w_ += gridDim.x) {             \
        const WorkItem it = (items)[w_];                                    \
        __syncthreads();                                                    \
        if (threadIdx.x == 0) S = scenes[it.scene];                         \
        __syncthreads();                                                    \
        const int64_t i = (int64_t)it.begin + threadIdx.x;                  \
        const bool active = i < (int64_t)it.end;

#define NAGA_END_ITEMS }

// rho, u; Q1 = (f~ + f~_prev) dt/2, Q2 = (Q1 + Q1_prev) dt/2
// (fluids/.../detail/pml_absorption.inl:531-631); layer sums of Q1, Q2
template <class L>
__global__ void __launch_bounds__(kBlock) k_macro_pml(const WorkItem* __restrict__ items, int nitems,
                                                      const SceneDev* __restrict__ scenes) {
    constexpr int Q = L::Q;
    __shared__ double red[kBlock / 32][2 * Q];
    NAGA_FOR_ITEMS(items, nitems)
    const int par = (int)(*S.step & 1ull);
    float* Q1cur = par ? S.Q1b : S.Q1a;
    const float* Q1prev = par ? S.Q1a : S.Q1b;
    const bool layer = active && i >= S.nb && i < S.nb + S.nl;
    float s1[Q], s2[Q];
    if (active) {
        float g[L::QP], q1p[L::QP], q1[L::QP];
        load_row_rw<L>(S.G, i, g);
        float drho, u[3] = {0.f, 0.f, 0.f};
        macros<L>(g, drho, u);
        const float4 mp = S.M[i];
        const float up[3] = {mp.y, mp.z, mp.w};
        S.M[i] = make_float4(drho, u[0], u[1], L::D == 3 ? u[2] : 0.f);
        load_row_rw<L>(Q1prev, i, q1p);
#pragma unroll
        for (int a = 0; a < Q; ++a) {
            const float ft = feq_c<L>(a, drho, u);
            const float ftp = feq_c<L>(a, mp.x, up);
            q1[a] = (ft + ftp) * S.dt_lat / 2.f;
            const float q2 = (q1[a] + q1p[a]) * S.dt_lat / 2.f;
            s1[a] = layer ? q1[a] : 0.f;
            s2[a] = layer ? q2 : 0.f;
        }
        store_row<L>(Q1cur, i, q1);
    } else {
#pragma unroll
        for (int a = 0; a < Q; ++a) s1[a] = s2[a] = 0.f;
    }
    // per-item layer sums in FP64, fixed order
    const bool touches = (int64_t)it.end > S.nb && (int64_t)it.begin < S.nb + S.nl;
    if (touches) {
        const int wid = threadIdx.x >> 5;
#pragma unroll
        for (int a = 0; a < Q; ++a) {
            double v1 = warp_sum((double)s1[a]);
            double v2 = warp_sum((double)s2[a]);
            if (lane_id() == 0) {
                red[wid][a] = v1;
                red[wid][Q + a] = v2;
            }
        }
    }
    __syncthreads();
    if (threadIdx.x < 2 * Q) {
        double v = 0.0;
        if (touches)
            for (int wv = 0; wv < kBlock / 32; ++wv) v += red[wv][threadIdx.x];
        S.partials[(int64_t)it.local * 2 * Q + threadIdx.x] = v;
    }
    NAGA_END_ITEMS
}

// layer means of Q1 and Q2 per scene (the reductions of
// pml_absorption.inl:776-836), summed in item order
template <int Q>
__global__ void k_pml_means(const SceneDev* __restrict__ scenes) {
    const SceneDev& S = scenes[blockIdx.x];
    const int t = threadIdx.x;
    if (t >= 2 * Q) return;
    double acc = 0.0;
    for (int it = 0; it < S.n_all_items; ++it) acc += S.partials[(int64_t)it * 2 * Q + t];
    S.means[t] = S.nl > 0 ? (float)acc / (float)S.nl : 0.f;
}

// probe densities (rho - rho0) from the RPIM probe weights
// (simulation_observers/density_observer.cuh:99-113)
__global__ void k_probe(const SceneDev* __restrict__ scenes) {
    const SceneDev& S = scenes[blockIdx.x];
    if (S.np == 0) return;
    const unsigned long long step = *S.step;
    const int slot = (int)(step % (unsigned long long)S.probe_cap);
    for (int p = threadIdx.x >> 5; p < S.np; p += blockDim.x >> 5) {
        float v = 0.f;
        for (int s = lane_id(); s < S.kp; s += 32) {
            const uint32_t j = S.pidx[(int64_t)s * S.np + p];
            v += S.pw[(int64_t)s * S.np + p] * S.M[j].x;
        }
        v = warp_sum(v);
        if (lane_id() == 0) S.probe_ring[(int64_t)slot * S.np + p] = v * S.rho0;
    }
}

// bulk + layer: s1 = g - sigma(3 f~ + 3 sigma Q1 + sigma^2 Q2)  (layer only)
//   + div(-2 c sigma (Q1 - <Q1>)) + div(c sigma^2 (Q2 - <Q2>))
//   [+ collision]  (pml_absorption.inl:770-855; simulation_engine.cuh:469-531)
template <class L>
__global__ void __launch_bounds__(kBlock) k_pml_collide(const WorkItem* __restrict__ items, int nitems,
                                                        const SceneDev* __restrict__ scenes) {
    constexpr int Q = L::Q;
    NAGA_FOR_ITEMS(items, nitems)
    if (active) {
        const int par = (int)(*S.step & 1ull);
        const float* Q1cur = par ? S.Q1b : S.Q1a;
        const float* Q1prev = par ? S.Q1a : S.Q1b;
        float acc[L::QP];
        load_row<L>(S.G, i, acc);
        float drho, u[3] = {0.f, 0.f, 0.f};
        macros<L>(acc, drho, u);
        float dcol[Q];
        collide<L>(acc, drho, u, S, dcol);
        const float hdt = S.half_dt;
        if (i >= S.nb && i < S.nb + S.nl) {
            const float sg = __ldg(S.sigma + (i - S.nb));
            float q1[L::QP], q1p[L::QP];
            load_row<L>(Q1cur, i, q1);
            load_row<L>(Q1prev, i, q1p);
#pragma unroll
            for (int a = 0; a < Q; ++a) {
                const float ft = feq_c<L>(a, drho, u);
                const float q2 = (q1[a] + q1p[a]) * S.dt_lat / 2.f;
                acc[a] -= sg * (3.f * ft + 3.f * sg * q1[a] + sg * sg * q2);
            }
        }
        (void)hdt;
        if (S.nl > 0) {
            float m1[Q], m2[Q];
#pragma unroll
            for (int a = 0; a < Q; ++a) {
                m1[a] = S.means[a];
                m2[a] = S.means[Q + a];
            }
            float div[Q];
#pragma unroll
            for (int a = 0; a < Q; ++a) div[a] = 0.f;
            for (int s = 0; s < S.k; ++s) {
                float wx, wy, wz;
                uint32_t j;
                stencil<L>(S, s, i, wx, wy, wz, j);
                if ((int64_t)j < S.nb || (int64_t)j >= S.nb + S.nl) continue;
                const float sg = __ldg(S.sigma + ((int64_t)j - S.nb));
                const int64_t jq = (int64_t)j - S.pml_shift;
                const float4* r1 = reinterpret_cast<const float4*>(Q1cur + jq * L::QP);
                const float4* r0 = reinterpret_cast<const float4*>(Q1prev + jq * L::QP);
#pragma unroll
                for (int c = 0; c < L::QP / 4; ++c) {
                    const float4 a4 = __ldg(r1 + c), b4 = __ldg(r0 + c);
                    const float qa[4] = {a4.x, a4.y, a4.z, a4.w};
                    const float qb[4] = {b4.x, b4.y, b4.z, b4.w};
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        const int a = 4 * c + e;
                        if (a >= Q) continue;
                        const float p = proj<L>(a, wx, wy, wz);
                        if (a == 0) continue;
                        const float q2 = (qa[e] + qb[e]) * S.dt_lat / 2.f;
                        const float phi = -2.f * sg * (qa[e] - m1[a]) + sg * sg * (q2 - m2[a]);
                        div[a] = fmaf(p, phi, div[a]);
                    }
                }
            }
#pragma unroll
            for (int a = 0; a < Q; ++a) acc[a] += div[a];
        }
        if (S.is_src[i]) store_row<L>(S.S1P, i, acc);
#pragma unroll
        for (int a = 0; a < Q; ++a) acc[a] += dcol[a];
        store_row<L>(S.S1, i, acc);
    }
    NAGA_END_ITEMS
}

// boundary: s1 = interp(s1 of bulk + layer, before collision) + collision;
// ghost: s1 = g + collision
template <class L>
__global__ void __launch_bounds__(kBlock) k_edge_collide(const WorkItem* __restrict__ items, int nitems,
                                                         const SceneDev* __restrict__ scenes) {
    constexpr int Q = L::Q;
    NAGA_FOR_ITEMS(items, nitems)
    if (active) {
        float g[L::QP];
        load_row<L>(S.G, i, g);
        float drho, u[3] = {0.f, 0.f, 0.f};
        macros<L>(g, drho, u);
        float dcol[Q];
        collide<L>(g, drho, u, S, dcol);
        float acc[L::QP];
        const int64_t b = i - S.nbl;
        if (b < S.nbd) {
#pragma unroll
            for (int a = 0; a < Q; ++a) acc[a] = 0.f;
            for (int s = 0; s < S.kb; ++s) {
                const uint32_t j = __ldg(S.bidx + (int64_t)s * S.nbd + b);
                const float w = __ldg(S.bw + (int64_t)s * S.nbd + b);
                float v[L::QP];
                load_row<L>(S.S1P, j, v);
#pragma unroll
                for (int a = 0; a < Q; ++a) acc[a] = fmaf(w, v[a], acc[a]);
            }
        } else {
#pragma unroll
            for (int a = 0; a < Q; ++a) acc[a] = g[a];
        }
#pragma unroll
        for (int a = 0; a < Q; ++a) acc[a] += dcol[a];
        store_row<L>(S.S1, i, acc);
    }
    NAGA_END_ITEMS
}

// bulk + layer: f = s1 + 0.75 sum_s w_s (s1_s - s1) (simulation_engine.cuh:
// 1233-1323); boundary: bounce-back f_a <- f_bb(a) where c_a . n > 0
// (:789-944); ghost: copy
template <class L>
__global__ void __launch_bounds__(kBlock) k_filter(const WorkItem* __restrict__ items, int nitems,
                                                   const SceneDev* __restrict__ scenes) {
    using T = Lat<L>;
    constexpr int Q = L::Q;
    NAGA_FOR_ITEMS(items, nitems)
    if (active) {
        float f[L::QP];
        load_row<L>(S.S1, i, f);
        float out[L::QP];
        if (i < S.nbl) {
            float sum[Q];
#pragma unroll
            for (int a = 0; a < Q; ++a) sum[a] = 0.f;
            for (int s = 0; s < S.k; ++s) {
                const float2 r = __ldg(S.stF + (int64_t)s * S.N + i);
                const uint32_t j = __float_as_uint(r.y);
                float v[L::QP];
                load_row<L>(S.S1, j, v);
#pragma unroll
                for (int a = 0; a < Q; ++a) sum[a] = fmaf(r.x, v[a] - f[a], sum[a]);
            }
#pragma unroll
            for (int a = 0; a < Q; ++a) out[a] = fmaf(0.75f, sum[a], f[a]);
        } else if (i - S.nbl < S.nbd) {
            const int64_t b = i - S.nbl;
            float n[3] = {0.f, 0.f, 0.f};
#pragma unroll
            for (int d = 0; d < L::D; ++d) n[d] = __ldg(S.normals + b * L::D + d);
#pragma unroll
            for (int a = 0; a < Q; ++a) {
                float cn = (float)T::cx(a) * n[0] + (float)T::cy(a) * n[1];
                if (L::D == 3) cn += (float)T::cz(a) * n[2];
                out[a] = cn > 0.f ? f[T::bb(a)] : f[a];
            }
        } else {
#pragma unroll
            for (int a = 0; a < Q; ++a) out[a] = f[a];
        }
        store_row<L>(S.G, i, out);
    }
    NAGA_END_ITEMS
}

// RK4 stage STAGE (detail/rk4_solver.cuh:48-171) with the streaming rates
// rate_a(i) = -sum_s (c_a . W_s) g_a(j_s) (pde_right_hand_side.cuh:82-176,
// divergence.cuh:377-488). Boundary and ghost nodes keep zero rates, so
// their stage values equal the step's start values (read from G).
template <class L, int STAGE>
__global__ void __launch_bounds__(kBlock) k_rk(const WorkItem* __restrict__ items, int nitems,
                                               const SceneDev* __restrict__ scenes) {
    constexpr int Q = L::Q;
    NAGA_FOR_ITEMS(items, nitems)
    if (active) {
        const float* src = (STAGE == 1) ? S.G : (STAGE == 2) ? S.G1 : (STAGE == 3) ? S.G2 : S.G1;
        float r[Q];
#pragma unroll
        for (int a = 0; a < Q; ++a) r[a] = 0.f;
        for (int s = 0; s < S.k; ++s) {
            float wx, wy, wz;
            uint32_t j;
            stencil<L>(S, s, i, wx, wy, wz, j);
            const float* row = ((int64_t)j < S.nbl ? src : S.G);
            float v[L::QP];
            load_row<L>(row, j, v);
#pragma unroll
            for (int a = 1; a < Q; ++a) r[a] = fmaf(proj<L>(a, wx, wy, wz), v[a], r[a]);
        }
        float f0[L::QP];
        load_row<L>(S.G, i, f0);
        float out[L::QP];
        if (STAGE == 1) {
            float acc[L::QP];
#pragma unroll
            for (int a = 0; a < Q; ++a) {
                const float kv = -r[a];
                out[a] = fmaf(S.a_half, kv, f0[a]);
                acc[a] = kv * S.b1;
            }
            store_row<L>(S.G1, i, out);
            store_row<L>(S.ACC, i, acc);
        } else {
            float acc[L::QP];
            load_row_rw<L>(S.ACC, i, acc);
            if (STAGE == 4) {
#pragma unroll
                for (int a = 0; a < Q; ++a) {
                    const float kv = -r[a];
                    const float df = acc[a] + kv * S.b1;
                    out[a] = fmaf(S.a_full, df, f0[a]);
                }
                store_row<L>(S.G, i, out);
            } else {
#pragma unroll
                for (int a = 0; a < Q; ++a) {
                    const float kv = -r[a];
                    out[a] = fmaf(STAGE == 2 ? S.a_half : S.a_full, kv, f0[a]);
                    acc[a] = acc[a] + kv * S.b2;
                }
                store_row<L>(STAGE == 2 ? S.G2 : S.G1, i, out);
                store_row<L>(S.ACC, i, acc);
            }
        }
    }
    NAGA_END_ITEMS
}

// boundary: f = interp(f of bulk + layer) (simulation_engine.cuh:1370)
template <class L>
__global__ void __launch_bounds__(kBlock) k_edge_interp(const WorkItem* __restrict__ items, int nitems,
                                                        const SceneDev* __restrict__ scenes) {
    constexpr int Q = L::Q;
    NAGA_FOR_ITEMS(items, nitems)
    const int64_t b = i - S.nbl;
    if (active && b < S.nbd) {
        float acc[L::QP];
#pragma unroll
        for (int a = 0; a < L::QP; ++a) acc[a] = 0.f;
        for (int s = 0; s < S.kb; ++s) {
            const uint32_t j = __ldg(S.bidx + (int64_t)s * S.nbd + b);
            const float w = __ldg(S.bw + (int64_t)s * S.nbd + b);
            float v[L::QP];
            load_row<L>(S.G, j, v);
#pragma unroll
            for (int a = 0; a < Q; ++a) acc[a] = fmaf(w, v[a], acc[a]);
        }
        store_row<L>(S.G, i, acc);
    }
    NAGA_END_ITEMS
}

__global__ void k_step_end(const SceneDev* __restrict__ scenes, int nscenes) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < nscenes) *scenes[s].step += 1ull;
}

}  // namespace

// ------------------------------------------------------------- launches
enum {
    K_MACRO = 0,
    K_MEANS,
    K_PROBE,
    K_PML,
    K_EDGE_COLLIDE,
    K_FILTER,
    K_RK1,
    K_RK2,
    K_RK3,
    K_RK4,
    K_EDGE_INTERP,
    K_STEP_END,
    K_COUNT
};

const char* kernel_name(int id) {
    static const char* names[K_COUNT] = {"macro_pml", "pml_means", "probe", "pml_collide", "edge_collide", "filter",
                                         "rk_stage1", "rk_stage2", "rk_stage3", "rk_stage4", "edge_interp",
                                         "step_end"};
    return (id >= 0 && id < K_COUNT) ? names[id] : "?";
}
int kernel_count() { return K_COUNT; }

template <class L>
int enqueue_step_t(const StepLaunch& P, cudaStream_t st) {
    const int cap = sm_count() * 8;
    auto grid = [&](int n) { return n < cap ? n : cap; };
    const bool prof = prof_on();
#define LAUNCH(id, n, ...)                      \
    if ((n) > 0) {                              \
        if (prof) prof_begin(id, st);           \
        __VA_ARGS__;                            \
        if (prof) prof_end(id, st);             \
    }
    LAUNCH(K_MACRO, P.n_all, (k_macro_pml<L><<<grid(P.n_all), kBlock, 0, st>>>(P.all, P.n_all, P.scenes)));
    LAUNCH(K_MEANS, P.nscenes, (k_pml_means<L::Q><<<P.nscenes, 64, 0, st>>>(P.scenes)));
    LAUNCH(K_PROBE, P.nscenes, (k_probe<<<P.nscenes, 128, 0, st>>>(P.scenes)));
    LAUNCH(K_PML, P.n_fluid, (k_pml_collide<L><<<grid(P.n_fluid), kBlock, 0, st>>>(P.fluid, P.n_fluid, P.scenes)));
    LAUNCH(K_EDGE_COLLIDE, P.n_edge,
           (k_edge_collide<L><<<grid(P.n_edge), kBlock, 0, st>>>(P.edge, P.n_edge, P.scenes)));
    LAUNCH(K_FILTER, P.n_all, (k_filter<L><<<grid(P.n_all), kBlock, 0, st>>>(P.all, P.n_all, P.scenes)));
    LAUNCH(K_RK1, P.n_fluid, (k_rk<L, 1><<<grid(P.n_fluid), kBlock, 0, st>>>(P.fluid, P.n_fluid, P.scenes)));
    LAUNCH(K_RK2, P.n_fluid, (k_rk<L, 2><<<grid(P.n_fluid), kBlock, 0, st>>>(P.fluid, P.n_fluid, P.scenes)));
    LAUNCH(K_RK3, P.n_fluid, (k_rk<L, 3><<<grid(P.n_fluid), kBlock, 0, st>>>(P.fluid, P.n_fluid, P.scenes)));
    LAUNCH(K_RK4, P.n_fluid, (k_rk<L, 4><<<grid(P.n_fluid), kBlock, 0, st>>>(P.fluid, P.n_fluid, P.scenes)));
    LAUNCH(K_EDGE_INTERP, P.n_edge,
           (k_edge_interp<L><<<grid(P.n_edge), kBlock, 0, st>>>(P.edge, P.n_edge, P.scenes)));
    LAUNCH(K_STEP_END, P.nscenes, (k_step_end<<<(P.nscenes + 127) / 128, 128, 0, st>>>(P.scenes, P.nscenes)));
#undef LAUNCH
    NAGA_CUDA_TRY(cudaGetLastError());
    return NAGA_OK;
}

int enqueue_step(int dim, const StepLaunch& P, cudaStream_t st) {
    return dim == 2 ? enqueue_step_t<D2Q9>(P, st) : enqueue_step_t<D3Q27>(P, st);
}

}  // namespace naga
