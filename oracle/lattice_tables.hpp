// Lattice tables and the central-moment collision of NAGA, restated for the
// CPU oracle. TEST INFRASTRUCTURE ONLY (see naga_oracle.h).
//
// The velocity sets, weights, collision matrices and the moment-projection
// formulas define the reference's collision model; they are data and algebra
// that must be alike for parity:
//   D3Q27: naga/fluids/nonlocal_lattice_boltzmann/detail/d3q27_lattice.cuh
//          velocities :45-55, weights :57-66, K :69-98, k formulas :125-378,
//          bounce-back map :380-387, central moment :390-412.
//   D2Q9:  detail/d2q9_lattice.cuh velocities :44-55, weights :57-68,
//          K :72-82, k formulas :120-299, bounce-back :142-155.
#pragma once
#include <cmath>

namespace orc {

// ---------------------------------------------------------------- D3Q27
static const int D3_C[27][3] = {
    {0, 0, 0},   {1, 0, 0},   {-1, 0, 0},  {0, 1, 0},   {0, -1, 0},
    {0, 0, 1},   {0, 0, -1},  {1, 1, 0},   {-1, 1, 0},  {1, -1, 0},
    {-1, -1, 0}, {1, 0, 1},   {-1, 0, 1},  {1, 0, -1},  {-1, 0, -1},
    {0, 1, 1},   {0, -1, 1},  {0, 1, -1},  {0, -1, -1}, {1, 1, 1},
    {-1, 1, 1},  {1, -1, 1},  {-1, -1, 1}, {1, 1, -1},  {-1, 1, -1},
    {1, -1, -1}, {-1, -1, -1}};

static const double D3_W[27] = {
    8. / 27.,  2. / 27.,  2. / 27.,  2. / 27.,  2. / 27.,  2. / 27.,  2. / 27.,
    1. / 54.,  1. / 54.,  1. / 54.,  1. / 54.,  1. / 54.,  1. / 54.,  1. / 54.,
    1. / 54.,  1. / 54.,  1. / 54.,  1. / 54.,  1. / 54.,  1. / 216., 1. / 216.,
    1. / 216., 1. / 216., 1. / 216., 1. / 216., 1. / 216., 1. / 216.};

static const int D3_BB[27] = {0,  2,  1,  4,  3,  6,  5,  10, 9,
                              8,  7,  14, 13, 12, 11, 18, 17, 16,
                              15, 26, 25, 24, 23, 22, 21, 20, 19};

// Collision matrix: row = population, column = moment increment k[j].
static const int D3_K[27][27] = {
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

// ----------------------------------------------------------------- D2Q9
// Direction order: rest, nw, w, sw, s, se, e, ne, n.
static const int D2_C[9][2] = {{0, 0},  {-1, 1}, {-1, 0}, {-1, -1}, {0, -1},
                               {1, -1}, {1, 0},  {1, 1},  {0, 1}};
static const double D2_W[9] = {4. / 9.,  1. / 36., 1. / 9.,  1. / 36., 1. / 9.,
                               1. / 36., 1. / 9.,  1. / 36., 1. / 9.};
enum { R_ = 0, NW_ = 1, W_ = 2, SW_ = 3, S_ = 4, SE_ = 5, E_ = 6, NE_ = 7, N_ = 8 };
static const int D2_BB[9] = {R_, SE_, E_, NE_, N_, NW_, W_, SW_, S_};
static const int D2_K[9][9] = {{1, 0, 0, -4, 0, 0, 0, 0, 4},
                               {1, -1, 1, 2, 0, 1, -1, 1, 1},
                               {1, -1, 0, -1, 1, 0, 0, -2, -2},
                               {1, -1, -1, 2, 0, -1, 1, 1, 1},
                               {1, 0, -1, -1, -1, 0, -2, 0, -2},
                               {1, 1, -1, 2, 0, 1, 1, -1, 1},
                               {1, 1, 0, -1, 1, 0, 0, 2, -2},
                               {1, 1, 1, 2, 0, -1, -1, -1, 1},
                               {1, 0, 1, -1, -1, 0, 2, 0, -2}};

// lattice speed of sound 1/sqrt(3), as lattices.cuh:46-49 spells it
template <class T>
inline T lattice_cs() {
    return static_cast<T>(0.57735026918962576450914878050196);
}

// x^m by repeated squaring as math.hpp:184-197 (m = 0 gives exactly 1)
template <class T>
inline T ipow(T x, int m) {
    if (m == 0) return T(1);
    if (m == 1) return x;
    T y = ipow(x, m / 2);
    return (m % 2 == 0) ? y * y : y * y * x;
}

// Central moment sum_a f_a (cx-ux)^m (cy-uy)^n (cz-uz)^p, accumulated in
// population order (d3q27_lattice.cuh:390-412).
template <class T>
inline T central_moment3(const T* f, const T* u, int m, int n, int p) {
    T sum = 0;
    for (int a = 0; a < 27; ++a) {
        sum += f[a] * ipow<T>(T(D3_C[a][0]) - u[0], m) *
               ipow<T>(T(D3_C[a][1]) - u[1], n) *
               ipow<T>(T(D3_C[a][2]) - u[2], p);
    }
    return sum;
}

// Relaxation rate for a fixed dimensionless omega (d3q27_lattice.cuh:200-321)
template <class T>
inline T fixed_rate(T omega_fixed, T dt) {
    T unit_nu = (T(1) / omega_fixed - T(0.5)) / T(3);
    return T(1) / (T(3) * unit_nu + T(0.5)) / dt;
}

// D3Q27 moment projection k[27] (d3q27_lattice.cuh:125-378).
template <class T>
void d3q27_projection(T* k, const T* f, T rho, const T* u, T nu, T dt) {
    k[0] = k[1] = k[2] = k[3] = 0;
    const T v0 = u[0], v1 = u[1], v2 = u[2];
    const T v0sq = v0 * v0, v1sq = v1 * v1, v2sq = v2 * v2;
    auto M = [&](int m, int n, int p) { return central_moment3<T>(f, u, m, n, p); };
    const T Kxy = M(1, 1, 0), Kxz = M(1, 0, 1), Kyz = M(0, 1, 1);
    const T Kxx = M(2, 0, 0), Kyy = M(0, 2, 0), Kzz = M(0, 0, 2);
    const T Kxxy = M(2, 1, 0), Kxxz = M(2, 0, 1), Kxyy = M(1, 2, 0);
    const T Kyyz = M(0, 2, 1), Kxzz = M(1, 0, 2), Kyzz = M(0, 1, 2);
    const T Kxyz = M(1, 1, 1), Kxyzz = M(1, 1, 2), Kxxyz = M(2, 1, 1);
    const T Kxyyz = M(1, 2, 1), Kxxyy = M(2, 2, 0), Kxxzz = M(2, 0, 2);
    const T Kyyzz = M(0, 2, 2), Kxxyzz = M(2, 1, 2), Kxyyzz = M(1, 2, 2);
    const T Kxxyyz = M(2, 2, 1), Kxxyyzz = M(2, 2, 2);

    T om = T(1) / (T(3) * nu + T(0.5)) / dt;
    k[4] = om * (-Kxy / 12);
    k[5] = om * (-Kxz / 12);
    k[6] = om * (-Kyz / 12);
    k[7] = om * (-(Kxx - Kyy) / 12);
    k[8] = om * (-(Kxx + Kyy - 2 * Kzz) / 36);
    k[9] = om * (-(Kxx + Kyy + Kzz - rho) / 18);

    om = fixed_rate<T>(T(1.5f), dt);
    k[10] = om * (-(6 * Kxy * v1 + 3 * Kxyy + 6 * Kxz * v2 + 3 * Kxzz + 3 * Kyy * v0 +
                    3 * Kzz * v0 - 2 * rho * v0) / 72);
    k[11] = om * (-(3 * Kxx * v1 + 3 * Kxxy + 6 * Kxy * v0 + 6 * Kyz * v2 + 3 * Kyzz +
                    3 * Kzz * v1 - 2 * rho * v1) / 72);
    k[12] = om * (-(3 * Kxx * v2 + 3 * Kxxz + 6 * Kxz * v0 + 3 * Kyy * v2 + 3 * Kyyz +
                    6 * Kyz * v1 - 2 * rho * v2) / 72);

    om = fixed_rate<T>(T(1.83f), dt);
    k[13] = om * (-(2 * Kxy * v1 + Kxyy - 2 * Kxz * v2 - Kxzz + Kyy * v0 - Kzz * v0) / 8);
    k[14] = om * (-(Kxx * v1 + Kxxy + 2 * Kxy * v0 - 2 * Kyz * v2 - Kyzz - Kzz * v1) / 8);
    k[15] = om * (-(Kxx * v2 + Kxxz + 2 * Kxz * v0 - Kyy * v2 - Kyyz - 2 * Kyz * v1) / 8);

    om = fixed_rate<T>(T(1.4f), dt);
    k[16] = om * (-(Kxy * v2 + Kxyz + Kxz * v1 + Kyz * v0) / 8);

    om = fixed_rate<T>(T(1.61f), dt);
    k[17] = om * (-(3 * Kxx * v1sq + 3 * Kxx * v2sq - 4 * Kxx + 6 * Kxxy * v1 + 3 * Kxxyy +
                    6 * Kxxz * v2 + 3 * Kxxzz + 12 * Kxy * v0 * v1 + 6 * Kxyy * v0 +
                    12 * Kxz * v0 * v2 + 6 * Kxzz * v0 + 3 * Kyy * v0sq + 3 * Kyy * v2sq -
                    4 * Kyy + 6 * Kyyz * v2 + 3 * Kyyzz + 12 * Kyz * v1 * v2 +
                    6 * Kyzz * v1 + 3 * Kzz * v0sq + 3 * Kzz * v1sq - 4 * Kzz -
                    2 * rho * v0sq - 2 * rho * v1sq - 2 * rho * v2sq + 3 * rho) / 36);

    om = fixed_rate<T>(T(1.98f), dt);
    k[18] = om * (-(3 * Kxx * v1sq + 3 * Kxx * v2sq - 4 * Kxx + 6 * Kxxy * v1 + 3 * Kxxyy +
                    6 * Kxxz * v2 + 3 * Kxxzz + 12 * Kxy * v0 * v1 + 6 * Kxyy * v0 +
                    12 * Kxz * v0 * v2 + 6 * Kxzz * v0 + 3 * Kyy * v0sq - 6 * Kyy * v2sq +
                    2 * Kyy - 12 * Kyyz * v2 - 6 * Kyyzz - 24 * Kyz * v1 * v2 -
                    12 * Kyzz * v1 + 3 * Kzz * v0sq - 6 * Kzz * v1sq + 2 * Kzz -
                    2 * rho * v0sq + rho * v1sq + rho * v2sq) / 72);
    k[19] = om * (-(3 * Kxx * v1sq - 3 * Kxx * v2sq + 6 * Kxxy * v1 + 3 * Kxxyy -
                    6 * Kxxz * v2 - 3 * Kxxzz + 12 * Kxy * v0 * v1 + 6 * Kxyy * v0 -
                    12 * Kxz * v0 * v2 - 6 * Kxzz * v0 + 3 * Kyy * v0sq - 2 * Kyy -
                    3 * Kzz * v0sq + 2 * Kzz - rho * v1sq + rho * v2sq) / 24);

    om = fixed_rate<T>(T(1.98f), dt);
    k[20] = om * (-(3 * Kxx * v1 * v2 + 3 * Kxxy * v2 + 3 * Kxxyz + 3 * Kxxz * v1 +
                    6 * Kxy * v0 * v2 + 6 * Kxyz * v0 + 6 * Kxz * v0 * v1 + 3 * Kyz * v0sq -
                    2 * Kyz - rho * v1 * v2) / 24);
    k[21] = om * (-(6 * Kxy * v1 * v2 + 3 * Kxyy * v2 + 3 * Kxyyz + 6 * Kxyz * v1 +
                    3 * Kxz * v1sq - 2 * Kxz + 3 * Kyy * v0 * v2 + 3 * Kyyz * v0 +
                    6 * Kyz * v0 * v1 - rho * v0 * v2) / 24);
    k[22] = om * (-(3 * Kxy * v2sq - 2 * Kxy + 6 * Kxyz * v2 + 3 * Kxyzz + 6 * Kxz * v1 * v2 +
                    3 * Kxzz * v1 + 6 * Kyz * v0 * v2 + 3 * Kyzz * v0 + 3 * Kzz * v0 * v1 -
                    rho * v0 * v1) / 24);

    om = fixed_rate<T>(T(1.74f), dt);
    k[23] = om * (-(6 * Kxy * v1 * v2sq - 4 * Kxy * v1 + 3 * Kxyy * v2sq - 2 * Kxyy +
                    6 * Kxyyz * v2 + 3 * Kxyyzz + 12 * Kxyz * v1 * v2 + 6 * Kxyzz * v1 +
                    6 * Kxz * v1sq * v2 - 4 * Kxz * v2 + 3 * Kxzz * v1sq - 2 * Kxzz +
                    3 * Kyy * v0 * v2sq - 2 * Kyy * v0 + 6 * Kyyz * v0 * v2 + 3 * Kyyzz * v0 +
                    12 * Kyz * v0 * v1 * v2 + 6 * Kyzz * v0 * v1 + 3 * Kzz * v0 * v1sq -
                    2 * Kzz * v0 - rho * v0 * v1sq - rho * v0 * v2sq + rho * v0) / 24);
    k[24] = om * (-(3 * Kxx * v1 * v2sq - 2 * Kxx * v1 + 3 * Kxxy * v2sq - 2 * Kxxy +
                    6 * Kxxyz * v2 + 3 * Kxxyzz + 6 * Kxxz * v1 * v2 + 3 * Kxxzz * v1 +
                    6 * Kxy * v0 * v2sq - 4 * Kxy * v0 + 12 * Kxyz * v0 * v2 + 6 * Kxyzz * v0 +
                    12 * Kxz * v0 * v1 * v2 + 6 * Kxzz * v0 * v1 + 6 * Kyz * v0sq * v2 -
                    4 * Kyz * v2 + 3 * Kyzz * v0sq - 2 * Kyzz + 3 * Kzz * v0sq * v1 -
                    2 * Kzz * v1 - rho * v0sq * v1 - rho * v1 * v2sq + rho * v1) / 24);
    k[25] = om * (-(3 * Kxx * v1sq * v2 - 2 * Kxx * v2 + 6 * Kxxy * v1 * v2 + 3 * Kxxyy * v2 +
                    3 * Kxxyyz + 6 * Kxxyz * v1 + 3 * Kxxz * v1sq - 2 * Kxxz +
                    12 * Kxy * v0 * v1 * v2 + 6 * Kxyy * v0 * v2 + 6 * Kxyyz * v0 +
                    12 * Kxyz * v0 * v1 + 6 * Kxz * v0 * v1sq - 4 * Kxz * v0 +
                    3 * Kyy * v0sq * v2 - 2 * Kyy * v2 + 3 * Kyyz * v0sq - 2 * Kyyz +
                    6 * Kyz * v0sq * v1 - 4 * Kyz * v1 - rho * v0sq * v2 - rho * v1sq * v2 +
                    rho * v2) / 24);
    k[26] = om * (-(27 * Kxx * v1sq * v2sq - 18 * Kxx * v1sq - 18 * Kxx * v2sq + 12 * Kxx +
                    54 * Kxxy * v1 * v2sq - 36 * Kxxy * v1 + 27 * Kxxyy * v2sq -
                    18 * Kxxyy + 54 * Kxxyyz * v2 + 27 * Kxxyyzz + 108 * Kxxyz * v1 * v2 +
                    54 * Kxxyzz * v1 + 54 * Kxxz * v1sq * v2 - 36 * Kxxz * v2 +
                    27 * Kxxzz * v1sq - 18 * Kxxzz + 108 * Kxy * v0 * v1 * v2sq -
                    72 * Kxy * v0 * v1 + 54 * Kxyy * v0 * v2sq - 36 * Kxyy * v0 +
                    108 * Kxyyz * v0 * v2 + 54 * Kxyyzz * v0 + 216 * Kxyz * v0 * v1 * v2 +
                    108 * Kxyzz * v0 * v1 + 108 * Kxz * v0 * v1sq * v2 - 72 * Kxz * v0 * v2 +
                    54 * Kxzz * v0 * v1sq - 36 * Kxzz * v0 + 27 * Kyy * v0sq * v2sq -
                    18 * Kyy * v0sq - 18 * Kyy * v2sq + 12 * Kyy + 54 * Kyyz * v0sq * v2 -
                    36 * Kyyz * v2 + 27 * Kyyzz * v0sq - 18 * Kyyzz +
                    108 * Kyz * v0sq * v1 * v2 - 72 * Kyz * v1 * v2 + 54 * Kyzz * v0sq * v1 -
                    36 * Kyzz * v1 + 27 * Kzz * v0sq * v1sq - 18 * Kzz * v0sq -
                    18 * Kzz * v1sq + 12 * Kzz - 9 * rho * v0sq * v1sq -
                    9 * rho * v0sq * v2sq + 9 * rho * v0sq - 9 * rho * v1sq * v2sq +
                    9 * rho * v1sq + 9 * rho * v2sq - 7 * rho) / 216);
}

// D2Q9 moment projection k[9] (d2q9_lattice.cuh:120-299).
template <class T>
void d2q9_projection(T* k, const T* f, T rho, const T* u, T nu, T dt) {
    const T om = T(1) / (T(3) * nu + T(0.5) * dt);
    const T inv_dt = T(1) / dt;
    const T u0 = u[0], u1 = u[1];
    k[0] = k[1] = k[2] = 0;
    k[3] = inv_dt *
           (rho * (u0 * u0 + u1 * u1) - f[E_] - f[N_] - f[S_] - f[W_] -
            2 * (f[SE_] + f[SW_] + f[NE_] + f[NW_] - rho / T(3))) /
           T(12);
    k[4] = om * (f[N_] + f[S_] - f[E_] - f[W_] + rho * (u0 * u0 - u1 * u1)) / T(4);
    k[5] = om * (f[NE_] + f[SW_] - f[NW_] - f[SE_] + rho * (u0 * u1)) / T(4);
    {
        T t1 = (f[SE_] + f[SW_] - f[NE_] - f[NW_] - 2 * u0 * u0 * u1 * rho +
                u1 * (rho - f[N_] - f[S_] - f[R_])) / T(4);
        T t2 = u0 / T(2) * (f[NE_] - f[NW_] - f[SE_] + f[SW_]);
        T t3 = -u1 / T(2) * (-3 * k[3] - k[4]) - 2 * u0 * k[5];
        k[6] = -inv_dt * (t1 + t2) + t3;
    }
    {
        T t1 = (f[SW_] + f[NW_] - f[SE_] - f[NE_] - 2 * u0 * u1 * u1 * rho +
                u0 * (rho - f[W_] - f[E_] - f[R_])) / T(4);
        T t2 = u1 / T(2) * (f[NE_] + f[SW_] - f[SE_] - f[NW_]);
        T t3 = -u0 / T(2) * (-3 * k[3] + k[4]) - 2 * u1 * k[5];
        k[7] = -inv_dt * (t1 + t2) + t3;
    }
    {
        T t1 = rho / T(9) - f[NE_] - f[NW_] - f[SE_] - f[SW_];
        T t2 = 2 * (u0 * (f[NE_] - f[NW_] + f[SE_] - f[SW_]) +
                    u1 * (f[NE_] + f[NW_] - f[SE_] - f[SW_]));
        T t3 = 4 * u0 * u1 * (f[NW_] - f[NE_] + f[SE_] - f[SW_]);
        T t4 = -u0 * u0 * (f[N_] + f[NE_] + f[NW_] + f[S_] + f[SE_] + f[SW_]);
        T t5 = u1 * u1 * (3 * u0 * u0 * rho - f[E_] - f[NE_] - f[NW_] - f[SE_] - f[SW_] - f[W_]);
        T t6 = -2 * k[3] - 2 * u0 * k[7] - 2 * u1 * k[6] + 4 * u0 * u1 * k[5] -
               (T(3) / T(2) * k[3] - k[4] / T(2)) * (u0 * u0 + u1 * u1);
        k[8] = inv_dt * (T(1) / T(4) * (t1 + t2 + t3 + t4 + t5)) + t6;
    }
}

}  // namespace orc
