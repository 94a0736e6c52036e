// CPU oracle for the NAGA nonlocal LBM acoustics step.
// TEST INFRASTRUCTURE ONLY: the reference the CUDA product is tested against. See
// naga_oracle.h for what may call it. Build with -ffp-contract=off so that
// FP32 distances match the reference formula bit for bit.
//
// Parity status: the step restates NAGA's D3Q27 engine; nothing in the
// reference pins step values (the reference cannot be built here: its
// runtime submodule is empty), so the step is anchored on the reference's
// known-answer programs (3x3 inverse, exact kNN sets, analytic RPIM and
// divergence fields) and on the algebra of the cited files.

#include "naga_oracle.h"
#include "lattice_tables.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <numeric>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

// ====================================================== distances / kNN
// Squared distance as distance_functions.hpp:138-161: the highest dimension
// is added last: d2 = dz^2 + (dy^2 + dx^2). Requires -ffp-contract=off.
static inline float dist2f(const float* a, const float* b, int dim) {
    float s = (a[0] - b[0]) * (a[0] - b[0]);
    for (int d = 1; d < dim; ++d) {
        float t = (a[d] - b[d]) * (a[d] - b[d]);
        s = t + s;
    }
    return s;
}

struct Cand {
    float d2;
    uint32_t idx;
};
static inline bool cand_less(const Cand& a, const Cand& b) {
    return a.d2 < b.d2 || (a.d2 == b.d2 && a.idx < b.idx);
}

// keeps the k smallest candidates, sorted ascending
struct KBest {
    int k, n = 0;
    Cand* c;
    void offer(float d2, uint32_t idx) {
        Cand x{d2, idx};
        if (n == k && !cand_less(x, c[k - 1])) return;
        int pos = (n < k) ? n++ : k - 1;
        while (pos > 0 && cand_less(x, c[pos - 1])) {
            c[pos] = c[pos - 1];
            --pos;
        }
        c[pos] = x;
    }
};

static void knn_brute(const float* src, int64_t n, const float* q, int64_t nq, int dim,
                      int k, uint32_t* idx, float* d2) {
#pragma omp parallel
    {
        std::vector<Cand> buf(k);
#pragma omp for schedule(static)
        for (int64_t i = 0; i < nq; ++i) {
            KBest kb{k, 0, buf.data()};
            for (int64_t j = 0; j < n; ++j) kb.offer(dist2f(q + i * dim, src + j * dim, dim), (uint32_t)j);
            for (int s = 0; s < k; ++s) {
                idx[i * k + s] = s < kb.n ? buf[s].idx : 0xffffffffu;
                d2[i * k + s] = s < kb.n ? buf[s].d2 : INFINITY;
            }
        }
    }
}

// Exact search over a uniform cell grid, expanding Chebyshev shells until
// the k-th candidate is strictly closer than anything outside the searched
// block (the bound carries a relative margin that covers FP32 rounding).
static void knn_grid(const float* src, int64_t n, const float* q, int64_t nq, int dim,
                     int k, uint32_t* idx, float* d2) {
    double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    for (int d = 0; d < dim; ++d) {
        lo[d] = INFINITY;
        hi[d] = -INFINITY;
    }
    for (int64_t j = 0; j < n; ++j)
        for (int d = 0; d < dim; ++d) {
            lo[d] = std::min(lo[d], (double)src[j * dim + d]);
            hi[d] = std::max(hi[d], (double)src[j * dim + d]);
        }
    double vol = 1;
    for (int d = 0; d < dim; ++d) {
        if (hi[d] - lo[d] < 1e-6) hi[d] = lo[d] + 1e-6;
        vol *= hi[d] - lo[d];
    }
    double w = std::pow(2.0 * vol / (double)std::max<int64_t>(n, 1), 1.0 / dim);
    int64_t dims[3] = {1, 1, 1};
    for (int d = 0; d < dim; ++d) dims[d] = std::max<int64_t>(1, (int64_t)std::ceil((hi[d] - lo[d]) / w));
    auto cell_of = [&](const float* p, int64_t* c) {
        for (int d = 0; d < dim; ++d) {
            int64_t v = (int64_t)std::floor(((double)p[d] - lo[d]) / w);
            c[d] = std::min(std::max<int64_t>(v, 0), dims[d] - 1);
        }
    };
    int64_t ncell = dims[0] * dims[1] * dims[2];
    std::vector<int64_t> start(ncell + 1, 0);
    std::vector<int64_t> cell(n);
    for (int64_t j = 0; j < n; ++j) {
        int64_t c[3] = {0, 0, 0};
        cell_of(src + j * dim, c);
        cell[j] = c[0] + dims[0] * (c[1] + dims[1] * c[2]);
        start[cell[j] + 1]++;
    }
    for (int64_t c = 0; c < ncell; ++c) start[c + 1] += start[c];
    std::vector<uint32_t> order(n);
    {
        std::vector<int64_t> fill(start.begin(), start.end() - 1);
        for (int64_t j = 0; j < n; ++j) order[fill[cell[j]]++] = (uint32_t)j;
    }
#pragma omp parallel
    {
        std::vector<Cand> buf(k);
#pragma omp for schedule(dynamic, 64)
        for (int64_t i = 0; i < nq; ++i) {
            const float* p = q + i * dim;
            int64_t c0[3] = {0, 0, 0};
            cell_of(p, c0);
            KBest kb{k, 0, buf.data()};
            for (int64_t r = 0;; ++r) {
                int64_t lo_c[3], hi_c[3];
                for (int d = 0; d < 3; ++d) {
                    lo_c[d] = d < dim ? c0[d] - r : 0;
                    hi_c[d] = d < dim ? c0[d] + r : 0;
                }
                for (int64_t z = std::max<int64_t>(lo_c[2], 0); z <= std::min(hi_c[2], dims[2] - 1); ++z)
                    for (int64_t y = std::max<int64_t>(lo_c[1], 0); y <= std::min(hi_c[1], dims[1] - 1); ++y)
                        for (int64_t x = std::max<int64_t>(lo_c[0], 0); x <= std::min(hi_c[0], dims[0] - 1); ++x) {
                            bool shell = (x == lo_c[0] || x == hi_c[0]) ||
                                         (dim > 1 && (y == lo_c[1] || y == hi_c[1])) ||
                                         (dim > 2 && (z == lo_c[2] || z == hi_c[2]));
                            if (!shell) continue;
                            int64_t cid = x + dims[0] * (y + dims[1] * z);
                            for (int64_t t = start[cid]; t < start[cid + 1]; ++t) {
                                uint32_t j = order[t];
                                kb.offer(dist2f(p, src + (int64_t)j * dim, dim), j);
                            }
                        }
                // distance from p to the nearest face of the block that does
                // not already reach the edge of the grid
                double bound = INFINITY;
                bool all_covered = true;
                for (int d = 0; d < dim; ++d) {
                    if (lo_c[d] > 0) {
                        all_covered = false;
                        bound = std::min(bound, (double)p[d] - (lo[d] + (double)lo_c[d] * w));
                    }
                    if (hi_c[d] < dims[d] - 1) {
                        all_covered = false;
                        bound = std::min(bound, (lo[d] + (double)(hi_c[d] + 1) * w) - (double)p[d]);
                    }
                }
                if (all_covered) break;
                if (kb.n == k && bound > 0 && (double)buf[k - 1].d2 < bound * bound * (1.0 - 1e-5)) break;
            }
            for (int s = 0; s < k; ++s) {
                idx[i * k + s] = s < kb.n ? buf[s].idx : 0xffffffffu;
                d2[i * k + s] = s < kb.n ? buf[s].d2 : INFINITY;
            }
        }
    }
}

// Restatement of NAGA's own search, used only to show that it returns the
// same neighbour SETS as the exact search on the benchmark clouds.
// Cells: nd_cubic_segmentation.cuh:227-303 (FP32 bounds, +1e-3 on a
// degenerate axis, width = (approx / N * volume)^(1/D), shape = ceil(extent /
// width)) and get_partition_index :376-392. Search:
// nearest_neighbors.cuh:207-411 -- Chebyshev rings r = 0, 1, ...; the first k
// candidates are appended and then sorted (insertion_sort :59-93), later ones
// replace the last entry only when strictly closer; the search continues
// while the previous ring added a first-k candidate or fewer than k are
// known, and stops at radius max((shape + 1) / 2). The reference visits the
// cells of a ring in a pseudo-random order and a cell's points in the order
// its atomic scatter left them; here both are in index order, which can
// change the result only where candidates tie at the k-th distance. The
// cell index is clamped to the grid (the reference's floor can reach `shape`
// through rounding).
struct CubicSeg {
    int dim = 0;
    float lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0}, w = 0;
    int64_t shape[3] = {1, 1, 1};
    std::vector<int64_t> start;  // [cells + 1], exclusive prefix sums of the sizes
    std::vector<uint32_t> order; // point indices grouped by cell, ascending within a cell
    void cell_of(const float* p, int64_t* c) const {
        for (int d = 0; d < dim; ++d) {
            if (p[d] < lo[d]) c[d] = 0;
            else if (p[d] >= hi[d]) c[d] = shape[d] - 1;
            else c[d] = std::min<int64_t>((int64_t)std::floor((p[d] - lo[d]) / w), shape[d] - 1);
        }
    }
};

static void cubic_segmentation(const float* src, int64_t n, int dim, int approx, CubicSeg& S) {
    S.dim = dim;
    for (int d = 0; d < dim; ++d) {
        S.lo[d] = INFINITY;
        S.hi[d] = -INFINITY;
    }
    for (int64_t j = 0; j < n; ++j)
        for (int d = 0; d < dim; ++d) {
            S.lo[d] = std::min(S.lo[d], src[j * dim + d]);
            S.hi[d] = std::max(S.hi[d], src[j * dim + d]);
        }
    const float tol = 1e-3f;
    float vol = 1.0f;
    for (int d = 0; d < dim; ++d) {
        if (S.hi[d] - S.lo[d] < tol) S.hi[d] = S.lo[d] + tol;
        vol *= S.hi[d] - S.lo[d];
    }
    S.w = std::pow((float)approx / (float)n * vol, 1.0f / (float)dim);
    for (int d = 0; d < dim; ++d) {
        S.shape[d] = (int64_t)std::ceil((S.hi[d] - S.lo[d]) / S.w);
        S.hi[d] = S.lo[d] + (float)S.shape[d] * S.w;
    }
    const int64_t ncell = S.shape[0] * S.shape[1] * S.shape[2];
    S.start.assign(ncell + 1, 0);
    std::vector<int64_t> cell(n);
    for (int64_t j = 0; j < n; ++j) {
        int64_t c[3] = {0, 0, 0};
        S.cell_of(src + j * dim, c);
        cell[j] = c[0] + S.shape[0] * (c[1] + S.shape[1] * c[2]);
        S.start[cell[j] + 1]++;
    }
    for (int64_t c = 0; c < ncell; ++c) S.start[c + 1] += S.start[c];
    S.order.assign(n, 0);
    std::vector<int64_t> fill(S.start.begin(), S.start.end() - 1);
    for (int64_t j = 0; j < n; ++j) S.order[fill[cell[j]]++] = (uint32_t)j;
}

static void knn_ring_reference(const float* src, int64_t n, const float* q, int64_t nq, int dim,
                               int k, int approx, uint32_t* idx, float* d2) {
    CubicSeg S;
    cubic_segmentation(src, n, dim, approx, S);
    const int64_t* shape = S.shape;
    const std::vector<int64_t>& start = S.start;
    const std::vector<uint32_t>& order = S.order;
    auto cell_of = [&](const float* p, int64_t* c) { S.cell_of(p, c); };
    int64_t max_r = 0;
    for (int d = 0; d < dim; ++d) max_r = std::max<int64_t>(max_r, (shape[d] + 1) / 2);
#pragma omp parallel
    {
        std::vector<float> bd(k);
        std::vector<uint32_t> bi(k);
#pragma omp for schedule(dynamic, 64)
        for (int64_t i = 0; i < nq; ++i) {
            const float* p = q + i * dim;
            int64_t c0[3] = {0, 0, 0};
            cell_of(p, c0);
            int nf = 0;
            bool fresh = true;
            for (int64_t r = 0; (fresh || nf < k) && r <= max_r; ++r) {
                fresh = false;
                int64_t a[3], b[3];
                for (int d = 0; d < 3; ++d) {
                    a[d] = d < dim ? c0[d] - r : 0;
                    b[d] = d < dim ? c0[d] + r : 0;
                }
                for (int64_t z = std::max<int64_t>(a[2], 0); z <= std::min(b[2], shape[2] - 1); ++z)
                    for (int64_t y = std::max<int64_t>(a[1], 0); y <= std::min(b[1], shape[1] - 1); ++y)
                        for (int64_t x = std::max<int64_t>(a[0], 0); x <= std::min(b[0], shape[0] - 1); ++x) {
                            bool shell = x == a[0] || x == b[0] || (dim > 1 && (y == a[1] || y == b[1])) ||
                                         (dim > 2 && (z == a[2] || z == b[2]));
                            if (!shell) continue;
                            int64_t cid = x + shape[0] * (y + shape[1] * z);
                            for (int64_t t = start[cid]; t < start[cid + 1]; ++t) {
                                const uint32_t j = order[t];
                                const float dd = dist2f(p, src + (int64_t)j * dim, dim);
                                if (nf < k) {
                                    bd[nf] = dd;
                                    bi[nf] = j;
                                    if (++nf == k) {
                                        for (int u = 1; u < k; ++u) {  // stable insertion sort
                                            float kd = bd[u];
                                            uint32_t ki = bi[u];
                                            int v = u - 1;
                                            for (; v >= 0 && bd[v] > kd; --v) {
                                                bd[v + 1] = bd[v];
                                                bi[v + 1] = bi[v];
                                            }
                                            bd[v + 1] = kd;
                                            bi[v + 1] = ki;
                                        }
                                    }
                                    fresh = true;
                                } else if (dd < bd[k - 1]) {
                                    int v = k - 1;
                                    for (; v > 0 && bd[v - 1] > dd; --v) {
                                        bd[v] = bd[v - 1];
                                        bi[v] = bi[v - 1];
                                    }
                                    bd[v] = dd;
                                    bi[v] = j;
                                }
                            }
                        }
            }
            for (int s = 0; s < k; ++s) {
                idx[i * k + s] = s < nf ? bi[s] : 0xffffffffu;
                d2[i * k + s] = s < nf ? bd[s] : INFINITY;
            }
        }
    }
}

// ================================================================== LU
// LU with partial pivoting (first row of maximal |a| in the column), as
// LAPACK getrf; cuBLAS {S,D}getrfBatched is called with these semantics at
// linalg/batched_matrix_inverse.cuh:229-250. A is n x n column-major.
static int lu_factor(double* A, int n, int* piv) {
    int info = 0;
    for (int j = 0; j < n; ++j) {
        int p = j;
        double best = std::fabs(A[j + n * j]);
        for (int i = j + 1; i < n; ++i)
            if (std::fabs(A[i + n * j]) > best) {
                best = std::fabs(A[i + n * j]);
                p = i;
            }
        piv[j] = p;
        if (A[p + n * j] == 0.0) {
            if (!info) info = j + 1;
            continue;
        }
        if (p != j)
            for (int c = 0; c < n; ++c) std::swap(A[j + n * c], A[p + n * c]);
        double inv = 1.0 / A[j + n * j];
        for (int i = j + 1; i < n; ++i) A[i + n * j] *= inv;
        for (int c = j + 1; c < n; ++c) {
            double a = A[j + n * c];
            if (a == 0.0) continue;
            for (int i = j + 1; i < n; ++i) A[i + n * c] -= A[i + n * j] * a;
        }
    }
    return info;
}

// solve A x = b in place with the factors of lu_factor (b: n x nrhs col-major)
static void lu_solve(const double* LU, int n, const int* piv, double* b, int nrhs) {
    for (int r = 0; r < nrhs; ++r) {
        double* x = b + (size_t)n * r;
        for (int j = 0; j < n; ++j)
            if (piv[j] != j) std::swap(x[j], x[piv[j]]);
        for (int j = 0; j < n; ++j)
            for (int i = j + 1; i < n; ++i) x[i] -= LU[i + n * j] * x[j];
        for (int j = n - 1; j >= 0; --j) {
            x[j] /= LU[j + n * j];
            for (int i = 0; i < j; ++i) x[i] -= LU[i + n * j] * x[j];
        }
    }
}

// ======================================================== RBF (RPIM)
// Shape functions of interpolation/radial_point_method.cuh:44-66 (MQ,
// q = 0.5, alpha_c = 0.1) and the cubic polyharmonic spline; evaluated in
// coordinates centred on the group's node and scaled by the spacing. Both
// shapes are radial, so the interpolation weights are invariant under the
// shift and the uniform scale (the RBF block scales by a constant factor and
// the linear monomial space is shift- and scale-invariant); the scaled
// system is far better conditioned in finite precision.
static inline double shape_fn(double r2, int shape) {
    if (shape == 0) return std::sqrt(r2 + 0.1 * 0.1);
    double r = std::sqrt(r2);
    return r * r * r;
}

// Augmented moment matrix G0 = [[Phi, P], [P^T, 0]], P = [1, x]
// (interpolation/detail/radial_point_method.cuh:390-431). xs: k scaled points.
static void build_G0(const double* xs, int k, int dim, int shape, double* G) {
    int n = k + dim + 1;
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
            double v;
            if (i >= k && j >= k)
                v = 0;
            else if (i >= k)
                v = (i == k) ? 1.0 : xs[j * dim + (i - k - 1)];
            else if (j >= k)
                v = (j == k) ? 1.0 : xs[i * dim + (j - k - 1)];
            else {
                double r2 = 0;
                for (int d = 0; d < dim; ++d) {
                    double t = xs[i * dim + d] - xs[j * dim + d];
                    r2 += t * t;
                }
                v = shape_fn(r2, shape);
            }
            G[i + n * j] = v;
        }
}

// G_x = [phi(|x - x_s|); 1; x] (radial_point_method detail :433-453)
static void build_Gx(const double* xs, int k, int dim, int shape, const double* x, double* g) {
    for (int s = 0; s < k; ++s) {
        double r2 = 0;
        for (int d = 0; d < dim; ++d) {
            double t = xs[s * dim + d] - x[d];
            r2 += t * t;
        }
        g[s] = shape_fn(r2, shape);
    }
    g[k] = 1.0;
    for (int d = 0; d < dim; ++d) g[k + 1 + d] = x[d];
}

}  // namespace orc

using namespace orc;

extern "C" int orc_knn(const float* src, int64_t n, const float* qry, int64_t nq, int dim, int k,
                       int grid, uint32_t* idx, float* d2) {
    if (dim < 1 || dim > 3 || k < 1 || n < 0 || nq < 0) return 1;
    if (grid)
        knn_grid(src, n, qry, nq, dim, k, idx, d2);
    else
        knn_brute(src, n, qry, nq, dim, k, idx, d2);
    return 0;
}

extern "C" int orc_cubic_segmentation(const float* src, int64_t n, int dim, int approx, float* lower,
                                      float* upper, float* width, int64_t* shape, int64_t* n_cells,
                                      uint32_t* sizes, uint32_t* offsets, uint32_t* indices) {
    if (n < 1 || (dim != 2 && dim != 3) || approx < 1) return 1;
    orc::CubicSeg S;
    orc::cubic_segmentation(src, n, dim, approx, S);
    const int64_t cells = S.shape[0] * S.shape[1] * S.shape[2];
    for (int d = 0; d < dim; ++d) {
        if (lower) lower[d] = S.lo[d];
        if (upper) upper[d] = S.hi[d];
        if (shape) shape[d] = S.shape[d];
    }
    if (width) *width = S.w;
    if (n_cells) *n_cells = cells;
    for (int64_t c = 0; c < cells; ++c) {
        if (sizes) sizes[c] = (uint32_t)(S.start[c + 1] - S.start[c]);
        if (offsets) offsets[c] = (uint32_t)S.start[c];
    }
    if (indices) std::copy(S.order.begin(), S.order.end(), indices);
    return 0;
}

extern "C" int orc_knn_ring_reference(const float* src, int64_t n, const float* qry, int64_t nq,
                                      int dim, int k, int approx, uint32_t* idx, float* d2) {
    if (dim < 1 || dim > 3 || k < 1 || n < 1 || nq < 0 || approx < 1) return 1;
    knn_ring_reference(src, n, qry, nq, dim, k, approx, idx, d2);
    return 0;
}

// explicit inverse via the LU factors (getri semantics: inv(A) from getrf)
extern "C" int orc_batched_inverse_f64(const double* A, int n, int64_t batch, double* Ainv,
                                       int* info) {
    if (n < 1 || batch < 0) return 1;
#pragma omp parallel
    {
        std::vector<double> LU((size_t)n * n);
        std::vector<int> piv(n);
#pragma omp for schedule(static)
        for (int64_t b = 0; b < batch; ++b) {
            std::memcpy(LU.data(), A + (size_t)b * n * n, sizeof(double) * n * n);
            int inf = lu_factor(LU.data(), n, piv.data());
            if (info) info[b] = inf;
            double* X = Ainv + (size_t)b * n * n;
            for (int c = 0; c < n; ++c)
                for (int r = 0; r < n; ++r) X[r + n * c] = (r == c) ? 1.0 : 0.0;
            if (inf == 0) lu_solve(LU.data(), n, piv.data(), X, n);
        }
    }
    return 0;
}

// Weights w_s(x) = sum_j (G0^-1)_{j,s} G_x(j) for every query of a group
// (interpolation/detail/radial_point_method.cuh:92-472), FP64.
extern "C" int orc_rbf_weights(const float* src, int64_t n, int dim, const uint32_t* support, int k,
                               const double* qry, int64_t ngroups, int group, double spacing,
                               int shape, double* weights) {
    if (dim < 1 || dim > 3 || k < 1 || group < 1 || !(spacing > 0)) return 1;
    int nn = k + dim + 1;
    int bad = 0;
#pragma omp parallel
    {
        std::vector<double> xs((size_t)k * dim), G((size_t)nn * nn), rhs((size_t)nn * group), xq(dim);
        std::vector<int> piv(nn);
#pragma omp for schedule(static) reduction(| : bad)
        for (int64_t g = 0; g < ngroups; ++g) {
            const uint32_t* sup = support + g * k;
            // centre: first query point of the group
            const double* o = qry + (g * group) * dim;
            for (int s = 0; s < k; ++s) {
                if ((int64_t)sup[s] >= n) bad = 1;
                for (int d = 0; d < dim; ++d)
                    xs[s * dim + d] = ((double)src[(int64_t)sup[s] * dim + d] - o[d]) / spacing;
            }
            build_G0(xs.data(), k, dim, shape, G.data());
            for (int q = 0; q < group; ++q) {
                for (int d = 0; d < dim; ++d) xq[d] = (qry[(g * group + q) * dim + d] - o[d]) / spacing;
                build_Gx(xs.data(), k, dim, shape, xq.data(), rhs.data() + (size_t)nn * q);
            }
            if (lu_factor(G.data(), nn, piv.data()) != 0) bad = 1;
            lu_solve(G.data(), nn, piv.data(), rhs.data(), group);
            for (int q = 0; q < group; ++q)
                for (int s = 0; s < k; ++s) weights[(g * group + q) * k + s] = rhs[(size_t)nn * q + s];
        }
    }
    return bad ? 2 : 0;
}

// ============================================== divergence stencil build
namespace orc {
// 4-point Gauss-Legendre nodes and weights with the six-digit values of
// nonlocal_calculus/detail/quadrature_points.cuh:49-61.
static const double GL_W[4] = {0.652145, 0.652145, 0.347855, 0.347855};
static const double GL_X[4] = {0.339981, -0.339981, 0.861136, -0.861136};

// unit quadrature offsets (quadrature_points.cuh:74-157): radius
// (x_gl + 1)/2, theta = t * pi/2, phi = p * pi/4 + pi/8; q = r + 4 t (+ 16 p)
static void unit_quad_point(int dim, int q, double* x) {
    const double pi = M_PI;
    int ri = q % 4;
    double r = (GL_X[ri] + 1.0) / 2.0;
    if (dim == 2) {
        int ti = q / 4;
        double th = ti * (3.0 * pi / 2.0 / 3.0);
        x[0] = r * std::cos(th);
        x[1] = r * std::sin(th);
    } else {
        int ti = (q / 4) % 4, pi_ = q / 16;
        double th = ti * (3.0 * pi / 2.0 / 3.0);
        double ph = pi_ * (3.0 * pi / 2.0 / 3.0 / 2.0) + pi / 4.0 / 2.0;
        x[0] = r * std::sin(ph) * std::cos(th);
        x[1] = r * std::sin(ph) * std::sin(th);
        x[2] = r * std::cos(ph);
    }
}

// antisymmetric w4 B-spline kernel alpha(x, y) with xy = y - x
// (nonlocal_calculus/detail/divergence.inl:55-133)
static void div_kernel(int dim, double delta, const double* xy, double* a) {
    const double pi = M_PI;
    if (dim == 2) {
        double r = std::sqrt(xy[0] * xy[0] + xy[1] * xy[1]);
        double ct = xy[0] / r, st = xy[1] / r;
        double den = pi * std::pow(delta, 5);
        double m;
        if (2.0 * r / delta < 1)
            m = (240.0 / 7.0) * r * (2.0 * delta - 3.0 * r);
        else if (2.0 * r / delta < 2)
            m = (240.0 / 7.0) * (delta - r) * (delta - r);
        else
            m = 0;
        a[0] = m * ct / den;
        a[1] = m * st / den;
    } else {
        double r = std::sqrt(xy[0] * xy[0] + xy[1] * xy[1] + xy[2] * xy[2]);
        double rxy = std::sqrt(xy[0] * xy[0] + xy[1] * xy[1]);
        double sp = rxy / r, cp = xy[2] / r;
        double ct = rxy != 0 ? xy[0] / rxy : 0, st = rxy != 0 ? xy[1] / rxy : 0;
        double den = pi * std::pow(delta, 6);
        double m;
        if (2.0 * r / delta < 1)
            m = 48.0 * r * (2.0 * delta - 3.0 * r);
        else if (2.0 * r / delta < 2)
            m = 48.0 * (delta - r) * (delta - r);
        else
            m = 0;
        a[0] = m * sp * ct / den;
        a[1] = m * sp * st / den;
        a[2] = m * cp / den;
    }
}

// Builds W[d,s,i] for queries [0, nq) over the domain pts[0, n): kNN(k),
// delta_i = 0.05 * |x_i - x_nn|, RPIM weights at every quadrature point and
// W(d,s) = sum_q alpha_d w_q (phi_s(x_q) + [s == 0]). The MQ spacing is the
// mean nearest-neighbour distance of each 16384-query batch, as
// divergence.cuh:85-160 builds the operator in such batches.
static int divergence_stencil(const float* pts, int64_t n, int dim, int k, int shape,
                              uint32_t* idx, double* W, double* delta_out) {
    std::vector<float> d2((size_t)n * k);
    knn_grid(pts, n, pts, n, dim, k, idx, d2.data());
    std::vector<double> nn(n);
    for (int64_t i = 0; i < n; ++i) {
        const float* a = pts + i * dim;
        const float* b = pts + (int64_t)idx[i * k + 1] * dim;
        double s = 0;
        for (int d = 0; d < dim; ++d) s += ((double)a[d] - b[d]) * ((double)a[d] - b[d]);
        nn[i] = std::sqrt(s);
    }
    const int64_t batch = 16384;
    std::vector<double> spacing((n + batch - 1) / batch);
    for (size_t b = 0; b < spacing.size(); ++b) {
        int64_t e = std::min<int64_t>(n, (int64_t)(b + 1) * batch);
        double s = 0;
        for (int64_t i = (int64_t)b * batch; i < e; ++i) s += nn[i];
        spacing[b] = s / (double)(e - (int64_t)b * batch);
    }
    const int nq = dim == 2 ? 16 : 64;
    const int nn_ = k + dim + 1;
    int bad = 0;
#pragma omp parallel
    {
        std::vector<double> xs((size_t)k * dim), G((size_t)nn_ * nn_), Ginv((size_t)nn_ * nn_), gx(nn_);
        std::vector<int> piv(nn_);
        std::vector<double> acc((size_t)k * dim);
#pragma omp for schedule(static) reduction(| : bad)
        for (int64_t i = 0; i < n; ++i) {
            const double delta = 0.05 * nn[i];
            const double sp = spacing[i / batch];
            const float* xi = pts + i * dim;
            for (int s = 0; s < k; ++s)
                for (int d = 0; d < dim; ++d)
                    xs[s * dim + d] = ((double)pts[(int64_t)idx[i * k + s] * dim + d] - xi[d]) / sp;
            build_G0(xs.data(), k, dim, shape, G.data());
            if (lu_factor(G.data(), nn_, piv.data()) != 0) bad = 1;
            for (int c = 0; c < nn_; ++c)
                for (int r = 0; r < nn_; ++r) Ginv[r + nn_ * c] = (r == c) ? 1.0 : 0.0;
            lu_solve(G.data(), nn_, piv.data(), Ginv.data(), nn_);
            std::fill(acc.begin(), acc.end(), 0.0);
            for (int q = 0; q < nq; ++q) {
                double u[3] = {0, 0, 0}, xy[3] = {0, 0, 0}, a[3] = {0, 0, 0}, xq[3] = {0, 0, 0};
                unit_quad_point(dim, q, u);
                for (int d = 0; d < dim; ++d) xy[d] = delta * u[d];
                div_kernel(dim, delta, xy, a);
                double wq = GL_W[q % 4] * delta / 2.0;
                wq *= 2.0 * M_PI / 4.0;
                if (dim == 3) wq *= M_PI / 4.0;
                if (dim == 2) {
                    wq *= std::sqrt(xy[0] * xy[0] + xy[1] * xy[1]);
                } else {
                    double r = std::sqrt(xy[0] * xy[0] + xy[1] * xy[1] + xy[2] * xy[2]);
                    double rxy = std::sqrt(xy[0] * xy[0] + xy[1] * xy[1]);
                    wq *= r * rxy;
                }
                for (int d = 0; d < dim; ++d) xq[d] = xy[d] / sp;
                build_Gx(xs.data(), k, dim, shape, xq, gx.data());
                for (int s = 0; s < k; ++s) {
                    double phi = 0;
                    for (int j = 0; j < nn_; ++j) phi += Ginv[j + nn_ * s] * gx[j];
                    for (int d = 0; d < dim; ++d) acc[s * dim + d] += a[d] * wq * (phi + (s == 0 ? 1.0 : 0.0));
                }
            }
            for (int s = 0; s < k * dim; ++s) W[i * k * dim + s] = acc[s];
            if (delta_out) delta_out[i] = delta;
        }
    }
    return bad ? 2 : 0;
}
}  // namespace orc

extern "C" int orc_divergence_stencil(const float* pts, int64_t n, int dim, int k, int shape,
                                      uint32_t* idx, double* W, double* delta) {
    if (dim < 2 || dim > 3 || k < dim + 2 || n < k) return 1;
    return divergence_stencil(pts, n, dim, k, shape, idx, W, delta);
}

// ====================================================== lattice helpers
namespace orc {
struct Lat {
    int dim, Q;
    double c[27][3];
    double w[27];
    int bb[27];
    int K[27][27];
};
static Lat make_lat(int dim) {
    Lat L{};
    L.dim = dim;
    L.Q = dim == 2 ? 9 : 27;
    for (int a = 0; a < L.Q; ++a) {
        for (int d = 0; d < dim; ++d) L.c[a][d] = dim == 2 ? D2_C[a][d] : D3_C[a][d];
        L.w[a] = dim == 2 ? D2_W[a] : D3_W[a];
        L.bb[a] = dim == 2 ? D2_BB[a] : D3_BB[a];
        for (int b = 0; b < L.Q; ++b) L.K[a][b] = dim == 2 ? D2_K[a][b] : D3_K[a][b];
    }
    return L;
}

// equilibrium w rho (1 + u.c/cs^2 + (u.c)^2/(2 cs^4) - u.u)
// (detail/equilibrium_distribution.cuh:41-64; note the - u.u term)
template <class T>
static inline T feq(T rho, const T* u, const double* c, T w, int dim) {
    T uu = 0, uc = 0;
    for (int d = 0; d < dim; ++d) uu += u[d] * u[d];
    for (int d = 0; d < dim; ++d) uc += u[d] * T(c[d]);
    const T cs = lattice_cs<T>();
    const T cs2 = cs * cs;
    const T cs4 = cs2 * cs2;
    return w * rho * (1 + uc / cs2 + (uc * uc) / (2 * cs4) - uu);
}
}  // namespace orc

extern "C" int orc_lattice(int dim, int* Q, double* c, double* w, int* bb, double* K) {
    if (dim != 2 && dim != 3) return 1;
    Lat L = make_lat(dim);
    *Q = L.Q;
    for (int a = 0; a < L.Q; ++a) {
        for (int d = 0; d < dim; ++d) c[a * dim + d] = L.c[a][d];
        w[a] = L.w[a];
        bb[a] = L.bb[a];
        for (int b = 0; b < L.Q; ++b) K[a * L.Q + b] = L.K[a][b];
    }
    return 0;
}

extern "C" int orc_collision(int dim, const double* f, double rho, const double* u, double nu,
                             double dt, double* df) {
    if (dim != 2 && dim != 3) return 1;
    Lat L = make_lat(dim);
    double k[27];
    if (dim == 3)
        d3q27_projection<double>(k, f, rho, u, nu, dt);
    else
        d2q9_projection<double>(k, f, rho, u, nu, dt);
    for (int l = 0; l < L.Q; ++l) {
        double s = 0;
        for (int j = 0; j < L.Q; ++j) s += L.K[l][j] * k[j];
        df[l] = s;
    }
    return 0;
}

// ============================================================== scene
namespace orc {

struct SceneBase {
    virtual ~SceneBase() = default;
    virtual int set_density(const float* drho) = 0;
    virtual int step(int nsteps, double* probes) = 0;
    virtual int phase(int ph) = 0;
    virtual int read_state(double* g, double* drho) const = 0;
    virtual int write_state(const double* g) = 0;
    virtual int tables(uint32_t*, double*, double*, uint32_t*, double*, uint32_t*, double*) const = 0;
    virtual int pml_state(double* q1, double* q2) const = 0;
    virtual int set_sources(const int64_t* nodes, int64_t n, const float* values, int64_t n_steps) = 0;
};

// One scene, T = double (the FP64 oracle) or T = float (the reference's
// own arithmetic). Follows detail/simulation_engine.cuh: init_domain
// :126-339, step_forward :1325-1375, reset :1377-1431.
template <class T>
struct Scene : SceneBase {
    int dim, Q, k, kb, kp, shape, pml_idx;
    int64_t N, nb, nl, nbd, ng, nbl, nd;
    double h;
    T nu, rho0, dt, c, dt_lat, nu_lat;
    Lat L;
    std::vector<float> ptsf;
    std::vector<float> normals;
    std::vector<T> sigma;  // [nl]
    // stencils (FP64 at set-up, used in T)
    std::vector<uint32_t> idx;  // [N][k]
    std::vector<double> W;      // [N][k][dim]
    std::vector<double> fw;     // [N][k]
    std::vector<uint32_t> bidx; // [nbd][kb]
    std::vector<double> bw;
    int np;
    std::vector<uint32_t> pidx;  // [np][kp]
    std::vector<double> pw;
    // state (reference layout: population-major f[a][i])
    std::vector<T> f, s1, s2, q1, q2, rho, u, f0, df, kk;
    T time = 0;
    // density sources: per-step values (dimensional density, FLT_MAX = no
    // term this step) of a set of nodes; frame = steps since set_density
    std::vector<int64_t> src_nodes;
    std::vector<float> src_vals;  // [src_steps][n]
    int64_t src_steps = 0, frame = 0;

    T& F(std::vector<T>& v, int a, int64_t i) { return v[(size_t)a * N + i]; }

    int init(const orc_scene_desc* d) {
        dim = d->dim;
        if (dim != 2 && dim != 3) return 1;
        L = make_lat(dim);
        Q = L.Q;
        k = d->k;
        kb = d->k_boundary;
        kp = d->k_probe;
        shape = d->shape;
        pml_idx = d->pml_indexing;
        nb = d->n_bulk;
        nl = d->n_layer;
        nbd = d->n_boundary;
        ng = d->n_ghost;
        N = nb + nl + nbd + ng;
        nbl = nb + nl;
        nd = N - ng;
        h = d->nodal_spacing;
        if (k < dim + 2 || k > 64 || kb < dim + 2 || kp < dim + 2 || nd < k || nbl < kb || N < kp) return 1;
        ptsf.assign(d->points, d->points + N * dim);
        normals.assign(d->normals, d->normals + nbd * dim);
        sigma.resize(nl);
        for (int64_t i = 0; i < nl; ++i) sigma[i] = (T)d->sigma[i];
        // set_problem_parameters (detail/simulation_engine.cuh:94-124)
        nu = (T)d->viscosity;
        rho0 = (T)d->rho0;
        dt = (T)d->time_step;
        c = (T)d->speed_of_sound;
        T ratio = lattice_cs<T>() / c;
        dt_lat = dt / ratio;
        nu_lat = nu / ratio;

        // divergence operator over [0, nd); ghost rows stay zero
        idx.assign((size_t)N * k, 0);
        W.assign((size_t)N * k * dim, 0.0);
        int rc = divergence_stencil(ptsf.data(), nd, dim, k, shape, idx.data(), W.data(), nullptr);
        if (rc) return rc;
        // selective-filter weights: normalised Gaussian, sigma_g = h / 2.5
        // (detail/simulation_engine.cuh:1233-1323), computed once here
        fw.assign((size_t)N * k, 0.0);
        const double sg = h / 2.5;
        for (int64_t i = 0; i < nd; ++i) {
            double sum = 0;
            for (int s = 0; s < k; ++s) {
                const float* a = &ptsf[i * dim];
                const float* b = &ptsf[(int64_t)idx[i * k + s] * dim];
                double r2 = 0;
                for (int dd = 0; dd < dim; ++dd) r2 += ((double)a[dd] - b[dd]) * ((double)a[dd] - b[dd]);
                double w = std::exp(-0.5 * r2 / (sg * sg));
                fw[i * k + s] = w;
                sum += w;
            }
            for (int s = 0; s < k; ++s) fw[i * k + s] /= sum;
        }
        // boundary interpolator: kNN among bulk+layer, RPIM with spacing h
        // (detail/simulation_engine.cuh:223-258)
        bidx.assign((size_t)nbd * kb, 0);
        bw.assign((size_t)nbd * kb, 0.0);
        if (nbd > 0) {
            std::vector<float> d2((size_t)nbd * kb);
            knn_grid(ptsf.data(), nbl, &ptsf[nbl * dim], nbd, dim, kb, bidx.data(), d2.data());
            std::vector<double> q((size_t)nbd * dim);
            for (int64_t i = 0; i < nbd * dim; ++i) q[i] = ptsf[nbl * dim + i];
            rc = orc_rbf_weights(ptsf.data(), nbl, dim, bidx.data(), kb, q.data(), nbd, 1, h, shape, bw.data());
            if (rc) return rc;
        }
        // probes: kNN among all points, RPIM with spacing h
        // (simulation_observers/density_observer.cuh:62-97)
        np = d->n_probes;
        pidx.assign((size_t)np * kp, 0);
        pw.assign((size_t)np * kp, 0.0);
        if (np > 0) {
            std::vector<float> d2((size_t)np * kp);
            knn_grid(ptsf.data(), N, d->probes, np, dim, kp, pidx.data(), d2.data());
            std::vector<double> q((size_t)np * dim);
            for (int64_t i = 0; i < np * dim; ++i) q[i] = d->probes[i];
            rc = orc_rbf_weights(ptsf.data(), N, dim, pidx.data(), kp, q.data(), np, 1, h, shape, pw.data());
            if (rc) return rc;
        }
        size_t QN = (size_t)Q * N;
        f.assign(QN, 0);
        s1.assign(QN, 0);
        s2.assign(QN, 0);
        f0.assign(QN, 0);
        df.assign(QN, 0);
        kk.assign(QN, 0);
        q1.assign(QN, 0);
        q2.assign(QN, 0);
        rho.assign(N, 0);
        u.assign((size_t)dim * N, 0);
        // PML operator construction: Q1 = w, Q2 = 0 (pml_absorption.inl:744-768)
        for (int a = 0; a < Q; ++a)
            for (int64_t i = 0; i < N; ++i) F(q1, a, i) = (T)L.w[a];
        // reset(): f = w, macros (detail/simulation_engine.cuh:1377-1431)
        for (int a = 0; a < Q; ++a)
            for (int64_t i = 0; i < N; ++i) F(f, a, i) = (T)L.w[a];
        macros();
        time = 0;
        return 0;
    }

    // rho = sum f, u = sum f c / rho, stored dimensional: rho*rho0, u*c/cs
    // (detail/simulation_engine.cuh:53-82,366-433)
    void macros() {
        const T cs = lattice_cs<T>();
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < N; ++i) {
            T r = 0, uu[3] = {0, 0, 0};
            for (int a = 0; a < Q; ++a) {
                T fa = f[(size_t)a * N + i];
                r += fa;
                for (int d = 0; d < dim; ++d) uu[d] += fa * (T)L.c[a][d];
            }
            for (int d = 0; d < dim; ++d) uu[d] /= r;
            rho[i] = r * rho0;
            for (int d = 0; d < dim; ++d) u[(size_t)d * N + i] = uu[d] * c / cs;
        }
    }

    int set_density(const float* drho) override {
        for (int a = 0; a < Q; ++a)
            for (int64_t i = 0; i < N; ++i) F(f, a, i) = (T)L.w[a] * (T(1) + (T)drho[i]);
        macros();
        frame = 0;
        return 0;
    }

    // apply_density_source_termsv5 (detail/simulation_engine.cuh:1057-1107)
    // with the race over the Q threads of a node (N2) resolved: the
    // population update f_a += (s / rho0) w_a once per population, and the
    // density statement rho <- (rho + (rho + s)) / 2 once per node.
    void apply_sources() {
        if (src_nodes.empty() || frame >= src_steps) return;
        const int64_t n = (int64_t)src_nodes.size();
        for (int64_t t = 0; t < n; ++t) {
            const float sv = src_vals[(size_t)frame * n + t];
            if (sv == std::numeric_limits<float>::max()) continue;
            const int64_t i = src_nodes[t];
            const T st = (T)sv;
            const T ds = st / rho0;
            for (int a = 0; a < Q; ++a) F(f, a, i) += ds * (T)L.w[a];
            const T imposed = (rho[i] + st) / rho0;
            rho[i] = (rho[i] + imposed * rho0) / T(2);
        }
    }

    // sum_s sum_d W(d,s,i) field_d(j_s): FP64 sums sequentially; FP32
    // reproduces the reference's pairwise shared-memory tree over s
    // (divergence.cuh:452-483).
    template <class Field>
    T divergence(int64_t i, Field&& field) const {
        T part[64];
        const double* Wi = &W[(size_t)i * k * dim];
        for (int s = 0; s < k; ++s) {
            uint32_t j = idx[(size_t)i * k + s];
            T fv[3];
            field(j, fv);
            T dv = 0;
            for (int d = 0; d < dim; ++d) dv += (T)Wi[s * dim + d] * fv[d];
            part[s] = dv;
        }
        if (std::is_same<T, double>::value) {
            T sum = 0;
            for (int s = 0; s < k; ++s) sum += part[s];
            return sum;
        }
        for (int st = 1; st < k; st *= 2)
            for (int t = 0; 2 * st * t + st < k; ++t) part[2 * st * t] += part[2 * st * t + st];
        return part[0];
    }

    // boundary RPIM interpolation f_b = w_a + sum W (f_j - w_a)
    // (radial_point_method.cuh:211-250 via simulation_engine.cuh:434-467)
    void interpolate_boundaries(std::vector<T>& v) {
#pragma omp parallel for schedule(static)
        for (int64_t b = 0; b < nbd; ++b)
            for (int a = 0; a < Q; ++a) {
                T off = (T)L.w[a], sum = 0;
                for (int s = 0; s < kb; ++s)
                    sum += (T)bw[b * kb + s] * (v[(size_t)a * N + bidx[b * kb + s]] - off);
                v[(size_t)a * N + nbl + b] = sum + off;
            }
    }

    double probe(int p) const {
        T sum = 0;
        for (int s = 0; s < kp; ++s) sum += (T)pw[p * kp + s] * (rho[pidx[p * kp + s]] - rho0);
        return (double)((sum + rho0) - rho0);
    }

    void pre_streaming() {
        const T cs = lattice_cs<T>();
        const T vscale = c / cs;  // velocity_scale of the PML/equilibrium subtasks
        s1 = f;  // scratchpad1 <- f (simulation_engine.cuh:1339-1344)
        // ---- PML Q update + local absorption (pml_absorption.inl:531-631)
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < N; ++i) {
            T ru = rho[i] / rho0, uu[3] = {0, 0, 0};
            for (int d = 0; d < dim; ++d) uu[d] = u[(size_t)d * N + i] / vscale;
            for (int a = 0; a < Q; ++a) {
                T wa = (T)L.w[a];
                T ft = feq<T>(ru, uu, L.c[a], wa, dim) - wa;
                T ftp = F(q1, a, i) - wa;
                T Q1v = (ft + ftp) * dt_lat / T(2);
                F(q1, a, i) = Q1v;
                T Q2v = (Q1v + F(q2, a, i)) * dt_lat / T(2);
                F(q2, a, i) = Q2v;
                if (i >= nb && i < nb + nl) {
                    T sg = sigma[i - nb];
                    F(s1, a, i) -= sg * (T(3) * ft + T(3) * sg * Q1v + sg * sg * Q2v);
                }
            }
        }
        // ---- PML divergence terms (pml_absorption.inl:770-855). The field
        // maps read sigma[j - nb] and, in the reference, Q[j - nb] as well
        // (pml_absorption.inl:438-448, 501-510): a node's field value uses the
        // Q of the node n_bulk places earlier. pml_indexing = 1 reads Q[j].
        const int64_t qshift = pml_idx == 0 ? nb : 0;
        for (int a = 0; a < Q; ++a) {
            double sum1 = 0, sum2 = 0;
            for (int64_t i = nb; i < nb + nl; ++i) {
                sum1 += (double)F(q1, a, i);
                sum2 += (double)F(q2, a, i);
            }
            const T m1 = (T)sum1 / (T)nl, m2 = (T)sum2 / (T)nl;
            const double* ca = L.c[a];
            const T* Q1a = &q1[(size_t)a * N];
            const T* Q2a = &q2[(size_t)a * N];
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < nd; ++i) {
                auto field1 = [&](uint32_t j, T* v) {
                    for (int d = 0; d < dim; ++d) v[d] = 0;
                    if ((int64_t)j < nb || (int64_t)j >= nb + nl) return;
                    T sg = sigma[j - nb];
                    T qv = Q1a[j - qshift];
                    for (int d = 0; d < dim; ++d) v[d] = T(-2) * (T)ca[d] * sg * (qv - m1);
                };
                T d1 = divergence(i, field1);
                F(s1, a, i) += d1;
            }
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < nd; ++i) {
                auto field2 = [&](uint32_t j, T* v) {
                    for (int d = 0; d < dim; ++d) v[d] = 0;
                    if ((int64_t)j < nb || (int64_t)j >= nb + nl) return;
                    T sg = sigma[j - nb];
                    T qv = Q2a[j - qshift];
                    for (int d = 0; d < dim; ++d) v[d] = (T)ca[d] * sg * sg * (qv - m2);
                };
                T d2 = divergence(i, field2);
                F(s1, a, i) += d2;
            }
        }
        // post_collision: Q2 <- Q1, Q1 <- feq(rho, u) (pml_absorption.inl:875-896)
        q2 = q1;
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < N; ++i) {
            T ru = rho[i] / rho0, uu[3] = {0, 0, 0};
            for (int d = 0; d < dim; ++d) uu[d] = u[(size_t)d * N + i] / vscale;
            for (int a = 0; a < Q; ++a) F(q1, a, i) = feq<T>(ru, uu, L.c[a], (T)L.w[a], dim);
        }
        interpolate_boundaries(s1);
        // ---- collision (simulation_engine.cuh:469-531)
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < N; ++i) {
            T fi[27], kv[27], uu[3] = {0, 0, 0};
            for (int a = 0; a < Q; ++a) fi[a] = f[(size_t)a * N + i];
            T r = rho[i] / rho0;
            for (int d = 0; d < dim; ++d) uu[d] = u[(size_t)d * N + i] * (cs / c);
            if (dim == 3)
                d3q27_projection<T>(kv, fi, r, uu, nu_lat, dt_lat);
            else
                d2q9_projection<T>(kv, fi, r, uu, nu_lat, dt_lat);
            for (int l = 0; l < Q; ++l) {
                T dfl = 0;
                for (int j = 0; j < Q; ++j) dfl += (T)L.K[l][j] * kv[j];
                s1[(size_t)l * N + i] += dfl * dt_lat;
            }
        }
        // ---- selective filter into s2 (simulation_engine.cuh:1233-1323)
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < N; ++i)
            for (int a = 0; a < Q; ++a) {
                const T* s1a = &s1[(size_t)a * N];
                if (i >= nbl) {
                    s2[(size_t)a * N + i] = s1a[i];
                    continue;
                }
                T fi = s1a[i], sum = 0;
                for (int s = 0; s < k; ++s) sum += (T)fw[i * k + s] * (s1a[idx[i * k + s]] - fi);
                s2[(size_t)a * N + i] = fi + T(0.75f) * sum;
            }
        std::swap(f, s2);
        // ---- bounce-back on boundary nodes (simulation_engine.cuh:789-944)
#pragma omp parallel for schedule(static)
        for (int64_t b = 0; b < nbd; ++b) {
            int64_t i = nbl + b;
            T nrm[3] = {0, 0, 0};
            for (int d = 0; d < dim; ++d) nrm[d] = (T)normals[b * dim + d];
            for (int a = 0; a < Q; ++a) {
                T cn = 0;
                for (int d = 0; d < dim; ++d) cn += (T)L.c[a][d] * nrm[d];
                if (cn <= 0) continue;
                f[(size_t)a * N + i] = f[(size_t)L.bb[a] * N + i];
            }
            for (int d = 0; d < dim; ++d) u[(size_t)d * N + i] = 0;
        }
    }

    // rates_a(i) = div(c_a (-(f_a - w_a))), zero on boundary and ghost
    // nodes (detail/pde_right_hand_side.cuh:82-176)
    void rates(const std::vector<T>& fs, std::vector<T>& out) {
        for (int a = 0; a < Q; ++a) {
            const T* fa = &fs[(size_t)a * N];
            const T wa = (T)L.w[a];
            const double* ca = L.c[a];
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < N; ++i) {
                if (i >= nbl) {
                    out[(size_t)a * N + i] = 0;
                    continue;
                }
                auto field = [&](uint32_t j, T* v) {
                    T sc = fa[j];
                    for (int d = 0; d < dim; ++d) v[d] = (T)ca[d] * (-(sc - wa));
                };
                out[(size_t)a * N + i] = divergence(i, field);
            }
        }
    }

    // classic RK4 as detail/rk4_solver.cuh:48-171
    void rk4() {
        const T h = dt_lat;
        const T a1 = h * T(0.5), a3 = h * T(1);
        const T b1 = T(1. / 6.), b2 = T(2. / 6.);
        const size_t QN = (size_t)Q * N;
        f0 = f;
        rates(f, kk);
#pragma omp parallel for schedule(static)
        for (size_t t = 0; t < QN; ++t) {
            f[t] = f0[t] + a1 * kk[t];
            df[t] = kk[t] * b1;
        }
        rates(f, kk);
#pragma omp parallel for schedule(static)
        for (size_t t = 0; t < QN; ++t) {
            f[t] = f0[t] + a1 * kk[t];
            df[t] = df[t] + kk[t] * b2;
        }
        rates(f, kk);
#pragma omp parallel for schedule(static)
        for (size_t t = 0; t < QN; ++t) {
            f[t] = f0[t] + a3 * kk[t];
            df[t] = df[t] + kk[t] * b2;
        }
        rates(f, kk);
#pragma omp parallel for schedule(static)
        for (size_t t = 0; t < QN; ++t) {
            df[t] = df[t] + kk[t] * b1;
            f[t] = f0[t] + h * df[t];
        }
    }

    int step(int nsteps, double* probes) override {
        for (int n = 0; n < nsteps; ++n) {
            macros();
            if (probes)
                for (int p = 0; p < np; ++p) probes[(size_t)n * np + p] = probe(p);
            apply_sources();
            pre_streaming();
            rk4();
            interpolate_boundaries(f);
            time += dt;
            ++frame;
        }
        return 0;
    }

    int phase(int ph) override {
        if (ph == 1) {
            macros();
            apply_sources();
            pre_streaming();
        } else if (ph == 2) {
            rk4();
            interpolate_boundaries(f);
            time += dt;
            ++frame;
        } else {
            return 1;
        }
        return 0;
    }

    int read_state(double* g, double* drho) const override {
        for (int64_t i = 0; i < N; ++i) {
            double r = 0;
            for (int a = 0; a < Q; ++a) {
                double v = (double)f[(size_t)a * N + i];
                if (g) g[i * Q + a] = v - L.w[a];
                r += v;
            }
            if (drho) drho[i] = r * (double)rho0 - (double)rho0;
        }
        return 0;
    }

    int set_sources(const int64_t* nodes, int64_t n, const float* values, int64_t n_steps) override {
        if (n < 0 || n_steps < 0 || (n > 0 && (!nodes || (n_steps > 0 && !values)))) return 1;
        for (int64_t t = 0; t < n; ++t)
            if (nodes[t] < 0 || nodes[t] >= N) return 1;
        src_nodes.assign(nodes, nodes + n);
        src_vals.assign(values, values + (size_t)n * n_steps);
        src_steps = n_steps;
        return 0;
    }

    int write_state(const double* g) override {
        for (int64_t i = 0; i < N; ++i)
            for (int a = 0; a < Q; ++a) f[(size_t)a * N + i] = (T)(L.w[a] + g[i * Q + a]);
        macros();
        return 0;
    }

    int tables(uint32_t* oidx, double* oW, double* ofw, uint32_t* obidx, double* obw, uint32_t* opidx,
               double* opw) const override {
        if (oidx) std::copy(idx.begin(), idx.end(), oidx);
        if (oW) std::copy(W.begin(), W.end(), oW);
        if (ofw) std::copy(fw.begin(), fw.end(), ofw);
        if (obidx) std::copy(bidx.begin(), bidx.end(), obidx);
        if (obw) std::copy(bw.begin(), bw.end(), obw);
        if (opidx) std::copy(pidx.begin(), pidx.end(), opidx);
        if (opw) std::copy(pw.begin(), pw.end(), opw);
        return 0;
    }

    int pml_state(double* oq1, double* oq2) const override {
        for (int64_t i = 0; i < N; ++i)
            for (int a = 0; a < Q; ++a) {
                if (oq1) oq1[i * Q + a] = (double)q1[(size_t)a * N + i];
                if (oq2) oq2[i * Q + a] = (double)q2[(size_t)a * N + i];
            }
        return 0;
    }
};

}  // namespace orc

struct orc_scene {
    std::unique_ptr<orc::SceneBase> impl;
};

extern "C" int orc_scene_create(const orc_scene_desc* d, orc_scene** out) {
    if (!d || !out) return 1;
    auto s = new orc_scene;
    int rc;
    if (d->precision == 1) {
        auto p = new orc::Scene<float>();
        rc = p->init(d);
        s->impl.reset(p);
    } else {
        auto p = new orc::Scene<double>();
        rc = p->init(d);
        s->impl.reset(p);
    }
    if (rc) {
        delete s;
        return rc;
    }
    *out = s;
    return 0;
}
extern "C" void orc_scene_destroy(orc_scene* s) { delete s; }
extern "C" int orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}
extern "C" int orc_scene_set_sources(orc_scene* s, const int64_t* nodes, int64_t n, const float* values,
                                     int64_t n_steps) {
    return s->impl->set_sources(nodes, n, values, n_steps);
}
extern "C" int orc_scene_set_density(orc_scene* s, const float* d) { return s->impl->set_density(d); }
extern "C" int orc_scene_step(orc_scene* s, int n, double* p) { return s->impl->step(n, p); }
extern "C" int orc_scene_step_phase(orc_scene* s, int ph) { return s->impl->phase(ph); }
extern "C" int orc_scene_read_state(const orc_scene* s, double* g, double* r) {
    return s->impl->read_state(g, r);
}
extern "C" int orc_scene_write_state(orc_scene* s, const double* g) { return s->impl->write_state(g); }
extern "C" int orc_scene_tables(const orc_scene* s, uint32_t* a, double* b, double* c, uint32_t* d,
                                double* e, uint32_t* f, double* g) {
    return s->impl->tables(a, b, c, d, e, f, g);
}
extern "C" int orc_scene_pml_state(const orc_scene* s, double* q1, double* q2) {
    return s->impl->pml_state(q1, q2);
}
