// Radial-point-interpolation weights and the nonlocal divergence stencil,
// built on the GPU in FP64 (or FP32 LU + FP64-residual refinement).
//
// NAGA builds the augmented moment matrix G0 = [[Phi, P], [P^T, 0]] per
// support set, inverts it with cuBLAS and contracts the inverse with G_x
// (interpolation/detail/radial_point_method.cuh:349-453). Here one warp
// owns one support set: it assembles G0 in shared memory, factors it with
// partial pivoting and solves for the right-hand sides directly (the
// contraction W = G0^-T G_x equals G0^-1 G_x because G0 is symmetric).
//
// Coordinates are shifted to the group's centre and divided by the spacing
// parameter before assembly. Both shape functions are radial, so this
// leaves the interpolation weights unchanged in exact arithmetic (the RBF
// block scales by a constant and span{1, x} is shift- and scale-invariant)
// while it removes most of the ill-conditioning of the absolute-coordinate
// system.
#include "warp_lu.cuh"
#include "scene_dev.hpp"

#include <algorithm>
#include <mutex>
#include <vector>

namespace naga {

// systems whose FP32 refinement failed in the last refined call (per thread)
static thread_local int64_t g_fallbacks = 0;

namespace {

// multiquadric (r^2 + (0.1 h)^2)^0.5 in units of h (radial_point_method.cuh:
// 44-66 with q = 0.5, alpha_c = 0.1), or the cubic polyharmonic spline r^3
__device__ __forceinline__ double shape_fn(double r2, int shape) {
    if (shape == 0) return sqrt(r2 + 0.01);
    double r = sqrt(r2);
    return r * r * r;
}

template <int D>
__device__ void build_G0(const double* xs, int k, int shape, double* G) {
    const int n = k + D + 1;
    for (int e = lane_id(); e < n * n; e += 32) {
        const int i = e % n, j = e / n;
        double v;
        if (i >= k && j >= k)
            v = 0.0;
        else if (i >= k)
            v = (i == k) ? 1.0 : xs[j * D + (i - k - 1)];
        else if (j >= k)
            v = (j == k) ? 1.0 : xs[i * D + (j - k - 1)];
        else {
            double r2 = 0;
#pragma unroll
            for (int d = 0; d < D; ++d) {
                double t = xs[i * D + d] - xs[j * D + d];
                r2 += t * t;
            }
            v = shape_fn(r2, shape);
        }
        G[e] = v;
    }
    __syncwarp();
}

// G_x row r for the scaled query point x
template <int D>
__device__ __forceinline__ double gx_row(const double* xs, int k, int shape, const double* x, int r) {
    if (r < k) {
        double r2 = 0;
#pragma unroll
        for (int d = 0; d < D; ++d) {
            double t = xs[r * D + d] - x[d];
            r2 += t * t;
        }
        return shape_fn(r2, shape);
    }
    if (r == k) return 1.0;
    return x[r - k - 1];
}

// y = A x for x distributed over the warp (rows r = lane, lane + 32)
__device__ void warp_matvec(const double* A, int n, double x0, double x1, double& y0, double& y1) {
    const int lane = lane_id();
    y0 = 0;
    y1 = 0;
    for (int j = 0; j < n; ++j) {
        double xj = warp_get(x0, x1, j);
        if (lane < n) y0 += A[lane + n * j] * xj;
        if (lane + 32 < n) y1 += A[lane + 32 + n * j] * xj;
    }
}

// Solves G0 x = b for the distributed right-hand side (x0, x1) in place:
// precision 0: FP64 LU (factors in G); precision 1: FP32 LU in Gf with
// FP64-residual refinement against G (unfactored). Refinement stops when
// the correction falls below 1e-14 of the solution or stops shrinking; it
// has converged when the last correction is below 1e-10 of the solution
// (the relative weight error the FP64 path is held to). Returns false when
// it has not.
__device__ bool solve_rhs(const double* G, const float* Gf, const int* piv, int n, int precision, double& x0,
                          double& x1) {
    if (precision == 0) {
        warp_lu_solve_reg(G, n, piv, x0, x1);
        return true;
    }
    const double b0 = x0, b1 = x1;
    float f0 = (float)b0, f1 = (float)b1;
    warp_lu_solve_reg(Gf, n, piv, f0, f1);
    x0 = f0;
    x1 = f1;
    double prev = INFINITY, dm = INFINITY, xm = 0;
    for (int it = 0; it < 30; ++it) {
        double y0, y1;
        warp_matvec(G, n, x0, x1, y0, y1);
        float r0 = (float)(b0 - y0), r1 = (float)(b1 - y1);
        warp_lu_solve_reg(Gf, n, piv, r0, r1);
        x0 += r0;
        x1 += r1;
        dm = fmax(fabs((double)r0), fabs((double)r1));
        xm = fmax(fabs(x0), fabs(x1));
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            dm = fmax(dm, __shfl_xor_sync(kFull, dm, o));
            xm = fmax(xm, __shfl_xor_sync(kFull, xm, o));
        }
        if (dm <= 1e-14 * xm || dm > 0.5 * prev) break;
        prev = dm;
    }
    return dm <= 1e-10 * xm;
}

__device__ __forceinline__ size_t rbf_smem_per_warp(int n, int k, int D, int precision) {
    size_t s = (size_t)8 * n * n + (size_t)8 * k * D + 16 * ((n + 3) / 4);
    if (precision) s += (size_t)4 * n * n + 16;
    return (s + 15) / 16 * 16;
}
size_t rbf_smem_per_warp_h(int n, int k, int D, int precision) {
    size_t s = (size_t)8 * n * n + (size_t)8 * k * D + 16 * ((n + 3) / 4);
    if (precision) s += (size_t)4 * n * n + 16;
    return (s + 15) / 16 * 16;
}

struct WarpSmem {
    double* G;
    double* xs;
    int* piv;
    float* Gf;
};
__device__ WarpSmem carve(unsigned char* base, int n, int k, int D, int precision) {
    WarpSmem w;
    w.G = reinterpret_cast<double*>(base);
    w.xs = w.G + n * n;
    w.piv = reinterpret_cast<int*>(w.xs + k * D);
    w.Gf = reinterpret_cast<float*>(reinterpret_cast<unsigned char*>(w.piv) + 16 * ((n + 3) / 4));
    return w;
}

// Factor G (and its FP32 copy when refining); returns the LU info.
__device__ int factor(WarpSmem& s, int n, int precision) {
    if (precision == 0) return warp_lu(s.G, n, s.piv);
    for (int e = lane_id(); e < n * n; e += 32) s.Gf[e] = (float)s.G[e];
    __syncwarp();
    return warp_lu(s.Gf, n, s.piv);
}

template <int D>
__global__ void rbf_weights_kernel(const float* __restrict__ src, int64_t nsrc, const uint32_t* __restrict__ support,
                                   int k, const double* __restrict__ qry, int64_t ngroups, int group, double spacing,
                                   int shape, int precision, double* __restrict__ weights, int* __restrict__ status,
                                   int wpb) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int w = threadIdx.x >> 5, lane = lane_id();
    const int n = k + D + 1;
    WarpSmem s = carve(smem + rbf_smem_per_warp(n, k, D, precision) * w, n, k, D, precision);
    for (int64_t g = (int64_t)blockIdx.x * wpb + w; g < ngroups; g += (int64_t)gridDim.x * wpb) {
        double o[D];
#pragma unroll
        for (int d = 0; d < D; ++d) o[d] = qry[(g * group) * D + d];
        for (int t = lane; t < k; t += 32) {
            uint32_t j = support[g * k + t];
            if ((int64_t)j >= nsrc) {
                atomicOr(status, 1);
                j = 0;
            }
#pragma unroll
            for (int d = 0; d < D; ++d) s.xs[t * D + d] = ((double)src[(int64_t)j * D + d] - o[d]) / spacing;
        }
        __syncwarp();
        build_G0<D>(s.xs, k, shape, s.G);
        int prec = precision;
        int info = factor(s, n, prec);
        if (info) atomicOr(status, 2);
        for (int q = 0; q < group; ++q) {
            double x[D];
#pragma unroll
            for (int d = 0; d < D; ++d) x[d] = (qry[(g * group + q) * D + d] - o[d]) / spacing;
            double x0 = lane < n ? gx_row<D>(s.xs, k, shape, x, lane) : 0.0;
            double x1 = lane + 32 < n ? gx_row<D>(s.xs, k, shape, x, lane + 32) : 0.0;
            if (!solve_rhs(s.G, s.Gf, s.piv, n, prec, x0, x1)) {
                // FP32 refinement failed: factor in FP64 and redo the group
                prec = 0;
                if (lane == 0) atomicAdd(status + 1, 1);
                if (warp_lu(s.G, n, s.piv)) atomicOr(status, 2);
                q = -1;
                continue;
            }
            double* out = weights + (g * group + q) * k;
            if (lane < k) out[lane] = x0;
            if (lane + 32 < k) out[lane + 32] = x1;
        }
        __syncwarp();
    }
}

// ------------------------------------------------- divergence stencil build
// 4-point Gauss-Legendre nodes/weights with the six-digit values NAGA uses
// (nonlocal_calculus/detail/quadrature_points.cuh:49-61).
__constant__ double c_gl_w[4] = {0.652145, 0.652145, 0.347855, 0.347855};
__constant__ double c_gl_x[4] = {0.339981, -0.339981, 0.861136, -0.861136};

// unit quadrature offset q (quadrature_points.cuh:74-157): radius
// (x_gl + 1) / 2; theta = t pi / 2; phi = p pi / 4 + pi / 8.
template <int D>
__device__ __forceinline__ void unit_quad(int q, double* u) {
    const double r = (c_gl_x[q & 3] + 1.0) / 2.0;
    const int t = (q >> 2) & 3;
    double st, ct;
    sincospi(0.5 * t, &st, &ct);
    if (D == 2) {
        u[0] = r * ct;
        u[1] = r * st;
    } else {
        const int p = q >> 4;
        double sp, cp;
        sincospi((2.0 * p + 1.0) / 8.0, &sp, &cp);
        u[0] = r * sp * ct;
        u[1] = r * sp * st;
        u[2] = r * cp;
    }
}

// antisymmetric w4 B-spline kernel (nonlocal_calculus/detail/divergence.inl:
// 55-133) and the quadrature weight of divergence.inl:171-197
template <int D>
__device__ __forceinline__ void kernel_and_weight(double delta, const double* xy, int q, double* a, double& wq) {
    const double pi = 3.141592653589793;
    double r2 = 0;
#pragma unroll
    for (int d = 0; d < D; ++d) r2 += xy[d] * xy[d];
    const double r = sqrt(r2);
    double m;
    if (2.0 * r / delta < 1)
        m = (D == 2 ? 240.0 / 7.0 : 48.0) * r * (2.0 * delta - 3.0 * r);
    else if (2.0 * r / delta < 2)
        m = (D == 2 ? 240.0 / 7.0 : 48.0) * (delta - r) * (delta - r);
    else
        m = 0;
    wq = c_gl_w[q & 3] * delta / 2.0 * (2.0 * pi / 4.0);
    if (D == 2) {
        const double den = pi * delta * delta * delta * delta * delta;
        a[0] = m * (xy[0] / r) / den;
        a[1] = m * (xy[1] / r) / den;
        wq *= r;
    } else {
        const double rxy = sqrt(xy[0] * xy[0] + xy[1] * xy[1]);
        const double den = pi * delta * delta * delta * delta * delta * delta;
        const double sp = rxy / r, cp = xy[2] / r;
        const double ct = rxy != 0 ? xy[0] / rxy : 0, st = rxy != 0 ? xy[1] / rxy : 0;
        a[0] = m * sp * ct / den;
        a[1] = m * sp * st / den;
        a[2] = m * cp / den;
        wq *= pi / 4.0;
        wq *= r * rxy;
    }
}

// The quadrature of the stencil build depends on the node only through
// delta: xy = delta u_q, and the product a_d(xy) w_q scales exactly as
// 1 / delta (3-D: a ~ delta^2 / delta^6, w ~ delta^3; 2-D: a ~ delta^2 /
// delta^5, w ~ delta^2). One launch tabulates u_q and K_qd = a_d w_q at
// delta = 1 with the functions above; the per-node loop scales them.
struct QuadTable {
    double u[64][3];
    double K[64][3];
    double ksum[3];  // sum_q K_qd
};
__device__ QuadTable g_quad[2];  // D2Q9, D3Q27 (filled once per device)

template <int D>
__global__ void quad_table_kernel() {
    QuadTable& g_q = g_quad[D - 2];
    constexpr int nq = D == 2 ? 16 : 64;
    const int q = threadIdx.x;
    if (q < nq) {
        double u[D], a[D], wq;
        unit_quad<D>(q, u);
        kernel_and_weight<D>(1.0, u, q, a, wq);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            g_q.u[q][d] = d < D ? u[d] : 0.0;
            g_q.K[q][d] = d < D ? a[d] * wq : 0.0;
        }
    }
    __syncthreads();
    if (q < 3) {
        double sum = 0;
        for (int t = 0; t < nq; ++t) sum += g_q.K[t][q];  // fixed order
        g_q.ksum[q] = sum;
    }
}

// nearest-neighbour distance |x_i - x_{idx[i][1]}| in FP64
template <int D>
__global__ void nn_kernel(const float* __restrict__ pts, const uint32_t* __restrict__ idx, int k, int64_t n,
                          double* __restrict__ nn) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t j = idx[i * k + 1];
        double s = 0;
#pragma unroll
        for (int d = 0; d < D; ++d) {
            double t = (double)pts[i * D + d] - (double)pts[(int64_t)j * D + d];
            s += t * t;
        }
        nn[i] = sqrt(s);
    }
}

// mean nearest-neighbour distance per batch of `batch` consecutive nodes
__global__ void batch_mean_kernel(const double* __restrict__ nn, int64_t n, int64_t batch, double* __restrict__ out) {
    __shared__ double red[32];
    const int64_t b = blockIdx.x;
    const int64_t s = b * batch, e = min(n, s + batch);
    double acc = 0;
    for (int64_t i = s + threadIdx.x; i < e; i += blockDim.x) acc += nn[i];
    acc = warp_sum(acc);
    if (lane_id() == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        v = warp_sum(v);
        if (threadIdx.x == 0) out[b] = v / (double)(e - s);
    }
}

}  // namespace

namespace {

// Per-node pieces shared by the two build kernels. One warp per node i:
// the support coordinates, shifted to x_i and divided by the spacing, go to
// xs (shared); lane t keeps support index t (and t + 32) and its squared
// distance; delta is the interaction radius 0.05 |x_i - x_nn|
// (operators.cuh:84-117). A support index outside [0, n) (a kNN sentinel)
// is replaced by i and reported in bad (warp-uniform).
template <int D>
struct NodeStencil {
    uint32_t jl[2];
    double r2own[2];
    double delta, sp;
    bool bad;
};
template <int D>
__device__ __forceinline__ NodeStencil<D> load_node(const float* __restrict__ pts, int64_t n,
                                                    const uint32_t* __restrict__ idx, int k, int64_t i, double sp,
                                                    double* xs) {
    const int lane = lane_id();
    NodeStencil<D> ns;
    ns.sp = sp;
    double xi[D];
#pragma unroll
    for (int d = 0; d < D; ++d) xi[d] = (double)pts[i * D + d];
    ns.jl[0] = ns.jl[1] = 0;
    ns.r2own[0] = ns.r2own[1] = 0;
    bool bad = false;
    for (int t = lane, r = 0; t < k; t += 32, ++r) {
        const uint32_t jr = idx[i * k + t];
        bad = bad || (int64_t)jr >= n;
        const uint32_t j = (int64_t)jr < n ? jr : (uint32_t)i;
        ns.jl[r] = j;
        double rr = 0;
#pragma unroll
        for (int d = 0; d < D; ++d) {
            const double xj = (double)pts[(int64_t)j * D + d];
            xs[t * D + d] = (xj - xi[d]) / sp;
            rr += (xj - xi[d]) * (xj - xi[d]);
        }
        ns.r2own[r] = rr;
    }
    ns.delta = 0.05 * sqrt(__shfl_sync(kFull, ns.r2own[0], 1));
    ns.bad = __any_sync(kFull, bad);
    __syncwarp();
    return ns;
}

// right-hand sides b_d = sum_q alpha_d(q) w_q G_x(q), rows lane / lane + 32,
// from the delta = 1 table: x_q = delta u_q / h, alpha_d w_q = K_qd / delta;
// cself_d = sum_q alpha_d w_q (the [s = 0] term of the weight)
template <int D>
__device__ __forceinline__ void quad_rhs(const double* xs, int k, int nsys, int shape, const NodeStencil<D>& ns,
                                         double* b0, double* b1, double* cself) {
    constexpr int nq = D == 2 ? 16 : 64;
    const int lane = lane_id();
    const QuadTable& tq = g_quad[D - 2];
    const double rdel = 1.0 / ns.delta, us = ns.delta / ns.sp;
#pragma unroll
    for (int d = 0; d < D; ++d) {
        b0[d] = b1[d] = 0;
        cself[d] = tq.ksum[d] * rdel;
    }
    // rows lane and lane + 32: support coordinates kept in registers (RBF
    // rows), the table read through the read-only path; same arithmetic as
    // gx_row
    const int r0 = lane, r1 = lane + 32;
    double x0[D], x1[D];
#pragma unroll
    for (int d = 0; d < D; ++d) {
        x0[d] = r0 < k ? xs[r0 * D + d] : 0.0;
        x1[d] = r1 < k ? xs[r1 * D + d] : 0.0;
    }
    const double* tu = &tq.u[0][0];
    const double* tk = &tq.K[0][0];
#pragma unroll 4
    for (int q = 0; q < nq; ++q) {
        double xq[D];
#pragma unroll
        for (int d = 0; d < D; ++d) xq[d] = us * __ldg(tu + 3 * q + d);
        auto row = [&](int r, const double* xr) -> double {
            if (r >= nsys) return 0.0;
            if (r < k) {
                double r2 = 0;
#pragma unroll
                for (int d = 0; d < D; ++d) {
                    const double t = xr[d] - xq[d];
                    r2 += t * t;
                }
                return shape_fn(r2, shape);
            }
            if (r == k) return 1.0;
            double v = xq[0];
#pragma unroll
            for (int d = 1; d < D; ++d)
                if (r - k - 1 == d) v = xq[d];
            return v;
        };
        const double g0 = row(r0, x0), g1 = row(r1, x1);
#pragma unroll
        for (int d = 0; d < D; ++d) {
            const double aw = __ldg(tk + 3 * q + d) * rdel;
            b0[d] += aw * g0;
            b1[d] += aw * g1;
        }
    }
}

// filter weights and the stencil records of node i (weights W0: support
// lane, W1: support lane + 32)
template <int D>
__device__ __forceinline__ void write_node(const StencilOut& out, int64_t i, int k, const NodeStencil<D>& ns,
                                           const double* W0, const double* W1) {
    const int lane = lane_id();
    // selective-filter weights: normalised Gaussian of the distance
    // (detail/simulation_engine.cuh:1233-1323), computed once
    double fw0 = 0, fw1 = 0;
    if (out.Ff || (D == 2 && out.Wf)) {
        const double inv2s2 = 0.5 / (out.filter_sigma * out.filter_sigma);
        fw0 = lane < k ? exp(-ns.r2own[0] * inv2s2) : 0.0;
        fw1 = lane + 32 < k ? exp(-ns.r2own[1] * inv2s2) : 0.0;
        const double tot = warp_sum(fw0 + fw1);
        fw0 /= tot;
        fw1 /= tot;
    }
    for (int r = 0; r < 2; ++r) {
        const int t = lane + 32 * r;
        if (t >= k) break;
        const double* Wt = r == 0 ? W0 : W1;
        if (out.W64)
#pragma unroll
            for (int d = 0; d < D; ++d) out.W64[(i * k + t) * D + d] = Wt[d];
        if (out.W32)
#pragma unroll
            for (int d = 0; d < D; ++d) out.W32[(i * k + t) * D + d] = (float)Wt[d];
        const int64_t at = out.npb > 0 ? pass_record(i, t, k, out.split, out.n_total, out.npb) : i * k + t;
        if (out.Wf) {
            const float fz = D == 3 ? (float)Wt[D - 1] : (float)(r == 0 ? fw0 : fw1);
            out.Wf[at] = make_float4((float)Wt[0], (float)Wt[1], fz, __uint_as_float(ns.jl[r]));
        }
        if (out.Ff) out.Ff[at] = make_float2((float)(r == 0 ? fw0 : fw1), __uint_as_float(ns.jl[r]));
    }
    if (out.delta && lane == 0) out.delta[i] = ns.delta;
    if (out.delta32 && lane == 0) out.delta32[i] = (float)ns.delta;
}

// Any k and both precisions: G0 column-major, factored by warp_lu, the D
// right-hand sides solved one after the other.
template <int D>
__global__ void divergence_build_kernel(const float* __restrict__ pts, int64_t n, const uint32_t* __restrict__ idx,
                                        int k, const double* __restrict__ spacing, int64_t spacing_batch,
                                        int shape, int precision, StencilOut out, int* __restrict__ status,
                                        int wpb) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int w = threadIdx.x >> 5, lane = lane_id();
    const int nsys = k + D + 1;
    WarpSmem s = carve(smem + rbf_smem_per_warp(nsys, k, D, precision) * w, nsys, k, D, precision);
    for (int64_t i = (int64_t)blockIdx.x * wpb + w; i < n; i += (int64_t)gridDim.x * wpb) {
        const NodeStencil<D> ns = load_node<D>(pts, n, idx, k, i, spacing[i / spacing_batch], s.xs);
        if (ns.bad && lane == 0) atomicOr(status, 1);
        build_G0<D>(s.xs, k, shape, s.G);
        double b0[D], b1[D], cself[D];
        quad_rhs<D>(s.xs, k, nsys, shape, ns, b0, b1, cself);
        const int info = factor(s, nsys, precision);
        if (info) atomicOr(status, 2);
        double W0[D], W1[D];
        bool ok = true;
#pragma unroll
        for (int d = 0; d < D; ++d) {
            double x0 = b0[d], x1 = b1[d];
            ok = ok && solve_rhs(s.G, s.Gf, s.piv, nsys, precision, x0, x1);
            W0[d] = x0 + (lane == 0 ? cself[d] : 0.0);
            W1[d] = x1;
        }
        if (!ok) {
            // FP32 refinement failed for this system: solve it in FP64
            if (lane == 0) atomicAdd(status + 1, 1);
            if (warp_lu(s.G, nsys, s.piv)) atomicOr(status, 2);
#pragma unroll
            for (int d = 0; d < D; ++d) {
                double x0 = b0[d], x1 = b1[d];
                warp_lu_solve_reg(s.G, nsys, s.piv, x0, x1);
                W0[d] = x0 + (lane == 0 ? cself[d] : 0.0);
                W1[d] = x1;
            }
        }
        write_node<D>(out, i, k, ns, W0, W1);
        __syncwarp();
    }
}

// ---- fixed stencil size, FP64: the augmented system [G0 | b_1 .. b_D] is
// factored in place, row-major with a padded row stride, so the forward
// substitution rides along with the elimination and one back substitution
// serves the D right-hand sides. Pivoting is warp_lu's (first maximal |a|
// of the column, rows swapped whole), the updates are the same operations
// in the same order; the back substitution multiplies by the pivot's
// reciprocal (computed once per column) instead of dividing.
template <int D, int KC>
struct AugSize {
    static constexpr int N = KC + D + 1;              // system size
    static constexpr int NC = (N + D + 1) / 2 * 2;    // columns with the right-hand sides, even
    static constexpr int LD = NC % 4 == 2 ? NC : NC + 2;  // row stride: 16-B rows, lanes' rows on distinct banks
    static constexpr int OFF = N > 32 ? N - 32 : 0;   // lane l owns row OFF + l, lanes < OFF also row l
    // per-warp block, a multiple of 128 B so every warp's rows stay 16-B aligned
    static constexpr size_t smem_per_warp = (sizeof(double) * ((size_t)N * LD + (size_t)KC * D + N) + 127) / 128 * 128;
};
static_assert(AugSize<3, 32>::LD % 2 == 0 && AugSize<2, 16>::LD % 2 == 0, "16-B aligned rows");
static_assert(AugSize<3, 32>::smem_per_warp % 16 == 0 && AugSize<2, 16>::smem_per_warp % 16 == 0, "aligned warps");

// G0 row-major with stride LD (G0 is symmetric, so this is also its transpose)
template <int D, int KC>
__device__ __forceinline__ void build_G0_rows(const double* xs, int shape, double* A) {
    using Z = AugSize<D, KC>;
    if constexpr (KC == 32) {
        // RBF block by symmetry: lane l evaluates the pairs (l, l + t mod 32),
        // t = 0..16, and writes both mirror entries (the t = 16 pairs twice,
        // with the same value)
        const int l = lane_id();
        double xl[D];
#pragma unroll
        for (int d = 0; d < D; ++d) xl[d] = xs[l * D + d];
#pragma unroll 4
        for (int t = 0; t <= 16; ++t) {
            const int c = (l + t) & 31;
            double r2 = 0;
#pragma unroll
            for (int d = 0; d < D; ++d) {
                const double u = xl[d] - xs[c * D + d];
                r2 += u * u;
            }
            const double v = shape_fn(r2, shape);
            A[l * Z::LD + c] = v;
            A[c * Z::LD + l] = v;
        }
        // border [1, x] in row / column l, and the zero corner
        A[l * Z::LD + KC] = 1.0;
        A[KC * Z::LD + l] = 1.0;
#pragma unroll
        for (int d = 0; d < D; ++d) {
            A[l * Z::LD + KC + 1 + d] = xl[d];
            A[(KC + 1 + d) * Z::LD + l] = xl[d];
        }
        if (l < (D + 1) * (D + 1)) A[(KC + l / (D + 1)) * Z::LD + KC + l % (D + 1)] = 0.0;
        return;
    }
#pragma unroll 4
    for (int e = lane_id(); e < Z::N * Z::N; e += 32) {
        const int r = e / Z::N, c = e % Z::N;
        double v;
        if (r >= KC && c >= KC)
            v = 0.0;
        else if (r >= KC)
            v = (r == KC) ? 1.0 : xs[c * D + (r - KC - 1)];
        else if (c >= KC)
            v = (c == KC) ? 1.0 : xs[r * D + (c - KC - 1)];
        else {
            double r2 = 0;
#pragma unroll
            for (int d = 0; d < D; ++d) {
                const double t = xs[r * D + d] - xs[c * D + d];
                r2 += t * t;
            }
            v = shape_fn(r2, shape);
        }
        A[r * Z::LD + c] = v;
    }
}

// row i -= l_i * row j over columns j+1 .. NC-1, l_i = a_ij / a_jj stored
template <int NC>
__device__ __forceinline__ void eliminate_row(double* ri, const double* rj, int j, double inv) {
    const double l = ri[j] * inv;
    ri[j] = l;
    int c = j + 1;
    if (c & 1) {
        ri[c] -= l * rj[c];
        ++c;
    }
    for (; c < NC; c += 2) {
        double2 a = *reinterpret_cast<double2*>(ri + c);
        const double2 b = *reinterpret_cast<const double2*>(rj + c);
        a.x -= l * b.x;
        a.y -= l * b.y;
        *reinterpret_cast<double2*>(ri + c) = a;
    }
}

// In-place LU of the augmented rows; rdiag[j] = 1 / u_jj. Returns 0, or
// j + 1 for the first column whose pivot is exactly zero (left unreduced).
template <int D, int KC>
__device__ int aug_lu(double* A, double* rdiag) {
    using Z = AugSize<D, KC>;
    constexpr int N = Z::N, LD = Z::LD, OFF = Z::OFF;
    const int lane = lane_id();
    const int p1 = OFF + lane;
    const bool has1 = p1 < N, has2 = lane < OFF;
    int info = 0;
    for (int j = 0; j < N; ++j) {
        // NaN never becomes a candidate, so the comparisons order totally and
        // every lane ends with the same pivot; lane 0's is broadcast anyway,
        // and a column with no candidate (all NaN) pivots on its own row
        double best = -1.0;
        int bi = N;
        if (has2 && lane >= j) {
            const double v = fabs(A[lane * LD + j]);
            if (v > best) {
                best = v;
                bi = lane;
            }
        }
        if (has1 && p1 >= j) {
            const double v = fabs(A[p1 * LD + j]);
            if (v > best) {
                best = v;
                bi = p1;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double ov = __shfl_xor_sync(kFull, best, o);
            const int oi = __shfl_xor_sync(kFull, bi, o);
            if (ov > best || (ov == best && oi < bi)) {
                best = ov;
                bi = oi;
            }
        }
        bi = __shfl_sync(kFull, bi, 0);
        const int p = bi < N ? bi : j;
        if (A[p * LD + j] == 0.0) {
            if (!info) info = j + 1;
            if (lane == 0) rdiag[j] = 0.0;
            __syncwarp();
            continue;
        }
        if (p != j)
            for (int c = lane; c < Z::NC; c += 32) {
                const double t = A[j * LD + c];
                A[j * LD + c] = A[p * LD + c];
                A[p * LD + c] = t;
            }
        __syncwarp();
        const double inv = 1.0 / A[j * LD + j];
        if (lane == 0) rdiag[j] = inv;
        if (has1 && p1 > j) eliminate_row<Z::NC>(A + p1 * LD, A + j * LD, j, inv);
        if (has2 && lane > j) eliminate_row<Z::NC>(A + lane * LD, A + j * LD, j, inv);
        __syncwarp();
    }
    return info;
}

template <int D, int KC>
__global__ void divergence_build_fixed_kernel(const float* __restrict__ pts, int64_t n,
                                              const uint32_t* __restrict__ idx, const double* __restrict__ spacing,
                                              int64_t spacing_batch, int shape, StencilOut out,
                                              int* __restrict__ status, int wpb) {
    using Z = AugSize<D, KC>;
    constexpr int N = Z::N, LD = Z::LD, OFF = Z::OFF;
    static_assert(KC <= 32, "one support per lane");
    extern __shared__ __align__(16) unsigned char smem[];
    const int w = threadIdx.x >> 5, lane = lane_id();
    double* A = reinterpret_cast<double*>(smem + Z::smem_per_warp * w);
    double* xs = A + N * LD;
    double* rdiag = xs + KC * D;
    const int p1 = OFF + lane;
    const bool has1 = p1 < N, has2 = lane < OFF;
    for (int64_t i = (int64_t)blockIdx.x * wpb + w; i < n; i += (int64_t)gridDim.x * wpb) {
        const NodeStencil<D> ns = load_node<D>(pts, n, idx, KC, i, spacing[i / spacing_batch], xs);
        if (ns.bad && lane == 0) atomicOr(status, 1);
        build_G0_rows<D, KC>(xs, shape, A);
        double b0[D], b1[D], cself[D];
        quad_rhs<D>(xs, KC, N, shape, ns, b0, b1, cself);
        // right-hand-side columns N .. N+D-1 (original row order), zero padding
        for (int r = 0; r < 2; ++r) {
            const int row = lane + 32 * r;
            if (row < N) {
#pragma unroll
                for (int d = 0; d < D; ++d) A[row * LD + N + d] = r == 0 ? b0[d] : b1[d];
                for (int c = N + D; c < Z::NC; ++c) A[row * LD + c] = 0.0;
            }
        }
        __syncwarp();
        if (aug_lu<D, KC>(A, rdiag)) atomicOr(status, 2);
        // back substitution, all right-hand sides at once: y1 holds row
        // OFF + lane, y2 row lane (lanes < OFF)
        double y1[D], y2[D];
#pragma unroll
        for (int d = 0; d < D; ++d) {
            y1[d] = has1 ? A[p1 * LD + N + d] : 0.0;
            y2[d] = has2 ? A[lane * LD + N + d] : 0.0;
        }
        for (int j = N - 1; j >= 0; --j) {
            const double rj = rdiag[j];
            double xj[D];
#pragma unroll
            for (int d = 0; d < D; ++d)
                xj[d] = (j >= OFF ? __shfl_sync(kFull, y1[d], j - OFF) : __shfl_sync(kFull, y2[d], j)) * rj;
            if (has1) {
                if (p1 == j) {
#pragma unroll
                    for (int d = 0; d < D; ++d) y1[d] = xj[d];
                } else if (p1 < j) {
                    const double u = A[p1 * LD + j];
#pragma unroll
                    for (int d = 0; d < D; ++d) y1[d] -= u * xj[d];
                }
            }
            if (has2) {
                if (lane == j) {
#pragma unroll
                    for (int d = 0; d < D; ++d) y2[d] = xj[d];
                } else if (lane < j) {
                    const double u = A[lane * LD + j];
#pragma unroll
                    for (int d = 0; d < D; ++d) y2[d] -= u * xj[d];
                }
            }
        }
        // weight of support t = lane: row t sits in lane t - OFF (or in y2)
        double W0[D], W1[D];
#pragma unroll
        for (int d = 0; d < D; ++d) {
            const double v = __shfl_sync(kFull, y1[d], (lane - OFF) & 31);
            W0[d] = (lane >= OFF ? v : y2[d]) + (lane == 0 ? cself[d] : 0.0);
            W1[d] = 0.0;
        }
        write_node<D>(out, i, KC, ns, W0, W1);
        __syncwarp();
    }
}

int warps_per_block_for(size_t per_warp) {
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    size_t lim = v > 0 ? (size_t)v : 48 * 1024;
    return (int)std::min<size_t>(8, lim / per_warp);
}

}  // namespace

// RBF weights on the device; status bits: 1 bad index, 2 singular, 4 no convergence
int rbf_weights_device(const float* src, int64_t nsrc, int dim, const uint32_t* support, int k, const double* qry,
                       int64_t ngroups, int group, double spacing, int shape, int precision, double* weights,
                       cudaStream_t st) {
    const int n = k + dim + 1;
    if (dim != 2 && dim != 3) return set_error(NAGA_EINVAL, "naga_rbf_weights: dim must be 2 or 3");
    if (k < dim + 1 || n > 64) return set_error(NAGA_EINVAL, "naga_rbf_weights: need dim + 1 <= k <= 60");
    if (group < 1 || ngroups < 0) return set_error(NAGA_EINVAL, "naga_rbf_weights: bad group size");
    if (!(spacing > 0)) return set_error(NAGA_EINVAL, "naga_rbf_weights: spacing must be > 0");
    if (shape != 0 && shape != 1) return set_error(NAGA_EINVAL, "naga_rbf_weights: unknown shape");
    if (precision != 0 && precision != 1) return set_error(NAGA_EINVAL, "naga_rbf_weights: unknown precision");
    if (ngroups == 0) return NAGA_OK;
    const size_t per_warp = rbf_smem_per_warp_h(n, k, dim, precision);
    const int wpb = warps_per_block_for(per_warp);
    if (wpb < 1) return set_error(NAGA_EINVAL, "naga_rbf_weights: system too large");
    int* d_status = nullptr;
    NAGA_CUDA_TRY(cudaMallocAsync(&d_status, 2 * sizeof(int), st));
    NAGA_CUDA_TRY(cudaMemsetAsync(d_status, 0, 2 * sizeof(int), st));
    const int blocks = (int)std::min<int64_t>((ngroups + wpb - 1) / wpb, (int64_t)sm_count() * 32);
    const size_t smem = per_warp * wpb;
    if (dim == 2) {
        NAGA_CUDA_TRY(cudaFuncSetAttribute(rbf_weights_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        rbf_weights_kernel<2><<<blocks, 32 * wpb, smem, st>>>(src, nsrc, support, k, qry, ngroups, group, spacing,
                                                              shape, precision, weights, d_status, wpb);
    } else {
        NAGA_CUDA_TRY(cudaFuncSetAttribute(rbf_weights_kernel<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        rbf_weights_kernel<3><<<blocks, 32 * wpb, smem, st>>>(src, nsrc, support, k, qry, ngroups, group, spacing,
                                                              shape, precision, weights, d_status, wpb);
    }
    NAGA_CUDA_TRY(cudaGetLastError());
    int h_st[2] = {0, 0};
    NAGA_CUDA_TRY(cudaMemcpyAsync(h_st, d_status, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
    NAGA_CUDA_TRY(cudaFreeAsync(d_status, st));
    NAGA_CUDA_TRY(cudaStreamSynchronize(st));
    const int h_status = h_st[0];
    g_fallbacks = h_st[1];
    if (h_status & 1) return set_error(NAGA_EINVAL, "naga_rbf_weights: support index out of range");
    if (h_status & 2) return set_error(NAGA_ESINGULAR, "naga_rbf_weights: singular moment matrix");
    return NAGA_OK;
}

// kNN + interaction radii + MQ spacing + stencil weights for pts[0, n)
int divergence_build_device(const float* pts, int64_t n, int dim, int k, int shape, int precision, uint32_t* idx,
                            StencilOut out, cudaStream_t st) {
    const int nsys = k + dim + 1;
    if (dim != 2 && dim != 3) return set_error(NAGA_EINVAL, "divergence build: dim must be 2 or 3");
    if (k < dim + 2 || nsys > 64) return set_error(NAGA_EINVAL, "divergence build: need dim + 2 <= k <= 60");
    if (n < k) return set_error(NAGA_EINVAL, "divergence build: fewer points than k");
    {
        // the quadrature table of this lattice, once per device
        static std::mutex mu;
        static bool filled[64][2] = {};
        int dev = 0;
        NAGA_CUDA_TRY(cudaGetDevice(&dev));
        std::lock_guard<std::mutex> lk(mu);
        if (dev >= 0 && dev < 64 && !filled[dev][dim - 2]) {
            if (dim == 2)
                quad_table_kernel<2><<<1, 64, 0, st>>>();
            else
                quad_table_kernel<3><<<1, 64, 0, st>>>();
            NAGA_CUDA_TRY(cudaGetLastError());
            NAGA_CUDA_TRY(cudaStreamSynchronize(st));
            filled[dev][dim - 2] = true;
        }
    }
    float* d2 = nullptr;
    double* nn = nullptr;
    double* sp = nullptr;
    int* d_status = nullptr;
    const int64_t batch = 16384;
    const int64_t nb = (n + batch - 1) / batch;
    NAGA_CUDA_TRY(cudaMallocAsync(&d2, sizeof(float) * n * k, st));
    int rc = knn_device(pts, n, pts, n, dim, k, idx, d2, st);
    if (rc) {
        cudaFreeAsync(d2, st);
        return rc;
    }
    NAGA_CUDA_TRY(cudaMallocAsync(&nn, sizeof(double) * n, st));
    NAGA_CUDA_TRY(cudaMallocAsync(&sp, sizeof(double) * nb, st));
    NAGA_CUDA_TRY(cudaMallocAsync(&d_status, 2 * sizeof(int), st));
    NAGA_CUDA_TRY(cudaMemsetAsync(d_status, 0, 2 * sizeof(int), st));
    {
        const int blocks = (int)std::min<int64_t>((n + 255) / 256, (int64_t)sm_count() * 8);
        if (dim == 2)
            nn_kernel<2><<<blocks, 256, 0, st>>>(pts, idx, k, n, nn);
        else
            nn_kernel<3><<<blocks, 256, 0, st>>>(pts, idx, k, n, nn);
        batch_mean_kernel<<<(unsigned)nb, 256, 0, st>>>(nn, n, batch, sp);
        NAGA_CUDA_TRY(cudaGetLastError());
    }
    auto fixed = [&](auto kern, size_t per_warp) -> int {
        const int wpb = warps_per_block_for(per_warp);
        const size_t smem = per_warp * wpb;
        const int blocks = (int)std::min<int64_t>((n + wpb - 1) / wpb, (int64_t)sm_count() * 32);
        NAGA_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        kern<<<blocks, 32 * wpb, smem, st>>>(pts, n, idx, sp, batch, shape, out, d_status, wpb);
        return NAGA_OK;
    };
    const size_t per_warp = rbf_smem_per_warp_h(nsys, k, dim, precision);
    const int wpb = warps_per_block_for(per_warp);
    const size_t smem = per_warp * wpb;
    const int blocks = (int)std::min<int64_t>((n + wpb - 1) / wpb, (int64_t)sm_count() * 32);
    int lrc = NAGA_OK;
    // FP64 builds of the benchmark stencil sizes take the fixed-size kernel
    if (precision == 0 && dim == 3 && k == 32) {
        lrc = fixed(divergence_build_fixed_kernel<3, 32>, AugSize<3, 32>::smem_per_warp);
    } else if (precision == 0 && dim == 2 && k == 16) {
        lrc = fixed(divergence_build_fixed_kernel<2, 16>, AugSize<2, 16>::smem_per_warp);
    } else if (dim == 2) {
        NAGA_CUDA_TRY(cudaFuncSetAttribute(divergence_build_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        divergence_build_kernel<2><<<blocks, 32 * wpb, smem, st>>>(pts, n, idx, k, sp, batch, shape, precision, out,
                                                                   d_status, wpb);
    } else {
        NAGA_CUDA_TRY(cudaFuncSetAttribute(divergence_build_kernel<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        divergence_build_kernel<3><<<blocks, 32 * wpb, smem, st>>>(pts, n, idx, k, sp, batch, shape, precision, out,
                                                                   d_status, wpb);
    }
    if (lrc) return lrc;
    NAGA_CUDA_TRY(cudaGetLastError());
    int h_st[2] = {0, 0};
    NAGA_CUDA_TRY(cudaMemcpyAsync(h_st, d_status, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
    NAGA_CUDA_TRY(cudaStreamSynchronize(st));
    const int h_status = h_st[0];
    g_fallbacks = h_st[1];
    cudaFreeAsync(d2, st);
    cudaFreeAsync(nn, st);
    cudaFreeAsync(sp, st);
    cudaFreeAsync(d_status, st);
    if (h_status & 1) return set_error(NAGA_EINVAL, "divergence build: support index out of range");
    if (h_status & 2) return set_error(NAGA_ESINGULAR, "divergence build: singular moment matrix");
    return NAGA_OK;
}

}  // namespace naga

using namespace naga;

extern "C" int64_t naga_refinement_fallbacks(void) { return naga::g_fallbacks; }

extern "C" int naga_rbf_weights(const float* src, int64_t n, int dim, const uint32_t* support, int k,
                                const double* qry, int64_t ngroups, int group, double spacing, int shape,
                                int precision, double* weights, void* stream) {
    if (ngroups > 0 && (!src || !support || !qry || !weights))
        return set_error(NAGA_EINVAL, "naga_rbf_weights: null pointer");
    return rbf_weights_device(src, n, dim, support, k, qry, ngroups, group, spacing, shape, precision, weights,
                              (cudaStream_t)stream);
}

extern "C" int naga_divergence_build(const float* pts, int64_t n, int dim, int k, int shape, int precision,
                                     uint32_t* idx, double* W, double* delta, void* stream) {
    if (!pts || !idx) return set_error(NAGA_EINVAL, "naga_divergence_build: null pointer");
    StencilOut out{};
    out.W64 = W;
    out.delta = delta;
    return divergence_build_device(pts, n, dim, k, shape, precision, idx, out, (cudaStream_t)stream);
}

extern "C" int naga_divergence_build_f32(const float* pts, int64_t n, int dim, int k, int shape, int precision,
                                         uint32_t* idx, float* W, float* delta, void* stream) {
    if (!pts || !idx) return set_error(NAGA_EINVAL, "naga_divergence_build_f32: null pointer");
    StencilOut out{};
    out.W32 = W;
    out.delta32 = delta;
    return divergence_build_device(pts, n, dim, k, shape, precision, idx, out, (cudaStream_t)stream);
}
