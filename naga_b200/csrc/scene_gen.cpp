// Synthetic scene inputs: jittered uniform grids in the unit square / cube,
// classified into the node classes NAGA's solver expects (bulk, absorbing
// layer, boundary), with PML absorption coefficients, inward boundary
// normals and Gaussian pressure pulses.
//
// The classification and the absorption profile follow NAGA's
// uniform_grid_provider (fluids/nonlocal_lattice_boltzmann/node_providers/
// uniform_grid_provider.cuh:65-161, detail/uniform_grid_provider.inl:
// 111-171): a node belongs to the layer when its squared distance to the
// nearest boundary node is <= L^2, and sigma = peak * ((L - d) / L)^2 in
// FP32. Boundary nodes sit on the walls, unjittered, with the outward grid
// normal (ranges/uniform_grid.cuh:255-293) negated to point inward.
//
// Node order within each class is Morton order of the grid indices, which
// keeps stencil neighbours close in memory for the GPU gathers.
#include "naga_b200.h"
#include "naga_internal.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace naga {

namespace {

inline uint64_t splitmix64(uint64_t& s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
inline double uniform01(uint64_t& s) { return (double)(splitmix64(s) >> 11) * (1.0 / 9007199254740992.0); }

inline uint64_t spread_bits3(uint64_t v) {
    v &= 0x1fffff;
    v = (v | v << 32) & 0x1f00000000ffffull;
    v = (v | v << 16) & 0x1f0000ff0000ffull;
    v = (v | v << 8) & 0x100f00f00f00f00full;
    v = (v | v << 4) & 0x10c30c30c30c30c3ull;
    v = (v | v << 2) & 0x1249249249249249ull;
    return v;
}
inline uint64_t spread_bits2(uint64_t v) {
    v &= 0xffffffff;
    v = (v | v << 16) & 0x0000ffff0000ffffull;
    v = (v | v << 8) & 0x00ff00ff00ff00ffull;
    v = (v | v << 4) & 0x0f0f0f0f0f0f0f0full;
    v = (v | v << 2) & 0x3333333333333333ull;
    v = (v | v << 1) & 0x5555555555555555ull;
    return v;
}

// squared distance with the highest dimension added last, FP32
inline float d2_ref(const float* a, const float* b, int dim) {
    float s = (a[0] - b[0]) * (a[0] - b[0]);
    for (int d = 1; d < dim; ++d) {
        float t = (a[d] - b[d]) * (a[d] - b[d]);
        s = t + s;
    }
    return s;
}

struct GridNode {
    uint64_t morton;
    int64_t lin;  // row-major grid index
};

}  // namespace

// Builds the full node set; returns 0 on success.
int build_grid_scene(const naga_grid_spec& sp, GridScene& out) {
    const int dim = sp.dim;
    const int64_t n1 = sp.n_side;
    if ((dim != 2 && dim != 3) || n1 < 3 || !(sp.jitter >= 0 && sp.jitter < 0.5) || sp.n_layers < 0)
        return NAGA_EINVAL;
    int64_t total = n1 * n1 * (dim == 3 ? n1 : 1);
    if (total > (int64_t)UINT32_MAX / 2) return NAGA_EINVAL;
    const double h = 1.0 / (double)(n1 - 1);
    out.dim = dim;
    out.h = h;

    // positions in row-major order (x fastest); every node draws `dim`
    // uniforms so the stream does not depend on the node's class
    std::vector<float> pos((size_t)total * dim);
    std::vector<char> is_bnd(total, 0);
    uint64_t state = sp.seed;
    for (int64_t n = 0; n < total; ++n) {
        int64_t g[3] = {n % n1, (n / n1) % n1, dim == 3 ? n / (n1 * n1) : 0};
        bool bnd = false;
        for (int d = 0; d < dim; ++d) bnd = bnd || g[d] == 0 || g[d] == n1 - 1;
        is_bnd[n] = bnd;
        for (int d = 0; d < dim; ++d) {
            double u = uniform01(state);
            double x = (double)g[d] * h;
            if (!bnd) x += (2.0 * u - 1.0) * sp.jitter * h;
            pos[(size_t)n * dim + d] = (float)x;
        }
    }

    // nearest boundary node: the boundary nodes of each wall form a regular
    // grid, so the nearest one on a wall is found by rounding the in-wall
    // coordinates (neighbours +-1 are checked to stay exact in FP32)
    const float Lt = (float)sp.n_layers * (float)h;
    std::vector<float> dist2(total, INFINITY);
    for (int64_t n = 0; n < total; ++n) {
        if (is_bnd[n]) continue;
        const float* p = &pos[(size_t)n * dim];
        float best = INFINITY;
        for (int wd = 0; wd < dim; ++wd)
            for (int side = 0; side < 2; ++side) {
                int64_t base[3];
                for (int d = 0; d < dim; ++d)
                    base[d] = std::min<int64_t>(std::max<int64_t>(std::llround((double)p[d] / h), 0), n1 - 1);
                base[wd] = side ? n1 - 1 : 0;
                int64_t lo0 = -1, hi0 = 1;
                for (int64_t a = lo0; a <= hi0; ++a)
                    for (int64_t b = (dim == 3 ? lo0 : 0); b <= (dim == 3 ? hi0 : 0); ++b) {
                        int64_t g[3] = {base[0], base[1], base[2]};
                        int od[2], c = 0;
                        for (int d = 0; d < dim; ++d)
                            if (d != wd) od[c++] = d;
                        g[od[0]] += a;
                        if (dim == 3) g[od[1]] += b;
                        bool ok = true;
                        for (int d = 0; d < dim; ++d) ok = ok && g[d] >= 0 && g[d] < n1;
                        if (!ok) continue;
                        float q[3];
                        for (int d = 0; d < dim; ++d) q[d] = (float)((double)g[d] * h);
                        best = std::min(best, d2_ref(p, q, dim));
                    }
            }
        dist2[n] = best;
    }

    std::vector<GridNode> bulk, layer, bnd;
    for (int64_t n = 0; n < total; ++n) {
        int64_t g[3] = {n % n1, (n / n1) % n1, dim == 3 ? n / (n1 * n1) : 0};
        uint64_t m = dim == 3 ? (spread_bits3(g[0]) | spread_bits3(g[1]) << 1 | spread_bits3(g[2]) << 2)
                              : (spread_bits2(g[0]) | spread_bits2(g[1]) << 1);
        GridNode gn{m, n};
        if (is_bnd[n])
            bnd.push_back(gn);
        else if (sp.n_layers > 0 && dist2[n] <= Lt * Lt)
            layer.push_back(gn);
        else
            bulk.push_back(gn);
    }
    auto by_morton = [](const GridNode& a, const GridNode& b) { return a.morton < b.morton; };
    std::sort(bulk.begin(), bulk.end(), by_morton);
    std::sort(layer.begin(), layer.end(), by_morton);
    std::sort(bnd.begin(), bnd.end(), by_morton);

    out.n_bulk = (int64_t)bulk.size();
    out.n_layer = (int64_t)layer.size();
    out.n_boundary = (int64_t)bnd.size();
    out.points.resize((size_t)total * dim);
    out.normals.resize((size_t)out.n_boundary * dim);
    out.sigma.resize((size_t)out.n_layer);
    out.grid_index.resize((size_t)total);
    int64_t w = 0;
    auto emit = [&](const GridNode& gn) {
        std::memcpy(&out.points[(size_t)w * dim], &pos[(size_t)gn.lin * dim], sizeof(float) * dim);
        out.grid_index[w] = gn.lin;
        ++w;
    };
    for (auto& gn : bulk) emit(gn);
    for (size_t t = 0; t < layer.size(); ++t) {
        float d = std::sqrt(dist2[layer[t].lin]);
        float r = (Lt - d) / Lt;
        out.sigma[t] = (float)sp.sigma_peak * (r * r);
        emit(layer[t]);
    }
    for (size_t t = 0; t < bnd.size(); ++t) {
        int64_t n = bnd[t].lin;
        int64_t g[3] = {n % n1, (n / n1) % n1, dim == 3 ? n / (n1 * n1) : 0};
        float nv[3] = {0, 0, 0};
        for (int d = 0; d < dim; ++d) nv[d] = g[d] == 0 ? -1.f : (g[d] == n1 - 1 ? 1.f : 0.f);
        float nn = 0;
        for (int d = 0; d < dim; ++d) nn += nv[d] * nv[d];
        nn = std::sqrt(nn);
        for (int d = 0; d < dim; ++d) out.normals[t * dim + d] = -(nv[d] / (nn == 0 ? 1.f : nn));
        emit(bnd[t]);
    }
    return NAGA_OK;
}

}  // namespace naga

using namespace naga;

extern "C" int naga_grid_counts(const naga_grid_spec* spec, int64_t* n_bulk, int64_t* n_layer,
                                int64_t* n_boundary) {
    if (!spec) return set_error(NAGA_EINVAL, "naga_grid_counts: null spec");
    GridScene s;
    int rc = build_grid_scene(*spec, s);
    if (rc) return set_error(rc, "naga_grid_counts: invalid grid spec");
    if (n_bulk) *n_bulk = s.n_bulk;
    if (n_layer) *n_layer = s.n_layer;
    if (n_boundary) *n_boundary = s.n_boundary;
    return NAGA_OK;
}

extern "C" int naga_grid_generate(const naga_grid_spec* spec, float* points, float* normals,
                                  float* sigma, double* nodal_spacing) {
    if (!spec) return set_error(NAGA_EINVAL, "naga_grid_generate: null spec");
    GridScene s;
    int rc = build_grid_scene(*spec, s);
    if (rc) return set_error(rc, "naga_grid_generate: invalid grid spec");
    if (points) std::memcpy(points, s.points.data(), s.points.size() * sizeof(float));
    if (normals) std::memcpy(normals, s.normals.data(), s.normals.size() * sizeof(float));
    if (sigma) std::memcpy(sigma, s.sigma.data(), s.sigma.size() * sizeof(float));
    if (nodal_spacing) *nodal_spacing = s.h;
    return NAGA_OK;
}

extern "C" int naga_gaussian_pulse(const float* points, int64_t n, int dim, const double* center,
                                   double amplitude, double width, float* drho) {
    if (!points || !center || !drho || n < 0 || dim < 1 || dim > 3 || !(width > 0))
        return set_error(NAGA_EINVAL, "naga_gaussian_pulse: invalid argument");
    for (int64_t i = 0; i < n; ++i) {
        double r2 = 0;
        for (int d = 0; d < dim; ++d) {
            double t = (double)points[i * dim + d] - center[d];
            r2 += t * t;
        }
        drho[i] = (float)(amplitude * std::exp(-r2 / (2.0 * width * width)));
    }
    return NAGA_OK;
}
