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
// keeps stencil neighbours close in memory for the GPU gathers. The per-node
// loops run on all host threads; the result does not depend on their number.
#include "naga_b200.h"
#include "naga_internal.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

namespace naga {

namespace {

// splitmix64: draw k (0-based) of the stream seeded with `seed` is the mix
// of seed + (k + 1) * gamma, so any draw can be computed directly
inline uint64_t splitmix64_at(uint64_t seed, uint64_t k) {
    uint64_t z = seed + (k + 1) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
inline double uniform01_at(uint64_t seed, uint64_t k) {
    return (double)(splitmix64_at(seed, k) >> 11) * (1.0 / 9007199254740992.0);
}

// fn(begin, end) over [0, n) in contiguous chunks on the host's threads
template <class Fn>
void parallel_for(int64_t n, Fn fn) {
    const int64_t hw = std::max(1u, std::thread::hardware_concurrency());
    const int64_t nt = std::max<int64_t>(1, std::min<int64_t>(hw, n / 16384));
    if (nt == 1) {
        fn((int64_t)0, n);
        return;
    }
    std::vector<std::thread> th;
    for (int64_t t = 0; t < nt; ++t) th.emplace_back(fn, n * t / nt, n * (t + 1) / nt);
    for (auto& x : th) x.join();
}

// row-major grid indices of the n1^dim grid in increasing Morton order
// (interleaved bits, x lowest), by walking the octants (quadrants) in order
void morton_walk(int dim, int64_t n1, int64_t x0, int64_t y0, int64_t z0, int64_t size,
                 std::vector<int64_t>& out) {
    if (x0 >= n1 || y0 >= n1 || z0 >= n1) return;
    if (size == 1) {
        out.push_back(x0 + n1 * (y0 + n1 * z0));
        return;
    }
    const int64_t hs = size / 2;
    const int nc = dim == 3 ? 8 : 4;
    for (int c = 0; c < nc; ++c)
        morton_walk(dim, n1, x0 + (c & 1) * hs, y0 + ((c >> 1) & 1) * hs, z0 + ((c >> 2) & 1) * hs, hs, out);
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
    // uniforms (draws n dim + d of the seed's stream), so the stream does not
    // depend on the node's class
    std::vector<float> pos((size_t)total * dim);
    std::vector<char> is_bnd(total, 0);
    const uint64_t seed = sp.seed;
    parallel_for(total, [&](int64_t b0, int64_t b1) {
        for (int64_t n = b0; n < b1; ++n) {
            int64_t g[3] = {n % n1, (n / n1) % n1, dim == 3 ? n / (n1 * n1) : 0};
            bool bnd = false;
            for (int d = 0; d < dim; ++d) bnd = bnd || g[d] == 0 || g[d] == n1 - 1;
            is_bnd[n] = bnd;
            for (int d = 0; d < dim; ++d) {
                double u = uniform01_at(seed, (uint64_t)n * dim + d);
                double x = (double)g[d] * h;
                if (!bnd) x += (2.0 * u - 1.0) * sp.jitter * h;
                pos[(size_t)n * dim + d] = (float)x;
            }
        }
    });

    // nearest boundary node: the boundary nodes of each wall form a regular
    // grid, so the nearest one on a wall is found by rounding the in-wall
    // coordinates (neighbours +-1 are checked to stay exact in FP32)
    const float Lt = (float)sp.n_layers * (float)h;
    std::vector<float> dist2(total, INFINITY);
    parallel_for(total, [&](int64_t b0, int64_t b1) {
        for (int64_t n = b0; n < b1; ++n) {
            if (is_bnd[n]) continue;
            const float* p = &pos[(size_t)n * dim];
            float best = INFINITY;
            for (int wd = 0; wd < dim; ++wd)
                for (int side = 0; side < 2; ++side) {
                    int64_t base[3];
                    for (int d = 0; d < dim; ++d)
                        base[d] = std::min<int64_t>(std::max<int64_t>(std::llround((double)p[d] / h), 0), n1 - 1);
                    base[wd] = side ? n1 - 1 : 0;
                    for (int64_t a = -1; a <= 1; ++a)
                        for (int64_t b = (dim == 3 ? -1 : 0); b <= (dim == 3 ? 1 : 0); ++b) {
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
    });

    // classes in Morton order of the grid indices
    std::vector<int64_t> order;
    order.reserve((size_t)total);
    int64_t size = 1;
    while (size < n1) size *= 2;
    morton_walk(dim, n1, 0, 0, 0, size, order);
    std::vector<int64_t> bulk, layer, bnd;  // row-major grid indices
    for (int64_t n : order) {
        if (is_bnd[n])
            bnd.push_back(n);
        else if (sp.n_layers > 0 && dist2[n] <= Lt * Lt)
            layer.push_back(n);
        else
            bulk.push_back(n);
    }

    out.n_bulk = (int64_t)bulk.size();
    out.n_layer = (int64_t)layer.size();
    out.n_boundary = (int64_t)bnd.size();
    out.points.resize((size_t)total * dim);
    out.normals.resize((size_t)out.n_boundary * dim);
    out.sigma.resize((size_t)out.n_layer);
    out.grid_index.resize((size_t)total);
    int64_t w = 0;
    auto emit = [&](int64_t lin) {
        std::memcpy(&out.points[(size_t)w * dim], &pos[(size_t)lin * dim], sizeof(float) * dim);
        out.grid_index[w] = lin;
        ++w;
    };
    for (int64_t n : bulk) emit(n);
    for (size_t t = 0; t < layer.size(); ++t) {
        float d = std::sqrt(dist2[layer[t]]);
        float r = (Lt - d) / Lt;
        out.sigma[t] = (float)sp.sigma_peak * (r * r);
        emit(layer[t]);
    }
    for (size_t t = 0; t < bnd.size(); ++t) {
        int64_t n = bnd[t];
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


namespace {
// grid indices of an nx x ny x nz box in increasing Morton order (x lowest)
void morton_walk_box(int dim, const int64_t* n, int64_t x0, int64_t y0, int64_t z0, int64_t size,
                     std::vector<int64_t>& out) {
    if (x0 >= n[0] || y0 >= n[1] || z0 >= n[2]) return;
    if (size == 1) {
        out.push_back(x0 + n[0] * (y0 + n[1] * z0));
        return;
    }
    const int64_t hs = size / 2;
    const int nc = dim == 3 ? 8 : 4;
    for (int c = 0; c < nc; ++c)
        morton_walk_box(dim, n, x0 + (c & 1) * hs, y0 + ((c >> 1) & 1) * hs, z0 + ((c >> 2) & 1) * hs, hs, out);
}
}  // namespace

// NAGA's uniform_grid_provider (node_providers/uniform_grid_provider.cuh:
// 53-161) restated on the host, in its FP32 arithmetic: per axis
// ceil((max - min) / h) + 1 nodes at the spacing that fits the box
// (ranges/uniform_grid.cuh:58-64, node n at min + (n % size) * spacing, x
// fastest); the outer shell is the boundary with the normalised outward
// face normal negated (uniform_grid.cuh:243-293, provider :89-94); a
// non-boundary node is in the layer when the squared distance to its
// nearest boundary node -- the projection onto its nearest face -- is
// <= L^2, with sigma = peak ((L - d) / L)^2 (detail/uniform_grid_provider.
// inl:111-171). Classes come in NAGA's order [bulk, layer, boundary]; inside
// each, Morton order (NAGA's is the order of atomic increments, not
// reproducible) or the grid order.
int build_box_scene(const naga_box_grid_spec& sp, GridScene& out) {
    const int dim = sp.dim;
    if (dim != 2 && dim != 3) return NAGA_EINVAL;
    const float h = (float)sp.spacing;
    if (!(h > 0) || !(sp.layer_thickness >= 0)) return NAGA_EINVAL;
    float mn[3] = {0, 0, 0}, sp_[3] = {1, 1, 1};
    int64_t n[3] = {1, 1, 1};
    int64_t total = 1;
    for (int d = 0; d < dim; ++d) {
        mn[d] = (float)sp.min[d];
        const float ext = (float)sp.max[d] - mn[d];
        if (!(ext > 0)) return NAGA_EINVAL;
        n[d] = (int64_t)std::ceil(ext / h) + 1;
        if (n[d] < 3) return NAGA_EINVAL;
        sp_[d] = ext / (float)(n[d] - 1);
        total *= n[d];
    }
    if (total > (int64_t)UINT32_MAX / 2) return NAGA_EINVAL;
    float hi[3] = {0, 0, 0};  // coordinate of the high face's nodes
    for (int d = 0; d < dim; ++d) hi[d] = mn[d] + (float)(n[d] - 1) * sp_[d];
    const float L = (float)sp.layer_thickness;
    out.dim = dim;
    out.h = h;

    std::vector<float> pos((size_t)total * dim);
    std::vector<char> is_bnd(total, 0);
    std::vector<float> dist2(total, 0.f);
    parallel_for(total, [&](int64_t b, int64_t e) {
        for (int64_t t = b; t < e; ++t) {
            int64_t r = t;
            bool bnd = false;
            float best = 0.f;
            bool first = true;
            for (int d = 0; d < dim; ++d) {
                const int64_t g = r % n[d];
                r /= n[d];
                const float x = mn[d] + (float)g * sp_[d];
                pos[(size_t)t * dim + d] = x;
                if (g == 0 || g == n[d] - 1) bnd = true;
                const float lo = (x - mn[d]) * (x - mn[d]), up = (x - hi[d]) * (x - hi[d]);
                const float m = std::min(lo, up);
                if (first || m < best) best = m;
                first = false;
            }
            is_bnd[t] = bnd;
            dist2[t] = best;
        }
    });

    std::vector<int64_t> order;
    order.reserve((size_t)total);
    if (sp.morton) {
        int64_t size = 1;
        while (size < std::max(n[0], std::max(n[1], n[2]))) size *= 2;
        morton_walk_box(dim, n, 0, 0, 0, size, order);
    } else {
        for (int64_t t = 0; t < total; ++t) order.push_back(t);
    }
    std::vector<int64_t> bulk, layer, bnd;
    for (int64_t t : order) {
        if (is_bnd[t])
            bnd.push_back(t);
        else if (L > 0 && dist2[t] <= L * L)
            layer.push_back(t);
        else
            bulk.push_back(t);
    }
    out.n_bulk = (int64_t)bulk.size();
    out.n_layer = (int64_t)layer.size();
    out.n_boundary = (int64_t)bnd.size();
    out.points.resize((size_t)total * dim);
    out.normals.resize((size_t)out.n_boundary * dim);
    out.sigma.resize((size_t)out.n_layer);
    out.grid_index.resize((size_t)total);
    int64_t w = 0;
    auto emit = [&](int64_t lin) {
        std::memcpy(&out.points[(size_t)w * dim], &pos[(size_t)lin * dim], sizeof(float) * dim);
        out.grid_index[w] = lin;
        ++w;
    };
    for (int64_t t : bulk) emit(t);
    for (size_t q = 0; q < layer.size(); ++q) {
        const float d = std::sqrt(dist2[layer[q]]);
        const float r = (L - d) / L;
        out.sigma[q] = (float)sp.peak_absorption * (r * r);
        emit(layer[q]);
    }
    for (size_t q = 0; q < bnd.size(); ++q) {
        int64_t r = bnd[q];
        float nv[3] = {0, 0, 0};
        for (int d = 0; d < dim; ++d) {
            const int64_t g = r % n[d];
            r /= n[d];
            nv[d] = g == 0 ? -1.f : (g == n[d] - 1 ? 1.f : 0.f);
        }
        float nn = 0;
        for (int d = 0; d < dim; ++d) nn += nv[d] * nv[d];
        nn = std::sqrt(nn);
        for (int d = 0; d < dim; ++d) out.normals[q * dim + d] = -(nv[d] / (nn == 0 ? 1.f : nn));
        emit(bnd[q]);
    }
    return NAGA_OK;
}

}  // namespace naga

using namespace naga;

namespace {
// the last grid built on this thread: the usual call pair (counts to size
// the buffers, then generate) builds it once
struct GridCache {
    bool valid = false;
    naga_grid_spec spec{};
    GridScene scene;
};
thread_local GridCache g_grid_cache;

bool same_spec(const naga_grid_spec& a, const naga_grid_spec& b) {
    return a.dim == b.dim && a.n_layers == b.n_layers && a.n_side == b.n_side && a.jitter == b.jitter &&
           a.sigma_peak == b.sigma_peak && a.seed == b.seed;
}

int cached_grid(const naga_grid_spec& spec, const GridScene** out) {
    GridCache& c = g_grid_cache;
    if (!c.valid || !same_spec(c.spec, spec)) {
        c.valid = false;
        c.scene = GridScene{};
        int rc = build_grid_scene(spec, c.scene);
        if (rc) return rc;
        c.spec = spec;
        c.valid = true;
    }
    *out = &c.scene;
    return NAGA_OK;
}
}  // namespace

extern "C" int naga_grid_counts(const naga_grid_spec* spec, int64_t* n_bulk, int64_t* n_layer,
                                int64_t* n_boundary) {
    if (!spec) return set_error(NAGA_EINVAL, "naga_grid_counts: null spec");
    const GridScene* sp = nullptr;
    int rc = cached_grid(*spec, &sp);
    if (rc) return set_error(rc, "naga_grid_counts: invalid grid spec");
    const GridScene& s = *sp;
    if (n_bulk) *n_bulk = s.n_bulk;
    if (n_layer) *n_layer = s.n_layer;
    if (n_boundary) *n_boundary = s.n_boundary;
    return NAGA_OK;
}

extern "C" int naga_grid_generate(const naga_grid_spec* spec, float* points, float* normals,
                                  float* sigma, double* nodal_spacing) {
    if (!spec) return set_error(NAGA_EINVAL, "naga_grid_generate: null spec");
    const GridScene* sp = nullptr;
    int rc = cached_grid(*spec, &sp);
    if (rc) return set_error(rc, "naga_grid_generate: invalid grid spec");
    const GridScene& s = *sp;
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

namespace {
struct BoxCache {
    bool valid = false;
    naga_box_grid_spec spec{};
    GridScene scene;
};
thread_local BoxCache g_box_cache;

int cached_box(const naga_box_grid_spec& spec, const GridScene** out) {
    BoxCache& c = g_box_cache;
    if (!c.valid || std::memcmp(&c.spec, &spec, sizeof spec) != 0) {
        c.valid = false;
        c.scene = GridScene{};
        int rc = build_box_scene(spec, c.scene);
        if (rc) return rc;
        c.spec = spec;
        c.valid = true;
    }
    *out = &c.scene;
    return NAGA_OK;
}
}  // namespace

extern "C" int naga_box_grid_counts(const naga_box_grid_spec* spec, int64_t* n_bulk, int64_t* n_layer,
                                    int64_t* n_boundary) {
    if (!spec) return set_error(NAGA_EINVAL, "naga_box_grid_counts: null spec");
    naga_box_grid_spec key = *spec;
    const GridScene* g = nullptr;
    int rc = cached_box(key, &g);
    if (rc) return set_error(rc, "naga_box_grid_counts: invalid box grid spec");
    if (n_bulk) *n_bulk = g->n_bulk;
    if (n_layer) *n_layer = g->n_layer;
    if (n_boundary) *n_boundary = g->n_boundary;
    return NAGA_OK;
}

extern "C" int naga_box_grid_generate(const naga_box_grid_spec* spec, float* points, float* normals, float* sigma,
                                      double* nodal_spacing) {
    if (!spec) return set_error(NAGA_EINVAL, "naga_box_grid_generate: null spec");
    naga_box_grid_spec key = *spec;
    const GridScene* g = nullptr;
    int rc = cached_box(key, &g);
    if (rc) return set_error(rc, "naga_box_grid_generate: invalid box grid spec");
    if (points) std::memcpy(points, g->points.data(), g->points.size() * sizeof(float));
    if (normals) std::memcpy(normals, g->normals.data(), g->normals.size() * sizeof(float));
    if (sigma) std::memcpy(sigma, g->sigma.data(), g->sigma.size() * sizeof(float));
    if (nodal_spacing) *nodal_spacing = g->h;
    return NAGA_OK;
}
