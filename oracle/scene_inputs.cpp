// Synthetic scene inputs for the oracle: jittered unit grids with the node
// classes of NAGA's uniform_grid_provider, and Gaussian pulses.
// TEST INFRASTRUCTURE ONLY (see naga_oracle.h). The benchmark's CPU
// baseline and the fixture scripts build their scenes with these, so they
// never load the product library; tests/test_oracle.py checks the output bit
// for bit against the library's naga_grid_generate / naga_gaussian_pulse.
//
// Definition of the grid (the benchmark configurations' "regular grid with
// spacing h, each point jittered uniformly by up to +-jitter h"):
//   * node (i, j[, l]) of an n^dim grid, h = 1 / (n - 1), row-major index
//     m = i + n (j + n l);
//   * coordinate d of node m uses draw m dim + d of the splitmix64 stream of
//     `seed` (Steele, Lea, Flood, "Fast splittable pseudorandom number
//     generators", OOPSLA 2014: state seed + (t + 1) 0x9E3779B97F4A7C15, then
//     the variant-13 finaliser), u = top 53 bits / 2^53, and is
//     x = i h + (2u - 1) jitter h in FP64, stored FP32; wall nodes are not
//     jittered;
//   * classes as NAGA's uniform_grid_provider (node_providers/
//     uniform_grid_provider.cuh:65-161, detail/uniform_grid_provider.inl:
//     111-171): walls = boundary with the inward unit normal; a non-wall node
//     is in the layer when its FP32 squared distance to the nearest wall node
//     is <= (n_layers h)^2, sigma = peak ((L - d) / L)^2 in FP32; the rest is
//     bulk;
//   * order: bulk, layer, boundary, each by increasing Morton key of the grid
//     indices (bits interleaved, x lowest).
// The nearest wall node is searched here in a 5-wide window around the
// rounded in-wall coordinates of each wall, by a plain minimum.

#include "naga_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace {

uint64_t splitmix64(uint64_t seed, uint64_t t) {
    uint64_t z = seed + (t + 1) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// squared distance, highest dimension added last (distance_functions.hpp:
// 138-161); the Makefile's -ffp-contract=off keeps it unfused
float sqdist(const float* a, const float* b, int dim) {
    float s = (a[0] - b[0]) * (a[0] - b[0]);
    for (int d = 1; d < dim; ++d) s = (a[d] - b[d]) * (a[d] - b[d]) + s;
    return s;
}

uint64_t morton_key(int dim, const int64_t* g) {
    uint64_t key = 0;
    for (int b = 0; b < 21; ++b)
        for (int d = 0; d < dim; ++d) key |= (uint64_t)((g[d] >> b) & 1) << (b * dim + d);
    return key;
}

struct Grid {
    int dim = 0;
    double h = 0;
    std::vector<int64_t> order;  // grid indices: bulk, layer, boundary
    int64_t counts[3] = {0, 0, 0};
    std::vector<float> pos;      // row-major grid order
    std::vector<float> dist2;
};

int make_grid(int dim, int64_t n1, int n_layers, double jitter, uint64_t seed, Grid& G) {
    if ((dim != 2 && dim != 3) || n1 < 3 || n_layers < 0 || !(jitter >= 0 && jitter < 0.5)) return 1;
    const int64_t total = n1 * n1 * (dim == 3 ? n1 : 1);
    const double h = 1.0 / (double)(n1 - 1);
    G.dim = dim;
    G.h = h;
    G.pos.assign((size_t)total * dim, 0.f);
    std::vector<char> wall(total, 0);
    for (int64_t m = 0; m < total; ++m) {
        int64_t g[3] = {m % n1, (m / n1) % n1, m / (n1 * n1)};
        bool w = false;
        for (int d = 0; d < dim; ++d) w = w || g[d] == 0 || g[d] == n1 - 1;
        wall[m] = w;
        for (int d = 0; d < dim; ++d) {
            double u = (double)(splitmix64(seed, (uint64_t)m * dim + d) >> 11) / 9007199254740992.0;
            double x = (double)g[d] * h;
            if (!w) x += (2.0 * u - 1.0) * jitter * h;
            G.pos[(size_t)m * dim + d] = (float)x;
        }
    }
    const float L = (float)n_layers * (float)h;
    G.dist2.assign(total, INFINITY);
    for (int64_t m = 0; m < total; ++m) {
        if (wall[m]) continue;
        const float* p = &G.pos[(size_t)m * dim];
        int64_t c[3] = {0, 0, 0};
        for (int d = 0; d < dim; ++d) c[d] = std::llround((double)p[d] / h);
        float best = INFINITY;
        for (int wd = 0; wd < dim; ++wd)
            for (int64_t side : {(int64_t)0, n1 - 1}) {
                int od[2] = {-1, -1}, no = 0;
                for (int d = 0; d < dim; ++d)
                    if (d != wd) od[no++] = d;
                const int span1 = dim == 3 ? 2 : 0;
                for (int64_t a = -2; a <= 2; ++a)
                    for (int64_t b = -span1; b <= span1; ++b) {
                        int64_t g[3] = {c[0], c[1], c[2]};
                        g[wd] = side;
                        g[od[0]] += a;
                        if (dim == 3) g[od[1]] += b;
                        bool inside = true;
                        for (int d = 0; d < dim; ++d) inside = inside && g[d] >= 0 && g[d] < n1;
                        if (!inside) continue;
                        float q[3];
                        for (int d = 0; d < dim; ++d) q[d] = (float)((double)g[d] * h);
                        best = std::min(best, sqdist(p, q, dim));
                    }
            }
        G.dist2[m] = best;
    }
    std::vector<std::pair<uint64_t, int64_t>> keyed((size_t)total);
    for (int64_t m = 0; m < total; ++m) {
        int64_t g[3] = {m % n1, (m / n1) % n1, m / (n1 * n1)};
        keyed[m] = {morton_key(dim, g), m};
    }
    std::sort(keyed.begin(), keyed.end());
    std::vector<int64_t> cls[3];
    for (auto& km : keyed) {
        const int64_t m = km.second;
        int c = wall[m] ? 2 : (n_layers > 0 && G.dist2[m] <= L * L ? 1 : 0);
        cls[c].push_back(m);
    }
    G.order.clear();
    for (int c = 0; c < 3; ++c) {
        G.counts[c] = (int64_t)cls[c].size();
        G.order.insert(G.order.end(), cls[c].begin(), cls[c].end());
    }
    return 0;
}

}  // namespace

extern "C" int orc_grid_generate(int dim, int64_t n_side, int n_layers, double jitter,
                                 double sigma_peak, uint64_t seed, int64_t* counts, float* points,
                                 float* normals, float* sigma, double* h) {
    Grid G;
    if (make_grid(dim, n_side, n_layers, jitter, seed, G)) return 1;
    if (counts) std::memcpy(counts, G.counts, sizeof G.counts);
    if (h) *h = G.h;
    const int64_t nb = G.counts[0], nl = G.counts[1], nw = G.counts[2];
    const float L = (float)n_layers * (float)G.h;
    for (int64_t t = 0; t < nb + nl + nw; ++t) {
        const int64_t m = G.order[t];
        if (points) std::memcpy(points + t * dim, &G.pos[(size_t)m * dim], sizeof(float) * dim);
        if (t >= nb && t < nb + nl && sigma) {
            float r = (L - std::sqrt(G.dist2[m])) / L;
            sigma[t - nb] = (float)sigma_peak * (r * r);
        }
        if (t >= nb + nl && normals) {
            int64_t g[3] = {m % n_side, (m / n_side) % n_side, m / (n_side * n_side)};
            float out[3] = {0, 0, 0}, len2 = 0;
            for (int d = 0; d < dim; ++d) {
                out[d] = g[d] == 0 ? -1.f : (g[d] == n_side - 1 ? 1.f : 0.f);
                len2 += out[d] * out[d];
            }
            float len = std::sqrt(len2);
            for (int d = 0; d < dim; ++d) normals[(t - nb - nl) * dim + d] = -(out[d] / len);
        }
    }
    return 0;
}

extern "C" int orc_gaussian_pulse(const float* points, int64_t n, int dim, const double* center,
                                  double amplitude, double width, float* drho) {
    if (!points || !center || !drho || n < 0 || dim < 1 || dim > 3 || !(width > 0)) return 1;
    for (int64_t i = 0; i < n; ++i) {
        double r2 = 0;
        for (int d = 0; d < dim; ++d) {
            const double t = (double)points[i * dim + d] - center[d];
            r2 += t * t;
        }
        drho[i] = (float)(amplitude * std::exp(-r2 / (2.0 * width * width)));
    }
    return 0;
}
