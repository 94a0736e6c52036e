// A NAGA-style density source through the C++ facade: a sinusoidal point
// source at the node nearest the centre of a D2Q9 domain, registered with
// register_density_source and evaluated by the engine before every step.
// Prints one line per step: t, the source value used, rho_a - 1, rho_b - 1.
#include <naga/naga.hpp>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

using namespace naga::fluids::nonlocal_lbm;
using lattice_t = d2q9_lattice<float>;

struct point_source : density_source<lattice_t> {
    size_t node = 0;
    float period = 1;
    std::vector<float> used;
    void add_density_source(const simulation_nodes<float>&, const problem_parameters<float>&, const float& time,
                            std::vector<float>& terms) override {
        const float v = (float)(2e-4 * std::sin(2.0 * 3.14159265358979 * time / period));
        terms[node] = v;
        used.push_back(v);
    }
};

int main(int argc, char** argv) {
    const int steps = argc > 1 ? std::atoi(argv[1]) : 20;
    jittered_grid_provider<lattice_t> provider(40, 4, 0.1, 0);
    auto nodes = provider.get();
    engine_options opt;
    opt.k = 16;
    opt.shape = 1;
    simulation_engine<lattice_t> engine(opt);
    const float dt = 0.5f * nodes.nodal_spacing;
    engine.set_problem_parameters(1e-5f, 1.0f, dt, 1.0f);
    engine.init_domain(nodes);
    density_observer<lattice_t> a({0.3f, 0.5f}), b({0.5f, 0.45f});
    engine.attach_observer(a);
    engine.attach_observer(b);
    const size_t N = nodes.points.size() / 2;
    point_source src;
    double best = 1e30;
    for (size_t i = 0; i < N; ++i) {
        double dx = nodes.points[2 * i] - 0.5, dy = nodes.points[2 * i + 1] - 0.5;
        if (dx * dx + dy * dy < best) {
            best = dx * dx + dy * dy;
            src.node = i;
        }
    }
    src.period = 17 * dt;
    engine.register_density_source(src);
    engine.set_initial_density(std::vector<float>(N, 0.f));
    for (int s = 0; s < steps; ++s) engine.step_forward();
    std::printf("%zu\n", src.node);
    for (int s = 0; s < steps; ++s)
        std::printf("%.9e %.9e %.9e %.9e\n", a.time_values()[s], src.used[s], a.density_values()[s] - 1.0f,
                    b.density_values()[s] - 1.0f);
    return 0;
}
