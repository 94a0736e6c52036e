// A NAGA-style driver program written against the C++ facade: builds a
// jittered D2Q9 domain, attaches two density observers, runs a Gaussian
// pulse and prints the probe traces (one line per step: t rho_a rho_b).
#include <naga/naga.hpp>

#include <cmath>
#include <cstdio>
#include <cstdlib>

using namespace naga::fluids::nonlocal_lbm;
using lattice_t = d2q9_lattice<float>;

int main(int argc, char** argv) {
    const int steps = argc > 1 ? std::atoi(argv[1]) : 20;
    jittered_grid_provider<lattice_t> provider(40, 4, 0.1, 0);
    auto nodes = provider.get();
    engine_options opt;
    opt.k = 16;
    opt.shape = 1;
    simulation_engine<lattice_t> engine(opt);
    engine.set_problem_parameters(1e-5f, 1.0f, 0.5f * nodes.nodal_spacing, 1.0f);
    engine.init_domain(nodes);
    density_observer<lattice_t> a({0.3f, 0.5f}), b({0.7f, 0.5f});
    engine.attach_observer(a);
    engine.attach_observer(b);
    const size_t N = nodes.points.size() / 2;
    std::vector<float> drho(N);
    for (size_t i = 0; i < N; ++i) {
        double dx = nodes.points[2 * i] - 0.5, dy = nodes.points[2 * i + 1] - 0.5;
        drho[i] = (float)(1e-3 * std::exp(-(dx * dx + dy * dy) / (2 * 0.08 * 0.08)));
    }
    engine.set_initial_density(drho);
    for (int s = 0; s < steps; ++s) engine.step_forward();
    for (int s = 0; s < steps; ++s)
        std::printf("%.9e %.9e %.9e\n", a.time_values()[s], a.density_values()[s] - 1.0f,
                    b.density_values()[s] - 1.0f);
    return 0;
}
