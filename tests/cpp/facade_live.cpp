// Observers and parameters changed on a running facade engine: an observer
// attached after some steps samples exactly like the same observer attached
// from the start (from the step it joined on), and the others are
// unaffected; set_problem_parameters on the running engine equals an engine
// that had those parameters when it was reset. Prints "ok" or exits 1.
#include <naga/naga.hpp>

#include <cmath>
#include <cstdio>
#include <cstdlib>

using namespace naga::fluids::nonlocal_lbm;
using lattice_t = d2q9_lattice<float>;

static std::vector<float> pulse(const simulation_nodes<float>& nodes) {
    const size_t N = nodes.points.size() / 2;
    std::vector<float> drho(N);
    for (size_t i = 0; i < N; ++i) {
        double dx = nodes.points[2 * i] - 0.5, dy = nodes.points[2 * i + 1] - 0.5;
        drho[i] = (float)(1e-3 * std::exp(-(dx * dx + dy * dy) / (2 * 0.08 * 0.08)));
    }
    return drho;
}

int main() {
    jittered_grid_provider<lattice_t> provider(36, 4, 0.1, 3);
    auto nodes = provider.get();
    const auto drho = pulse(nodes);
    engine_options opt;
    opt.k = 16;
    opt.shape = 1;
    const float dt = 0.5f * nodes.nodal_spacing;

    // observers
    simulation_engine<lattice_t> e1(opt), e2(opt);
    density_observer<lattice_t> a1({0.3f, 0.5f}), b1({0.6f, 0.55f}), a2({0.3f, 0.5f}), b2({0.6f, 0.55f});
    for (auto* e : {&e1, &e2}) {
        e->set_problem_parameters(1e-5f, 1.0f, dt, 1.0f);
        e->init_domain(nodes);
    }
    e1.attach_observer(a1);
    e1.attach_observer(b1);
    e2.attach_observer(a2);
    e1.set_initial_density(drho);
    e2.set_initial_density(drho);
    for (int s = 0; s < 6; ++s) {
        e1.step_forward();
        e2.step_forward();
    }
    e2.attach_observer(b2);
    for (int s = 0; s < 6; ++s) {
        e1.step_forward();
        e2.step_forward();
    }
    if (a1.density_values() != a2.density_values()) return std::puts("observer a differs"), 1;
    const auto& v1 = b1.density_values();
    const auto& v2 = b2.density_values();
    if (v2.size() != 6 || !std::equal(v2.begin(), v2.end(), v1.end() - 6)) return std::puts("late observer differs"), 1;

    // parameters
    simulation_engine<lattice_t> e3(opt), e4(opt);
    density_observer<lattice_t> c3({0.4f, 0.5f}), c4({0.4f, 0.5f});
    e3.set_problem_parameters(3e-5f, 1.1f, 0.8f * dt, 1.0f);
    e3.init_domain(nodes);
    e3.attach_observer(c3);
    e3.set_initial_density(drho);
    e4.set_problem_parameters(1e-5f, 1.0f, dt, 1.0f);
    e4.init_domain(nodes);
    e4.attach_observer(c4);
    e4.set_initial_density(drho);
    e4.step_forward();  // the engine is live
    e4.set_problem_parameters(3e-5f, 1.1f, 0.8f * dt, 1.0f);
    e4.reset();
    density_observer<lattice_t> d3({0.5f, 0.45f}), d4({0.5f, 0.45f});
    e3.attach_observer(d3);
    e4.attach_observer(d4);
    for (int s = 0; s < 8; ++s) {
        e3.step_forward();
        e4.step_forward();
    }
    if (d3.density_values() != d4.density_values()) return std::puts("parameters differ"), 1;

    // detach on a running engine: the other observers and the state carry on
    e1.detach_observer(a1);
    e2.detach_observer(a2);
    for (int s = 0; s < 3; ++s) {
        e1.step_forward();
        e2.step_forward();
    }
    if (a1.density_values().size() != 12 || a2.density_values().size() != 12)
        return std::puts("detached observer still updated"), 1;
    if (b1.density_values().size() != 15 || b2.density_values().size() != 9 ||
        !std::equal(b2.density_values().begin(), b2.density_values().end(), b1.density_values().end() - 9))
        return std::puts("observers after detach differ"), 1;
    if (e1.populations() != e2.populations()) return std::puts("state after detach differs"), 1;

    // solution(): populations per direction and the dimensional macros
    const auto sol = e4.solution();
    const size_t N = nodes.points.size() / 2;
    if (sol.lattice_distributions[0].size() != N || sol.macroscopic_values.fluid_density.size() != N ||
        sol.macroscopic_values.fluid_velocity.size() != 2 * N)
        return std::puts("solution sizes"), 1;
    double mass = 0;
    for (const auto& f : sol.lattice_distributions) mass += f[N / 2];
    if (std::fabs(mass - 1.0) > 1e-2) return std::puts("solution populations"), 1;
    if (std::fabs(sol.macroscopic_values.fluid_density[N / 2] / 1.1 - 1.0) > 1e-2)
        return std::puts("solution density"), 1;
    std::puts("ok");
    return 0;
}
