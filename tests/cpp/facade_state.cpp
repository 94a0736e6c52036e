// save_state / load_state through the facade with a minimal cereal-style
// archive: an engine restored from a snapshot taken after 8 steps continues
// bit for bit like the engine that took it, observers included. Prints "ok"
// or exits 1.
#include <naga/naga.hpp>

#include <cmath>
#include <cstdio>
#include <cstring>

using namespace naga::fluids::nonlocal_lbm;
using lattice_t = d3q27_lattice<float>;

// cereal-style archives: the output one appends every argument's bytes in
// order (vectors with their length), the input one reads them back
struct OutArchive {
    std::vector<unsigned char> data;
    template <class T>
    void one(const T& v) {
        const auto* p = reinterpret_cast<const unsigned char*>(&v);
        data.insert(data.end(), p, p + sizeof(T));
    }
    template <class T>
    void one(const std::vector<T>& v) {
        const uint64_t n = v.size();
        one(n);
        const auto* p = reinterpret_cast<const unsigned char*>(v.data());
        data.insert(data.end(), p, p + n * sizeof(T));
    }
    template <class... A>
    void operator()(const A&... a) {
        (one(a), ...);
    }
};
struct InArchive {
    const std::vector<unsigned char>& data;
    size_t at = 0;
    template <class T>
    void one(T& v) {
        std::memcpy(&v, data.data() + at, sizeof(T));
        at += sizeof(T);
    }
    template <class T>
    void one(std::vector<T>& v) {
        uint64_t n = 0;
        one(n);
        v.resize(n);
        std::memcpy(v.data(), data.data() + at, n * sizeof(T));
        at += n * sizeof(T);
    }
    template <class... A>
    void operator()(A&... a) {
        (one(a), ...);
    }
};

int main() {
    jittered_grid_provider<lattice_t> provider(14, 3, 0.1, 5);
    auto nodes = provider.get();
    const size_t N = nodes.points.size() / 3;
    std::vector<float> drho(N);
    for (size_t i = 0; i < N; ++i) {
        double dx = nodes.points[3 * i] - 0.5, dy = nodes.points[3 * i + 1] - 0.5, dz = nodes.points[3 * i + 2] - 0.5;
        drho[i] = (float)(1e-3 * std::exp(-(dx * dx + dy * dy + dz * dz) / (2 * 0.1 * 0.1)));
    }
    engine_options opt;
    opt.k = 32;
    opt.shape = 0;
    simulation_engine<lattice_t> a(opt), b(opt);
    density_observer<lattice_t> pa({0.4f, 0.5f, 0.5f}), pb({0.4f, 0.5f, 0.5f});
    for (auto* e : {&a, &b}) {
        e->set_problem_parameters(1e-5f, 1.0f, 0.5f * nodes.nodal_spacing, 1.0f);
        e->init_domain(nodes);
    }
    a.attach_observer(pa);
    b.attach_observer(pb);
    a.set_initial_density(drho);
    b.set_initial_density(std::vector<float>(N, 0.f));
    for (int s = 0; s < 8; ++s) a.step_forward();
    OutArchive out;
    a.save_state(out);
    pa.save_state(out);
    for (int s = 0; s < 8; ++s) a.step_forward();
    b.step_forward();  // b is live, in another state
    InArchive in{out.data};
    b.load_state(in);
    pb.load_state(in);
    for (int s = 0; s < 8; ++s) b.step_forward();
    if (pa.density_values() != pb.density_values()) return std::puts("observer traces differ"), 1;
    if (a.populations() != b.populations()) return std::puts("states differ"), 1;
    if (a.time() != b.time()) return std::puts("times differ"), 1;
    std::puts("ok");
    return 0;
}
