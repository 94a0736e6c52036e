// Header-only C++ facade over libnaga_b200.so with the shape of NAGA's C++
// API (NAGAGroup/NAGA), so a program written against NAGA's engine keeps its
// structure:
//
//   NAGA                                         here
//   fluids/nonlocal_lattice_boltzmann/           naga::fluids::nonlocal_lbm::
//     simulation_engine.cuh:40-121                 simulation_engine<Lattice>
//     simulation_nodes.cuh:41-66                   simulation_nodes<T>
//     simulation_variables.cuh:40-60               problem_parameters<T>
//     node_provider.cuh:41-50                      node_provider<Lattice>
//     simulation_observer.cuh:41-55                simulation_observer<Lattice>
//     simulation_observers/density_observer.cuh    density_observer<Lattice>
//     d2q9_lattice.cuh / d3q27_lattice.cuh         d2q9_lattice<T>, d3q27_lattice<T>
//   segmentation/nearest_neighbors.cuh:444-477   naga::segmentation::batched_nearest_neighbors
//   linalg/batched_matrix_inverse.cuh:389-397    naga::linalg::batched_matrix_inverse
//
// Differences a caller sees: arrays are std::vector on the host (NAGA used
// its unified-memory sclx::array); the engine owns device state; errors
// from the C ABI are rethrown as std::invalid_argument (bad arguments) or
// std::runtime_error (everything else), the exception types NAGA throws.
#pragma once

#include <cuda_runtime.h>
#include <naga_b200.h>

#include <algorithm>
#include <limits>
#include <array>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

namespace naga {

namespace detail {
inline void check(int rc, const char* where) {
    if (rc == NAGA_OK) return;
    std::string msg = std::string(where) + ": " + naga_last_error();
    if (rc == NAGA_EINVAL) throw std::invalid_argument(msg);
    throw std::runtime_error(msg);
}
}  // namespace detail

template <class T, unsigned D>
using point_t = std::array<T, D>;

namespace fluids::nonlocal_lbm {

template <class T>
struct d2q9_lattice {
    static constexpr unsigned size = 9;
    static constexpr unsigned dimensions = 2;
    using value_type = T;
};

template <class T>
struct d3q27_lattice {
    static constexpr unsigned size = 27;
    static constexpr unsigned dimensions = 3;
    using value_type = T;
};

template <class Lattice>
struct lattice_traits {
    static constexpr unsigned size = Lattice::size;
    static constexpr unsigned dimensions = Lattice::dimensions;
    using value_type = typename Lattice::value_type;
    static constexpr value_type lattice_speed_of_sound =
        static_cast<value_type>(0.57735026918962576450914878050196);
};

// Node order: bulk, absorbing layer, boundary, ghost. points holds
// dimensions x N values with the coordinates of a node adjacent (NAGA's
// {D, N} column-major array).
template <class T>
struct simulation_nodes {
    std::vector<T> points;
    std::vector<T> boundary_normals;  // inward, dimensions x num_boundary_points
    std::vector<T> layer_absorption;  // num_layer_points
    size_t num_bulk_points{};
    size_t num_layer_points{};
    size_t num_ghost_nodes{0};
    size_t num_boundary_points{};
    T nodal_spacing{};
};

// simulation_engine::solution() (simulation_variables.cuh:52-62) as host
// copies: f per direction (library population order, naga_lattice), the
// density rho rho0 and velocity u c / c_s ({dimensions, N}, a node's
// components adjacent)
template <class Lattice>
struct state_variables {
    using value_type = typename Lattice::value_type;
    std::array<std::vector<value_type>, Lattice::size> lattice_distributions{};
    struct {
        std::vector<value_type> fluid_velocity;
        std::vector<value_type> fluid_density;
    } macroscopic_values;
};

template <class T>
struct problem_parameters {
    T fluid_viscosity;
    T time_step;
    T speed_of_sound;
    T nominal_density;
    T lattice_viscosity;
    T lattice_time_step;
    T lattice_characteristic_frequency;
};

template <class Lattice>
class node_provider {
  public:
    using value_type = typename lattice_traits<Lattice>::value_type;
    virtual ~node_provider() = default;
    virtual simulation_nodes<value_type> get() const = 0;
};

// Jittered uniform grid in the unit square / cube (naga_grid_generate): the
// synthetic counterpart of NAGA's uniform_grid_provider.
template <class Lattice>
class jittered_grid_provider : public node_provider<Lattice> {
  public:
    using value_type = typename lattice_traits<Lattice>::value_type;
    jittered_grid_provider(int64_t n_side, int n_layers, double sigma_peak, uint64_t seed, double jitter = 0.25)
        : spec_{static_cast<int>(Lattice::dimensions), n_layers, n_side, jitter, sigma_peak, seed} {}

    simulation_nodes<value_type> get() const override {
        int64_t nb, nl, nbd;
        detail::check(naga_grid_counts(&spec_, &nb, &nl, &nbd), "jittered_grid_provider");
        const int D = spec_.dim;
        std::vector<float> pts((nb + nl + nbd) * D), nrm(nbd * D), sig(nl);
        double h = 0;
        detail::check(naga_grid_generate(&spec_, pts.data(), nrm.data(), sig.data(), &h), "jittered_grid_provider");
        simulation_nodes<value_type> out;
        out.points.assign(pts.begin(), pts.end());
        out.boundary_normals.assign(nrm.begin(), nrm.end());
        out.layer_absorption.assign(sig.begin(), sig.end());
        out.num_bulk_points = (size_t)nb;
        out.num_layer_points = (size_t)nl;
        out.num_boundary_points = (size_t)nbd;
        out.nodal_spacing = (value_type)h;
        return out;
    }

  private:
    naga_grid_spec spec_;
};

// NAGA's uniform_grid_provider (node_providers/uniform_grid_provider.cuh:
// 53-161) with its constructor: an axis-aligned box [min, max] at
// grid_spacing, absorbing layer of the given thickness and peak rate
// (naga_box_grid_generate). Nodes within each class come in Morton order.
template <class Lattice>
class uniform_grid_provider : public node_provider<Lattice> {
  public:
    using value_type = typename lattice_traits<Lattice>::value_type;
    static constexpr unsigned dimensions = Lattice::dimensions;
    uniform_grid_provider(const point_t<value_type, dimensions>& min, const point_t<value_type, dimensions>& max,
                          const value_type& grid_spacing, const value_type& absorption_layer_thickness = 0,
                          const value_type& peak_absorption_rate = 0) {
        spec_.dim = (int)dimensions;
        spec_.morton = 1;
        for (unsigned d = 0; d < 3; ++d) {
            spec_.min[d] = d < dimensions ? (double)min[d] : 0.0;
            spec_.max[d] = d < dimensions ? (double)max[d] : 1.0;
        }
        spec_.spacing = grid_spacing;
        spec_.layer_thickness = absorption_layer_thickness;
        spec_.peak_absorption = peak_absorption_rate;
    }

    simulation_nodes<value_type> get() const override {
        int64_t nb, nl, nbd;
        detail::check(naga_box_grid_counts(&spec_, &nb, &nl, &nbd), "uniform_grid_provider");
        const int D = spec_.dim;
        std::vector<float> pts((nb + nl + nbd) * D), nrm(nbd * D), sig(nl);
        double h = 0;
        detail::check(naga_box_grid_generate(&spec_, pts.data(), nrm.data(), sig.data(), &h),
                      "uniform_grid_provider");
        simulation_nodes<value_type> out;
        out.points.assign(pts.begin(), pts.end());
        out.boundary_normals.assign(nrm.begin(), nrm.end());
        out.layer_absorption.assign(sig.begin(), sig.end());
        out.num_bulk_points = (size_t)nb;
        out.num_layer_points = (size_t)nl;
        out.num_boundary_points = (size_t)nbd;
        out.nodal_spacing = (value_type)h;
        return out;
    }

  private:
    naga_box_grid_spec spec_{};
};

template <class Lattice>
class simulation_observer {
  public:
    using value_type = typename lattice_traits<Lattice>::value_type;
    virtual ~simulation_observer() = default;
    // time of the step start and the probe density there (density observers)
    virtual void update(const value_type& time, const value_type& density) = 0;
    virtual point_t<value_type, Lattice::dimensions> location() const = 0;
};

// Probe of the fluid density at a fixed point, sampled at the start of each
// step by RPIM interpolation (density_observer.cuh:47-145).
template <class Lattice>
class density_observer : public simulation_observer<Lattice> {
  public:
    using value_type = typename lattice_traits<Lattice>::value_type;
    explicit density_observer(const point_t<value_type, Lattice::dimensions>& loc, value_type time_multiplier = 1)
        : loc_(loc), time_multiplier_(time_multiplier) {}
    void update(const value_type& t, const value_type& density) override {
        time_values_.push_back(t * time_multiplier_);
        density_values_.push_back(density);
    }
    point_t<value_type, Lattice::dimensions> location() const override { return loc_; }
    const std::vector<value_type>& density_values() const { return density_values_; }
    const std::vector<value_type>& time_values() const { return time_values_; }

    // density_observer::save_state / load_state (density_observer.cuh:
    // 115-133) for a cereal-style archive (ar(values...)); the RPIM tables
    // of the probe live in the engine's scene (its save_state)
    template <class Archive>
    void save_state(Archive& ar) const {
        ar(loc_, density_values_, time_values_, time_multiplier_);
    }
    template <class Archive>
    void load_state(Archive& ar) {
        ar(loc_, density_values_, time_values_, time_multiplier_);
    }

  private:
    point_t<value_type, Lattice::dimensions> loc_;
    value_type time_multiplier_;
    std::vector<value_type> density_values_, time_values_;
};

// A density source (density_source.cuh:41-82): before each step the engine
// fills `source_terms` [N] with the sentinel std::numeric_limits<float>::
// max() and calls every registered source, which writes the dimensional
// density terms of its nodes for that step's time. NAGA's callback also
// receives the device state (state_variables); here the state stays on the
// GPU, so sources depend on the domain, the parameters and time.
template <class Lattice>
class density_source {
  public:
    using value_type = typename lattice_traits<Lattice>::value_type;
    virtual void add_density_source(const simulation_nodes<value_type>& domain,
                                    const problem_parameters<value_type>& params, const value_type& time,
                                    std::vector<value_type>& source_terms) = 0;
    virtual ~density_source() = default;
};

// Options of the B200 engine that NAGA fixes at compile time.
struct engine_options {
    int k = 0;                 // stencil size; 0 = 32 (NAGA's num_interp_support)
    int k_boundary = 0;        // 0 = k
    int k_probe = 0;           // 0 = k
    int shape = 0;             // 0 = multiquadric (NAGA's default), 1 = r^3
    int pml_indexing = 0;      // 0 = as NAGA, 1 = corrected
    int weight_precision = 0;  // 0 = FP64 solves, 1 = FP32 + FP64 refinement
};

template <class Lattice>
class simulation_engine {
  public:
    using value_type = typename lattice_traits<Lattice>::value_type;
    static constexpr unsigned lattice_size = Lattice::size;
    static constexpr unsigned dimensions = Lattice::dimensions;
    using simulation_domain_t = simulation_nodes<value_type>;
    using problem_parameters_t = fluids::nonlocal_lbm::problem_parameters<value_type>;

    explicit simulation_engine(engine_options opt = {}) : impl_(std::make_shared<impl>()) { impl_->opt = opt; }

    void set_problem_parameters(value_type fluid_viscosity, value_type nominal_density, value_type time_step,
                                value_type speed_of_sound, value_type characteristic_frequency = 0) {
        auto& p = impl_->params;
        p.fluid_viscosity = fluid_viscosity;
        p.nominal_density = nominal_density;
        p.time_step = time_step;
        p.speed_of_sound = speed_of_sound;
        const value_type ratio = lattice_traits<Lattice>::lattice_speed_of_sound / speed_of_sound;
        p.lattice_time_step = time_step / ratio;
        p.lattice_viscosity = fluid_viscosity / ratio;
        const value_type fc = characteristic_frequency == 0 ? value_type(1) / time_step : characteristic_frequency;
        p.lattice_characteristic_frequency = fc * ratio;
        // a live scene takes the new parameters at its next step (its state
        // and stencils stay); otherwise they apply when the scene is built
        if (impl_->scene)
            detail::check(naga_scene_set_params(impl_->scene, fluid_viscosity, nominal_density, time_step,
                                                speed_of_sound),
                          "set_problem_parameters");
    }

    void init_domain(const simulation_domain_t& domain) {
        const size_t N = domain.num_bulk_points + domain.num_layer_points + domain.num_boundary_points +
                         domain.num_ghost_nodes;
        if (domain.points.size() != N * dimensions)
            throw std::invalid_argument(
                "The number of points in the simulation domain does not match the sum of the number of bulk, "
                "layer, and boundary points.");
        if (domain.boundary_normals.size() != domain.num_boundary_points * dimensions)
            throw std::invalid_argument("The number of boundary normals does not match the number of boundary points.");
        if (domain.layer_absorption.size() != domain.num_layer_points)
            throw std::invalid_argument(
                "The number of layer absorption coefficients does not match the number of layer points.");
        impl_->domain = domain;
        impl_->drho.assign(N, 0.f);
        impl_->invalidate();
    }

    void init_domain(const node_provider<Lattice>& nodes) { init_domain(nodes.get()); }

    // initial density perturbation (units of the nominal density), u = 0
    void set_initial_density(const std::vector<value_type>& drho) {
        impl_->drho.assign(drho.begin(), drho.end());
        if (impl_->scene) detail::check(naga_scene_set_density(impl_->scene, impl_->drho.data()), "set_initial_density");
        impl_->time = 0;
    }

    void step_forward() {
        impl_->ensure();
        const int64_t t = naga_scene_step_count(impl_->scene);
        if (!impl_->sources.empty()) impl_->upload_sources(t);
        detail::check(naga_scene_step(impl_->scene, 1), "step_forward");
        if (!impl_->observers.empty()) {
            std::vector<float> pr((size_t)impl_->n_probes);
            detail::check(naga_scene_read_probes(impl_->scene, t, 1, pr.data()), "step_forward");
            for (size_t o = 0; o < impl_->observers.size(); ++o)
                impl_->observers[o]->update(impl_->time,
                                            impl_->params.nominal_density + (value_type)pr[impl_->probe_of[o]]);
        }
        impl_->time += impl_->params.time_step;
    }

    void reset() {
        impl_->ensure();
        detail::check(naga_scene_set_density(impl_->scene, impl_->drho.data()), "reset");
        impl_->time = 0;
    }

    value_type time() const { return impl_->time; }
    value_type speed_of_sound() const { return impl_->params.speed_of_sound; }
    const simulation_domain_t& domain() const { return impl_->domain; }
    const problem_parameters_t& problem_parameters() const { return impl_->params; }

    // simulation_engine::register_density_source (simulation_engine.cuh:80-82)
    void register_density_source(density_source<Lattice>& src) {
        auto& v = impl_->sources;
        if (std::find(v.begin(), v.end(), &src) != v.end())
            throw std::runtime_error("Density source already registered with an engine.");
        v.push_back(&src);
    }
    void unregister_density_source(density_source<Lattice>& src) {
        auto& v = impl_->sources;
        v.erase(std::remove(v.begin(), v.end(), &src), v.end());
        if (v.empty() && impl_->scene)
            detail::check(naga_scene_set_density_source(impl_->scene, nullptr, 0, nullptr, 0, 0),
                          "unregister_density_source");
    }

    void attach_observer(simulation_observer<Lattice>& o) {
        if (impl_->scene) {
            // a live scene gains a probe; it samples from the next step on
            const auto l = o.location();
            std::vector<float> x(l.begin(), l.end());
            int index = 0;
            detail::check(naga_scene_add_probe(impl_->scene, x.data(), &index), "attach_observer");
            impl_->probe_of.push_back(index);
            impl_->n_probes = index + 1;
        } else {
            impl_->probe_of.push_back((int)impl_->observers.size());
        }
        impl_->observers.push_back(&o);
    }
    // the observer stops receiving updates; a live scene keeps its probe
    // (and its state), as NAGA's detach only drops the observer
    void detach_observer(simulation_observer<Lattice>& o) {
        auto& v = impl_->observers;
        for (size_t k = 0; k < v.size();) {
            if (v[k] == &o) {
                v.erase(v.begin() + (long)k);
                impl_->probe_of.erase(impl_->probe_of.begin() + (long)k);
            } else {
                ++k;
            }
        }
        if (!impl_->scene)
            for (size_t k = 0; k < v.size(); ++k) impl_->probe_of[k] = (int)k;
    }

    // density perturbation rho - rho0 of every node and the centred
    // populations f - w (node-major), copied to the host
    std::vector<float> density() {
        impl_->ensure();
        int64_t N;
        int Q;
        naga_scene_size(impl_->scene, &N, &Q);
        std::vector<float> r(N);
        detail::check(naga_scene_read_state(impl_->scene, nullptr, r.data()), "density");
        return r;
    }
    std::vector<float> populations() {
        impl_->ensure();
        int64_t N;
        int Q;
        naga_scene_size(impl_->scene, &N, &Q);
        std::vector<float> g(N * Q);
        detail::check(naga_scene_read_state(impl_->scene, g.data(), nullptr), "populations");
        return g;
    }

    // simulation_engine::save_state / load_state (simulation_engine.cuh:
    // 108-116) for a cereal-style archive (ar(values...)): the scene's
    // snapshot (populations, PML history, macros, probe ring, step count;
    // naga_scene_save) and the engine time. Load into an engine initialised
    // with the same domain, parameters and observers.
    template <class Archive>
    void save_state(Archive& ar) const {
        impl_->ensure();
        std::vector<unsigned char> bytes((size_t)naga_scene_snapshot_bytes(impl_->scene));
        detail::check(naga_scene_save(impl_->scene, bytes.data(), (int64_t)bytes.size()), "save_state");
        ar(bytes, impl_->time);
    }
    template <class Archive>
    void load_state(Archive& ar) {
        impl_->ensure();
        std::vector<unsigned char> bytes;
        ar(bytes, impl_->time);
        detail::check(naga_scene_load(impl_->scene, bytes.data(), (int64_t)bytes.size()), "load_state");
    }

    // simulation_engine::solution() (simulation_engine.cuh:100): the
    // populations f = w + g per direction and the dimensional macroscopic
    // values of the last step, copied to the host
    state_variables<Lattice> solution() {
        impl_->ensure();
        int64_t N;
        int Q;
        naga_scene_size(impl_->scene, &N, &Q);
        std::vector<float> g((size_t)N * Q);
        detail::check(naga_scene_read_state(impl_->scene, g.data(), nullptr), "solution");
        std::vector<float> w(Q);
        detail::check(naga_lattice((int)dimensions, nullptr, w.data(), nullptr), "solution");
        state_variables<Lattice> out;
        for (int a = 0; a < Q; ++a) {
            auto& f = out.lattice_distributions[a];
            f.resize((size_t)N);
            for (int64_t i = 0; i < N; ++i) f[i] = w[a] + g[(size_t)i * Q + a];
        }
        out.macroscopic_values.fluid_density.resize((size_t)N);
        out.macroscopic_values.fluid_velocity.resize((size_t)N * dimensions);
        detail::check(naga_scene_read_macros(impl_->scene, out.macroscopic_values.fluid_density.data(),
                                             out.macroscopic_values.fluid_velocity.data()),
                      "solution");
        return out;
    }

    naga_scene* handle() {
        impl_->ensure();
        return impl_->scene;
    }

  private:
    // copies share state, as NAGA's pimpl engine does (simulation_engine.cuh:119-120)
    struct impl {
        engine_options opt;
        problem_parameters_t params{};
        simulation_domain_t domain{};
        std::vector<float> drho;
        std::vector<simulation_observer<Lattice>*> observers;
        std::vector<int> probe_of;  // the scene probe each observer reads
        int n_probes = 0;           // probes of the live scene
        std::vector<density_source<Lattice>*> sources;
        std::vector<value_type> terms;  // per-step source terms [N]
        std::vector<int64_t> src_nodes;
        std::vector<float> src_row;
        naga_scene* scene = nullptr;
        value_type time = 0;

        // the registered sources' terms for step t (time `time`) as one row
        void upload_sources(int64_t t) {
            const size_t N = domain.num_bulk_points + domain.num_layer_points + domain.num_boundary_points +
                             domain.num_ghost_nodes;
            const value_type none = std::numeric_limits<float>::max();
            terms.assign(N, none);
            for (auto* src : sources) src->add_density_source(domain, params, time, terms);
            src_nodes.clear();
            src_row.clear();
            for (size_t i = 0; i < N; ++i)
                if (terms[i] != none) {
                    src_nodes.push_back((int64_t)i);
                    src_row.push_back((float)terms[i]);
                }
            detail::check(naga_scene_set_density_source(scene, src_nodes.data(), (int64_t)src_nodes.size(),
                                                        src_row.data(), t, src_nodes.empty() ? 0 : 1),
                          "step_forward: density sources");
        }

        void invalidate() {
            if (scene) naga_scene_destroy(scene);
            scene = nullptr;
            n_probes = 0;
        }
        void ensure() {
            if (scene) return;
            const size_t N = domain.num_bulk_points + domain.num_layer_points + domain.num_boundary_points +
                             domain.num_ghost_nodes;
            if (N == 0) throw std::invalid_argument("simulation_engine: init_domain has not been called");
            std::vector<float> pts(domain.points.begin(), domain.points.end());
            std::vector<float> nrm(domain.boundary_normals.begin(), domain.boundary_normals.end());
            std::vector<float> sig(domain.layer_absorption.begin(), domain.layer_absorption.end());
            std::vector<float> prb;
            for (auto* o : observers) {
                auto l = o->location();
                prb.insert(prb.end(), l.begin(), l.end());
            }
            naga_scene_desc d{};
            d.dim = (int)dimensions;
            d.k = opt.k ? opt.k : 32;
            d.k_boundary = opt.k_boundary ? opt.k_boundary : d.k;
            d.k_probe = opt.k_probe ? opt.k_probe : d.k;
            d.shape = opt.shape;
            d.pml_indexing = opt.pml_indexing;
            d.weight_precision = opt.weight_precision;
            d.n_probes = (int)observers.size();
            d.n_bulk = (int64_t)domain.num_bulk_points;
            d.n_layer = (int64_t)domain.num_layer_points;
            d.n_boundary = (int64_t)domain.num_boundary_points;
            d.n_ghost = (int64_t)domain.num_ghost_nodes;
            d.nodal_spacing = domain.nodal_spacing;
            d.viscosity = params.fluid_viscosity;
            d.rho0 = params.nominal_density;
            d.time_step = params.time_step;
            d.speed_of_sound = params.speed_of_sound;
            d.points = pts.data();
            d.normals = nrm.data();
            d.sigma = sig.data();
            d.probes = prb.empty() ? nullptr : prb.data();
            d.probe_capacity = 1024;
            detail::check(naga_scene_create(&d, &scene), "simulation_engine::init_domain");
            n_probes = (int)observers.size();
            probe_of.resize(observers.size());
            for (size_t o = 0; o < observers.size(); ++o) probe_of[o] = (int)o;
            detail::check(naga_scene_set_density(scene, drho.data()), "simulation_engine::reset");
            time = 0;
        }
        ~impl() { invalidate(); }
    };
    std::shared_ptr<impl> impl_;
};

}  // namespace fluids::nonlocal_lbm

namespace detail {
// device copy of a host vector, freed on scope exit
template <class T>
struct device_vec {
    T* p = nullptr;
    explicit device_vec(size_t n) {
        if (cudaMalloc((void**)&p, sizeof(T) * (n ? n : 1)) != cudaSuccess)
            throw std::runtime_error("naga: cudaMalloc failed");
    }
    device_vec(const std::vector<T>& v) : device_vec(v.size()) {
        if (!v.empty() && cudaMemcpy(p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice) != cudaSuccess)
            throw std::runtime_error("naga: cudaMemcpy failed");
    }
    std::vector<T> host(size_t n, cudaStream_t st) const {
        std::vector<T> v(n);
        if (cudaStreamSynchronize(st) != cudaSuccess ||
            (n && cudaMemcpy(v.data(), p, sizeof(T) * n, cudaMemcpyDeviceToHost) != cudaSuccess))
            throw std::runtime_error("naga: cudaMemcpy failed");
        return v;
    }
    ~device_vec() { cudaFree(p); }
    device_vec(const device_vec&) = delete;
    device_vec& operator=(const device_vec&) = delete;
};
}  // namespace detail

namespace segmentation {
// Exact k nearest neighbours of `queries` among `points` (host arrays,
// D x count with a point's coordinates adjacent). Returns {dist^2, indices},
// k x count with a query's k entries adjacent, ascending in (dist^2, index).
template <unsigned D>
std::tuple<std::vector<float>, std::vector<uint32_t>> batched_nearest_neighbors(unsigned k,
                                                                               const std::vector<float>& queries,
                                                                               const std::vector<float>& points,
                                                                               cudaStream_t stream = nullptr) {
    const int64_t nq = (int64_t)(queries.size() / D), n = (int64_t)(points.size() / D);
    detail::device_vec<float> dq(queries), dp(points), dd(nq * k);
    detail::device_vec<uint32_t> di(nq * k);
    detail::check(naga_knn(dp.p, n, dq.p, nq, (int)D, (int)k, di.p, dd.p, stream), "batched_nearest_neighbors");
    return {dd.host(nq * k, stream), di.host(nq * k, stream)};
}
}  // namespace segmentation

namespace linalg {
// Inverse of `batch` n x n matrices stored back to back, column-major
// (NAGA's {n, n, batch} array); FP64, or FP32 LU + FP64 refinement.
inline std::vector<double> batched_matrix_inverse(const std::vector<double>& A, int n, bool refined = false,
                                                  cudaStream_t stream = nullptr) {
    const int64_t batch = (int64_t)(A.size() / ((size_t)n * n));
    detail::device_vec<double> dA(A), dX(A.size());
    detail::device_vec<int> info(batch);
    if (refined)
        detail::check(naga_batched_inverse_f32r(dA.p, dX.p, n, batch, 30, 1e-14, info.p, stream), "batched_matrix_inverse");
    else
        detail::check(naga_batched_inverse_f64(dA.p, dX.p, n, batch, info.p, stream), "batched_matrix_inverse");
    auto inf = info.host(batch, stream);
    for (int v : inf)
        if (v != 0) throw std::runtime_error("batched_matrix_inverse: singular or unconverged matrix in the batch");
    return dX.host(A.size(), stream);
}
}  // namespace linalg

}  // namespace naga
