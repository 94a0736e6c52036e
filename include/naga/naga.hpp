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
//   segmentation/nd_cubic_segmentation.cuh       naga::segmentation::nd_cubic_segmentation<T, D>
//   segmentation/nearest_neighbors.cuh:444-477   naga::segmentation::batched_nearest_neighbors
//   interpolation/radial_point_method.cuh        naga::interpolation::radial_point_method<T>
//   nonlocal_calculus/divergence.cuh, operators.cuh
//                                                naga::nonlocal_calculus::divergence_operator<T, D>,
//                                                operator_builder<T, D>
//   linalg/batched_matrix_inverse.cuh:389-397    naga::linalg::batched_matrix_inverse
//
// Differences a caller sees: the engine's arrays are std::vector on the host
// and the primitives' are naga::device_array (NAGA used its unified-memory
// sclx::array for both); the engine owns device state; errors
// from the C ABI are rethrown as std::invalid_argument (bad arguments) or
// std::runtime_error (everything else), the exception types NAGA throws.
#pragma once

#include <cuda_runtime.h>
#include <naga_b200.h>

#include <algorithm>
#include <cmath>
#include <future>
#include <limits>
#include <array>
#include <type_traits>
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

// ------------------------------------------------------------ device arrays
// A typed device buffer in the role of NAGA's sclx::array: a reference-
// counted handle (copies share the buffer), either owning memory it
// allocated (freed with its last copy) or viewing memory the caller owns
// (never freed here), so the primitives below run on the caller's device
// pointers without a copy. Sizes are element counts; a NAGA array of shape
// {D, N} is D * N elements with a point's coordinates adjacent.
template <class T>
class device_array {
  public:
    using value_type = T;
    using mutable_type = std::remove_const_t<T>;

    device_array() = default;
    explicit device_array(size_t n) : n_(n) {
        mutable_type* p = nullptr;
        if (cudaMalloc((void**)&p, sizeof(T) * (n ? n : 1)) != cudaSuccess)
            throw std::runtime_error("naga::device_array: cudaMalloc failed");
        p_ = std::shared_ptr<T>(p, [](T* q) { cudaFree((void*)q); });
    }
    // a view of caller memory (device pointer, n elements); not freed here
    static device_array view(T* p, size_t n) {
        device_array a;
        a.p_ = std::shared_ptr<T>(p, [](T*) {});
        a.n_ = n;
        return a;
    }
    static device_array from_host(const std::vector<mutable_type>& v, cudaStream_t st = nullptr) {
        device_array a(v.size());
        if (!v.empty() && (cudaMemcpyAsync((void*)a.data(), v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice,
                                           st) != cudaSuccess ||
                           cudaStreamSynchronize(st) != cudaSuccess))
            throw std::runtime_error("naga::device_array: host to device copy failed");
        return a;
    }
    // copy to the host after the work queued on `st` has finished
    std::vector<mutable_type> to_host(cudaStream_t st = nullptr) const {
        std::vector<mutable_type> v(n_);
        if (cudaStreamSynchronize(st) != cudaSuccess ||
            (n_ && cudaMemcpy(v.data(), (const void*)p_.get(), sizeof(T) * n_, cudaMemcpyDeviceToHost) != cudaSuccess))
            throw std::runtime_error("naga::device_array: device to host copy failed");
        return v;
    }
    // a read-only handle on the same buffer
    template <class U = T, class = std::enable_if_t<!std::is_const_v<U>>>
    operator device_array<const U>() const {
        return device_array<const U>::share(p_, n_);
    }
    static device_array share(std::shared_ptr<T> p, size_t n) {
        device_array a;
        a.p_ = std::move(p);
        a.n_ = n;
        return a;
    }
    T* data() const { return p_.get(); }
    size_t size() const { return n_; }
    size_t elements() const { return n_; }
    bool empty() const { return n_ == 0; }

  private:
    std::shared_ptr<T> p_;
    size_t n_ = 0;
};

// NAGA's default_point_map (point_map.cuh:45-81): the points of a {D, N}
// array, here a device array of D * N values.
template <class T, unsigned D>
struct default_point_map {
    using value_type = T;
    static constexpr unsigned dimensions = D;
    device_array<const T> points;
    default_point_map() = default;
    default_point_map(device_array<const T> p) : points(std::move(p)) {
        if (points.size() % D != 0) throw std::invalid_argument("naga::default_point_map: size is not a multiple of D");
    }
    template <class U = T, class = std::enable_if_t<!std::is_const_v<U>>>
    default_point_map(const device_array<U>& p) : default_point_map(device_array<const T>(p)) {}
    size_t size() const { return points.size() / D; }
};

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

// NAGA's asynchronous calls return std::future<void>; here the work is
// queued on a stream and the future's get() waits for it
inline std::future<void> stream_future(cudaStream_t st) {
    return std::async(std::launch::deferred, [st] {
        if (cudaStreamSynchronize(st) != cudaSuccess) throw std::runtime_error("naga: stream synchronisation failed");
    });
}
}  // namespace detail

namespace segmentation {
// NAGA's nd_cubic_segmentation<T, D>(points, approx_partition_size)
// (segmentation/nd_cubic_segmentation.cuh:227-303): the uniform partition of
// a point cloud into cells of about approx_partition_size points, built on
// the device (naga_segmentation_shape / _build). Bounds, width and shape
// follow NAGA's FP32 arithmetic; every partition lists its points in
// ascending index order. T = float.
template <class T, unsigned D>
class nd_cubic_segmentation {
    static_assert(std::is_same_v<T, float>, "nd_cubic_segmentation: T = float");
    static_assert(D == 2 || D == 3, "nd_cubic_segmentation: D = 2 or 3");

  public:
    nd_cubic_segmentation() = default;
    nd_cubic_segmentation(const device_array<const T>& points, unsigned approx_partition_size,
                          cudaStream_t stream = nullptr)
        : points_(points) {
        if (points.size() % D != 0)
            throw std::invalid_argument(
                "The number of dimensions in the points array does not match the number of dimensions in the "
                "segmentation");
        const int64_t n = (int64_t)(points.size() / D);
        float lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0}, w = 0;
        int64_t shape[3] = {1, 1, 1};
        detail::check(naga_segmentation_shape(points.data(), n, (int)D, (int)approx_partition_size, lo, hi, &w, shape,
                                              stream),
                      "nd_cubic_segmentation");
        size_t cells = 1;
        for (unsigned d = 0; d < D; ++d) {
            lower_[d] = lo[d];
            upper_[d] = hi[d];
            shape_[d] = (size_t)shape[d];
            cells *= shape_[d];
        }
        width_ = w;
        sizes_ = device_array<uint32_t>(cells);
        offsets_ = device_array<uint32_t>(cells);
        indices_ = device_array<uint32_t>((size_t)n);
        detail::check(naga_segmentation_build(points.data(), n, (int)D, lo, hi, w, shape, sizes_.data(),
                                              offsets_.data(), indices_.data(), stream),
                      "nd_cubic_segmentation");
        if (cudaStreamSynchronize(stream) != cudaSuccess)
            throw std::runtime_error("nd_cubic_segmentation: stream synchronisation failed");
    }

    // get_partition_index (nd_cubic_segmentation.cuh:376-392) on the host,
    // in the same FP32 arithmetic (a quotient that rounds up to the shape is
    // clamped to the last cell)
    template <class PointType>
    std::array<size_t, D> get_partition_index(const PointType& p) const {
        std::array<size_t, D> c{};
        for (unsigned d = 0; d < D; ++d) {
            const float x = (float)p[d];
            if (x < lower_[d])
                c[d] = 0;
            else if (x >= upper_[d])
                c[d] = shape_[d] - 1;
            else
                c[d] = std::min((size_t)std::floor((x - lower_[d]) / width_), shape_[d] - 1);
        }
        return c;
    }
    size_t linear_index(const std::array<size_t, D>& c) const {
        size_t lin = 0, mul = 1;
        for (unsigned d = 0; d < D; ++d) {
            lin += c[d] * mul;
            mul *= shape_[d];
        }
        return lin;
    }
    // point indices of one partition (get_partition), copied to the host
    std::vector<uint32_t> get_partition(size_t linear) const {
        if (linear >= partition_count()) throw std::invalid_argument("nd_cubic_segmentation: partition out of range");
        uint32_t size = 0, off = 0;
        if (cudaMemcpy(&size, sizes_.data() + linear, 4, cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemcpy(&off, offsets_.data() + linear, 4, cudaMemcpyDeviceToHost) != cudaSuccess)
            throw std::runtime_error("nd_cubic_segmentation: copy failed");
        std::vector<uint32_t> v(size);
        if (size && cudaMemcpy(v.data(), indices_.data() + off, 4 * size, cudaMemcpyDeviceToHost) != cudaSuccess)
            throw std::runtime_error("nd_cubic_segmentation: copy failed");
        return v;
    }

    const std::array<size_t, D>& shape() const { return shape_; }
    size_t partition_count() const {
        size_t c = 1;
        for (unsigned d = 0; d < D; ++d) c *= shape_[d];
        return c;
    }
    size_t point_count() const { return points_.size() / D; }
    T partition_width() const { return width_; }
    const std::array<T, D>& lower_bounds() const { return lower_; }
    const std::array<T, D>& upper_bounds() const { return upper_; }
    device_array<const T> points() const { return points_; }
    // device arrays: partition sizes and their exclusive prefix sums (one per
    // partition, linear index x + shape[0] (y + shape[1] z)), point indices
    // grouped by partition
    device_array<const uint32_t> partition_sizes() const { return sizes_; }
    device_array<const uint32_t> partition_index_offsets() const { return offsets_; }
    device_array<const uint32_t> indices() const { return indices_; }

  private:
    device_array<const T> points_;
    device_array<uint32_t> sizes_, offsets_, indices_;
    std::array<T, D> lower_{}, upper_{};
    std::array<size_t, D> shape_{};
    T width_{};
};

// batched_nearest_neighbors(k, distances_squared, indices, query_points,
// segmented_ref_points) (nearest_neighbors.cuh:95-108): the exact k nearest
// of every query among the segmentation's points under the (dist^2, index)
// order (naga_knn), into caller arrays of k * n_queries elements (a query's
// k entries adjacent, ascending). Queued on `stream`.
template <class T, unsigned D>
void batched_nearest_neighbors(unsigned k, device_array<T>& distances_squared, device_array<uint32_t>& indices,
                               const default_point_map<T, D>& query_points,
                               const nd_cubic_segmentation<T, D>& segmented_ref_points,
                               cudaStream_t stream = nullptr) {
    const size_t nq = query_points.size();
    if (distances_squared.size() != (size_t)k * nq || indices.size() != (size_t)k * nq)
        throw std::invalid_argument("batched_nearest_neighbors: output arrays must hold k x n_queries values");
    detail::check(naga_knn(segmented_ref_points.points().data(), (int64_t)segmented_ref_points.point_count(),
                           query_points.points.data(), (int64_t)nq, (int)D, (int)k, indices.data(),
                           distances_squared.data(), stream),
                  "batched_nearest_neighbors");
}

// batched_nearest_neighbors(k, query_points, segmented_ref_points)
// (nearest_neighbors.cuh:444-477): returns {distances_squared, indices}.
template <class T, unsigned D>
std::tuple<device_array<T>, device_array<uint32_t>> batched_nearest_neighbors(
    unsigned k, const default_point_map<T, D>& query_points, const nd_cubic_segmentation<T, D>& segmented_ref_points,
    cudaStream_t stream = nullptr) {
    device_array<T> d2((size_t)k * query_points.size());
    device_array<uint32_t> idx((size_t)k * query_points.size());
    batched_nearest_neighbors(k, d2, idx, query_points, segmented_ref_points, stream);
    return {d2, idx};
}

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

namespace interpolation {
// NAGA's multiquadric (interpolation/radial_point_method.cuh:44-66):
// (r^2 + (alpha_c h)^2)^q; the device solves implement q = 1/2, alpha_c =
// 1/10 (NAGA's defaults and the only values its callers use)
template <class T = float>
struct mq_shape_function {
    static constexpr int id = 0;
    T q_ = T(0.5), alpha_c_ = T(0.1);
    mq_shape_function(const T& q = T(0.5), const T& alpha_c = T(0.1)) : q_(q), alpha_c_(alpha_c) {}
    void check() const {
        if (q_ != T(0.5) || alpha_c_ != T(0.1))
            throw std::invalid_argument("mq_shape_function: the device solves implement q = 0.5, alpha_c = 0.1");
    }
};
// the cubic polyharmonic spline r^3 (no NAGA counterpart; the benchmark
// configurations name it)
template <class T = float>
struct cubic_shape_function {
    static constexpr int id = 1;
    void check() const {}
};

// NAGA's radial_point_method<T> (interpolation/radial_point_method.cuh:
// 92-280) for T = float: weights from augmented RBF systems solved on the
// device (FP64, or FP32 with FP64-residual refinement when precision = 1),
// and the interpolation gather. interpolate() queues the gather on the
// stream and returns a future whose get() waits for it, as NAGA's does.
template <class T = float>
class radial_point_method {
    static_assert(std::is_same_v<T, float>, "radial_point_method: T = float");

  public:
    radial_point_method() = default;

    // weights [n_queries][k] (NAGA's {k, n_queries}); interpolating_indices
    // [n_queries / group_size][k], indices into source_points (D x N)
    template <unsigned D, class ShapeFunctionType = mq_shape_function<T>>
    static device_array<T> compute_weights(const device_array<const T>& source_points,
                                           const device_array<const uint32_t>& interpolating_indices,
                                           const default_point_map<T, D>& query_points,
                                           const T& approx_particle_spacing, unsigned group_size = 1,
                                           const ShapeFunctionType& shape_function = ShapeFunctionType{},
                                           int precision = 0, cudaStream_t stream = nullptr) {
        shape_function.check();
        const size_t nq = query_points.size();
        if (group_size == 0 || nq % group_size != 0)
            throw std::invalid_argument("query_size must be a multiple of group_size");
        const size_t ngroups = nq / group_size;
        if (ngroups == 0) return device_array<T>(0);
        if (interpolating_indices.size() % ngroups != 0)
            throw std::invalid_argument("radial_point_method: indices must hold k x (n_queries / group_size) values");
        const int k = (int)(interpolating_indices.size() / ngroups);
        device_array<T> w(nq * (size_t)k);
        detail::check(naga_rbf_weights_f32(source_points.data(), (int64_t)(source_points.size() / D), (int)D,
                                           interpolating_indices.data(), k, query_points.points.data(),
                                           (int64_t)ngroups, (int)group_size, approx_particle_spacing,
                                           ShapeFunctionType::id, precision, w.data(), stream),
                      "radial_point_method::compute_weights");
        return w;
    }

    template <unsigned D, class ShapeFunctionType = mq_shape_function<T>>
    static radial_point_method create_interpolator(const device_array<const T>& source_points,
                                                   const device_array<const uint32_t>& interpolating_indices,
                                                   const default_point_map<T, D>& query_points,
                                                   const T& approx_particle_spacing, unsigned group_size = 1,
                                                   const ShapeFunctionType& shape_function = ShapeFunctionType{},
                                                   int precision = 0, cudaStream_t stream = nullptr) {
        radial_point_method r;
        r.weights_ = compute_weights<D>(source_points, interpolating_indices, query_points, approx_particle_spacing,
                                        group_size, shape_function, precision, stream);
        r.indices_ = interpolating_indices;
        r.group_size_ = group_size;
        r.n_queries_ = query_points.size();
        r.k_ = r.n_queries_ ? r.weights_.size() / r.n_queries_ : 0;
        r.source_points_size_ = source_points.size() / D;
        return r;
    }

    // destination = sum_s w (field(support) - offset) + offset for every
    // query; field holds C values per source point and destination C per
    // query (C = 1: NAGA's one-dimensional overload, C > 1: its {C, N} one)
    std::future<void> interpolate(const device_array<const T>& field, const device_array<T>& destination,
                                  T centering_offset = T(0), cudaStream_t stream = nullptr) const {
        if (source_points_size_ == 0 || field.size() % source_points_size_ != 0)
            throw std::invalid_argument(
                "field array must have the same number of rows as the number of source points used to construct "
                "the interpolator");
        const size_t C = field.size() / source_points_size_;
        if (destination.size() != C * n_queries_)
            throw std::invalid_argument(
                "destination array must have the same number of columns as the number of points used to "
                "construct the interpolator");
        detail::check(naga_rbf_interpolate(weights_.data(), indices_.data(), (int64_t)n_queries_, (int)group_size_,
                                           (int)k_, field.data(), (int64_t)source_points_size_, (int)C,
                                           centering_offset, destination.data(), stream),
                      "radial_point_method::interpolate");
        return detail::stream_future(stream);
    }

    device_array<const T> weights() const { return weights_; }
    device_array<const uint32_t> indices() const { return indices_; }
    unsigned group_size() const { return group_size_; }
    size_t support_size() const { return k_; }

  private:
    device_array<T> weights_;
    device_array<const uint32_t> indices_;
    unsigned group_size_ = 1;
    size_t n_queries_ = 0, k_ = 0, source_points_size_ = 0;
};
}  // namespace interpolation

namespace nonlocal_calculus {
// NAGA's divergence_operator<T, D> (nonlocal_calculus/divergence.cuh:44-
// 212): the nonlocal divergence stencil of a point cloud (kNN, interaction
// radii, quadrature RPIM weights; naga_divergence_build[_f32]) and its
// gather apply(field, result, centering_offset) (naga_divergence_apply
// [_f64]). T = float stores FP32 weights (the engine's instantiation), T =
// double FP64 ones (NAGA's nonlocal_divergence_3d example). The stencil
// size is NAGA's num_interp_support, 32, unless `k` says otherwise;
// `shape` picks the RBF (0 multiquadric, NAGA's; 1 r^3).
template <class T, unsigned D>
class divergence_operator {
    static_assert(std::is_same_v<T, float> || std::is_same_v<T, double>, "divergence_operator: float or double");

  public:
    using default_field_map = default_point_map<T, D>;
    divergence_operator() = default;

    // create(domain, query_points, override_query_size): NAGA's weight
    // kernel reads the node position from the domain array
    // (detail/divergence.inl:171), so its every caller passes the domain as
    // the query set; so must callers here (the same array). Rows past the
    // point count up to override_query_size are zero, as NAGA's.
    static divergence_operator create(const device_array<const T>& domain, const device_array<const T>& query_points,
                                      size_t override_query_size = 0, int k = 32, int shape = 0, int precision = 0,
                                      cudaStream_t stream = nullptr) {
        if (query_points.data() != domain.data() || query_points.size() != domain.size())
            throw std::invalid_argument(
                "divergence_operator::create: the query points must be the domain (the stencil weights are built at "
                "the domain's nodes)");
        const size_t n = domain.size() / D;
        const size_t rows = override_query_size == 0 ? n : override_query_size;
        if (rows < n)
            throw std::invalid_argument("override_query_size must be at least as large as the number of query points.");
        device_array<float> pts32;
        const float* pts = nullptr;
        if constexpr (std::is_same_v<T, float>) {
            pts = domain.data();
        } else {
            std::vector<double> h = domain.to_host(stream);
            pts32 = device_array<float>::from_host(std::vector<float>(h.begin(), h.end()), stream);
            pts = pts32.data();
        }
        divergence_operator op;
        op.k_ = (size_t)k;
        op.rows_ = rows;
        op.weights_ = device_array<T>(rows * (size_t)k * D);
        op.support_indices_ = device_array<uint32_t>(rows * (size_t)k);
        if (cudaMemsetAsync(op.weights_.data(), 0, sizeof(T) * op.weights_.size(), stream) != cudaSuccess ||
            cudaMemsetAsync(op.support_indices_.data(), 0, 4 * op.support_indices_.size(), stream) != cudaSuccess)
            throw std::runtime_error("divergence_operator::create: memset failed");
        if constexpr (std::is_same_v<T, float>)
            detail::check(naga_divergence_build_f32(pts, (int64_t)n, (int)D, k, shape, precision,
                                                    op.support_indices_.data(), op.weights_.data(), nullptr, stream),
                          "divergence_operator::create");
        else
            detail::check(naga_divergence_build(pts, (int64_t)n, (int)D, k, shape, precision,
                                                op.support_indices_.data(), op.weights_.data(), nullptr, stream),
                          "divergence_operator::create");
        return op;
    }
    static divergence_operator create(const device_array<const T>& domain, cudaStream_t stream = nullptr) {
        return create(domain, domain, 0, 32, 0, 0, stream);
    }

    // result_i = sum_s sum_d W(d, s, i) (field_d(support(s, i)) - offset),
    // queued on `stream` (divergence.cuh:377-488)
    void apply(const default_field_map& field, const device_array<T>& result, const T& centering_offset = T(0),
               cudaStream_t stream = nullptr) const {
        if (result.size() != rows_) throw std::invalid_argument("Result array has incorrect shape.");
        if (result.size() != field.size()) throw std::invalid_argument("Result array has incorrect size.");
        if constexpr (std::is_same_v<T, float>)
            detail::check(naga_divergence_apply(weights_.data(), support_indices_.data(), (int64_t)rows_, (int)D,
                                                (int)k_, field.points.data(), centering_offset, result.data(), stream),
                          "divergence_operator::apply");
        else
            detail::check(naga_divergence_apply_f64(weights_.data(), support_indices_.data(), (int64_t)rows_,
                                                    (int)D, (int)k_, field.points.data(), centering_offset,
                                                    result.data(), stream),
                          "divergence_operator::apply");
    }

    // weights [rows][k][D] (NAGA's {D, k, rows}); support indices [rows][k]
    device_array<const T> weights() const { return weights_; }
    device_array<const uint32_t> support_indices() const { return support_indices_; }
    size_t support_size() const { return k_; }

  private:
    device_array<T> weights_;
    device_array<uint32_t> support_indices_;
    size_t k_ = 0, rows_ = 0;
};
// NAGA's operator_builder<T, D> (nonlocal_calculus/operators.cuh:43-166):
// holds the domain (and query points) and creates an operator over them,
// builder.create<divergence_operator>() as in NAGA's examples
// (examples/nonlocal_divergence_3d.cu:110-113). The query points must be
// the domain, as for divergence_operator::create.
template <class T, unsigned D>
class operator_builder {
  public:
    explicit operator_builder(const device_array<const T>& domain) : domain_(domain), query_(domain) {}
    operator_builder(const device_array<const T>& domain, const device_array<const T>& query_points)
        : domain_(domain), query_(query_points) {}
    template <template <class, unsigned> class Operator>
    Operator<T, D> create(int k = 32, int shape = 0, int precision = 0, cudaStream_t stream = nullptr) const {
        return Operator<T, D>::create(domain_, query_, 0, k, shape, precision, stream);
    }

  private:
    device_array<const T> domain_, query_;
};
}  // namespace nonlocal_calculus

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

// batched_matrix_inverse(A, A_inv) (linalg/batched_matrix_inverse.cuh:
// 389-397) on caller device arrays of `batch` column-major n x n matrices;
// info (batch entries, or empty) receives getrf's status per matrix. Queued
// on `stream`; the future's get() waits for it.
inline std::future<void> batched_matrix_inverse(const device_array<const double>& A, const device_array<double>& A_inv,
                                                int n, const device_array<int>& info = {}, bool refined = false,
                                                cudaStream_t stream = nullptr) {
    if (n < 1 || A.size() % ((size_t)n * n) != 0 || A_inv.size() != A.size())
        throw std::invalid_argument("batched_matrix_inverse: A and A_inv must hold batch x n x n values");
    const int64_t batch = (int64_t)(A.size() / ((size_t)n * n));
    if (!info.empty() && info.size() != (size_t)batch)
        throw std::invalid_argument("batched_matrix_inverse: info must hold one entry per matrix");
    if (refined)
        detail::check(naga_batched_inverse_f32r(A.data(), A_inv.data(), n, batch, 30, 1e-14,
                                                info.empty() ? nullptr : info.data(), stream),
                      "batched_matrix_inverse");
    else
        detail::check(naga_batched_inverse_f64(A.data(), A_inv.data(), n, batch, info.empty() ? nullptr : info.data(),
                                               stream),
                      "batched_matrix_inverse");
    return detail::stream_future(stream);
}
}  // namespace linalg

}  // namespace naga
