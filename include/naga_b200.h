/*
 * naga_b200: B200-native (sm_100a) nonlocal lattice-Boltzmann acoustics step.
 *
 * C ABI of libnaga_b200.so. Plain pointers and sizes only; no exceptions
 * cross this boundary. Every entry point returns an int status (NAGA_OK on
 * success); naga_last_error() gives a message for the calling thread.
 *
 * Each declaration names the NAGA (NAGAGroup/NAGA) interface it replaces,
 * as path:line within that project. The header-only C++ facade in
 * include/naga/ maps the reference's template API onto these calls.
 *
 * Memory: "host" arguments are ordinary host memory; "device" arguments are
 * CUDA device pointers on the current device. Scene and batch handles own
 * their device buffers. Streams are passed as void* (a cudaStream_t; NULL is
 * the legacy default stream).
 *
 * Threading: a handle is not thread-safe; distinct handles may be used from
 * distinct threads. The library starts no threads of its own.
 */
#ifndef NAGA_B200_H
#define NAGA_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
/* replaces the exceptions of sclx::throw_exception<std::invalid_argument |
 * std::runtime_error> (e.g. fluids/nonlocal_lattice_boltzmann/detail/
 * simulation_engine.cuh:128-167, linalg/batched_matrix_inverse.cuh:252-272) */
enum {
    NAGA_OK = 0,
    NAGA_EINVAL = 1,       /* invalid argument / shape mismatch            */
    NAGA_ENOMEM = 2,       /* allocation failed or over the memory budget  */
    NAGA_ECUDA = 3,        /* a CUDA runtime call failed                   */
    NAGA_ENOCONVERGE = 4,  /* refinement did not reach the tolerance       */
    NAGA_ETIMEOUT = 5,     /* a bounded device wait gave up                */
    NAGA_ESINGULAR = 6,    /* exactly singular matrix in a factorisation   */
    NAGA_ENODEVICE = 7     /* no CUDA device / extension not usable        */
};

/* message for the last failing call on this thread ("" if none) */
const char* naga_last_error(void);
/* library version: major * 10000 + minor * 100 + patch */
int naga_version(void);

/* ------------------------------------------------------ synthetic scenes */
/* Jittered uniform grid in the unit square/cube with the node classes of
 * NAGA's uniform_grid_provider (fluids/nonlocal_lattice_boltzmann/
 * node_providers/uniform_grid_provider.cuh:65-161): interior nodes jittered
 * by U(-jitter h, +jitter h) per coordinate (splitmix64 stream from `seed`,
 * `dim` draws per grid node in row-major order), walls unjittered, layer =
 * squared distance to the nearest boundary node <= (n_layers h)^2,
 * sigma = sigma_peak ((L - d) / L)^2. Output order: bulk, layer, boundary,
 * each in Morton order of the grid indices.                                 */
typedef struct naga_grid_spec {
    int dim;            /* 2 or 3 */
    int n_layers;       /* absorbing-layer thickness in grid spacings */
    int64_t n_side;     /* grid nodes per side, spacing h = 1 / (n_side - 1) */
    double jitter;      /* jitter as a fraction of h, in [0, 0.5) */
    double sigma_peak;  /* peak absorption coefficient */
    uint64_t seed;
} naga_grid_spec;

int naga_grid_counts(const naga_grid_spec* spec, int64_t* n_bulk,
                     int64_t* n_layer, int64_t* n_boundary);
/* host outputs: points [N][dim], normals [n_boundary][dim] (inward),
 * sigma [n_layer]; any output may be NULL.                                  */
int naga_grid_generate(const naga_grid_spec* spec, float* points,
                       float* normals, float* sigma, double* nodal_spacing);
/* NAGA's uniform_grid_provider(min, max, grid_spacing, layer_thickness,
 * peak_absorption_rate) (node_providers/uniform_grid_provider.cuh:53-161),
 * on the host in its FP32 arithmetic: an axis-aligned box gridded with
 * ceil((max - min) / spacing) + 1 nodes per axis, boundary = outer shell
 * (inward normals), layer = nodes within layer_thickness of the nearest
 * boundary node, sigma = peak ((L - d) / L)^2; classes [bulk, layer,
 * boundary], each in Morton order (morton = 1) or grid order (0). Fill the
 * unused coordinates of min / max for dim = 2 with anything.              */
typedef struct naga_box_grid_spec {
    int dim;
    int morton;
    double min[3], max[3];
    double spacing, layer_thickness, peak_absorption;
} naga_box_grid_spec;

int naga_box_grid_counts(const naga_box_grid_spec* spec, int64_t* n_bulk,
                         int64_t* n_layer, int64_t* n_boundary);
/* host outputs as naga_grid_generate; nodal_spacing = spacing            */
int naga_box_grid_generate(const naga_box_grid_spec* spec, float* points,
                           float* normals, float* sigma,
                           double* nodal_spacing);
/* drho_i = amplitude * exp(-|x_i - center|^2 / (2 width^2)), host arrays    */
int naga_gaussian_pulse(const float* points, int64_t n, int dim,
                        const double* center, double amplitude, double width,
                        float* drho);

/* ------------------------------------------------------------ primitives */
/* Exact k nearest neighbours of each query among src under the
 * (dist^2, index) order; dist^2 is the FP32 value of
 * distance_functions.hpp:138-161 (highest dimension added last). Device
 * arrays: src [n][dim], qry [nq][dim] float; idx, d2 [nq][k] (ascending).
 * With fewer than k sources the slots past the n found hold index
 * 0xffffffff and d2 = +inf (NAGA prints a warning and leaves them unset,
 * segmentation/nearest_neighbors.cuh:421-425). nq = 0 is a no-op. A NaN or
 * infinite source coordinate returns NAGA_EINVAL before the search runs
 * (so does every call that builds stencils from points: the divergence
 * build, scene creation and probes).
 * Replaces nd_cubic_segmentation<T,D>(points, approx_size)
 * (segmentation/nd_cubic_segmentation.cuh:227-303) followed by
 * batched_nearest_neighbors(k, query_map, segmentation)
 * (segmentation/nearest_neighbors.cuh:95-108, 444-477).                     */
int naga_knn(const float* src, int64_t n, const float* qry, int64_t nq,
             int dim, int k, uint32_t* idx, float* d2, void* stream);

/* The same search without allocating device memory, for callers that
 * cannot call cudaMalloc while they run: processes that handed the free
 * device memory to their own caching allocator at start-up and live on a
 * fixed budget, and paths that must not let cudaMalloc / cudaFree
 * synchronise the whole device and stall other streams. No reference
 * counterpart (NAGA allocates its segmentation arrays on every call).
 * Scratch is one fixed device array of ~1.8 MB inside the library, held by
 * every GPU that loads it until the process exits; hence n <= 65536 source
 * points (larger n returns NAGA_EINVAL), any number of queries. The first
 * call on a device looks up the array's device address
 * (cudaGetSymbolAddress), and so does the first call after the device's
 * context was re-created (cudaDeviceReset); make that first call before any
 * stream capture. Each call synchronises `stream` once: it reads the
 * cloud's bounding box back to the host to size its cell grid, then queues
 * the search behind it and returns. Every call shares the one array: calls
 * that overlap on the GPU (other streams, other host threads) race, so
 * serialise them. Each call resets the counters it needs. Results equal
 * naga_knn's bit for bit.                                                  */
int naga_knn_noalloc(const float* src, int64_t n, const float* qry,
                     int64_t nq, int dim, int k, uint32_t* idx, float* d2,
                     void* stream);

/* Self-kNN of many independent clouds in one launch. pts: device
 * [total][dim], clouds back to back; offsets: host [n_clouds + 1]. Output
 * indices are local to each cloud. No reference counterpart as a single
 * call: the reference runs one segmentation + search per cloud
 * (examples/batched_knn_search.cu:96-157 runs it per partition size).       */
int naga_knn_clouds(const float* pts, const int64_t* offsets, int n_clouds,
                    int dim, int k, uint32_t* idx, float* d2, void* stream);

/* Batched inverse of n x n matrices, each column-major, batch back to back
 * (device arrays A, A_inv [batch][n][n]; info [batch] or NULL: 0 = ok,
 * j > 0 = zero pivot at column j). One warp per matrix, LU with partial
 * pivoting (first maximal |a|) then inversion. Replaces
 * linalg::batched_matrix_inverse(A, A_inv, copy_A)
 * (linalg/batched_matrix_inverse.cuh:325-397; cuBLAS getrf/getri at
 * linalg/detail/batched_matrix_inverse.cuh:46-72). n <= 64.               */
int naga_batched_inverse_f64(const double* A, double* A_inv, int n,
                             int64_t batch, int* info, void* stream);
/* Same result computed from an FP32 LU with FP64-residual iterative
 * refinement of each column; a column stops at max_iter, when its
 * correction is below rel_tol relative to the column, or when the
 * correction stops shrinking (the FP64 residual's floor). info: as above,
 * or -1 when some column ended with a correction above both rel_tol and
 * 1e-10 of the column.                                                      */
int naga_batched_inverse_f32r(const double* A, double* A_inv, int n,
                              int64_t batch, int max_iter, double rel_tol,
                              int* info, void* stream);

/* RBF (radial point interpolation) weights: for every group g with support
 * indices support[g][k] into src [n][dim], and its `group` query points
 * qry [ngroups*group][dim], weights[q][k] such that the interpolant at
 * query q is sum_s weights[q][s] * value(support[g][s]). Augmented system
 * [[Phi, P], [P^T, 0]] with P = [1, x] (n_sys = k + dim + 1 <= 64).
 * shape: 0 = multiquadric (r^2 + (0.1 spacing)^2)^0.5, 1 = cubic r^3.
 * precision: 0 = FP64 LU, 1 = FP32 LU + FP64-residual refinement.
 * Replaces radial_point_method<T>::compute_weights
 * (interpolation/radial_point_method.cuh:118-139; detail :92-472).
 * Device arrays; weights are FP64.                                          */
int naga_rbf_weights(const float* src, int64_t n, int dim,
                     const uint32_t* support, int k, const double* qry,
                     int64_t ngroups, int group, double spacing, int shape,
                     int precision, double* weights, void* stream);

/* Number of systems of the calling thread's last naga_rbf_weights /
 * naga_divergence_build / scene set-up with precision 1 whose FP32
 * refinement did not reach 1e-10 and were re-solved in FP64.                */
int64_t naga_refinement_fallbacks(void);

/* Nonlocal divergence stencil over the points pts [n][dim] (device):
 * idx [n][k] (kNN), W [n][k][dim] (FP64) with W(d,s,i) the weight of
 * support s of node i in dimension d, delta [n] (interaction radius) or
 * NULL. Replaces divergence_operator<T,D>::create(domain, queries)
 * (nonlocal_calculus/divergence.cuh:53-166; operators.cuh:77-136;
 * detail/divergence.inl:135-227).                                           */
int naga_divergence_build(const float* pts, int64_t n, int dim, int k,
                          int shape, int precision, uint32_t* idx, double* W,
                          double* delta, void* stream);
/* The same stencil with FP32 outputs: W [n][k][dim] and delta [n] (or
 * NULL) as floats (the solves stay FP64 or refined FP32 as `precision`
 * says). Replaces divergence_operator<float, D>::create(domain) (the
 * engine's T = float instantiation, detail/simulation_engine.cuh:169-181). */
int naga_divergence_build_f32(const float* pts, int64_t n, int dim, int k,
                              int shape, int precision, uint32_t* idx,
                              float* W, float* delta, void* stream);
/* result_i = sum_s t_s, t_s = sum_d W(d,s,i) (field[idx(s,i)][d] - offset)
 * with W stored [n][k][dim] and field [n][dim] (device); the t_s are summed
 * by NAGA's pairwise tree (stride 1, 2, 4, ...), k <= 64. Replaces
 * divergence_operator<T, D>::apply(field, result, centering_offset) with
 * default_point_map (nonlocal_calculus/divergence.cuh:183-212, 377-488):
 * FP32 here, FP64 in naga_divergence_apply_f64.                            */
int naga_divergence_apply(const float* W, const uint32_t* idx, int64_t n,
                          int dim, int k, const float* field,
                          float centering_offset, float* result, void* stream);
int naga_divergence_apply_f64(const double* W, const uint32_t* idx, int64_t n,
                              int dim, int k, const double* field,
                              double centering_offset, double* result,
                              void* stream);

/* RBF weights with FP32 queries and FP32 weights (the solves are FP64, or
 * refined FP32 with precision 1): radial_point_method<float>::
 * compute_weights(source_points, interpolating_indices, query_points,
 * approx_particle_spacing, group_size, shape_function)
 * (interpolation/radial_point_method.cuh:118-139). Arguments as
 * naga_rbf_weights; weights [ngroups * group][k] (NAGA's {k, n_queries}).  */
int naga_rbf_weights_f32(const float* src, int64_t n, int dim,
                         const uint32_t* support, int k, const float* qry,
                         int64_t ngroups, int group, float spacing, int shape,
                         int precision, float* weights, void* stream);
/* out[q][c] = sum_s weights[q][s] (field[support[q / group][s]][c] - offset)
 * + offset, summed over s in order in FP32: radial_point_method<float>::
 * interpolate(field, destination, centering_offset)
 * (interpolation/radial_point_method.cuh:172-280) for n_fields components
 * per point (field [n_src][n_fields], out [nq][n_fields]; n_fields = 1 is
 * the one-dimensional overload). Device arrays.                           */
int naga_rbf_interpolate(const float* weights, const uint32_t* support,
                         int64_t nq, int group, int k, const float* field,
                         int64_t n_src, int n_fields, float centering_offset,
                         float* out, void* stream);

/* NAGA's nd_cubic_segmentation<float, D>(points, approx_partition_size)
 * (segmentation/nd_cubic_segmentation.cuh:227-303) in two calls. First the
 * partition grid, on the host in NAGA's FP32 arithmetic from the device
 * bounds: lower / upper bounds (an axis thinner than 1e-3 widened to 1e-3),
 * width = (approx / n * volume)^(1/dim), shape[d] = ceil(extent / width),
 * upper = lower + shape * width (host outputs, dim entries each; the call
 * synchronises the stream). Then the partitions: every point's partition
 * as get_partition_index (:376-392; x >= upper -> shape - 1, and a
 * quotient that rounds up to shape is clamped to shape - 1), linear index
 * x + shape[0] (y + shape[1] z); sizes [n_partitions], their exclusive
 * prefix sums offsets [n_partitions] and the point indices grouped by
 * partition indices [n] (device outputs; n_partitions = product of
 * shape). Within a partition the indices ascend (NAGA's order there is that
 * of its atomic increments).                                              */
int naga_segmentation_shape(const float* pts, int64_t n, int dim,
                            int approx_partition_size, float* lower,
                            float* upper, float* width, int64_t* shape,
                            void* stream);
int naga_segmentation_build(const float* pts, int64_t n, int dim,
                            const float* lower, const float* upper,
                            float width, const int64_t* shape,
                            uint32_t* sizes, uint32_t* offsets,
                            uint32_t* indices, void* stream);

/* ---------------------------------------------------------------- scenes */
/* One acoustic scene: domain, stencils and device-resident state.
 * Replaces naga::fluids::nonlocal_lbm::simulation_engine<Lattice>
 * (fluids/nonlocal_lattice_boltzmann/simulation_engine.cuh:40-121):
 * set_problem_parameters :52-66, init_domain :68-74, step_forward :76,
 * reset :78, attach_observer(density_observer) :90-96, time() :98.        */
typedef struct naga_scene naga_scene;

typedef struct naga_scene_desc {
    int dim;              /* 2 -> D2Q9, 3 -> D3Q27 */
    int k;                /* divergence and filter stencil size (<= 64)   */
    int k_boundary;       /* boundary-interpolation support size          */
    int k_probe;          /* probe-interpolation support size             */
    int shape;            /* RBF: 0 = multiquadric (NAGA default), 1 = r^3 */
    int pml_indexing;     /* 0 = as NAGA (layer fields read Q of the node
                             n_bulk places earlier, pml_absorption.inl:
                             438-448), 1 = each layer node reads its own Q */
    int weight_precision; /* 0 = FP64 weight solves, 1 = FP32 + refinement */
    int n_probes;
    int64_t n_bulk, n_layer, n_boundary, n_ghost;
    double nodal_spacing;
    /* set_problem_parameters(nu, rho0, dt, c) */
    double viscosity, rho0, time_step, speed_of_sound;
    /* host arrays, copied at creation */
    const float* points;   /* [N][dim], order bulk, layer, boundary, ghost */
    const float* normals;  /* [n_boundary][dim], inward                     */
    const float* sigma;    /* [n_layer]                                     */
    const float* probes;   /* [n_probes][dim]                               */
    int probe_capacity;    /* probe samples kept on the device (ring)       */
} naga_scene_desc;

/* builds stencils and weights on the device and sets the rest state:
 * simulation_engine::set_problem_parameters + init_domain
 * (simulation_engine.cuh:52-74) in one call                              */
int naga_scene_create(const naga_scene_desc* desc, naga_scene** out);
int naga_scene_destroy(naga_scene* scene);
/* simulation_engine::set_problem_parameters (simulation_engine.cuh:52-66)
 * on an existing scene: nu, rho0, dt, c take effect at the next step (the
 * lattice-unit rates are recomputed; the stencils do not depend on them) */
int naga_scene_set_params(naga_scene* scene, double viscosity, double rho0,
                          double time_step, double speed_of_sound);
/* simulation_engine::init_domain (simulation_engine.cuh:68-74) on an
 * existing handle: the scene is rebuilt from desc (new nodes, stencils,
 * probes; rest state, step 0). The scene must not belong to a user batch.
 * On error the scene keeps its previous domain.                          */
int naga_scene_init_domain(naga_scene* scene, const naga_scene_desc* desc);
/* the initial condition: the same as naga_scene_set_density             */
int naga_scene_set_initial_condition(naga_scene* scene, const float* drho);
/* attach_observer of a density probe (density_observer.cuh:47-97) after
 * creation: its RPIM tables are built, the probe ring gains a column
 * (earlier samples of the other probes are kept; the new probe reads 0
 * for steps before it was added); *index receives its probe index.      */
int naga_scene_add_probe(naga_scene* scene, const float* xyz, int* index);
/* stream the scene's work is issued on (a cudaStream_t) */
void* naga_scene_stream(naga_scene* scene);
/* rest state plus a density perturbation (host [N], units of rho0), u = 0;
 * resets time and the probe ring. drho == NULL gives NAGA's reset().     */
int naga_scene_set_density(naga_scene* scene, const float* drho);
/* enqueue nsteps time steps on the scene's stream (asynchronous)         */
int naga_scene_step(naga_scene* scene, int nsteps);
int naga_scene_sync(naga_scene* scene);
/* steps taken since the last set_density                                 */
int64_t naga_scene_step_count(const naga_scene* scene);
/* probe samples (rho - rho0, sampled at the start of each step) for steps
 * [first, first + count), host out [count][n_probes]; the ring keeps the
 * last probe_capacity steps. Synchronises the scene's stream.            */
int naga_scene_read_probes(naga_scene* scene, int64_t first, int64_t count,
                           float* out);
/* as naga_scene_read_probes, but only enqueues the copy on the scene's
 * stream behind the steps already enqueued and returns: out (page-locked
 * host memory for a truly asynchronous copy) is filled once the stream
 * reaches it, e.g. after naga_scene_sync. An observer of a running
 * simulation reads every step this way without stalling the device
 * (NAGA's density_observer reads inside step_forward,
 * density_observer.cuh:99-113). first + count may run up to the steps
 * enqueued so far; the ring must still hold step `first` when the copy
 * runs (count <= probe_capacity, and at most probe_capacity - count steps
 * enqueued after it).                                                     */
int naga_scene_read_probes_async(naga_scene* scene, int64_t first,
                                 int64_t count, float* out);
/* centred populations g = f - w, host [N][Q], and rho - rho0, host [N]   */
int naga_scene_read_state(naga_scene* scene, float* g, float* drho);
/* the lattice in the library's population order (the order of g in
 * naga_scene_read_state / write_state): Q, weights [Q] and velocities
 * [Q][dim] (integers); outputs may be NULL. The order and values are NAGA's
 * (detail/d2q9_lattice.cuh:44-88, detail/d3q27_lattice.cuh:45-123).        */
int naga_lattice(int dim, int* q, float* weights, int* velocities);
/* the macroscopic values of simulation_engine::solution()
 * (simulation_variables.cuh:52-62: fluid_density, fluid_velocity), as NAGA
 * stores them -- dimensional, rho rho0 and u c / c_s -- and computed where
 * NAGA computes them, at the start of the last step (after its density
 * sources; boundary velocities 0, as its bounce-back leaves them). Host
 * out: density [N], velocity [N][dim]; either may be NULL.               */
int naga_scene_read_macros(naga_scene* scene, float* density, float* velocity);
/* Density sources (replace simulation_engine::register_density_source,
 * simulation_engine.cuh:80-82, and density_source::add_density_source,
 * density_source.cuh:41-82): values [n_steps][n_nodes] of the listed nodes
 * (dimensional density; FLT_MAX = no term that step, NAGA's sentinel), kept
 * on the device; step first_step + r (steps counted from the last
 * set_density) applies row r after the probes sample the macros:
 * f_a += (s / rho0) w_a, rho <- rho + s / 2 once per node (NAGA's pass does
 * these from racing threads, detail/simulation_engine.cuh:1057-1107). Other
 * steps have no source. Replaces any earlier sources (the device node map
 * is reused when the node list is unchanged, so a caller may upload one row
 * per step cheaply); n_nodes = 0 removes them.                             */
int naga_scene_set_density_source(naga_scene* scene, const int64_t* nodes,
                                  int64_t n_nodes, const float* values,
                                  int64_t first_step, int64_t n_steps);
/* Snapshots (replace NAGA's cereal save/load of its observers and state,
 * density_observer.cuh:115-133, pml_absorption.inl:902-920): the dynamic
 * state -- populations, macros, PML integrals, step counters, probe ring --
 * as one host buffer with a versioned header. Loading it into a scene
 * created from the same description resumes stepping bit for bit (the
 * eviction / resume format of a serving loop). Stencil tables are rebuilt
 * from the description, not stored.                                       */
int64_t naga_scene_snapshot_bytes(const naga_scene* scene);
int naga_scene_save(naga_scene* scene, void* buf, int64_t capacity);
int naga_scene_load(naga_scene* scene, const void* buf, int64_t size);
int naga_scene_write_state(naga_scene* scene, const float* g);
/* set-up tables as stored for the step: idx [N][k], W [N][k][dim],
 * filter weights [N][k], boundary idx/weights [n_boundary][k_boundary],
 * probe idx/weights [n_probes][k_probe]. Any output may be NULL.         */
int naga_scene_read_tables(naga_scene* scene, uint32_t* idx, float* W,
                           float* filter_w, uint32_t* bidx, float* bw,
                           uint32_t* pidx, float* pw);
/* device bytes held by the scene                                          */
int64_t naga_scene_device_bytes(const naga_scene* scene);
/* number of nodes N and populations Q                                     */
int naga_scene_size(const naga_scene* scene, int64_t* n_nodes, int* q);

/* ---------------------------------------------------------------- batches */
/* Many independent scenes of one lattice advanced together: one launch per
 * kernel of the step covers every member scene, and the whole step is a
 * CUDA graph. No reference counterpart: NAGA steps one engine at a time.  */
typedef struct naga_batch naga_batch;

int naga_batch_create(int dim, naga_batch** out);
/* priority 1 creates the batch stream at the device's highest stream
 * priority, so its steps run ahead of work queued on other streams (scene
 * set-up); 0 is naga_batch_create                                         */
int naga_batch_create_with_priority(int dim, int priority, naga_batch** out);
int naga_batch_destroy(naga_batch* batch);
/* membership changes take effect at the next naga_batch_step             */
int naga_batch_add(naga_batch* batch, naga_scene* scene);
int naga_batch_remove(naga_batch* batch, naga_scene* scene);
int naga_batch_size(const naga_batch* batch);
void* naga_batch_stream(naga_batch* batch);
/* applies pending membership changes now: rebuilds the work lists, tunes
 * the launch shape of a new batch shape (naga_tuning_report) and captures
 * the step graph; naga_batch_step does the same when it is still pending.
 * Lets a caller keep that one-off work out of a timed window.            */
int naga_batch_prepare(naga_batch* batch);
/* enqueue nsteps steps of every member scene (asynchronous)              */
int naga_batch_step(naga_batch* batch, int nsteps);
int naga_batch_sync(naga_batch* batch);

/* --------------------------------------------------------------- serving */
/* Continuous-batching request loop: requests (a scene and a step count)
 * queue FIFO. A set-up thread of the server admits them -- scene set-up
 * (kNN, RPIM and stencil weight solves) on each scene's own stream,
 * overlapping the running batch on the device -- while the requests fit
 * the device-memory budget and the slot limit and, with a per-step latency
 * target, while the batch's step time with them (estimated from the
 * measured time per node-step) stays within the target; it also frees the
 * scenes of retired requests. Every naga_server_tick, on the caller's
 * thread, advances all active scenes by steps_per_tick steps as one batch
 * (a CUDA event after each step gives the per-step latency samples), then
 * retires finished requests (their probe traces kept on the host) and adds
 * the scenes whose set-up finished; batch changes (naga_batch_prepare)
 * happen before the timed steps of a tick. The tick never waits for
 * set-up. No reference counterpart: NAGA steps one engine at a time
 * (simulation_engine.cuh:76).                                              */
typedef struct naga_server naga_server;

typedef struct naga_server_config {
    int dim;               /* lattice of every request                       */
    int steps_per_tick;    /* steps per tick (>= 1)                          */
    int max_active;        /* scene slots, 0 = limited by memory only        */
    int step_priority;     /* 0: the batch's steps and admissions' set-up
                              share the device; 1: steps first
                              (naga_batch_create_with_priority)             */
    int64_t memory_budget; /* device bytes the active scenes may hold        */
    double target_step_ms; /* per-step latency target of the batch, 0 = none:
                              admission stops while the estimated step time
                              with the next request would exceed it (an
                              empty batch always takes one request)        */
} naga_server_config;

typedef struct naga_server_stats {
    int64_t ticks, steps, node_updates;
    double busy_ms;         /* device time of the batch steps               */
    double p50_step_ms, p99_step_ms;  /* per-step device time (events)     */
    int64_t bytes_in_use, peak_bytes;
    int64_t done, failed;
    int active, queued;     /* queued includes requests in set-up          */
    /* host wall time summed per activity: preparing the batch (membership
     * changes, graph capture), scene set-up (on the set-up thread), waiting
     * for the batch's steps, retiring and growing the batch               */
    double prepare_ms, admit_ms, wait_ms, retire_ms;
    /* wall time from submission to completion of the finished requests,
     * and from submission to the end of set-up of the admitted ones        */
    double p50_request_ms, p99_request_ms, p50_queue_ms;
    int64_t admitted;
} naga_server_stats;

/* estimated device bytes of a scene (resident state plus set-up scratch)  */
int64_t naga_scene_estimate_bytes(const naga_scene_desc* desc);
int naga_server_create(const naga_server_config* cfg, naga_server** out);
int naga_server_destroy(naga_server* server);
/* copies the host inputs; drho as in naga_scene_set_density; probe
 * capacity is set from steps                                              */
int naga_server_submit(naga_server* server, const naga_scene_desc* desc,
                       const float* drho, int64_t steps, int64_t* id);
int naga_server_tick(naga_server* server, int* n_active, int* n_queued);
/* state: 0 queued, 1 active, 2 done, 3 failed (naga_last_error has why)  */
int naga_server_request_state(naga_server* server, int64_t id, int* state,
                              int64_t* steps_done);
/* probe trace of a finished request, host [steps][n_probes]; releases it  */
int naga_server_result(naga_server* server, int64_t id, float* probes);
int naga_server_read_stats(naga_server* server, naga_server_stats* out);

/* ---------------------------------------------------------------- timing */
/* Per-kernel CUDA-event timing of the step kernels (off by default).
 * When on, every step kernel launch is bracketed by events on the stream
 * it runs on; naga_profile_read returns, per kernel id, the launch count
 * and the summed milliseconds. Enabling it disables graph replay.         */
int naga_profile_enable(int on);
int naga_profile_reset(void);
/* names[i] (static strings), launches[i], ms[i] for i < *count (in/out)  */
int naga_profile_read(int* count, const char** names, int64_t* launches,
                      double* ms);

/* ---------------------------------------------------------- launch shapes */
/* The launch shape of the gather kernels is tuned once per batch shape
 * (lattice, stencil sizes, size class) the first time such a batch steps:
 * RK stage 1 is timed on the batch's own items for every candidate pair of
 * threads per node of the RK stages (D3Q27: 8, 7, 4; D2Q9: 2, 1 -- the
 * first is the default, one float4 chunk of the row per thread) and
 * resident blocks per SM (the driver's default shared-memory carveout,
 * then 2 .. max), and the fastest kept; a shape other than the default must
 * beat it by 3%. NAGA_GATHER_BPS=<n> and NAGA_GATHER_TPN=<t> in the
 * environment fix it instead. Results never depend on the shape. Nodes per
 * pass (32 in 3-D, 64 in 2-D) are fixed by the layout of the stencil tables
 * at scene creation. No NAGA counterpart (its launch shapes are fixed by
 * its runtime). Writes the tuner's log (one line per tuned shape:
 * candidates and microseconds per launch) into buf (NUL-terminated,
 * truncated to cap) and returns its full length.                          */
int64_t naga_tuning_report(char* buf, int64_t cap);

/* ------------------------------------------------------ failure detection */
/* Every wait of the step kernels (tile copies into shared memory, on an
 * mbarrier) gives up after a fixed number of polls (about a second on
 * B200), the kernel returns, and the next naga_scene_sync /
 * naga_batch_sync / step reports NAGA_ETIMEOUT with the context still
 * usable. This call exercises that path on the current device: the same
 * wait, on a barrier that nothing completes, with `polls` polls (0 = the
 * step kernels' own limit); it returns NAGA_ETIMEOUT when the wait gave up
 * and the error was reported (and cleared). Run it while no step is in
 * flight: the timeout flag is shared by the device's step kernels.
 * No NAGA counterpart (NAGA's kernels have no bounded waits).             */
int naga_selftest_wait_timeout(int polls);

#ifdef __cplusplus
}
#endif

#endif /* NAGA_B200_H */
