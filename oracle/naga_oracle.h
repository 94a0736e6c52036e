/*
 * CPU oracle for the NAGA nonlocal lattice-Boltzmann acoustics step.
 *
 * TEST INFRASTRUCTURE ONLY. The CUDA product is tested against it: tests/, the smoke
 * entry and bench.py's CPU-baseline leg may call it. The product
 * (naga_b200/, include/) never links, loads or executes anything here.
 *
 * It restates, in plain C++, the algorithms of NAGAGroup/NAGA that sit on
 * the step's path (file:line citations are on each function in
 * naga_oracle.cpp). Precision: every routine computes in FP64; the step can
 * also run in the reference's own FP32 arithmetic (the reference instantiates
 * everything with T = float, e.g. examples/nonlocal_lbm_pulse_3d.cu:35) for
 * the timed CPU baseline and for error-budget studies.
 *
 * All arrays are host memory, row-major, with the layouts stated per call.
 */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- exact k nearest neighbours under the (dist^2, index) order ------- */
/* src: [n][dim] float, qry: [nq][dim] float -> idx/d2: [nq][k].
 * dist^2 is evaluated exactly as distance_functions.hpp:138-161 (highest
 * dimension first, no FMA contraction). grid=0 selects brute force.       */
int orc_knn(const float* src, int64_t n, const float* qry, int64_t nq, int dim,
            int k, int grid, uint32_t* idx, float* d2);

/* ---- NAGA's own ring search (cells of ~approx points, stops one ring
 * after the k-th candidate), restated to compare neighbour SETS with the
 * exact search: nd_cubic_segmentation.cuh:227-303, nearest_neighbors.cuh:
 * 207-411. Cells are visited in index order, not NAGA's random order.    */
int orc_knn_ring_reference(const float* src, int64_t n, const float* qry,
                           int64_t nq, int dim, int k, int approx,
                           uint32_t* idx, float* d2);

/* ---- NAGA's cubic segmentation (nd_cubic_segmentation.cuh:227-303,
 * get_partition_index :376-392) in its FP32 arithmetic: bounds, width,
 * shape; per partition (linear index x + shape0 (y + shape1 z)) its size,
 * the exclusive prefix sums and the point indices grouped by partition,
 * ascending within one. Call with NULL arrays to learn n_cells first.   */
int orc_cubic_segmentation(const float* src, int64_t n, int dim, int approx,
                           float* lower, float* upper, float* width,
                           int64_t* shape, int64_t* n_cells, uint32_t* sizes,
                           uint32_t* offsets, uint32_t* indices);

/* ---- batched LU inverse (getrf + getri semantics), FP64 -------------- */
/* A, Ainv: [batch][n][n] column-major per matrix; info[batch] (0 = ok,
 * j>0 = U(j,j) exactly zero, LAPACK convention).                          */
int orc_batched_inverse_f64(const double* A, int n, int64_t batch,
                            double* Ainv, int* info);

/* ---- RBF (radial point interpolation) weights, FP64 ----------------- */
/* shape: 0 = multiquadric (r^2 + (0.1 h)^2)^0.5, 1 = cubic polyharmonic r^3.
 * support: [ngroups][k] indices into src ([n][dim]); qry: [ngroups*group][dim]
 * (double); weights out: [ngroups*group][k] double.                        */
int orc_rbf_weights(const float* src, int64_t n, int dim,
                    const uint32_t* support, int k, const double* qry,
                    int64_t ngroups, int group, double spacing, int shape,
                    double* weights);

/* ---- nonlocal divergence stencil (W[d,s,i]) -------------------------- */
/* pts: [n][dim] float. Out: idx [n][k], W [n][k][dim] (double),
 * delta [n] (interaction radius). Restates divergence.cuh:53-166,
 * operators.cuh:77-136, divergence.inl:135-227.                          */
int orc_divergence_stencil(const float* pts, int64_t n, int dim, int k,
                           int shape, uint32_t* idx, double* W,
                           double* delta);

/* ---- scene: domain, set-up and time step ---------------------------- */
typedef struct orc_scene_desc {
    int dim;               /* 2 (D2Q9) or 3 (D3Q27) */
    int k;                 /* divergence / filter stencil size */
    int k_boundary;        /* boundary RPIM support size */
    int k_probe;           /* probe RPIM support size */
    int shape;             /* 0 = MQ, 1 = PHS r^3 */
    int pml_indexing;      /* 0 = as the reference, 1 = corrected */
    int precision;         /* 0 = FP64, 1 = FP32 (reference arithmetic) */
    int64_t n_bulk, n_layer, n_boundary, n_ghost;
    double nodal_spacing;
    double viscosity, rho0, time_step, speed_of_sound;
    const float* points;   /* [N][dim] */
    const float* normals;  /* [n_boundary][dim] (inward) */
    const float* sigma;    /* [n_layer] */
    int n_probes;
    const float* probes;   /* [n_probes][dim] */
} orc_scene_desc;

typedef struct orc_scene orc_scene;

int orc_scene_create(const orc_scene_desc* desc, orc_scene** out);
void orc_scene_destroy(orc_scene* s);
/* drho: [N] float, density perturbation in units of rho0; u = 0.        */
int orc_scene_set_density(orc_scene* s, const float* drho);
/* advance nsteps; probe densities (rho - rho0) sampled at the start of
 * every step are appended to out_probes [nsteps][n_probes] (may be NULL). */
int orc_scene_step(orc_scene* s, int nsteps, double* out_probes);
/* density sources (per-step values of a node set, dimensional density,
 * FLT_MAX = no term that step), applied after the probes of each step as
 * detail/simulation_engine.cuh:1057-1107 without its race               */
int orc_scene_set_sources(orc_scene* s, const int64_t* nodes, int64_t n,
                          const float* values, int64_t n_steps);
/* centred populations g = f - w, [N][Q] double, and rho - rho0 [N].      */
int orc_scene_read_state(const orc_scene* s, double* g, double* drho);
/* replace the populations (centred, [N][Q]) and recompute macros.        */
int orc_scene_write_state(orc_scene* s, const double* g);
/* stencil / weight tables built at set-up (for kernel-level tests).      */
int orc_scene_tables(const orc_scene* s, uint32_t* idx, double* W,
                     double* filter_w, uint32_t* bidx, double* bw,
                     uint32_t* pidx, double* pw);
/* individual phases of one step, for stage-level comparisons:
 * phase 1: after the pre-streaming part (macros .. bounce-back);
 * phase 2: after RK4 and the final boundary interpolation.               */
int orc_scene_step_phase(orc_scene* s, int phase);
int orc_scene_pml_state(const orc_scene* s, double* q1, double* q2);

/* OpenMP threads of the calling thread's later parallel regions (n <= 0
 * leaves it); returns the number now in effect (1 without OpenMP).      */
int orc_set_threads(int n);

/* ---- synthetic scene inputs (scene_inputs.cpp) ---------------------- */
/* Jittered n_side^dim grid of the unit square / cube with NAGA's node
 * classes; counts[3] = {bulk, layer, boundary}; outputs may be NULL (call
 * once with NULL outputs for the counts). points [N][dim], normals
 * [n_boundary][dim] (inward), sigma [n_layer], h = 1 / (n_side - 1).      */
int orc_grid_generate(int dim, int64_t n_side, int n_layers, double jitter,
                      double sigma_peak, uint64_t seed, int64_t* counts,
                      float* points, float* normals, float* sigma, double* h);
/* drho_i = amplitude exp(-|x_i - center|^2 / (2 width^2)) (FP64, stored FP32) */
int orc_gaussian_pulse(const float* points, int64_t n, int dim,
                       const double* center, double amplitude, double width,
                       float* drho);

/* ---- lattice tables (for tests of the product's tables) -------------- */
int orc_lattice(int dim, int* Q, double* c /*[Q][dim]*/, double* w /*[Q]*/,
                int* bb /*[Q]*/, double* K /*[Q][Q]*/);
/* collision increment dF = (K k) for given f, rho, u (lattice units).     */
int orc_collision(int dim, const double* f, double rho, const double* u,
                  double nu_lat, double dt_lat, double* df);

#ifdef __cplusplus
}
#endif
