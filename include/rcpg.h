/* rcpgenerator_b200 -- C ABI of the B200 packing engine.
 *
 * Drop-in replacement for the relaxation path of RCPGenerator
 * (KD-physics/RCPGenerator, paths relative to its python_code/python/):
 *   rcpgenerator::run_packing / run_packing_observed
 *       include/rcpgenerator/rcp_generator.hpp:269-280, bound to Python by
 *       src/bindings/module.cpp:236-296 as _rcpgenerator.run_packing(_observed)
 *   its exported per-step kernels
 *       get_pairs_nd_3 (rcp_generator.hpp:200-216), get_forces_nd_3 (:218-243),
 *       adam_update (:245-267), compute_mean_force (:150-155),
 *       scale_diameters_nd (:180-185)
 *   and the initializer
 *       rcpgenerator::initialize_particles (include/rcpgenerator/initialize_particles.hpp:90),
 *       bound as _rcpgenerator.initialize_particles (src/bindings/module.cpp:228-234).
 *
 * Conventions
 *   - Plain pointers and sizes only. Arrays of per-particle vectors are flat and
 *     particle-major: x[i*ndim + d] (the reference flattens its nested vectors
 *     the same way, rcp_generator.cpp:4357-4363).
 *   - "_dev" pointers are CUDA device pointers on the current device; `stream`
 *     is a cudaStream_t (NULL = legacy default stream).
 *   - Every function returns RCPG_OK (0) or a negative error code and, when
 *     `err` is non-NULL, writes a NUL-terminated message into err[errlen].
 *     RCPG_ERUNTIME carries the reference's std::runtime_error text (neighbour
 *     capacity overflow, box/walls length), RCPG_EINVAL an argument error
 *     (the reference's std::invalid_argument / ValueError cases).
 *   - No CPU fallback: without a usable CUDA device every compute entry point
 *     fails with RCPG_ECUDA.
 */
#ifndef RCPG_H
#define RCPG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RCPG_ABI_VERSION 3

#define RCPG_OK 0
#define RCPG_ERUNTIME (-1)
#define RCPG_ECUDA (-2)
#define RCPG_EINVAL (-22)
#define RCPG_ENOSPC (-28)

/* PackingInput + PackingConfig (rcp_generator.hpp:18-33). box/walls may be
 * NULL with length 0 (the reference's defaults: unit box, all periodic). */
typedef struct rcpg_packing_input {
    uint64_t N;
    int32_t ndim;
    const double* positions; /* [N*ndim] */
    const double* diameters; /* [N] */
    const double* box;       /* [box_len] */
    int32_t box_len;
    const int8_t* walls;     /* [walls_len]; walls[0] = -t: t-ball container */
    int32_t walls_len;
    uint32_t neighbor_max;   /* 0 = the reference's default per Ndim */
    uint32_t seed;           /* accepted and unused, as in the reference */
    int32_t fix_height;
} rcpg_packing_input;

/* PackingRunOptions (rcp_generator.hpp:102-123) plus engine selection. */
typedef struct rcpg_run_options {
    uint64_t max_steps;          /* 0 = schedule-derived cap */
    int32_t has_mu_override;
    double mu_override;
    int32_t fix_diameter;
    int32_t has_target_phi;
    double target_phi;
    uint64_t reorder_interval;   /* default 2000; 0 disables the spatial reorder */
    int32_t has_initial_phi_target;
    double initial_phi_target;
    int32_t exact;               /* 1: host-controlled steps + one-thread reduction order */
    int32_t device;              /* CUDA device ordinal */
    int32_t graph_steps;         /* steps per CUDA graph replay (graph mode), 0 = default */
    /* Pair arithmetic, graph mode only (no counterpart in the reference, which is FP64):
     * 0 = FP64 (default); 1 = mixed -- FP32 pair terms on FP64 displacements until the
     * first step whose max overlap (relative, as max_overlap_history) is below
     * mixed_switch, FP64 from that step on. Positions, ADAM state, diameters and all
     * global sums stay FP64. */
    int32_t pair_precision;
    double mixed_switch;         /* default 1e-5 */
    /* Length in steps of the growth rung (mu_flag = 1, rcp_generator.cpp:5834-5931);
     * 0 = the reference's deadline 6000 + 9*sqrt(N*ndim) (at least 1500). Set by a
     * warm start from its predicted growth curve; no counterpart in the reference. */
    uint64_t growth_steps;
} rcpg_run_options;

/* PackingObservation (rcp_generator.hpp:92-98). */
typedef struct rcpg_observation {
    uint64_t step;
    double phi;
    double force_magnitude;
    double energy;
    double max_min_dist;
} rcpg_observation;

/* Observer (PackingObserver, rcp_generator.hpp:125-127): positions is
 * [N*ndim] when the call captures this sample's positions, else NULL. */
typedef void (*rcpg_observer_fn)(const rcpg_observation* obs, const double* positions, void* user);

/* PackingResult (rcp_generator.hpp:35-90) + PackingTrace (:100-108).
 * Library-owned; release with rcpg_result_free. */
typedef struct rcpg_result {
    uint64_t N;
    int32_t ndim;
    uint64_t steps;
    double phi;                /* box-relative, as the reference's result.phi */
    double max_min_dist;
    double force_magnitude;
    double* positions;         /* [N*ndim] (after the spatial reorders) */
    double* diameters;         /* [N] */
    double* box;               /* [ndim] */
    int8_t* walls;             /* [ndim] (normalised) */
    double* phi_history;       /* [steps] each */
    double* force_history;
    double* energy_history;
    double* max_overlap_history;
    double* mu_history;
    double* alpha_history;
    int8_t* mu_flag_history;
    uint64_t* particle_origin; /* [N] */
    uint64_t trace_len;
    uint64_t* trace_steps;     /* [trace_len] */
    double* trace_positions;   /* [trace_len*N*ndim] (NULL unless captured) */
    double* trace_diameters;   /* [trace_len*N] (NULL unless captured) */
    double* trace_phi;
    double* trace_force;
    double* trace_energy;
    double* trace_max_min_dist;
    uint64_t pair_builds;      /* neighbour-list builds performed */
    uint32_t row_capacity;     /* neighbour row capacity in use at the end */
    uint64_t kernel_launches;  /* kernels launched by this run */
    /* mixed precision (pair_precision = 1): the step after which the pair terms were
     * FP64 (0 = never switched), and the relative error, on the final state, of the
     * pair energy sum and of the forces (max |F32 - F64| / max |F64|) with FP32 pair
     * terms against FP64 ones on the same rows. NaN when the run was FP64. */
    uint64_t fp64_switch_step;
    double pair_energy_rel_error;
    double pair_force_rel_error;
} rcpg_result;

const char* rcpg_version(void);
int32_t rcpg_abi_version(void);
/* Number of visible CUDA devices (0 when none / no driver). */
int32_t rcpg_device_count(void);

void rcpg_default_options(rcpg_run_options* opt);

/* run_packing_observed (rcp_generator.hpp:272-280; module.cpp:247-296).
 * progress_interval / trajectory_interval 0 = off. */
int32_t rcpg_run_packing(const rcpg_packing_input* in, const rcpg_run_options* opt,
                         uint64_t progress_interval, int32_t capture_positions,
                         uint64_t trajectory_interval, rcpg_observer_fn observer, void* user,
                         rcpg_result** out, char* err, size_t errlen);
void rcpg_result_free(rcpg_result* r);

/* Many independent packings (the reference's throughput pattern: one process
 * per core, rcptools/jobs.py:392-401, each calling run_packing), all with the
 * run options `opt` (graph engine).
 *   concurrency < 0: the persistent batch engine -- one kernel per ndim in
 *     which every thread block runs whole packings taken from a queue (no
 *     kernel launch per step).
 *   concurrency = 0: the persistent engine for the cheap packings (N x 3^ndim
 *     up to 3e4, diameters within a factor 2.5) and 32 ordinary engines on CUDA
 *     streams for the others, at the same time.
 *   concurrency > 0: that many host threads each drive one ordinary engine at
 *     a time on their own CUDA stream of device opt->device.
 * Exact runs and runs that can reach a target-phi lock always take the stream
 * path.
 * results[k] receives packing k's result (free each with rcpg_result_free) or
 * NULL, and status[k] its RCPG_* code. Returns RCPG_OK when every packing
 * succeeded, else the first failing code, with that packing's index and
 * message in err. */
int32_t rcpg_run_batch(const rcpg_packing_input* inputs, uint64_t count, const rcpg_run_options* opt,
                       int32_t concurrency, rcpg_result** results, int32_t* status, char* err,
                       size_t errlen);
/* Autotuned launch shape of the persistent batch kernel for packings of
 * `ndim` (pair_precision as in rcpg_run_options): the same synthetic batch is
 * timed at 1 and 2 resident blocks per SM (steps_per_s[2], packing-steps per
 * second) and the faster is kept for the process (*blocks_per_sm). Runs the
 * tuning on first use; rcpg_run_batch uses it when every packing goes to the
 * persistent kernel. No counterpart in the reference. */
int32_t rcpg_batch_tuning(int32_t ndim, int32_t device, int32_t pair_precision, int32_t* blocks_per_sm,
                          double* steps_per_s, char* err, size_t errlen);
/* rcpg_run_batch with a growth-rung length per packing (growth_steps[k],
 * 0 = the reference's deadline), overriding opt->growth_steps: the batch form
 * of a learned warm start. No counterpart in the reference. */
int32_t rcpg_run_batch_growth(const rcpg_packing_input* inputs, uint64_t count, const rcpg_run_options* opt,
                              const uint64_t* growth_steps, int32_t concurrency, rcpg_result** results,
                              int32_t* status, char* err, size_t errlen);

/* Step-wise control of one packing (the loop of run_packing_observed,
 * rcp_generator.cpp:5511-6662, advanced in slices). */
typedef struct rcpg_engine rcpg_engine;
int32_t rcpg_engine_create(const rcpg_packing_input* in, const rcpg_run_options* opt,
                           void* stream, rcpg_engine** out, char* err, size_t errlen);
/* Advance by at most max_new_steps (0 = to completion); *finished = 1 once
 * the run has converged or reached its step cap. */
int32_t rcpg_engine_advance(rcpg_engine* e, uint64_t max_new_steps, int32_t* finished,
                            char* err, size_t errlen);
uint64_t rcpg_engine_steps(const rcpg_engine* e);
uint64_t rcpg_engine_kernel_launches(const rcpg_engine* e);
int32_t rcpg_engine_result(rcpg_engine* e, rcpg_result** out, char* err, size_t errlen);
void rcpg_engine_destroy(rcpg_engine* e);
/* Engine diagnostics (no reference counterpart): times `reps` launches of the
 * pair-force kernel on the engine's current state with CUDA events on its
 * stream; *avg_ms = mean launch time, *alg_bytes = algorithmic bytes of one
 * launch, *mean_row = mean neighbour-row length. The run state is unchanged. */
int32_t rcpg_engine_profile_pair_kernel(rcpg_engine* e, uint32_t reps, double* avg_ms,
                                        double* alg_bytes, double* mean_row, char* err,
                                        size_t errlen);
/* The same for the neighbour build's search kernel (the rebuild of
 * get_pairs_kdtree, ENG:2758-3526; in graph mode the tiled build with the
 * step's forces fused): `reps` full rebuilds of the current state, each from a
 * cold L2, timed around the search kernel only. The rows are left rebuilt for
 * the current positions; the control block is restored. */
int32_t rcpg_engine_profile_build_kernel(rcpg_engine* e, uint32_t reps, double* avg_ms,
                                         double* alg_bytes, char* err, size_t errlen);

/* ---- per-step kernels on device buffers ---------------------------------- */

/* Pair shell of a full refresh: min(max(median*1.02, Dmin*2.25), Dmax)*0.5
 * (rcp_generator.cpp:2846, :1210). Host arrays. */
double rcpg_t_shell(const double* D, uint64_t N);

/* Full-refresh neighbour rows (get_pairs_kdtree for ndim <= 3, get_pairs_nd_3
 * otherwise, with every particle refreshed): row i holds every j != i with
 * MIC |x_j - x_i|^2 < r_c^2 (the reference's predicate), ascending, stored
 * column-major: nbr_dev[k*N + i], k < cnt_dev[i] <= row_capacity.
 * *row_need_out = longest row; when it exceeds row_capacity the rows are
 * truncated and RCPG_ENOSPC is returned. box/walls are host arrays [ndim]. */
int32_t rcpg_pairs_full(uint64_t N, int32_t ndim, const double* x_dev, const double* D_dev,
                        const double* box, const int8_t* walls, double t_shell,
                        uint32_t row_capacity, uint32_t* nbr_dev, uint32_t* cnt_dev,
                        uint32_t* row_need_out, void* stream, char* err, size_t errlen);

/* rcpg_pairs_full without device allocation. No counterpart in the reference
 * (its engine allocates host memory only). For callers that must not
 * allocate device memory while they run: applications whose device memory is
 * reserved up front by their own allocator, where an extra cudaMalloc fails or
 * fragments the pool, and time-critical loops, where cudaMalloc / cudaFree
 * would synchronise the device and stall other streams. Same arguments and
 * results as rcpg_pairs_full; the caller still passes every input and output.
 * The scratch is a fixed 8 MiB array of static device memory that every GPU
 * loading this library keeps until the process exits. A working set larger
 * than that -- about N*(16*P + 8*ndim + 24 + 4*row_capacity) bytes plus the
 * cell grid, P = 4 for ndim <= 3, i.e. roughly 20,000 particles in 3-D at
 * row_capacity 64 -- is rejected with RCPG_ENOSPC before any work. The first
 * call on a device looks up the array's device address (cudaGetSymbolAddress)
 * and should be made before any stream capture. Every call waits for `stream`
 * to finish, because it reads the longest row back to the host to report it.
 * All calls share the array and it keeps the previous call's contents (the
 * build clears what must start at zero); calls whose GPU work overlaps in time
 * race and must be serialised. */
int32_t rcpg_pairs_full_noalloc(uint64_t N, int32_t ndim, const double* x_dev, const double* D_dev,
                                const double* box, const int8_t* walls, double t_shell,
                                uint32_t row_capacity, uint32_t* nbr_dev, uint32_t* cnt_dev,
                                uint32_t* row_need_out, void* stream, char* err, size_t errlen);

/* One neighbour build of the graph engine on a given state, with that state's
 * forces: get_pairs_kdtree (ENG:2758-3526) with every particle refreshed, then
 * get_forces_nd_3 (rcp_generator.hpp:218-243) + compute_mean_force
 * (:150-155), the way a rebuild step of the graph engine does them. Rows hold
 * the same partners as rcpg_pairs_full but in the build's scan order (mixed
 * precision: a superset, see below), returned in particle order like
 * rcpg_pairs_full; F_dev [N*ndim] and scalars[7] as rcpg_forces with tree-order
 * sums. Where the build computes the forces in the same pass (the cell-unit
 * search: ndim <= 3, N >= 20,000, one size class) *fused_out = 1, else the
 * pair kernel computes them on the new rows and *fused_out = 0.
 * pair_precision 1 = the graph engine's mixed precision (FP32 pair terms on
 * FP64 differences; the row test is widened by 1e-5 relative, so rows hold
 * every pair of the FP64 shell and a few just outside it), 0 = FP64; plus 2:
 * F_dev and scalars from the pair kernel on the new rows, also when the build
 * fused the forces. Diagnostic entry point for parity tests; no counterpart in
 * the reference. */
int32_t rcpg_pairs_forces_scan(uint64_t N, int32_t ndim, const double* x_dev, const double* D_dev,
                               const double* box, const int8_t* walls, double t_shell, double mu,
                               int32_t pair_precision, uint32_t row_capacity, uint32_t* nbr_dev,
                               uint32_t* cnt_dev, uint32_t* row_need_out, double* F_dev,
                               double* scalars, int32_t* fused_out, void* stream, char* err,
                               size_t errlen);

/* get_forces_nd_3 (rcp_generator.hpp:218-243) on rows from rcpg_pairs_full
 * (any superset of the overlapping pairs gives the same result), followed by
 * compute_mean_force (:150-155). Writes F_dev [N*ndim] and
 * scalars[7] = {U, max_min_dist, Lc, Fmean, dkappa, mean_force, count}.
 * exact_order = 1 reduces the scalars in the reference's one-thread order. */
int32_t rcpg_forces(uint64_t N, int32_t ndim, const double* x_dev, const double* D_dev,
                    const double* box, const int8_t* walls, const uint32_t* nbr_dev,
                    const uint32_t* cnt_dev, uint32_t row_capacity, double mu,
                    int32_t exact_order, double* F_dev, double* scalars, void* stream,
                    char* err, size_t errlen);

/* compute_mean_force (rcp_generator.hpp:150-155) of F_dev [N*ndim]. */
int32_t rcpg_mean_force(uint64_t N, int32_t ndim, const double* F_dev, double* mean_out,
                        void* stream, char* err, size_t errlen);

/* adam_update (rcp_generator.hpp:245-267) for the particles followed by the
 * position step and the single-box wrap, i.e. the fused pass of
 * rcp_generator.cpp:6410-6521, at bias-correction step t >= 1. */
int32_t rcpg_adam_step(uint64_t N, int32_t ndim, const double* F_dev, double* m_dev,
                       double* v_dev, double* x_dev, const double* box, double alpha,
                       uint64_t t, void* stream, char* err, size_t errlen);

/* Growth-aware displacement refresh trigger (rcp_generator.cpp:6104-6145):
 * updates D_last (running min), theta_anchor and, for refreshed particles,
 * x_last; refresh_dev[i] in {0,1}; *count_out = refreshed particles. */
int32_t rcpg_refresh_check(uint64_t N, int32_t ndim, const double* x_dev, double* x_last_dev,
                           const double* D_dev, double* D_last_dev, double* theta_dev,
                           double theta_new, uint8_t* refresh_dev, uint64_t* count_out,
                           void* stream, char* err, size_t errlen);

/* scale_diameters_nd (rcp_generator.hpp:180-185), host arrays; returns the factor. */
double rcpg_scale_diameters_nd(const double* D, uint64_t N, double phi_target, const double* box,
                               int32_t ndim, int32_t fix_height, double* D_out);

/* ---- initializer ---------------------------------------------------------- */

/* Distribution (initialize_particles.hpp:18-31); type is a NUL-terminated
 * name: mono, gaussian, bigaussian, bidisperse, lognormal, flat, powerlaw,
 * exponential, weibull, custom. */
typedef struct rcpg_distribution {
    const char* type;
    double d, mu, sigma, mu1, sigma1, mu2, sigma2, p, d1, d2, d_min, d_max, exponent, scale,
        shape;
    const double* custom; /* [custom_len] */
    uint64_t custom_len;
} rcpg_distribution;

/* initialize_particles (initialize_particles.hpp:33-53, :90). Host arrays:
 * positions_out [N*ndim], diameters_out [N], box_out [ndim], walls_out [ndim];
 * box/walls inputs may be NULL with length 0. */
int32_t rcpg_initialize_particles(double phi, uint64_t N, int32_t ndim, const double* box,
                                  int32_t box_len, const int8_t* walls, int32_t walls_len,
                                  int32_t fix_height, const rcpg_distribution* dist,
                                  uint64_t seed, double* positions_out, double* diameters_out,
                                  double* box_out, int8_t* walls_out, double* scale_factor_out,
                                  double* phi_modifier_out, char* err, size_t errlen);

/* ---- analysis ------------------------------------------------------------- */

/* overlap_report of the reference's analysis package (rcptools/overlap.py:7-113):
 * candidates are the pairs i < j within 2 * max(D)/2 (minimum image on every
 * axis when box != NULL, as the reference does whatever the walls); a candidate
 * overlaps when (r_i + r_j) - |pos_i - pos_j| > 0. Host arrays in and out:
 * *n_candidate_out, *n_overlap_out; for the first min(n_overlap, capacity)
 * overlapping pairs in ascending (i, j): pairs_out[2m] = {i, j},
 * frac_sum_out[m] = overlap / (r_i + r_j), frac_min_out[m] = overlap / min(r_i, r_j).
 * RCPG_ENOSPC when n_overlap > capacity (the counts are still set). */
int32_t rcpg_overlap_report(uint64_t N, int32_t ndim, const double* positions, const double* diameters,
                            const double* box, uint64_t* n_candidate_out, uint64_t* n_overlap_out,
                            uint64_t capacity, uint32_t* pairs_out, double* frac_sum_out,
                            double* frac_min_out, int32_t device, char* err, size_t errlen);

/* ---- learned warm start (no counterpart in the reference) ----------------
 *
 * A fully connected network with layer widths widths[0..layers]: hidden
 * layers GELU(z) = 0.5 z (1 + erf(z / sqrt 2)), linear output. Parameters are
 * one FP32 array (the master copy) and a BF16 copy of the same layout: for
 * layer l, W_l [widths[l+1] x widths[l]] row-major, then b_l [widths[l+1]].
 * Inputs X [batch x widths[0]] and targets T [batch x widths[layers]] are
 * FP32, row-major. The kernels multiply BF16 weights and BF16 activations with
 * FP32 accumulation; pre-activations, gradients and the loss are FP32. All
 * pointers except `widths` are device pointers; `workspace` holds at least
 * rcpg_mlp_workspace_bytes(...) bytes, 256-byte aligned. Calls are
 * asynchronous on `stream`. */
uint64_t rcpg_mlp_param_count(const int32_t* widths, int32_t layers);
uint64_t rcpg_mlp_workspace_bytes(const int32_t* widths, int32_t layers, int32_t batch);
/* Y [batch x widths[layers]] = network(X). */
int32_t rcpg_mlp_forward(const int32_t* widths, int32_t layers, int32_t batch, const void* w_bf16,
                         const float* w_fp32, const float* X, float* Y, void* workspace,
                         uint64_t workspace_bytes, void* stream, char* err, size_t errlen);
/* One training step on the loss L = sum_{b,o} out_weight[o] (Y[b,o] - T[b,o])^2 / (batch * widths[layers])
 * (out_weight NULL = all ones): grad [param_count] = dL/dparams (FP32), and
 * loss_terms [batch x widths[layers]] (optional) the summands. With lr > 0 and
 * adam_m / adam_v non-NULL, Adam (beta 0.9 / 0.999, eps 1e-8, bias correction
 * at `step` >= 1) updates w_fp32 and refreshes w_bf16. */
int32_t rcpg_mlp_train_step(const int32_t* widths, int32_t layers, int32_t batch, float* w_fp32,
                            void* w_bf16, float* adam_m, float* adam_v, float* grad, const float* X,
                            const float* T, const float* out_weight, float lr, int32_t step,
                            float* loss_terms, void* workspace, uint64_t workspace_bytes, void* stream,
                            char* err, size_t errlen);
/* y = BF16(x), round to nearest even; n elements. */
int32_t rcpg_mlp_to_bf16(uint64_t n, const float* x, void* y, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* RCPG_H */
