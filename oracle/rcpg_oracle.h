/* CPU restatement of the reference packing engine's per-step kernels.
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker the parity tests compare the
 * CUDA path against; nothing in the product library links, loads or calls it.
 * Every function cites the reference code it restates (paths relative to the
 * reference project; ENG = python_code/python/src/core/rcp_generator.cpp).
 *
 * Parity pinning: each function is checked against the reference engine
 * itself (oracle/_ref, built from the reference sources) and against the
 * committed golden vectors in tests/golden (tests/test_oracle_pin.py).
 *
 * Layouts follow the reference: positions / forces / ADAM moments are flat
 * particle-major arrays x[i*ndim + d]; a half neighbour list is CSR
 * (counts[i], then the ids of row i, ascending, all > i).
 */
#ifndef RCPG_ORACLE_H
#define RCPG_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Pair shell t = min(max(median*1.02, Dmin*2.25), Dmax) * 0.5  (ENG:2846, :1210). */
double rcpo_t_shell(size_t N, const double* D);

/* Full-refresh half list: rows hold every j > i with
 *   MIC d2 < r_c^2,  r_c = (Di + Dj)*0.5 + t            for ndim <= 3 (ENG:3276-3297)
 *                    r_c = Di*0.5 + t + (double)(float)(Dj*0.5)  for ndim > 3 (ENG:1357)
 * Returns the total entry count; writes ids only while total <= cap. */
size_t rcpo_pairs_full(size_t N, size_t ndim, const double* x, const double* D,
                       const double* box, double t_shell, uint32_t* counts, uint32_t* ids,
                       size_t cap);

/* Soft-sphere energy/gradient + walls + containment + scalar finalise
 * (get_forces_nd_3, ENG:3597-4269), one-thread summation order.
 * scalars = {U, max_min_dist, Lc, Fmean, dkappa, count}. */
void rcpo_forces(size_t N, size_t ndim, const double* x, const double* D, const double* box,
                 const int8_t* walls, const uint32_t* counts, const uint32_t* ids, double mu,
                 double* F, double* scalars);

/* Mean |F_i| over |F_i|^2 > 1e-16, divided by sqrt(ndim) (compute_mean_force, ENG:769-803). */
double rcpo_mean_force(const double* F, size_t N, size_t ndim);

/* Fused particle ADAM + position step + single-box wrap (ENG:6410-6521,
 * scalar branch :6499-6519) with inv_b1 = 1/(1-beta1^t), inv_b2 = 1/(1-beta2^t). */
void rcpo_adam_step(size_t N, size_t ndim, const double* F, double alpha, double inv_b1,
                    double inv_b2, const double* box, double* m, double* v, double* x);

/* kappa ADAM moments (ENG:6354-6358) and kappa step (ENG:6405-6407).
 * state = {m_kappa, v_kappa, m_hat_kappa, v_hat_kappa}; returns the new kappa.
 * pow_b1 = beta1^t, pow_b2 = beta2^t. */
double rcpo_kappa_step(double* state, double dkappa, double pow_b1, double pow_b2, double alpha,
                       double kappa);

/* Growth-aware displacement refresh trigger (ENG:6104-6145). Updates D_last
 * (running min), theta_anchor, x_last for refreshed particles; refresh[k] in {0,1}.
 * Returns the number of refreshed particles. */
size_t rcpo_refresh_check(size_t N, size_t ndim, const double* x, double* x_last,
                          const double* D, double* D_last, double* theta_anchor,
                          double theta_new, uint8_t* refresh);

/* Spatial reorder permutation (ENG:4850-4948): 21-bit 3D Morton order for
 * ndim == 3 (ENG:1107-1160), x-column order otherwise (ENG:1081-1105); ties by index.
 * perm[k] = old index of the particle moved to slot k. */
void rcpo_reorder_perm(size_t N, size_t ndim, const double* x, const double* box, uint32_t* perm);

/* Per-row neighbour capacity (compute_pair_layout, ENG:4527-4566). */
void rcpo_pair_caps(size_t N, size_t ndim, const double* D, uint32_t neighbor_max, uint32_t* caps);

#ifdef __cplusplus
}
#endif

#endif
