// Test infrastructure only (the checker, never the product): a flat-pointer C
// shim over the reference engine's own exported kernels, compiled from the
// reference sources by oracle/Makefile into oracle/_ref/librcpg_ref.so.
//
// Every entry point calls the reference implementation itself; the only code
// here is layout conversion (CSR <-> the reference's slotted pair rows).
//
// Reference functions used (python_code/python/src/core/rcp_generator.cpp):
//   get_pairs_kdtree      :2758-3526  (run_packing's pair backend for Ndim <= 3)
//   get_pairs_nd_3        :1198-1478  (pair backend for Ndim > 3, dispatch :3533-3560)
//   get_forces_nd_3       :3597-4269
//   compute_mean_force    :769-803
//   adam_update           :4271-4335  (+ position step / wrap :6522-6573)
//   scale_diameters_nd    :1162-1196
// and the pair-capacity formula of compute_pair_layout :4527-4566.
#include "rcpgenerator/rcp_generator.hpp"

#include <omp.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

namespace rcpgenerator {
// External linkage in the reference TU but not declared in its header.
void get_pairs_kdtree(
    std::size_t N, std::size_t Ndim, const double* x, const std::vector<double>& D,
    const std::vector<double>& box, const std::vector<std::int8_t>& walls,
    const std::vector<std::uint32_t>& refresh, const std::uint32_t* max_neighbors_per_particle,
    const std::uint64_t* pair_offsets, std::uint32_t* pairs_data,
    std::uint32_t* out_max_observed, std::uint32_t* out_min_observed,
    double* packed_d0, const double* D0_data);
}  // namespace rcpgenerator

namespace {

void put_err(char* err, std::size_t errlen, const std::string& msg) {
    if (err && errlen) {
        std::snprintf(err, errlen, "%s", msg.c_str());
    }
}

// Per-row capacity exactly as compute_pair_layout (rcp_generator.cpp:4527-4566).
void pair_layout(std::size_t N, std::size_t Ndim, const double* D, std::uint32_t neighbor_max,
                 std::vector<std::uint32_t>& caps, std::vector<std::uint64_t>& offsets) {
    static const std::uint32_t table[4] = {300, 750, 5500, 5500};
    if (neighbor_max == 0) {
        std::size_t idx = (Ndim >= 2 ? std::min<std::size_t>(Ndim - 2, 3) : 0);
        neighbor_max = table[idx];
    }
    double dmin = D[0];
    for (std::size_t i = 1; i < N; ++i) if (D[i] < dmin) dmin = D[i];
    if (dmin <= 0.0) dmin = 1.0;
    const std::uint32_t base = neighbor_max;
    const double scaling = static_cast<double>(Ndim) / 3.0;
    const double omega = 1.0 + static_cast<double>(Ndim) / 6.0;
    caps.assign(N, 0);
    offsets.assign(N + 1, 0);
    std::uint64_t off = 0;
    for (std::size_t i = 0; i < N; ++i) {
        const double ratio = D[i] / dmin;
        const double cap_d = scaling * (50.0 * std::pow(ratio, omega) + static_cast<double>(base));
        std::uint32_t cap = static_cast<std::uint32_t>(std::ceil(cap_d));
        if (static_cast<std::uint64_t>(cap) > N) cap = static_cast<std::uint32_t>(N);
        caps[i] = cap;
        offsets[i] = off;
        off += static_cast<std::uint64_t>(cap) + 1;
    }
    offsets[N] = off;
}

}  // namespace

extern "C" {

int ref_set_num_threads(int n) {
    if (n < 1) return -1;
    omp_set_num_threads(n);
    return 0;
}

int ref_get_num_threads(void) { return omp_get_max_threads(); }

// Full-refresh half neighbour list (rows hold j > i, ascending), built by the
// backend run_packing dispatches to. counts[N]; ids packed row after row.
// Returns 0, 1 (ids_cap too small; *total_out holds the need) or -1 (engine
// error, message in err).
int ref_pairs_full(std::size_t N, std::size_t Ndim, const double* x, const double* D,
                   const double* box, const std::int8_t* walls, std::uint32_t neighbor_max,
                   std::uint32_t* counts, std::uint32_t* ids, std::size_t ids_cap,
                   std::size_t* total_out, char* err, std::size_t errlen) {
    try {
        std::vector<double> Dv(D, D + N);
        std::vector<double> bv(box, box + Ndim);
        std::vector<std::int8_t> wv(Ndim, 0);
        if (walls) wv.assign(walls, walls + Ndim);
        std::vector<std::uint32_t> caps;
        std::vector<std::uint64_t> offs;
        pair_layout(N, Ndim, D, neighbor_max, caps, offs);
        std::vector<std::uint32_t> data(offs[N], 0u);
        std::vector<std::uint32_t> refresh(N, 1u);
        if (Ndim <= 3) {
            // A one-particle call first: the kd-tree keeps function-static
            // caches keyed on N (D-stat indices, tree); changing N forces the
            // full recompute that a fresh run_packing would see.
            double x1[3] = {0.0, 0.0, 0.0};
            std::vector<double> D1(1, D[0]);
            std::vector<std::uint32_t> r1(1, 1u), c1(1, 1u);
            std::vector<std::uint64_t> o1 = {0, 2};
            std::uint32_t d1[2] = {0, 0};
            rcpgenerator::get_pairs_kdtree(1, Ndim, x1, D1, bv, wv, r1, c1.data(), o1.data(), d1,
                                           nullptr, nullptr, nullptr, nullptr);
            rcpgenerator::get_pairs_kdtree(N, Ndim, x, Dv, bv, wv, refresh, caps.data(),
                                           offs.data(), data.data(), nullptr, nullptr, nullptr,
                                           nullptr);
        } else {
            rcpgenerator::get_pairs_nd_3(N, Ndim, x, Dv, bv, wv, refresh, caps.data(), offs.data(),
                                         data.data(), nullptr, nullptr, nullptr, nullptr);
        }
        std::size_t total = 0;
        for (std::size_t i = 0; i < N; ++i) total += data[offs[i]];
        if (total_out) *total_out = total;
        if (total > ids_cap) return 1;
        std::size_t k = 0;
        for (std::size_t i = 0; i < N; ++i) {
            const std::uint32_t c = data[offs[i]];
            counts[i] = c;
            for (std::uint32_t q = 1; q <= c; ++q) ids[k++] = data[offs[i] + q];
        }
        return 0;
    } catch (const std::exception& e) {
        put_err(err, errlen, e.what());
        return -1;
    }
}

// get_forces_nd_3 on a half list given as CSR (counts + packed ids).
// scalars_out = {U, max_min_dist, Lc, Fmean, dkappa}.
int ref_forces(std::size_t N, std::size_t Ndim, const double* x, const double* D,
               const double* box, const std::int8_t* walls, const std::uint32_t* counts,
               const std::uint32_t* ids, double mu, double* F_out, double* scalars_out) {
    std::vector<std::uint64_t> offs(N + 1, 0);
    for (std::size_t i = 0; i < N; ++i) offs[i + 1] = offs[i] + counts[i] + 1;
    std::vector<std::uint32_t> data(offs[N], 0u);
    std::size_t k = 0;
    for (std::size_t i = 0; i < N; ++i) {
        data[offs[i]] = counts[i];
        for (std::uint32_t q = 1; q <= counts[i]; ++q) data[offs[i] + q] = ids[k++];
    }
    std::vector<double> Dv(D, D + N);
    std::vector<double> bv(box, box + Ndim);
    std::vector<std::int8_t> wv(Ndim, 0);
    if (walls) wv.assign(walls, walls + Ndim);
    std::vector<std::vector<double>> min_dist;
    std::vector<std::size_t> z(N, 0);
    double U = 0, maxov = 0, Lc = 0, Fmean = 0, dkappa = 0;
    rcpgenerator::get_forces_nd_3(data.data(), offs.data(), x, N, Ndim, Dv, bv, wv, F_out, U,
                                  min_dist, maxov, Lc, Fmean, mu, dkappa, z);
    scalars_out[0] = U;
    scalars_out[1] = maxov;
    scalars_out[2] = Lc;
    scalars_out[3] = Fmean;
    scalars_out[4] = dkappa;
    return 0;
}

double ref_mean_force(const double* F, std::size_t N, std::size_t Ndim) {
    std::vector<std::size_t> z;
    return rcpgenerator::compute_mean_force(F, N, Ndim, 0.0, z);
}

// One particle ADAM step at bias-correction counter t followed by the
// position step and the single-box wrap, i.e. the unfused path of
// run_packing_observed (adam_update + :6522-6573), which the fused pass
// (:6410-6521) reproduces element for element.
// kappa_state = {m_kappa, v_kappa, m_hat_kappa, v_hat_kappa} (in/out).
int ref_adam_step(std::size_t N, std::size_t Ndim, const double* F, double dkappa,
                  std::size_t t, double alpha, const double* box, double* m, double* v,
                  double* x, double* kappa_state) {
    const std::size_t total = N * Ndim;
    std::vector<double> v_update(total), m_hat(total), v_hat(total);
    std::vector<std::vector<double>> v_max, a, v_verlet, a_old;
    double m_k = kappa_state[0], v_k = kappa_state[1], vu_k = 0.0;
    double mh_k = kappa_state[2], vh_k = kappa_state[3];
    rcpgenerator::adam_update("ADAM", N, Ndim, F, dkappa, 0.9, 0.999, t, 0.1, 2.0, m, v, v_max,
                              v_update.data(), m_hat.data(), v_hat.data(), a, v_verlet, a_old, m_k,
                              v_k, vu_k, mh_k, vh_k);
    for (std::size_t k = 0; k < total; ++k) {
        x[k] -= alpha * m_hat[k] / (std::sqrt(v_hat[k]) + 1e-8);
    }
    for (std::size_t i = 0; i < N; ++i) {
        for (std::size_t d = 0; d < Ndim; ++d) {
            double val = x[i * Ndim + d];
            const double L = box[d];
            if (val >= L) val -= L;
            else if (val < 0) val += L;
            x[i * Ndim + d] = val;
        }
    }
    kappa_state[0] = m_k;
    kappa_state[1] = v_k;
    kappa_state[2] = mh_k;
    kappa_state[3] = vh_k;
    return 0;
}

double ref_scale_diameters(const double* D, std::size_t N, double phi_target, const double* box,
                           std::size_t Ndim, int fix_height, double* D_out) {
    std::vector<double> Dv(D, D + N);
    std::vector<double> bv(box, box + Ndim);
    auto res = rcpgenerator::scale_diameters_nd(Dv, phi_target, bv, Ndim, fix_height != 0);
    std::memcpy(D_out, res.first.data(), N * sizeof(double));
    return res.second;
}

}  // extern "C"
