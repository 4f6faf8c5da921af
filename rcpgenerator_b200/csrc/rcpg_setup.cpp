// Run setup of run_packing_observed (python_code/python/src/core/rcp_generator.cpp,
// "ENG", :4353-4990) on the host.
#include "rcpg_setup.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <numeric>
#include <stdexcept>
#include <thread>

namespace rcpg {

namespace {

constexpr double kPi = 3.14159265358979323846;

// fn(i) for i in [0, n) on up to 16 host threads (large n only). Used for
// per-particle terms that the caller then sums in index order, so results do
// not depend on the thread count.
template <typename Fn>
void parallel_for(std::size_t n, Fn fn) {
    unsigned T = std::thread::hardware_concurrency();
    T = T < 1 ? 1 : (T > 16 ? 16 : T);
    if (n < (std::size_t{1} << 16) || T == 1) {
        for (std::size_t i = 0; i < n; ++i) fn(i);
        return;
    }
    std::vector<std::thread> pool;
    const std::size_t chunk = (n + T - 1) / T;
    for (unsigned t = 0; t < T; ++t) {
        const std::size_t lo = t * chunk, hi = std::min(n, lo + chunk);
        if (lo >= hi) break;
        pool.emplace_back([lo, hi, &fn]() {
            for (std::size_t i = lo; i < hi; ++i) fn(i);
        });
    }
    for (auto& th : pool) th.join();
}

}  // namespace

double sphere_volume(double r, std::size_t ndim) {
    return std::pow(kPi, ndim / 2.0) * std::pow(r, static_cast<double>(ndim)) /
           std::tgamma(ndim / 2.0 + 1.0);
}

std::vector<double> scale_diameters_nd(const std::vector<double>& D, double phi_target,
                                       const std::vector<double>& box, std::size_t ndim,
                                       bool fix_height, double* factor_out) {
    double V_box = 1.0;
    for (double L : box) V_box *= L;
    // sphere_volume(Di * 0.5, ndim) per particle, its constant factors
    // evaluated once (same operations in the same order), summed in order
    const double c_pi = std::pow(kPi, ndim / 2.0), c_gamma = std::tgamma(ndim / 2.0 + 1.0);
    // the volumes go through the output buffer, which then takes the scaled diameters
    std::vector<double> out(D.size());
    parallel_for(D.size(), [&](std::size_t i) {
        out[i] = c_pi * std::pow(D[i] * 0.5, static_cast<double>(ndim)) / c_gamma;
    });
    double sumVol = 0.0;
    for (double v : out) sumVol += v;
    const double factor = fix_height ? std::pow(phi_target * V_box / sumVol, 1.0 / double(ndim - 1))
                                     : std::pow(phi_target * V_box / sumVol, 1.0 / double(ndim));
    parallel_for(D.size(), [&](std::size_t i) { out[i] = D[i] * factor; });
    if (factor_out) *factor_out = factor;
    return out;
}

std::vector<std::uint32_t> pair_caps(const std::vector<double>& D, int ndim,
                                     std::uint32_t neighbor_max) {
    const std::size_t N = D.size();
    std::vector<std::uint32_t> caps(N, 0);
    if (N == 0) return caps;
    double dmin = D[0];
    for (std::size_t i = 1; i < N; ++i)
        if (D[i] < dmin) dmin = D[i];
    if (dmin <= 0.0) dmin = 1.0;
    const double scaling = static_cast<double>(ndim) / 3.0;
    const double omega = 1.0 + static_cast<double>(ndim) / 6.0;
    parallel_for(N, [&](std::size_t i) {
        const double cap_d = scaling * (50.0 * std::pow(D[i] / dmin, omega) + static_cast<double>(neighbor_max));
        std::uint32_t cap = static_cast<std::uint32_t>(std::ceil(cap_d));
        if (static_cast<std::uint64_t>(cap) > N) cap = static_cast<std::uint32_t>(N);
        caps[i] = cap;
    });
    return caps;
}

// ---------------------------------------------------------------------------
// setup (ENG:4353-4990)
// ---------------------------------------------------------------------------
void check_run_input(const EngineInput& in) {
    const std::size_t nd = static_cast<std::size_t>(in.ndim);
    if (in.positions.size() != in.N * nd || in.diameters.size() != in.N)
        throw std::invalid_argument("rcpgenerator_b200: positions/diameters size mismatch");
    // the reference's own checks and texts (ENG:4440, :4446)
    if (!in.box.empty() && in.box.size() != nd) throw std::runtime_error("Error: --box length mismatch");
    if (!in.walls.empty() && in.walls.size() != nd)
        throw std::runtime_error("Error: --walls expects Ndim entries");
}

RunSetup prepare_run(const EngineInput& in) {
    RunSetup out;
    if (in.N == 0) throw std::invalid_argument("rcpgenerator_b200: no particles");
    if (in.ndim < 2 || in.ndim > kMaxDim)
        throw std::invalid_argument("rcpgenerator_b200: Ndim must be in [2, 8]");
    if (in.N >= 0xFFFFFFF0ull) throw std::invalid_argument("rcpgenerator_b200: N too large");
    const std::size_t N = in.N, nd = static_cast<std::size_t>(in.ndim);
    out.N = in.N;
    out.ndim = in.ndim;
    std::vector<double> x = in.positions;
    std::vector<double> D = in.diameters;
    if (x.size() != N * nd || D.size() != N)
        throw std::invalid_argument("rcpgenerator_b200: positions/diameters size mismatch");

    // refresh-trigger scale from the caller's diameters (ENG:4401-4430)
    double trigger_scale;
    double med_in;  // median of the caller's diameters (rank N/2)
    {
        double dmx = 0.0, dmn = std::numeric_limits<double>::max();
        for (double dv : D) {
            if (dv > dmx) dmx = dv;
            if (dv < dmn) dmn = dv;
        }
        std::vector<double> Ds = D;
        std::nth_element(Ds.begin(), Ds.begin() + Ds.size() / 2, Ds.end());
        const double med = Ds[Ds.size() / 2];
        med_in = med;
        const double t_shell = std::min(std::max(med * 1.02, dmn * 2.25), dmx) * 0.5;
        const double rho = t_shell / dmn;
        trigger_scale = std::min(1.28 * rho, 1.9);
    }

    check_run_input(in);
    std::vector<double> box = in.box;
    std::vector<std::int8_t> walls = in.walls;
    if (box.empty()) box.assign(nd, 1.0);
    if (walls.empty()) walls.assign(nd, 0);

    double phi_modifier = 1;
    if (walls[0] < 0) {
        if (walls[0] == -1) walls[0] = -2;
        for (std::size_t k = 1; k < static_cast<std::size_t>(-walls[0]) && k < nd; ++k) {
            walls[k] = -1;
            box[k] = box[0];
        }
        phi_modifier = sphere_volume(1 / 2., static_cast<std::size_t>(-walls[0]));
    }
    if (in.fix_height) box[nd - 1] = box[nd - 1] * D[0];

    double phi = 0.025;
    if (in.has_initial_phi_target) phi = in.initial_phi_target;
    else if (nd == 2) phi = 0.575;
    else if (nd == 3) phi = 0.33;
    else if (nd == 4) phi = 0.15;
    else if (nd == 5) phi = 0.10;
    else if (nd > 5) phi = 0.10 / std::pow(2, (nd - 4));
    double factor = 1.0;  // diameter scale of the start (1 with fix_diameter)
    if (!in.fix_diameter) {
        std::vector<double> Ds = scale_diameters_nd(D, phi * phi_modifier, box, nd, in.fix_height, &factor);
        if (in.fix_height) {
            box[nd - 1] = box[nd - 1] * factor;
            for (std::size_t i = 0; i < N; ++i) x[i * nd + (nd - 1)] = x[i * nd + (nd - 1)] * factor;
        }
        D = std::move(Ds);
    }
    const double coeff = std::pow(kPi, nd / 2.0) / std::tgamma(nd / 2.0 + 1.0);
    std::vector<double> terms(N);
    parallel_for(N, [&](std::size_t i) { terms[i] = coeff * std::pow(D[i] / 2.0, static_cast<double>(nd)); });
    double current_volume = 0.0;
    for (double v : terms) current_volume += v;
    double box_volume = std::accumulate(box.begin(), box.end(), 1.0, std::multiplies<double>());
    phi = current_volume / box_volume / phi_modifier;
    const double Dmin = *std::min_element(D.begin(), D.end());

    std::uint32_t neighbor_max = in.neighbor_max;
    if (neighbor_max == 0) {
        static const std::uint32_t table[4] = {300, 750, 5500, 5500};
        neighbor_max = table[std::min<std::size_t>(nd - 2, 3)];
    }
    out.neighbor_max = neighbor_max;
    // per-row capacity of the reference layout (ENG:4527-4566): the overflow
    // threshold of its own-write rows, reported with the reference's message.
    out.caps = pair_caps(D, static_cast<int>(nd), neighbor_max);
    // step cap and rung-1 deadline (ENG:4713-4737, :5862-5891), RCP_SPEED=quick
    std::uint64_t rung1_deadline;
    {
        double dl = 2.0 * 4000.0 + 9.0 * std::sqrt(static_cast<double>(N) * static_cast<double>(nd)) - 2000.0;
        if (dl < 1500.0) dl = 1500.0;
        rung1_deadline = static_cast<std::uint64_t>(dl);
        // a warm start may shorten (or lengthen) the growth rung; no reference counterpart
        if (in.growth_steps > 0) rung1_deadline = in.growth_steps;
    }
    std::uint64_t step_cap;
    if (in.max_steps > 0) {
        step_cap = in.max_steps;
    } else {
        double rung1 = 2.0 * 4000.0 + 9.0 * std::sqrt(static_cast<double>(N) * static_cast<double>(nd)) - 2000.0;
        if (rung1 < 1500.0) rung1 = 1500.0;
        const std::uint64_t formula = static_cast<std::uint64_t>(rung1 * static_cast<double>(2 + 3));
        step_cap = std::max<std::uint64_t>(60000, formula);
    }
    double alpha = 0.005, alpha_max = 0.005;
    if (nd == 3) alpha = alpha_max = 0.0045;
    if (nd == 4) alpha = alpha_max = 0.0035;
    if (nd >= 5) alpha = alpha_max = 0.0025;

    // D0 statistics (ENG:4800-4838); D is not used after this point
    out.D0 = std::move(D);
    const std::vector<double>& D0_ = out.D0;
    double D0min = D0_[0], S = 0.0, D0max = 0.0;
    for (std::size_t i = 0; i < N; ++i) {
        if (D0_[i] < D0min) D0min = D0_[i];
        double r = D0_[i] * 0.5, rN = 1.0;
        for (std::size_t k = 0; k < nd; ++k) rN *= r;
        S += rN;
        if (D0_[i] > D0max) D0max = D0_[i];
    }
    // the median of D0 = D * factor: a positive scale keeps every rank, and
    // the element at rank N/2 was scaled by the same rounded multiplication
    const double D0med = in.fix_diameter ? med_in : med_in * factor;

    Controller& c = out.c;
    std::memset(&c, 0, sizeof(c));
    c.N = N;
    c.ndim = static_cast<int>(nd);
    c.alpha_max = alpha_max;
    c.phi_modifier = phi_modifier;
    c.coeff = coeff;
    c.trigger_scale = trigger_scale;
    c.step_cap = step_cap;
    c.rung1_deadline = rung1_deadline;
    c.reorder_interval = in.reorder_interval;
    c.fix_height = in.fix_height ? 1 : 0;
    c.has_target_phi = in.has_target_phi ? 1 : 0;
    c.target_phi = in.target_phi;
    c.D0_min = D0min;
    c.D0_max = D0max;
    c.D0_med = D0med;
    c.S_D0 = S;
    c.t = 0.0;
    c.alpha = alpha;
    c.mu = in.has_mu_override ? in.mu_override : 2.5e-4;
    c.mu_flag = 1;
    c.mu_change = 0.0;
    c.phi = phi;
    c.phi_max = 0.0;
    c.kappa = 1.0;
    c.kappa_D = 1.0;
    c.kappa_D_prev = 1.0;
    c.Dmin = Dmin;
    for (std::size_t d = 0; d < nd; ++d) c.box[d] = box[d];
    double bv = 1.0;
    for (std::size_t d = 0; d < nd; ++d) bv *= box[d];
    c.box_volume = bv;
    c.runtime_fix_diameter = in.fix_diameter ? 1 : 0;
    c.theta = Dmin * 0.25 * trigger_scale;
    c.mu_eff = c.mu;
    c.t_shell = shell_of(D0min, D0med, D0max);
    c.Dmax_cur = D0max;
    c.fix_height_scale = 1.0;

    out.walls = walls;
    out.x = std::move(x);
    return out;
}


}  // namespace rcpg
