// Initial configurations for Packing(...): seeded diameter distributions and
// random sequential addition (RSA) on a fine cell grid.
//
// Restates initialize_particles of the reference
// (python_code/python/src/core/initialize_particles.cpp, "INI"): the same
// libstdc++ engines (std::mt19937 for diameters, std::mt19937_64 for
// placement) and distributions are drawn in the same order, so with the same
// standard library the outputs are identical value for value.
#include "rcpg_init.h"

#include <algorithm>
#include <cmath>
#include <numeric>
#include <random>
#include <stdexcept>

namespace rcpg {

namespace {

constexpr double kPi = 3.14159265358979323846;

double ball_volume(double r, std::size_t ndim) {
    return std::pow(kPi, ndim / 2.0) * std::pow(r, static_cast<double>(ndim)) / std::tgamma(ndim / 2.0 + 1.0);
}

// Linear map of the realised [min, max] onto [lo, hi] (INI:58-66, :83-93, :107-116).
void stretch_to(std::vector<double>& D, double lo, double hi) {
    const double mn = *std::min_element(D.begin(), D.end());
    const double mx = *std::max_element(D.begin(), D.end());
    if (mx > mn + 1e-12) {
        for (double& v : D) v = lo + (v - mn) * (hi - lo) / (mx - mn);
    } else {
        std::fill(D.begin(), D.end(), lo);
    }
}

}  // namespace

// INI:17-130
std::vector<double> draw_diameters(std::size_t N, const DistSpec& dist, std::mt19937& rng) {
    std::vector<double> D(N);
    const std::string& t = dist.type;
    if (t == "mono") {
        std::fill(D.begin(), D.end(), dist.d);
    } else if (t == "gaussian") {
        std::normal_distribution<> nd(dist.mu, dist.sigma);
        for (auto& v : D) v = std::abs(nd(rng));
    } else if (t == "bigaussian") {
        const std::size_t n1 = static_cast<std::size_t>(std::round(dist.p * N));
        std::normal_distribution<> g1(dist.mu1, dist.sigma1), g2(dist.mu2, dist.sigma2);
        for (std::size_t i = 0; i < n1; ++i) D[i] = std::abs(g1(rng));
        for (std::size_t i = n1; i < N; ++i) D[i] = std::abs(g2(rng));
        std::shuffle(D.begin(), D.end(), rng);
    } else if (t == "bidisperse") {
        const std::size_t n1 = static_cast<std::size_t>(std::round(dist.p * N));
        for (std::size_t i = 0; i < n1; ++i) D[i] = dist.d1;
        for (std::size_t i = n1; i < N; ++i) D[i] = dist.d2;
        std::shuffle(D.begin(), D.end(), rng);
    } else if (t == "lognormal") {
        std::lognormal_distribution<> ld(dist.mu, dist.sigma);
        for (auto& v : D) v = std::clamp(ld(rng), 0.0025, 30.0);
    } else if (t == "flat") {
        std::uniform_real_distribution<> ud(dist.d_min, dist.d_max);
        for (auto& v : D) v = ud(rng);
        stretch_to(D, dist.d_min, dist.d_max);
    } else if (t == "powerlaw") {
        std::uniform_real_distribution<> ud(0.0, 1.0);
        const double a = dist.exponent + 1.0;
        for (std::size_t i = 0; i < N; ++i) {
            const double u = ud(rng);
            if (std::abs(a) < 1e-12) {
                D[i] = dist.d_min * std::exp(u * std::log(dist.d_max / dist.d_min));
            } else {
                const double top = std::pow(dist.d_max, a) - std::pow(dist.d_min, a);
                D[i] = std::pow(top * u + std::pow(dist.d_min, a), 1.0 / a);
            }
        }
        stretch_to(D, dist.d_min, dist.d_max);
    } else if (t == "exponential") {
        const double lambda = -std::log(0.5) / (dist.d_max - dist.d_min);
        std::uniform_real_distribution<> ud(0.0, 1.0);
        for (std::size_t i = 0; i < N; ++i) {
            const double u = ud(rng);
            D[i] = dist.d_min - (1.0 / lambda) * std::log(1.0 - u);
            if (D[i] > dist.d_max) D[i] = dist.d_max;
        }
        stretch_to(D, dist.d_min, dist.d_max);
    } else if (t == "weibull") {
        std::weibull_distribution<> wd(dist.shape, dist.scale);
        for (auto& v : D) v = wd(rng);
    } else if (t == "custom") {
        if (dist.custom.size() != N) throw std::runtime_error("custom distribution needs N entries");
        D = dist.custom;
    } else {
        // The reference prints and calls std::exit(1) here (INI:124-127); a
        // library reports it instead.
        throw std::invalid_argument("Unsupported distribution: " + t);
    }
    return D;
}

// RSA with largest-first insertion and halo registration (INI:184-343).
void place_rsa(std::vector<double>& x, const std::vector<double>& D, const std::vector<double>& box,
               const std::vector<std::int8_t>& walls, std::uint64_t seed) {
    const std::size_t N = D.size(), nd = box.size();
    if (N == 0) return;
    double Dmax = 0.0;
    for (double v : D)
        if (v > Dmax) Dmax = v;
    if (Dmax <= 0.0) Dmax = 1e-12;
    double box_vol = 1.0;
    for (std::size_t d = 0; d < nd; ++d) box_vol *= box[d];
    double edge = std::pow(box_vol / std::max(1.0, static_cast<double>(N) / 2.0), 1.0 / static_cast<double>(nd));
    if (!(edge > 0.0)) edge = Dmax;
    std::vector<long> ncell(nd);
    std::vector<double> csize(nd);
    std::vector<std::size_t> stride(nd, 1);
    std::size_t total = 1;
    for (std::size_t d = 0; d < nd; ++d) {
        long nc = std::lround(box[d] / edge);
        if (nc < 1) nc = 1;
        ncell[d] = nc;
        csize[d] = box[d] / static_cast<double>(nc);
        total *= static_cast<std::size_t>(nc);
    }
    for (std::size_t d = 1; d < nd; ++d) stride[d] = stride[d - 1] * static_cast<std::size_t>(ncell[d - 1]);
    // cell -> registered particles, as a CSR-free vector of vectors
    std::vector<std::vector<std::uint32_t>> cells(total);
    const bool sph = walls[0] < 0;
    const std::size_t ksph = sph ? static_cast<std::size_t>(-walls[0]) : 0;
    const double rsph = box[0] * 0.5;
    std::mt19937_64 rng{seed ? seed : 0x9E3779B97F4A7C15ULL};
    std::uniform_real_distribution<double> ud(0.0, 1.0);
    auto wrap_axis = [&](long c, std::size_t d, long& out) -> bool {
        if (walls[d] == 0) {
            const long n = ncell[d];
            if (n == 1) {
                out = 0;
                return true;
            }
            c %= n;
            if (c < 0) c += n;
            out = c;
            return true;
        }
        if (c < 0 || c >= ncell[d]) return false;
        out = c;
        return true;
    };
    std::vector<double> xt(nd);
    std::vector<long> ci(nd), hw(nd);
    const std::size_t max_attempts = std::size_t{1} << 22;
    for (std::size_t n = 0; n < N; ++n) {
        const double Dc = D[n];
        std::size_t attempts = 0;
        for (;;) {
            if (++attempts > max_attempts)
                throw std::runtime_error(
                    "initializer: could not place a non-overlapping particle "
                    "(phi_init too high for random sequential addition; "
                    "lower the initial packing fraction)");
            for (std::size_t d = 0; d < nd; ++d) {
                if (walls[d] == 0) xt[d] = ud(rng) * box[d];
                else xt[d] = Dc * 0.5 + ud(rng) * (box[d] - Dc);
            }
            if (sph) {
                double s = 0.0;
                for (std::size_t d = 0; d < ksph; ++d) {
                    const double q = xt[d] - rsph;
                    s += q * q;
                }
                if (s > (rsph - Dc * 0.5) * (rsph - Dc * 0.5)) continue;
            }
            for (std::size_t d = 0; d < nd; ++d) {
                long c = static_cast<long>(xt[d] / csize[d]);
                if (c < 0) c = 0;
                if (c >= ncell[d]) c = ncell[d] - 1;
                ci[d] = c;
            }
            std::size_t center = 0;
            for (std::size_t d = 0; d < nd; ++d) center += static_cast<std::size_t>(ci[d]) * stride[d];
            bool ok = true;
            for (std::uint32_t idx : cells[center]) {
                double s = 0.0;
                for (std::size_t d = 0; d < nd; ++d) {
                    double q = xt[d] - x[idx * nd + d];
                    if (walls[d] == 0) q -= box[d] * std::nearbyint(q / box[d]);
                    s += q * q;
                }
                const double r = 0.5 * (D[idx] + Dc);
                if (s <= r * r) {
                    ok = false;
                    break;
                }
            }
            if (!ok) continue;
            for (std::size_t d = 0; d < nd; ++d) x[n * nd + d] = xt[d];
            std::size_t halo = 1;
            for (std::size_t d = 0; d < nd; ++d) {
                long h = static_cast<long>(std::ceil(Dc / csize[d])) + 1;
                if (h > ncell[d]) h = ncell[d];
                hw[d] = h;
                halo *= static_cast<std::size_t>(2 * h + 1);
            }
            for (std::size_t m = 0; m < halo; ++m) {
                std::size_t t = m, hidx = 0;
                bool valid = true;
                double md2 = 0.0;
                for (std::size_t d = 0; d < nd; ++d) {
                    const long span = 2 * hw[d] + 1;
                    const long o = static_cast<long>(t % static_cast<std::size_t>(span)) - hw[d];
                    t /= static_cast<std::size_t>(span);
                    double gap = 0.0;
                    if (o > 0) gap = static_cast<double>(ci[d] + o) * csize[d] - xt[d];
                    else if (o < 0) gap = xt[d] - static_cast<double>(ci[d] + o + 1) * csize[d];
                    if (gap > 0.0) md2 += gap * gap;
                    long wc;
                    if (!wrap_axis(ci[d] + o, d, wc)) {
                        valid = false;
                        break;
                    }
                    hidx += static_cast<std::size_t>(wc) * stride[d];
                }
                if (valid && md2 < Dc * Dc) cells[hidx].push_back(static_cast<std::uint32_t>(n));
            }
            break;
        }
    }
}

// INI:399-474
InitResult initialize_particles(const InitSpec& spec) {
    double phi = spec.phi;
    const std::size_t N = spec.N, nd = spec.ndim;
    std::vector<double> box = spec.box;
    std::vector<std::int8_t> walls = spec.walls;
    if (nd < 2) throw std::runtime_error("--Ndim must be >=2");
    if (walls.size() != nd) walls.resize(nd, 0);
    if (box.empty()) box.assign(nd, 1.0);
    if (phi <= 0 || phi >= 1 || N == 0) throw std::runtime_error("Missing or invalid phi/N");
    if (box.size() != nd) throw std::runtime_error("Error: --box length mismatch");
    const double Llast = box[0];
    double h = 1;
    if (spec.fix_height) {
        h = box[nd - 1];
        box[nd - 1] = box[0];
    }
    double phi_modifier = 1.0;
    if (walls[0] < 0) phi_modifier = ball_volume(1 / 2., static_cast<std::size_t>(-walls[0]));
    std::mt19937 rng{static_cast<std::mt19937::result_type>(spec.seed)};
    std::vector<double> raw = draw_diameters(N, spec.dist, rng);
    // scale to phi*phi_modifier (the initializer's own scale_diameters_nd, INI:132-150)
    double V_box = 1.0;
    for (double L : box) V_box *= L;
    double sumVol = 0.0;
    for (double Di : raw) {
        const double r = Di * 0.5;
        const double unit = std::pow(kPi, nd / 2.0) / std::tgamma(nd / 2.0 + 1.0);
        sumVol += unit * std::pow(r, double(nd));
    }
    const double factor = std::pow(phi * phi_modifier * V_box / sumVol, 1.0 / double(nd));
    std::vector<double> Ds = raw;
    for (auto& v : Ds) v *= factor;
    std::vector<std::size_t> idx(N);
    std::iota(idx.begin(), idx.end(), 0);
    std::sort(idx.begin(), idx.end(), [&](std::size_t a, std::size_t b) { return Ds[a] > Ds[b]; });
    std::vector<double> D(N);
    for (std::size_t i = 0; i < N; ++i) D[i] = Ds[idx[i]];
    if (spec.fix_height) {
        const double s = std::pow(h * D[0] / Llast, 1.0 / (nd - 1));
        const double eps = std::pow(s, nd);
        for (auto& v : D) v *= s;
        box[nd - 1] *= eps;
    }
    InitResult r;
    r.positions.assign(N * nd, 0.0);
    place_rsa(r.positions, D, box, walls, spec.seed);
    r.diameters = std::move(D);
    r.box = std::move(box);
    r.walls = std::move(walls);
    r.scale_factor = factor;
    r.phi_modifier = phi_modifier;
    return r;
}

}  // namespace rcpg
