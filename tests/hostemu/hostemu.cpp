// Test infrastructure: a CPU emulation of the engine's exact mode, built from
// the product's own per-particle arithmetic (rcpg_core.h), controller
// (rcpg_schedule.h) and run setup (rcpg_setup.cpp), with a brute-force
// neighbour list. The CPU test suite runs it against the reference engine to
// pin the schedule and the per-particle arithmetic before any GPU run.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>

#include "rcpg_core.h"
#include "rcpg_device.h"
#include "rcpg_noalloc_plan.h"
#include "rcpg_schedule.h"
#include "rcpg_setup.h"

using namespace rcpg;

namespace {

template <int ND>
struct Emu {
    std::uint64_t N;
    RunSetup s;
    Controller& c;
    Geometry g{};
    std::vector<double> x, D0, F, m, v, x_last;
    std::vector<std::uint64_t> origin;
    std::vector<std::vector<std::uint32_t>> rows;
    std::vector<double> hphi, hforce, henergy, hmaxov, hmu, halpha;
    std::vector<std::int8_t> hflag;
    Histories h{};
    double kappa_min = 1.0;
    double theta = 0.0;
    std::uint64_t builds = 0;
    bool adam_pending = false;
    double a_alpha = 0, a_ib1 = 0, a_ib2 = 0;
    double a_box[kMaxDim];

    explicit Emu(RunSetup&& rs) : N(rs.N), s(std::move(rs)), c(s.c) {
        x = s.x;
        D0 = s.D0;
        F.assign(N * ND, 0.0);
        m.assign(N * ND, 0.0);
        v.assign(N * ND, 0.0);
        x_last = x;
        origin.resize(N);
        std::iota(origin.begin(), origin.end(), 0ull);
        const std::size_t hs = c.step_cap + 1;
        hphi.assign(hs, 0.0); hforce.assign(hs, 0.0); henergy.assign(hs, 0.0);
        hmaxov.assign(hs, 0.0); hmu.assign(hs, 0.0); halpha.assign(hs, 0.0); hflag.assign(hs, 0);
        h = Histories{hphi.data(), hforce.data(), henergy.data(), hmaxov.data(), hmu.data(),
                      halpha.data(), hflag.data()};
        g.ndim = ND;
        g.circle_k = s.walls[0] < 0 ? -s.walls[0] : 0;
        g.any_flat_wall = 0;
        for (int d = 0; d < ND; ++d) {
            g.walls[d] = s.walls[d];
            if (s.walls[d] == 1) g.any_flat_wall = 1;
        }
        set_box(c.box);
        theta = c.theta;
    }
    void set_box(const double* b) {
        for (int d = 0; d < ND; ++d) {
            g.box[d] = b[d];
            g.inv_box[d] = 1.0 / b[d];
        }
    }
    void build(double kap, double t_shell) {
        rows.assign(N, {});
        for (std::uint64_t i = 0; i < N; ++i) {
            const double Di = D0[i] * kap;
            for (std::uint64_t j = 0; j < N; ++j) {
                if (j == i) continue;
                const double Dj = D0[j] * kap;
                const bool ok = (ND <= 3 || j > i)
                                    ? in_shell<ND>(&x[i * ND], &x[j * ND], Di, Dj, g.box, g.inv_box, t_shell)
                                    : in_shell<ND>(&x[i * ND], &x[j * ND], Dj, Di, g.box, g.inv_box, t_shell);
                if (ok) rows[i].push_back(static_cast<std::uint32_t>(j));
            }
        }
        x_last = x;
        kappa_min = kap;
        ++builds;
    }
    ForceSums forces(double kap) {
        ForceSums s;
        sums_zero(s);
        std::vector<std::vector<PairTerms>> terms(N);
        for (std::uint64_t i = 0; i < N; ++i) {
            double fi[ND];
            for (int d = 0; d < ND; ++d) fi[d] = 0.0;
            const double Di = D0[i] * kap;
            for (std::uint32_t j : rows[i]) {
                PairTerms pt;
                if (!pair_force<ND>(&x[i * ND], Di, &x[j * ND], D0[j] * kap, g, fi, pt)) continue;
                if (j > i) terms[i].push_back(pt);
            }
            double wu = 0, wd = 0, wf = 0;
            unsigned long long wc = 0;
            wall_forces<ND>(&x[i * ND], Di, g, fi, wu, wd, wf, wc);
            for (int d = 0; d < ND; ++d) F[i * ND + d] = fi[d];
        }
        for (std::uint64_t i = 0; i < N; ++i)
            for (const PairTerms& pt : terms[i]) {
                s.pair_U = xadd(s.pair_U, pt.U);
                s.pair_count += 1;
                s.pair_Lc = xadd(s.pair_Lc, pt.Lc);
                if (pt.U > s.pair_maxov) s.pair_maxov = pt.U;
                s.pair_dk = xadd(s.pair_dk, pt.dk);
                s.pair_Fm = xadd(s.pair_Fm, pt.Fm);
            }
        for (std::uint64_t i = 0; i < N; ++i) {
            double fd[ND];
            for (int d = 0; d < ND; ++d) fd[d] = 0.0;
            wall_forces<ND>(&x[i * ND], D0[i] * kap, g, fd, s.pair_U, s.pair_dk, s.pair_Fm, s.wall_count);
        }
        for (std::uint64_t i = 0; i < N; ++i) s.sum_D = xadd(s.sum_D, D0[i] * kap);
        std::uint32_t mc = 0;
        for (std::uint64_t i = 0; i < N; ++i) {
            const double f2 = force_norm2<ND>(&F[i * ND]);
            if (f2 > 1.0E-16) {
                s.sum_mag = xadd(s.sum_mag, xsqrt(f2));
                ++mc;
            }
        }
        s.mag_count = mc;
        return s;
    }
    void reorder() {
        std::vector<std::uint64_t> key(N);
        for (std::uint64_t i = 0; i < N; ++i) {
            if (ND == 3) {
                std::uint64_t code = 0;
                for (int d = 0; d < 3; ++d) {
                    const double scale = (static_cast<double>(1u << 21) - 1.0) / g.box[d];
                    code |= morton_spread21(morton_axis(x[i * ND + d], g.box[d], scale)) << d;
                }
                key[i] = code;
            } else {
                key[i] = double_order_key(x[i * ND]);
            }
        }
        std::vector<std::uint32_t> perm(N);
        std::iota(perm.begin(), perm.end(), 0u);
        std::stable_sort(perm.begin(), perm.end(), [&](std::uint32_t a, std::uint32_t b) { return key[a] < key[b]; });
        auto apply = [&](auto& arr, int w) {
            auto tmp = arr;
            for (std::uint64_t k = 0; k < N; ++k)
                for (int q = 0; q < w; ++q) tmp[k * w + q] = arr[static_cast<std::uint64_t>(perm[k]) * w + q];
            arr.swap(tmp);
        };
        apply(x, ND); apply(D0, 1); apply(m, ND); apply(v, ND); apply(origin, 1); apply(s.caps, 1);
    }
    void adam(double fix_scale) {
        for (std::uint64_t i = 0; i < N; ++i) {
            for (int d = 0; d < ND; ++d) {
                const std::uint64_t idx = i * ND + d;
                x[idx] = adam_coord(F[idx], m[idx], v[idx], x[idx], a_alpha, a_ib1, a_ib2, a_box[d]);
            }
            if (fix_scale != 1.0) x[i * ND + ND - 1] = xmul(x[i * ND + ND - 1], fix_scale);
        }
    }
    bool any_trigger(double kap) {
        bool any = false;
        for (std::uint64_t i = 0; i < N; ++i) {
            double d2 = 0.0;
            for (int d = 0; d < ND; ++d) {
                const double dd = xsub(x[i * ND + d], x_last[i * ND + d]);
                d2 = xadd(d2, xmul(dd, dd));
            }
            if (refresh_trigger(d2, xmul(D0[i], kap), xmul(D0[i], kappa_min), theta)) any = true;
        }
        return any;
    }
    void initial() {
        if (c.reorder_interval > 0) reorder();
        build(1.0, c.t_shell);
        const ForceSums fs = forces(1.0);
        (void)fs;
    }
    bool step() {
        const std::uint64_t step = c.hist_filled + 1;
        if (step > c.step_cap) return false;
        begin_step(c, h, step);
        if (adam_pending) {
            adam(1.0);
            adam_pending = false;
        }
        if (c.done) return false;
        if (c.reorder) {
            const double kp = c.runtime_fix_diameter ? 1.0 : c.kappa_D_prev;
            reorder();
            build(kp, shell_of(xmul(c.D0_min, kp), xmul(c.D0_med, kp), xmul(c.D0_max, kp)));
        }
        if (c.fix_height && !c.runtime_fix_diameter && c.fix_height_scale != 1.0)
            for (std::uint64_t i = 0; i < N; ++i) x[i * ND + ND - 1] = xmul(x[i * ND + ND - 1], c.fix_height_scale);
        set_box(c.box);
        theta = c.theta;
        bool rebuild = false;
        if (c.rebuild_mode == REBUILD_FULL) {
            rebuild = true;
        } else {
            kappa_min = std::fmin(kappa_min, c.kappa_D);
            rebuild = any_trigger(c.kappa_D);
        }
        if (rebuild) build(c.kappa_D, c.t_shell);
        const ForceSums fs = forces(c.kappa_D);
        const double count = static_cast<double>(1ull + fs.pair_count + fs.wall_count);
        StepScalars sc;
        sc.U = std::pow(xdiv(xadd(fs.pair_U, fs.wall_U), count), 2.0);
        sc.max_overlap = fs.pair_maxov;
        sc.Lc = xdiv(fs.pair_Lc, count);
        sc.dkappa = xadd(xadd(fs.pair_dk, fs.wall_dk), xmul(c.mu_eff, fs.sum_D));
        sc.Fmean = xdiv(-xadd(fs.pair_Fm, fs.wall_Fm), count);
        sc.mean_force = xdiv(xdiv(fs.sum_mag, static_cast<double>(static_cast<std::uint32_t>(fs.mag_count))),
                             xsqrt(static_cast<double>(ND)));
        sc.count = count;
        end_step(c, h, sc);
        for (int d = 0; d < ND; ++d) a_box[d] = c.box[d];
        a_alpha = c.adam_alpha;
        a_ib1 = c.inv_b1;
        a_ib2 = c.inv_b2;
        adam_pending = true;
        return true;
    }
};

template <int ND>
int run_nd(const EngineInput& in, double* pos_out, double* dia_out, double* hist_out,
           std::uint64_t hist_cap, std::uint64_t* origin_out, double* scal_out) {
    Emu<ND> e(prepare_run(in));
    e.initial();
    while (e.step()) {}
    if (e.adam_pending) e.adam(1.0);
    const Controller& c = e.c;
    const std::uint64_t n = c.hist_filled;
    for (std::uint64_t i = 0; i < e.N * ND; ++i) pos_out[i] = e.x[i];
    const double kd = c.runtime_fix_diameter ? 1.0 : c.kappa_D;
    for (std::uint64_t i = 0; i < e.N; ++i) {
        dia_out[i] = c.runtime_fix_diameter ? e.D0[i] : e.D0[i] * kd;
        origin_out[i] = e.origin[i];
    }
    const std::uint64_t k = std::min(n, hist_cap);
    for (std::uint64_t q = 0; q < k; ++q) {
        hist_out[0 * hist_cap + q] = e.hphi[q];
        hist_out[1 * hist_cap + q] = e.hforce[q];
        hist_out[2 * hist_cap + q] = e.henergy[q];
        hist_out[3 * hist_cap + q] = e.hmaxov[q];
        hist_out[4 * hist_cap + q] = e.hmu[q];
        hist_out[5 * hist_cap + q] = e.halpha[q];
        hist_out[6 * hist_cap + q] = e.hflag[q];
    }
    scal_out[0] = static_cast<double>(n);
    scal_out[1] = c.phi;
    scal_out[2] = c.max_min_dist;
    scal_out[3] = c.F_magnitude;
    scal_out[4] = static_cast<double>(e.builds);
    for (int d = 0; d < ND; ++d) scal_out[5 + d] = c.box[d];
    return 0;
}

}  // namespace

extern "C" int hostemu_run_packing(std::uint64_t N, int ndim, const double* positions,
                                   const double* diameters, const double* box,
                                   const std::int8_t* walls, std::uint32_t neighbor_max,
                                   int fix_height, std::uint64_t max_steps, double mu, int has_mu,
                                   int fix_diameter, std::uint64_t reorder_interval,
                                   double* pos_out, double* dia_out, double* hist_out,
                                   std::uint64_t hist_cap, std::uint64_t* origin_out,
                                   double* scal_out, std::uint64_t growth_steps) {
    EngineInput in;
    in.N = N;
    in.ndim = ndim;
    in.positions.assign(positions, positions + N * ndim);
    in.diameters.assign(diameters, diameters + N);
    if (box) in.box.assign(box, box + ndim);
    if (walls) in.walls.assign(walls, walls + ndim);
    in.neighbor_max = neighbor_max;
    in.fix_height = fix_height != 0;
    in.max_steps = max_steps;
    in.has_mu_override = has_mu != 0;
    in.mu_override = mu;
    in.fix_diameter = fix_diameter != 0;
    in.reorder_interval = reorder_interval;
    in.growth_steps = growth_steps;
    switch (ndim) {
        case 2: return run_nd<2>(in, pos_out, dia_out, hist_out, hist_cap, origin_out, scal_out);
        case 3: return run_nd<3>(in, pos_out, dia_out, hist_out, hist_cap, origin_out, scal_out);
        case 4: return run_nd<4>(in, pos_out, dia_out, hist_out, hist_cap, origin_out, scal_out);
        default: return -22;
    }
}

// Layout of the allocation-free build's fixed scratch array (the product's
// own sizing, rcpg_noalloc_plan.h) for a CPU test: out[0..13] = byte offsets
// of ctl, pos, spos, x_last, caps, cell_of, cell_rank, cell_list, work,
// nbr_cnt, nbr, scan_tmp, cell_count, cell_start; out[14] = cell capacity,
// out[15] = bytes used, out[16] = array size. Returns 1 when the plan fits.
extern "C" int hostemu_noalloc_plan(std::uint64_t N, int ndim, std::uint32_t row_capacity,
                                    std::uint64_t* out) {
    const NoAllocPlan p = plan_noalloc(N, ndim, row_capacity, sizeof(DevCtl));
    const std::size_t offs[14] = {p.ctl, p.pos, p.spos, p.x_last, p.caps, p.cell_of, p.cell_rank,
                                  p.cell_list, p.work, p.nbr_cnt, p.nbr, p.scan_tmp, p.cell_count,
                                  p.cell_start};
    for (int k = 0; k < 14; ++k) out[k] = offs[k];
    out[14] = p.cell_capacity;
    out[15] = p.used;
    out[16] = kNoAllocScratchBytes;
    return p.ok ? 1 : 0;
}
