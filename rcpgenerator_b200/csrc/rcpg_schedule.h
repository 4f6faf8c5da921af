// The relaxation controller of Packing.pack(): growth (kappa), learning
// rate (alpha), pressure (mu) rungs, oscillation and the convergence gate.
//
// Restates the step loop of run_packing_observed
// (python_code/python/src/core/rcp_generator.cpp, "ENG", :5511-6662) with the
// reference's defaults for every RCP_* environment knob (clean environment):
// RCP_SPEED=quick, adaptive oscillation on, mu1 boost B=5 / tau=350,
// adaptive shell off (s_dyn = 1), K_BATCH = 1, no sign-flip reset, no
// per-particle alpha multipliers, no state save/load, no cascade mask.
//
// The same code runs on the host (exact mode: host libm, the reference's own
// pow/exp/sin) and inside the one-warp controller kernel (graph mode: CUDA
// libm; identical control flow, last-ulp differences in pow/exp/sin).
#pragma once

#include <cstddef>
#include <cstdint>

#include "rcpg_core.h"

namespace rcpg {

enum : int { OSC_INACTIVE = 0, OSC_ACTIVE = 1, OSC_FINAL = 2, OSC_DONE = 3 };

// What the particle kernels must do before the forces of the step that
// begin_step() opened.
enum : int { REBUILD_CHECK = 1, REBUILD_FULL = 2 };

// Device/host-resident histories, each hist_size = step_cap + 1 long and
// zero-initialised like the reference's (ENG:4739-4748).
struct Histories {
    double* phi;
    double* force;
    double* energy;
    double* max_overlap;
    double* mu;
    double* alpha;
    std::int8_t* mu_flag;
};

// Reduced scalars of one force evaluation, finalised (ENG:4259-4268) plus
// compute_mean_force (ENG:769-803).
struct StepScalars {
    double U;            // (sum overlap / count)^2
    double max_overlap;  // max_min_dist
    double Lc;
    double Fmean;        // -sum(F_mag) / count
    double dkappa;       // sum r(d - r) + walls + mu_eff * sum D
    double mean_force;   // mean |F_i| / sqrt(ndim)  (NaN when no contacts)
    double count;        // 1 + contacts
};

struct Controller {
    // ---- constants of the run -------------------------------------------
    std::uint64_t N;
    int ndim;
    double alpha_max;
    double phi_modifier;
    double coeff;             // pi^(d/2) / Gamma(d/2 + 1)
    double trigger_scale;     // theta = Dmin/4 * trigger_scale (ENG:4376-4430)
    std::uint64_t step_cap;
    std::uint64_t rung1_deadline;
    std::uint64_t reorder_interval;
    int fix_height;
    int has_target_phi;
    double target_phi;
    // D0 statistics: D = D0 * kappa keeps their order (monotone rounding),
    // so min/max/median of D are these times kappa (ENG:5749-5781, :2795-2846).
    double D0_min, D0_max, D0_med;
    double S_D0;              // sum (D0/2)^ndim (ENG:4816-4828)

    // ---- dynamic state ----------------------------------------------------
    double t;                 // ADAM counter
    double alpha;
    double mu;
    int mu_flag;
    double mu_change;
    std::uint64_t last_alpha_update;
    double phi;
    double phi_max;
    std::uint64_t phi_max_step;
    double kappa;             // current growth variable
    double kappa_D;           // kappa of the last diameter update (D = D0*kappa_D)
    double kappa_D_prev;      // kappa_D of the previous step (used by the reorder rebuild)
    double m_kappa, v_kappa, m_hat_kappa, v_hat_kappa;
    double F_magnitude;
    double max_min_dist;
    double U;
    double Dmin;              // Dmin at the last full rebuild (ENG:4518, :6038)
    double box[kMaxDim];
    double box_volume;        // box volume used for this step's phi
    int runtime_fix_diameter;
    int target_phi_locked;
    int mu_decay_active;
    double mu_decay_target;
    std::uint64_t mu_decay_next_tick;
    int osc_phase;
    double osc_mu_0, osc_mu_m1;
    std::uint64_t osc_start, osc_period, osc_t_relax, osc_final_start, osc_consec;
    std::uint64_t steps;
    std::uint64_t hist_filled;

    // ---- outputs of begin_step for the particle kernels -------------------
    int done;                 // convergence gate fired at the top of step `steps`
    int reorder;              // spatial reorder before this step's refresh
    int rebuild_mode;         // REBUILD_CHECK or REBUILD_FULL
    int lock_now;             // target-phi lock requested (host-only action)
    double theta;             // refresh budget Dmin/4 * trigger_scale
    double mu_eff;            // pressure fed to the forces (ENG:6214-6218)
    double t_shell;           // pair shell for a rebuild in this step
    double Dmax_cur;          // current max diameter
    double fix_height_scale;  // factor applied to the last coordinate this step
    // ---- outputs of end_step for the ADAM pass ----------------------------
    double adam_alpha, inv_b1, inv_b2;
};

// ---- helpers -------------------------------------------------------------

RCPG_HD double phi_range(const double* h, std::uint64_t lo, std::uint64_t hi) {
    // max - min over h[lo, hi) (std::minmax_element, ENG:5533-5536)
    double mn = h[lo], mx = h[lo];
    for (std::uint64_t k = lo + 1; k < hi; ++k) {
        const double v = h[k];
        if (v < mn) mn = v;
        if (v > mx) mx = v;
    }
    return xsub(mx, mn);
}

// mean(v, start, end) with inclusive end (ENG:757-767).
RCPG_HD double hist_mean(const double* v, std::uint64_t start, std::uint64_t end) {
    double s = 0.0;
    for (std::uint64_t k = start; k <= end; ++k) s = xadd(s, v[k]);
    return xdiv(s, static_cast<double>(end - start + 1));
}

RCPG_HD double dmin2(double a, double b) { return (b < a) ? b : a; }  // std::min
RCPG_HD double dmax2(double a, double b) { return (a < b) ? b : a; }  // std::max

// Pair shell t = min(max(median*1.02, Dmin*2.25), Dmax)*0.5 (ENG:2846).
RCPG_HD double shell_of(double Dmin, double Dmed, double Dmax) {
    return xmul(dmin2(dmax2(xmul(Dmed, 1.02), xmul(Dmin, 2.25)), Dmax), 0.5);
}

// Window statistics of the histories that begin_step(step) reads: the phi
// range over [step - 250, step - 1) and the force means of the learning-rate
// rule. The graph-mode controller computes them with its whole block before
// the serial schedule; the host computes them in the reference's order.
struct HistStats {
    double phi_range_250;  // phi_range(h.phi, step - 250, step - 1)
    double f_450_250;      // hist_mean(h.force, step - 450, step - 250)
    double f_75_1;         // hist_mean(h.force, step - 75, step - 1)
    double f_200_1;        // hist_mean(h.force, step - 200, step - 1)
    double f_3000_2500;    // hist_mean(h.force, step - 3000, step - 2500)
};

// ---- top of step (ENG:5520-6042) ------------------------------------------
// Everything the reference does before its pair refresh, except the two
// particle-wide actions it requests through flags: reorder and lock_now.
// `pre` (optional) holds the history window statistics of this step.
RCPG_HD void begin_step(Controller& c, const Histories& h, std::uint64_t step, const HistStats* pre = nullptr) {
    const std::uint64_t cooldown = 250;
    const double flat = 5e-3, decay = 0.85;
    c.steps = step;
    c.done = 0;
    c.reorder = 0;
    c.lock_now = 0;
    c.fix_height_scale = 1.0;
    c.t = xadd(c.t, 1.0);

    // feedback mu decay (ENG:5528-5544)
    if (c.mu_decay_active && step >= c.mu_decay_next_tick && step > 250) {
        const double rng = pre ? pre->phi_range_250 : phi_range(h.phi, step - 250, step - 1);
        if (rng < flat) {
            c.mu = xmul(c.mu, decay);
            if (c.mu <= c.mu_decay_target) {
                c.mu = c.mu_decay_target;
                c.mu_decay_active = 0;
            }
            c.mu_decay_next_tick = step + cooldown;
        }
    }
    // oscillation start (ENG:5553-5571)
    if (c.osc_phase == OSC_INACTIVE && c.mu_flag == 0 && !c.mu_decay_active &&
        c.mu_change > 0 && static_cast<double>(step) > c.mu_change) {
        c.osc_mu_0 = c.mu;
        c.osc_mu_m1 = xdiv(c.mu, 10.0);
        c.osc_t_relax = step - static_cast<std::uint64_t>(c.mu_change);
        if (c.osc_t_relax < 250) c.osc_t_relax = 250;
        c.osc_start = step;
        c.osc_period = static_cast<std::uint64_t>(xmul(0.5, c.mu_change));
        if (c.osc_period < 1000) c.osc_period = 1000;
        c.osc_phase = OSC_ACTIVE;
        c.mu_flag = -1;
        c.mu_change = static_cast<double>(step);
        c.alpha = xdiv(c.alpha, 2.0);
    }
    const double cycles = 2.0;
    if (c.osc_phase == OSC_ACTIVE) {
        const double t_into = static_cast<double>(step - c.osc_start);
        const double cp = xdiv(t_into, static_cast<double>(c.osc_period));
        if (cp >= cycles) {
            c.mu = c.osc_mu_m1;
            c.osc_phase = OSC_FINAL;
            c.osc_final_start = step;
            c.mu_decay_next_tick = step + cooldown;
        } else {
            const double ph = xsub(cp, floor(cp));
            const double sin_val = -sin(xmul(xmul(2.0, 3.14159265358979323846), ph));
            const double mu_ref =
                xadd(xmul(xsub(c.osc_mu_0, c.osc_mu_m1),
                          exp(xdiv(-t_into, static_cast<double>(c.osc_t_relax)))),
                     c.osc_mu_m1);
            c.mu = xmul(mu_ref, pow(10.0, sin_val));
            if (cp >= xsub(cycles, 0.25)) {
                // F_history[step-1] is not written yet at the top of the step,
                // so the reference reads its zero (ENG:5615-5616).
                const double F_now = (step >= 1) ? h.force[step - 1] : 0.0;
                const bool met = (F_now < 5e-3) && (c.max_min_dist < 5e-4);
                if (met) {
                    c.osc_consec += 1;
                    if (c.osc_consec >= 3) c.osc_phase = OSC_DONE;
                } else {
                    c.osc_consec = 0;
                }
            }
        }
    } else if (c.osc_phase == OSC_FINAL && step >= c.mu_decay_next_tick && step > 250) {
        const double rng = pre ? pre->phi_range_250 : phi_range(h.phi, step - 250, step - 1);
        if (rng < flat) {
            const double F_now = (step >= 1) ? h.force[step - 1] : 0.0;
            const bool met = (F_now < 5e-3) && (c.max_min_dist < 5e-4);
            if (met) {
                c.osc_consec += 1;
                if (c.osc_consec >= 3) c.osc_phase = OSC_DONE;
            } else {
                c.osc_consec = 0;
                c.mu = xmul(c.mu, decay);
            }
            if (step - c.osc_final_start > 50000) c.osc_phase = OSC_DONE;
            c.mu_decay_next_tick = step + cooldown;
        }
    }
    if (c.osc_phase == OSC_DONE) {
        c.done = 1;
        return;
    }
    // periodic spatial reorder (ENG:5661-5663)
    if (c.reorder_interval > 0 && step > 1 && (step % c.reorder_interval == 0)) c.reorder = 1;

    // learning rate (ENG:5665-5721)
    {
        const std::uint64_t s250 = (step > 251) ? step - 250 : 1;  // max(step-250, 1)
        if ((step - c.last_alpha_update > 500) && (xsub(c.phi, h.phi[s250]) < 5e-4) &&
            (step > 2500) && static_cast<double>(step) > xadd(c.mu_change, 500.0)) {
            double trend1 = pre ? xdiv(pre->f_450_250, pre->f_75_1)
                                : xdiv(hist_mean(h.force, step - 450, step - 250), hist_mean(h.force, step - 75, step - 1));
            const double trend2 = xsub(c.phi, h.phi[s250]);
            if ((c.mu_flag < 1 && trend1 < 0.85) || trend2 < -5E-4) {
                c.last_alpha_update = step;
                c.alpha = xdiv(c.alpha, 1.5);
            } else if (c.mu_flag < 1 && step - c.last_alpha_update > 1500) {
                trend1 = pre ? xdiv(pre->f_200_1, pre->f_3000_2500)
                             : xdiv(hist_mean(h.force, step - 200, step - 1), hist_mean(h.force, step - 3000, step - 2500));
                if (trend1 > 0.5) {
                    c.last_alpha_update = step;
                    c.alpha = xmul(c.alpha, 1.15);
                }
            }
            if (c.mu_flag == 1) c.alpha = dmax2(c.alpha, xdiv(c.alpha_max, 10.0));
        }
        c.alpha = dmin2(xmul(c.alpha, 1.00005), c.alpha_max);
        if (step % 500 == 0) c.alpha = dmin2(c.alpha_max, xmul(1.1, c.alpha));
        if (c.mu_flag == -1) {
            const double cap = xmul(c.alpha_max, 0.01);
            if (c.alpha > cap) c.alpha = cap;
        }
    }

    // diameters, phi (ENG:5723-5781)
    c.kappa_D_prev = c.kappa_D;
    if (!c.runtime_fix_diameter) c.kappa_D = c.kappa;
    const double kap = c.runtime_fix_diameter ? 1.0 : c.kappa;
    double Dmin_latest = xmul(c.D0_min, kap);
    double k_nd = 1.0;
    if (!c.runtime_fix_diameter)
        for (int k = 0; k < c.ndim; ++k) k_nd = xmul(k_nd, c.kappa);
    const double current_volume = xmul(xmul(c.coeff, c.S_D0), k_nd);
    // box volume before this step's fix_height stretch (ENG:5775-5783)
    double box_volume = 1.0;
    for (int k = 0; k < c.ndim; ++k) box_volume = xmul(box_volume, c.box[k]);
    c.box_volume = box_volume;
    if (c.fix_height && !c.runtime_fix_diameter) {
        c.box[c.ndim - 1] = xmul(c.box[c.ndim - 1], c.kappa);
        c.fix_height_scale = c.kappa;
    }
    c.phi = xdiv(current_volume, box_volume);
    if (c.has_target_phi && !c.target_phi_locked && !c.runtime_fix_diameter) {
        if (xdiv(c.phi, c.phi_modifier) >= c.target_phi) {
            // Rescaling D0 to the target needs a pass over all diameters; the
            // host performs it and calls finish_lock() (ENG:5783-5832).
            c.lock_now = 1;
            return;
        }
    }
    h.phi[step - 1] = xdiv(c.phi, c.phi_modifier);
    if (c.phi > c.phi_max) {
        c.phi_max = c.phi;
        c.phi_max_step = step;
    }
    // rung-1 deadline (ENG:5834-5931)
    if (step > 500 && c.mu_flag == 1) {
        if (step > c.rung1_deadline) {
            c.mu_decay_target = xdiv(c.mu, 10.0);
            c.mu_decay_active = 1;
            c.mu_decay_next_tick = step + cooldown;
            c.alpha = xdiv(c.alpha, 2.0);
            c.mu_flag = 0;
            c.mu_change = static_cast<double>(step);
        }
    }
    // full rebuild on Dmin growth, else the displacement trigger (ENG:6022-6047)
    const double ts = c.trigger_scale;
    if (xdiv(Dmin_latest, c.Dmin) > 1.05) {
        c.rebuild_mode = REBUILD_FULL;
        c.Dmin = Dmin_latest;
    } else {
        c.rebuild_mode = REBUILD_CHECK;
    }
    c.theta = xmul(xmul(c.Dmin, 0.25), ts);
    c.mu_eff = (c.mu_flag == 1)
                   ? xmul(c.mu, xadd(1.0, xmul(4.0, exp(xdiv(-static_cast<double>(step), 350.0)))))
                   : c.mu;
    const double Dmin_cur = xmul(c.D0_min, kap);
    const double Dmed_cur = xmul(c.D0_med, kap);
    c.Dmax_cur = xmul(c.D0_max, kap);
    c.t_shell = shell_of(Dmin_cur, Dmed_cur, c.Dmax_cur);
}

// Completes a step whose target-phi lock the host has just applied: D0 is
// the rescaled diameter set, kappa = 1, the pair list rebuilt (ENG:5783-5832).
RCPG_HD void finish_lock(Controller& c, const Histories& h, std::uint64_t step, double D0_min,
                         double D0_max, double D0_med, double S_D0) {
    const std::uint64_t cooldown = 250;
    c.kappa = 1.0;
    c.kappa_D = 1.0;
    c.mu = 0.0;
    c.runtime_fix_diameter = 1;
    c.target_phi_locked = 1;
    c.lock_now = 0;
    c.D0_min = D0_min;
    c.D0_max = D0_max;
    c.D0_med = D0_med;
    c.S_D0 = S_D0;
    const double Dmin_latest = D0_min;
    c.phi = xdiv(xmul(c.coeff, S_D0), c.box_volume);
    c.Dmin = Dmin_latest;
    h.phi[step - 1] = xdiv(c.phi, c.phi_modifier);
    if (c.phi > c.phi_max) {
        c.phi_max = c.phi;
        c.phi_max_step = step;
    }
    if (step > 500 && c.mu_flag == 1 && step > c.rung1_deadline) {
        c.mu_decay_target = xdiv(c.mu, 10.0);
        c.mu_decay_active = 1;
        c.mu_decay_next_tick = step + cooldown;
        c.alpha = xdiv(c.alpha, 2.0);
        c.mu_flag = 0;
        c.mu_change = static_cast<double>(step);
    }
    // Dmin_latest / Dmin == 1: the displacement trigger runs (and finds the
    // freshly anchored particles unmoved).
    c.rebuild_mode = REBUILD_CHECK;
    c.theta = xmul(xmul(c.Dmin, 0.25), c.trigger_scale);
    c.mu_eff = (c.mu_flag == 1)
                   ? xmul(c.mu, xadd(1.0, xmul(4.0, exp(xdiv(-static_cast<double>(step), 350.0)))))
                   : c.mu;
    c.Dmax_cur = D0_max;
    c.t_shell = shell_of(D0_min, D0_med, D0_max);
}

// ---- end of step (ENG:6249-6577) ------------------------------------------
RCPG_HD void end_step(Controller& c, const Histories& h, const StepScalars& s) {
    const std::uint64_t step = c.steps;
    c.U = s.U;
    c.max_min_dist = s.max_overlap;
    c.F_magnitude = xdiv(s.mean_force, s.Fmean);
    h.force[step - 1] = c.F_magnitude;
    h.max_overlap[step - 1] = c.max_min_dist;
    h.mu[step - 1] = c.mu;
    h.alpha[step - 1] = c.alpha;
    h.mu_flag[step - 1] = static_cast<std::int8_t>(c.mu_flag);
    // kappa half of the fused ADAM (ENG:6354-6358)
    const double dk = s.dkappa;
    c.m_kappa = xsub(xmul(0.9, c.m_kappa), xmul(xsub(1.0, 0.9), dk));
    c.v_kappa = xadd(xmul(0.999, c.v_kappa), xmul(xsub(1.0, 0.999), xmul(dk, dk)));
    const double pb1 = pow(0.9, c.t);
    const double pb2 = pow(0.999, c.t);
    c.m_hat_kappa = xdiv(c.m_kappa, xsub(1.0, pb1));
    c.v_hat_kappa = xdiv(c.v_kappa, xsub(1.0, pb2));
    if (!c.runtime_fix_diameter)
        c.kappa = xsub(c.kappa, xdiv(xmul(c.alpha, c.m_hat_kappa), xadd(xsqrt(c.v_hat_kappa), 1e-8)));
    c.adam_alpha = c.alpha;
    c.inv_b1 = xdiv(1.0, xsub(1.0, pb1));
    c.inv_b2 = xdiv(1.0, xsub(1.0, pb2));
    h.energy[step - 1] = c.U;
    c.hist_filled = step;
}

}  // namespace rcpg
