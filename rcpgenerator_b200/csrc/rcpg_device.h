// Device-resident state of one packing and the launchers of its kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "rcpg_core.h"
#include "rcpg_schedule.h"

namespace rcpg {

constexpr int kMaxClass = 8;

// Scalars the particle kernels read, plus status words they write. Lives in
// device memory; in exact (host-controlled) mode the host rewrites it every
// step, in graph mode the controller kernel does.
struct DevCtl {
    Controller c;        // schedule state (graph mode: owned by the controller kernel)
    Geometry g;          // box / walls of the current step
    ForceSums sums;      // reduced sums of the last force evaluation
    StepScalars scal;    // finalised scalars of the last force evaluation
    // ADAM pass parameters (of the step being finished)
    double adam_box[kMaxDim];
    double adam_alpha, adam_inv_b1, adam_inv_b2;
    double fix_height_scale;
    // pair-list build parameters
    double build_kappa;  // D = D0 * build_kappa during the build
    double build_t_shell;
    double build_Dmax;
    // refresh anchor (shared by all particles: every rebuild re-anchors all)
    double refresh_kappa;  // D = D0 * refresh_kappa in the trigger
    double kappa_min;      // running minimum of kappa since the anchor
    double theta;          // budget
    double force_kappa;    // D = D0 * force_kappa in the forces
    double force_mu;       // mu fed to the forces
    // cell grid of the current build (one grid, or class 0's of several)
    int ncell[kMaxDim];
    double cell_scale[kMaxDim];
    std::uint32_t ncells;         // cells of all grids
    // Size classes (wide size distributions): class k holds the particles with
    // D0 in [class_d0[k], class_d0[k+1]) and has its own grid, as wide as the
    // pair cutoff of its largest member (class_d0max[k]); nclass <= 1: one grid
    int nclass;
    int tile_rows;       // 2-D tiled build: tile height in cells (set by k_build_prepare)
    double class_d0[kMaxClass + 1];
    double class_d0max[kMaxClass];
    int cls_ncell[kMaxClass][kMaxDim];
    double cls_scale[kMaxClass][kMaxDim];
    std::uint32_t cls_base[kMaxClass + 1];  // first cell of class k
    // control words
    std::uint32_t rebuild_flag;   // rebuild the pair list before the forces
    std::uint32_t adam_go;        // ADAM pass of the finished step is pending
    std::uint32_t stopped;        // graph steps after this point do nothing
    std::uint32_t halted;         // stopped because of an error / capacity overflow
    std::uint32_t row_need;       // largest full row seen by a build
    std::uint32_t cap_error;      // a half row exceeded the reference capacity
    // ~(particle << 32 | capacity) of the lowest-indexed particle over its
    // capacity (the maximum of the complements: the reference's loop reports
    // the first particle in index order); 0 = none
    unsigned long long cap_error_key;
    std::uint32_t nbuilds;        // pair-list builds performed
    std::uint32_t fuse_forces;    // a tiled build also computes the step's forces (graph mode)
    std::uint32_t forces_done;    // this step's forces were computed by the build
    std::uint32_t nsum_blocks;    // number of valid entries in block_sums
    std::uint64_t graph_steps;    // steps completed by the controller kernel
    // mixed-precision pair arithmetic (graph mode): FP32 pair terms while the
    // max overlap of the last step is >= mixed_switch, FP64 from then on
    std::uint32_t pair_fp32;      // the forces of the current step use FP32 pair terms
    std::uint32_t pad0;
    double mixed_switch;
    std::uint64_t fp64_switch_step;  // step whose max overlap fell below mixed_switch (0: none)
    // cell-order storage (graph mode): which of the two buffer sets holds the
    // particle state, flipped by each build's permutation; blocks of the
    // permutation kernel that have finished (the last one flips)
    std::uint32_t buf;
    std::uint32_t permute_done;
    std::uint64_t pair_kernel_runs;  // launches of the pair kernel that computed forces
    // Cell units of the cell-order kernels (graph mode, one size class, set by
    // each build): a unit is unit_w consecutive cells of one grid row (the last
    // unit of a row may be shorter); unit_chunks units per grid row, unit_count
    // units in all.
    std::uint32_t unit_w;
    std::uint32_t unit_chunks;
    std::uint32_t unit_count;
    std::uint32_t pad1;
};

// In graph mode every pair-list build stores the particles in cell order
// ("cell-order storage"): the build permutes the per-particle state (pos, m,
// v, origin, caps, ref_rank) into the second buffer set (*_alt) in the order of
// the cell grid -- cells in grid order, each cell's members in their previous
// order -- and flips DevCtl::buf, so the search and the pair kernel read each
// particle's neighbours from a few contiguous ranges. Rows then hold partner
// indices of that order and F is in that order too. ref_rank[i] is the
// particle's index in the reference's own order (input order permuted by its
// spatial reorders), used to return results in that order. Kernels call
// bind_buffers() first, which points pos/m/v/origin/caps/ref_rank at the
// current set; without *_alt (exact mode, the stand-alone C ABI kernels) the
// arrays never move.
struct DevArrays {
    std::uint64_t N;
    int ndim;
    int P;                  // pos stride
    double* pos;            // [N*P] x_0..x_{d-1}, D0 (32-byte aligned records for the force kernel)
    double* pos_tmp;        // [N*P] reorder gather target
    double* spos;           // [N*P] positions in cell order (build scratch; may alias pos_tmp)
    double* F;              // [N*ndim]
    double* m;              // [N*ndim]
    double* v;              // [N*ndim]
    double* vec_tmp;        // [N*ndim] reorder gather target
    double* x_last;         // [N*ndim] refresh anchor positions
    std::uint32_t* nbr;     // [S*N] column-major full rows (see sorted_rows)
    std::uint32_t* nbr_cnt; // [N]
    // Row slot -> particle map. Row t (nbr[k*N + t], nbr_cnt[t]) belongs to
    // particle work[t]; rows are kept in cell order (a build writes work: the
    // members of each cell in ascending particle order) so a warp's particles,
    // and their partners, are spatial neighbours. nullptr = identity (rows in
    // particle order).
    std::uint32_t* work;
    std::uint32_t S;        // row capacity
    // 1: rows sorted by partner index (exact mode, pairs_full: the reference's
    // summation order); 0: rows in the build's fixed scan order (graph mode)
    int sorted_rows;
    // 1: the run may use FP32 pair terms (mixed precision), so the force
    // kernel is launched in both variants; each checks ctl->pair_fp32
    int mixed;
    std::uint32_t* caps;    // [N] half-row capacity of the reference layout
    std::uint64_t* origin;  // [N] particle_origin
    std::uint64_t* u64_tmp; // [N]
    std::uint32_t* cell_of;    // [N]
    std::uint32_t* cell_rank;  // [N]
    std::uint32_t* cell_count; // [C_alloc + 1]
    std::uint32_t* cell_start; // [C_alloc + 1]
    std::uint32_t* cell_list;  // [N] members of each cell in arrival order (k_build_scatter)
    std::uint32_t C_alloc;
    std::uint32_t* scan_tmp;   // block sums of the scan
    ForceSums* block_sums;     // [nblocks of the force kernel]
    PairTerms* pterm;          // [S*N] exact-order pair terms (exact mode only)
    std::uint32_t* pterm_cnt;  // [N]
    // radix sort
    std::uint64_t* sort_keys[2];
    std::uint32_t* sort_vals[2];
    std::uint32_t* sort_hist;  // [256 * nblocks]
    DevCtl* ctl;
    Histories hist;            // device histories (graph mode)
    // cell-order storage (graph mode; nullptr otherwise): the second buffer
    // set and the reference-order rank of each particle
    int permute;               // 1: every build permutes into cell order
    double* pos_alt;
    double* m_alt;
    double* v_alt;
    std::uint64_t* origin_alt;
    std::uint32_t* caps_alt;
    std::uint32_t* ref_rank;
    std::uint32_t* ref_rank_alt;
    // Captured step graphs with conditional nodes (graph mode): the handle of
    // the step's pair-kernel switch (0 = FP64 kernel, 1 = mixed kernel,
    // 2 = none), set by the step gate and by the build's last kernel; 0 when
    // the kernels are launched outside such a graph.
    unsigned long long cond_forces;
};

// Particle index and capacity of the first over-capacity particle.
inline std::uint32_t cap_error_particle(const DevCtl& c) { return static_cast<std::uint32_t>((~c.cap_error_key) >> 32); }
inline std::uint32_t cap_error_capacity(const DevCtl& c) { return static_cast<std::uint32_t>(~c.cap_error_key); }

// The arrays of the buffer set `buf` (host twin of bind_buffers).
RCPG_HD DevArrays bound_arrays(DevArrays a, std::uint32_t buf) {
    if (a.permute && buf) {
        a.pos = a.pos_alt;
        a.m = a.m_alt;
        a.v = a.v_alt;
        a.origin = a.origin_alt;
        a.caps = a.caps_alt;
        a.ref_rank = a.ref_rank_alt;
    }
    return a;
}

constexpr int kForceBlock = 256;

RCPG_HD unsigned force_blocks(std::uint64_t N) {
    return static_cast<unsigned>((N + kForceBlock - 1) / kForceBlock);
}

// ---- launchers (rcpg_kernels.cu) ------------------------------------------
// All take the device arrays by value and enqueue on `st`.
void launch_adam_refresh(const DevArrays& a, int do_adam, int do_refresh, cudaStream_t st);
void launch_rebuild(const DevArrays& a, cudaStream_t st);
// the same, with e0 / e1 recorded just before and after the search kernels
// (the tiled build and the warp search; the one that has nothing to do returns)
void launch_rebuild_timed(const DevArrays& a, cudaStream_t st, cudaEvent_t e0, cudaEvent_t e1);
void launch_forces(const DevArrays& a, int exact_terms, cudaStream_t st);
// One variant of the pair kernel (mixed = 0: FP64 pair terms, 1: FP32 pair
// terms), the body of a step graph's pair-kernel switch.
void launch_forces_variant(const DevArrays& a, int mixed, cudaStream_t st);
// The step gate of a captured step graph: opens the build (cond_build = 1
// when the step rebuilds its rows) and sets the pair-kernel switch for a step
// without a build.
void launch_step_gate(const DevArrays& a, unsigned long long cond_build, cudaStream_t st);
void launch_reduce_exact(const DevArrays& a, cudaStream_t st);
void launch_reduce_fast(const DevArrays& a, cudaStream_t st);
// out[0] = max |ref[k]|, out[1] = max |cmp[k] - ref[k]| over k < n, as the bit
// patterns of the non-negative doubles (out zeroed first by the caller).
void launch_diff_max(const double* ref, const double* cmp, std::uint64_t n, unsigned long long* out,
                     cudaStream_t st);
void launch_controller(const DevArrays& a, int open_only, cudaStream_t st);
void launch_reorder(const DevArrays& a, cudaStream_t st);
void launch_fix_height(const DevArrays& a, cudaStream_t st);

void launch_pack(std::uint64_t N, int ndim, const double* x, const double* D, double* pos,
                 cudaStream_t st);
void launch_unpack(std::uint64_t N, int ndim, const double* pos, double* x, cudaStream_t st);
void launch_refresh_arrays(std::uint64_t N, int ndim, const double* x, double* x_last,
                           const double* D, double* D_last, double* theta, double theta_new,
                           std::uint8_t* refresh, unsigned long long* count, cudaStream_t st);
void launch_mean_force_blocks(const DevArrays& a, cudaStream_t st);
// Cell-order storage -> the input's particle order (origin holds each
// particle's input index): rows (partners mapped too), counts and forces.
void launch_cell_order_to_particle_order(const DevArrays& a, std::uint32_t* nbr_out, std::uint32_t* cnt_out,
                                         double* F_out, cudaStream_t st);
void launch_rows_to_particle_order(std::uint64_t N, const std::uint32_t* work, const std::uint32_t* src,
                                   const std::uint32_t* src_cnt, std::uint32_t* dst,
                                   std::uint32_t* dst_cnt, cudaStream_t st);

// Host-side finalisation shared with the controller kernel (ENG:4259-4268, :769-803).
RCPG_HD StepScalars finalize_sums(const ForceSums& s, double mu_eff, int ndim) {
    StepScalars r;
    const double count = static_cast<double>(1ull + s.pair_count + s.wall_count);
    const double U_tot = xadd(s.pair_U, s.wall_U);
    r.U = pow(xdiv(U_tot, count), 2.0);
    r.max_overlap = s.pair_maxov;
    r.Lc = xdiv(s.pair_Lc, count);
    r.dkappa = xadd(xadd(s.pair_dk, s.wall_dk), xmul(mu_eff, s.sum_D));
    r.Fmean = xdiv(-xadd(s.pair_Fm, s.wall_Fm), count);
    const double mean_mag = xdiv(s.sum_mag, static_cast<double>(static_cast<std::uint32_t>(s.mag_count)));
    r.mean_force = xdiv(mean_mag, xsqrt(static_cast<double>(ndim)));
    r.count = count;
    return r;
}

}  // namespace rcpg
