// CUDA kernels of the packing step (sm_100a).
//
// One thread per particle everywhere except the controller (one block) and the
// scans / radix sort. The pair list is a full list (both directions) stored
// column-major, nbr[k*N + t], so a warp reading entry k of 32 consecutive rows
// issues one coalesced 128-byte load, and every particle sums its own pair
// forces without atomics. In exact mode each row is sorted by partner index,
// the order in which the reference's one-thread loop accumulates the forces;
// in graph mode a row keeps the build's fixed scan order (deterministic run to
// run). Pair scalars (energy, dkappa, ...) are counted once per pair, by the
// lower index.
#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <type_traits>

#include "rcpg_device.h"
#include "rcpg_devutil.cuh"

namespace rcpg {

namespace {

// Early-exit guards. The flags are combined with bitwise operators so that
// all of their loads are issued before the first branch: one round trip to
// memory per block instead of one per flag (kernels that have nothing to do
// in a step otherwise cost several microseconds at N = 1M).
__device__ __forceinline__ bool ctl_idle(const DevCtl* ctl) {
    const std::uint32_t st = ctl->stopped, ha = ctl->halted;
    return (st | ha) != 0u;
}

// Value of a step graph's pair-kernel switch: 0 = FP64 kernel, 1 = mixed
// kernel, 2 = no pair kernel (the forces are computed elsewhere or the run
// has stopped).
__device__ __forceinline__ unsigned forces_case(bool run, std::uint32_t pair_fp32, int mixed) {
    return !run ? 2u : ((pair_fp32 != 0u && mixed) ? 1u : 0u);
}

// no pair-list build in this step
__device__ __forceinline__ bool build_off(const DevCtl* ctl) {
    const std::uint32_t st = ctl->stopped, ha = ctl->halted, rb = ctl->rebuild_flag;
    return ((st | ha) != 0u) | (rb == 0u);
}

// ===========================================================================
// A. ADAM step of the finished step + refresh trigger of the next step
// ===========================================================================
// Persistent grid (resident_grid): each thread loads the step's parameters
// once and then walks the particles with a grid stride, two at a time, so the
// loads of both are in flight together.
template <int ND>
__global__ void __launch_bounds__(256) k_adam_refresh(DevArrays a, int do_adam, int do_refresh) {
    const DevCtl* ctl = a.ctl;
    const std::uint32_t halted = ctl->halted, adam_go = ctl->adam_go, stopped = ctl->stopped;
    const int mode = ctl->c.rebuild_mode;
    if (halted) return;
    const bool adam = do_adam && adam_go;
    const bool refresh = do_refresh && !stopped && mode == REBUILD_CHECK;
    if (!adam && !refresh) return;
    bind_buffers(a);
    const double alpha = ctl->adam_alpha, ib1 = ctl->adam_inv_b1, ib2 = ctl->adam_inv_b2;
    const double fh = ctl->fix_height_scale;
    const double rk = ctl->refresh_kappa, kmin = ctl->kappa_min, theta = ctl->theta;
    double abox[ND];
    RCPG_UNROLL
    for (int d = 0; d < ND; ++d) abox[d] = ctl->adam_box[d];
    const std::uint64_t N = a.N;
    const std::uint64_t stride = static_cast<std::uint64_t>(gridDim.x) * blockDim.x;
    bool trig = false;
    for (std::uint64_t i0 = blockIdx.x * static_cast<std::uint64_t>(blockDim.x) + threadIdx.x; i0 < N;
         i0 += 2 * stride) {
        constexpr int U = 2;
        double x[U][ND], D0[U], F[U][ND], m[U][ND], v[U][ND], xl[U][ND];
        RCPG_UNROLL
        for (int u = 0; u < U; ++u) {
            const std::uint64_t i = i0 + u * stride;
            if (i >= N) continue;
            load_pos<ND>(a.pos, i, x[u], D0[u]);
            RCPG_UNROLL
            for (int d = 0; d < ND; ++d) {
                if (adam) {
                    F[u][d] = a.F[i * ND + d];
                    m[u][d] = a.m[i * ND + d];
                    v[u][d] = a.v[i * ND + d];
                }
                if (refresh) xl[u][d] = a.x_last[i * ND + d];
            }
        }
        RCPG_UNROLL
        for (int u = 0; u < U; ++u) {
            const std::uint64_t i = i0 + u * stride;
            if (i >= N) continue;
            if (adam) {
                RCPG_UNROLL
                for (int d = 0; d < ND; ++d) {
                    x[u][d] = adam_coord(F[u][d], m[u][d], v[u][d], x[u][d], alpha, ib1, ib2, abox[d]);
                    a.m[i * ND + d] = m[u][d];
                    a.v[i * ND + d] = v[u][d];
                }
                if (fh != 1.0) x[u][ND - 1] = xmul(x[u][ND - 1], fh);
                store_pos<ND>(a.pos, i, x[u], D0[u]);
            }
            if (refresh) {
                double d2 = 0.0;
                RCPG_UNROLL
                for (int d = 0; d < ND; ++d) {
                    const double dd = xsub(x[u][d], xl[u][d]);
                    d2 = xadd(d2, xmul(dd, dd));
                }
                trig = trig || refresh_trigger(d2, xmul(D0[u], rk), xmul(D0[u], kmin), theta);
            }
        }
    }
    // one flag write per block (a million same-address stores would serialise in L2)
    if (__syncthreads_or(trig) && threadIdx.x == 0) a.ctl->rebuild_flag = 1u;
}

// ===========================================================================
// B. pair-list rebuild: grid -> bin -> scan -> scatter -> search
// ===========================================================================
// Height of the 2-D tiles of the tiled search (k_build_search_tiled), chosen
// per build from the mean cell occupancy.
constexpr int kTileRowsMin = 4, kTileRowsMax = 12, kTileRowsPref = 8;
constexpr int kTileStage2 = 1024;  // staged particles per 2-D tile (TileShape<2>::stage)

// Shape of the cell units of the cell-order search (k_cells, below).
template <int ND>
struct UnitShape {
    static constexpr int ndc = ND <= 3 ? ND : 3;
    static constexpr int rows = ndc == 2 ? 3 : 9;        // neighbour rows of a unit
    static constexpr int threads = ndc == 2 ? 128 : 64;  // block size
    static constexpr int target = ndc == 2 ? 112 : 56;   // particles per unit
    static constexpr int stage = ndc == 2 ? 640 : 768;   // staged records (32 bytes each)
    static constexpr int maxw = ndc == 2 ? 256 : 128;    // cells per unit at most
    static constexpr int slice = maxw + 3;               // cell_start entries per row (build)
    static constexpr int windows = 3 * rows;             // main, wrapped x-1, wrapped x+1 per row
    static constexpr int min_blocks = 6;                 // resident blocks per SM (register budget)
};

// Cells per unit for a build with `cells` cells in a grid of nc0 cells per row:
// about `target` particles at the mean occupancy, windows that fit the stage
// with 30 % headroom, at most maxw cells.
template <int ND>
__device__ __forceinline__ std::uint32_t unit_width(std::uint64_t N, double cells, int nc0) {
    using US = UnitShape<ND>;
    const double ppc = static_cast<double>(N) / (cells > 1.0 ? cells : 1.0);
    const double occ = ppc > 1e-3 ? ppc : 1e-3;
    double w = floor(static_cast<double>(US::target) / occ);
    const double ws = floor(static_cast<double>(US::stage) / (1.3 * US::rows * occ)) - 2.0;
    if (ws < w) w = ws;
    if (w > static_cast<double>(US::maxw)) w = US::maxw;
    if (w > static_cast<double>(nc0)) w = nc0;
    if (!(w >= 1.0)) w = 1.0;
    return static_cast<std::uint32_t>(w);
}

__global__ void k_build_prepare(DevArrays a) {
    DevCtl* ctl = a.ctl;
    if (build_off(ctl)) return;
    const std::uint32_t n = a.C_alloc + 1;
    for (std::uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
        a.cell_count[k] = 0u;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        const int nd = a.ndim;
        const int K = ctl->nclass > 1 ? ctl->nclass : 1;
        // per class: cells at least one largest-member cutoff wide
        long long nc[kMaxClass][kMaxDim];
        double cells_k[kMaxClass];
        double total = 0.0;
        for (int k = 0; k < K; ++k) {
            const double dmax = K > 1 ? xmul(ctl->class_d0max[k], ctl->build_kappa) : ctl->build_Dmax;
            const double cutoff = (dmax + ctl->build_t_shell) * (1.0 + 1e-6);
            cells_k[k] = 1.0;
            for (int d = 0; d < nd; ++d) {
                double q = floor(ctl->g.box[d] / cutoff);
                if (!(q >= 1.0)) q = 1.0;
                if (q > 1048576.0) q = 1048576.0;
                nc[k][d] = static_cast<long long>(q);
                cells_k[k] *= q;
            }
            total += cells_k[k];
        }
        // coarsen the class with the most cells until all fit
        while (total > static_cast<double>(a.C_alloc)) {
            int km = 0;
            for (int k = 1; k < K; ++k)
                if (cells_k[k] > cells_k[km]) km = k;
            int dm = 0;
            for (int d = 1; d < nd; ++d)
                if (nc[km][d] > nc[km][dm]) dm = d;
            const long long nn = (nc[km][dm] * 3) / 4;
            total -= cells_k[km];
            cells_k[km] = cells_k[km] / static_cast<double>(nc[km][dm]) * static_cast<double>(nn < 1 ? 1 : nn);
            total += cells_k[km];
            nc[km][dm] = nn < 1 ? 1 : nn;
            if (cells_k[km] <= 1.0 && total > static_cast<double>(a.C_alloc)) break;
        }
        std::uint32_t cells = 0;
        for (int k = 0; k < K; ++k) {
            ctl->cls_base[k] = cells;
            std::uint32_t ck = 1;
            for (int d = 0; d < nd; ++d) {
                ctl->cls_ncell[k][d] = static_cast<int>(nc[k][d]);
                ctl->cls_scale[k][d] = static_cast<double>(nc[k][d]) / ctl->g.box[d];
                ck *= static_cast<std::uint32_t>(nc[k][d]);
            }
            cells += ck;
        }
        ctl->cls_base[K] = cells;
        for (int d = 0; d < nd; ++d) {
            ctl->ncell[d] = ctl->cls_ncell[0][d];
            ctl->cell_scale[d] = ctl->cls_scale[0][d];
        }
        ctl->ncells = cells;
        // cell units of the cell-order kernels (one grid: class 0's)
        if (nd == 2 || nd == 3) {
            const double c0 = cells_k[0];
            const int nc0 = static_cast<int>(nc[0][0]);
            const std::uint32_t w = nd == 2 ? unit_width<2>(a.N, c0, nc0) : unit_width<3>(a.N, c0, nc0);
            const std::uint32_t chunks = (static_cast<std::uint32_t>(nc0) + w - 1) / w;
            std::uint32_t rows = static_cast<std::uint32_t>(nc[0][1]);
            if (nd == 3) rows *= static_cast<std::uint32_t>(nc[0][2]);
            ctl->unit_w = w;
            ctl->unit_chunks = chunks;
            ctl->unit_count = chunks * rows;
        } else {
            ctl->unit_w = ctl->unit_chunks = ctl->unit_count = 0u;
        }
        // 2-D tiles: kTileRowsPref cells high, lower where the halo's
        // particles at the mean cell occupancy (with 30 % headroom) would not
        // fit the staging area
        if (nd == 2) {
            const double ppc = static_cast<double>(a.N) / static_cast<double>(cells ? cells : 1u);
            const double fit = floor(static_cast<double>(kTileStage2) / (18.0 * 1.3 * (ppc > 1e-3 ? ppc : 1e-3))) - 2.0;
            double r = fit < static_cast<double>(kTileRowsPref) ? fit : static_cast<double>(kTileRowsPref);
            if (!(r >= kTileRowsMin)) r = kTileRowsMin;
            ctl->tile_rows = static_cast<int>(r);
        } else {
            ctl->tile_rows = 0;
        }
        // every rebuild re-anchors every particle (x_last is written by k_bin)
        ctl->kappa_min = ctl->build_kappa;
        // graph mode: the tiled build also computes this step's forces
        // (only with unsorted rows: a sorted row is summed after its sort)
        ctl->forces_done = a.sorted_rows ? 0u : ctl->fuse_forces;
        ctl->row_need = 0u;
        ctl->nbuilds += 1u;
    }
}

template <int ND>
__global__ void __launch_bounds__(256) k_build_bin(DevArrays a) {
    const DevCtl* ctl = a.ctl;
    if (build_off(ctl)) return;
    const std::uint64_t i = blockIdx.x * static_cast<std::uint64_t>(blockDim.x) + threadIdx.x;
    if (i >= a.N) return;
    bind_buffers(a);
    double x[ND], D0;
    load_pos<ND>(a.pos, i, x, D0);
    int k = 0;  // size class
    while (k + 1 < ctl->nclass && D0 >= ctl->class_d0[k + 1]) ++k;
    std::uint32_t c = ctl->cls_base[k], mul = 1;
#pragma unroll
    for (int d = 0; d < ND; ++d) {
        const int cd = cell_coord(x[d], ctl->cls_scale[k][d], ctl->cls_ncell[k][d]);
        c += static_cast<std::uint32_t>(cd) * mul;
        mul *= static_cast<std::uint32_t>(ctl->cls_ncell[k][d]);
        if (!a.permute) a.x_last[i * ND + d] = x[d];  // cell-order storage: the permutation writes it
    }
    a.cell_of[i] = c;
    a.cell_rank[i] = atomicAdd(&a.cell_count[c], 1u);
}

// Exclusive scan of n uint32 in tiles of 4096 (1024 threads x 4).
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

__global__ void __launch_bounds__(kScanThreads)
    k_scan_tiles(const std::uint32_t* in, std::uint32_t* out, std::uint32_t n,
                 std::uint32_t* block_sums, const DevCtl* gate) {
    if (gate && build_off(gate)) return;
    __shared__ std::uint32_t smem[32];
    const std::uint64_t base = static_cast<std::uint64_t>(blockIdx.x) * kScanTile + threadIdx.x * kScanItems;
    std::uint32_t v[kScanItems];
    std::uint32_t sum = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        v[k] = (base + k < n) ? in[base + k] : 0u;
        sum += v[k];
    }
    std::uint32_t total;
    std::uint32_t off = block_exclusive_scan(sum, smem, total);
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        if (base + k < n) out[base + k] = off;
        off += v[k];
    }
    if (threadIdx.x == 0 && block_sums) block_sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanThreads)
    k_scan_add(std::uint32_t* out, std::uint32_t n, const std::uint32_t* block_offsets,
               const DevCtl* gate) {
    if (gate && build_off(gate)) return;
    const std::uint32_t add = block_offsets[blockIdx.x];
    const std::uint64_t base = static_cast<std::uint64_t>(blockIdx.x) * kScanTile + threadIdx.x * kScanItems;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
        if (base + k < n) out[base + k] += add;
}

// Exclusive scan of n <= kScanTile^2 values, gated on a rebuild when gate != null.
void scan_exclusive(const std::uint32_t* in, std::uint32_t* out, std::uint32_t n,
                    std::uint32_t* tmp, const DevCtl* gate, cudaStream_t st) {
    const std::uint32_t tiles = (n + kScanTile - 1) / kScanTile;
    if (tiles > static_cast<std::uint32_t>(kScanTile)) throw std::length_error("rcpg scan: more than 4096^2 elements");
    if (tiles <= 1) {
        k_scan_tiles<<<1, kScanThreads, 0, st>>>(in, out, n, nullptr, gate);
        return;
    }
    k_scan_tiles<<<tiles, kScanThreads, 0, st>>>(in, out, n, tmp, gate);
    k_scan_tiles<<<1, kScanThreads, 0, st>>>(tmp, tmp + kScanTile, tiles, nullptr, gate);
    k_scan_add<<<tiles, kScanThreads, 0, st>>>(out, n, tmp + kScanTile, gate);
}

__global__ void __launch_bounds__(256) k_build_scatter(DevArrays a) {
    const DevCtl* ctl = a.ctl;
    if (build_off(ctl)) return;
    const std::uint64_t i = blockIdx.x * static_cast<std::uint64_t>(blockDim.x) + threadIdx.x;
    if (i >= a.N) return;
    a.cell_list[a.cell_start[a.cell_of[i]] + a.cell_rank[i]] = static_cast<std::uint32_t>(i);
}

template <int ND>
__device__ __forceinline__ bool tiled_build_ok(const DevCtl* ctl);

// Particles below which the tiled search is not used: a small packing has too
// few tiles to fill the GPU, and the warp search (k_build_search) spreads one
// particle over 32 lanes instead.
constexpr std::uint64_t kTiledMinN = 20000;

// the tiled search builds the rows (rows in particle order: exact mode and
// the stand-alone pair build)
template <int ND>
__device__ __forceinline__ bool use_tiled(const DevArrays& a) {
    return !a.permute && a.sorted_rows && (a.N >= kTiledMinN) && tiled_build_ok<ND>(a.ctl);
}

// the cell-unit search builds the rows (graph mode, ndim 2 and 3, one size
// class, at least 3 cells per axis)
template <int ND>
__device__ __forceinline__ bool use_cells(const DevArrays& a) {
    if (ND > 3 || !a.permute || a.N < kTiledMinN) return false;
    const DevCtl* ctl = a.ctl;
    bool ok = ctl->nclass <= 1;
    RCPG_UNROLL
    for (int d = 0; d < (ND <= 3 ? ND : 3); ++d) ok = ok & (ctl->ncell[d] >= 3);
    return ok;
}

// Builds without the tiled search: the members of each cell in ascending
// particle order in work (the atomic ranks of k_build_bin are arrival order;
// row slots and per-block force sums must not depend on it), and a copy of
// their positions in that order (spos), so the search reads each cell's
// candidates from contiguous memory. The tiled search orders its cells itself.
template <int ND>
__global__ void __launch_bounds__(256) k_build_cell_sort(DevArrays a) {
    const DevCtl* ctl = a.ctl;
    if (build_off(ctl) || use_tiled<ND>(a)) return;
    const std::uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ctl->ncells) return;
    const std::uint32_t q0 = a.cell_start[c], q1 = a.cell_start[c + 1];
    constexpr std::uint32_t kRegSort = 8;  // cells up to this size are sorted in registers
    if (q1 - q0 <= kRegSort) {
        // all members loaded at once, an odd-even transposition network over
        // kRegSort slots (empty slots hold the largest key), then the stores
        const std::uint32_t n = q1 - q0;
        std::uint32_t v[kRegSort];
        RCPG_UNROLL
        for (std::uint32_t k = 0; k < kRegSort; ++k) v[k] = k < n ? a.cell_list[q0 + k] : 0xFFFFFFFFu;
        if (n > 1) {
            RCPG_UNROLL
            for (std::uint32_t pass = 0; pass < kRegSort; ++pass) {
                RCPG_UNROLL
                for (std::uint32_t k = pass & 1u; k + 1 < kRegSort; k += 2) {
                    const std::uint32_t lo = min(v[k], v[k + 1]), hi = max(v[k], v[k + 1]);
                    v[k] = lo;
                    v[k + 1] = hi;
                }
            }
        }
        RCPG_UNROLL
        for (std::uint32_t k = 0; k < kRegSort; ++k)
            if (k < n) a.work[q0 + k] = v[k];
    } else {
        for (std::uint32_t k = q0; k < q1; ++k) {
            const std::uint32_t v = a.cell_list[k];
            std::uint32_t p = k;
            while (p > q0 && a.work[p - 1] > v) {
                a.work[p] = a.work[p - 1];
                --p;
            }
            a.work[p] = v;
        }
    }
    if (a.permute) return;  // cell-order storage: k_build_permute moves the particles themselves
    constexpr int P = pos_stride(ND);
    for (std::uint32_t q = q0; q < q1; ++q) {
        const double2* src = reinterpret_cast<const double2*>(a.pos + static_cast<std::uint64_t>(a.work[q]) * P);
        double2* dst = reinterpret_cast<double2*>(a.spos + static_cast<std::uint64_t>(q) * P);
        RCPG_UNROLL
        for (int h = 0; h < P / 2; ++h) dst[h] = src[h];
    }
}

// Cell-order storage (graph mode): particle q of the new order is particle
// work[q] of the current one (cells in grid order, each cell's members in
// their current order, written by k_build_cell_sort). Moves the per-particle
// state into the other buffer set, anchors the refresh trigger there
// (x_last = x, every build re-anchors every particle) and, once every block
// has finished (all have read the current set), flips DevCtl::buf.
template <int ND>
__global__ void __launch_bounds__(256) k_build_permute(DevArrays a) {
    DevCtl* ctl = a.ctl;
    if (build_off(ctl)) return;
    const std::uint32_t b = ctl->buf;
    const DevArrays src = bound_arrays(a, b), dst = bound_arrays(a, b ^ 1u);
    constexpr int P = pos_stride(ND);
    const std::uint64_t N = a.N;
    // two particles per thread, every load of both before any store
    const std::uint64_t stride = static_cast<std::uint64_t>(gridDim.x) * blockDim.x;
    for (std::uint64_t q0 = blockIdx.x * static_cast<std::uint64_t>(blockDim.x) + threadIdx.x; q0 < N;
         q0 += 2 * stride) {
        constexpr int U = 2;
        double2 rec[U][P / 2];
        double mv[U][2 * ND];
        std::uint64_t org[U];
        std::uint32_t cap[U], rr[U];
        RCPG_UNROLL
        for (int u = 0; u < U; ++u) {
            const std::uint64_t q = q0 + u * stride;
            if (q >= N) continue;
            const std::uint64_t o = a.work[q];
            const double2* ps = reinterpret_cast<const double2*>(src.pos + o * P);
            RCPG_UNROLL
            for (int h = 0; h < P / 2; ++h) rec[u][h] = ps[h];
            RCPG_UNROLL
            for (int d = 0; d < ND; ++d) {
                mv[u][d] = src.m[o * ND + d];
                mv[u][ND + d] = src.v[o * ND + d];
            }
            org[u] = src.origin[o];
            cap[u] = src.caps[o];
            rr[u] = src.ref_rank[o];
        }
        RCPG_UNROLL
        for (int u = 0; u < U; ++u) {
            const std::uint64_t q = q0 + u * stride;
            if (q >= N) continue;
            double2* pd = reinterpret_cast<double2*>(dst.pos + q * P);
            RCPG_UNROLL
            for (int h = 0; h < P / 2; ++h) {
                pd[h] = rec[u][h];
                if (2 * h < ND) a.x_last[q * ND + 2 * h] = rec[u][h].x;
                if (2 * h + 1 < ND) a.x_last[q * ND + 2 * h + 1] = rec[u][h].y;
            }
            RCPG_UNROLL
            for (int d = 0; d < ND; ++d) {
                dst.m[q * ND + d] = mv[u][d];
                dst.v[q * ND + d] = mv[u][ND + d];
            }
            dst.origin[q] = org[u];
            dst.caps[q] = cap[u];
            dst.ref_rank[q] = rr[u];
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const std::uint32_t done = atomicAdd(&ctl->permute_done, 1u);
        if (done == gridDim.x - 1) {
            ctl->permute_done = 0u;
            ctl->buf = b ^ 1u;
        }
    }
}

// Warp search (every build the tiled search does not take: ndim > 3, small
// packings, grids narrower than a tile). One warp per row slot t (particle
// work[t]). The neighbour cells are taken 32 at a time: each lane reads one
// cell's member range, a warp scan numbers the chunk's candidates, and the
// lanes test consecutive candidates (each finds its cell by a binary search
// over the lanes' ranges), so every lane has a candidate in every round
// whatever the cell occupancy. Accepted partners take row slots in candidate
// order (ballot + popc): the row is in a fixed scan order. Rows that must be
// sorted (sorted_rows: exact mode) are then sorted ascending by a bitonic
// sort in the warp.
constexpr int kWarpSearchWarps = 4;    // warps per block
constexpr int kWarpRowSmem = 256;      // row entries held (and sorted) in shared memory

template <int ND>
__global__ void __launch_bounds__(32 * kWarpSearchWarps) k_build_search(DevArrays a) {
    DevCtl* ctl = a.ctl;
    const std::uint64_t N = a.N;
    const bool other = use_tiled<ND>(a) || use_cells<ND>(a);
    if (a.cond_forces && blockIdx.x == 0 && threadIdx.x == 0 && !build_off(ctl)) {
        // last kernel of the build in a step graph: the pair kernel runs
        // unless another search computed this step's forces
        const std::uint32_t fd = other ? ctl->forces_done : 0u;
        cudaGraphSetConditional(a.cond_forces, forces_case(fd == 0u, ctl->pair_fp32, a.mixed));
    }
    if (build_off(ctl) || other) return;
    if (blockIdx.x == 0 && threadIdx.x == 0) ctl->forces_done = 0u;
    __shared__ std::uint32_t buf[kWarpSearchWarps][kWarpRowSmem];
    __shared__ std::uint32_t block_need;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (threadIdx.x == 0) block_need = 0u;
    __syncthreads();
    const std::uint32_t S = a.S;
    const Geometry& g = ctl->g;
    const double kap = ctl->build_kappa, t_shell = ctl->build_t_shell;
    double bx[ND], ibx[ND];
    RCPG_UNROLL
    for (int d = 0; d < ND; ++d) {
        bx[d] = g.box[d];
        ibx[d] = g.inv_box[d];
    }
    const int K = ctl->nclass > 1 ? ctl->nclass : 1;
    std::uint32_t* row = buf[w];
    // cell-order storage: slot t is particle t, and the cells' members are
    // contiguous in pos itself
    bind_buffers(a);
    const bool perm = a.permute != 0;
    const double* cpos = perm ? a.pos : a.spos;
    const std::uint64_t warps = static_cast<std::uint64_t>(gridDim.x) * kWarpSearchWarps;
    for (std::uint64_t t = blockIdx.x * static_cast<std::uint64_t>(kWarpSearchWarps) + w; t < N; t += warps) {
        const std::uint32_t i = perm ? static_cast<std::uint32_t>(t) : a.work[t];
        const std::uint32_t ri = perm ? a.ref_rank[i] : i;  // the reference's index (half-row count)
        double xi[ND], D0i;
        load_pos<ND>(cpos, t, xi, D0i);
        const double Di = xmul(D0i, kap);
        std::uint32_t n = 0, n_half = 0;  // n: warp-uniform row length so far
        // every grid: cells within the largest cutoff of particle i and a member
        // of the class (one cell for its own and smaller classes, more for
        // classes of smaller particles than i, whose cells are narrower)
        for (int kc = 0; kc < K; ++kc) {
            int nc[ND], nn[ND], lo[ND];
            int total_combo = 1;
            const double dmax = K > 1 ? xmul(ctl->class_d0max[kc], kap) : ctl->build_Dmax;
            const double rcut = (Di + dmax) * 0.5 + t_shell;
            RCPG_UNROLL
            for (int d = 0; d < ND; ++d) {
                const double scale = ctl->cls_scale[kc][d];
                nc[d] = ctl->cls_ncell[kc][d];
                // cells per cutoff on this axis: 1 with one grid (cells are at
                // least one cutoff wide), computed per class otherwise
                double mm = 1.0;
                if (K > 1) {
                    mm = ceil(rcut * scale * (1.0 + 1e-6));
                    if (!(mm >= 1.0)) mm = 1.0;
                }
                if (!(2.0 * mm + 1.0 <= static_cast<double>(nc[d]))) {
                    nn[d] = nc[d];  // every cell of the axis, once
                    lo[d] = 0;
                } else {
                    const int m = static_cast<int>(mm);
                    nn[d] = 2 * m + 1;
                    lo[d] = cell_coord(xi[d], scale, nc[d]) - m;
                }
                total_combo *= nn[d];
            }
            const std::uint32_t base = ctl->cls_base[kc];
            for (int cb = 0; cb < total_combo; cb += 32) {
                // this lane's cell of the chunk and its member range
                const int combo = cb + lane;
                std::uint32_t q0 = 0, cntc = 0;
                if (combo < total_combo) {
                    std::uint32_t cell = base, mul = 1;
                    int r = combo;
                    RCPG_UNROLL
                    for (int d = 0; d < ND; ++d) {
                        const int kk = r % nn[d];
                        r /= nn[d];
                        int c = lo[d] + kk;
                        if (c < 0) c += nc[d];
                        else if (c >= nc[d]) c -= nc[d];
                        cell += static_cast<std::uint32_t>(c) * mul;
                        mul *= static_cast<std::uint32_t>(nc[d]);
                    }
                    q0 = a.cell_start[cell];
                    cntc = a.cell_start[cell + 1] - q0;
                }
                // inclusive scan of the member counts over the lanes
                std::uint32_t incl = cntc;
                RCPG_UNROLL
                for (int o = 1; o < 32; o <<= 1) {
                    const std::uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl += v;
                }
                const std::uint32_t tot = __shfl_sync(0xffffffffu, incl, 31);
                for (std::uint32_t k0 = 0; k0 < tot; k0 += 32) {
                    const std::uint32_t k = k0 + lane;
                    bool ok = false;
                    std::uint32_t j = 0;
                    // owner lane of candidate k: the first lane whose inclusive
                    // count exceeds k (5-step search over the lanes)
                    int s_lo = 0;
                    RCPG_UNROLL
                    for (int step = 16; step > 0; step >>= 1) {
                        const std::uint32_t v = __shfl_sync(0xffffffffu, incl, s_lo + step - 1);
                        if (v <= k) s_lo += step;
                    }
                    const int own = s_lo < 31 ? s_lo : 31;
                    const std::uint32_t own_q0 = __shfl_sync(0xffffffffu, q0, own);
                    const std::uint32_t own_incl = __shfl_sync(0xffffffffu, incl, own);
                    const std::uint32_t own_cnt = __shfl_sync(0xffffffffu, cntc, own);
                    if (k < tot) {
                        const std::uint32_t q = own_q0 + (k - (own_incl - own_cnt));
                        j = perm ? q : a.work[q];
                        if (j != i) {
                            double xj[ND], D0j;
                            load_pos<ND>(cpos, q, xj, D0j);
                            const double Dj = xmul(D0j, kap);
                            ok = (ND <= 3 || j > i) ? in_shell<ND>(xi, xj, Di, Dj, bx, ibx, t_shell)
                                                    : in_shell<ND>(xi, xj, Dj, Di, bx, ibx, t_shell);
                        }
                    }
                    // row slots in candidate order
                    const unsigned mask = __ballot_sync(0xffffffffu, ok);
                    if (ok) {
                        const std::uint32_t slot = n + __popc(mask & ((1u << lane) - 1u));
                        if (slot < static_cast<std::uint32_t>(kWarpRowSmem)) row[slot] = j;
                        else if (slot < S) a.nbr[static_cast<std::uint64_t>(slot) * N + t] = j;
                        if (perm ? (a.ref_rank[j] > ri) : (j > i)) ++n_half;
                    }
                    n += static_cast<std::uint32_t>(__popc(mask));
                }
            }
        }
        __syncwarp();
        RCPG_UNROLL
        for (int o = 16; o > 0; o >>= 1) n_half += __shfl_xor_sync(0xffffffffu, n_half, o);
        if (lane == 0) {
            const std::uint32_t cap = a.caps[i];
            if (n_half > cap) report_cap_error(ctl, ri, cap);
            atomicMax(&block_need, n);
            a.nbr_cnt[t] = n > S ? 0u : n;  // overflow: empty row, rebuilt after the capacity grows
        }
        if (n > S) continue;
        if (!a.sorted_rows) {
            // scan-order row: the shared part goes out as it is
            const std::uint32_t ns = n < static_cast<std::uint32_t>(kWarpRowSmem) ? n : kWarpRowSmem;
            for (std::uint32_t e = lane; e < ns; e += 32) a.nbr[static_cast<std::uint64_t>(e) * N + t] = row[e];
        } else if (n <= static_cast<std::uint32_t>(kWarpRowSmem)) {
            // bitonic sort of the row padded to a power of two
            std::uint32_t p2 = 1;
            while (p2 < n) p2 <<= 1;
            for (std::uint32_t e = n + lane; e < p2; e += 32) row[e] = 0xffffffffu;
            __syncwarp();
            for (std::uint32_t kk = 2; kk <= p2; kk <<= 1) {
                for (std::uint32_t jj = kk >> 1; jj > 0; jj >>= 1) {
                    for (std::uint32_t e = lane; e < p2; e += 32) {
                        const std::uint32_t f = e ^ jj;
                        if (f > e) {
                            const std::uint32_t x = row[e], y = row[f];
                            const bool up = (e & kk) == 0;
                            if ((x > y) == up) {
                                row[e] = y;
                                row[f] = x;
                            }
                        }
                    }
                    __syncwarp();
                }
            }
            for (std::uint32_t e = lane; e < n; e += 32) a.nbr[static_cast<std::uint64_t>(e) * N + t] = row[e];
        } else if (lane == 0) {
            // longer than the shared buffer: the row in global memory, sorted there
            for (std::uint32_t e = 0; e < static_cast<std::uint32_t>(kWarpRowSmem); ++e)
                a.nbr[static_cast<std::uint64_t>(e) * N + t] = row[e];
            std::uint32_t* gr = a.nbr + t;
            for (std::uint32_t k = 1; k < n; ++k) {
                const std::uint32_t v = gr[static_cast<std::uint64_t>(k) * N];
                std::uint32_t p = k;
                while (p > 0 && gr[static_cast<std::uint64_t>(p - 1) * N] > v) {
                    gr[static_cast<std::uint64_t>(p) * N] = gr[static_cast<std::uint64_t>(p - 1) * N];
                    --p;
                }
                gr[static_cast<std::uint64_t>(p) * N] = v;
            }
        }
        __syncwarp();
    }
    __syncthreads();
    if (threadIdx.x == 0 && block_need) atomicMax(&ctl->row_need, block_need);
}

// ---- tiled search (ndim 2, 3) ---------------------------------------------
// One block per tile of cells (persistent over tiles). The particles of the
// tile and of its one-cell halo are staged in shared memory (positions, ids,
// row slots, local cell), then every particle of the tile tests its 3^ndim
// neighbour cells from shared memory only. Used when every axis has at least
// tile + 2 cells (no cell of the halo is loaded twice); otherwise, and for
// ndim > 3, k_build_search handles the build.
// 2-D tiles are 16 cells wide and ctl->tile_rows (kTileRowsMin..kTileRowsMax)
// high; t(1) is the largest height.
template <int ND> struct TileShape;
template <> struct TileShape<2> {
    __host__ __device__ static constexpr int t(int d) { return d == 0 ? 16 : kTileRowsMax; }
    static constexpr int halo_cells = 18 * (kTileRowsMax + 2);
    static constexpr int stage = kTileStage2;
};
template <> struct TileShape<3> {
    __host__ __device__ static constexpr int t(int) { return 4; }
    static constexpr int halo_cells = 6 * 6 * 6;
    static constexpr int stage = 1280;
};
constexpr int kTileThreads = 256;
constexpr int kTileRow = 32;  // staged row entries per thread

// dynamic shared memory of k_build_search_tiled<ND>: staged records, ids, row
// slots, halo cell offsets, inner list, local cells, then the staged rows
template <int ND>
constexpr std::size_t tile_smem_bytes() {
    using TS = TileShape<ND <= 3 ? ND : 3>;
    return static_cast<std::size_t>(TS::stage) * pos_stride(ND) * 8 + 2ull * TS::stage * 4 +
           (TS::halo_cells + 2) * 4 + 2ull * TS::stage * 2 + static_cast<std::size_t>(kTileRow) * kTileThreads * 2;
}

template <int ND>
__device__ __forceinline__ bool tiled_build_ok(const DevCtl* ctl) {
    if (ND > 3) return false;
    bool ok = ctl->nclass <= 1;
    RCPG_UNROLL
    for (int d = 0; d < (ND <= 3 ? ND : 3); ++d)
        ok = ok & (ctl->ncell[d] >= (ND == 2 && d == 1 ? ctl->tile_rows : TileShape<(ND <= 3 ? ND : 3)>::t(d)) + 2);
    return ok;
}

// Sorts a row gathered partly in shared memory (column `mine`, stride kTileThreads)
// and partly in the global row, and writes it to row slot q.
__device__ __forceinline__ void finish_row(std::uint32_t* mine, int stride, int smem_cap,
                                           std::uint32_t n, std::uint32_t S, std::uint32_t* nbr,
                                           std::uint32_t* nbr_cnt, std::uint64_t N, std::uint64_t q) {
    if (n > S) {
        // overflow: the row is incomplete. It is published empty, so that no
        // reader can meet an unwritten entry; the build reports row_need > S
        // and the caller rebuilds with a larger row capacity.
        nbr_cnt[q] = 0;
        return;
    }
    nbr_cnt[q] = n;
    if (smem_cap > 0 && n <= static_cast<std::uint32_t>(smem_cap)) {
        for (std::uint32_t k = 1; k < n; ++k) {
            const std::uint32_t v = mine[k * stride];
            std::uint32_t p = k;
            while (p > 0 && mine[(p - 1) * stride] > v) {
                mine[p * stride] = mine[(p - 1) * stride];
                --p;
            }
            mine[p * stride] = v;
        }
        for (std::uint32_t k = 0; k < n; ++k) nbr[static_cast<std::uint64_t>(k) * N + q] = mine[k * stride];
    } else {
        for (std::uint32_t k = 0; k < static_cast<std::uint32_t>(smem_cap); ++k)
            nbr[static_cast<std::uint64_t>(k) * N + q] = mine[k * stride];
        std::uint32_t* row = nbr + q;  // insertion sort of the whole row in place
        for (std::uint32_t k = 1; k < n; ++k) {
            const std::uint32_t v = row[static_cast<std::uint64_t>(k) * N];
            std::uint32_t p = k;
            while (p > 0 && row[static_cast<std::uint64_t>(p - 1) * N] > v) {
                row[static_cast<std::uint64_t>(p) * N] = row[static_cast<std::uint64_t>(p - 1) * N];
                --p;
            }
            row[static_cast<std::uint64_t>(p) * N] = v;
        }
    }
}

// Rows sorted by partner index (exact mode, rcpg_pairs_full): the reference's
// summation order. Particles stay in their own order; row slots follow the
// cells (work[q] = particle of slot q).
template <int ND>
__global__ void __launch_bounds__(kTileThreads, 3) k_build_search_tiled(DevArrays a) {
    constexpr int NDT = ND <= 3 ? ND : 3;
    using TS = TileShape<NDT>;
    constexpr int P = pos_stride(ND);
    constexpr int STAGE = TS::stage;
    constexpr int HC = TS::halo_cells;
    DevCtl* ctl = a.ctl;
    if (ND > 3) return;
    if (build_off(ctl) || !use_tiled<ND>(a)) return;
    extern __shared__ __align__(16) unsigned char tile_smem[];
    double* s_pos = reinterpret_cast<double*>(tile_smem);
    std::uint32_t* s_id = reinterpret_cast<std::uint32_t*>(s_pos + STAGE * P);
    std::uint32_t* s_slot = s_id + STAGE;
    std::uint32_t* s_cstart = s_slot + STAGE;
    std::uint16_t* s_inner = reinterpret_cast<std::uint16_t*>(s_cstart + HC + 2);
    std::uint16_t* s_cell = s_inner + STAGE;
    std::uint16_t* s_rows = s_cell + STAGE;  // [kTileRow][kTileThreads] staged row entries
    __shared__ unsigned long long s_warp2[kTileThreads / 32];
    __shared__ std::uint32_t s_need, s_ninner;
    const std::uint64_t N = a.N;
    const std::uint32_t S = a.S;
    // box of the minimum image in shared memory (the loops store through other
    // pointers, so loads through ctl would be repeated)
    __shared__ double bx[ND], ibx[ND];
    if (threadIdx.x < ND) {
        bx[threadIdx.x] = ctl->g.box[threadIdx.x];
        ibx[threadIdx.x] = ctl->g.inv_box[threadIdx.x];
    }
    const double kap = ctl->build_kappa, t_shell = ctl->build_t_shell;
    int nc[ND], nt[ND];
    // tile extent per axis (the 2-D height is chosen per build)
    __shared__ int s_ts[ND];
    std::uint32_t tiles = 1;
    RCPG_UNROLL
    for (int d = 0; d < ND; ++d) {
        nc[d] = ctl->ncell[d];
        const int tsd = (ND == 2 && d == 1) ? ctl->tile_rows : TS::t(d);
        if (threadIdx.x == 0) s_ts[d] = tsd;
        nt[d] = (nc[d] + tsd - 1) / tsd;
        tiles *= static_cast<std::uint32_t>(nt[d]);
    }
    __syncthreads();  // s_ts, bx, ibx
    if (threadIdx.x == 0) s_need = 0u;
    std::uint16_t* mine = s_rows + threadIdx.x;
    for (std::uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        int t0[ND], hw[ND];
        std::uint32_t rem = tile;
        int H = 1;
        RCPG_UNROLL
        for (int d = 0; d < ND; ++d) {
            const int tc = static_cast<int>(rem % static_cast<std::uint32_t>(nt[d]));
            rem /= static_cast<std::uint32_t>(nt[d]);
            t0[d] = tc * s_ts[d];
            const int tw = min(s_ts[d], nc[d] - t0[d]);
            hw[d] = tw + 2;
            H *= hw[d];
        }
        __syncthreads();  // the previous tile is done with shared memory
        // 1. particle count of every halo cell, 2. block scans -> staging offsets
        std::uint32_t cs = 0, cnt = 0;
        bool inner_cell = false;
        if (static_cast<int>(threadIdx.x) < H) {
            int r = threadIdx.x;
            std::uint32_t c = 0, mul = 1;
            inner_cell = true;
            RCPG_UNROLL
            for (int d = 0; d < ND; ++d) {
                const int l = r % hw[d];
                r /= hw[d];
                inner_cell = inner_cell && l >= 1 && l <= hw[d] - 2;
                int gc = t0[d] - 1 + l;
                if (gc < 0) gc += nc[d];
                else if (gc >= nc[d]) gc -= nc[d];
                c += static_cast<std::uint32_t>(gc) * mul;
                mul *= static_cast<std::uint32_t>(nc[d]);
            }
            cs = a.cell_start[c];
            cnt = a.cell_start[c + 1] - cs;
        }
        // one scan of (inner count << 32 | count): staging offsets and inner-list offsets
        unsigned long long tot2;
        const unsigned long long off2 = block_exclusive_scan<unsigned long long>(
            (static_cast<unsigned long long>(inner_cell ? cnt : 0u) << 32) | cnt, s_warp2, tot2);
        const std::uint32_t off = static_cast<std::uint32_t>(off2), total = static_cast<std::uint32_t>(tot2);
        const std::uint32_t ioff = static_cast<std::uint32_t>(off2 >> 32), ninner = static_cast<std::uint32_t>(tot2 >> 32);
        if (static_cast<int>(threadIdx.x) < H) s_cstart[threadIdx.x] = off;
        if (threadIdx.x == 0) {
            s_cstart[H] = total;
            s_ninner = ninner;
        }
        const bool fits = total <= static_cast<std::uint32_t>(STAGE);
        // 3. stage the halo particles (one thread per halo cell) and list the tile's own
        if (fits && static_cast<int>(threadIdx.x) < H) {
            // the cell's members in ascending particle order (the bin's atomic
            // ranks are arrival order); the owner tile of a cell publishes that
            // order as the cell's row slots (work)
            std::uint32_t* ids = s_id + off;
            for (std::uint32_t k = 0; k < cnt; ++k) {
                const std::uint32_t v = a.cell_list[cs + k];
                std::uint32_t p = k;
                while (p > 0 && ids[p - 1] > v) {
                    ids[p] = ids[p - 1];
                    --p;
                }
                ids[p] = v;
            }
            for (std::uint32_t k = 0; k < cnt; ++k) {
                const std::uint32_t q = cs + k, dst = off + k;
                const std::uint32_t id = ids[k];
                const double2* src = reinterpret_cast<const double2*>(a.pos + static_cast<std::uint64_t>(id) * P);
                double2* sp = reinterpret_cast<double2*>(s_pos + dst * P);
                RCPG_UNROLL
                for (int h = 0; h < P / 2; ++h) sp[h] = src[h];
                s_slot[dst] = q;
                s_cell[dst] = static_cast<std::uint16_t>(threadIdx.x);
                if (inner_cell) {
                    s_inner[ioff + k] = static_cast<std::uint16_t>(dst);
                    a.work[q] = id;
                }
            }
        }
        __syncthreads();
        if (!fits) {
            // more halo particles than the staging area: rows of this tile from
            // global memory
            for (int h = threadIdx.x; h < H; h += blockDim.x) {
                int hl[ND];
                int r = h;
                bool inner = true;
                RCPG_UNROLL
                for (int d = 0; d < ND; ++d) {
                    hl[d] = r % hw[d];
                    r /= hw[d];
                    inner = inner && hl[d] >= 1 && hl[d] <= hw[d] - 2;
                }
                if (!inner) continue;
                std::uint32_t c = 0, mul = 1;
                RCPG_UNROLL
                for (int d = 0; d < ND; ++d) {
                    c += static_cast<std::uint32_t>(t0[d] - 1 + hl[d]) * mul;
                    mul *= static_cast<std::uint32_t>(nc[d]);
                }
                // this tile owns the cell: its members in ascending order as row slots
                const std::uint32_t q0 = a.cell_start[c], q1 = a.cell_start[c + 1];
                for (std::uint32_t k = q0; k < q1; ++k) {
                    const std::uint32_t v = a.cell_list[k];
                    std::uint32_t p = k;
                    while (p > q0 && a.work[p - 1] > v) {
                        a.work[p] = a.work[p - 1];
                        --p;
                    }
                    a.work[p] = v;
                }
                for (std::uint32_t q = q0; q < q1; ++q) {
                    const std::uint32_t i = a.work[q];
                    double xi[ND], D0i;
                    load_pos<ND>(a.pos, i, xi, D0i);
                    const double Di = xmul(D0i, kap);
                    std::uint32_t n = 0, n_half = 0;
                    int odo[ND];
                    RCPG_UNROLL
                    for (int d = 0; d < ND; ++d) odo[d] = 0;
                    constexpr int NCOMBO = (ND == 2) ? 9 : 27;
                    for (int combo = 0; combo < NCOMBO; ++combo) {
                        std::uint32_t cn = 0, mm = 1;
                        RCPG_UNROLL
                        for (int d = 0; d < ND; ++d) {
                            int gc = t0[d] - 1 + hl[d] - 1 + odo[d];
                            if (gc < 0) gc += nc[d];
                            else if (gc >= nc[d]) gc -= nc[d];
                            cn += static_cast<std::uint32_t>(gc) * mm;
                            mm *= static_cast<std::uint32_t>(nc[d]);
                        }
                        RCPG_UNROLL
                        for (int d = 0; d < ND; ++d) {
                            if (++odo[d] < 3) break;
                            odo[d] = 0;
                        }
                        for (std::uint32_t pp = a.cell_start[cn]; pp < a.cell_start[cn + 1]; ++pp) {
                            const std::uint32_t j = a.cell_list[pp];  // any order: the row is sorted at the end
                            if (j == i) continue;
                            double xj[ND], D0j;
                            load_pos<ND>(a.pos, j, xj, D0j);
                            if (!in_shell<ND>(xi, xj, Di, xmul(D0j, kap), bx, ibx, t_shell)) continue;
                            if (n < S) a.nbr[static_cast<std::uint64_t>(n) * N + q] = j;
                            ++n;
                            if (j > i) ++n_half;
                        }
                    }
                    const std::uint32_t cap = a.caps[i];
                    if (n_half > cap) report_cap_error(ctl, i, cap);
                    atomicMax(&s_need, n);
                    finish_row(nullptr, 0, 0, n, S, a.nbr, a.nbr_cnt, N, q);
                }
            }
            continue;
        }
        // 4. rows of the tile's own particles from shared memory
        for (std::uint32_t u = threadIdx.x; u < s_ninner; u += blockDim.x) {
            const std::uint32_t k = s_inner[u];
            int hl[ND];
            {
                int r = s_cell[k];
                RCPG_UNROLL
                for (int d = 0; d < ND; ++d) {
                    hl[d] = r % hw[d];
                    r /= hw[d];
                }
            }
            const std::uint32_t i = s_id[k];
            const std::uint64_t q = s_slot[k];
            double xi[ND], D0i;
            load_pos<ND>(s_pos, k, xi, D0i);
            const double Di = xmul(D0i, kap);
            std::uint32_t n = 0, n_half = 0;
            // the cells x-1, x, x+1 of one halo row are consecutive halo cells,
            // so their staged particles form one contiguous range: 3^(ndim-1)
            // ranges, visited in the order of the 3^ndim cells (axis 0 fastest)
            constexpr int NROW = (ND == 2) ? 3 : 9;
            const int hbase = hl[0] - 1 + (ND == 2 ? (hl[1] - 1) * hw[0]
                                                   : (hl[1] - 1) * hw[0] + (hl[ND - 1] - 1) * hw[0] * hw[1]);
            for (int rr = 0; rr < NROW; ++rr) {
                const int hc = hbase + (rr % 3) * hw[0] + (ND == 2 ? 0 : (rr / 3) * hw[0] * hw[1]);
                const std::uint32_t p0 = s_cstart[hc], p1 = s_cstart[hc + 3];
                for (std::uint32_t pp = p0; pp < p1; ++pp) {
                    if (pp == k) continue;
                    double xj[ND], D0j;
                    load_pos<ND>(s_pos, pp, xj, D0j);
                    const double Dj = xmul(D0j, kap);
                    double dx[ND];
                    const double d2 = pair_disp<ND>(xi, xj, bx, ibx, dx);
                    const double r_c = shell_cut<ND>(Di, Dj, t_shell);  // ndim <= 3: symmetric
                    if (!(d2 < xmul(r_c, r_c))) continue;
                    const std::uint32_t j = s_id[pp];
                    if (n < static_cast<std::uint32_t>(kTileRow)) mine[n * kTileThreads] = static_cast<std::uint16_t>(pp);
                    else if (n < S) a.nbr[static_cast<std::uint64_t>(n) * N + q] = j;
                    ++n;
                    if (j > i) ++n_half;
                }
            }
            const std::uint32_t cap = a.caps[i];
            if (n_half > cap) report_cap_error(ctl, i, cap);
            atomicMax(&s_need, n);
            if (n > S) {
                a.nbr_cnt[q] = 0;  // overflow: empty row, rebuilt after the capacity grows
                continue;
            }
            if (n <= static_cast<std::uint32_t>(kTileRow)) {
                // sort the staged indices by particle id, write the row
                for (std::uint32_t e = 1; e < n; ++e) {
                    const std::uint16_t v = mine[e * kTileThreads];
                    const std::uint32_t vid = s_id[v];
                    std::uint32_t p = e;
                    while (p > 0 && s_id[mine[(p - 1) * kTileThreads]] > vid) {
                        mine[p * kTileThreads] = mine[(p - 1) * kTileThreads];
                        --p;
                    }
                    mine[p * kTileThreads] = v;
                }
                a.nbr_cnt[q] = n;
                for (std::uint32_t e = 0; e < n; ++e)
                    a.nbr[static_cast<std::uint64_t>(e) * N + q] = s_id[mine[e * kTileThreads]];
            } else {
                // long row (kTileRow < n <= S): the first kTileRow entries go to
                // the global row too, sorted there
                for (std::uint32_t e = 0; e < static_cast<std::uint32_t>(kTileRow); ++e)
                    a.nbr[static_cast<std::uint64_t>(e) * N + q] = s_id[mine[e * kTileThreads]];
                finish_row(nullptr, 0, 0, n, S, a.nbr, a.nbr_cnt, N, q);
            }
        }
    }
    __syncthreads();
    if (threadIdx.x == 0 && s_need) atomicMax(&ctl->row_need, s_need);
}

// ---- cell units: the cell-order search (graph mode) -------------------------
// With cell-order storage the members of consecutive cells of one grid row
// are one contiguous range of particles. A unit is a chunk of unit_w
// consecutive cells of one grid row (2-D: row y; 3-D: row (y, z)), sized by
// each build so that it holds about UnitShape::target particles and its
// windows fit the stage. A block takes one unit at a time:
//   1. the cell_start entries of the unit's 3^(ndim-1) neighbour rows: cells
//      cx0-1 .. cx1 of each (the main window), plus, where the unit touches
//      the end of the grid row, the cell at the row's other end (the wrapped
//      x-1 / x+1 cell);
//   2. the FP64 records of those windows -- contiguous ranges of pos -- into
//      shared memory, with coalesced 256-bit loads by the whole block (2-D:
//      the record's spare slot takes the FP32 diameter of the mixed test);
//   3. one thread per particle of the unit tests its candidates from shared
//      memory (windows that do not fit the stage are read from pos instead:
//      the same code instantiated for global records).
// A particle's candidates in scan order: the cells x-1, x, x+1 of each
// neighbour row, rows in order (row offset r = (dy+1) + 3 (dz+1)), then the
// wrapped cell of each row where the particle sits at the row's end (2-D: the
// three rows' ranges are walked as one sequence, so the lanes of a warp run
// about as many rounds as their longest candidate list, and each round probes
// two candidates before committing them in order). Each goes through
// the reference's predicate in FP64, or (MX) the mixed-precision shell test
// (FP32 on FP64 differences, widened by kShellMarginF so that the rows hold
// every pair of the FP64 shell); rows hold the partners in that order and the
// step's forces are computed in the same pass, summed in row order with the
// arithmetic of k_forces (which gives the same forces on these rows bit for
// bit). MX: each variant returns at once when the step's pair precision is
// the other one.

// 32-byte particle record (ndim <= 3) from global memory, one 256-bit load
__device__ __forceinline__ void ld_record(const double* p, double2& lo, double2& hi) {
    asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];"
        : "=d"(lo.x), "=d"(lo.y), "=d"(hi.x), "=d"(hi.y)
        : "l"(p));
}

template <int ND>
__device__ __forceinline__ void unpack_record(const double2& lo, const double2& hi, double* x, double& D0) {
    x[0] = lo.x;
    x[1] = lo.y;
    if constexpr (ND == 3) {
        x[2] = hi.x;
        D0 = hi.y;
    } else {
        D0 = hi.x;
    }
}

// FP32 diameter kept in the spare slot of a staged 2-D record
__device__ __forceinline__ double pack_f32(float f) {
    return __longlong_as_double(static_cast<long long>(__float_as_uint(f)));
}
__device__ __forceinline__ float unpack_f32(double d) {
    return __uint_as_float(static_cast<unsigned>(__double_as_longlong(d)));
}

// One particle's candidate tests and its pair sums in the arithmetic of
// k_forces: FP32 (MX) or FP64 accumulators for the pair scalars, the force in
// FP32 (MX) or FP64.
template <int ND, bool MX>
struct UnitPair {
    using Acc = std::conditional_t<MX, float, double>;
    double xi[ND], Di, kap;
    float Dif, kapf;
    double fi[ND];
    float fif[ND];
    Acc sU, sLc, sdk, sFm, smax;
    std::uint32_t scount;

    __device__ __forceinline__ void begin(const double* x, double D0, double k) {
        kap = k;
        kapf = static_cast<float>(k);
        Di = xmul(D0, k);
        Dif = static_cast<float>(D0) * kapf;
        RCPG_UNROLL
        for (int d = 0; d < ND; ++d) {
            xi[d] = x[d];
            fi[d] = 0.0;
            fif[d] = 0.0f;
        }
        sU = sLc = sdk = sFm = smax = Acc(0);
        scount = 0;
    }

    // The tests of one candidate (xj, D0j; D0jf = its FP32 diameter), kept
    // for commit(): the displacement, its square and the pair's r_ij; pass =
    // the shell test, ov = overlapping (with `fuse`; an overlapping pair also
    // passes the shell test). Two candidates are probed side by side and
    // committed in scan order.
    struct Probe {
        using T = std::conditional_t<MX, float, double>;
        T dx[ND], d2, r;
        bool pass, ov;
    };
    __device__ __forceinline__ void probe(Probe& pr, const double* xj, double D0j, float D0jf, const double* bx,
                                          const double* ibx, const float* hbf, double t_shell, float tf,
                                          bool fuse) const {
        if constexpr (MX) {
            pr.d2 = mixed_disp<ND>(xi, xj, bx, hbf, pr.dx);
            pr.r = 0.5f * (Dif + D0jf * kapf);
            const float rc = pr.r + tf;
            pr.pass = pr.d2 < rc * rc * kShellMarginF;
            pr.ov = fuse && pr.d2 < pr.r * pr.r;
        } else {
            const double Dj = xmul(D0j, kap);
            pr.d2 = pair_disp<ND>(xi, xj, bx, ibx, pr.dx);
            const double r_c = shell_cut<ND>(Di, Dj, t_shell);  // ndim <= 3: symmetric
            pr.pass = pr.d2 < xmul(r_c, r_c);
            pr.r = xmul(0.5, xadd(Di, Dj));
            pr.ov = fuse && pr.d2 < xmul(pr.r, pr.r);
        }
    }
    // The pair terms of a probed overlapping pair; the scalars once per pair
    // (from the lower index).
    __device__ __forceinline__ void commit(bool upper, const Probe& pr) {
        if (!pr.ov) return;
        if constexpr (MX) {
            PairTermsF pf;
            pair_terms_mixed_f<ND>(pr.dx, pr.d2, pr.r, fif, pf);
            if (upper) {
                sU += pf.U;
                sLc += pf.Lc;
                sdk += pf.dk;
                sFm += pf.Fm;
                smax = fmaxf(smax, pf.U);
                ++scount;
            }
        } else {
            PairTerms pt;
            pair_terms_f64<ND>(pr.dx, pr.d2, pr.r, fi, pt);
            if (upper) {
                sU = xadd(sU, pt.U);
                sLc = xadd(sLc, pt.Lc);
                sdk = xadd(sdk, pt.dk);
                sFm = xadd(sFm, pt.Fm);
                smax = fmax(smax, pt.U);
                ++scount;
            }
        }
    }
    // One candidate probed and committed: whether it is a partner.
    __device__ __forceinline__ bool candidate(bool upper, const double* xj, double D0j, float D0jf,
                                              const double* bx, const double* ibx, const float* hbf,
                                              double t_shell, float tf, bool fuse) {
        Probe pr;
        probe(pr, xj, D0j, D0jf, bx, ibx, hbf, t_shell, tf, fuse);
        if (!pr.pass) return false;
        commit(upper, pr);
        return true;
    }

    __device__ __forceinline__ void force(double* f) const {
        RCPG_UNROLL
        for (int d = 0; d < ND; ++d) f[d] = MX ? static_cast<double>(fif[d]) : fi[d];
    }
};

template <int ND, bool MX>
__global__ void __launch_bounds__(UnitShape<ND>::threads, UnitShape<ND>::min_blocks) k_cells(DevArrays a) {
    using US = UnitShape<ND>;
    constexpr int NDC = US::ndc, R = US::rows, T = US::threads, NW = US::windows;
    constexpr int CR = NDC == 2 ? 1 : 4;  // row offset of the unit's own row
    DevCtl* ctl = a.ctl;
    if (build_off(ctl) || !use_cells<ND>(a) || MX != (ctl->pair_fp32 != 0u)) return;
    bind_buffers(a);
    extern __shared__ __align__(16) double u_stage[];  // [US::stage][4]: the staged records
    std::uint32_t* s_cs = reinterpret_cast<std::uint32_t*>(u_stage + 4 * US::stage);  // [R][US::slice]
    // windows, flat index w = 3 r + kind (0 main, 1 wrapped x-1, 2 wrapped x+1):
    // first particle, length, index of the first record in the stage (or in
    // pos, for a unit that is not staged)
    __shared__ std::uint32_t s_wb[NW], s_wl[NW], s_ws[NW];
    __shared__ std::uint32_t s_qa, s_qb, s_total, s_need;
    __shared__ ForceSums s_red[T / 32];
    // the thread's column of the block sums (its particles in order), in
    // shared memory: they change once per particle
    __shared__ double s_acc[7][T];
    __shared__ std::uint32_t s_accn[2][T];
    const std::uint64_t N = a.N;
    const std::uint32_t S = a.S;
    const Geometry& g = ctl->g;
    double bx[ND], ibx[ND];
    float hbf[ND];
    RCPG_UNROLL
    for (int d = 0; d < ND; ++d) {
        bx[d] = g.box[d];
        ibx[d] = g.inv_box[d];
        hbf[d] = static_cast<float>(0.5 * g.box[d]);
    }
    int nc[NDC];
    RCPG_UNROLL
    for (int d = 0; d < NDC; ++d) nc[d] = ctl->ncell[d];
    const double scale0 = ctl->cell_scale[0];
    const std::uint32_t W = ctl->unit_w, chunks = ctl->unit_chunks, units = ctl->unit_count;
    const double kap = ctl->build_kappa;
    const double t_shell = ctl->build_t_shell;
    const float tf = static_cast<float>(t_shell);
    const bool fuse = ctl->forces_done != 0u;
    if (blockIdx.x == 0 && threadIdx.x == 0 && fuse) ctl->nsum_blocks = gridDim.x;
    if (threadIdx.x == 0) s_need = 0u;
    const int col = threadIdx.x;
    RCPG_UNROLL
    for (int f = 0; f < 7; ++f) s_acc[f][col] = 0.0;
    s_accn[0][col] = s_accn[1][col] = 0u;
    std::uint32_t need = 0;
    bool overflow = false;
    for (std::uint32_t u = blockIdx.x; u < units; u += gridDim.x) {
        const std::uint32_t row0 = u / chunks;
        const int cx0 = static_cast<int>((u - row0 * chunks) * W);
        const int cx1 = min(cx0 + static_cast<int>(W), nc[0]);
        const int y0 = static_cast<int>(row0 % static_cast<std::uint32_t>(nc[1]));
        const int z0 = NDC == 3 ? static_cast<int>(row0 / static_cast<std::uint32_t>(nc[1])) : 0;
        const int cl = max(cx0 - 1, 0), ch = min(cx1 + 1, nc[0]);
        const int cnt = ch - cl + 1;  // cell_start entries of one row's slice
        // first cell of the grid row at row offset r
        auto rowbase = [&](int r) -> std::uint64_t {
            int y = y0 + (r % 3) - 1;
            y = y < 0 ? y + nc[1] : (y >= nc[1] ? y - nc[1] : y);
            std::uint64_t row = static_cast<std::uint64_t>(y);
            if constexpr (NDC == 3) {
                int z = z0 + (r / 3) - 1;
                z = z < 0 ? z + nc[2] : (z >= nc[2] ? z - nc[2] : z);
                row += static_cast<std::uint64_t>(z) * static_cast<std::uint64_t>(nc[1]);
            }
            return row * static_cast<std::uint64_t>(nc[0]);
        };
        __syncthreads();  // the previous unit is finished with the shared arrays
        // 1. cell_start entries: the rows' slices and windows
        for (int r = 0; r < R; ++r) {
            const std::uint32_t* cs = a.cell_start + rowbase(r) + cl;
            for (int c = threadIdx.x; c < cnt; c += T) s_cs[r * US::slice + c] = cs[c];
        }
        if (threadIdx.x < R) {
            const int r = threadIdx.x;
            const std::uint32_t* cs = a.cell_start + rowbase(r);
            const std::uint32_t mb = cs[cl], me = cs[ch];
            std::uint32_t lb = 0, le = 0, rb = 0, re = 0;
            if (cx0 == 0) {
                lb = cs[nc[0] - 1];
                le = cs[nc[0]];
            }
            if (cx1 == nc[0]) {
                rb = cs[0];
                re = cs[1];
            }
            s_wb[3 * r] = mb;
            s_wl[3 * r] = me - mb;
            s_wb[3 * r + 1] = lb;
            s_wl[3 * r + 1] = le - lb;
            s_wb[3 * r + 2] = rb;
            s_wl[3 * r + 2] = re - rb;
            if (r == CR) {
                s_qa = cs[cx0];
                s_qb = cs[cx1];
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            std::uint32_t tot = 0;
            for (int w = 0; w < NW; ++w) {
                s_ws[w] = tot;
                tot += s_wl[w];
            }
            s_total = tot;
            if (tot > static_cast<std::uint32_t>(US::stage))  // not staged: records read from pos
                for (int w = 0; w < NW; ++w) s_ws[w] = s_wb[w];
        }
        __syncthreads();
        const std::uint32_t total = s_total;
        const bool staged = total <= static_cast<std::uint32_t>(US::stage);
        // 2. stage the windows: each thread copies records tid, tid + T, ... of
        // their concatenation, four loads in flight before the stores
        if (staged) {
            int wc = 0;
            for (std::uint32_t e0 = threadIdx.x; e0 < total; e0 += 4u * T) {
                double2 lo[4], hi[4];
                RCPG_UNROLL
                for (int k = 0; k < 4; ++k) {
                    const std::uint32_t e = e0 + static_cast<std::uint32_t>(k * T);
                    if (e < total) {
                        while (e - s_ws[wc] >= s_wl[wc]) ++wc;
                        const std::uint64_t p = s_wb[wc] + (e - s_ws[wc]);
                        ld_record(a.pos + 4 * p, lo[k], hi[k]);
                    }
                }
                RCPG_UNROLL
                for (int k = 0; k < 4; ++k) {
                    const std::uint32_t e = e0 + static_cast<std::uint32_t>(k * T);
                    if (e < total) {
                        if constexpr (NDC == 2) hi[k].y = pack_f32(static_cast<float>(hi[k].x));
                        double2* dst = reinterpret_cast<double2*>(u_stage + 4 * static_cast<std::size_t>(e));
                        dst[0] = lo[k];
                        dst[1] = hi[k];
                    }
                }
            }
        }
        __syncthreads();
        const std::uint32_t own_b = s_wb[3 * CR], own_s = s_ws[3 * CR];
        // 3. the unit's particles; records from the stage or, for a unit whose
        // windows did not fit, from pos
        auto particles = [&](auto staged_tag) {
            constexpr bool STG = decltype(staged_tag)::value;
            const double* recs = STG ? static_cast<const double*>(u_stage) : a.pos;  // record s at recs + 4 s
            for (std::uint32_t q = s_qa + threadIdx.x; q < s_qb; q += T) {
                double xq[ND], D0q;
                {
                    const double2* r2 =
                        reinterpret_cast<const double2*>(recs + 4 * static_cast<std::size_t>(own_s + (q - own_b)));
                    unpack_record<ND>(r2[0], r2[1], xq, D0q);
                }
                UnitPair<ND, MX> up;
                up.begin(xq, D0q, kap);
                std::uint32_t n = 0;
                // candidate p, record s of `recs`
                auto test = [&](std::uint32_t p, std::uint32_t s) {
                    const double2* r2 = reinterpret_cast<const double2*>(recs + 4 * static_cast<std::size_t>(s));
                    const double2 lo = r2[0], hi = r2[1];
                    double xj[ND], D0j;
                    unpack_record<ND>(lo, hi, xj, D0j);
                    float D0jf = 0.0f;
                    if constexpr (MX) D0jf = (STG && NDC == 2) ? unpack_f32(hi.y) : static_cast<float>(D0j);
                    if (up.candidate(p > q, xj, D0j, D0jf, bx, ibx, hbf, t_shell, tf, fuse)) {
                        if (n < S) a.nbr[static_cast<std::uint64_t>(n) * N + q] = p;
                        ++n;
                    }
                };
                // the binning's cell (same arithmetic and positions), held
                // inside the unit so that every slice index stays in range
                const int cx = min(max(cell_coord(xq[0], scale0, nc[0]), cx0), cx1 - 1);
                const int lo = cx == 0 ? 0 : cx - 1, hi = cx == nc[0] - 1 ? nc[0] : cx + 2;
                // the main ranges: cells lo .. hi-1 of each row
                if constexpr (NDC == 2) {
                    std::uint32_t pb[3], ns[3], sb[3];
                    RCPG_UNROLL
                    for (int r = 0; r < 3; ++r) {
                        const std::uint32_t* sl = s_cs + r * US::slice;
                        pb[r] = sl[lo - cl];
                        ns[r] = sl[hi - cl] - pb[r];
                        sb[r] = s_ws[3 * r] + (pb[r] - s_wb[3 * r]);
                    }
                    const std::uint32_t c1 = ns[0], c2 = ns[0] + ns[1], tot = c2 + ns[2];
                    // two candidates per round: both probed (independent
                    // work for the lane), then committed in scan order
                    for (std::uint32_t k = 0; k < tot; k += 2) {
                        std::uint32_t pp[2];
                        typename UnitPair<ND, MX>::Probe pr[2];
                        RCPG_UNROLL
                        for (int v = 0; v < 2; ++v) {
                            const std::uint32_t kk = min(k + static_cast<std::uint32_t>(v), tot - 1);
                            const bool r0 = kk < c1, r1 = kk < c2;
                            const std::uint32_t o = r0 ? kk : (r1 ? kk - c1 : kk - c2);
                            pp[v] = (r0 ? pb[0] : (r1 ? pb[1] : pb[2])) + o;
                            const std::uint32_t st = (r0 ? sb[0] : (r1 ? sb[1] : sb[2])) + o;
                            const double2* r2 = reinterpret_cast<const double2*>(recs + 4 * static_cast<std::size_t>(st));
                            const double2 rl = r2[0], rh = r2[1];
                            double xj[ND], D0j;
                            unpack_record<ND>(rl, rh, xj, D0j);
                            float D0jf = 0.0f;
                            if constexpr (MX) D0jf = STG ? unpack_f32(rh.y) : static_cast<float>(D0j);
                            up.probe(pr[v], xj, D0j, D0jf, bx, ibx, hbf, t_shell, tf, fuse);
                        }
                        RCPG_UNROLL
                        for (int v = 0; v < 2; ++v) {
                            if (k + static_cast<std::uint32_t>(v) < tot && pp[v] != q && pr[v].pass) {
                                if (n < S) a.nbr[static_cast<std::uint64_t>(n) * N + q] = pp[v];
                                ++n;
                                up.commit(pp[v] > q, pr[v]);
                            }
                        }
                    }
                } else {
                    for (int r = 0; r < R; ++r) {
                        const std::uint32_t* sl = s_cs + r * US::slice;
                        const std::uint32_t pb = sl[lo - cl], pe = sl[hi - cl];
                        const std::uint32_t sb = s_ws[3 * r] + (pb - s_wb[3 * r]);
                        for (std::uint32_t p = pb; p < pe; ++p)
                            if (p != q) test(p, sb + (p - pb));
                    }
                }
                // the wrapped cells: the x-1 cell of a particle at x = 0, the
                // x+1 cell of one at x = nc0-1
                if (cx == 0 || cx == nc[0] - 1) {
                    const int wk = cx == 0 ? 1 : 2;
                    for (int r = 0; r < R; ++r) {
                        const std::uint32_t wb = s_wb[3 * r + wk], wl = s_wl[3 * r + wk], ws = s_ws[3 * r + wk];
                        for (std::uint32_t o = 0; o < wl; ++o)
                            if (wb + o != q) test(wb + o, ws + o);
                    }
                }
                // the reference's capacity check counts the partners after q in
                // its own order; a row that fits the capacity in full needs no count
                const std::uint32_t cap = a.caps[q];
                if (n > cap && n <= S) {
                    const std::uint32_t rq = a.ref_rank[q];
                    std::uint32_t n_half = 0;
                    for (std::uint32_t k = 0; k < n; ++k)
                        n_half += a.ref_rank[a.nbr[static_cast<std::uint64_t>(k) * N + q]] > rq;
                    if (n_half > cap) report_cap_error(ctl, rq, cap);
                }
                need = max(need, n);
                if (n > S) {
                    a.nbr_cnt[q] = 0u;  // overflow: empty row, rebuilt after the capacity grows
                    overflow = true;
                    continue;
                }
                a.nbr_cnt[q] = n;
                if (!fuse) continue;
                double f[ND];
                up.force(f);
                s_acc[0][col] = xadd(s_acc[0][col], static_cast<double>(up.sU));
                s_acc[1][col] = xadd(s_acc[1][col], static_cast<double>(up.sLc));
                s_acc[2][col] = xadd(s_acc[2][col], static_cast<double>(up.sdk));
                s_acc[3][col] = xadd(s_acc[3][col], static_cast<double>(up.sFm));
                s_acc[4][col] = fmax(s_acc[4][col], static_cast<double>(up.smax));
                std::uint32_t wc = 0;
                wall_forces<ND>(xq, up.Di, g, f, s_acc[0][col], s_acc[2][col], s_acc[3][col], wc);
                s_accn[0][col] += up.scount + wc;
                const double f2 = force_norm2<ND>(f);
                if (f2 > 1.0E-16) {
                    s_acc[5][col] = xadd(s_acc[5][col], xsqrt(f2));
                    ++s_accn[1][col];
                }
                s_acc[6][col] = xadd(s_acc[6][col], up.Di);
                RCPG_UNROLL
                for (int d = 0; d < ND; ++d) a.F[static_cast<std::uint64_t>(q) * ND + d] = f[d];
            }
        };
        if (staged) particles(std::true_type{});
        else particles(std::false_type{});
    }
    if (overflow && fuse) ctl->forces_done = 0u;
    // block maximum of the row lengths, one atomic per block
    RCPG_UNROLL
    for (int o = 16; o > 0; o >>= 1) need = max(need, __shfl_xor_sync(0xffffffffu, need, o));
    __syncthreads();
    if ((threadIdx.x & 31) == 0 && need) atomicMax(&s_need, need);
    if (fuse) {
        ForceSums fs;
        sums_zero(fs);
        fs.pair_U = s_acc[0][col];
        fs.pair_Lc = s_acc[1][col];
        fs.pair_dk = s_acc[2][col];
        fs.pair_Fm = s_acc[3][col];
        fs.pair_maxov = s_acc[4][col];
        fs.sum_mag = s_acc[5][col];
        fs.sum_D = s_acc[6][col];
        fs.pair_count = s_accn[0][col];
        fs.mag_count = s_accn[1][col];
        block_reduce_sums<T>(fs, s_red);  // ends with a block barrier before thread 0 reads
        if (threadIdx.x == 0) a.block_sums[blockIdx.x] = fs;
    } else {
        __syncthreads();
    }
    if (threadIdx.x == 0 && s_need) atomicMax(&ctl->row_need, s_need);
}

// dynamic shared memory of k_cells<ND, *>: the stage and the rows' cell_start slices
template <int ND>
constexpr std::size_t cells_smem_bytes() {
    using US = UnitShape<ND>;
    return static_cast<std::size_t>(US::stage) * 4 * sizeof(double) +
           static_cast<std::size_t>(US::rows) * US::slice * sizeof(std::uint32_t);
}

// ===========================================================================
// C. forces + walls + per-block sums
// ===========================================================================
// EXACT: the pair terms of every counted pair are also stored (pterm) for the
// one-thread-order reduction; the block sums are not used then. Otherwise the
// block sums are the step's reduction input and the wall terms join the pair
// chains (the reduction adds pair and wall terms anyway). MIXED: FP32 pair
// terms; the graph launches both variants and the one that does not match the
// step's precision returns at once.
template <int ND, bool EXACT, bool MIXED>
__global__ void __launch_bounds__(kForceBlock, EXACT ? 1 : ((MIXED && ND == 2) ? 3 : 2)) k_forces(DevArrays a) {
    const DevCtl* ctl = a.ctl;
    __shared__ ForceSums red[kForceBlock / 32];
    {
        // one round trip for every flag of the early exit
        const std::uint32_t st = ctl->stopped, ha = ctl->halted, fd = ctl->forces_done, p32 = ctl->pair_fp32;
        if ((st | ha | fd) != 0u || MIXED != (!EXACT && p32 != 0u)) return;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.ctl->nsum_blocks = gridDim.x;
        a.ctl->pair_kernel_runs += 1ull;
    }
    bind_buffers(a);
    const std::uint64_t N = a.N;
    const Geometry& g = ctl->g;
    double bx[ND];
    RCPG_UNROLL
    for (int d = 0; d < ND; ++d) bx[d] = g.box[d];
    const double kap = ctl->force_kappa;
    // the block's running sums live in shared memory, one column per thread
    // (they change once per particle); a particle's pair terms are summed in
    // registers first
    __shared__ double acc[7][kForceBlock];
    __shared__ std::uint32_t accn[2][kForceBlock];
    RCPG_UNROLL
    for (int f = 0; f < 7; ++f) acc[f][threadIdx.x] = 0.0;
    accn[0][threadIdx.x] = accn[1][threadIdx.x] = 0u;
    // persistent grid: row slots t = blockIdx*256 + tid, then strides of the grid
    for (std::uint64_t t = blockIdx.x * static_cast<std::uint64_t>(blockDim.x) + threadIdx.x; t < N;
         t += static_cast<std::uint64_t>(gridDim.x) * blockDim.x) {
        // row slot t belongs to particle work[t] (rows in cell order over
        // particles in their own order) or to particle t (cell-order storage,
        // rows in particle order)
        const std::uint64_t i = (a.permute || !a.work) ? t : a.work[t];
        double xi[ND], D0i;
        load_pos_g<ND>(a.pos, i, xi, D0i, 1);
        const double Di = xmul(D0i, kap);
        double fi[ND];
        const std::uint32_t n = min(a.nbr_cnt[t], a.S);
        std::uint32_t nterm = 0, scount = 0;
        using Acc = std::conditional_t<MIXED, float, double>;
        Acc sU = 0, sLc = 0, sdk = 0, sFm = 0, smax = 0;
        // Partners in chunks of kChunk: the row ids and then the partner
        // positions of a chunk are loaded before any of its arithmetic, so a
        // thread keeps kChunk gathers in flight; the pairs are still summed in
        // row order.
        auto rows = [&](auto mixed_tag) {
            constexpr bool MX = decltype(mixed_tag)::value;
            constexpr std::uint32_t kChunk = 4;
            float fif[ND], hbf[ND];
            double ibx[ND];
            RCPG_UNROLL
            for (int d = 0; d < ND; ++d) {
                fi[d] = 0.0;
                fif[d] = 0.0f;
                hbf[d] = static_cast<float>(0.5 * bx[d]);
                if constexpr (!MX) ibx[d] = g.inv_box[d];
            }
            const float kapf = static_cast<float>(kap);
            const float Dif = static_cast<float>(D0i) * kapf;
            for (std::uint32_t k0 = 0; k0 < n; k0 += kChunk) {
                std::uint32_t jj[kChunk];
                double xj[kChunk][ND], D0j[kChunk];
                RCPG_UNROLL
                for (std::uint32_t u = 0; u < kChunk; ++u)
                    jj[u] = (k0 + u < n) ? __ldg(a.nbr + static_cast<std::uint64_t>(k0 + u) * N + t) : 0u;
                RCPG_UNROLL
                for (std::uint32_t u = 0; u < kChunk; ++u)
                    if (k0 + u < n && jj[u] < N) load_pos_g<ND>(a.pos, jj[u], xj[u], D0j[u], 1);
                // the chunk's displacements and overlap tests first (independent
                // work), then the overlapping pairs' terms in row order
                using PT = std::conditional_t<MX, float, double>;
                PT pdx[kChunk][ND], pd2[kChunk], pr[kChunk];
                bool pov[kChunk];
                RCPG_UNROLL
                for (std::uint32_t u = 0; u < kChunk; ++u) {
                    const bool live = k0 + u < n && jj[u] < N;
                    if (!live) {  // a defined record for the unused slots
                        RCPG_UNROLL
                        for (int d = 0; d < ND; ++d) xj[u][d] = xi[d];
                        D0j[u] = 0.0;
                    }
                    if constexpr (MX) {
                        pd2[u] = mixed_disp<ND>(xi, xj[u], bx, hbf, pdx[u]);
                        pr[u] = 0.5f * (Dif + static_cast<float>(D0j[u]) * kapf);
                        pov[u] = live && pd2[u] < pr[u] * pr[u];
                    } else {
                        pr[u] = xmul(0.5, xadd(Di, xmul(D0j[u], kap)));
                        pd2[u] = pair_disp<ND>(xi, xj[u], bx, ibx, pdx[u]);
                        pov[u] = live && pd2[u] < xmul(pr[u], pr[u]);
                    }
                }
                RCPG_UNROLL
                for (std::uint32_t u = 0; u < kChunk; ++u) {
                    if (!pov[u]) continue;
                    const std::uint32_t j = jj[u];
                    if constexpr (MX) {
                        // FP32 terms summed in FP32 (EXACT never takes FP32 terms)
                        PairTermsF pf;
                        pair_terms_mixed_f<ND>(pdx[u], pd2[u], pr[u], fif, pf);
                        if (j > i) {
                            sU += pf.U;
                            sLc += pf.Lc;
                            sdk += pf.dk;
                            sFm += pf.Fm;
                            smax = fmaxf(smax, pf.U);
                            ++scount;
                        }
                    } else {
                        PairTerms pt;
                        pair_terms_f64<ND>(pdx[u], pd2[u], pr[u], fi, pt);
                        if (j > i) {
                            if constexpr (EXACT) {
                                a.pterm[static_cast<std::uint64_t>(nterm) * N + i] = pt;
                                ++nterm;
                            } else {
                                sU = xadd(sU, pt.U);
                                sLc = xadd(sLc, pt.Lc);
                                sdk = xadd(sdk, pt.dk);
                                sFm = xadd(sFm, pt.Fm);
                                smax = fmax(smax, pt.U);
                                ++scount;
                            }
                        }
                    }
                }
            }
            if constexpr (MX) {
                RCPG_UNROLL
                for (int d = 0; d < ND; ++d) fi[d] = static_cast<double>(fif[d]);
            }
        };
        rows(std::integral_constant<bool, MIXED>{});
        if constexpr (EXACT) {
            a.pterm_cnt[i] = nterm;
            double wU = 0.0, wdk = 0.0, wFm = 0.0;  // recomputed in order by k_reduce_exact
            std::uint32_t wc = 0;
            wall_forces<ND>(xi, Di, g, fi, wU, wdk, wFm, wc);
        } else {
            const int c = threadIdx.x;
            acc[0][c] = xadd(acc[0][c], static_cast<double>(sU));
            acc[1][c] = xadd(acc[1][c], static_cast<double>(sLc));
            acc[2][c] = xadd(acc[2][c], static_cast<double>(sdk));
            acc[3][c] = xadd(acc[3][c], static_cast<double>(sFm));
            acc[4][c] = fmax(acc[4][c], static_cast<double>(smax));
            std::uint32_t wc = 0;
            wall_forces<ND>(xi, Di, g, fi, acc[0][c], acc[2][c], acc[3][c], wc);
            accn[0][c] += scount + wc;
            const double f2 = force_norm2<ND>(fi);
            if (f2 > 1.0E-16) {
                acc[5][c] = xadd(acc[5][c], xsqrt(f2));
                ++accn[1][c];
            }
            acc[6][c] = xadd(acc[6][c], Di);
        }
#pragma unroll
        for (int d = 0; d < ND; ++d) a.F[i * ND + d] = fi[d];
    }
    if constexpr (!EXACT) {
        ForceSums s;
        sums_zero(s);
        const int c = threadIdx.x;
        s.pair_U = acc[0][c];
        s.pair_Lc = acc[1][c];
        s.pair_dk = acc[2][c];
        s.pair_Fm = acc[3][c];
        s.pair_maxov = acc[4][c];
        s.sum_mag = acc[5][c];
        s.sum_D = acc[6][c];
        s.pair_count = accn[0][c];
        s.mag_count = accn[1][c];
        block_reduce_sums<kForceBlock>(s, red);
        if (threadIdx.x == 0) a.block_sums[blockIdx.x] = s;
    }
}

// ===========================================================================
// D. reductions and controller
// ===========================================================================
// Sums in the one-thread order of the reference: all pair terms row after
// row, then the wall terms particle after particle (ENG:4086-4257), the
// diameter sum and the force-magnitude sum in index order (ENG:4262, :785).
template <int ND>
__global__ void k_reduce_exact(DevArrays a) {
    DevCtl* ctl = a.ctl;
    if (ctl_idle(ctl)) return;
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    const std::uint64_t N = a.N;
    ForceSums s;
    sums_zero(s);
    for (std::uint64_t i = 0; i < N; ++i) {
        const std::uint32_t n = a.pterm_cnt[i];
        for (std::uint32_t k = 0; k < n; ++k) {
            const PairTerms pt = a.pterm[static_cast<std::uint64_t>(k) * N + i];
            s.pair_U = xadd(s.pair_U, pt.U);
            s.pair_count += 1ull;
            s.pair_Lc = xadd(s.pair_Lc, pt.Lc);
            if (pt.U > s.pair_maxov) s.pair_maxov = pt.U;
            s.pair_dk = xadd(s.pair_dk, pt.dk);
            s.pair_Fm = xadd(s.pair_Fm, pt.Fm);
        }
    }
    const Geometry g = ctl->g;  // register copy: the loops below store through other pointers
    const double kap = ctl->force_kappa;
    for (std::uint64_t i = 0; i < N; ++i) {
        double xi[ND], D0i, fdummy[ND];
        load_pos<ND>(a.pos, i, xi, D0i);
#pragma unroll
        for (int d = 0; d < ND; ++d) fdummy[d] = 0.0;
        // wall terms continue the pair chains, as in the reference
        wall_forces<ND>(xi, xmul(D0i, kap), g, fdummy, s.pair_U, s.pair_dk, s.pair_Fm, s.wall_count);
    }
    for (std::uint64_t i = 0; i < N; ++i) {
        double xi[ND], D0i;
        load_pos<ND>(a.pos, i, xi, D0i);
        s.sum_D = xadd(s.sum_D, xmul(D0i, kap));
    }
    std::uint32_t mc = 0;
    for (std::uint64_t i = 0; i < N; ++i) {
        const double f2 = force_norm2<ND>(a.F + i * ND);
        if (f2 > 1.0E-16) {
            s.sum_mag = xadd(s.sum_mag, xsqrt(f2));
            ++mc;
        }
    }
    s.mag_count = mc;
    ctl->sums = s;
}

// Fixed-order reduction of the per-block partial sums by one block.
constexpr int kCtlThreads = 256;

__device__ void reduce_blocks(const DevArrays& a, ForceSums* smem, ForceSums& out) {
    const unsigned nb = a.ctl->nsum_blocks;
    ForceSums s;
    sums_zero(s);
    for (unsigned b = threadIdx.x; b < nb; b += blockDim.x) sums_add(s, a.block_sums[b]);
    block_reduce_sums<kCtlThreads>(s, smem);
    if (threadIdx.x == 0) out = s;
}

__global__ void __launch_bounds__(kCtlThreads) k_reduce_fast(DevArrays a) {
    __shared__ ForceSums red[kCtlThreads / 32];
    DevCtl* ctl = a.ctl;
    if (ctl_idle(ctl)) return;
    ForceSums s;
    reduce_blocks(a, red, s);
    if (threadIdx.x == 0) ctl->sums = s;
}

// Graph-mode controller: reduce, finish step s (end_step), open step s+1
// (begin_step) and publish the parameters of the kernels that follow. With
// open_only it just opens the next step (the first step of a run).
// Window statistics of the histories for begin_step(step), computed by the
// whole block: sums in a fixed tree (graph mode; the host sums in order).
__device__ void hist_stats_block(const Histories& h, std::uint64_t step, HistStats& out, double* red) {
    // (lo, hi) inclusive index ranges of the four force means
    const long long S = static_cast<long long>(step);
    const long long lo[4] = {S - 450, S - 75, S - 200, S - 3000};
    const long long hi[4] = {S - 250, S - 1, S - 1, S - 2500};
    double sum[4] = {0.0, 0.0, 0.0, 0.0};
    // a window whose start precedes step 1 wraps in the unsigned step
    // arithmetic of hist_mean, which then sums nothing: the same here
    RCPG_UNROLL
    for (int w = 0; w < 4; ++w)
        if (lo[w] >= 0)
            for (long long k = lo[w] + threadIdx.x; k <= hi[w]; k += blockDim.x) sum[w] = xadd(sum[w], h.force[k]);
    // phi range over [step - 250, step - 1)
    double mn = HUGE_VAL, mx = -HUGE_VAL;
    for (long long k = S - 250 + threadIdx.x; k < S - 1; k += blockDim.x)
        if (k >= 0) {
            mn = fmin(mn, h.phi[k]);
            mx = fmax(mx, h.phi[k]);
        }
    RCPG_UNROLL
    for (int o = 16; o > 0; o >>= 1) {
        RCPG_UNROLL
        for (int w = 0; w < 4; ++w) sum[w] = xadd(sum[w], __shfl_down_sync(0xffffffffu, sum[w], o));
        mn = fmin(mn, __shfl_down_sync(0xffffffffu, mn, o));
        mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (lane == 0) {
        RCPG_UNROLL
        for (int w = 0; w < 4; ++w) red[warp * 6 + w] = sum[w];
        red[warp * 6 + 4] = mn;
        red[warp * 6 + 5] = mx;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < nw; ++k) {
            RCPG_UNROLL
            for (int w = 0; w < 4; ++w) red[w] = xadd(red[w], red[k * 6 + w]);
            red[4] = fmin(red[4], red[k * 6 + 4]);
            red[5] = fmax(red[5], red[k * 6 + 5]);
        }
        // the divisors of hist_mean: end - start + 1 in unsigned step arithmetic
        const std::uint64_t u = step;
        out.f_450_250 = xdiv(red[0], static_cast<double>((u - 250) - (u - 450) + 1));
        out.f_75_1 = xdiv(red[1], static_cast<double>((u - 1) - (u - 75) + 1));
        out.f_200_1 = xdiv(red[2], static_cast<double>((u - 1) - (u - 200) + 1));
        out.f_3000_2500 = xdiv(red[3], static_cast<double>((u - 2500) - (u - 3000) + 1));
        out.phi_range_250 = xsub(red[5], red[4]);
    }
}

__global__ void __launch_bounds__(kCtlThreads) k_controller(DevArrays a, int open_only) {
    __shared__ ForceSums red[kCtlThreads / 32];
    __shared__ double s_hred[(kCtlThreads / 32) * 6];
    // the controller state is worked on in shared memory: one coalesced copy
    // in and out instead of a chain of dependent global loads in one thread
    __shared__ Controller cs;
    __shared__ HistStats s_stats;
    __shared__ int s_publish, s_go;
    DevCtl* ctl = a.ctl;
    if (ctl_idle(ctl)) {
        if (threadIdx.x == 0) ctl->adam_go = 0u;
        return;
    }
    static_assert(sizeof(Controller) % 8 == 0, "controller copy by 8-byte words");
    constexpr int kWords = sizeof(Controller) / 8;
    {
        const unsigned long long* src = reinterpret_cast<const unsigned long long*>(&ctl->c);
        unsigned long long* dst = reinterpret_cast<unsigned long long*>(&cs);
        for (int w = threadIdx.x; w < kWords; w += blockDim.x) dst[w] = src[w];
    }
    // the control words thread 0 needs, loaded before the reduction so that
    // their latency overlaps it
    std::uint32_t row_need = 0, cap_error = 0, pair_fp32 = 0;
    double force_mu = 0.0, mixed_switch = 0.0;
    if (threadIdx.x == 0) {
        row_need = ctl->row_need;
        cap_error = ctl->cap_error;
        pair_fp32 = ctl->pair_fp32;
        force_mu = ctl->force_mu;
        mixed_switch = ctl->mixed_switch;
    }
    __syncthreads();
    ForceSums s;
    if (!open_only) reduce_blocks(a, red, s);
    // 1. end of the finished step (thread 0)
    if (threadIdx.x == 0) {
        Controller& c = cs;
        s_publish = 0;
        bool go = true;
        if (!open_only) {
            ctl->sums = s;
            // capacity problems of the last build stop the run before its results are used
            if (row_need > a.S || cap_error) {
                ctl->halted = 1u;
                ctl->adam_go = 0u;
                go = false;
            } else {
                const StepScalars sc = finalize_sums(s, force_mu, a.ndim);
                ctl->scal = sc;
                end_step(c, a.hist, sc);
                // mixed precision: FP64 pair terms from the first step whose
                // (nonzero) max overlap is below the switch, for the rest of the run
                if (pair_fp32 && sc.max_overlap > 0.0 && sc.max_overlap < mixed_switch) {
                    ctl->pair_fp32 = 0u;
                    ctl->fp64_switch_step = c.steps;
                }
                ctl->graph_steps += 1ull;
                for (int d = 0; d < a.ndim; ++d) ctl->adam_box[d] = c.box[d];
                ctl->adam_alpha = c.adam_alpha;
                ctl->adam_inv_b1 = c.inv_b1;
                ctl->adam_inv_b2 = c.inv_b2;
                ctl->adam_go = 1u;
            }
        } else {
            ctl->adam_go = 0u;
        }
        if (go) {
            ctl->fix_height_scale = 1.0;
            if (c.steps + 1 > c.step_cap) {
                ctl->stopped = 1u;
                go = false;
            }
        }
        s_go = go ? 1 : 0;
    }
    __syncthreads();
    // 2. the history windows the next step's schedule may read (the block)
    const std::uint64_t next = cs.steps + 1;
    const bool stats = s_go && next > 250 &&
                       ((next >= cs.mu_decay_next_tick) || (next > 2500 && next - cs.last_alpha_update > 500));
    if (stats) hist_stats_block(a.hist, next, s_stats, s_hred);
    __syncthreads();
    // 3. top of the next step (thread 0)
    if (threadIdx.x == 0 && s_go) {
        Controller& c = cs;
        begin_step(c, a.hist, next, stats ? &s_stats : nullptr);
        // the stretch of a reorder step waits until after the reorder (ENG:5661 < :5758)
        ctl->fix_height_scale = c.reorder ? 1.0 : c.fix_height_scale;
        if (c.done || c.reorder || c.lock_now) ctl->stopped = 1u;
        else s_publish = 1;
    }
    __syncthreads();
    {
        const unsigned long long* src = reinterpret_cast<const unsigned long long*>(&cs);
        unsigned long long* dst = reinterpret_cast<unsigned long long*>(&ctl->c);
        for (int w = threadIdx.x; w < kWords; w += blockDim.x) dst[w] = src[w];
    }
    if (threadIdx.x == 0 && s_publish) publish_step(ctl, cs, a.ndim);
}

// First node of a step in a captured step graph: opens the build when the
// step rebuilds its rows, and sets the pair-kernel switch for a step without
// a build (a build's last kernel sets it once the search has decided).
__global__ void k_step_gate(DevArrays a, unsigned long long cond_build) {
    const DevCtl* ctl = a.ctl;
    const std::uint32_t st = ctl->stopped, ha = ctl->halted, rb = ctl->rebuild_flag, p32 = ctl->pair_fp32;
    const bool live = (st | ha) == 0u;
    const bool build = live && rb != 0u;
    cudaGraphSetConditional(cond_build, build ? 1u : 0u);
    cudaGraphSetConditional(a.cond_forces, forces_case(live && !build, p32, a.mixed));
}

// fix_height stretch of the last coordinate without an ADAM step (used when
// the stretch and the ADAM pass are not fused).
template <int ND>
__global__ void k_fix_height(DevArrays a) {
    const std::uint64_t i = blockIdx.x * static_cast<std::uint64_t>(blockDim.x) + threadIdx.x;
    if (i >= a.N) return;
    bind_buffers(a);
    const double s = a.ctl->fix_height_scale;
    double* p = a.pos + i * pos_stride(ND) + (ND - 1);
    *p = xmul(*p, s);
}

// Rows in cell order -> rows in particle order (dst[k*N + work[t]] = src[k*N + t]).
__global__ void k_rows_to_particle_order(std::uint64_t N, const std::uint32_t* work,
                                         const std::uint32_t* src, const std::uint32_t* src_cnt,
                                         std::uint32_t* dst, std::uint32_t* dst_cnt) {
    const std::uint64_t t = blockIdx.x * static_cast<std::uint64_t>(blockDim.x) + threadIdx.x;
    if (t >= N) return;
    const std::uint64_t i = work[t];
    const std::uint32_t n = src_cnt[t];
    dst_cnt[i] = n;
    for (std::uint32_t k = 0; k < n; ++k) dst[static_cast<std::uint64_t>(k) * N + i] = src[static_cast<std::uint64_t>(k) * N + t];
}

template <int ND>
__global__ void k_cell_order_to_particle_order(DevArrays a, std::uint32_t* nbr_out, std::uint32_t* cnt_out,
                                               double* F_out) {
    const std::uint64_t q = blockIdx.x * static_cast<std::uint64_t>(blockDim.x) + threadIdx.x;
    if (q >= a.N) return;
    bind_buffers(a);
    const std::uint64_t N = a.N, i = a.origin[q];
    const std::uint32_t n = min(a.nbr_cnt[q], a.S);
    cnt_out[i] = n;
    for (std::uint32_t k = 0; k < n; ++k)
        nbr_out[static_cast<std::uint64_t>(k) * N + i] =
            static_cast<std::uint32_t>(a.origin[a.nbr[static_cast<std::uint64_t>(k) * N + q]]);
    RCPG_UNROLL
    for (int d = 0; d < ND; ++d) F_out[i * ND + d] = a.F[q * ND + d];
}

// ===========================================================================
// R. spatial reorder: key -> stable LSD radix sort -> gather
// ===========================================================================
// Sort key of the reference's spatial reorder: 21-bit Morton code in 3-D,
// the x coordinate otherwise (ENG:4850-4948).
template <int ND>
__device__ __forceinline__ std::uint64_t reorder_key(const double* x, const Geometry& g) {
    if (ND == 3) {
        std::uint64_t code = 0;
#pragma unroll
        for (int d = 0; d < 3 && d < ND; ++d) {
            const double scale = (static_cast<double>(1u << 21) - 1.0) / g.box[d];
            code |= morton_spread21(morton_axis(x[d], g.box[d], scale)) << d;
        }
        return code;
    }
    return double_order_key(x[0]);
}

template <int ND>
__global__ void k_reorder_keys(DevArrays a) {
    const std::uint64_t i = blockIdx.x * static_cast<std::uint64_t>(blockDim.x) + threadIdx.x;
    if (i >= a.N) return;
    double x[ND], D0;
    load_pos<ND>(a.pos, i, x, D0);
    a.sort_keys[0][i] = reorder_key<ND>(x, a.ctl->g);
    a.sort_vals[0][i] = static_cast<std::uint32_t>(i);
}

// Cell-order storage: the reference's reorder only changes the order in which
// results are returned. Keys are placed at each particle's reference index,
// so the stable sort breaks ties by the previous reference order as the
// reference's sort does; the particles themselves do not move.
template <int ND>
__global__ void k_reorder_keys_ranked(DevArrays a) {
    const std::uint64_t q = blockIdx.x * static_cast<std::uint64_t>(blockDim.x) + threadIdx.x;
    if (q >= a.N) return;
    bind_buffers(a);
    double x[ND], D0;
    load_pos<ND>(a.pos, q, x, D0);
    const std::uint32_t r = a.ref_rank[q];
    a.sort_keys[0][r] = reorder_key<ND>(x, a.ctl->g);
    a.sort_vals[0][r] = static_cast<std::uint32_t>(q);
}

__global__ void k_reorder_ranks(DevArrays a, const std::uint32_t* perm) {
    const std::uint64_t k = blockIdx.x * static_cast<std::uint64_t>(blockDim.x) + threadIdx.x;
    if (k >= a.N) return;
    bind_buffers(a);
    a.ref_rank[perm[k]] = static_cast<std::uint32_t>(k);
}

constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;

// Per-tile digit histogram, digit-major: hist[digit * tiles + tile].
__global__ void __launch_bounds__(kSortThreads)
    k_sort_hist(const std::uint64_t* keys, std::uint32_t n, int shift, std::uint32_t* hist,
                std::uint32_t tiles) {
    __shared__ std::uint32_t h[256];
    h[threadIdx.x] = 0u;
    __syncthreads();
    const std::uint64_t base = static_cast<std::uint64_t>(blockIdx.x) * kSortTile;
    for (int k = threadIdx.x; k < kSortTile; k += kSortThreads) {
        const std::uint64_t idx = base + k;
        if (idx < n) atomicAdd(&h[(keys[idx] >> shift) & 0xFFu], 1u);
    }
    __syncthreads();
    hist[static_cast<std::uint64_t>(threadIdx.x) * tiles + blockIdx.x] = h[threadIdx.x];
}

// Stable scatter: elements of a tile are ranked in index order, chunk by
// chunk of 256 (one per thread), with per-warp match masks.
__global__ void __launch_bounds__(kSortThreads)
    k_sort_scatter(const std::uint64_t* keys_in, const std::uint32_t* vals_in, std::uint64_t* keys_out,
                   std::uint32_t* vals_out, std::uint32_t n, int shift, const std::uint32_t* offsets,
                   std::uint32_t tiles) {
    __shared__ std::uint32_t base_d[256];
    __shared__ std::uint32_t wcnt[kSortThreads / 32][256];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    base_d[threadIdx.x] = offsets[static_cast<std::uint64_t>(threadIdx.x) * tiles + blockIdx.x];
    const std::uint64_t tile0 = static_cast<std::uint64_t>(blockIdx.x) * kSortTile;
    for (int chunk = 0; chunk < kSortItems; ++chunk) {
#pragma unroll
        for (int w = 0; w < kSortThreads / 32; ++w) wcnt[w][threadIdx.x] = 0u;
        __syncthreads();
        const std::uint64_t idx = tile0 + static_cast<std::uint64_t>(chunk) * kSortThreads + threadIdx.x;
        const bool valid = idx < n;
        std::uint64_t key = 0;
        std::uint32_t val = 0, digit = 0xFFFFFFFFu;
        if (valid) {
            key = keys_in[idx];
            val = vals_in[idx];
            digit = static_cast<std::uint32_t>((key >> shift) & 0xFFu);
        }
        const unsigned peers = __match_any_sync(0xffffffffu, digit);
        const unsigned lt = (1u << lane) - 1u;
        const std::uint32_t rank_w = __popc(peers & lt);
        if (valid && rank_w == 0) wcnt[warp][digit] = __popc(peers);
        __syncthreads();
        std::uint32_t before = 0;
        if (valid) {
            for (int w = 0; w < warp; ++w) before += wcnt[w][digit];
            const std::uint32_t pos = base_d[digit] + before + rank_w;
            keys_out[pos] = key;
            vals_out[pos] = val;
        }
        __syncthreads();
        // advance the per-digit base by this chunk's count (thread d owns digit d)
        std::uint32_t tot = 0;
#pragma unroll
        for (int w = 0; w < kSortThreads / 32; ++w) tot += wcnt[w][threadIdx.x];
        base_d[threadIdx.x] += tot;
        __syncthreads();
    }
}

template <int ND>
__global__ void k_reorder_gather(DevArrays a, const std::uint32_t* perm) {
    const std::uint64_t k = blockIdx.x * static_cast<std::uint64_t>(blockDim.x) + threadIdx.x;
    if (k >= a.N) return;
    const std::uint64_t src = perm[k];
    constexpr int P = pos_stride(ND);
#pragma unroll
    for (int q = 0; q < P; ++q) a.pos_tmp[k * P + q] = a.pos[src * P + q];
#pragma unroll
    for (int d = 0; d < ND; ++d) a.vec_tmp[k * ND + d] = a.m[src * ND + d];
    a.u64_tmp[k] = a.origin[src];
    a.cell_rank[k] = a.caps[src];  // cell_rank doubles as scratch here
}

template <int ND>
__global__ void k_reorder_gather_v(DevArrays a, const std::uint32_t* perm) {
    const std::uint64_t k = blockIdx.x * static_cast<std::uint64_t>(blockDim.x) + threadIdx.x;
    if (k >= a.N) return;
    const std::uint64_t src = perm[k];
#pragma unroll
    for (int d = 0; d < ND; ++d) a.x_last[k * ND + d] = a.v[src * ND + d];
}

template <int ND>
__global__ void k_reorder_commit(DevArrays a) {
    const std::uint64_t k = blockIdx.x * static_cast<std::uint64_t>(blockDim.x) + threadIdx.x;
    if (k >= a.N) return;
    constexpr int P = pos_stride(ND);
#pragma unroll
    for (int q = 0; q < P; ++q) a.pos[k * P + q] = a.pos_tmp[k * P + q];
#pragma unroll
    for (int d = 0; d < ND; ++d) {
        a.m[k * ND + d] = a.vec_tmp[k * ND + d];
        a.v[k * ND + d] = a.x_last[k * ND + d];
    }
    a.origin[k] = a.u64_tmp[k];
    a.caps[k] = a.cell_rank[k];
}

// ===========================================================================
// P. layout conversion and stand-alone kernels of the C ABI
// ===========================================================================
template <int ND>
__global__ void k_pack(std::uint64_t N, const double* __restrict__ x, const double* __restrict__ D,
                       double* __restrict__ pos) {
    const std::uint64_t i = blockIdx.x * static_cast<std::uint64_t>(blockDim.x) + threadIdx.x;
    if (i >= N) return;
    double xi[ND];
#pragma unroll
    for (int d = 0; d < ND; ++d) xi[d] = x[i * ND + d];
    store_pos<ND>(pos, i, xi, D ? D[i] : 0.0);
}

template <int ND>
__global__ void k_unpack(std::uint64_t N, const double* __restrict__ pos, double* __restrict__ x) {
    const std::uint64_t i = blockIdx.x * static_cast<std::uint64_t>(blockDim.x) + threadIdx.x;
    if (i >= N) return;
    double xi[ND], D0;
    load_pos<ND>(pos, i, xi, D0);
#pragma unroll
    for (int d = 0; d < ND; ++d) x[i * ND + d] = xi[d];
}

// Per-particle anchors, as the reference keeps them (ENG:6104-6145).
template <int ND>
__global__ void k_refresh_arrays(std::uint64_t N, const double* __restrict__ x, double* x_last,
                                 const double* __restrict__ D, double* D_last, double* theta,
                                 double theta_new, std::uint8_t* refresh,
                                 unsigned long long* count) {
    const std::uint64_t k = blockIdx.x * static_cast<std::uint64_t>(blockDim.x) + threadIdx.x;
    if (k >= N) return;
    double d2 = 0.0;
#pragma unroll
    for (int d = 0; d < ND; ++d) {
        const double dd = xsub(x[k * ND + d], x_last[k * ND + d]);
        d2 = xadd(d2, xmul(dd, dd));
    }
    double Dl = D_last[k];
    if (D[k] < Dl) Dl = D[k];
    double th = theta[k];
    if (th > theta_new) th = theta_new;
    std::uint8_t r = 0;
    if (refresh_trigger(d2, D[k], Dl, th)) {
        r = 1;
#pragma unroll
        for (int d = 0; d < ND; ++d) x_last[k * ND + d] = x[k * ND + d];
        Dl = D[k];
        th = theta_new;
        atomicAdd(count, 1ull);
    }
    D_last[k] = Dl;
    theta[k] = th;
    refresh[k] = r;
}

template <int ND>
__global__ void __launch_bounds__(kForceBlock) k_mean_force_blocks(DevArrays a) {
    __shared__ ForceSums red[kForceBlock / 32];
    if (blockIdx.x == 0 && threadIdx.x == 0) a.ctl->nsum_blocks = gridDim.x;
    const std::uint64_t i = blockIdx.x * static_cast<std::uint64_t>(blockDim.x) + threadIdx.x;
    ForceSums s;
    sums_zero(s);
    if (i < a.N) {
        const double f2 = force_norm2<ND>(a.F + i * ND);
        if (f2 > 1.0E-16) {
            s.sum_mag = xsqrt(f2);
            s.mag_count = 1ull;
        }
    }
    block_reduce_sums<kForceBlock>(s, red);
    if (threadIdx.x == 0) a.block_sums[blockIdx.x] = s;
}

template <int ND>
void reorder_impl(const DevArrays& a, cudaStream_t st) {
    const unsigned nb = force_blocks(a.N);
    const std::uint32_t n = static_cast<std::uint32_t>(a.N);
    if (a.permute) k_reorder_keys_ranked<ND><<<nb, kForceBlock, 0, st>>>(a);
    else k_reorder_keys<ND><<<nb, kForceBlock, 0, st>>>(a);
    const std::uint32_t tiles = (n + kSortTile - 1) / kSortTile;
    int cur = 0;
    for (int pass = 0; pass < 8; ++pass) {
        const int shift = pass * 8;
        k_sort_hist<<<tiles, kSortThreads, 0, st>>>(a.sort_keys[cur], n, shift, a.sort_hist, tiles);
        scan_exclusive(a.sort_hist, a.sort_hist, 256u * tiles, a.scan_tmp, nullptr, st);
        k_sort_scatter<<<tiles, kSortThreads, 0, st>>>(a.sort_keys[cur], a.sort_vals[cur],
                                                       a.sort_keys[cur ^ 1], a.sort_vals[cur ^ 1], n,
                                                       shift, a.sort_hist, tiles);
        cur ^= 1;
    }
    const std::uint32_t* perm = a.sort_vals[cur];
    if (a.permute) {
        k_reorder_ranks<<<nb, kForceBlock, 0, st>>>(a, perm);
        return;
    }
    k_reorder_gather<ND><<<nb, kForceBlock, 0, st>>>(a, perm);
    k_reorder_gather_v<ND><<<nb, kForceBlock, 0, st>>>(a, perm);
    k_reorder_commit<ND><<<nb, kForceBlock, 0, st>>>(a);
}

// Blocks of `Kernel` that are resident on the whole GPU at once (SMs x
// occupancy), cached per device: the grid of the persistent kernels.
template <auto Kernel>
unsigned resident_grid(int threads, std::size_t smem = 0) {
    static int grid[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return 148u;
    if (grid[dev] == 0) {
        int sms = 148, per_sm = 1;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, Kernel, threads, smem);
        grid[dev] = sms * (per_sm > 0 ? per_sm : 1);
    }
    return static_cast<unsigned>(grid[dev]);
}

template <int ND>
void adam_nd(const DevArrays& a, int do_adam, int do_refresh, cudaStream_t st) {
    const unsigned need = (force_blocks(a.N) + 1) / 2, g = resident_grid<k_adam_refresh<ND>>(kForceBlock);
    k_adam_refresh<ND><<<need < g ? need : g, kForceBlock, 0, st>>>(a, do_adam, do_refresh);
}

// persistent force grid: at most the blocks resident at once (the block-sum
// buffers hold at least force_blocks(N) entries)
// persistent grid of the cell-unit search: the blocks resident at once (at
// most 4096, the engine's block-sum entries)
template <int ND, bool MX>
void launch_cells_variant(const DevArrays& a, cudaStream_t st) {
    if constexpr (ND <= 3) {
        int dev = 0;
        cudaGetDevice(&dev);
        constexpr std::size_t smem = cells_smem_bytes<ND>();
        constexpr int T = UnitShape<ND>::threads;
        static int grid[64] = {};
        if (dev >= 0 && dev < 64 && grid[dev] == 0) {
            cudaFuncSetAttribute(k_cells<ND, MX>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
            int sms = 148, per_sm = 1;
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_cells<ND, MX>, T, smem);
            const int gr = sms * (per_sm > 0 ? per_sm : 1);
            grid[dev] = gr < 4096 ? gr : 4096;
        }
        const unsigned g = (dev >= 0 && dev < 64) ? static_cast<unsigned>(grid[dev]) : 148u;
        k_cells<ND, MX><<<g, T, smem, st>>>(a);
    }
}

// persistent force grid: at most the blocks resident at once (the block-sum
// buffers hold at least force_blocks(N) entries)
template <int ND, bool EXACT, bool MIXED>
void forces_nd(const DevArrays& a, cudaStream_t st) {
    const unsigned need = force_blocks(a.N), g = resident_grid<k_forces<ND, EXACT, MIXED>>(kForceBlock);
    k_forces<ND, EXACT, MIXED><<<need < g ? need : g, kForceBlock, 0, st>>>(a);
}

// persistent grid of the tiled build: as many blocks as fit on the GPU at once
template <int ND>
void launch_tiled(const DevArrays& a, cudaStream_t st) {
    int dev = 0;
    cudaGetDevice(&dev);
    constexpr std::size_t smem = tile_smem_bytes<ND>();
    static int grid[64] = {};
    if (dev >= 0 && dev < 64 && grid[dev] == 0) {
        cudaFuncSetAttribute(k_build_search_tiled<ND>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(smem));
        int sms = 148, per_sm = 1;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_build_search_tiled<ND>, kTileThreads, smem);
        grid[dev] = sms * (per_sm > 0 ? per_sm : 1);
    }
    const int blocks = (dev >= 0 && dev < 64) ? grid[dev] : 148;
    k_build_search_tiled<ND><<<static_cast<unsigned>(blocks), kTileThreads, smem, st>>>(a);
}

// both precisions where the run may use FP32 pair terms (the one that does
// not match the step returns at once)
template <int ND>
void launch_cells(const DevArrays& a, cudaStream_t st) {
    launch_cells_variant<ND, false>(a, st);
    if (a.mixed) launch_cells_variant<ND, true>(a, st);
}

// e0 / e1 (optional): events recorded around the search kernels only
template <int ND>
void rebuild_impl(const DevArrays& a, cudaStream_t st, cudaEvent_t e0 = nullptr, cudaEvent_t e1 = nullptr) {
    const unsigned nb = force_blocks(a.N);
    const unsigned cb = (a.C_alloc + 1 + 255) / 256;
    k_build_prepare<<<cb < 1024 ? cb : 1024, 256, 0, st>>>(a);
    k_build_bin<ND><<<nb, kForceBlock, 0, st>>>(a);
    scan_exclusive(a.cell_count, a.cell_start, a.C_alloc + 1, a.scan_tmp, a.ctl, st);
    k_build_scatter<<<nb, kForceBlock, 0, st>>>(a);
    k_build_cell_sort<ND><<<(a.C_alloc + 255) / 256, 256, 0, st>>>(a);
    if (a.permute) {
        // persistent grid, two particles per thread and round
        const unsigned need = (nb + 1) / 2, g = resident_grid<k_build_permute<ND>>(256);
        k_build_permute<ND><<<need < g ? need : g, 256, 0, st>>>(a);
    }
    if (e0) cudaEventRecord(e0, st);
    if (ND <= 3 && a.N >= kTiledMinN) {  // smaller packings take the warp search
        if (a.permute) {
            launch_cells<ND>(a, st);
        } else if (a.sorted_rows) {
            launch_tiled<ND>(a, st);
        }
    }
    const unsigned need = static_cast<unsigned>((a.N + kWarpSearchWarps - 1) / kWarpSearchWarps),
                   g = resident_grid<k_build_search<ND>>(32 * kWarpSearchWarps);
    k_build_search<ND><<<need < g ? need : g, 32 * kWarpSearchWarps, 0, st>>>(a);
    if (e1) cudaEventRecord(e1, st);
}

}  // namespace

#define RCPG_DISPATCH_ND(nd, CALL)                 \
    switch (nd) {                                  \
        case 2: { constexpr int ND = 2; CALL; } break; \
        case 3: { constexpr int ND = 3; CALL; } break; \
        case 4: { constexpr int ND = 4; CALL; } break; \
        case 5: { constexpr int ND = 5; CALL; } break; \
        case 6: { constexpr int ND = 6; CALL; } break; \
        case 7: { constexpr int ND = 7; CALL; } break; \
        case 8: { constexpr int ND = 8; CALL; } break; \
        default: break;                            \
    }

void launch_adam_refresh(const DevArrays& a, int do_adam, int do_refresh, cudaStream_t st) {
    RCPG_DISPATCH_ND(a.ndim, (adam_nd<ND>(a, do_adam, do_refresh, st)));
}

void launch_rebuild(const DevArrays& a, cudaStream_t st) {
    RCPG_DISPATCH_ND(a.ndim, (rebuild_impl<ND>(a, st)));
}

void launch_rebuild_timed(const DevArrays& a, cudaStream_t st, cudaEvent_t e0, cudaEvent_t e1) {
    RCPG_DISPATCH_ND(a.ndim, (rebuild_impl<ND>(a, st, e0, e1)));
}

void launch_forces(const DevArrays& a, int exact_terms, cudaStream_t st) {
    // k_forces (and the cell-unit search) read a 4-double particle record
    // (ndim <= 3) with one 256-bit load
    if (a.P == 4 && (((reinterpret_cast<std::uintptr_t>(a.pos) | reinterpret_cast<std::uintptr_t>(a.pos_alt)) & 31u) != 0))
        throw std::invalid_argument("rcpgenerator_b200: particle records must be 32-byte aligned");
    if (exact_terms) {
        RCPG_DISPATCH_ND(a.ndim, (forces_nd<ND, true, false>(a, st)));
    } else {
        RCPG_DISPATCH_ND(a.ndim, (forces_nd<ND, false, false>(a, st)));
        if (a.mixed) RCPG_DISPATCH_ND(a.ndim, (forces_nd<ND, false, true>(a, st)));
    }
}

void launch_forces_variant(const DevArrays& a, int mixed, cudaStream_t st) {
    if (mixed) {
        RCPG_DISPATCH_ND(a.ndim, (forces_nd<ND, false, true>(a, st)));
    } else {
        RCPG_DISPATCH_ND(a.ndim, (forces_nd<ND, false, false>(a, st)));
    }
}

void launch_step_gate(const DevArrays& a, unsigned long long cond_build, cudaStream_t st) {
    k_step_gate<<<1, 1, 0, st>>>(a, cond_build);
}

void launch_reduce_exact(const DevArrays& a, cudaStream_t st) {
    RCPG_DISPATCH_ND(a.ndim, (k_reduce_exact<ND><<<1, 1, 0, st>>>(a)));
}

// max |ref| and max |cmp - ref| (mixed-precision error report): a
// non-negative double's bit pattern orders like its value, so the block
// maxima combine with an integer atomicMax
__global__ void __launch_bounds__(256) k_diff_max(const double* __restrict__ ref, const double* __restrict__ cmp,
                                                  std::uint64_t n, unsigned long long* out) {
    double m0 = 0.0, m1 = 0.0;
    for (std::uint64_t k = blockIdx.x * 256ull + threadIdx.x; k < n; k += static_cast<std::uint64_t>(gridDim.x) * 256ull) {
        const double r = ref[k];
        m0 = fmax(m0, fabs(r));
        m1 = fmax(m1, fabs(cmp[k] - r));
    }
    RCPG_UNROLL
    for (int o = 16; o > 0; o >>= 1) {
        m0 = fmax(m0, __shfl_down_sync(0xffffffffu, m0, o));
        m1 = fmax(m1, __shfl_down_sync(0xffffffffu, m1, o));
    }
    __shared__ double s0[8], s1[8];
    if ((threadIdx.x & 31) == 0) {
        s0[threadIdx.x >> 5] = m0;
        s1[threadIdx.x >> 5] = m1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < 8; ++w) {
            m0 = fmax(m0, s0[w]);
            m1 = fmax(m1, s1[w]);
        }
        atomicMax(out, static_cast<unsigned long long>(__double_as_longlong(m0)));
        atomicMax(out + 1, static_cast<unsigned long long>(__double_as_longlong(m1)));
    }
}

void launch_diff_max(const double* ref, const double* cmp, std::uint64_t n, unsigned long long* out,
                     cudaStream_t st) {
    std::uint64_t blocks = (n + 255) / 256;
    if (blocks > 1184) blocks = 1184;
    if (blocks < 1) blocks = 1;
    k_diff_max<<<static_cast<unsigned>(blocks), 256, 0, st>>>(ref, cmp, n, out);
}

void launch_reduce_fast(const DevArrays& a, cudaStream_t st) {
    k_reduce_fast<<<1, kCtlThreads, 0, st>>>(a);
}

void launch_controller(const DevArrays& a, int open_only, cudaStream_t st) {
    k_controller<<<1, kCtlThreads, 0, st>>>(a, open_only);
}

void launch_reorder(const DevArrays& a, cudaStream_t st) {
    RCPG_DISPATCH_ND(a.ndim, (reorder_impl<ND>(a, st)));
}

void launch_fix_height(const DevArrays& a, cudaStream_t st) {
    const unsigned nb = force_blocks(a.N);
    RCPG_DISPATCH_ND(a.ndim, (k_fix_height<ND><<<nb, kForceBlock, 0, st>>>(a)));
}

void launch_pack(std::uint64_t N, int ndim, const double* x, const double* D, double* pos,
                 cudaStream_t st) {
    const unsigned nb = force_blocks(N);
    RCPG_DISPATCH_ND(ndim, (k_pack<ND><<<nb, kForceBlock, 0, st>>>(N, x, D, pos)));
}

void launch_unpack(std::uint64_t N, int ndim, const double* pos, double* x, cudaStream_t st) {
    const unsigned nb = force_blocks(N);
    RCPG_DISPATCH_ND(ndim, (k_unpack<ND><<<nb, kForceBlock, 0, st>>>(N, pos, x)));
}

void launch_refresh_arrays(std::uint64_t N, int ndim, const double* x, double* x_last,
                           const double* D, double* D_last, double* theta, double theta_new,
                           std::uint8_t* refresh, unsigned long long* count, cudaStream_t st) {
    const unsigned nb = force_blocks(N);
    RCPG_DISPATCH_ND(ndim, (k_refresh_arrays<ND><<<nb, kForceBlock, 0, st>>>(
                               N, x, x_last, D, D_last, theta, theta_new, refresh, count)));
}

void launch_rows_to_particle_order(std::uint64_t N, const std::uint32_t* work, const std::uint32_t* src,
                                   const std::uint32_t* src_cnt, std::uint32_t* dst,
                                   std::uint32_t* dst_cnt, cudaStream_t st) {
    k_rows_to_particle_order<<<force_blocks(N), kForceBlock, 0, st>>>(N, work, src, src_cnt, dst, dst_cnt);
}

void launch_cell_order_to_particle_order(const DevArrays& a, std::uint32_t* nbr_out, std::uint32_t* cnt_out,
                                         double* F_out, cudaStream_t st) {
    RCPG_DISPATCH_ND(a.ndim, (k_cell_order_to_particle_order<ND><<<force_blocks(a.N), kForceBlock, 0, st>>>(
                                 a, nbr_out, cnt_out, F_out)));
}

void launch_mean_force_blocks(const DevArrays& a, cudaStream_t st) {
    const unsigned nb = force_blocks(a.N);
    RCPG_DISPATCH_ND(a.ndim, (k_mean_force_blocks<ND><<<nb, kForceBlock, 0, st>>>(a)));
}

}  // namespace rcpg
