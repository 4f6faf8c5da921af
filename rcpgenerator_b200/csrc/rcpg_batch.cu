// Persistent batch engine: many independent packings in one launch.
//
// Each thread block runs whole packings, one at a time, taken from a queue:
// the same step as the graph engine (rcpg_engine.cu, graph mode) -- build when
// triggered, forces, controller, ADAM + refresh trigger, periodic reorder --
// but with every phase done by the block and separated by block barriers, so
// a step of a small packing costs no kernel launch at all. Packings of uneven
// N share the GPU through the queue (a block that finishes one takes the
// next). All instances of one launch have the same ndim (the host groups them).
//
// A launch runs every unfinished instance for at most `chunk` steps; the host
// relaunches until all are done, so each launch stays short. An instance
// whose neighbour rows outgrow their capacity is stopped (status 3) and the
// host runs it again from the start with twice the capacity.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <map>
#include <mutex>
#include <tuple>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <stdexcept>
#include <string>
#include <vector>

#include "rcpg_batch.h"
#include "rcpg_devutil.cuh"
#include "rcpg_setup.h"

namespace rcpg {

namespace {

constexpr int kBT = 256;            // threads per block (one per digit of the reorder's radix sort)
constexpr int kBW = kBT / 32;       // warps per block

// One instance's arrays (pointers already offset to the instance).
struct View {
    std::uint64_t N;
    std::uint32_t S, C_alloc;
    double *pos, *spos, *F, *m, *v, *x_last, *pos_tmp, *vec_tmp;
    std::uint32_t *nbr, *nbr_cnt, *caps, *cell_of, *cell_rank, *cell_list, *work, *cell_count, *cell_start;
    std::uint64_t *origin, *u64_tmp, *keys0, *keys1;
    std::uint32_t *vals0, *vals1;
    Histories hist;
    DevCtl* ctl;
    BatchInst* inst;
};

__device__ View make_view(const BatchArrays& B, std::uint32_t k, int ndim) {
    BatchInst* I = B.inst + k;
    View V;
    const std::uint64_t o = I->off;
    const int P = pos_stride(ndim);
    V.N = I->N;
    V.S = I->S;
    V.C_alloc = I->C_alloc;
    V.pos = B.pos + o * P;
    V.spos = B.spos + o * P;
    V.pos_tmp = B.pos_tmp + o * P;
    V.F = B.F + o * ndim;
    V.m = B.m + o * ndim;
    V.v = B.v + o * ndim;
    V.x_last = B.x_last + o * ndim;
    V.vec_tmp = B.vec_tmp + o * ndim;
    V.nbr = B.nbr + I->nbr_off;
    V.nbr_cnt = B.nbr_cnt + o;
    V.caps = B.caps + o;
    V.cell_of = B.cell_of + o;
    V.cell_rank = B.cell_rank + o;
    V.cell_list = B.cell_list + o;
    V.work = B.work + o;
    V.cell_count = B.cell_count + I->cell_off;
    V.cell_start = B.cell_start + I->cell_off;
    V.origin = B.origin + o;
    V.u64_tmp = B.u64_tmp + o;
    V.keys0 = B.keys0 + o;
    V.keys1 = B.keys1 + o;
    V.vals0 = B.vals0 + o;
    V.vals1 = B.vals1 + o;
    const std::uint64_t h = I->hist_off;
    V.hist = Histories{B.h_phi + h, B.h_force + h, B.h_energy + h, B.h_maxov + h,
                       B.h_mu + h, B.h_alpha + h, B.h_muflag + h};
    V.ctl = B.ctl + k;
    V.inst = I;
    return V;
}

struct Shared {
    Controller cs;
    ForceSums red[kBW];
    std::uint32_t wsum[kBW];
    unsigned long long wsum64[kBW];
    std::uint32_t hist[256];
    std::uint32_t base[256];
    std::uint32_t wcnt[kBW][256];
    std::uint32_t need, carry, flag;
    int publish;
};

// ---- A. ADAM of the finished step + refresh trigger (k_adam_refresh) -------
template <int ND>
__device__ bool b_adam_refresh(const View& V, bool do_adam, bool do_refresh) {
    const DevCtl* ctl = V.ctl;
    const bool adam = do_adam && ctl->adam_go;
    const bool refresh = do_refresh && !ctl->stopped && ctl->c.rebuild_mode == REBUILD_CHECK;
    bool trig = false;
    if (adam || refresh) {
        const double alpha = ctl->adam_alpha, ib1 = ctl->adam_inv_b1, ib2 = ctl->adam_inv_b2;
        const double fh = ctl->fix_height_scale;
        const double rk = ctl->refresh_kappa, kmin = ctl->kappa_min, theta = ctl->theta;
        double abox[ND];
#pragma unroll
        for (int d = 0; d < ND; ++d) abox[d] = ctl->adam_box[d];
        for (std::uint64_t i = threadIdx.x; i < V.N; i += kBT) {
            double x[ND], D0;
            load_pos<ND>(V.pos, i, x, D0);
            if (adam) {
#pragma unroll
                for (int d = 0; d < ND; ++d) {
                    double mm = V.m[i * ND + d], vv = V.v[i * ND + d];
                    x[d] = adam_coord(V.F[i * ND + d], mm, vv, x[d], alpha, ib1, ib2, abox[d]);
                    V.m[i * ND + d] = mm;
                    V.v[i * ND + d] = vv;
                }
                if (fh != 1.0) x[ND - 1] = xmul(x[ND - 1], fh);
                store_pos<ND>(V.pos, i, x, D0);
            }
            if (refresh) {
                double d2 = 0.0;
#pragma unroll
                for (int d = 0; d < ND; ++d) {
                    const double dd = xsub(x[d], V.x_last[i * ND + d]);
                    d2 = xadd(d2, xmul(dd, dd));
                }
                trig = trig || refresh_trigger(d2, xmul(D0, rk), xmul(D0, kmin), theta);
            }
        }
    }
    return __syncthreads_or(trig) != 0;
}

// ---- B. pair-list build (k_build_prepare / bin / scan / scatter / cell sort
// / warp search, one block) ------------------------------------------------
template <int ND>
__device__ void b_build(const View& V, Shared& sh) {
    DevCtl* ctl = V.ctl;
    const std::uint64_t N = V.N;
    if (threadIdx.x == 0) {
        const double cutoff = (ctl->build_Dmax + ctl->build_t_shell) * (1.0 + 1e-6);
        long long nc[ND];
        double total = 1.0;
        for (int d = 0; d < ND; ++d) {
            double q = floor(ctl->g.box[d] / cutoff);
            if (!(q >= 1.0)) q = 1.0;
            if (q > 1048576.0) q = 1048576.0;
            nc[d] = static_cast<long long>(q);
            total *= q;
        }
        while (total > static_cast<double>(V.C_alloc)) {
            int dm = 0;
            for (int d = 1; d < ND; ++d)
                if (nc[d] > nc[dm]) dm = d;
            const long long nn = (nc[dm] * 3) / 4;
            total = total / static_cast<double>(nc[dm]) * static_cast<double>(nn < 1 ? 1 : nn);
            nc[dm] = nn < 1 ? 1 : nn;
        }
        std::uint32_t cells = 1;
        for (int d = 0; d < ND; ++d) {
            ctl->ncell[d] = static_cast<int>(nc[d]);
            ctl->cell_scale[d] = static_cast<double>(nc[d]) / ctl->g.box[d];
            cells *= static_cast<std::uint32_t>(nc[d]);
        }
        ctl->ncells = cells;
        ctl->kappa_min = ctl->build_kappa;  // every build re-anchors every particle
        ctl->forces_done = 0u;
        ctl->row_need = 0u;
        ctl->nbuilds += 1u;
        sh.need = 0u;
    }
    __syncthreads();
    const std::uint32_t ncells = ctl->ncells;
    for (std::uint32_t c = threadIdx.x; c <= ncells; c += kBT) V.cell_count[c] = 0u;
    __syncthreads();
    int nc[ND];
    double scale[ND];
#pragma unroll
    for (int d = 0; d < ND; ++d) {
        nc[d] = ctl->ncell[d];
        scale[d] = ctl->cell_scale[d];
    }
    // bin
    for (std::uint64_t i = threadIdx.x; i < N; i += kBT) {
        double x[ND], D0;
        load_pos<ND>(V.pos, i, x, D0);
        std::uint32_t c = 0, mul = 1;
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            c += static_cast<std::uint32_t>(cell_coord(x[d], scale[d], nc[d])) * mul;
            mul *= static_cast<std::uint32_t>(nc[d]);
            V.x_last[i * ND + d] = x[d];
        }
        V.cell_of[i] = c;
        V.cell_rank[i] = atomicAdd(&V.cell_count[c], 1u);
    }
    __syncthreads();
    // exclusive scan of the counts, a block-wide chunk at a time
    if (threadIdx.x == 0) sh.carry = 0u;
    __syncthreads();
    for (std::uint32_t c0 = 0; c0 <= ncells; c0 += kBT) {
        const std::uint32_t c = c0 + threadIdx.x;
        const std::uint32_t v = c <= ncells ? V.cell_count[c] : 0u;
        std::uint32_t total;
        const std::uint32_t off = block_exclusive_scan<std::uint32_t>(v, sh.wsum, total);
        if (c <= ncells) V.cell_start[c] = sh.carry + off;
        __syncthreads();
        if (threadIdx.x == 0) sh.carry += total;
        __syncthreads();
    }
    // scatter (arrival order)
    for (std::uint64_t i = threadIdx.x; i < N; i += kBT)
        V.cell_list[V.cell_start[V.cell_of[i]] + V.cell_rank[i]] = static_cast<std::uint32_t>(i);
    __syncthreads();
    // each cell's members in ascending order (work) and their positions (spos)
    constexpr int P = pos_stride(ND);
    for (std::uint32_t c = threadIdx.x; c < ncells; c += kBT) {
        const std::uint32_t q0 = V.cell_start[c], q1 = V.cell_start[c + 1];
        for (std::uint32_t k = q0; k < q1; ++k) {
            const std::uint32_t v = V.cell_list[k];
            std::uint32_t p = k;
            while (p > q0 && V.work[p - 1] > v) {
                V.work[p] = V.work[p - 1];
                --p;
            }
            V.work[p] = v;
        }
        for (std::uint32_t q = q0; q < q1; ++q) {
            const double2* src = reinterpret_cast<const double2*>(V.pos + static_cast<std::uint64_t>(V.work[q]) * P);
            double2* dst = reinterpret_cast<double2*>(V.spos + static_cast<std::uint64_t>(q) * P);
#pragma unroll
            for (int h = 0; h < P / 2; ++h) dst[h] = src[h];
        }
    }
    __syncthreads();
    // search: one thread per row slot, partners in the fixed scan order (cells
    // of the 3^ndim neighbourhood in odometer order, members ascending), so the
    // rows are deterministic without a sort
    const std::uint32_t S = V.S;
    const Geometry& g = ctl->g;
    const double kap = ctl->build_kappa, t_shell = ctl->build_t_shell;
    double bx[ND], ibx[ND];
    int nn[ND];
    int total_combo = 1;
#pragma unroll
    for (int d = 0; d < ND; ++d) {
        bx[d] = g.box[d];
        ibx[d] = g.inv_box[d];
        nn[d] = nc[d] < 3 ? nc[d] : 3;
        total_combo *= nn[d];
    }
    std::uint32_t need = 0;
    for (std::uint64_t t = threadIdx.x; t < N; t += kBT) {
        const std::uint32_t i = V.work[t];
        double xi[ND], D0i;
        load_pos<ND>(V.spos, t, xi, D0i);
        const double Di = xmul(D0i, kap);
        int cc[ND];
#pragma unroll
        for (int d = 0; d < ND; ++d) cc[d] = cell_coord(xi[d], scale[d], nc[d]);
        std::uint32_t n = 0, n_half = 0;
        for (int combo = 0; combo < total_combo; ++combo) {
            std::uint32_t cell = 0, mul = 1;
            int r = combo;
#pragma unroll
            for (int d = 0; d < ND; ++d) {
                const int k = r % nn[d];
                r /= nn[d];
                int c = (nc[d] >= 3) ? cc[d] - 1 + k : k;
                if (c < 0) c += nc[d];
                else if (c >= nc[d]) c -= nc[d];
                cell += static_cast<std::uint32_t>(c) * mul;
                mul *= static_cast<std::uint32_t>(nc[d]);
            }
            const std::uint32_t q0 = V.cell_start[cell], q1 = V.cell_start[cell + 1];
            for (std::uint32_t q = q0; q < q1; ++q) {
                const std::uint32_t j = V.work[q];
                double xj[ND], D0j;
                load_pos<ND>(V.spos, q, xj, D0j);
                if (j == i) continue;
                const double Dj = xmul(D0j, kap);
                const bool ok = (ND <= 3 || j > i) ? in_shell<ND>(xi, xj, Di, Dj, bx, ibx, t_shell)
                                                   : in_shell<ND>(xi, xj, Dj, Di, bx, ibx, t_shell);
                if (!ok) continue;
                if (n < S) V.nbr[static_cast<std::uint64_t>(n) * N + t] = j;
                ++n;
                if (j > i) ++n_half;
            }
        }
        const std::uint32_t cap = V.caps[i];
        if (n_half > cap) report_cap_error(ctl, i, cap);
        need = need > n ? need : n;
        V.nbr_cnt[t] = n > S ? 0u : n;
    }
    atomicMax(&sh.need, need);
    __syncthreads();
    if (threadIdx.x == 0) {
        ctl->row_need = sh.need;
        ctl->rebuild_flag = 0u;
    }
    __syncthreads();
}

// ---- C. forces + walls + block sums (k_forces, graph variant) --------------
template <int ND>
__device__ ForceSums b_forces(const View& V, Shared& sh, bool mixed) {
    const DevCtl* ctl = V.ctl;
    const std::uint64_t N = V.N;
    const Geometry& g = ctl->g;
    double bx[ND], ibx[ND];
    float hbf[ND];
#pragma unroll
    for (int d = 0; d < ND; ++d) {
        bx[d] = g.box[d];
        ibx[d] = g.inv_box[d];
        hbf[d] = static_cast<float>(0.5 * bx[d]);
    }
    const double kap = ctl->force_kappa;
    const float kapf = static_cast<float>(kap);
    // the wall terms join the pair chains (the finalisation adds them anyway)
    double sU = 0.0, sLc = 0.0, sdk = 0.0, sFm = 0.0, smax = 0.0, smag = 0.0, sD = 0.0;
    std::uint32_t scount = 0, smagc = 0;
    for (std::uint64_t t = threadIdx.x; t < N; t += kBT) {
        const std::uint64_t i = V.work[t];
        double xi[ND], D0i;
        load_pos<ND>(V.pos, i, xi, D0i);
        const double Di = xmul(D0i, kap);
        const float Dif = static_cast<float>(D0i) * kapf;
        double fi[ND];
        float fif[ND];
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            fi[d] = 0.0;
            fif[d] = 0.0f;
        }
        const std::uint32_t n = min(V.nbr_cnt[t], V.S);
        // partners in chunks: the ids, then the positions of a chunk are loaded
        // before its arithmetic (several gathers in flight per thread)
        constexpr std::uint32_t kC = 2;
        for (std::uint32_t k0 = 0; k0 < n; k0 += kC) {
          std::uint32_t jj[kC];
          double xjc[kC][ND], D0c[kC];
#pragma unroll
          for (std::uint32_t u = 0; u < kC; ++u)
              jj[u] = (k0 + u < n) ? V.nbr[static_cast<std::uint64_t>(k0 + u) * N + t] : 0xffffffffu;
#pragma unroll
          for (std::uint32_t u = 0; u < kC; ++u)
              if (jj[u] < N) load_pos<ND>(V.pos, jj[u], xjc[u], D0c[u]);
#pragma unroll
          for (std::uint32_t u = 0; u < kC; ++u) {
            const std::uint32_t j = jj[u];
            if (j >= N) continue;
            const double* xj = xjc[u];
            const double D0j = D0c[u];
            PairTerms pt;
            if (mixed) {
                float dxf[ND];
                const float d2f = mixed_disp<ND>(xi, xj, bx, hbf, dxf);
                const float rsum = 0.5f * (Dif + static_cast<float>(D0j) * kapf);
                if (!(d2f < rsum * rsum)) continue;
                pair_terms_mixed<ND>(dxf, d2f, rsum, fif, pt);
            } else {
                const double r_ij = xmul(0.5, xadd(Di, xmul(D0j, kap)));
                double dx[ND];
                const double d2 = pair_disp<ND>(xi, xj, bx, ibx, dx);
                if (!(d2 < xmul(r_ij, r_ij))) continue;
                pair_terms_f64<ND>(dx, d2, r_ij, fi, pt);
            }
            if (j > i) {
                sU = xadd(sU, pt.U);
                sLc = xadd(sLc, pt.Lc);
                sdk = xadd(sdk, pt.dk);
                sFm = xadd(sFm, pt.Fm);
                smax = fmax(smax, pt.U);
                ++scount;
            }
          }
        }
        if (mixed) {
#pragma unroll
            for (int d = 0; d < ND; ++d) fi[d] = static_cast<double>(fif[d]);
        }
        wall_forces<ND>(xi, Di, g, fi, sU, sdk, sFm, scount);
        const double f2 = force_norm2<ND>(fi);
        if (f2 > 1.0E-16) {
            smag = xadd(smag, xsqrt(f2));
            ++smagc;
        }
        sD = xadd(sD, Di);
#pragma unroll
        for (int d = 0; d < ND; ++d) V.F[i * ND + d] = fi[d];
    }
    ForceSums s;
    sums_zero(s);
    s.pair_U = sU;
    s.pair_Lc = sLc;
    s.pair_dk = sdk;
    s.pair_Fm = sFm;
    s.pair_maxov = smax;
    s.pair_count = scount;
    s.sum_mag = smag;
    s.mag_count = smagc;
    s.sum_D = sD;
    block_reduce_sums<kBT>(s, sh.red);
    __syncthreads();
    if (threadIdx.x == 0) sh.red[0] = s;
    __syncthreads();
    return sh.red[0];
}

// ---- R. spatial reorder (k_reorder_keys + LSD radix sort + gather) -------
template <int ND>
__device__ void b_reorder(const View& V, Shared& sh) {
    const std::uint64_t N = V.N;
    const std::uint32_t n = static_cast<std::uint32_t>(N);
    const Geometry& g = V.ctl->g;
    for (std::uint64_t i = threadIdx.x; i < N; i += kBT) {
        double x[ND], D0;
        load_pos<ND>(V.pos, i, x, D0);
        std::uint64_t key;
        if (ND == 3) {
            std::uint64_t code = 0;
#pragma unroll
            for (int d = 0; d < 3 && d < ND; ++d) {
                const double scale = (static_cast<double>(1u << 21) - 1.0) / g.box[d];
                code |= morton_spread21(morton_axis(x[d], g.box[d], scale)) << d;
            }
            key = code;
        } else {
            key = double_order_key(x[0]);
        }
        V.keys0[i] = key;
        V.vals0[i] = static_cast<std::uint32_t>(i);
    }
    __syncthreads();
    std::uint64_t* kin = V.keys0;
    std::uint64_t* kout = V.keys1;
    std::uint32_t* vin = V.vals0;
    std::uint32_t* vout = V.vals1;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int pass = 0; pass < 8; ++pass) {
        const int shift = pass * 8;
        sh.hist[threadIdx.x] = 0u;
        __syncthreads();
        for (std::uint32_t e = threadIdx.x; e < n; e += kBT) atomicAdd(&sh.hist[(kin[e] >> shift) & 0xFFu], 1u);
        __syncthreads();
        std::uint32_t total;
        const std::uint32_t off = block_exclusive_scan<std::uint32_t>(sh.hist[threadIdx.x], sh.wsum, total);
        sh.base[threadIdx.x] = off;
        __syncthreads();
        for (std::uint32_t c0 = 0; c0 < n; c0 += kBT) {
#pragma unroll
            for (int ww = 0; ww < kBW; ++ww) sh.wcnt[ww][threadIdx.x] = 0u;
            __syncthreads();
            const std::uint32_t e = c0 + threadIdx.x;
            const bool valid = e < n;
            std::uint64_t key = 0;
            std::uint32_t val = 0, digit = 0xFFFFFFFFu;
            if (valid) {
                key = kin[e];
                val = vin[e];
                digit = static_cast<std::uint32_t>((key >> shift) & 0xFFu);
            }
            const unsigned peers = __match_any_sync(0xffffffffu, digit);
            const std::uint32_t rank_w = __popc(peers & ((1u << lane) - 1u));
            if (valid && rank_w == 0) sh.wcnt[warp][digit] = __popc(peers);
            __syncthreads();
            if (valid) {
                std::uint32_t before = 0;
                for (int ww = 0; ww < warp; ++ww) before += sh.wcnt[ww][digit];
                const std::uint32_t p = sh.base[digit] + before + rank_w;
                kout[p] = key;
                vout[p] = val;
            }
            __syncthreads();
            std::uint32_t tot = 0;
#pragma unroll
            for (int ww = 0; ww < kBW; ++ww) tot += sh.wcnt[ww][threadIdx.x];
            sh.base[threadIdx.x] += tot;
            __syncthreads();
        }
        std::uint64_t* tk = kin;
        kin = kout;
        kout = tk;
        std::uint32_t* tv = vin;
        vin = vout;
        vout = tv;
    }
    // after 8 passes the sorted permutation is in vin (= vals0)
    constexpr int P = pos_stride(ND);
    for (std::uint64_t k = threadIdx.x; k < N; k += kBT) {
        const std::uint64_t src = vin[k];
#pragma unroll
        for (int q = 0; q < P; ++q) V.pos_tmp[k * P + q] = V.pos[src * P + q];
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            V.vec_tmp[k * ND + d] = V.m[src * ND + d];
            V.x_last[k * ND + d] = V.v[src * ND + d];
        }
        V.u64_tmp[k] = V.origin[src];
        V.cell_rank[k] = V.caps[src];
    }
    __syncthreads();
    for (std::uint64_t k = threadIdx.x; k < N; k += kBT) {
#pragma unroll
        for (int q = 0; q < P; ++q) V.pos[k * P + q] = V.pos_tmp[k * P + q];
#pragma unroll
        for (int d = 0; d < ND; ++d) {
            V.m[k * ND + d] = V.vec_tmp[k * ND + d];
            V.v[k * ND + d] = V.x_last[k * ND + d];
        }
        V.origin[k] = V.u64_tmp[k];
        V.caps[k] = V.cell_rank[k];
    }
    __syncthreads();
}

// Rebuild flag from the refresh trigger, set by thread 0 after the block OR.
__device__ __forceinline__ void set_trigger(DevCtl* ctl, bool trig) {
    if (threadIdx.x == 0 && trig) ctl->rebuild_flag = 1u;
    __syncthreads();
}

// Controller step (k_controller): finish the step just computed, open the
// next one. Thread 0 works on the shared copy of the controller.
__device__ void b_controller(const View& V, Shared& sh, const ForceSums& s, int ndim, bool open_only) {
    DevCtl* ctl = V.ctl;
    if (threadIdx.x == 0) {
        sh.cs = ctl->c;
        Controller& c = sh.cs;
        sh.publish = 0;
        bool go = true;
        if (!open_only) {
            ctl->sums = s;
            if (ctl->row_need > V.S || ctl->cap_error) {
                ctl->halted = 1u;
                ctl->adam_go = 0u;
                go = false;
            } else {
                const StepScalars sc = finalize_sums(s, ctl->force_mu, ndim);
                ctl->scal = sc;
                end_step(c, V.hist, sc);
                if (ctl->pair_fp32 && sc.max_overlap > 0.0 && sc.max_overlap < ctl->mixed_switch) {
                    ctl->pair_fp32 = 0u;
                    ctl->fp64_switch_step = c.steps;
                }
                ctl->graph_steps += 1ull;
                for (int d = 0; d < ndim; ++d) ctl->adam_box[d] = c.box[d];
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
            } else {
                begin_step(c, V.hist, c.steps + 1);
                ctl->fix_height_scale = c.reorder ? 1.0 : c.fix_height_scale;
                if (c.done || c.reorder || c.lock_now) ctl->stopped = 1u;
                else sh.publish = 1;
            }
        }
        ctl->c = c;
        if (sh.publish) publish_step(ctl, c, ndim);
    }
    __syncthreads();
}

// Reorder step, fix_height stretch and reopening after a stop (the graph
// engine's host-side after_stop, here on the device).
template <int ND>
__device__ void b_after_stop(const View& V, Shared& sh) {
    DevCtl* ctl = V.ctl;
    const Controller& c = ctl->c;
    if (c.reorder) {
        if (threadIdx.x == 0) {
            const double kp = c.runtime_fix_diameter ? 1.0 : c.kappa_D_prev;
            ctl->build_kappa = kp;
            ctl->build_t_shell = shell_of(xmul(c.D0_min, kp), xmul(c.D0_med, kp), xmul(c.D0_max, kp));
            ctl->build_Dmax = xmul(c.D0_max, kp);
        }
        __syncthreads();
        b_reorder<ND>(V, sh);
        b_build<ND>(V, sh);
        if (ctl->row_need > V.S || ctl->cap_error) {
            if (threadIdx.x == 0) ctl->halted = 1u;
            __syncthreads();
            return;
        }
    }
    if (c.fix_height && !c.runtime_fix_diameter && c.fix_height_scale != 1.0 && c.reorder) {
        const double sc = c.fix_height_scale;
        for (std::uint64_t i = threadIdx.x; i < V.N; i += kBT) {
            double* p = V.pos + i * pos_stride(ND) + (ND - 1);
            *p = xmul(*p, sc);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        publish_step(ctl, ctl->c, ND);
        ctl->adam_go = 0u;
        ctl->stopped = 0u;
        ctl->halted = 0u;
    }
    __syncthreads();
    if (ctl->c.rebuild_mode == REBUILD_CHECK) set_trigger(ctl, b_adam_refresh<ND>(V, false, true));
}

// Instance finished (2), stopped for a larger row capacity (3) or a capacity
// error of the reference layout (4), or unsupported (5: a target-phi lock).
__device__ void b_finish(const View& V, std::uint32_t status) {
    if (threadIdx.x == 0) V.inst->status = status;
    __syncthreads();
}

template <int ND>
__device__ void run_instance(const View& V, Shared& sh, std::uint32_t chunk, int mixed) {
    DevCtl* ctl = V.ctl;
    std::uint32_t status = V.inst->status;
    __syncthreads();
    if (status == 0u) {
        // set-up of the graph engine (Engine::upload_initial + the opening of step 1)
        if (ctl->c.reorder_interval > 0) b_reorder<ND>(V, sh);
        b_build<ND>(V, sh);
        if (ctl->row_need > V.S || ctl->cap_error) {
            b_finish(V, ctl->cap_error ? 4u : 3u);
            return;
        }
        const ForceSums s0 = b_forces<ND>(V, sh, false);
        if (threadIdx.x == 0) {
            ctl->sums = s0;
            const StepScalars sc = finalize_sums(s0, ctl->c.mu, ND);
            ctl->c.U = sc.U;
            ctl->c.max_min_dist = sc.max_overlap;
            ctl->rebuild_flag = 0u;
            ctl->stopped = 0u;
            ctl->halted = 0u;
            ctl->pair_fp32 = mixed ? 1u : 0u;
        }
        __syncthreads();
        b_controller(V, sh, s0, ND, true);
        if (ctl->stopped) {
            const Controller& c = ctl->c;
            if (c.done || c.steps + 1 > c.step_cap) {
                b_finish(V, 2u);
                return;
            }
            if (c.lock_now) {
                b_finish(V, 5u);
                return;
            }
            b_after_stop<ND>(V, sh);
        } else if (ctl->c.rebuild_mode == REBUILD_CHECK) {
            set_trigger(ctl, b_adam_refresh<ND>(V, false, true));
        }
        if (threadIdx.x == 0) V.inst->status = 1u;
        __syncthreads();
    }
    for (std::uint32_t it = 0; it < chunk; ++it) {
        if (ctl->halted) {
            b_finish(V, ctl->cap_error ? 4u : 3u);
            return;
        }
        if (ctl->rebuild_flag) b_build<ND>(V, sh);
        const ForceSums s = b_forces<ND>(V, sh, ctl->pair_fp32 != 0u);
        b_controller(V, sh, s, ND, false);
        set_trigger(ctl, b_adam_refresh<ND>(V, true, true));
        if (ctl->halted) {
            b_finish(V, ctl->cap_error ? 4u : 3u);
            return;
        }
        if (ctl->stopped) {
            const Controller& c = ctl->c;
            if (c.done || c.steps + 1 > c.step_cap || c.hist_filled >= c.step_cap) {
                b_finish(V, 2u);
                return;
            }
            if (c.lock_now) {
                b_finish(V, 5u);
                return;
            }
            b_after_stop<ND>(V, sh);
        }
    }
}

template <int ND>
__global__ void __launch_bounds__(kBT, 2) k_batch(BatchArrays B, std::uint32_t chunk, int mixed) {
    extern __shared__ __align__(16) unsigned char batch_smem[];
    Shared& sh = *reinterpret_cast<Shared*>(batch_smem);
    __shared__ std::uint32_t s_k;
    for (;;) {
        if (threadIdx.x == 0) s_k = atomicAdd(B.queue, 1u);
        __syncthreads();
        const std::uint32_t q = s_k;
        __syncthreads();
        if (q >= B.nactive) return;
        const std::uint32_t k = B.active[q];
        const View V = make_view(B, k, ND);
        run_instance<ND>(V, sh, chunk, mixed);
    }
}

}  // namespace

void launch_batch(const BatchArrays& B, int ndim, std::uint32_t chunk, int mixed, int device,
                  int blocks_per_sm, cudaStream_t st) {
    const std::size_t smem = sizeof(Shared);
    int sms = 148, per = 1;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    switch (ndim) {
#define RCPG_BATCH_CASE(D)                                                                          \
    case D: {                                                                                       \
        cudaFuncSetAttribute(k_batch<D>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)); \
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_batch<D>, kBT, smem);                 \
        if (per > blocks_per_sm) per = blocks_per_sm;                                               \
        const unsigned grid = static_cast<unsigned>(sms * (per > 0 ? per : 1));                     \
        k_batch<D><<<grid, kBT, smem, st>>>(B, chunk, mixed);                                       \
    } break;
        RCPG_BATCH_CASE(2)
        RCPG_BATCH_CASE(3)
        RCPG_BATCH_CASE(4)
        RCPG_BATCH_CASE(5)
        RCPG_BATCH_CASE(6)
        RCPG_BATCH_CASE(7)
        RCPG_BATCH_CASE(8)
#undef RCPG_BATCH_CASE
        default:
            break;
    }
}


// ---------------------------------------------------------------------------
// host driver
// ---------------------------------------------------------------------------
namespace {

// Row capacity to start from (grown by doubling for the packings that outgrow it).
std::uint32_t base_row_capacity(int ndim) {
    switch (ndim) {
        case 2: return 32;
        case 3: return 64;
        case 4: return 160;
        default: return 320;
    }
}

struct Pool {
    cudaStream_t st;
    std::vector<void*> ptrs;
    explicit Pool(cudaStream_t s) : st(s) {}
    template <typename T>
    T* get(std::size_t n) {
        void* p = nullptr;
        const cudaError_t e = pool_alloc_async(&p, n * sizeof(T), st);
        if (e != cudaSuccess) {
            cudaGetLastError();
            throw EngineError(-2, std::string("rcpgenerator_b200: batch allocation failed: ") + cudaGetErrorString(e));
        }
        ptrs.push_back(p);
        return static_cast<T*>(p);
    }
    ~Pool() {
        for (void* p : ptrs) cudaFreeAsync(p, st);
        cudaStreamSynchronize(st);
    }
};

void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw EngineError(-2, std::string("rcpgenerator_b200: CUDA error in ") + what + ": " + cudaGetErrorString(e));
    }
}

// One launch group: packings of one ndim, run to completion. Returns the
// final status of each.
std::vector<std::uint32_t> run_group(const std::vector<EngineInput>& ins, const std::vector<RunSetup>& su,
                                     const std::vector<std::size_t>& idx, std::uint32_t mult,
                                     std::uint32_t chunk, int blocks_per_sm, cudaStream_t st,
                                     std::vector<BatchOutcome>& out) {
    const int nd = su[idx[0]].ndim;
    const int P = pos_stride(nd);
    const std::size_t K = idx.size();
    std::vector<BatchInst> inst(K);
    std::uint64_t Ntot = 0, nbr_tot = 0, cell_tot = 0, hist_tot = 0;
    for (std::size_t q = 0; q < K; ++q) {
        const RunSetup& r = su[idx[q]];
        BatchInst& I = inst[q];
        I.N = static_cast<std::uint32_t>(r.N);
        std::uint64_t S = static_cast<std::uint64_t>(base_row_capacity(nd)) * mult;
        if (S > r.N) S = std::max<std::uint64_t>(r.N, 1);
        I.S = static_cast<std::uint32_t>(S);
        const double cutoff = (r.c.Dmax_cur + r.c.t_shell) * (1.0 + 1e-6);
        double cells = 1.0;
        for (int d = 0; d < nd; ++d) cells *= std::max(1.0, std::floor(r.c.box[d] / cutoff));
        const double cap = std::min(cells * 1.5 + 64.0, 8.0 * static_cast<double>(r.N) + 1024.0);
        I.C_alloc = static_cast<std::uint32_t>(cap);
        I.off = Ntot;
        I.nbr_off = nbr_tot;
        I.cell_off = cell_tot;
        I.hist_off = hist_tot;
        I.status = 0u;
        Ntot += r.N;
        nbr_tot += static_cast<std::uint64_t>(I.S) * r.N;
        cell_tot += I.C_alloc + 1ull;
        hist_tot += r.c.step_cap + 1;
    }
    Pool pool(st);
    BatchArrays B{};
    B.pos = pool.get<double>(Ntot * P);
    B.spos = pool.get<double>(Ntot * P);
    B.pos_tmp = pool.get<double>(Ntot * P);
    B.F = pool.get<double>(Ntot * nd);
    B.m = pool.get<double>(Ntot * nd);
    B.v = pool.get<double>(Ntot * nd);
    B.x_last = pool.get<double>(Ntot * nd);
    B.vec_tmp = pool.get<double>(Ntot * nd);
    B.nbr = pool.get<std::uint32_t>(nbr_tot);
    B.nbr_cnt = pool.get<std::uint32_t>(Ntot);
    B.caps = pool.get<std::uint32_t>(Ntot);
    B.cell_of = pool.get<std::uint32_t>(Ntot);
    B.cell_rank = pool.get<std::uint32_t>(Ntot);
    B.cell_list = pool.get<std::uint32_t>(Ntot);
    B.work = pool.get<std::uint32_t>(Ntot);
    B.cell_count = pool.get<std::uint32_t>(cell_tot);
    B.cell_start = pool.get<std::uint32_t>(cell_tot);
    B.origin = pool.get<std::uint64_t>(Ntot);
    B.u64_tmp = pool.get<std::uint64_t>(Ntot);
    B.keys0 = pool.get<std::uint64_t>(Ntot);
    B.keys1 = pool.get<std::uint64_t>(Ntot);
    B.vals0 = pool.get<std::uint32_t>(Ntot);
    B.vals1 = pool.get<std::uint32_t>(Ntot);
    B.h_phi = pool.get<double>(hist_tot);
    B.h_force = pool.get<double>(hist_tot);
    B.h_energy = pool.get<double>(hist_tot);
    B.h_maxov = pool.get<double>(hist_tot);
    B.h_mu = pool.get<double>(hist_tot);
    B.h_alpha = pool.get<double>(hist_tot);
    B.h_muflag = pool.get<std::int8_t>(hist_tot);
    B.ctl = pool.get<DevCtl>(K);
    B.inst = pool.get<BatchInst>(K);
    B.active = pool.get<std::uint32_t>(K);
    B.queue = pool.get<std::uint32_t>(1);

    // initial state of every packing (Engine::upload_initial)
    std::vector<double> pos(Ntot * P, 0.0);
    std::vector<std::uint64_t> origin(Ntot);
    std::vector<std::uint32_t> caps(Ntot);
    std::vector<DevCtl> ctl(K);
    const bool mixed = ins[idx[0]].pair_precision == 1;
    for (std::size_t q = 0; q < K; ++q) {
        const RunSetup& r = su[idx[q]];
        const std::uint64_t o = inst[q].off;
        for (std::uint64_t i = 0; i < r.N; ++i) {
            for (int d = 0; d < nd; ++d) pos[(o + i) * P + d] = r.x[i * nd + d];
            pos[(o + i) * P + nd] = r.D0[i];
            origin[o + i] = i;
            caps[o + i] = r.caps[i];
        }
        DevCtl& h = ctl[q];
        std::memset(&h, 0, sizeof(h));
        Geometry& g = h.g;
        g.ndim = nd;
        g.circle_k = r.walls[0] < 0 ? -r.walls[0] : 0;
        for (int d = 0; d < nd; ++d) {
            g.walls[d] = r.walls[d];
            if (r.walls[d] == 1) g.any_flat_wall = 1;
            g.box[d] = r.c.box[d];
            g.inv_box[d] = 1.0 / r.c.box[d];
        }
        h.c = r.c;
        h.fix_height_scale = 1.0;
        h.build_kappa = 1.0;
        h.build_t_shell = r.c.t_shell;
        h.build_Dmax = r.c.Dmax_cur;
        h.refresh_kappa = 1.0;
        h.kappa_min = 1.0;
        h.theta = r.c.theta;
        h.force_kappa = 1.0;
        h.force_mu = r.c.mu;
        h.rebuild_flag = 1u;
        h.mixed_switch = ins[idx[q]].mixed_switch > 0.0 ? ins[idx[q]].mixed_switch : 1e-5;
    }
    ck(cudaMemcpyAsync(B.pos, pos.data(), pos.size() * 8, cudaMemcpyHostToDevice, st), "H2D pos");
    ck(cudaMemcpyAsync(B.origin, origin.data(), Ntot * 8, cudaMemcpyHostToDevice, st), "H2D origin");
    ck(cudaMemcpyAsync(B.caps, caps.data(), Ntot * 4, cudaMemcpyHostToDevice, st), "H2D caps");
    ck(cudaMemcpyAsync(B.ctl, ctl.data(), K * sizeof(DevCtl), cudaMemcpyHostToDevice, st), "H2D ctl");
    ck(cudaMemcpyAsync(B.inst, inst.data(), K * sizeof(BatchInst), cudaMemcpyHostToDevice, st), "H2D inst");
    ck(cudaMemsetAsync(B.m, 0, Ntot * nd * 8, st), "memset");
    ck(cudaMemsetAsync(B.v, 0, Ntot * nd * 8, st), "memset");
    ck(cudaMemsetAsync(B.F, 0, Ntot * nd * 8, st), "memset");
    ck(cudaMemsetAsync(B.nbr_cnt, 0, Ntot * 4, st), "memset");
    for (double* hp : {B.h_phi, B.h_force, B.h_energy, B.h_maxov, B.h_mu, B.h_alpha})
        ck(cudaMemsetAsync(hp, 0, hist_tot * 8, st), "memset");
    ck(cudaMemsetAsync(B.h_muflag, 0, hist_tot, st), "memset");

    int device = 0;
    cudaGetDevice(&device);
    std::vector<std::uint32_t> active(K);
    std::iota(active.begin(), active.end(), 0u);
    std::vector<BatchInst> now(K);
    while (!active.empty()) {
        ck(cudaMemcpyAsync(B.active, active.data(), active.size() * 4, cudaMemcpyHostToDevice, st), "H2D active");
        ck(cudaMemsetAsync(B.queue, 0, 4, st), "memset");
        B.nactive = static_cast<std::uint32_t>(active.size());
        launch_batch(B, nd, chunk, mixed ? 1 : 0, device, blocks_per_sm, st);
        ck(cudaGetLastError(), "batch launch");
        ck(cudaMemcpyAsync(now.data(), B.inst, K * sizeof(BatchInst), cudaMemcpyDeviceToHost, st), "D2H inst");
        ck(cudaStreamSynchronize(st), "batch kernel");
        std::vector<std::uint32_t> next;
        for (std::uint32_t q : active)
            if (now[q].status <= 1u) next.push_back(q);
        active.swap(next);
    }

    // results
    ck(cudaMemcpyAsync(pos.data(), B.pos, pos.size() * 8, cudaMemcpyDeviceToHost, st), "D2H pos");
    ck(cudaMemcpyAsync(origin.data(), B.origin, Ntot * 8, cudaMemcpyDeviceToHost, st), "D2H origin");
    ck(cudaMemcpyAsync(ctl.data(), B.ctl, K * sizeof(DevCtl), cudaMemcpyDeviceToHost, st), "D2H ctl");
    std::vector<double> hv[6];
    std::vector<std::int8_t> hm(hist_tot);
    double* hsrc[6] = {B.h_phi, B.h_force, B.h_energy, B.h_maxov, B.h_mu, B.h_alpha};
    for (int a = 0; a < 6; ++a) {
        hv[a].resize(hist_tot);
        ck(cudaMemcpyAsync(hv[a].data(), hsrc[a], hist_tot * 8, cudaMemcpyDeviceToHost, st), "D2H hist");
    }
    ck(cudaMemcpyAsync(hm.data(), B.h_muflag, hist_tot, cudaMemcpyDeviceToHost, st), "D2H hist");
    ck(cudaStreamSynchronize(st), "D2H");
    std::vector<std::uint32_t> status(K);
    for (std::size_t q = 0; q < K; ++q) {
        status[q] = now[q].status;
        if (status[q] != 2u) continue;
        const RunSetup& r = su[idx[q]];
        const Controller& c = ctl[q].c;
        BatchOutcome& o = out[idx[q]];
        EngineResult& R = o.result;
        const std::uint64_t off = inst[q].off, N = r.N;
        R.positions.resize(N * nd);
        R.diameters.resize(N);
        const double kd = c.runtime_fix_diameter ? 1.0 : c.kappa_D;
        for (std::uint64_t i = 0; i < N; ++i) {
            for (int d = 0; d < nd; ++d) R.positions[i * nd + d] = pos[(off + i) * P + d];
            const double D0 = pos[(off + i) * P + nd];
            R.diameters[i] = c.runtime_fix_diameter ? D0 : D0 * kd;
        }
        R.particle_origin.assign(origin.begin() + off, origin.begin() + off + N);
        R.box.assign(c.box, c.box + nd);
        R.walls = r.walls;
        const std::size_t n = c.hist_filled, h0 = inst[q].hist_off;
        std::vector<double>* dst[6] = {&R.phi_history, &R.force_history, &R.energy_history,
                                       &R.max_overlap_history, &R.mu_history, &R.alpha_history};
        for (int a = 0; a < 6; ++a) dst[a]->assign(hv[a].begin() + h0, hv[a].begin() + h0 + n);
        R.mu_flag_history.assign(hm.begin() + h0, hm.begin() + h0 + n);
        R.steps = n;
        R.phi = c.phi;
        R.max_min_dist = c.max_min_dist;
        R.force_magnitude = c.F_magnitude;
        R.builds = ctl[q].nbuilds;
        R.row_capacity = inst[q].S;
        R.fp64_switch_step = ctl[q].fp64_switch_step;
        R.pair_energy_rel_error = R.pair_force_rel_error = std::nan("");
        o.N = N;
        o.ndim = nd;
        o.code = 0;
    }
    return status;
}

}  // namespace

namespace {
constexpr std::uint64_t kTunePackingN = 256;
constexpr std::uint64_t kTuneSteps = 200;
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int>, BatchTuning> g_tuned;
}  // namespace

BatchTuning tune_batch(int ndim, int device, bool mixed) {
    const auto key = std::make_tuple(device, ndim, mixed ? 1 : 0);
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tuned.find(key);
        if (it != g_tuned.end()) return it->second;
    }
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    std::vector<EngineInput> ins(static_cast<std::size_t>(2 * sms));
    std::uint64_t rng = 0x9E3779B97F4A7C15ull;
    for (std::size_t k = 0; k < ins.size(); ++k) {
        EngineInput& e = ins[k];
        e.N = kTunePackingN;
        e.ndim = ndim;
        e.positions.resize(kTunePackingN * ndim);
        for (double& v : e.positions) {  // xorshift uniforms in [0, 1)
            rng ^= rng << 13;
            rng ^= rng >> 7;
            rng ^= rng << 17;
            v = static_cast<double>(rng >> 11) * (1.0 / 9007199254740992.0);
        }
        e.diameters.assign(kTunePackingN, 1.0);
        e.max_steps = kTuneSteps;
        e.device = device;
        e.pair_precision = mixed ? 1 : 0;
    }
    BatchTuning t;
    for (int b = 1; b <= 2; ++b) {
        const auto t0 = std::chrono::steady_clock::now();
        const std::vector<BatchOutcome> r = run_batch_persistent(ins, 2048u, b);
        const double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        std::uint64_t steps = 0;
        for (const BatchOutcome& o : r) steps += o.code == 0 ? o.result.steps : 0;
        t.steps_per_s[b - 1] = s > 0.0 ? static_cast<double>(steps) / s : 0.0;
    }
    t.blocks_per_sm = t.steps_per_s[1] > t.steps_per_s[0] ? 2 : 1;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tuned[key] = t;
    return t;
}

std::vector<BatchOutcome> run_batch_persistent(const std::vector<EngineInput>& ins, std::uint32_t chunk,
                                               int blocks_per_sm) {
    std::vector<BatchOutcome> out(ins.size());
    if (ins.empty()) return out;
    std::vector<RunSetup> su(ins.size());
    std::vector<std::size_t> pending;
    for (std::size_t k = 0; k < ins.size(); ++k) {
        try {
            if (ins[k].exact || ins[k].has_target_phi)
                throw std::invalid_argument(
                    "rcpgenerator_b200: the batch engine runs the graph engine; exact runs and "
                    "target_phi runs are not batched");
            su[k] = prepare_run(ins[k]);
            pending.push_back(k);
        } catch (const std::invalid_argument& e) {
            out[k].code = -22;
            out[k].message = e.what();
        } catch (const std::exception& e) {
            out[k].code = -1;
            out[k].message = e.what();
        }
    }
    ck(cudaSetDevice(ins[0].device), "cudaSetDevice");
    cudaStream_t st = nullptr;
    ck(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "cudaStreamCreate");
    try {
        for (std::uint32_t mult = 1; !pending.empty(); mult *= 2) {
            std::vector<std::size_t> again;
            for (int nd = 2; nd <= kMaxDim; ++nd) {
                std::vector<std::size_t> grp;
                for (std::size_t k : pending)
                    if (su[k].ndim == nd) grp.push_back(k);
                if (grp.empty()) continue;
                const int bps = blocks_per_sm > 0 ? blocks_per_sm
                                                  : tune_batch(nd, ins[0].device, ins[0].pair_precision == 1).blocks_per_sm;
                const std::vector<std::uint32_t> st_k = run_group(ins, su, grp, mult, chunk, bps, st, out);
                for (std::size_t q = 0; q < grp.size(); ++q) {
                    const std::size_t k = grp[q];
                    if (st_k[q] == 2u) continue;
                    if (st_k[q] == 3u && mult < 64) {
                        again.push_back(k);
                    } else if (st_k[q] == 4u) {
                        out[k].code = -1;
                        out[k].message = "rcpgenerator: a particle exceeded its neighbor capacity during "
                                         "pair-list construction (kdtree own-write); pass a larger neighbor_max";
                    } else if (st_k[q] == 5u) {
                        out[k].code = -22;
                        out[k].message = "rcpgenerator_b200: target_phi runs are not batched";
                    } else {
                        out[k].code = -1;
                        out[k].message = "rcpgenerator_b200: neighbour rows outgrew the batch row capacity";
                    }
                }
            }
            pending.swap(again);
        }
    } catch (...) {
        cudaStreamDestroy(st);
        throw;
    }
    cudaStreamDestroy(st);
    return out;
}

}  // namespace rcpg
