// Device helpers shared by the kernels of one packing (rcpg_kernels.cu) and
// by the persistent batch kernel (rcpg_batch.cu): position records, cell
// coordinates and the fixed-order reductions of the force sums.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "rcpg_device.h"

namespace rcpg {
namespace {

// A half row over its reference capacity (the reference's overflow error,
// ENG:647-658); the lowest particle index is kept.
__device__ __forceinline__ void report_cap_error(DevCtl* ctl, std::uint32_t particle, std::uint32_t cap) {
    atomicMax(&ctl->cap_error_key, ~((static_cast<unsigned long long>(particle) << 32) | cap));
    ctl->cap_error = 1u;
}

// Points the per-particle arrays of `a` at the buffer set that holds the
// particle state now (cell-order storage, graph mode); no-op otherwise.
__device__ __forceinline__ void bind_buffers(DevArrays& a) {
    if (a.permute && a.ctl->buf) {
        a.pos = a.pos_alt;
        a.m = a.m_alt;
        a.v = a.v_alt;
        a.origin = a.origin_alt;
        a.caps = a.caps_alt;
        a.ref_rank = a.ref_rank_alt;
    }
}

template <int ND>
__device__ __forceinline__ void load_pos(const double* __restrict__ pos, std::uint64_t i,
                                         double* x, double& D0) {
    constexpr int P = pos_stride(ND);
    const double2* p2 = reinterpret_cast<const double2*>(pos + i * P);
#pragma unroll
    for (int h = 0; h < P / 2; ++h) {
        const double2 w = p2[h];
        if (2 * h < ND) x[2 * h] = w.x;
        else if (2 * h == ND) D0 = w.x;
        if (2 * h + 1 < ND) x[2 * h + 1] = w.y;
        else if (2 * h + 1 == ND) D0 = w.y;
    }
}

// load_pos from global memory: with ld256 (P == 4, 32-byte aligned records,
// data not written by the running kernel; the caller checks the alignment)
// the record is one 256-bit read-only load instead of two 128-bit loads.
template <int ND>
__device__ __forceinline__ void load_pos_g(const double* __restrict__ pos, std::uint64_t i, double* x,
                                           double& D0, int ld256) {
    if constexpr (pos_stride(ND) == 4) {
        if (ld256) {
            double w[4];
            asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];"
                : "=d"(w[0]), "=d"(w[1]), "=d"(w[2]), "=d"(w[3])
                : "l"(pos + i * 4));
#pragma unroll
            for (int d = 0; d < ND; ++d) x[d] = w[d];
            D0 = w[ND];
            return;
        }
    }
    load_pos<ND>(pos, i, x, D0);
}

template <int ND>
__device__ __forceinline__ void store_pos(double* __restrict__ pos, std::uint64_t i,
                                          const double* x, double D0) {
    constexpr int P = pos_stride(ND);
    double2* p2 = reinterpret_cast<double2*>(pos + i * P);
#pragma unroll
    for (int h = 0; h < P / 2; ++h) {
        double2 w;
        w.x = (2 * h < ND) ? x[2 * h] : ((2 * h == ND) ? D0 : 0.0);
        w.y = (2 * h + 1 < ND) ? x[2 * h + 1] : ((2 * h + 1 == ND) ? D0 : 0.0);
        p2[h] = w;
    }
}

// Cell coordinate of one axis; the grid cell is at least as wide as the
// largest pair cutoff, so partners sit in the 3^ndim neighbourhood.
__device__ __forceinline__ int cell_coord(double x, double scale, int nc) {
    double s = x * scale;
    if (!(s > 0.0)) return 0;  // negative, zero or NaN
    int c = static_cast<int>(s);
    return c >= nc ? nc - 1 : c;
}

// ---- deterministic reductions of ForceSums ---------------------------------
__device__ __forceinline__ double shfl_down_d(double v, int o) {
    return __shfl_down_sync(0xffffffffu, v, o);
}

__device__ __forceinline__ void warp_reduce_sums(ForceSums& s) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        s.pair_U = xadd(s.pair_U, shfl_down_d(s.pair_U, o));
        s.pair_Lc = xadd(s.pair_Lc, shfl_down_d(s.pair_Lc, o));
        s.pair_dk = xadd(s.pair_dk, shfl_down_d(s.pair_dk, o));
        s.pair_Fm = xadd(s.pair_Fm, shfl_down_d(s.pair_Fm, o));
        s.pair_maxov = fmax(s.pair_maxov, shfl_down_d(s.pair_maxov, o));
        s.wall_U = xadd(s.wall_U, shfl_down_d(s.wall_U, o));
        s.wall_dk = xadd(s.wall_dk, shfl_down_d(s.wall_dk, o));
        s.wall_Fm = xadd(s.wall_Fm, shfl_down_d(s.wall_Fm, o));
        s.sum_mag = xadd(s.sum_mag, shfl_down_d(s.sum_mag, o));
        s.sum_D = xadd(s.sum_D, shfl_down_d(s.sum_D, o));
        s.pair_count += __shfl_down_sync(0xffffffffu, s.pair_count, o);
        s.wall_count += __shfl_down_sync(0xffffffffu, s.wall_count, o);
        s.mag_count += __shfl_down_sync(0xffffffffu, s.mag_count, o);
    }
}

__device__ __forceinline__ void sums_add(ForceSums& a, const ForceSums& b) {
    a.pair_U = xadd(a.pair_U, b.pair_U);
    a.pair_Lc = xadd(a.pair_Lc, b.pair_Lc);
    a.pair_dk = xadd(a.pair_dk, b.pair_dk);
    a.pair_Fm = xadd(a.pair_Fm, b.pair_Fm);
    a.pair_maxov = fmax(a.pair_maxov, b.pair_maxov);
    a.wall_U = xadd(a.wall_U, b.wall_U);
    a.wall_dk = xadd(a.wall_dk, b.wall_dk);
    a.wall_Fm = xadd(a.wall_Fm, b.wall_Fm);
    a.sum_mag = xadd(a.sum_mag, b.sum_mag);
    a.sum_D = xadd(a.sum_D, b.sum_D);
    a.pair_count += b.pair_count;
    a.wall_count += b.wall_count;
    a.mag_count += b.mag_count;
}

// Deterministic block reduction (fixed shuffle tree, warps combined in order).
template <int NT>
__device__ __forceinline__ void block_reduce_sums(ForceSums& s, ForceSums* smem) {
    warp_reduce_sums(s);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) smem[warp] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        ForceSums t = smem[0];
#pragma unroll
        for (int w = 1; w < NT / 32; ++w) sums_add(t, smem[w]);
        s = t;
    }
}

// Exclusive scan of one value per thread over the block; total = block sum.
template <typename T>
__device__ __forceinline__ T block_exclusive_scan(T v, T* smem, T& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T s = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const T y = __shfl_up_sync(0xffffffffu, s, o);
        if (lane >= o) s += y;
    }
    if (lane == 31) smem[warp] = s;
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
        T w = lane < nw ? smem[lane] : T(0);
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const T y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < nw) smem[lane] = w;
    }
    __syncthreads();
    const T warp_off = warp ? smem[warp - 1] : T(0);
    total = smem[(blockDim.x >> 5) - 1];
    __syncthreads();
    return warp_off + s - v;
}

// Parameters of the kernels of the step that begin_step() just opened.
__device__ __forceinline__ void publish_step(DevCtl* ctl, const Controller& c, int ndim) {
    ctl->forces_done = 0u;
    for (int d = 0; d < ndim; ++d) {
        ctl->g.box[d] = c.box[d];
        ctl->g.inv_box[d] = 1.0 / c.box[d];
    }
    ctl->refresh_kappa = c.kappa_D;
    ctl->force_kappa = c.kappa_D;
    ctl->force_mu = c.mu_eff;
    ctl->build_kappa = c.kappa_D;
    ctl->build_t_shell = c.t_shell;
    ctl->build_Dmax = c.Dmax_cur;
    ctl->theta = c.theta;
    if (c.rebuild_mode == REBUILD_FULL) {
        ctl->rebuild_flag = 1u;
    } else {
        ctl->rebuild_flag = 0u;
        ctl->kappa_min = fmin(ctl->kappa_min, c.kappa_D);
    }
}

}  // namespace
}  // namespace rcpg
