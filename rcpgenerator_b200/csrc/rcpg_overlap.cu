// Overlap report of a packed state on the GPU: the pair-overlap diagnostic of
// the reference's analysis package (rcptools/overlap.py:7-113) -- candidate
// pairs i < j within 2 * R_max (its KD-tree query radius, overlap.py:53),
// minimum image by round-half-even of pos[i] - pos[j] over every axis when a
// box is given (overlap.py:63-65), overlap (r_i + r_j) - |d| > 0, fractions
// in the "sum" and "min" conventions (overlap.py:71-75).
//
// Cells at least 2 R_max wide (one grid, binned on the host), one thread per
// particle over the distinct neighbour cells (1, 2 or 3 per axis), two
// passes: counts, then the pairs of each particle at its offset, sorted by j.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/rcpg.h"
#include "rcpg_core.h"
#include "rcpg_engine.h"

namespace {

using rcpg::xadd;
using rcpg::xmul;
using rcpg::xsub;

constexpr int kOvMaxDim = 8;

struct OvGrid {
    int ndim;
    int periodic;
    int ncell[kOvMaxDim];
    double lo[kOvMaxDim], width[kOvMaxDim], box[kOvMaxDim];
    double rq;  // candidate radius 2 R_max
};

// |pos[i] - pos[j]| with the image removed, in the operation order of the
// reference's NumPy expression (no fused multiply-adds)
__device__ __forceinline__ double pair_dist(const double* __restrict__ x, std::uint64_t i, std::uint64_t j,
                                            const OvGrid& g) {
    double s = 0.0;
    for (int d = 0; d < g.ndim; ++d) {
        double dd = xsub(x[i * g.ndim + d], x[j * g.ndim + d]);
        if (g.periodic) dd = xsub(dd, xmul(nearbyint(dd / g.box[d]), g.box[d]));
        s = xadd(s, xmul(dd, dd));
    }
    return sqrt(s);
}

// PASS 0: counts (candidates, overlaps); PASS 1: writes the overlaps of i at off[i]
template <int PASS>
__global__ void __launch_bounds__(128) k_overlap(const double* __restrict__ x, const double* __restrict__ D,
                                                 std::uint64_t N, OvGrid g, const std::uint32_t* __restrict__ cell_of,
                                                 const std::uint32_t* __restrict__ cell_start,
                                                 const std::uint32_t* __restrict__ cell_list,
                                                 unsigned long long* __restrict__ ncand,
                                                 std::uint32_t* __restrict__ nov,
                                                 const unsigned long long* __restrict__ off,
                                                 std::uint32_t* __restrict__ pairs, double* __restrict__ fsum,
                                                 double* __restrict__ fmin_, unsigned long long capacity) {
    const std::uint64_t i = blockIdx.x * 128ull + threadIdx.x;
    if (i >= N) return;
    int ci[kOvMaxDim], span[kOvMaxDim], first[kOvMaxDim], odo[kOvMaxDim];
    {
        std::uint32_t c = cell_of[i];
        for (int d = 0; d < g.ndim; ++d) {
            ci[d] = static_cast<int>(c % static_cast<std::uint32_t>(g.ncell[d]));
            c /= static_cast<std::uint32_t>(g.ncell[d]);
            const int n = g.ncell[d];
            if (g.periodic) {
                span[d] = n >= 3 ? 3 : n;
                first[d] = n >= 3 ? -1 : 0;
            } else {
                first[d] = ci[d] > 0 ? -1 : 0;
                span[d] = (ci[d] < n - 1 ? 1 : 0) - first[d] + 1;
            }
            odo[d] = 0;
        }
    }
    const double Ri = D[i] / 2.0;
    unsigned long long cand = 0;
    std::uint32_t cnt = 0;
    const unsigned long long base = PASS ? off[i] : 0ull;
    while (true) {
        std::uint32_t cn = 0, mul = 1;
        for (int d = 0; d < g.ndim; ++d) {
            int cc = ci[d] + first[d] + odo[d];
            if (cc < 0) cc += g.ncell[d];
            else if (cc >= g.ncell[d]) cc -= g.ncell[d];
            cn += static_cast<std::uint32_t>(cc) * mul;
            mul *= static_cast<std::uint32_t>(g.ncell[d]);
        }
        for (std::uint32_t p = cell_start[cn]; p < cell_start[cn + 1]; ++p) {
            const std::uint32_t j = cell_list[p];
            if (j <= i) continue;
            const double dist = pair_dist(x, i, j, g);
            if (!(dist <= g.rq)) continue;
            ++cand;
            const double Rj = D[j] / 2.0;
            const double rsum = xadd(Ri, Rj);
            const double ov = xsub(rsum, dist);
            if (!(ov > 0.0)) continue;
            if (PASS) {
                const unsigned long long q = base + cnt;
                if (q < capacity) {
                    // insertion by j: the pairs of i end sorted
                    unsigned long long p2 = q;
                    while (p2 > base && pairs[2 * (p2 - 1) + 1] > j) {
                        pairs[2 * p2] = pairs[2 * (p2 - 1)];
                        pairs[2 * p2 + 1] = pairs[2 * (p2 - 1) + 1];
                        fsum[p2] = fsum[p2 - 1];
                        fmin_[p2] = fmin_[p2 - 1];
                        --p2;
                    }
                    pairs[2 * p2] = static_cast<std::uint32_t>(i);
                    pairs[2 * p2 + 1] = j;
                    fsum[p2] = ov / rsum;
                    fmin_[p2] = ov / fmin(Ri, Rj);
                }
            }
            ++cnt;
        }
        int d = 0;
        for (; d < g.ndim; ++d) {
            if (++odo[d] < span[d]) break;
            odo[d] = 0;
        }
        if (d == g.ndim) break;
    }
    if (!PASS) {
        ncand[i] = cand;
        nov[i] = cnt;
    }
}

int32_t fail(char* err, std::size_t errlen, int32_t code, const std::string& msg) {
    if (err && errlen) std::snprintf(err, errlen, "%s", msg.c_str());
    return code;
}

struct DevBuf {
    std::vector<void*> ptrs;
    cudaStream_t st;
    explicit DevBuf(cudaStream_t s) : st(s) {}
    template <typename T>
    T* get(std::size_t n) {
        void* p = nullptr;
        if (rcpg::pool_alloc_async(&p, n * sizeof(T) + 16, st) != cudaSuccess)
            throw std::runtime_error("rcpgenerator_b200: device allocation failed");
        ptrs.push_back(p);
        return static_cast<T*>(p);
    }
    ~DevBuf() {
        for (void* p : ptrs) cudaFreeAsync(p, st);
        cudaStreamSynchronize(st);
    }
};

}  // namespace

extern "C" int32_t rcpg_overlap_report(uint64_t N, int32_t ndim, const double* positions, const double* diameters,
                                       const double* box, uint64_t* n_candidate_out, uint64_t* n_overlap_out,
                                       uint64_t capacity, uint32_t* pairs_out, double* frac_sum_out,
                                       double* frac_min_out, int32_t device, char* err, size_t errlen) {
    if (n_candidate_out) *n_candidate_out = 0;
    if (n_overlap_out) *n_overlap_out = 0;
    if (ndim < 1 || ndim > kOvMaxDim || (N && (!positions || !diameters)) ||
        (capacity && (!pairs_out || !frac_sum_out || !frac_min_out)))
        return fail(err, errlen, RCPG_EINVAL, "rcpgenerator_b200: bad arguments to rcpg_overlap_report");
    if (N < 2) return RCPG_OK;
    if (N >= 0xFFFFFFF0ull) return fail(err, errlen, RCPG_EINVAL, "rcpgenerator_b200: N too large");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        cudaGetLastError();
        return fail(err, errlen, RCPG_ECUDA, "rcpgenerator_b200: no CUDA device available (this engine has no CPU path)");
    }
    try {
        if (cudaSetDevice(device) != cudaSuccess) throw std::runtime_error("cudaSetDevice failed");
        // grid: cells at least 2 R_max wide, at most about 2N + 64 cells
        OvGrid g{};
        g.ndim = ndim;
        g.periodic = box ? 1 : 0;
        double dmax = 0.0;
        for (uint64_t i = 0; i < N; ++i) dmax = std::max(dmax, diameters[i]);
        const double rq = 2.0 * (dmax / 2.0);
        g.rq = rq;
        const double cell_min = rq * (1.0 + 1e-6);  // binning slack: a pair within rq never skips a cell
        double cells = 1.0;
        for (int d = 0; d < ndim; ++d) {
            double lo, hi;
            if (box) {
                lo = 0.0;
                hi = box[d];
            } else {
                lo = hi = positions[d];
                for (uint64_t i = 1; i < N; ++i) {
                    lo = std::min(lo, positions[i * ndim + d]);
                    hi = std::max(hi, positions[i * ndim + d]);
                }
                hi = std::max(hi, lo + 1e-300);
            }
            const double L = hi - lo;
            double n = rq > 0.0 ? std::floor(L / cell_min) : 1.0;
            if (!(n >= 1.0)) n = 1.0;
            if (n > 1048576.0) n = 1048576.0;
            g.lo[d] = lo;
            g.box[d] = box ? box[d] : L;
            g.ncell[d] = static_cast<int>(n);
            cells *= n;
        }
        const double cap_cells = 2.0 * static_cast<double>(N) + 64.0;
        while (cells > cap_cells) {
            int dm = 0;
            for (int d = 1; d < ndim; ++d)
                if (g.ncell[d] > g.ncell[dm]) dm = d;
            const int nn = std::max(1, (g.ncell[dm] * 3) / 4);
            cells = cells / g.ncell[dm] * nn;
            g.ncell[dm] = nn;
        }
        for (int d = 0; d < ndim; ++d) g.width[d] = (box ? box[d] : (g.box[d])) / g.ncell[d];
        // host binning (counting sort by cell, ascending particle order in a cell)
        const std::uint64_t C = static_cast<std::uint64_t>(cells);
        std::vector<std::uint32_t> cell_of(N), start(C + 1, 0u), list(N);
        for (uint64_t i = 0; i < N; ++i) {
            std::uint32_t c = 0, mul = 1;
            for (int d = 0; d < ndim; ++d) {
                double v = positions[i * ndim + d] - g.lo[d];
                if (box) v -= std::floor(v / box[d]) * box[d];
                // cell index, clamped (a NaN from a zero box side goes to cell 0)
                const double q = std::floor(v / g.width[d]);
                long long k = 0;
                if (q >= static_cast<double>(g.ncell[d] - 1)) k = g.ncell[d] - 1;
                else if (q > 0.0) k = static_cast<long long>(q);
                c += static_cast<std::uint32_t>(k) * mul;
                mul *= static_cast<std::uint32_t>(g.ncell[d]);
            }
            cell_of[i] = c;
            ++start[c + 1];
        }
        for (std::uint64_t c = 0; c < C; ++c) start[c + 1] += start[c];
        {
            std::vector<std::uint32_t> fill(start.begin(), start.end() - 1);
            for (uint64_t i = 0; i < N; ++i) list[fill[cell_of[i]]++] = static_cast<std::uint32_t>(i);
        }
        cudaStream_t st = nullptr;
        if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess)
            throw std::runtime_error("cudaStreamCreate failed");
        std::uint64_t total_ov = 0, total_cand = 0;
        {
            DevBuf B(st);
            double* dx = B.get<double>(N * ndim);
            double* dD = B.get<double>(N);
            std::uint32_t* dcell = B.get<std::uint32_t>(N);
            std::uint32_t* dstart = B.get<std::uint32_t>(C + 1);
            std::uint32_t* dlist = B.get<std::uint32_t>(N);
            unsigned long long* dcand = B.get<unsigned long long>(N);
            std::uint32_t* dnov = B.get<std::uint32_t>(N);
            unsigned long long* doff = B.get<unsigned long long>(N);
            auto ok = [&](cudaError_t e, const char* what) {
                if (e != cudaSuccess)
                    throw std::runtime_error(std::string("rcpgenerator_b200: CUDA error in ") + what + ": " +
                                             cudaGetErrorString(e));
            };
            ok(cudaMemcpyAsync(dx, positions, N * ndim * 8, cudaMemcpyHostToDevice, st), "H2D");
            ok(cudaMemcpyAsync(dD, diameters, N * 8, cudaMemcpyHostToDevice, st), "H2D");
            ok(cudaMemcpyAsync(dcell, cell_of.data(), N * 4, cudaMemcpyHostToDevice, st), "H2D");
            ok(cudaMemcpyAsync(dstart, start.data(), (C + 1) * 4, cudaMemcpyHostToDevice, st), "H2D");
            ok(cudaMemcpyAsync(dlist, list.data(), N * 4, cudaMemcpyHostToDevice, st), "H2D");
            const unsigned blocks = static_cast<unsigned>((N + 127) / 128);
            k_overlap<0><<<blocks, 128, 0, st>>>(dx, dD, N, g, dcell, dstart, dlist, dcand, dnov, nullptr, nullptr,
                                                 nullptr, nullptr, 0ull);
            ok(cudaGetLastError(), "k_overlap count");
            std::vector<unsigned long long> cand(N);
            std::vector<std::uint32_t> nov(N);
            ok(cudaMemcpyAsync(cand.data(), dcand, N * 8, cudaMemcpyDeviceToHost, st), "D2H");
            ok(cudaMemcpyAsync(nov.data(), dnov, N * 4, cudaMemcpyDeviceToHost, st), "D2H");
            ok(cudaStreamSynchronize(st), "sync");
            std::vector<unsigned long long> off(N);
            for (uint64_t i = 0; i < N; ++i) {
                off[i] = total_ov;
                total_ov += nov[i];
                total_cand += cand[i];
            }
            const std::uint64_t m = std::min<std::uint64_t>(total_ov, capacity);
            if (m > 0) {
                std::uint32_t* dpairs = B.get<std::uint32_t>(2 * m);
                double* dfs = B.get<double>(m);
                double* dfm = B.get<double>(m);
                ok(cudaMemcpyAsync(doff, off.data(), N * 8, cudaMemcpyHostToDevice, st), "H2D");
                k_overlap<1><<<blocks, 128, 0, st>>>(dx, dD, N, g, dcell, dstart, dlist, nullptr, nullptr, doff, dpairs,
                                                     dfs, dfm, static_cast<unsigned long long>(m));
                ok(cudaGetLastError(), "k_overlap write");
                ok(cudaMemcpyAsync(pairs_out, dpairs, 2 * m * 4, cudaMemcpyDeviceToHost, st), "D2H");
                ok(cudaMemcpyAsync(frac_sum_out, dfs, m * 8, cudaMemcpyDeviceToHost, st), "D2H");
                ok(cudaMemcpyAsync(frac_min_out, dfm, m * 8, cudaMemcpyDeviceToHost, st), "D2H");
                ok(cudaStreamSynchronize(st), "sync");
            }
        }
        cudaStreamDestroy(st);
        if (n_candidate_out) *n_candidate_out = total_cand;
        if (n_overlap_out) *n_overlap_out = total_ov;
        if (total_ov > capacity)
            return fail(err, errlen, RCPG_ENOSPC, "rcpgenerator_b200: more overlapping pairs than the output capacity");
        return RCPG_OK;
    } catch (const std::exception& e) {
        return fail(err, errlen, RCPG_ECUDA, e.what());
    }
}
