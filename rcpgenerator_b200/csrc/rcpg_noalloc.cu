// rcpg_pairs_full_noalloc: the full-refresh neighbour-row build of
// rcpg_pairs_full without any device allocation.
//
// Who needs it: callers that must not allocate device memory while they run.
// Typical cases are applications whose device memory is reserved up front by
// their own allocator, so an extra cudaMalloc fails or fragments the pool, and
// time-critical loops, where cudaMalloc / cudaFree would synchronise the
// device and stall the other streams. rcpg_pairs_full needs ten scratch arrays
// per call (packed positions, cell grid, cell lists, rows in cell order); here
// they are carved out of one fixed array in the library's static device memory.
//
// The scratch array is kNoAllocScratchBytes (8 MiB) of __device__ memory that
// every GPU which loads this library keeps until the process exits. A call
// whose working set does not fit is rejected with RCPG_ENOSPC before anything
// runs. All calls share the array and it keeps the previous call's contents:
// the cell counters are cleared inside the build, and the control block is
// rewritten before every call. Calls whose GPU work overlaps in time (other
// streams, other host threads) race on the array and must be serialised by the
// caller.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include <stdexcept>

#include "../../include/rcpg.h"
#include "rcpg_device.h"
#include "rcpg_noalloc_plan.h"

namespace {

using rcpg::kNoAllocScratchBytes;
constexpr int kMaxDevices = 64;

// The scratch array. Host code must not use its name as a pointer: on the
// host it is a stand-in symbol, not a device address; the device address
// comes from cudaGetSymbolAddress below.
__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_addr_mutex;
void* g_addr[kMaxDevices] = {};

// Device max of D[0..N) into ctl->build_Dmax (the cutoff of the cell grid).
__global__ void k_noalloc_dmax(std::uint64_t N, const double* __restrict__ D, rcpg::DevCtl* ctl) {
    __shared__ double red[1024 / 32];
    double m = 0.0;
    for (std::uint64_t k = threadIdx.x; k < N; k += blockDim.x) m = fmax(m, D[k]);
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < static_cast<int>(blockDim.x >> 5); ++w) m = fmax(m, red[w]);
        ctl->build_Dmax = fmax(m, red[0]);
    }
}

void set_err(char* err, std::size_t errlen, const std::string& msg) {
    if (err && errlen) std::snprintf(err, errlen, "%s", msg.c_str());
}

// Device address of the scratch array on the current device, looked up once
// per device (with that device current) and cached.
int32_t scratch_address(void** out, char* err, std::size_t errlen) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        cudaGetLastError();
        set_err(err, errlen, "rcpgenerator_b200: no current CUDA device");
        return RCPG_ECUDA;
    }
    std::lock_guard<std::mutex> lock(g_addr_mutex);
    if (!g_addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            set_err(err, errlen, std::string("rcpgenerator_b200: cudaGetSymbolAddress failed: ") +
                                     cudaGetErrorString(e));
            return RCPG_ECUDA;
        }
        g_addr[dev] = p;
    }
    *out = g_addr[dev];
    return RCPG_OK;
}

}  // namespace

extern "C" int32_t rcpg_pairs_full_noalloc(uint64_t N, int32_t ndim, const double* x_dev,
                                           const double* D_dev, const double* box,
                                           const int8_t* walls, double t_shell,
                                           uint32_t row_capacity, uint32_t* nbr_dev,
                                           uint32_t* cnt_dev, uint32_t* row_need_out,
                                           void* stream, char* err, size_t errlen) {
    if (N == 0 || ndim < 2 || ndim > rcpg::kMaxDim || !x_dev || !D_dev || !nbr_dev || !cnt_dev ||
        row_capacity == 0) {
        set_err(err, errlen, "rcpgenerator_b200: bad arguments to rcpg_pairs_full_noalloc");
        return RCPG_EINVAL;
    }
    void* base = nullptr;
    const int32_t rc = scratch_address(&base, err, errlen);
    if (rc != RCPG_OK) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const rcpg::NoAllocPlan plan = rcpg::plan_noalloc(N, ndim, row_capacity, sizeof(rcpg::DevCtl));
    if (!plan.ok) {
        set_err(err, errlen,
                "rcpgenerator_b200: rcpg_pairs_full_noalloc needs more than its fixed 8 MiB "
                "device scratch for this N / ndim / row_capacity (use rcpg_pairs_full)");
        return RCPG_ENOSPC;
    }
    unsigned char* b = static_cast<unsigned char*>(base);
    rcpg::DevArrays a{};
    a.N = N;
    a.ndim = ndim;
    a.P = rcpg::pos_stride(ndim);
    a.ctl = reinterpret_cast<rcpg::DevCtl*>(b + plan.ctl);
    a.pos = reinterpret_cast<double*>(b + plan.pos);
    a.spos = reinterpret_cast<double*>(b + plan.spos);
    a.x_last = reinterpret_cast<double*>(b + plan.x_last);
    a.caps = reinterpret_cast<std::uint32_t*>(b + plan.caps);
    a.cell_of = reinterpret_cast<std::uint32_t*>(b + plan.cell_of);
    a.cell_rank = reinterpret_cast<std::uint32_t*>(b + plan.cell_rank);
    a.cell_list = reinterpret_cast<std::uint32_t*>(b + plan.cell_list);
    a.work = reinterpret_cast<std::uint32_t*>(b + plan.work);
    a.nbr_cnt = reinterpret_cast<std::uint32_t*>(b + plan.nbr_cnt);
    a.nbr = reinterpret_cast<std::uint32_t*>(b + plan.nbr);
    a.scan_tmp = reinterpret_cast<std::uint32_t*>(b + plan.scan_tmp);
    a.S = row_capacity;
    a.sorted_rows = 1;  // the reference's row order
    // the rest of the array holds the cell grid; the build coarsens its grid
    // to these many cells
    a.C_alloc = plan.cell_capacity;
    a.cell_count = reinterpret_cast<std::uint32_t*>(b + plan.cell_count);
    a.cell_start = reinterpret_cast<std::uint32_t*>(b + plan.cell_start);
    rcpg::DevCtl h;
    std::memset(&h, 0, sizeof(h));
    rcpg::Geometry& g = h.g;
    g.ndim = ndim;
    g.circle_k = (walls && walls[0] < 0) ? -walls[0] : 0;
    for (int d = 0; d < ndim; ++d) {
        g.walls[d] = walls ? walls[d] : 0;
        if (g.walls[d] == 1) g.any_flat_wall = 1;
        g.box[d] = box ? box[d] : 1.0;
        g.inv_box[d] = 1.0 / g.box[d];
    }
    h.build_kappa = 1.0;
    h.build_t_shell = t_shell;
    h.rebuild_flag = 1u;
    cudaError_t e = cudaMemcpyAsync(a.ctl, &h, sizeof(h), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(a.caps, 0xFF, N * 4, st);
    if (e != cudaSuccess) {
        cudaGetLastError();
        set_err(err, errlen, std::string("rcpgenerator_b200: ") + cudaGetErrorString(e));
        return RCPG_ECUDA;
    }
    try {
        k_noalloc_dmax<<<1, 1024, 0, st>>>(N, D_dev, a.ctl);
        rcpg::launch_pack(N, ndim, x_dev, D_dev, a.pos, st);
        rcpg::launch_rebuild(a, st);
        rcpg::launch_rows_to_particle_order(N, a.work, a.nbr, a.nbr_cnt, nbr_dev, cnt_dev, st);
    } catch (const std::length_error& ex) {
        set_err(err, errlen, std::string("rcpgenerator_b200: ") + ex.what());
        return RCPG_ENOSPC;
    } catch (const std::invalid_argument& ex) {
        set_err(err, errlen, std::string("rcpgenerator_b200: ") + ex.what());
        return RCPG_EINVAL;
    } catch (const std::exception& ex) {
        set_err(err, errlen, std::string("rcpgenerator_b200: ") + ex.what());
        return RCPG_ERUNTIME;
    }
    std::uint32_t need = 0;
    e = cudaMemcpyAsync(&need, &a.ctl->row_need, sizeof(need), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_err(err, errlen, std::string("rcpgenerator_b200: ") + cudaGetErrorString(e));
        return RCPG_ECUDA;
    }
    if (row_need_out) *row_need_out = need;
    if (need > row_capacity) {
        set_err(err, errlen, "rcpgenerator_b200: a neighbour row exceeds row_capacity");
        return RCPG_ENOSPC;
    }
    return RCPG_OK;
}
