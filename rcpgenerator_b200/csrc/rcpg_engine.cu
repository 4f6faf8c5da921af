// Host driver of one packing: the setup of run_packing_observed
// (python_code/python/src/core/rcp_generator.cpp, "ENG", :4353-5013), then the
// step loop in one of two modes:
//   graph mode  -- the controller runs on the GPU (k_controller) and whole
//                  steps are replayed from a captured CUDA graph; the host
//                  only intervenes every few dozen steps, at reorders and at
//                  the end.
//   exact mode  -- the controller runs on the host with the host libm and
//                  every force evaluation is reduced in the reference's
//                  one-thread order, so a run reproduces the reference engine
//                  at one OpenMP thread step for step.
#include "rcpg_engine.h"
#include "rcpg_setup.h"

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstring>
#include <mutex>
#include <numeric>

namespace rcpg {

// Device memory of an engine comes from this library's stream-ordered pool of
// the device (cudaMallocFromPoolAsync / cudaFreeAsync on the engine's stream),
// so creating and destroying engines never synchronises the device: engines
// on other streams (a batch) keep running. The pool keeps up to kPoolKeep
// bytes of freed memory reserved for the next engine (the default pool hands
// it back to the driver at every synchronisation, and the next engine pays a
// driver allocation again). The pinned control block used to read the device
// controller is recycled through a process-wide free list for the same reason.
namespace {
std::mutex g_pinned_mu;
std::vector<DevCtl*> g_pinned_free;
std::mutex g_pool_mu;
std::vector<cudaMemPool_t> g_pools;  // by device ordinal, created on first use
constexpr std::uint64_t kPoolKeep = std::uint64_t{16} << 30;
}  // namespace

cudaError_t pool_alloc_async(void** p, std::size_t bytes, cudaStream_t st) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    cudaMemPool_t pool = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_pool_mu);
        if (static_cast<int>(g_pools.size()) <= dev) g_pools.resize(dev + 1, nullptr);
        if (!g_pools[dev]) {
            cudaMemPoolProps props;
            std::memset(&props, 0, sizeof(props));
            props.allocType = cudaMemAllocationTypePinned;
            props.handleTypes = cudaMemHandleTypeNone;
            props.location.type = cudaMemLocationTypeDevice;
            props.location.id = dev;
            e = cudaMemPoolCreate(&g_pools[dev], &props);
            if (e != cudaSuccess) {
                g_pools[dev] = nullptr;
                return e;
            }
            std::uint64_t keep = kPoolKeep;
            e = cudaMemPoolSetAttribute(g_pools[dev], cudaMemPoolAttrReleaseThreshold, &keep);
            if (e != cudaSuccess) return e;
        }
        pool = g_pools[dev];
    }
    return cudaMallocFromPoolAsync(p, bytes < 16 ? 16 : bytes, pool, st);
}

DevCtl* pinned_ctl_acquire() {
    {
        std::lock_guard<std::mutex> lk(g_pinned_mu);
        if (!g_pinned_free.empty()) {
            DevCtl* p = g_pinned_free.back();
            g_pinned_free.pop_back();
            return p;
        }
    }
    void* p = nullptr;
    if (cudaMallocHost(&p, sizeof(DevCtl)) != cudaSuccess) {
        cudaGetLastError();
        throw EngineError(-2, "rcpgenerator_b200: cudaMallocHost of the control block failed");
    }
    return static_cast<DevCtl*>(p);
}

void pinned_ctl_release(DevCtl* p) {
    std::lock_guard<std::mutex> lk(g_pinned_mu);
    g_pinned_free.push_back(p);
}

// Size classes of the cell grids for a wide size distribution: class k holds
// D0 in [D0min*2^k, D0min*2^(k+1)) (the last class is unbounded); each class's
// grid is as wide as the cutoff of its largest member, so a small particle
// does not scan cells sized for the largest one. One class when
// D0max/D0min <= kClassRatio.
void set_size_classes(const std::vector<double>& D0, DevCtl& h) {
    constexpr double kClassRatio = 2.5;
    double lo = D0.empty() ? 1.0 : D0[0], hi = lo;
    for (double v : D0) {
        lo = std::min(lo, v);
        hi = std::max(hi, v);
    }
    int K = 1;
    if (lo > 0.0 && hi / lo > kClassRatio) K = std::min(kMaxClass, static_cast<int>(std::ceil(std::log2(hi / lo))));
    h.nclass = K;
    for (int k = 0; k <= K; ++k) h.class_d0[k] = (k == 0) ? 0.0 : (k == K ? HUGE_VAL : lo * std::ldexp(1.0, k));
    for (int k = 0; k < K; ++k) h.class_d0max[k] = 0.0;
    for (double v : D0) {
        int k = 0;
        while (k + 1 < K && v >= h.class_d0[k + 1]) ++k;
        h.class_d0max[k] = std::max(h.class_d0max[k], v);
    }
    for (int k = 0; k < K; ++k)
        if (h.class_d0max[k] <= 0.0) h.class_d0max[k] = k + 1 < K ? h.class_d0[k + 1] : hi;
}

void Engine::check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        throw EngineError(-2, std::string("rcpgenerator_b200: CUDA error in ") + what + ": " +
                                  cudaGetErrorString(e));
    }
}

// ---------------------------------------------------------------------------
// setup (ENG:4353-4990), shared with the host emulation (rcpg_setup.cpp)
// ---------------------------------------------------------------------------
void Engine::setup_host(const EngineInput& in) {
    // the target-phi lock rescales every diameter on the host, so runs that
    // can lock are host-controlled
    exact_ = in.exact || in.has_target_phi;
    mixed_ = !exact_ && in.pair_precision == 1;
    mixed_switch_ = in.mixed_switch;
    graph_steps_ = in.graph_steps > 0 ? in.graph_steps : 32;
    device_ = in.device;
    RunSetup s = prepare_run(in);
    N_ = s.N;
    ndim_ = s.ndim;
    host_c_ = s.c;
    x0_ = std::move(s.x);
    D0_ = std::move(s.D0);
    caps_ = std::move(s.caps);
    walls_ = std::move(s.walls);
    neighbor_max_ = s.neighbor_max;
    hist_size_ = host_c_.step_cap + 1;
}

void Engine::alloc_device() {
    check(cudaSetDevice(device_), "cudaSetDevice");
    const std::uint64_t N = N_;
    const int nd = ndim_;
    P_ = pos_stride(nd);
    auto dalloc = [&](std::size_t bytes) -> void* {
        void* p = nullptr;
        check(pool_alloc_async(&p, bytes, st_), "cudaMallocFromPoolAsync");
        allocs_.push_back(p);
        return p;
    };
    a_.N = N;
    a_.ndim = nd;
    a_.P = P_;
    // graph mode stores the particles in cell order (every build permutes them
    // into the second buffer set); exact mode keeps the reference's order
    a_.permute = exact_ ? 0 : 1;
    a_.pos = static_cast<double*>(dalloc(N * P_ * sizeof(double)));
    a_.F = static_cast<double*>(dalloc(N * nd * sizeof(double)));
    a_.m = static_cast<double*>(dalloc(N * nd * sizeof(double)));
    a_.v = static_cast<double*>(dalloc(N * nd * sizeof(double)));
    a_.vec_tmp = static_cast<double*>(dalloc(N * nd * sizeof(double)));
    a_.x_last = static_cast<double*>(dalloc(N * nd * sizeof(double)));
    a_.nbr_cnt = static_cast<std::uint32_t*>(dalloc(N * 4));
    a_.caps = static_cast<std::uint32_t*>(dalloc(N * 4));
    a_.origin = static_cast<std::uint64_t*>(dalloc(N * 8));
    if (a_.permute) {
        a_.pos_alt = static_cast<double*>(dalloc(N * P_ * sizeof(double)));
        a_.m_alt = static_cast<double*>(dalloc(N * nd * sizeof(double)));
        a_.v_alt = static_cast<double*>(dalloc(N * nd * sizeof(double)));
        a_.origin_alt = static_cast<std::uint64_t*>(dalloc(N * 8));
        a_.caps_alt = static_cast<std::uint32_t*>(dalloc(N * 4));
        a_.ref_rank = static_cast<std::uint32_t*>(dalloc(N * 4));
        a_.ref_rank_alt = static_cast<std::uint32_t*>(dalloc(N * 4));
    } else {
        // the reorder's gather targets and the sorted position copy of the build
        a_.pos_tmp = static_cast<double*>(dalloc(N * P_ * sizeof(double)));
        a_.spos = a_.pos_tmp;  // the reorder uses it only before a build
        a_.u64_tmp = static_cast<std::uint64_t*>(dalloc(N * 8));
    }
    a_.cell_of = static_cast<std::uint32_t*>(dalloc(N * 4));
    a_.cell_rank = static_cast<std::uint32_t*>(dalloc(N * 4));
    a_.cell_list = static_cast<std::uint32_t*>(dalloc(N * 4));
    a_.work = static_cast<std::uint32_t*>(dalloc(N * 4));  // row slot -> particle, written by each build
    // exact mode sums each row in ascending partner order, as the reference
    a_.sorted_rows = exact_ ? 1 : 0;
    a_.mixed = mixed_ ? 1 : 0;
    // cell grid capacity: the grids at the initial (smallest) cutoffs
    {
        DevCtl cls{};
        set_size_classes(D0_, cls);
        double cells = 0.0;
        for (int k = 0; k < cls.nclass; ++k) {
            const double dmax = cls.nclass > 1 ? cls.class_d0max[k] : host_c_.Dmax_cur;
            const double cutoff = (dmax + host_c_.t_shell) * (1.0 + 1e-6);
            double ck = 1.0;
            for (int d = 0; d < nd; ++d) ck *= std::max(1.0, std::floor(host_c_.box[d] / cutoff));
            cells += ck;
        }
        double cap = std::min(cells * 1.5 + 64.0, 8.0 * static_cast<double>(N) + 1024.0);
        cap = std::min(cap, 2.0e9);
        a_.C_alloc = static_cast<std::uint32_t>(cap);
    }
    a_.cell_count = static_cast<std::uint32_t*>(dalloc((a_.C_alloc + 1ull) * 4));
    a_.cell_start = static_cast<std::uint32_t*>(dalloc((a_.C_alloc + 1ull) * 4));
    a_.scan_tmp = static_cast<std::uint32_t*>(dalloc(2 * 4096 * 4 + 64));
    // per-block partial sums: one per force block, or one per block of the
    // persistent tiled build when it computes the forces
    a_.block_sums = static_cast<ForceSums*>(dalloc(std::max<std::size_t>(force_blocks(N), 4096) * sizeof(ForceSums)));
    a_.pterm_cnt = static_cast<std::uint32_t*>(dalloc(N * 4));
    for (int b = 0; b < 2; ++b) {
        a_.sort_keys[b] = static_cast<std::uint64_t*>(dalloc(N * 8));
        a_.sort_vals[b] = static_cast<std::uint32_t*>(dalloc(N * 4));
    }
    const std::uint64_t tiles = (N + 4095) / 4096;
    a_.sort_hist = static_cast<std::uint32_t*>(dalloc(256 * tiles * 4 + 64));
    a_.ctl = static_cast<DevCtl*>(dalloc(sizeof(DevCtl)));
    // row capacity: grown on demand when a build reports a longer row
    a_.S = 0;
    a_.nbr = nullptr;
    a_.pterm = nullptr;
    ensure_row_capacity(nd == 2 ? 24u : (nd == 3 ? 48u : 96u));
    histories_on_device_ = !exact_;
    if (histories_on_device_) {
        const std::size_t hs = hist_size_;
        a_.hist.phi = static_cast<double*>(dalloc(hs * 8));
        a_.hist.force = static_cast<double*>(dalloc(hs * 8));
        a_.hist.energy = static_cast<double*>(dalloc(hs * 8));
        a_.hist.max_overlap = static_cast<double*>(dalloc(hs * 8));
        a_.hist.mu = static_cast<double*>(dalloc(hs * 8));
        a_.hist.alpha = static_cast<double*>(dalloc(hs * 8));
        a_.hist.mu_flag = static_cast<std::int8_t*>(dalloc(hs));
        check(cudaMemsetAsync(a_.hist.phi, 0, hs * 8, st_), "memset");
        check(cudaMemsetAsync(a_.hist.force, 0, hs * 8, st_), "memset");
        check(cudaMemsetAsync(a_.hist.energy, 0, hs * 8, st_), "memset");
        check(cudaMemsetAsync(a_.hist.max_overlap, 0, hs * 8, st_), "memset");
        check(cudaMemsetAsync(a_.hist.mu, 0, hs * 8, st_), "memset");
        check(cudaMemsetAsync(a_.hist.alpha, 0, hs * 8, st_), "memset");
        check(cudaMemsetAsync(a_.hist.mu_flag, 0, hs, st_), "memset");
    } else {
        h_phi_.assign(hist_size_, 0.0);
        h_force_.assign(hist_size_, 0.0);
        h_energy_.assign(hist_size_, 0.0);
        h_maxov_.assign(hist_size_, 0.0);
        h_mu_.assign(hist_size_, 0.0);
        h_alpha_.assign(hist_size_, 0.0);
        h_muflag_.assign(hist_size_, 0);
        hh_ = Histories{h_phi_.data(), h_force_.data(), h_energy_.data(), h_maxov_.data(),
                        h_mu_.data(), h_alpha_.data(), h_muflag_.data()};
    }
    hctl_pinned_ = pinned_ctl_acquire();
}

void Engine::ensure_row_capacity(std::uint32_t need) {
    if (need <= a_.S && a_.nbr) return;
    std::uint32_t S = std::max<std::uint32_t>(a_.S, 8u);
    while (S < need) S = S + S / 2 + 8;
    if (static_cast<std::uint64_t>(S) > N_) S = static_cast<std::uint32_t>(std::max<std::uint64_t>(N_, 1));
    if (S < need) S = need;
    auto drop = [&](void* p) {
        if (!p) return;
        cudaFreeAsync(p, st_);
        allocs_.erase(std::remove(allocs_.begin(), allocs_.end(), p), allocs_.end());
    };
    drop(a_.nbr);
    drop(a_.pterm);
    a_.nbr = nullptr;
    a_.pterm = nullptr;
    void* p = nullptr;
    check(pool_alloc_async(&p, static_cast<std::size_t>(S) * N_ * 4, st_), "cudaMallocFromPoolAsync(nbr)");
    allocs_.push_back(p);
    a_.nbr = static_cast<std::uint32_t*>(p);
    if (exact_) {
        check(pool_alloc_async(&p, static_cast<std::size_t>(S) * N_ * sizeof(PairTerms), st_), "cudaMallocFromPoolAsync(pterm)");
        allocs_.push_back(p);
        a_.pterm = static_cast<PairTerms*>(p);
    }
    a_.S = S;
    destroy_graph();
}

void Engine::free_device() {
    destroy_graph();
    for (void* p : allocs_) cudaFreeAsync(p, st_);
    allocs_.clear();
    if (st_) cudaStreamSynchronize(st_);
    if (hctl_pinned_) pinned_ctl_release(hctl_pinned_);
    hctl_pinned_ = nullptr;
}

void Engine::push_ctl() {
    *hctl_pinned_ = hctl_;
    check(cudaMemcpyAsync(a_.ctl, hctl_pinned_, sizeof(DevCtl), cudaMemcpyHostToDevice, st_), "push ctl");
    check(cudaStreamSynchronize(st_), "sync");
}

void Engine::pull_ctl() {
    check(cudaMemcpyAsync(hctl_pinned_, a_.ctl, sizeof(DevCtl), cudaMemcpyDeviceToHost, st_), "pull ctl");
    if (sync_ev_) {
        check(cudaEventRecord(sync_ev_, st_), "event record");
        check(cudaEventSynchronize(sync_ev_), "sync");
    } else {
        check(cudaStreamSynchronize(st_), "sync");
    }
    hctl_ = *hctl_pinned_;
}

void Engine::set_blocking_sync(bool on) {
    if (on && !sync_ev_) {
        check(cudaEventCreateWithFlags(&sync_ev_, cudaEventBlockingSync | cudaEventDisableTiming), "event");
    } else if (!on && sync_ev_) {
        cudaEventDestroy(sync_ev_);
        sync_ev_ = nullptr;
    }
}

// Parameters of the kernels of the step that begin_step() just opened
// (the host twin of the tail of k_controller).
void Engine::publish_step_params() {
    const Controller& c = host_c_;
    hctl_.c = c;
    for (int d = 0; d < ndim_; ++d) {
        hctl_.g.box[d] = c.box[d];
        hctl_.g.inv_box[d] = 1.0 / c.box[d];
    }
    hctl_.refresh_kappa = c.kappa_D;
    hctl_.force_kappa = c.kappa_D;
    hctl_.force_mu = c.mu_eff;
    hctl_.build_kappa = c.kappa_D;
    hctl_.build_t_shell = c.t_shell;
    hctl_.build_Dmax = c.Dmax_cur;
    hctl_.theta = c.theta;
    hctl_.forces_done = 0u;
    if (c.rebuild_mode == REBUILD_FULL) {
        hctl_.rebuild_flag = 1u;
    } else {
        hctl_.rebuild_flag = 0u;
        hctl_.kappa_min = std::fmin(hctl_.kappa_min, c.kappa_D);
    }
}

void Engine::upload_initial() {
    const std::uint64_t N = N_;
    const int nd = ndim_;
    std::vector<double> pos(N * P_, 0.0);
    for (std::uint64_t i = 0; i < N; ++i) {
        for (int d = 0; d < nd; ++d) pos[i * P_ + d] = x0_[i * nd + d];
        pos[i * P_ + nd] = D0_[i];
    }
    std::vector<std::uint64_t> origin(N);
    std::iota(origin.begin(), origin.end(), 0ull);
    check(cudaMemcpyAsync(a_.pos, pos.data(), pos.size() * 8, cudaMemcpyHostToDevice, st_), "H2D pos");
    check(cudaMemcpyAsync(a_.origin, origin.data(), N * 8, cudaMemcpyHostToDevice, st_), "H2D origin");
    check(cudaMemcpyAsync(a_.caps, caps_.data(), N * 4, cudaMemcpyHostToDevice, st_), "H2D caps");
    std::vector<std::uint32_t> rank;
    if (a_.permute) {
        rank.resize(N);
        std::iota(rank.begin(), rank.end(), 0u);
        check(cudaMemcpyAsync(a_.ref_rank, rank.data(), N * 4, cudaMemcpyHostToDevice, st_), "H2D rank");
    }
    check(cudaMemsetAsync(a_.m, 0, N * nd * 8, st_), "memset m");
    check(cudaMemsetAsync(a_.v, 0, N * nd * 8, st_), "memset v");
    check(cudaMemsetAsync(a_.F, 0, N * nd * 8, st_), "memset F");
    check(cudaStreamSynchronize(st_), "sync");

    std::memset(&hctl_, 0, sizeof(hctl_));
    set_size_classes(D0_, hctl_);
    Geometry& g = hctl_.g;
    g.ndim = nd;
    g.circle_k = walls_[0] < 0 ? -walls_[0] : 0;
    g.any_flat_wall = 0;
    for (int d = 0; d < nd; ++d) {
        g.walls[d] = walls_[d];
        if (walls_[d] == 1) g.any_flat_wall = 1;
        g.box[d] = host_c_.box[d];
        g.inv_box[d] = 1.0 / host_c_.box[d];
    }
    hctl_.c = host_c_;
    hctl_.fix_height_scale = 1.0;
    hctl_.build_kappa = 1.0;
    hctl_.build_t_shell = host_c_.t_shell;
    hctl_.build_Dmax = host_c_.Dmax_cur;
    hctl_.refresh_kappa = 1.0;
    hctl_.kappa_min = 1.0;
    hctl_.theta = host_c_.theta;
    hctl_.force_kappa = 1.0;
    hctl_.force_mu = host_c_.mu;
    hctl_.rebuild_flag = 1u;
    hctl_.fuse_forces = 0u;  // set for the graph loop once the run starts
    hctl_.pair_fp32 = 0u;    // the initial energy is FP64; the graph loop may switch to mixed
    hctl_.mixed_switch = mixed_switch_;
    push_ctl();

    // initial spatial reorder + full build (ENG:4992-5009), initial forces (ENG:5011-5013)
    if (host_c_.reorder_interval > 0) {
        launch_reorder(a_, st_);
        launches_ += 3 + 8 * 4 + 3;
    }
    for (int attempt = 0; attempt < 8; ++attempt) {
        launch_rebuild(a_, st_);
        launches_ += 7;
        forces_and_reduce(exact_);
        pull_ctl();
        if (hctl_.cap_error) break;
        if (hctl_.row_need <= a_.S) break;
        ensure_row_capacity(hctl_.row_need);
        hctl_.rebuild_flag = 1u;
        push_ctl();
    }
    if (hctl_.cap_error) {
        throw EngineError(-ENOSPC, std::string("rcpgenerator: particle ") +
                                       std::to_string(cap_error_particle(hctl_)) +
                                       " exceeded its neighbor capacity (" +
                                       std::to_string(cap_error_capacity(hctl_)) +
                                       " slots) during pair-list construction (kdtree own-write). "
                                       "This usually means the per-particle neighbor allocation is too small for the size ratio in this packing. "
                                       "Recommendation: pass a larger neighbor_max (the per-particle base; e.g. neighbor_max=1500 -- capacity scales as 50*(D_i/D_min)^omega + neighbor_max), or reduce the size ratio.");
    }
    const StepScalars s0 = finalize_sums(hctl_.sums, host_c_.mu, ndim_);
    initial_U_ = s0.U;
    initial_maxov_ = s0.max_overlap;
    host_c_.U = s0.U;
    host_c_.max_min_dist = s0.max_overlap;
    hctl_.rebuild_flag = 0u;
    hctl_.c = host_c_;
    push_ctl();
}

Engine::Engine(const EngineInput& in, cudaStream_t stream) {
    setup_host(in);
    check(cudaSetDevice(in.device), "cudaSetDevice");
    if (stream) {
        st_ = stream;
    } else {
        check(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking), "cudaStreamCreate");
        own_stream_ = true;
    }
    try {
        alloc_device();
        upload_initial();
    } catch (...) {
        free_device();
        if (own_stream_) cudaStreamDestroy(st_);
        throw;
    }
}

Engine::~Engine() {
    cudaSetDevice(device_);
    if (sync_ev_) cudaEventDestroy(sync_ev_);
    free_device();
    if (body_st_) cudaStreamDestroy(body_st_);
    if (own_stream_ && st_) cudaStreamDestroy(st_);
}

std::uint64_t Engine::builds() {
    pull_ctl();
    return hctl_.nbuilds;
}

void Engine::profile_build_kernel(std::uint32_t reps, double* avg_ms, double* alg_bytes) {
    pull_ctl();
    const DevCtl saved = hctl_;
    const std::size_t flush_bytes = std::size_t{256} << 20;
    void* flush = nullptr;
    check(pool_alloc_async(&flush, flush_bytes, st_), "cudaMallocFromPoolAsync(flush)");
    cudaEvent_t e0, e1;
    check(cudaEventCreate(&e0), "event");
    check(cudaEventCreate(&e1), "event");
    double total_ms = 0.0;
    for (std::uint32_t k = 0; k <= reps; ++k) {  // launch 0 warms up
        // each build of cell-order storage moves the particles to the other
        // buffer set: keep the set the previous build left current
        if (k > 0) pull_ctl();
        const std::uint32_t cur = hctl_.buf;
        hctl_ = saved;
        hctl_.buf = cur;
        hctl_.stopped = 0u;
        hctl_.halted = 0u;
        hctl_.rebuild_flag = 1u;
        hctl_.fuse_forces = exact_ ? 0u : 1u;
        push_ctl();
        check(cudaMemsetAsync(flush, static_cast<int>(k & 0xFF), flush_bytes, st_), "flush");
        launch_rebuild_timed(a_, st_, e0, e1);
        check(cudaEventSynchronize(e1), "sync");
        float ms = 0.f;
        check(cudaEventElapsedTime(&ms, e0, e1), "elapsed");
        if (k > 0) total_ms += ms;
        launches_ += 9;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    check(cudaFreeAsync(flush, st_), "cudaFreeAsync(flush)");
    std::vector<std::uint32_t> cnt(N_);
    check(cudaMemcpyAsync(cnt.data(), a_.nbr_cnt, N_ * 4, cudaMemcpyDeviceToHost, st_), "D2H cnt");
    check(cudaStreamSynchronize(st_), "sync");
    double total = 0.0;
    for (std::uint32_t c : cnt) total += c;
    // per particle: its record (8P), row length (4) and row entries (4k); the
    // tiled search (exact mode) also stages id and row slot (8), the cell-order
    // search (graph mode) writes the fused force F_i (8*ndim)
    const double per = 8.0 * P_ + 4.0 + (exact_ ? 8.0 : 8.0 * ndim_);
    *avg_ms = reps ? total_ms / reps : 0.0;
    *alg_bytes = static_cast<double>(N_) * per + 4.0 * total;
    pull_ctl();
    const std::uint32_t cur = hctl_.buf;
    hctl_ = saved;
    hctl_.buf = cur;
    push_ctl();
}

void Engine::profile_pair_kernel(std::uint32_t reps, double* avg_ms, double* alg_bytes,
                                 double* mean_row) {
    pull_ctl();
    const DevCtl saved = hctl_;
    hctl_.stopped = 0u;
    hctl_.halted = 0u;
    hctl_.forces_done = 0u;
    push_ctl();
    // every launch starts from a cold L2: a 256 MiB write evicts the previous
    // launch's lines (L2 is 126 MB), then the launch alone is timed
    const std::size_t flush_bytes = std::size_t{256} << 20;
    void* flush = nullptr;
    check(pool_alloc_async(&flush, flush_bytes, st_), "cudaMallocFromPoolAsync(flush)");
    cudaEvent_t e0, e1;
    check(cudaEventCreate(&e0), "event");
    check(cudaEventCreate(&e1), "event");
    launch_forces(a_, 0, st_);  // warm the instruction cache / first-touch
    double total_ms = 0.0;
    for (std::uint32_t k = 0; k < reps; ++k) {
        check(cudaMemsetAsync(flush, static_cast<int>(k & 0xFF), flush_bytes, st_), "flush");
        check(cudaEventRecord(e0, st_), "record");
        launch_forces(a_, 0, st_);
        check(cudaEventRecord(e1, st_), "record");
        check(cudaEventSynchronize(e1), "sync");
        float ms = 0.f;
        check(cudaEventElapsedTime(&ms, e0, e1), "elapsed");
        total_ms += ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    check(cudaFreeAsync(flush, st_), "cudaFreeAsync(flush)");
    const double ms = total_ms;
    launches_ += reps + 1;
    std::vector<std::uint32_t> cnt(N_);
    check(cudaMemcpyAsync(cnt.data(), a_.nbr_cnt, N_ * 4, cudaMemcpyDeviceToHost, st_), "D2H cnt");
    check(cudaStreamSynchronize(st_), "sync");
    double total = 0.0;
    for (std::uint32_t c : cnt) total += c;
    // per particle: read x_i (8*ndim) + D0_i (8) + row length (4) + row ids (4*k), write F_i (8*ndim)
    const double bytes = static_cast<double>(N_) * (16.0 * ndim_ + 12.0) + 4.0 * total;
    *avg_ms = reps ? ms / reps : 0.0;
    *alg_bytes = bytes;
    *mean_row = total / static_cast<double>(N_);
    hctl_ = saved;
    push_ctl();
}

void Engine::forces_and_reduce(bool exact_reduce) {
    launch_forces(a_, exact_reduce ? 1 : 0, st_);
    if (exact_reduce) launch_reduce_exact(a_, st_);
    else launch_reduce_fast(a_, st_);
    launches_ += 2;
}

// Reorder of the step that begin_step() opened: permutes with the positions
// after the previous step and rebuilds with the previous diameters (ENG:4850-4948).
void Engine::do_reorder_and_rebuild() {
    const Controller& c = host_c_;
    const double kp = c.runtime_fix_diameter ? 1.0 : c.kappa_D_prev;
    hctl_.build_kappa = kp;
    hctl_.build_t_shell = shell_of(xmul(c.D0_min, kp), xmul(c.D0_med, kp), xmul(c.D0_max, kp));
    hctl_.build_Dmax = xmul(c.D0_max, kp);
    hctl_.rebuild_flag = 1u;
    hctl_.stopped = 0u;
    const std::uint32_t fuse = hctl_.fuse_forces;
    hctl_.fuse_forces = 0u;  // this build uses the previous step's diameters
    push_ctl();
    launch_reorder(a_, st_);
    launches_ += 3 + 8 * 4 + 3;
    for (int attempt = 0; attempt < 8; ++attempt) {
        launch_rebuild(a_, st_);
        launches_ += 7;
        pull_ctl();
        if (hctl_.cap_error || hctl_.row_need <= a_.S) break;
        ensure_row_capacity(hctl_.row_need);
        hctl_.rebuild_flag = 1u;
        push_ctl();
    }
    hctl_.fuse_forces = fuse;
    hctl_.forces_done = 0u;
}

// Target-phi lock (ENG:5783-5832): D0 := D rescaled to the target, kappa := 1.
void Engine::do_target_lock(std::uint64_t step) {
    Controller& c = host_c_;
    const std::uint64_t N = N_;
    const int nd = ndim_;
    std::vector<double> pos(N * P_);
    check(cudaMemcpyAsync(pos.data(), a_.pos, pos.size() * 8, cudaMemcpyDeviceToHost, st_), "D2H pos");
    check(cudaStreamSynchronize(st_), "sync");
    std::vector<double> D(N);
    for (std::uint64_t i = 0; i < N; ++i) D[i] = pos[i * P_ + nd] * c.kappa;
    std::vector<double> boxv(c.box, c.box + nd);
    double factor = 1.0;
    std::vector<double> Dn = scale_diameters_nd(D, c.target_phi * c.phi_modifier, boxv, nd, c.fix_height != 0, &factor);
    double D0min = Dn[0], D0max = 0.0, S = 0.0;
    for (std::uint64_t i = 0; i < N; ++i) {
        if (Dn[i] < D0min) D0min = Dn[i];
        if (Dn[i] > D0max) D0max = Dn[i];
        double r = Dn[i] * 0.5, rN = 1.0;
        for (int k = 0; k < nd; ++k) rN *= r;
        S += rN;
        pos[i * P_ + nd] = Dn[i];
    }
    std::vector<double> Dm = Dn;
    std::nth_element(Dm.begin(), Dm.begin() + N / 2, Dm.end());
    const double D0med = Dm[N / 2];
    check(cudaMemcpyAsync(a_.pos, pos.data(), pos.size() * 8, cudaMemcpyHostToDevice, st_), "H2D pos");
    // caps of the new diameters (ENG:5815-5819 recomputes the pair layout)
    {
        const double scaling = static_cast<double>(nd) / 3.0;
        const double omega = 1.0 + static_cast<double>(nd) / 6.0;
        const double dmin = D0min > 0.0 ? D0min : 1.0;
        for (std::uint64_t i = 0; i < N; ++i) {
            const double cap_d = scaling * (50.0 * std::pow(Dn[i] / dmin, omega) + static_cast<double>(neighbor_max_));
            std::uint32_t cap = static_cast<std::uint32_t>(std::ceil(cap_d));
            if (static_cast<std::uint64_t>(cap) > N) cap = static_cast<std::uint32_t>(N);
            caps_[i] = cap;
        }
        check(cudaMemcpyAsync(a_.caps, caps_.data(), N * 4, cudaMemcpyHostToDevice, st_), "H2D caps");
    }
    finish_lock(c, hh_, step, D0min, D0max, D0med, S);
    set_size_classes(Dn, hctl_);
    // full rebuild with the new diameters, re-anchor everything
    hctl_.build_kappa = 1.0;
    hctl_.build_t_shell = shell_of(D0min, D0med, D0max);
    hctl_.build_Dmax = D0max;
    hctl_.rebuild_flag = 1u;
    push_ctl();
    launch_rebuild(a_, st_);
    launches_ += 7;
}

}  // namespace rcpg

namespace rcpg {

// ---------------------------------------------------------------------------
// exact mode: one step with the controller on the host
// ---------------------------------------------------------------------------
// Returns false when the run has ended (convergence at the top of the step or
// step cap reached before it).
bool Engine::step_host() {
    Controller& c = host_c_;
    const std::uint64_t step = c.hist_filled + 1;
    if (step > c.step_cap) return false;
    begin_step(c, hh_, step);
    // 1. pending ADAM pass of the previous step (positions after step-1)
    if (adam_pending_) {
        hctl_.adam_go = 1u;
        hctl_.fix_height_scale = 1.0;
        hctl_.stopped = 0u;
        hctl_.halted = 0u;
        push_ctl();
        launch_adam_refresh(a_, 1, 0, st_);
        ++launches_;
        adam_pending_ = false;
        hctl_.adam_go = 0u;
    }
    if (c.done) return false;
    // 2. reorder at the top of the step, with the previous diameters
    if (c.reorder) {
        do_reorder_and_rebuild();
        if (hctl_.cap_error) pull_ctl();
    }
    // 3. fix_height stretch of the last axis (ENG:5758-5764)
    if (c.fix_height && !c.runtime_fix_diameter) {
        hctl_.fix_height_scale = c.fix_height_scale;
        push_ctl();
        launch_fix_height(a_, st_);
        ++launches_;
    }
    // 4. target-phi lock (rescale + full rebuild), else the refresh decision
    if (c.lock_now) {
        do_target_lock(step);
    }
    publish_step_params();
    hctl_.adam_go = 0u;
    hctl_.stopped = 0u;
    hctl_.halted = 0u;
    push_ctl();
    if (c.rebuild_mode == REBUILD_CHECK) {
        launch_adam_refresh(a_, 0, 1, st_);
        ++launches_;
    }
    // 5. rebuild (if flagged) + forces + one-thread-order reduction
    for (int attempt = 0; attempt < 8; ++attempt) {
        launch_rebuild(a_, st_);
        launches_ += 7;
        forces_and_reduce(true);
        pull_ctl();
        if (hctl_.cap_error || hctl_.row_need <= a_.S) break;
        ensure_row_capacity(hctl_.row_need);
        hctl_.rebuild_flag = 1u;
        push_ctl();
    }
    if (hctl_.cap_error) {
        throw EngineError(-ENOSPC, std::string("rcpgenerator: particle ") +
                                       std::to_string(cap_error_particle(hctl_)) +
                                       " exceeded its neighbor capacity (" +
                                       std::to_string(cap_error_capacity(hctl_)) +
                                       " slots) during pair-list construction (kdtree own-write). "
                                       "This usually means the per-particle neighbor allocation is too small for the size ratio in this packing. "
                                       "Recommendation: pass a larger neighbor_max (the per-particle base; e.g. neighbor_max=1500 -- capacity scales as 50*(D_i/D_min)^omega + neighbor_max), or reduce the size ratio.");
    }
    hctl_.rebuild_flag = 0u;
    // 6. end of step on the host
    const StepScalars sc = finalize_sums(hctl_.sums, c.mu_eff, ndim_);
    hctl_.scal = sc;
    end_step(c, hh_, sc);
    for (int d = 0; d < ndim_; ++d) hctl_.adam_box[d] = c.box[d];
    hctl_.adam_alpha = c.adam_alpha;
    hctl_.adam_inv_b1 = c.inv_b1;
    hctl_.adam_inv_b2 = c.inv_b2;
    adam_pending_ = true;
    return true;
}

// ---------------------------------------------------------------------------
// graph mode
// ---------------------------------------------------------------------------
void Engine::destroy_graph() {
    if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
    if (graph_) cudaGraphDestroy(graph_);
    graph_exec_ = nullptr;
    graph_ = nullptr;
}

// Kernels of one neighbour build (launch_rebuild): prepare, bin, the scan
// (one kernel, or three for more than 4096 tiles of cells), scatter, cell
// sort, the permutation of cell-order storage, the cell-unit search
// (ndim <= 3, N >= 20,000; one kernel per pair precision the run may use) or
// the tiled search, and the warp search.
std::uint64_t Engine::kernels_per_build() const {
    const std::uint64_t cells = static_cast<std::uint64_t>(a_.C_alloc) + 1;
    const std::uint64_t scans = cells <= 4096 ? 1 : 3;
    std::uint64_t k = 4 + scans + (a_.permute ? 1 : 0) + 1;
    if (ndim_ <= 3 && N_ >= 20000) {
        if (a_.permute) k += a_.mixed ? 2 : 1;
        else if (a_.sorted_rows) k += 1;
    }
    return k;
}

template <typename Body>
void Engine::add_conditional(int type, unsigned long long handle, unsigned size, Body body) {
    cudaStreamCaptureStatus status;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    std::size_t nd = 0;
    check(cudaStreamGetCaptureInfo(st_, &status, nullptr, &g, &deps, &nd), "capture info");
    cudaGraphNodeParams p = {cudaGraphNodeTypeConditional};
    p.conditional.handle = handle;
    p.conditional.type = static_cast<cudaGraphConditionalNodeType>(type);
    p.conditional.size = size;
    cudaGraphNode_t node = nullptr;
    check(cudaGraphAddNode(&node, g, deps, nd, &p), "add conditional node");
    for (unsigned b = 0; b < size; ++b) {
        check(cudaStreamBeginCaptureToGraph(body_st_, p.conditional.phGraph_out[b], nullptr, nullptr, 0,
                                            cudaStreamCaptureModeThreadLocal),
              "capture conditional body");
        body(body_st_, b);
        cudaGraph_t out = nullptr;
        check(cudaStreamEndCapture(body_st_, &out), "end conditional body");
    }
    check(cudaStreamUpdateCaptureDependencies(st_, &node, 1, cudaStreamSetCaptureDependencies),
          "capture dependencies");
}

void Engine::capture_step() {
    cudaStreamCaptureStatus status;
    cudaGraph_t g = nullptr;
    check(cudaStreamGetCaptureInfo(st_, &status, nullptr, &g, nullptr, nullptr), "capture info");
    cudaGraphConditionalHandle build = 0, forces = 0;
    check(cudaGraphConditionalHandleCreate(&build, g, 0, cudaGraphCondAssignDefault), "conditional handle");
    check(cudaGraphConditionalHandleCreate(&forces, g, 2, cudaGraphCondAssignDefault), "conditional handle");
    DevArrays ag = a_;
    ag.cond_forces = forces;
    launch_step_gate(ag, build, st_);
    add_conditional(cudaGraphCondTypeIf, build, 1, [&](cudaStream_t s, unsigned) { launch_rebuild(ag, s); });
    add_conditional(cudaGraphCondTypeSwitch, forces, mixed_ ? 2u : 1u,
                    [&](cudaStream_t s, unsigned variant) { launch_forces_variant(ag, static_cast<int>(variant), s); });
    launch_controller(ag, 0, st_);
    launch_adam_refresh(ag, 1, 1, st_);
}

// The step loop as one CUDA graph of graph_steps_ steps. Each step opens with
// a one-thread gate kernel; the build and the pair kernel sit in conditional
// nodes that the gate and the build set on the device, so a step without a
// rebuild launches four kernels (gate, pair kernel, controller, ADAM).
void Engine::capture_graph() {
    destroy_graph();
    if (!body_st_) check(cudaStreamCreateWithFlags(&body_st_, cudaStreamNonBlocking), "cudaStreamCreate");
    check(cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal), "begin capture");
    try {
        for (int k = 0; k < graph_steps_; ++k) capture_step();
    } catch (...) {
        cudaGraph_t partial = nullptr;
        cudaStreamEndCapture(st_, &partial);
        if (partial) cudaGraphDestroy(partial);
        cudaGetLastError();
        throw;
    }
    check(cudaStreamEndCapture(st_, &graph_), "end capture");
    check(cudaGraphInstantiate(&graph_exec_, graph_, 0), "graph instantiate");
    std::size_t nodes = 0;
    check(cudaGraphGetNodes(graph_, nullptr, &nodes), "graph nodes");
    graph_nodes_per_step_ = nodes / static_cast<std::uint64_t>(graph_steps_);
}

// Opening of step 1 (or of the step after a host intervention): the host
// already ran begin_step(); publish it and run the refresh trigger.
void Engine::after_stop() {
    Controller& c = host_c_;
    const std::uint64_t step = c.steps;
    if (c.reorder) do_reorder_and_rebuild();
    if (hctl_.cap_error) return;
    if (c.fix_height && !c.runtime_fix_diameter && c.fix_height_scale != 1.0 && c.reorder) {
        // the stretch was deferred past the reorder
        hctl_.fix_height_scale = c.fix_height_scale;
        push_ctl();
        launch_fix_height(a_, st_);
        ++launches_;
    }
    (void)step;
    publish_step_params();
    hctl_.adam_go = 0u;
    hctl_.stopped = 0u;
    hctl_.halted = 0u;
    push_ctl();
    if (c.rebuild_mode == REBUILD_CHECK) {
        launch_adam_refresh(a_, 0, 1, st_);
        ++launches_;
    }
}

bool Engine::advance_graph(std::uint64_t max_new_steps) {
    Controller& c = host_c_;
    const std::uint64_t start = c.hist_filled;
    if (c.hist_filled == 0 && c.steps == 0) {
        // step 1 opens on the device like every later step
        hctl_.c = c;
        hctl_.stopped = 0u;
        hctl_.halted = 0u;
        hctl_.fuse_forces = 1u;  // rebuild steps compute their forces in the tiled build
        hctl_.pair_fp32 = mixed_ ? 1u : 0u;
        push_ctl();
        launch_controller(a_, 1, st_);
        ++launches_;
        pull_ctl();
        c = hctl_.c;
        if (hctl_.stopped) {
            if (c.done || c.steps + 1 > c.step_cap) {
                finished_ = true;
                return true;
            }
            after_stop();
        } else if (c.rebuild_mode == REBUILD_CHECK) {
            launch_adam_refresh(a_, 0, 1, st_);
            ++launches_;
        }
    }
    while (!finished_) {
        const std::uint64_t done_steps = c.hist_filled - start;
        if (max_new_steps && done_steps >= max_new_steps) break;
        const std::uint64_t want = max_new_steps ? max_new_steps - done_steps : ~0ull;
        if (!graph_exec_) capture_graph();
        const std::uint64_t b0 = hctl_.nbuilds, f0 = hctl_.pair_kernel_runs;
        bool replay = false;
        if (want >= static_cast<std::uint64_t>(graph_steps_)) {
            check(cudaGraphLaunch(graph_exec_, st_), "graph launch");
            replay = true;
        } else {
            for (std::uint64_t k = 0; k < want; ++k) {
                launch_rebuild(a_, st_);
                launch_forces(a_, 0, st_);
                launch_controller(a_, 0, st_);
                launch_adam_refresh(a_, 1, 1, st_);
                launches_ += kernels_per_build() + (mixed_ ? 4 : 3);
            }
        }
        pull_ctl();
        c = hctl_.c;
        if (replay) {
            // kernels the replay ran: gate, controller and ADAM of each of its
            // steps (they return at once after a stop), and the builds and pair
            // kernels its conditional nodes opened
            launches_ += 3 * static_cast<std::uint64_t>(graph_steps_) +
                         (hctl_.nbuilds - b0) * kernels_per_build() + (hctl_.pair_kernel_runs - f0);
        }
        if (hctl_.halted) {
            if (hctl_.cap_error) {
                throw EngineError(-ENOSPC, std::string("rcpgenerator: particle ") +
                                               std::to_string(cap_error_particle(hctl_)) +
                                               " exceeded its neighbor capacity (" +
                                               std::to_string(cap_error_capacity(hctl_)) +
                                               " slots) during pair-list construction (kdtree own-write). "
                                               "This usually means the per-particle neighbor allocation is too small for the size ratio in this packing. "
                                               "Recommendation: pass a larger neighbor_max (the per-particle base; e.g. neighbor_max=1500 -- capacity scales as 50*(D_i/D_min)^omega + neighbor_max), or reduce the size ratio.");
            }
            handle_overflow_and_resume();
            continue;
        }
        if (hctl_.stopped) {
            if (c.done || c.steps + 1 > c.step_cap || c.hist_filled >= c.step_cap) {
                if (!c.done && c.hist_filled < c.step_cap) {
                    // stopped before opening the next step: nothing pending
                }
                finished_ = true;
                break;
            }
            after_stop();
            if (hctl_.cap_error) {
                pull_ctl();
                throw EngineError(-ENOSPC, "rcpgenerator: neighbor capacity exceeded during reorder rebuild");
            }
        }
    }
    return finished_;
}

// A build found a row longer than the allocated capacity: grow, rebuild and
// redo the interrupted step from its forces.
void Engine::handle_overflow_and_resume() {
    ensure_row_capacity(hctl_.row_need);
    hctl_.halted = 0u;
    hctl_.stopped = 0u;
    hctl_.rebuild_flag = 1u;
    hctl_.row_need = 0u;
    push_ctl();
    launch_rebuild(a_, st_);
    launch_forces(a_, 0, st_);
    launch_controller(a_, 0, st_);
    launch_adam_refresh(a_, 1, 1, st_);
    launches_ += kernels_per_build() + (mixed_ ? 4 : 3);
}

bool Engine::advance(std::uint64_t max_new_steps) {
    if (finished_) return true;
    if (exact_) {
        std::uint64_t n = 0;
        while (!max_new_steps || n < max_new_steps) {
            if (!step_host()) {
                finished_ = true;
                break;
            }
            ++n;
        }
        if (finished_ && adam_pending_) {
            hctl_.adam_go = 1u;
            hctl_.fix_height_scale = 1.0;
            push_ctl();
            launch_adam_refresh(a_, 1, 0, st_);
            ++launches_;
            adam_pending_ = false;
            hctl_.adam_go = 0u;
        }
        return finished_;
    }
    return advance_graph(max_new_steps);
}

void Engine::download_histories() {
    if (!histories_on_device_) return;
    const std::size_t n = host_c_.hist_filled;
    h_phi_.assign(n, 0.0);
    h_force_.assign(n, 0.0);
    h_energy_.assign(n, 0.0);
    h_maxov_.assign(n, 0.0);
    h_mu_.assign(n, 0.0);
    h_alpha_.assign(n, 0.0);
    h_muflag_.assign(n, 0);
    if (n) {
        check(cudaMemcpyAsync(h_phi_.data(), a_.hist.phi, n * 8, cudaMemcpyDeviceToHost, st_), "D2H");
        check(cudaMemcpyAsync(h_force_.data(), a_.hist.force, n * 8, cudaMemcpyDeviceToHost, st_), "D2H");
        check(cudaMemcpyAsync(h_energy_.data(), a_.hist.energy, n * 8, cudaMemcpyDeviceToHost, st_), "D2H");
        check(cudaMemcpyAsync(h_maxov_.data(), a_.hist.max_overlap, n * 8, cudaMemcpyDeviceToHost, st_), "D2H");
        check(cudaMemcpyAsync(h_mu_.data(), a_.hist.mu, n * 8, cudaMemcpyDeviceToHost, st_), "D2H");
        check(cudaMemcpyAsync(h_alpha_.data(), a_.hist.alpha, n * 8, cudaMemcpyDeviceToHost, st_), "D2H");
        check(cudaMemcpyAsync(h_muflag_.data(), a_.hist.mu_flag, n, cudaMemcpyDeviceToHost, st_), "D2H");
        check(cudaStreamSynchronize(st_), "sync");
    }
}

void Engine::download_particles(std::vector<double>& pos, std::vector<std::uint64_t>* origin) {
    const std::uint64_t N = N_;
    pos.resize(N * P_);
    if (origin) origin->resize(N);
    if (!a_.permute) {
        check(cudaMemcpyAsync(pos.data(), a_.pos, pos.size() * 8, cudaMemcpyDeviceToHost, st_), "D2H pos");
        if (origin)
            check(cudaMemcpyAsync(origin->data(), a_.origin, N * 8, cudaMemcpyDeviceToHost, st_), "D2H origin");
        check(cudaStreamSynchronize(st_), "sync");
        return;
    }
    // cell-order storage: the current buffer set, then particle q goes to its
    // reference index ref_rank[q]
    pull_ctl();
    const DevArrays cur = bound_arrays(a_, hctl_.buf);
    std::vector<double> cell(N * P_);
    std::vector<std::uint64_t> org(origin ? N : 0);
    std::vector<std::uint32_t> rank(N);
    check(cudaMemcpyAsync(cell.data(), cur.pos, cell.size() * 8, cudaMemcpyDeviceToHost, st_), "D2H pos");
    check(cudaMemcpyAsync(rank.data(), cur.ref_rank, N * 4, cudaMemcpyDeviceToHost, st_), "D2H rank");
    if (origin) check(cudaMemcpyAsync(org.data(), cur.origin, N * 8, cudaMemcpyDeviceToHost, st_), "D2H origin");
    check(cudaStreamSynchronize(st_), "sync");
    for (std::uint64_t q = 0; q < N; ++q) {
        const std::uint64_t r = rank[q];
        for (int k = 0; k < P_; ++k) pos[r * P_ + k] = cell[q * P_ + k];
        if (origin) (*origin)[r] = org[q];
    }
}

EngineResult Engine::result() {
    if (exact_ && adam_pending_) {
        hctl_.adam_go = 1u;
        hctl_.fix_height_scale = 1.0;
        push_ctl();
        launch_adam_refresh(a_, 1, 0, st_);
        ++launches_;
        adam_pending_ = false;
        hctl_.adam_go = 0u;
    }
    if (!exact_) {
        pull_ctl();
        host_c_ = hctl_.c;
    }
    const Controller& c = host_c_;
    const std::uint64_t N = N_;
    const int nd = ndim_;
    EngineResult r;
    std::vector<double> pos;
    download_particles(pos, &r.particle_origin);
    r.positions.resize(N * nd);
    r.diameters.resize(N);
    // diameters of the last diameter update: D = D0*kappa (ENG:5733)
    const double kd = c.runtime_fix_diameter ? 1.0 : c.kappa_D;
    for (std::uint64_t i = 0; i < N; ++i) {
        for (int d = 0; d < nd; ++d) r.positions[i * nd + d] = pos[i * P_ + d];
        r.diameters[i] = c.runtime_fix_diameter ? pos[i * P_ + nd] : pos[i * P_ + nd] * kd;
    }
    r.box.assign(c.box, c.box + nd);
    r.walls = walls_;
    download_histories();
    const std::size_t n = c.hist_filled;
    r.phi_history.assign(h_phi_.begin(), h_phi_.begin() + n);
    r.force_history.assign(h_force_.begin(), h_force_.begin() + n);
    r.energy_history.assign(h_energy_.begin(), h_energy_.begin() + n);
    r.max_overlap_history.assign(h_maxov_.begin(), h_maxov_.begin() + n);
    r.mu_history.assign(h_mu_.begin(), h_mu_.begin() + n);
    r.alpha_history.assign(h_alpha_.begin(), h_alpha_.begin() + n);
    r.mu_flag_history.assign(h_muflag_.begin(), h_muflag_.begin() + n);
    r.steps = n;
    r.phi = c.phi;
    r.max_min_dist = c.max_min_dist;
    r.force_magnitude = c.F_magnitude;
    pull_ctl();
    r.builds = hctl_.nbuilds;
    r.row_capacity = a_.S;
    r.fp64_switch_step = hctl_.fp64_switch_step;
    r.pair_energy_rel_error = r.pair_force_rel_error = std::nan("");
    if (mixed_) pair_precision_error(&r.pair_energy_rel_error, &r.pair_force_rel_error);
    return r;
}

void Engine::pair_precision_error(double* energy_rel, double* force_rel) {
    pull_ctl();
    const DevCtl saved = hctl_;
    const std::uint64_t n = N_ * static_cast<std::uint64_t>(ndim_);
    check(cudaMemcpyAsync(a_.vec_tmp, a_.F, n * 8, cudaMemcpyDeviceToDevice, st_), "save F");
    // the FP64 forces and the two maxima stay on the device
    void* scratch = nullptr;
    check(pool_alloc_async(&scratch, n * 8 + 16, st_), "cudaMallocFromPoolAsync(precision check)");
    double* F64 = static_cast<double*>(scratch);
    unsigned long long* mx = reinterpret_cast<unsigned long long*>(F64 + n);
    check(cudaMemsetAsync(mx, 0, 16, st_), "memset");
    double U[2] = {0.0, 0.0};
    for (int prec = 0; prec < 2; ++prec) {  // 0: FP64, 1: FP32 pair terms
        hctl_ = saved;
        hctl_.stopped = 0u;
        hctl_.halted = 0u;
        hctl_.forces_done = 0u;
        hctl_.pair_fp32 = static_cast<std::uint32_t>(prec);
        push_ctl();
        launch_forces(a_, 0, st_);
        launch_reduce_fast(a_, st_);
        launches_ += 2;
        if (prec == 0) {
            check(cudaMemcpyAsync(F64, a_.F, n * 8, cudaMemcpyDeviceToDevice, st_), "copy F");
        } else {
            launch_diff_max(F64, a_.F, n, mx, st_);
            ++launches_;
        }
        pull_ctl();
        U[prec] = hctl_.sums.pair_U;
    }
    unsigned long long bits[2] = {0ull, 0ull};
    check(cudaMemcpyAsync(bits, mx, 16, cudaMemcpyDeviceToHost, st_), "D2H max");
    check(cudaStreamSynchronize(st_), "sync");
    double fmax, dmax;
    std::memcpy(&fmax, &bits[0], 8);
    std::memcpy(&dmax, &bits[1], 8);
    *energy_rel = U[0] != 0.0 ? std::fabs(U[1] - U[0]) / std::fabs(U[0]) : std::fabs(U[1]);
    *force_rel = fmax > 0.0 ? dmax / fmax : dmax;
    check(cudaMemcpyAsync(a_.F, a_.vec_tmp, n * 8, cudaMemcpyDeviceToDevice, st_), "restore F");
    check(cudaFreeAsync(scratch, st_), "cudaFreeAsync");
    hctl_ = saved;
    push_ctl();
}

void Engine::observe(std::uint64_t step, bool capture, const ObserverFn& observer,
                     std::vector<TraceSample>* trace) {
    double vals[4] = {0, 0, 0, 0};
    if (step == 0) {
        vals[0] = host_c_.phi;  // setup phi (already divided by phi_modifier, ENG:4505)
        vals[1] = 0.0;
        vals[2] = initial_U_;
        vals[3] = initial_maxov_;
    } else if (histories_on_device_) {
        check(cudaMemcpyAsync(&vals[0], a_.hist.phi + step - 1, 8, cudaMemcpyDeviceToHost, st_), "D2H");
        check(cudaMemcpyAsync(&vals[1], a_.hist.force + step - 1, 8, cudaMemcpyDeviceToHost, st_), "D2H");
        check(cudaMemcpyAsync(&vals[2], a_.hist.energy + step - 1, 8, cudaMemcpyDeviceToHost, st_), "D2H");
        check(cudaMemcpyAsync(&vals[3], a_.hist.max_overlap + step - 1, 8, cudaMemcpyDeviceToHost, st_), "D2H");
        check(cudaStreamSynchronize(st_), "sync");
    } else {
        vals[0] = h_phi_[step - 1];
        vals[1] = h_force_[step - 1];
        vals[2] = h_energy_[step - 1];
        vals[3] = h_maxov_[step - 1];
    }
    Observation ob{step, vals[0], vals[1], vals[2], vals[3]};
    std::vector<double> xs;
    if (capture) {
        if (exact_ && adam_pending_) {
            hctl_.adam_go = 1u;
            hctl_.fix_height_scale = 1.0;
            push_ctl();
            launch_adam_refresh(a_, 1, 0, st_);
            ++launches_;
            adam_pending_ = false;
            hctl_.adam_go = 0u;
        }
        std::vector<double> pos;
        download_particles(pos, nullptr);
        xs.resize(N_ * ndim_);
        TraceSample ts;
        ts.step = step;
        ts.diameters.resize(N_);
        double kd = host_c_.kappa_D;
        if (!exact_ && step > 0) {
            pull_ctl();
            kd = hctl_.c.kappa_D_prev;
        }
        if (host_c_.runtime_fix_diameter) kd = 1.0;
        for (std::uint64_t i = 0; i < N_; ++i) {
            for (int d = 0; d < ndim_; ++d) xs[i * ndim_ + d] = pos[i * P_ + d];
            ts.diameters[i] = pos[i * P_ + ndim_] * kd;
        }
        ts.positions = xs;
        ts.phi = ob.phi;
        ts.force = ob.force_magnitude;
        ts.energy = ob.energy;
        ts.max_min_dist = ob.max_min_dist;
        if (trace) trace->push_back(std::move(ts));
    }
    if (observer) observer(ob, capture ? &xs : nullptr);
}

void Engine::run(std::uint64_t progress_interval, bool capture_positions,
                 std::uint64_t trajectory_interval, const ObserverFn& observer,
                 std::vector<TraceSample>* trace) {
    const bool want_obs = observer && progress_interval > 0;
    const bool want_cap = capture_positions && trajectory_interval > 0;
    if (want_obs || want_cap) observe(0, want_cap, observer, trace);
    if (!want_obs && !want_cap) {
        advance(0);
    } else {
        std::uint64_t every = 0;
        if (want_obs) every = progress_interval;
        if (want_cap) every = every ? std::gcd(every, trajectory_interval) : trajectory_interval;
        while (!finished_) {
            const std::uint64_t s0 = steps_done();
            const std::uint64_t next = (s0 / every + 1) * every;
            advance(next - s0);
            const std::uint64_t s = steps_done();
            if (s == next && s > 0) {
                const bool rep = want_obs && (s % progress_interval == 0);
                const bool cap = want_cap && (s % trajectory_interval == 0);
                if (rep || cap) observe(s, cap, rep ? observer : ObserverFn(), trace);
            }
        }
    }
    // final sample when the last step was not already recorded (ENG:6736-6762)
    const std::uint64_t last = host_c_.steps;
    const bool final_cap = want_cap && last > 0 && (last % trajectory_interval == 0);
    const bool final_rep = want_obs && last > 0 && (last % progress_interval == 0);
    if ((capture_positions && !final_cap) || (observer && !final_rep)) {
        EngineResult r = result();
        if (trace && capture_positions) {
            TraceSample ts;
            ts.step = last;
            ts.positions = r.positions;
            ts.diameters = r.diameters;
            ts.phi = r.phi;
            ts.force = r.force_magnitude;
            ts.energy = host_c_.U;
            ts.max_min_dist = r.max_min_dist;
            trace->push_back(std::move(ts));
        }
        if (observer) {
            Observation ob{last, r.phi, r.force_magnitude, host_c_.U, r.max_min_dist};
            observer(ob, capture_positions ? &r.positions : nullptr);
        }
    }
}

}  // namespace rcpg
