// Host driver of one packing on one GPU.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <functional>
#include <stdexcept>
#include <string>
#include <vector>

#include "rcpg_device.h"
#include "rcpg_setup.h"

namespace rcpg {

struct Observation {
    std::uint64_t step;
    double phi, force_magnitude, energy, max_min_dist;
};

// PackingResult (rcp_generator.hpp:35-90) minus the research-only fields.
struct EngineResult {
    std::vector<double> positions;  // [N*ndim]
    std::vector<double> diameters;
    std::vector<double> box;
    std::vector<std::int8_t> walls;
    std::vector<double> phi_history, force_history, energy_history, max_overlap_history,
        mu_history, alpha_history;
    std::vector<std::int8_t> mu_flag_history;
    std::uint64_t steps = 0;
    double phi = 0.0, max_min_dist = 0.0, force_magnitude = 0.0;
    std::vector<std::uint64_t> particle_origin;
    // engine statistics
    std::uint64_t builds = 0;
    std::uint32_t row_capacity = 0;
    // mixed precision: step after which the pair terms were FP64 (0: never
    // switched), and the relative error of the final state's energy sum and
    // forces with FP32 pair terms against FP64 ones (NaN when not mixed)
    std::uint64_t fp64_switch_step = 0;
    double pair_energy_rel_error = 0.0, pair_force_rel_error = 0.0;
};

struct TraceSample {
    std::uint64_t step;
    std::vector<double> positions;  // [N*ndim]
    std::vector<double> diameters;
    double phi, force, energy, max_min_dist;
};

using ObserverFn = std::function<void(const Observation&, const std::vector<double>* positions)>;

struct DevCtl;
// pinned host copies of the control block, recycled across engines
// Stream-ordered device allocation from this library's pool of the current
// device (freed memory stays reserved for the next engine; free with cudaFreeAsync).
cudaError_t pool_alloc_async(void** p, std::size_t bytes, cudaStream_t st);
DevCtl* pinned_ctl_acquire();
void pinned_ctl_release(DevCtl* p);

// Size classes of the cell grids (one grid per doubling of D0 when
// max/min D0 > 2.5, else one grid) into h.nclass, class_d0, class_d0max.
void set_size_classes(const std::vector<double>& D0, DevCtl& h);

class EngineError : public std::runtime_error {
   public:
    EngineError(int code, const std::string& msg) : std::runtime_error(msg), code_(code) {}
    int code() const { return code_; }

   private:
    int code_;
};

class Engine {
   public:
    explicit Engine(const EngineInput& in, cudaStream_t stream = nullptr);
    ~Engine();
    Engine(const Engine&) = delete;
    Engine& operator=(const Engine&) = delete;

    // Advance by at most max_new_steps steps (0 = to completion). Returns
    // true once the run is finished (converged or step cap).
    bool advance(std::uint64_t max_new_steps);
    // Run to completion with optional observation / trajectory capture.
    void run(std::uint64_t progress_interval, bool capture_positions,
             std::uint64_t trajectory_interval, const ObserverFn& observer,
             std::vector<TraceSample>* trace);
    EngineResult result();
    std::uint64_t steps_done() const { return host_c_.hist_filled; }
    bool finished() const { return finished_; }
    cudaStream_t stream() const { return st_; }
    std::uint64_t N() const { return N_; }
    int ndim() const { return ndim_; }
    // Kernel launches issued so far by this engine (the graph counts per node).
    std::uint64_t launches() const { return launches_; }
    std::uint64_t builds();
    // Times `reps` back-to-back launches of the pair-force kernel on the
    // current state (CUDA events on the engine stream); returns the average
    // duration and the kernel's algorithmic bytes per launch.
    void profile_pair_kernel(std::uint32_t reps, double* avg_ms, double* alg_bytes,
                             double* mean_row);
    // The same for the neighbour build's search (graph mode: the tiled build
    // with the step's forces fused), each launch after the binning stages of a
    // full rebuild of the current state and a cold L2. Leaves the rows rebuilt
    // for the current positions; the control block is restored.
    void profile_build_kernel(std::uint32_t reps, double* avg_ms, double* alg_bytes);
    // Mixed precision: the final state's forces evaluated with FP32 and with
    // FP64 pair terms on the same rows; relative difference of the pair
    // energy sum and max |F32 - F64| / max |F64|. Leaves the state unchanged.
    void pair_precision_error(double* energy_rel, double* force_rel);
    // Waits for the device by sleeping on a blocking event instead of spinning
    // (for many engines driven by more host threads than cores: a batch).
    void set_blocking_sync(bool on);

   private:
    void setup_host(const EngineInput& in);
    void alloc_device();
    void free_device();
    void upload_initial();
    void ensure_row_capacity(std::uint32_t need);
    void push_ctl();
    void pull_ctl();
    void publish_step_params();
    void do_reorder_and_rebuild();
    void do_target_lock(std::uint64_t step);
    void forces_and_reduce(bool exact_reduce);
    void finish_step_host();
    bool step_host();
    bool advance_graph(std::uint64_t max_new_steps);
    void capture_graph();
    // one step of the step graph: gate, conditional build, pair-kernel switch,
    // controller, ADAM (kernels run only where the step needs them)
    void capture_step();
    template <typename Body>
    void add_conditional(int type, unsigned long long handle, unsigned size, Body body);
    std::uint64_t kernels_per_build() const;
    void destroy_graph();
    void handle_overflow_and_resume();
    void after_stop();
    void observe(std::uint64_t step, bool capture, const ObserverFn& observer,
                 std::vector<TraceSample>* trace);
    void download_histories();
    // particle records [N*P] and particle_origin (optional) of the current
    // state in the reference's order (graph mode stores them in cell order)
    void download_particles(std::vector<double>& pos, std::vector<std::uint64_t>* origin);
    void check(cudaError_t e, const char* what);

    // configuration
    std::uint64_t N_ = 0;
    int ndim_ = 0;
    int P_ = 0;
    bool exact_ = false;
    bool mixed_ = false;          // FP32 pair terms until the max overlap falls below mixed_switch_
    double mixed_switch_ = 1e-5;
    int graph_steps_ = 32;
    int device_ = 0;
    cudaStream_t st_ = nullptr;
    bool own_stream_ = false;
    std::uint32_t neighbor_max_ = 0;

    // host copies
    std::vector<double> x0_;          // initial positions (after setup scaling)
    std::vector<double> D0_;          // D0 after setup
    std::vector<std::uint32_t> caps_;
    std::vector<std::int8_t> walls_;
    Controller host_c_{};
    DevCtl hctl_{};
    std::vector<double> h_phi_, h_force_, h_energy_, h_maxov_, h_mu_, h_alpha_;
    std::vector<std::int8_t> h_muflag_;
    Histories hh_{};
    std::uint64_t hist_size_ = 0;
    bool histories_on_device_ = false;
    bool finished_ = false;
    bool adam_pending_ = false;   // exact mode: ADAM pass of the last finished step not yet applied
    std::uint64_t launches_ = 0;
    double initial_U_ = 0.0, initial_maxov_ = 0.0;

    // device
    DevArrays a_{};
    void* d_block_ = nullptr;
    std::vector<void*> allocs_;
    cudaGraphExec_t graph_exec_ = nullptr;
    cudaGraph_t graph_ = nullptr;
    std::uint64_t graph_nodes_per_step_ = 0;
    cudaStream_t body_st_ = nullptr;  // captures the bodies of the step graph's conditional nodes
    std::uint32_t* pinned_ = nullptr;
    DevCtl* hctl_pinned_ = nullptr;
    cudaEvent_t sync_ev_ = nullptr;  // blocking-sync event (set_blocking_sync)
};

}  // namespace rcpg
