// Persistent batch engine (rcpg_batch.cu): many independent packings of one
// ndim run by one kernel, each thread block taking whole packings from a queue.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "rcpg_device.h"
#include "rcpg_engine.h"
#include "rcpg_setup.h"

namespace rcpg {

// One packing of a batch: where its arrays start in the concatenated buffers.
struct BatchInst {
    std::uint64_t off;       // first particle
    std::uint64_t nbr_off;   // first row entry (S*N entries, column-major in the packing)
    std::uint64_t cell_off;  // first cell counter (C_alloc + 1 entries)
    std::uint64_t hist_off;  // first history entry (step_cap + 1 entries)
    std::uint32_t N, S, C_alloc;
    // 0 not started, 1 running, 2 finished, 3 rows outgrew S (run again with a
    // larger S), 4 half row beyond the reference capacity, 5 needs a target-phi lock
    std::uint32_t status;
};

// The concatenated device arrays of one launch (same layouts as DevArrays).
struct BatchArrays {
    double *pos, *spos, *F, *m, *v, *x_last, *pos_tmp, *vec_tmp;
    std::uint32_t *nbr, *nbr_cnt, *caps, *cell_of, *cell_rank, *cell_list, *work, *cell_count, *cell_start;
    std::uint64_t *origin, *u64_tmp, *keys0, *keys1;
    std::uint32_t *vals0, *vals1;
    double *h_phi, *h_force, *h_energy, *h_maxov, *h_mu, *h_alpha;
    std::int8_t* h_muflag;
    DevCtl* ctl;              // [instances]
    BatchInst* inst;          // [instances]
    std::uint32_t* active;    // indices of the instances this launch advances
    std::uint32_t nactive;
    std::uint32_t* queue;     // next entry of `active` to take
};

void launch_batch(const BatchArrays& B, int ndim, std::uint32_t chunk, int mixed, int device,
                  int blocks_per_sm, cudaStream_t st);

// Outcome of one packing of run_batch_persistent.
struct BatchOutcome {
    int code = 0;             // 0 ok, else an RCPG_* error code
    std::string message;
    EngineResult result;
    std::uint64_t N = 0;
    int ndim = 0;
};

// Runs every packing to completion in persistent launches of at most `chunk`
// steps per packing, with at most `blocks_per_sm` resident blocks per SM
// (0: the autotuned value of each ndim, tune_batch). All share the run
// options of `ins[k]` (graph engine; packings that can reach a target-phi
// lock are reported as unsupported).
std::vector<BatchOutcome> run_batch_persistent(const std::vector<EngineInput>& ins, std::uint32_t chunk,
                                               int blocks_per_sm);

// Launch-shape autotuner of the persistent batch kernel for one (device,
// ndim, pair precision): the same synthetic batch -- two packings per SM of
// kTunePackingN particles, uniform positions, mono diameters, capped at
// kTuneSteps steps -- runs at 1 and at 2 resident blocks per SM, and the
// faster (packing-steps per second) is kept for the process. A result does
// not depend on the launch shape (each packing runs in one block of fixed
// size), so the choice only moves time.
struct BatchTuning {
    int blocks_per_sm = 1;
    double steps_per_s[2] = {0.0, 0.0};  // at 1 and 2 blocks per SM
};
BatchTuning tune_batch(int ndim, int device, bool mixed);

// Work of one build step of a packing in the persistent kernel, in candidate
// tests (N x 3^ndim x members per cell): the batch sends the packings above a
// budget to engines on streams, which spread one packing over the GPU.
inline double batch_cost(std::uint64_t N, int ndim) {
    double c = static_cast<double>(N);
    for (int d = 0; d < ndim; ++d) c *= 3.0;
    return c;
}

}  // namespace rcpg
