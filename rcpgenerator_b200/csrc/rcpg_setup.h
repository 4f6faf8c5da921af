// Run setup of run_packing_observed on the host (no CUDA): input checks,
// wall normalisation, the start-phi rescale, schedule constants and the
// initial controller state. Shared by the CUDA engine and the host emulation.
#pragma once

#include <cstddef>
#include <cstdint>
#include <vector>

#include "rcpg_schedule.h"

namespace rcpg {

// Inputs of run_packing_observed (rcp_generator.hpp:18-33, :102-123).
struct EngineInput {
    std::uint64_t N = 0;
    int ndim = 0;
    std::vector<double> positions;  // [N*ndim]
    std::vector<double> diameters;  // [N]
    std::vector<double> box;        // [ndim] or empty
    std::vector<std::int8_t> walls; // [ndim] or empty
    std::uint32_t neighbor_max = 0;
    std::uint32_t seed = 0;
    bool fix_height = false;
    // PackingRunOptions
    std::uint64_t max_steps = 0;
    bool has_mu_override = false;
    double mu_override = 0.0;
    bool fix_diameter = false;
    bool has_target_phi = false;
    double target_phi = 0.0;
    std::uint64_t reorder_interval = 2000;
    bool has_initial_phi_target = false;
    double initial_phi_target = 0.55;
    // engine selection
    bool exact = false;          // host-controlled steps, one-thread reduction order
    int device = 0;
    int graph_steps = 32;        // steps per captured graph (graph mode)
    // pair arithmetic (graph mode): 0 = FP64 throughout; 1 = mixed, FP32 pair
    // terms until the first step whose max overlap falls below mixed_switch
    int pair_precision = 0;
    double mixed_switch = 1e-5;
    // length of the growth rung (mu_flag = 1); 0 = the reference's deadline
    std::uint64_t growth_steps = 0;
};

struct RunSetup {
    std::uint64_t N = 0;
    int ndim = 0;
    Controller c{};                    // state before step 1
    std::vector<double> x;             // [N*ndim] positions after setup scaling
    std::vector<double> D0;            // [N] diameters after the start-phi rescale
    std::vector<std::uint32_t> caps;   // [N] half-row capacity (compute_pair_layout)
    std::vector<std::int8_t> walls;    // normalised walls
    std::uint32_t neighbor_max = 0;    // resolved neighbor_max
};

// Throws std::invalid_argument / std::runtime_error with the reference's messages.
// The input checks of the run set-up that need no GPU: sizes, box and walls
// lengths (std::invalid_argument / std::runtime_error with the reference's texts).
void check_run_input(const EngineInput& in);
RunSetup prepare_run(const EngineInput& in);

// Per-row capacity of the reference pair layout (ENG:4527-4566).
std::vector<std::uint32_t> pair_caps(const std::vector<double>& D, int ndim,
                                     std::uint32_t neighbor_max);

// scale_diameters_nd (rcp_generator.cpp:1162-1196).
std::vector<double> scale_diameters_nd(const std::vector<double>& D, double phi_target,
                                       const std::vector<double>& box, std::size_t ndim,
                                       bool fix_height, double* factor_out);
double sphere_volume(double r, std::size_t ndim);

}  // namespace rcpg
