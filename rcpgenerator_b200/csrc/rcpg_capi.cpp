// extern "C" entry points declared in include/rcpg.h.
#include "../../include/rcpg.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <exception>
#include <new>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "rcpg_batch.h"
#include "rcpg_engine.h"
#include "rcpg_init.h"
#include "rcpg_setup.h"

using rcpg::DevArrays;
using rcpg::DevCtl;

struct rcpg_engine {
    rcpg::Engine* eng;
};

namespace {

void put_err(char* err, std::size_t errlen, const std::string& msg) {
    if (err && errlen) std::snprintf(err, errlen, "%s", msg.c_str());
}

int32_t fail(char* err, std::size_t errlen, int32_t code, const std::string& msg) {
    put_err(err, errlen, msg);
    return code;
}

int32_t classify(const std::exception& e) {
    if (auto* ee = dynamic_cast<const rcpg::EngineError*>(&e)) {
        if (ee->code() == -EINVAL) return RCPG_EINVAL;
        if (ee->code() == -ENOSPC) return RCPG_ERUNTIME;
        if (ee->code() == -2) return RCPG_ECUDA;
        return RCPG_ERUNTIME;
    }
    if (dynamic_cast<const std::invalid_argument*>(&e)) return RCPG_EINVAL;
    return RCPG_ERUNTIME;
}

bool have_device(char* err, std::size_t errlen) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) {
        cudaGetLastError();
        put_err(err, errlen, "rcpgenerator_b200: no CUDA device available (this engine has no CPU path)");
        return false;
    }
    return true;
}

rcpg::EngineInput make_input(const rcpg_packing_input* in, const rcpg_run_options* opt) {
    rcpg::EngineInput e;
    e.N = in->N;
    e.ndim = in->ndim;
    if (!in->positions || !in->diameters)
        throw rcpg::EngineError(-EINVAL, "rcpgenerator_b200: positions and diameters are required");
    e.positions.assign(in->positions, in->positions + in->N * static_cast<std::uint64_t>(in->ndim));
    e.diameters.assign(in->diameters, in->diameters + in->N);
    if (in->box && in->box_len > 0) e.box.assign(in->box, in->box + in->box_len);
    if (in->walls && in->walls_len > 0) e.walls.assign(in->walls, in->walls + in->walls_len);
    e.neighbor_max = in->neighbor_max;
    e.seed = in->seed;
    e.fix_height = in->fix_height != 0;
    rcpg_run_options o;
    if (opt) o = *opt;
    else rcpg_default_options(&o);
    e.max_steps = o.max_steps;
    e.has_mu_override = o.has_mu_override != 0;
    e.mu_override = o.mu_override;
    e.fix_diameter = o.fix_diameter != 0;
    e.has_target_phi = o.has_target_phi != 0;
    e.target_phi = o.target_phi;
    e.reorder_interval = o.reorder_interval;
    e.has_initial_phi_target = o.has_initial_phi_target != 0;
    e.initial_phi_target = o.initial_phi_target;
    e.growth_steps = o.growth_steps;
    e.exact = o.exact != 0;
    e.device = o.device;
    e.graph_steps = o.graph_steps;
    e.pair_precision = o.pair_precision;
    e.mixed_switch = o.mixed_switch > 0.0 ? o.mixed_switch : 1e-5;
    return e;
}

template <typename T>
T* dup(const std::vector<T>& v) {
    T* p = static_cast<T*>(std::malloc(v.size() * sizeof(T) + 1));
    if (!p) throw std::bad_alloc();
    if (!v.empty()) std::memcpy(p, v.data(), v.size() * sizeof(T));
    return p;
}

rcpg_result* make_result(const rcpg::EngineResult& r, std::uint64_t N, int ndim,
                         const std::vector<rcpg::TraceSample>* trace, bool with_positions,
                         std::uint64_t launches) {
    rcpg_result* out = static_cast<rcpg_result*>(std::calloc(1, sizeof(rcpg_result)));
    if (!out) throw std::bad_alloc();
    out->N = N;
    out->ndim = ndim;
    out->steps = r.steps;
    out->phi = r.phi;
    out->max_min_dist = r.max_min_dist;
    out->force_magnitude = r.force_magnitude;
    out->positions = dup(r.positions);
    out->diameters = dup(r.diameters);
    out->box = dup(r.box);
    out->walls = dup(r.walls);
    out->phi_history = dup(r.phi_history);
    out->force_history = dup(r.force_history);
    out->energy_history = dup(r.energy_history);
    out->max_overlap_history = dup(r.max_overlap_history);
    out->mu_history = dup(r.mu_history);
    out->alpha_history = dup(r.alpha_history);
    out->mu_flag_history = dup(r.mu_flag_history);
    out->particle_origin = dup(r.particle_origin);
    out->pair_builds = r.builds;
    out->row_capacity = r.row_capacity;
    out->kernel_launches = launches;
    out->fp64_switch_step = r.fp64_switch_step;
    out->pair_energy_rel_error = r.pair_energy_rel_error;
    out->pair_force_rel_error = r.pair_force_rel_error;
    if (trace && !trace->empty()) {
        const std::size_t T = trace->size();
        out->trace_len = T;
        std::vector<std::uint64_t> steps(T);
        std::vector<double> ph(T), fo(T), en(T), mm(T);
        std::vector<double> pos, dia;
        for (std::size_t k = 0; k < T; ++k) {
            const auto& s = (*trace)[k];
            steps[k] = s.step;
            ph[k] = s.phi;
            fo[k] = s.force;
            en[k] = s.energy;
            mm[k] = s.max_min_dist;
            if (with_positions) {
                pos.insert(pos.end(), s.positions.begin(), s.positions.end());
                dia.insert(dia.end(), s.diameters.begin(), s.diameters.end());
            }
        }
        out->trace_steps = dup(steps);
        out->trace_phi = dup(ph);
        out->trace_force = dup(fo);
        out->trace_energy = dup(en);
        out->trace_max_min_dist = dup(mm);
        if (with_positions) {
            out->trace_positions = dup(pos);
            out->trace_diameters = dup(dia);
        }
    }
    return out;
}

// Scratch buffers of one stand-alone kernel call (stream-ordered).
struct Scratch {
    cudaStream_t st;
    std::vector<void*> ptrs;
    explicit Scratch(cudaStream_t s) : st(s) {}
    void* get(std::size_t bytes) {
        void* p = nullptr;
        if (rcpg::pool_alloc_async(&p, bytes, st) != cudaSuccess)
            throw rcpg::EngineError(-2, "rcpgenerator_b200: device allocation failed");
        ptrs.push_back(p);
        return p;
    }
    ~Scratch() {
        for (void* p : ptrs) cudaFreeAsync(p, st);
    }
};

void geometry_from(DevCtl& h, int ndim, const double* box, const int8_t* walls) {
    rcpg::Geometry& g = h.g;
    g.ndim = ndim;
    g.circle_k = (walls && walls[0] < 0) ? -walls[0] : 0;
    g.any_flat_wall = 0;
    for (int d = 0; d < ndim; ++d) {
        g.walls[d] = walls ? walls[d] : 0;
        if (g.walls[d] == 1) g.any_flat_wall = 1;
        g.box[d] = box ? box[d] : 1.0;
        g.inv_box[d] = 1.0 / g.box[d];
    }
}

void cuda_ok(cudaError_t e, const char* what) {
    if (e != cudaSuccess)
        throw rcpg::EngineError(-2, std::string("rcpgenerator_b200: CUDA error in ") + what + ": " +
                                        cudaGetErrorString(e));
}

}  // namespace

extern "C" {

const char* rcpg_version(void) { return "rcpgenerator_b200 0.1.0 (sm_100a)"; }

int32_t rcpg_abi_version(void) { return RCPG_ABI_VERSION; }

int32_t rcpg_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

void rcpg_default_options(rcpg_run_options* opt) {
    if (!opt) return;
    std::memset(opt, 0, sizeof(*opt));
    opt->reorder_interval = 2000;
    opt->initial_phi_target = 0.55;
    opt->graph_steps = 32;
    opt->pair_precision = 0;
    opt->mixed_switch = 1e-5;
}

int32_t rcpg_run_packing(const rcpg_packing_input* in, const rcpg_run_options* opt,
                         uint64_t progress_interval, int32_t capture_positions,
                         uint64_t trajectory_interval, rcpg_observer_fn observer, void* user,
                         rcpg_result** out, char* err, size_t errlen) {
    if (!in || !out) return fail(err, errlen, RCPG_EINVAL, "rcpgenerator_b200: null argument");
    *out = nullptr;
    try {
        // argument errors first (they need no GPU), then the device
        const rcpg::EngineInput ei = make_input(in, opt);
        rcpg::check_run_input(ei);
        if (!have_device(err, errlen)) return RCPG_ECUDA;
        rcpg::Engine eng(ei);
        std::vector<rcpg::TraceSample> trace;
        rcpg::ObserverFn fn;
        if (observer) {
            fn = [&](const rcpg::Observation& o, const std::vector<double>* pos) {
                rcpg_observation ob{o.step, o.phi, o.force_magnitude, o.energy, o.max_min_dist};
                observer(&ob, pos ? pos->data() : nullptr, user);
            };
        }
        eng.run(progress_interval, capture_positions != 0, trajectory_interval, fn, &trace);
        const rcpg::EngineResult r = eng.result();
        *out = make_result(r, eng.N(), eng.ndim(), &trace, capture_positions != 0, eng.launches());
        return RCPG_OK;
    } catch (const std::exception& e) {
        return fail(err, errlen, classify(e), e.what());
    }
}

namespace {

int32_t run_batch_impl(const rcpg_packing_input* inputs, uint64_t count, const rcpg_run_options* opt,
                       const uint64_t* growth_steps, int32_t concurrency, rcpg_result** results,
                       int32_t* status, char* err, size_t errlen) {
    if ((!inputs && count) || (!results && count))
        return fail(err, errlen, RCPG_EINVAL, "rcpgenerator_b200: null argument");
    for (uint64_t k = 0; k < count; ++k) {
        results[k] = nullptr;
        if (status) status[k] = RCPG_OK;
    }
    if (count == 0) return RCPG_OK;
    if (!have_device(err, errlen)) return RCPG_ECUDA;
    rcpg_run_options o;
    if (opt) o = *opt;
    else rcpg_default_options(&o);
    std::mutex mu;
    int32_t first_code = RCPG_OK;
    uint64_t first_index = 0;
    std::string first_msg;
    auto record = [&](uint64_t k, int32_t code, const std::string& msg) {
        if (status) status[k] = code;
        std::lock_guard<std::mutex> lk(mu);
        if (first_code == RCPG_OK || k < first_index) {
            first_code = code;
            first_index = k;
            first_msg = msg;
        }
    };
    auto input_of = [&](uint64_t k) {
        rcpg::EngineInput e = make_input(&inputs[k], &o);
        if (growth_steps) e.growth_steps = growth_steps[k];
        return e;
    };
    // concurrency 0: the cheap packings (graph engine, no target-phi lock, a
    // build step below kPersistentBudget candidate tests) go to the persistent
    // kernel, which runs on its own host thread with one block per SM, the
    // others to 32 engines on streams at the same time; concurrency < 0: every
    // eligible packing to the persistent kernel
    constexpr double kPersistentBudget = 3e4;
    std::vector<uint64_t> on_streams, persistent;
    for (uint64_t k = 0; k < count; ++k) {
        const bool eligible = concurrency <= 0 && !o.exact && !o.has_target_phi;
        // the persistent kernel keeps one cell grid: wide size distributions
        // (the engines' size-class grids) stay on the streams in the automatic split
        double dlo = 0.0, dhi = 0.0;
        if (inputs[k].diameters && inputs[k].N) {
            dlo = dhi = inputs[k].diameters[0];
            for (uint64_t i = 1; i < inputs[k].N; ++i) {
                dlo = std::min(dlo, inputs[k].diameters[i]);
                dhi = std::max(dhi, inputs[k].diameters[i]);
            }
        }
        const bool narrow = dlo > 0.0 && dhi <= 2.5 * dlo;
        const bool ok = eligible && (concurrency < 0 ||
                                     (narrow && rcpg::batch_cost(inputs[k].N, inputs[k].ndim) <= kPersistentBudget));
        (ok ? persistent : on_streams).push_back(k);
    }
    // the stream workers take the most expensive packings first (longest
    // processing time first), so that no large packing starts last and runs
    // alone at the end; results keep their input slots
    std::stable_sort(on_streams.begin(), on_streams.end(), [&](uint64_t x, uint64_t y) {
        return rcpg::batch_cost(inputs[x].N, inputs[x].ndim) > rcpg::batch_cost(inputs[y].N, inputs[y].ndim);
    });
    std::thread pthread;
    if (!persistent.empty()) {
        pthread = std::thread([&]() {
            try {
                std::vector<rcpg::EngineInput> ins;
                ins.reserve(persistent.size());
                for (uint64_t k : persistent) ins.push_back(input_of(k));
                const std::vector<rcpg::BatchOutcome> res =
                    rcpg::run_batch_persistent(ins, 2048u, on_streams.empty() ? 0 : 1);
                for (std::size_t q = 0; q < persistent.size(); ++q) {
                    const uint64_t k = persistent[q];
                    const rcpg::BatchOutcome& b = res[q];
                    if (b.code == 0) {
                        results[k] = make_result(b.result, b.N, b.ndim, nullptr, false, 0);
                    } else {
                        record(k, b.code == -22 ? RCPG_EINVAL : (b.code == -2 ? RCPG_ECUDA : RCPG_ERUNTIME),
                               b.message);
                    }
                }
            } catch (const std::exception& e) {
                for (uint64_t k : persistent) record(k, classify(e), e.what());
            }
        });
    }
    const uint64_t ns = on_streams.size();
    const uint64_t nthreads = ns ? std::max<uint64_t>(1, std::min<uint64_t>(ns, concurrency > 0 ? concurrency : 32)) : 0;
    std::atomic<uint64_t> next{0};
    auto worker = [&]() {
        if (cudaSetDevice(o.device) != cudaSuccess) {
            cudaGetLastError();
            for (uint64_t q; (q = next.fetch_add(1)) < ns;) record(on_streams[q], RCPG_ECUDA, "rcpgenerator_b200: cudaSetDevice failed");
            return;
        }
        cudaStream_t st = nullptr;
        if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
            cudaGetLastError();
            for (uint64_t q; (q = next.fetch_add(1)) < ns;) record(on_streams[q], RCPG_ECUDA, "rcpgenerator_b200: cudaStreamCreate failed");
            return;
        }
        for (uint64_t q; (q = next.fetch_add(1)) < ns;) {
            const uint64_t k = on_streams[q];
            try {
                rcpg::Engine eng(input_of(k), st);
                eng.set_blocking_sync(true);  // many host threads: sleep while the GPU works
                eng.run(0, false, 0, rcpg::ObserverFn(), nullptr);
                const rcpg::EngineResult r = eng.result();
                results[k] = make_result(r, eng.N(), eng.ndim(), nullptr, false, eng.launches());
            } catch (const std::exception& e) {
                record(k, classify(e), e.what());
            }
        }
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
    };
    std::vector<std::thread> pool;
    pool.reserve(nthreads);
    for (uint64_t t = 0; t < nthreads; ++t) pool.emplace_back(worker);
    for (auto& t : pool) t.join();
    if (pthread.joinable()) pthread.join();
    if (first_code != RCPG_OK)
        return fail(err, errlen, first_code, "packing " + std::to_string(first_index) + ": " + first_msg);
    return RCPG_OK;
}

}  // namespace

int32_t rcpg_run_batch(const rcpg_packing_input* inputs, uint64_t count, const rcpg_run_options* opt,
                       int32_t concurrency, rcpg_result** results, int32_t* status, char* err,
                       size_t errlen) {
    return run_batch_impl(inputs, count, opt, nullptr, concurrency, results, status, err, errlen);
}

int32_t rcpg_run_batch_growth(const rcpg_packing_input* inputs, uint64_t count, const rcpg_run_options* opt,
                              const uint64_t* growth_steps, int32_t concurrency, rcpg_result** results,
                              int32_t* status, char* err, size_t errlen) {
    return run_batch_impl(inputs, count, opt, growth_steps, concurrency, results, status, err, errlen);
}

int32_t rcpg_batch_tuning(int32_t ndim, int32_t device, int32_t pair_precision, int32_t* blocks_per_sm,
                          double* steps_per_s, char* err, size_t errlen) {
    if (ndim < 2 || ndim > rcpg::kMaxDim)
        return fail(err, errlen, RCPG_EINVAL, "rcpgenerator_b200: Ndim must be in [2, 8]");
    if (!have_device(err, errlen)) return RCPG_ECUDA;
    try {
        cuda_ok(cudaSetDevice(device), "cudaSetDevice");
        const rcpg::BatchTuning t = rcpg::tune_batch(ndim, device, pair_precision == 1);
        if (blocks_per_sm) *blocks_per_sm = t.blocks_per_sm;
        if (steps_per_s) {
            steps_per_s[0] = t.steps_per_s[0];
            steps_per_s[1] = t.steps_per_s[1];
        }
        return RCPG_OK;
    } catch (const std::exception& e) {
        return fail(err, errlen, classify(e), e.what());
    }
}

void rcpg_result_free(rcpg_result* r) {
    if (!r) return;
    void* fields[] = {r->positions,       r->diameters,        r->box,           r->walls,
                      r->phi_history,     r->force_history,    r->energy_history, r->max_overlap_history,
                      r->mu_history,      r->alpha_history,    r->mu_flag_history, r->particle_origin,
                      r->trace_steps,     r->trace_positions,  r->trace_diameters, r->trace_phi,
                      r->trace_force,     r->trace_energy,     r->trace_max_min_dist};
    for (void* p : fields) std::free(p);
    std::free(r);
}

int32_t rcpg_engine_create(const rcpg_packing_input* in, const rcpg_run_options* opt,
                           void* stream, rcpg_engine** out, char* err, size_t errlen) {
    if (!in || !out) return fail(err, errlen, RCPG_EINVAL, "rcpgenerator_b200: null argument");
    *out = nullptr;
    if (!have_device(err, errlen)) return RCPG_ECUDA;
    try {
        rcpg::Engine* e = new rcpg::Engine(make_input(in, opt), static_cast<cudaStream_t>(stream));
        *out = new rcpg_engine{e};
        return RCPG_OK;
    } catch (const std::exception& e) {
        return fail(err, errlen, classify(e), e.what());
    }
}

int32_t rcpg_engine_advance(rcpg_engine* e, uint64_t max_new_steps, int32_t* finished, char* err,
                            size_t errlen) {
    if (!e) return fail(err, errlen, RCPG_EINVAL, "rcpgenerator_b200: null engine");
    try {
        const bool f = e->eng->advance(max_new_steps);
        if (finished) *finished = f ? 1 : 0;
        return RCPG_OK;
    } catch (const std::exception& ex) {
        return fail(err, errlen, classify(ex), ex.what());
    }
}

uint64_t rcpg_engine_steps(const rcpg_engine* e) { return e ? e->eng->steps_done() : 0; }

uint64_t rcpg_engine_kernel_launches(const rcpg_engine* e) { return e ? e->eng->launches() : 0; }

int32_t rcpg_engine_result(rcpg_engine* e, rcpg_result** out, char* err, size_t errlen) {
    if (!e || !out) return fail(err, errlen, RCPG_EINVAL, "rcpgenerator_b200: null argument");
    try {
        const rcpg::EngineResult r = e->eng->result();
        *out = make_result(r, e->eng->N(), e->eng->ndim(), nullptr, false, e->eng->launches());
        return RCPG_OK;
    } catch (const std::exception& ex) {
        return fail(err, errlen, classify(ex), ex.what());
    }
}

int32_t rcpg_engine_profile_pair_kernel(rcpg_engine* e, uint32_t reps, double* avg_ms,
                                        double* alg_bytes, double* mean_row, char* err,
                                        size_t errlen) {
    if (!e || !avg_ms || !alg_bytes || !mean_row)
        return fail(err, errlen, RCPG_EINVAL, "rcpgenerator_b200: null argument");
    try {
        e->eng->profile_pair_kernel(reps, avg_ms, alg_bytes, mean_row);
        return RCPG_OK;
    } catch (const std::exception& ex) {
        return fail(err, errlen, classify(ex), ex.what());
    }
}

int32_t rcpg_engine_profile_build_kernel(rcpg_engine* e, uint32_t reps, double* avg_ms,
                                         double* alg_bytes, char* err, size_t errlen) {
    if (!e || !avg_ms || !alg_bytes)
        return fail(err, errlen, RCPG_EINVAL, "rcpgenerator_b200: null argument");
    try {
        e->eng->profile_build_kernel(reps, avg_ms, alg_bytes);
        return RCPG_OK;
    } catch (const std::exception& ex) {
        return fail(err, errlen, classify(ex), ex.what());
    }
}

void rcpg_engine_destroy(rcpg_engine* e) {
    if (!e) return;
    delete e->eng;
    delete e;
}

double rcpg_t_shell(const double* D, uint64_t N) {
    if (!D || N == 0) return 0.0;
    std::vector<double> s(D, D + N);
    const double dmin = *std::min_element(s.begin(), s.end());
    const double dmax = *std::max_element(s.begin(), s.end());
    std::nth_element(s.begin(), s.begin() + N / 2, s.end());
    return rcpg::shell_of(dmin, s[N / 2], dmax);
}

int32_t rcpg_pairs_full(uint64_t N, int32_t ndim, const double* x_dev, const double* D_dev,
                        const double* box, const int8_t* walls, double t_shell,
                        uint32_t row_capacity, uint32_t* nbr_dev, uint32_t* cnt_dev,
                        uint32_t* row_need_out, void* stream, char* err, size_t errlen) {
    if (N == 0 || ndim < 2 || ndim > rcpg::kMaxDim || !x_dev || !D_dev || !nbr_dev || !cnt_dev ||
        row_capacity == 0)
        return fail(err, errlen, RCPG_EINVAL, "rcpgenerator_b200: bad arguments to rcpg_pairs_full");
    if (!have_device(err, errlen)) return RCPG_ECUDA;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    try {
        const int P = rcpg::pos_stride(ndim);
        // largest diameter and the cell-grid capacity need D on the host
        std::vector<double> D(N);
        cuda_ok(cudaMemcpyAsync(D.data(), D_dev, N * 8, cudaMemcpyDeviceToHost, st), "D2H D");
        cuda_ok(cudaStreamSynchronize(st), "sync");
        const double Dmax = *std::max_element(D.begin(), D.end());
        Scratch sc(st);
        DevArrays a{};
        a.N = N;
        a.ndim = ndim;
        a.P = P;
        a.pos = static_cast<double*>(sc.get(N * P * 8));
        a.spos = static_cast<double*>(sc.get(N * P * 8));
        a.x_last = static_cast<double*>(sc.get(N * ndim * 8));
        // the build writes rows in cell order into scratch, then they are
        // transposed into the caller's particle-ordered buffers
        a.nbr = static_cast<std::uint32_t*>(sc.get(static_cast<std::size_t>(row_capacity) * N * 4));
        a.nbr_cnt = static_cast<std::uint32_t*>(sc.get(N * 4));
        a.S = row_capacity;
        a.sorted_rows = 1;  // the reference's row order
        a.caps = static_cast<std::uint32_t*>(sc.get(N * 4));
        a.cell_of = static_cast<std::uint32_t*>(sc.get(N * 4));
        a.cell_rank = static_cast<std::uint32_t*>(sc.get(N * 4));
        a.cell_list = static_cast<std::uint32_t*>(sc.get(N * 4));
        a.work = static_cast<std::uint32_t*>(sc.get(N * 4));
        {
            const double cutoff = (Dmax + t_shell) * (1.0 + 1e-6);
            double cells = 1.0;
            for (int d = 0; d < ndim; ++d) cells *= std::max(1.0, std::floor((box ? box[d] : 1.0) / cutoff));
            double cap = std::min(cells + 64.0, 8.0 * static_cast<double>(N) + 1024.0);
            a.C_alloc = static_cast<std::uint32_t>(std::min(cap, 2.0e9));
        }
        a.cell_count = static_cast<std::uint32_t*>(sc.get((a.C_alloc + 1ull) * 4));
        a.cell_start = static_cast<std::uint32_t*>(sc.get((a.C_alloc + 1ull) * 4));
        a.scan_tmp = static_cast<std::uint32_t*>(sc.get(2 * 4096 * 4 + 64));
        a.ctl = static_cast<DevCtl*>(sc.get(sizeof(DevCtl)));
        DevCtl h;
        std::memset(&h, 0, sizeof(h));
        geometry_from(h, ndim, box, walls);
        h.build_kappa = 1.0;
        h.build_t_shell = t_shell;
        h.build_Dmax = Dmax;
        h.rebuild_flag = 1u;
        cuda_ok(cudaMemcpyAsync(a.ctl, &h, sizeof(h), cudaMemcpyHostToDevice, st), "H2D ctl");
        cuda_ok(cudaMemsetAsync(a.caps, 0xFF, N * 4, st), "memset caps");
        rcpg::launch_pack(N, ndim, x_dev, D_dev, a.pos, st);
        rcpg::launch_rebuild(a, st);
        rcpg::launch_rows_to_particle_order(N, a.work, a.nbr, a.nbr_cnt, nbr_dev, cnt_dev, st);
        cuda_ok(cudaMemcpyAsync(&h, a.ctl, sizeof(h), cudaMemcpyDeviceToHost, st), "D2H ctl");
        cuda_ok(cudaStreamSynchronize(st), "sync");
        cuda_ok(cudaGetLastError(), "kernel launch");
        if (row_need_out) *row_need_out = h.row_need;
        if (h.row_need > row_capacity)
            return fail(err, errlen, RCPG_ENOSPC, "rcpgenerator_b200: a neighbour row exceeds row_capacity");
        return RCPG_OK;
    } catch (const std::exception& e) {
        return fail(err, errlen, classify(e), e.what());
    }
}

int32_t rcpg_pairs_forces_scan(uint64_t N, int32_t ndim, const double* x_dev, const double* D_dev,
                               const double* box, const int8_t* walls, double t_shell, double mu,
                               int32_t pair_precision, uint32_t row_capacity, uint32_t* nbr_dev,
                               uint32_t* cnt_dev, uint32_t* row_need_out, double* F_dev,
                               double* scalars, int32_t* fused_out, void* stream, char* err,
                               size_t errlen) {
    if (N == 0 || N > 0xFFFFFFFFull || ndim < 2 || ndim > rcpg::kMaxDim || !x_dev || !D_dev || !nbr_dev ||
        !cnt_dev || !F_dev || row_capacity == 0 || pair_precision < 0 || pair_precision > 3)
        return fail(err, errlen, RCPG_EINVAL, "rcpgenerator_b200: bad arguments to rcpg_pairs_forces_scan");
    // bit 1: the forces of the step's pair kernel on the new rows, also after a build that fused them
    const bool pair_kernel = (pair_precision & 2) != 0;
    pair_precision &= 1;
    if (!have_device(err, errlen)) return RCPG_ECUDA;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    try {
        const int P = rcpg::pos_stride(ndim);
        std::vector<double> D(N);
        cuda_ok(cudaMemcpyAsync(D.data(), D_dev, N * 8, cudaMemcpyDeviceToHost, st), "D2H D");
        cuda_ok(cudaStreamSynchronize(st), "sync");
        const double Dmax = *std::max_element(D.begin(), D.end());
        Scratch sc(st);
        DevArrays a{};
        a.N = N;
        a.ndim = ndim;
        a.P = P;
        // the graph engine's layout: cell-order storage in two buffer sets
        a.permute = 1;
        auto dbl = [&](std::size_t n) { return static_cast<double*>(sc.get(n * 8)); };
        auto u32 = [&](std::size_t n) { return static_cast<std::uint32_t*>(sc.get(n * 4)); };
        auto u64 = [&](std::size_t n) { return static_cast<std::uint64_t*>(sc.get(n * 8)); };
        a.pos = dbl(N * P);
        a.pos_alt = dbl(N * P);
        a.m = dbl(N * ndim);
        a.m_alt = dbl(N * ndim);
        a.v = dbl(N * ndim);
        a.v_alt = dbl(N * ndim);
        a.origin = u64(N);
        a.origin_alt = u64(N);
        a.caps = u32(N);
        a.caps_alt = u32(N);
        a.ref_rank = u32(N);
        a.ref_rank_alt = u32(N);
        a.x_last = dbl(N * ndim);
        a.F = dbl(N * ndim);
        a.nbr = u32(static_cast<std::size_t>(row_capacity) * N);
        a.nbr_cnt = u32(N);
        a.S = row_capacity;
        a.sorted_rows = 0;  // the graph engine's scan order
        a.mixed = pair_precision;
        a.cell_of = u32(N);
        a.cell_rank = u32(N);
        a.cell_list = u32(N);
        a.work = u32(N);
        // the engine's cell grids: one per size class for wide size distributions
        DevCtl cls;
        std::memset(&cls, 0, sizeof(cls));
        rcpg::set_size_classes(D, cls);
        {
            double cells = 0.0;
            for (int k = 0; k < cls.nclass; ++k) {
                const double dmax = cls.nclass > 1 ? cls.class_d0max[k] : Dmax;
                const double cutoff = (dmax + t_shell) * (1.0 + 1e-6);
                double ck = 1.0;
                for (int d = 0; d < ndim; ++d) ck *= std::max(1.0, std::floor((box ? box[d] : 1.0) / cutoff));
                cells += ck;
            }
            double cap = std::min(cells + 64.0, 8.0 * static_cast<double>(N) + 1024.0);
            a.C_alloc = static_cast<std::uint32_t>(std::min(cap, 2.0e9));
        }
        a.cell_count = u32(a.C_alloc + 1ull);
        a.cell_start = u32(a.C_alloc + 1ull);
        a.scan_tmp = u32(2 * 4096 + 16);
        a.block_sums = static_cast<rcpg::ForceSums*>(
            sc.get(std::max<std::size_t>(rcpg::force_blocks(N), 4096) * sizeof(rcpg::ForceSums)));
        a.ctl = static_cast<DevCtl*>(sc.get(sizeof(DevCtl)));
        DevCtl h;
        std::memset(&h, 0, sizeof(h));
        geometry_from(h, ndim, box, walls);
        h.build_kappa = 1.0;
        h.build_t_shell = t_shell;
        h.build_Dmax = Dmax;
        h.force_kappa = 1.0;
        h.force_mu = mu;
        h.rebuild_flag = 1u;
        h.fuse_forces = 1u;
        h.pair_fp32 = static_cast<std::uint32_t>(pair_precision);
        h.nclass = cls.nclass;
        std::memcpy(h.class_d0, cls.class_d0, sizeof(h.class_d0));
        std::memcpy(h.class_d0max, cls.class_d0max, sizeof(h.class_d0max));
        std::vector<std::uint64_t> ident(N);
        for (std::uint64_t i = 0; i < N; ++i) ident[i] = i;
        std::vector<std::uint32_t> ident32(ident.begin(), ident.end());
        cuda_ok(cudaMemcpyAsync(a.ctl, &h, sizeof(h), cudaMemcpyHostToDevice, st), "H2D ctl");
        cuda_ok(cudaMemcpyAsync(a.origin, ident.data(), N * 8, cudaMemcpyHostToDevice, st), "H2D origin");
        cuda_ok(cudaMemcpyAsync(a.ref_rank, ident32.data(), N * 4, cudaMemcpyHostToDevice, st), "H2D rank");
        cuda_ok(cudaMemsetAsync(a.caps, 0xFF, N * 4, st), "memset caps");
        cuda_ok(cudaMemsetAsync(a.m, 0, N * ndim * 8, st), "memset m");
        cuda_ok(cudaMemsetAsync(a.v, 0, N * ndim * 8, st), "memset v");
        rcpg::launch_pack(N, ndim, x_dev, D_dev, a.pos, st);
        rcpg::launch_rebuild(a, st);
        // the forces of the build, or (builds that do not fuse them) of the pair kernel
        DevCtl after;
        cuda_ok(cudaMemcpyAsync(&after, a.ctl, sizeof(after), cudaMemcpyDeviceToHost, st), "D2H ctl");
        cuda_ok(cudaStreamSynchronize(st), "sync");
        if (pair_kernel && after.forces_done)
            cuda_ok(cudaMemsetAsync(&a.ctl->forces_done, 0, sizeof(std::uint32_t), st), "memset forces_done");
        rcpg::launch_forces(a, 0, st);
        rcpg::launch_reduce_fast(a, st);
        // rows, counts and forces back in the caller's particle order
        rcpg::launch_cell_order_to_particle_order(a, nbr_dev, cnt_dev, F_dev, st);
        cuda_ok(cudaMemcpyAsync(&h, a.ctl, sizeof(h), cudaMemcpyDeviceToHost, st), "D2H ctl");
        cuda_ok(cudaStreamSynchronize(st), "sync");
        cuda_ok(cudaGetLastError(), "kernel launch");
        if (row_need_out) *row_need_out = h.row_need;
        if (fused_out) *fused_out = static_cast<int32_t>(after.forces_done);
        if (h.row_need > row_capacity)
            return fail(err, errlen, RCPG_ENOSPC, "rcpgenerator_b200: a neighbour row exceeds row_capacity");
        const rcpg::StepScalars s = rcpg::finalize_sums(h.sums, mu, ndim);
        if (scalars) {
            scalars[0] = s.U;
            scalars[1] = s.max_overlap;
            scalars[2] = s.Lc;
            scalars[3] = s.Fmean;
            scalars[4] = s.dkappa;
            scalars[5] = s.mean_force;
            scalars[6] = s.count;
        }
        return RCPG_OK;
    } catch (const std::exception& e) {
        return fail(err, errlen, classify(e), e.what());
    }
}

int32_t rcpg_forces(uint64_t N, int32_t ndim, const double* x_dev, const double* D_dev,
                    const double* box, const int8_t* walls, const uint32_t* nbr_dev,
                    const uint32_t* cnt_dev, uint32_t row_capacity, double mu,
                    int32_t exact_order, double* F_dev, double* scalars, void* stream,
                    char* err, size_t errlen) {
    if (N == 0 || ndim < 2 || ndim > rcpg::kMaxDim || !x_dev || !D_dev || !nbr_dev || !cnt_dev ||
        !F_dev || row_capacity == 0)
        return fail(err, errlen, RCPG_EINVAL, "rcpgenerator_b200: bad arguments to rcpg_forces");
    if (!have_device(err, errlen)) return RCPG_ECUDA;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    try {
        const int P = rcpg::pos_stride(ndim);
        Scratch sc(st);
        DevArrays a{};
        a.N = N;
        a.ndim = ndim;
        a.P = P;
        a.pos = static_cast<double*>(sc.get(N * P * 8));
        a.F = F_dev;
        a.nbr = const_cast<std::uint32_t*>(nbr_dev);
        a.nbr_cnt = const_cast<std::uint32_t*>(cnt_dev);
        a.S = row_capacity;
        a.block_sums = static_cast<rcpg::ForceSums*>(sc.get(rcpg::force_blocks(N) * sizeof(rcpg::ForceSums)));
        if (exact_order) {
            a.pterm = static_cast<rcpg::PairTerms*>(sc.get(static_cast<std::size_t>(row_capacity) * N * sizeof(rcpg::PairTerms)));
            a.pterm_cnt = static_cast<std::uint32_t*>(sc.get(N * 4));
        }
        a.ctl = static_cast<DevCtl*>(sc.get(sizeof(DevCtl)));
        DevCtl h;
        std::memset(&h, 0, sizeof(h));
        geometry_from(h, ndim, box, walls);
        h.force_kappa = 1.0;
        h.force_mu = mu;
        cuda_ok(cudaMemcpyAsync(a.ctl, &h, sizeof(h), cudaMemcpyHostToDevice, st), "H2D ctl");
        rcpg::launch_pack(N, ndim, x_dev, D_dev, a.pos, st);
        rcpg::launch_forces(a, exact_order ? 1 : 0, st);
        if (exact_order) rcpg::launch_reduce_exact(a, st);
        else rcpg::launch_reduce_fast(a, st);
        cuda_ok(cudaMemcpyAsync(&h, a.ctl, sizeof(h), cudaMemcpyDeviceToHost, st), "D2H ctl");
        cuda_ok(cudaStreamSynchronize(st), "sync");
        cuda_ok(cudaGetLastError(), "kernel launch");
        const rcpg::StepScalars s = rcpg::finalize_sums(h.sums, mu, ndim);
        if (scalars) {
            scalars[0] = s.U;
            scalars[1] = s.max_overlap;
            scalars[2] = s.Lc;
            scalars[3] = s.Fmean;
            scalars[4] = s.dkappa;
            scalars[5] = s.mean_force;
            scalars[6] = s.count;
        }
        return RCPG_OK;
    } catch (const std::exception& e) {
        return fail(err, errlen, classify(e), e.what());
    }
}

int32_t rcpg_mean_force(uint64_t N, int32_t ndim, const double* F_dev, double* mean_out,
                        void* stream, char* err, size_t errlen) {
    if (N == 0 || ndim < 2 || ndim > rcpg::kMaxDim || !F_dev || !mean_out)
        return fail(err, errlen, RCPG_EINVAL, "rcpgenerator_b200: bad arguments to rcpg_mean_force");
    if (!have_device(err, errlen)) return RCPG_ECUDA;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    try {
        Scratch sc(st);
        DevArrays a{};
        a.N = N;
        a.ndim = ndim;
        a.F = const_cast<double*>(F_dev);
        a.block_sums = static_cast<rcpg::ForceSums*>(sc.get(rcpg::force_blocks(N) * sizeof(rcpg::ForceSums)));
        a.ctl = static_cast<DevCtl*>(sc.get(sizeof(DevCtl)));
        DevCtl h;
        std::memset(&h, 0, sizeof(h));
        cuda_ok(cudaMemcpyAsync(a.ctl, &h, sizeof(h), cudaMemcpyHostToDevice, st), "H2D ctl");
        rcpg::launch_mean_force_blocks(a, st);
        rcpg::launch_reduce_fast(a, st);
        cuda_ok(cudaMemcpyAsync(&h, a.ctl, sizeof(h), cudaMemcpyDeviceToHost, st), "D2H ctl");
        cuda_ok(cudaStreamSynchronize(st), "sync");
        cuda_ok(cudaGetLastError(), "kernel launch");
        const double mean_mag = h.sums.sum_mag / static_cast<double>(static_cast<std::uint32_t>(h.sums.mag_count));
        *mean_out = mean_mag / std::sqrt(static_cast<double>(ndim));
        return RCPG_OK;
    } catch (const std::exception& e) {
        return fail(err, errlen, classify(e), e.what());
    }
}

int32_t rcpg_adam_step(uint64_t N, int32_t ndim, const double* F_dev, double* m_dev,
                       double* v_dev, double* x_dev, const double* box, double alpha,
                       uint64_t t, void* stream, char* err, size_t errlen) {
    if (N == 0 || ndim < 2 || ndim > rcpg::kMaxDim || !F_dev || !m_dev || !v_dev || !x_dev || t == 0)
        return fail(err, errlen, RCPG_EINVAL, "rcpgenerator_b200: bad arguments to rcpg_adam_step");
    if (!have_device(err, errlen)) return RCPG_ECUDA;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    try {
        const int P = rcpg::pos_stride(ndim);
        Scratch sc(st);
        DevArrays a{};
        a.N = N;
        a.ndim = ndim;
        a.P = P;
        a.pos = static_cast<double*>(sc.get(N * P * 8));
        a.F = const_cast<double*>(F_dev);
        a.m = m_dev;
        a.v = v_dev;
        a.ctl = static_cast<DevCtl*>(sc.get(sizeof(DevCtl)));
        DevCtl h;
        std::memset(&h, 0, sizeof(h));
        for (int d = 0; d < ndim; ++d) h.adam_box[d] = box ? box[d] : 1.0;
        const double pb1 = std::pow(0.9, static_cast<double>(t));
        const double pb2 = std::pow(0.999, static_cast<double>(t));
        h.adam_alpha = alpha;
        h.adam_inv_b1 = 1.0 / (1.0 - pb1);
        h.adam_inv_b2 = 1.0 / (1.0 - pb2);
        h.fix_height_scale = 1.0;
        h.adam_go = 1u;
        cuda_ok(cudaMemcpyAsync(a.ctl, &h, sizeof(h), cudaMemcpyHostToDevice, st), "H2D ctl");
        rcpg::launch_pack(N, ndim, x_dev, nullptr, a.pos, st);
        rcpg::launch_adam_refresh(a, 1, 0, st);
        rcpg::launch_unpack(N, ndim, a.pos, x_dev, st);
        cuda_ok(cudaStreamSynchronize(st), "sync");
        cuda_ok(cudaGetLastError(), "kernel launch");
        return RCPG_OK;
    } catch (const std::exception& e) {
        return fail(err, errlen, classify(e), e.what());
    }
}

int32_t rcpg_refresh_check(uint64_t N, int32_t ndim, const double* x_dev, double* x_last_dev,
                           const double* D_dev, double* D_last_dev, double* theta_dev,
                           double theta_new, uint8_t* refresh_dev, uint64_t* count_out,
                           void* stream, char* err, size_t errlen) {
    if (N == 0 || ndim < 2 || ndim > rcpg::kMaxDim || !x_dev || !x_last_dev || !D_dev ||
        !D_last_dev || !theta_dev || !refresh_dev)
        return fail(err, errlen, RCPG_EINVAL, "rcpgenerator_b200: bad arguments to rcpg_refresh_check");
    if (!have_device(err, errlen)) return RCPG_ECUDA;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    try {
        Scratch sc(st);
        auto* cnt = static_cast<unsigned long long*>(sc.get(8));
        cuda_ok(cudaMemsetAsync(cnt, 0, 8, st), "memset");
        rcpg::launch_refresh_arrays(N, ndim, x_dev, x_last_dev, D_dev, D_last_dev, theta_dev,
                                    theta_new, refresh_dev, cnt, st);
        unsigned long long c = 0;
        cuda_ok(cudaMemcpyAsync(&c, cnt, 8, cudaMemcpyDeviceToHost, st), "D2H");
        cuda_ok(cudaStreamSynchronize(st), "sync");
        cuda_ok(cudaGetLastError(), "kernel launch");
        if (count_out) *count_out = c;
        return RCPG_OK;
    } catch (const std::exception& e) {
        return fail(err, errlen, classify(e), e.what());
    }
}

double rcpg_scale_diameters_nd(const double* D, uint64_t N, double phi_target, const double* box,
                               int32_t ndim, int32_t fix_height, double* D_out) {
    std::vector<double> Dv(D, D + N);
    std::vector<double> bv(box, box + ndim);
    double factor = 1.0;
    std::vector<double> o = rcpg::scale_diameters_nd(Dv, phi_target, bv, ndim, fix_height != 0, &factor);
    if (D_out) std::memcpy(D_out, o.data(), N * sizeof(double));
    return factor;
}

int32_t rcpg_initialize_particles(double phi, uint64_t N, int32_t ndim, const double* box,
                                  int32_t box_len, const int8_t* walls, int32_t walls_len,
                                  int32_t fix_height, const rcpg_distribution* dist,
                                  uint64_t seed, double* positions_out, double* diameters_out,
                                  double* box_out, int8_t* walls_out, double* scale_factor_out,
                                  double* phi_modifier_out, char* err, size_t errlen) {
    try {
        rcpg::InitSpec s;
        s.phi = phi;
        s.N = N;
        s.ndim = static_cast<std::size_t>(ndim < 0 ? 0 : ndim);
        if (box && box_len > 0) s.box.assign(box, box + box_len);
        if (walls && walls_len > 0) s.walls.assign(walls, walls + walls_len);
        s.fix_height = fix_height != 0;
        s.seed = seed;
        if (dist) {
            if (dist->type) s.dist.type = dist->type;
            s.dist.d = dist->d;
            s.dist.mu = dist->mu;
            s.dist.sigma = dist->sigma;
            s.dist.mu1 = dist->mu1;
            s.dist.sigma1 = dist->sigma1;
            s.dist.mu2 = dist->mu2;
            s.dist.sigma2 = dist->sigma2;
            s.dist.p = dist->p;
            s.dist.d1 = dist->d1;
            s.dist.d2 = dist->d2;
            s.dist.d_min = dist->d_min;
            s.dist.d_max = dist->d_max;
            s.dist.exponent = dist->exponent;
            s.dist.scale = dist->scale;
            s.dist.shape = dist->shape;
            if (dist->custom && dist->custom_len) s.dist.custom.assign(dist->custom, dist->custom + dist->custom_len);
        }
        rcpg::InitResult r = rcpg::initialize_particles(s);
        if (positions_out) std::memcpy(positions_out, r.positions.data(), r.positions.size() * 8);
        if (diameters_out) std::memcpy(diameters_out, r.diameters.data(), r.diameters.size() * 8);
        if (box_out) std::memcpy(box_out, r.box.data(), r.box.size() * 8);
        if (walls_out) std::memcpy(walls_out, r.walls.data(), r.walls.size());
        if (scale_factor_out) *scale_factor_out = r.scale_factor;
        if (phi_modifier_out) *phi_modifier_out = r.phi_modifier;
        return RCPG_OK;
    } catch (const std::invalid_argument& e) {
        return fail(err, errlen, RCPG_EINVAL, e.what());
    } catch (const std::exception& e) {
        return fail(err, errlen, RCPG_ERUNTIME, e.what());
    }
}

}  // extern "C"
