// The reference-side binding: menos::SimulationEngine over the mb2 C ABI.
//
// This file belongs in the MENOS tree (src/engines/dense_b200/), compiled
// against MENOS's own headers and linked with libmenos_b200.so; it is the
// drop-in for engines::dense_cuda::CudaDenseEngine
// (src/engines/dense_cuda/cuda_dense_engine.cpp:325-412) behind the same
// (Engine::Dense, Backend::Cuda, Tier::InMemory) triple.  Registration: in
// src/plan/execution_engines.cpp:24-31 push `&b200_dense_engine()` instead of
// `&kCudaDense` when b200_device_available(), and fill the hardware
// profile's CUDA figures from measure_b200_calibration() instead of
// plan::measure_cuda_calibration() (src/plan/cuda_calibration.cpp:42-153).
// Nothing else in MENOS changes: planner, KIR, light cone, ledger and front
// ends call it through the interface.
//
// What differs from the reference's CUDA engine, by design:
//   * counts are drawn on the device: a sole region's histogram by the exact
//     device sampler (identical counts), a Factorized region's draws by a
//     device-side cumulative distribution (identical draws); neither copies
//     the state back, so only a statevector request needs the host budget;
//   * the estimate prices the sweep with the engine's calibrated per-pass
//     time model (mb2_estimate_sweep_time) in the planner's own terms.
#include <chrono>
#include <cmath>
#include <complex>
#include <cstring>
#include <exception>
#include <map>
#include <memory>
#include <string>
#include <type_traits>
#include <utility>
#include <variant>
#include <vector>

#include "b200_dense_engine.h"
#include "common/error.h"
#include "common/memory_ledger.h"
#include "common/rng.h"
#include "engines/dense/cumulative_distribution.h"
#include "ir/noise.h"
#include "mb2.h"
#include "menos/bitstring.h"
#include "menos/simulation_engine.h"
#include "plan/cuda_calibration.h"

namespace menos::engines::dense_b200 {
namespace {

// One context per process, opened on first use (device 0).
mb2_context* context() {
    static mb2_context* ctx = [] {
        mb2_context* c = nullptr;
        return mb2_context_create(0, &c) == MB2_OK ? c : nullptr;
    }();
    return ctx;
}

// Status codes to the reference's typed errors (src/common/error.h:11-43).
void check(int rc, const char* what) {
    if (rc == MB2_OK) return;
    char msg[512] = {0};
    if (context() != nullptr) mb2_last_error(context(), msg, sizeof(msg));
    const std::string text = std::string(what) + ": " + msg;
    if (rc == MB2_ERR_RESOURCE) throw common::ResourceExceeded(text);
    throw common::InternalError(text);
}

struct Ops {
    std::vector<mb2_op> ops;
    std::vector<std::vector<double>> matrices;  // storage for UnitaryOp entries
};

Ops to_mb2(std::span<const Operation> operations) {
    Ops out;
    out.ops.reserve(operations.size());
    out.matrices.reserve(operations.size());
    for (const Operation& operation : operations) {
        mb2_op o{};
        std::visit(
            [&](const auto& op) {
                using T = std::decay_t<decltype(op)>;
                if constexpr (std::is_same_v<T, GateOp>) {
                    o.opcode = static_cast<int32_t>(op.opcode);
                    o.num_qubits = static_cast<uint32_t>(op.qubits.size());
                    for (size_t j = 0; j < op.qubits.size(); ++j) o.qubits[j] = op.qubits[j];
                    for (size_t j = 0; j < op.params.size() && j < 3; ++j) o.params[j] = op.params[j];
                } else if constexpr (std::is_same_v<T, UnitaryOp>) {
                    o.opcode = MB2_UNITARY;
                    o.num_qubits = static_cast<uint32_t>(op.qubits.size());
                    for (size_t j = 0; j < op.qubits.size(); ++j) o.qubits[j] = op.qubits[j];
                    std::vector<double> m(2 * op.matrix.size());
                    std::memcpy(m.data(), op.matrix.data(), m.size() * sizeof(double));
                    out.matrices.push_back(std::move(m));
                    o.matrix = out.matrices.back().data();
                } else if constexpr (std::is_same_v<T, MeasureOp>) {
                    o.opcode = MB2_MEASURE;
                    o.num_qubits = 1;
                    o.qubits[0] = op.qubit;
                    o.clbit = op.clbit;
                } else {
                    throw common::InternalError("dense_b200: a noise channel reached a pure-state engine");
                }
            },
            operation);
        out.ops.push_back(o);
    }
    return out;
}

// A device state with its Device-space ledger charge (the reference's
// DeviceBuffer charges the same, src/kernels/cuda/device_buffer.cpp:33);
// freed on every exit, unwinding included (cuda_dense_engine.cpp:55-57).
struct StateGuard {
    mb2_state* s = nullptr;
    common::MemoryLedger::Charge charge;
    StateGuard() = default;
    StateGuard(const StateGuard&) = delete;
    StateGuard& operator=(const StateGuard&) = delete;
    ~StateGuard() { mb2_state_free(s); }
    mb2_state* release() {
        mb2_state* out = s;
        s = nullptr;
        return out;
    }
};

// The monitor crosses the C boundary as a callback; its exception is carried
// back and rethrown on this side.
struct MonitorBridge {
    const ExecutionMonitor* monitor;
    std::exception_ptr error;
};

int on_boundary(void* user, uint64_t blocks_done) {
    auto* b = static_cast<MonitorBridge*>(user);
    try {
        b->monitor->at_safe_boundary(blocks_done);
        return 0;
    } catch (...) {
        b->error = std::current_exception();
        return 1;
    }
}

BitString outcome_of(uint64_t index, const std::vector<std::pair<uint32_t, uint32_t>>& targets, uint32_t width) {
    BitString outcome(width);
    for (const auto& [qubit, clbit] : targets)
        if ((index >> qubit) & 1u) outcome.set(clbit, true);
    return outcome;
}

// A Factorized region's outcome distribution kept on the device: the
// answers of engines::dense::CumulativeDistribution::sample_one
// (src/engines/dense/cumulative_distribution.cpp:3-124) for the region's
// state, without copying the state back or building the 8 * 2^n cumulative
// array on the host.  combine_counts (src/runtime/combine_counts.cpp) draws
// one word per shot from the region's own Rng; the first call draws the
// next `batch` words from a copy of that Rng and resolves them all in one
// device walk (mb2_sample_basis); each call then takes one word from the
// caller's Rng and returns the precomputed outcome when the word is the
// expected one (always, in combine_counts), resolving it alone otherwise.
class DeviceRegionSampler final : public RegionCountsSampler {
public:
    DeviceRegionSampler(StateGuard& state, std::span<const std::pair<QubitId, ClbitId>> targets, uint32_t width,
                        uint64_t batch)
        : state_(state.release()),
          charge_(std::move(state.charge)),
          targets_(targets.begin(), targets.end()),
          width_(width),
          batch_(batch == 0 ? 1 : batch) {}
    DeviceRegionSampler(const DeviceRegionSampler&) = delete;
    DeviceRegionSampler& operator=(const DeviceRegionSampler&) = delete;
    ~DeviceRegionSampler() override { mb2_state_free(state_); }

    [[nodiscard]] BitString sample_one(common::Rng& rng) const override {
        if (next_ >= words_.size()) {
            common::Rng ahead = rng;
            words_.resize(batch_);
            std::vector<double> u(batch_);
            for (uint64_t i = 0; i < batch_; ++i) {
                words_[i] = ahead.next_word();
                u[i] = common::Rng::word_to_uniform(words_[i]);
            }
            basis_.assign(batch_, 0);
            check(mb2_sample_basis(state_, u.data(), batch_, basis_.data()), "region sampler");
            next_ = 0;
        }
        const uint64_t w = rng.next_word();
        if (w == words_[next_]) return outcome_of(basis_[next_++], targets_, width_);
        words_.clear();
        next_ = 0;
        const double u = common::Rng::word_to_uniform(w);
        uint64_t b = 0;
        check(mb2_sample_basis(state_, &u, 1, &b), "region sampler");
        return outcome_of(b, targets_, width_);
    }

private:
    mb2_state* state_;
    common::MemoryLedger::Charge charge_;
    std::vector<std::pair<uint32_t, uint32_t>> targets_;
    uint32_t width_;
    uint64_t batch_;
    mutable std::vector<uint64_t> words_, basis_;
    mutable uint64_t next_ = 0;
};

}  // namespace

bool b200_device_available() { return context() != nullptr; }

mb2_context* b200_context() { return context(); }

// The figures the planner's CUDA time model reads
// (src/plan/planner.cpp:415-433, plan::CudaCalibration), measured on this
// engine: a work unit is one amplitude of one state pass, priced at the
// autotuner's per-amplitude pass cost; a launch costs the autotuner's fixed
// per-pass cost; transfers are timed with pageable host memory, as the
// reference measures them.  present == false without a device.
plan::CudaCalibration measure_b200_calibration() {
    plan::CudaCalibration c;
    mb2_context* ctx = context();
    if (ctx == nullptr) return c;
    uint64_t total = 0, free_bytes = 0;
    if (mb2_device_info(ctx, nullptr, &total, &free_bytes) != MB2_OK) return c;
    mb2_tuning t{};
    if (mb2_context_tuning(ctx, &t) != MB2_OK) return c;
    if (t.probe_qubits == 0 && mb2_autotune(ctx, 0, &t) != MB2_OK) return c;
    using clock = std::chrono::steady_clock;
    // Transfers: a 64 MiB state both ways, best of three.
    constexpr uint32_t kQ = 22;
    mb2_state* s = nullptr;
    if (mb2_state_alloc(ctx, kQ, MB2_C128, ~uint64_t{0}, &s) != MB2_OK) return c;
    std::vector<std::complex<double>> host(uint64_t{1} << kQ);
    double h2d = 1e30, d2h = 1e30;
    for (int r = 0; r < 3; ++r) {
        auto t0 = clock::now();
        mb2_copy_in(s, host.data(), host.size());
        auto t1 = clock::now();
        mb2_copy_out(s, host.data(), host.size());
        auto t2 = clock::now();
        h2d = std::min(h2d, std::chrono::duration<double>(t1 - t0).count());
        d2h = std::min(d2h, std::chrono::duration<double>(t2 - t1).count());
    }
    mb2_state_free(s);
    // One execution's fixed cost beyond its launches: allocate, initialise,
    // synchronise and free a one-qubit state, best of five.
    double exec = 1e30;
    for (int r = 0; r < 5; ++r) {
        auto t0 = clock::now();
        mb2_state* e = nullptr;
        if (mb2_state_alloc(ctx, 1, MB2_C128, ~uint64_t{0}, &e) != MB2_OK) return c;
        mb2_init(e, 0.0);
        mb2_synchronize(e);
        mb2_state_free(e);
        exec = std::min(exec, std::chrono::duration<double>(clock::now() - t0).count());
    }
    const double bytes = static_cast<double>(host.size() * sizeof(std::complex<double>));
    c.present = true;
    c.device_total_bytes = total;
    c.device_available_bytes = free_bytes;
    c.host_to_device_bytes_per_second = bytes / h2d;
    c.device_to_host_bytes_per_second = bytes / d2h;
    c.kernel_launch_seconds = t.pass_s_fixed;
    c.execution_seconds = std::max(0.0, exec - t.pass_s_fixed);
    c.device_work_units_per_second = 1.0 / t.pass_s_per_amp;
    return c;
}

class B200DenseEngine : public SimulationEngine {
public:
    [[nodiscard]] std::string_view name() const override { return "dense_b200"; }
    [[nodiscard]] Engine engine_id() const override { return Engine::Dense; }
    [[nodiscard]] Backend backend() const override { return Backend::Cuda; }
    [[nodiscard]] EngineCapabilities capabilities() const override {
        return EngineCapabilities{/*counts=*/true, /*statevector=*/true, /*expectation=*/true};
    }

    // Never throws; infeasible is a value (include/menos/simulation_engine.h:349-359).
    [[nodiscard]] CostEstimate estimate(const EngineEstimateRequest& request) const override {
        try {
            return estimate_or_throw(request);
        } catch (const std::exception& e) {
            return CostEstimate{false, 0, 0, std::string("dense_b200: ") + e.what(), {}};
        }
    }

    [[nodiscard]] EngineExecutionResult execute(const EngineExecutionRequest& request) const override {
        common::ensure(b200_device_available(), "B200DenseEngine::execute: no device");
        Ops ops = to_mb2(request.operations);
        const uint64_t amps = uint64_t{1} << request.num_qubits;
        const uint64_t state_bytes = 16 * amps;
        uint64_t total = 0, free_bytes = 0;
        check(mb2_device_info(context(), nullptr, &total, &free_bytes), "device_info");
        StateGuard st;
        // Budgeted against the device's own free memory, refused before any
        // allocation (device_buffer.cpp:23), then charged to the Device space.
        check(mb2_state_alloc(context(), request.num_qubits, MB2_C128, free_bytes, &st.s), "state");
        st.charge = common::MemoryLedger::Charge(state_bytes, common::MemoryLedger::Space::Device);
        check(mb2_init(st.s, request.global_phase), "init");
        mb2_sweep_options o{request.fuse_gates ? 1 : 0, 0, 0, 0, 0, 0};
        if (request.monitor != nullptr) {
            MonitorBridge bridge{request.monitor, nullptr};
            const int rc = mb2_apply_program_monitored(st.s, ops.ops.data(), static_cast<uint32_t>(ops.ops.size()),
                                                       &o, &on_boundary, &bridge);
            if (bridge.error) std::rethrow_exception(bridge.error);
            check(rc, "sweep");
        } else {
            check(mb2_apply_program(st.s, ops.ops.data(), static_cast<uint32_t>(ops.ops.size()), &o), "sweep");
        }
        EngineExecutionResult result;
        result.actual_bytes = state_bytes;
        if (request.want_expectation) {
            const auto& terms = request.observable->terms;
            std::vector<uint64_t> xs, zs;
            for (const auto& t : terms) {
                xs.push_back(t.first.x_words[0]);
                zs.push_back(t.first.z_words[0]);
            }
            std::vector<std::complex<double>> out(terms.size());
            check(mb2_expectation(st.s, xs.data(), zs.data(), static_cast<uint32_t>(terms.size()),
                                  reinterpret_cast<double*>(out.data())),
                  "expectation");
            result.expectation_terms = std::move(out);
        }
        if (request.want_counts && request.is_sole_region) {
            std::vector<uint32_t> targets;
            for (const auto& [q, c] : request.measure_targets) {
                targets.push_back(q);
                targets.push_back(c);
            }
            std::vector<uint64_t> outcomes(request.shots), counts(request.shots);
            uint64_t distinct = request.shots;
            check(mb2_sample(st.s, request.shots, request.seed, targets.data(),
                             static_cast<uint32_t>(request.measure_targets.size()), outcomes.data(), counts.data(),
                             &distinct),
                  "sample");
            std::map<BitString, std::uint64_t> hist;
            for (uint64_t i = 0; i < distinct; ++i) {
                BitString key(request.bitstring_width);
                for (uint32_t b = 0; b < request.bitstring_width && b < 64; ++b)
                    if ((outcomes[i] >> b) & 1u) key.set(b, true);
                hist.emplace(std::move(key), counts[i]);
            }
            result.counts = std::move(hist);
        }
        if (request.want_statevector) {
            // The host copy is the only host memory this engine needs; it is
            // refused over budget before it is allocated, with the reference's
            // message (cuda_dense_engine.cpp:377-384).
            if (state_bytes > request.budget_bytes)
                throw common::ResourceExceeded("CUDA dense: the host copy needs " + std::to_string(state_bytes) +
                                               " bytes, budget is " + std::to_string(request.budget_bytes) +
                                               " bytes");
            std::vector<std::complex<double>> host(amps);
            common::MemoryLedger::Charge charge(state_bytes);
            check(mb2_copy_out(st.s, host.data(), amps), "copy_out");
            charge.release();
            result.statevector = std::move(host);
        }
        if (request.want_counts && !request.is_sole_region) {
            // The region's distribution stays on the device with the state.
            result.counts_sampler = std::make_unique<DeviceRegionSampler>(st, request.measure_targets,
                                                                          request.bitstring_width, request.shots);
        }
        return result;
    }

private:
    [[nodiscard]] CostEstimate estimate_or_throw(const EngineEstimateRequest& request) const {
        if (!b200_device_available()) return CostEstimate{false, 0, 0, "no B200 device is available", {}};
        if (auto reason = ir::first_noise_reason(*request.operations); reason.has_value())
            return CostEstimate{false, 0, 0, *reason, {}};
        if (request.num_qubits > 34) return CostEstimate{false, 0, 0, "more than 34 qubits on one B200", {}};
        if (request.num_qubits == 0)
            return CostEstimate{false, 0, 0, "a region of no qubits (one amplitude) is not worth a device", {}};
        Ops ops = to_mb2(*request.operations);
        const uint32_t n = request.num_qubits;
        mb2_sweep_options o{request.fuse_gates ? 1 : 0, 0, 0, 0, 0, 0};
        mb2_sweep_estimate e{};
        if (mb2_estimate_sweep(ops.ops.data(), static_cast<uint32_t>(ops.ops.size()), &o, n, &e) != MB2_OK)
            return CostEstimate{false, 0, 0, "dense_b200: operations rejected", {}};
        const uint64_t amps = uint64_t{1} << n;
        const uint64_t terms = request.want_expectation ? request.observable->terms.size() : 0;
        // Expectation scratch: masks, partial sums and results per term.
        const uint64_t device_bytes = e.device_bytes + terms * (16 + 512 * 16 + 16);
        uint64_t free_bytes = 0;
        mb2_device_info(context(), nullptr, nullptr, &free_bytes);
        if (device_bytes > free_bytes)
            return CostEstimate{false, 0, 0,
                                "dense_b200 needs " + std::to_string(device_bytes) + " device bytes, " +
                                    std::to_string(free_bytes) + " free",
                                {}};
        // Device work in the planner's units (one unit = one amplitude of one
        // state pass): the calibrated sweep time beyond its launches, plus the
        // output passes (a statevector copy reads the state once: half a
        // pass; the sampler reads it three times; each group of Pauli terms
        // that shares a read, once).
        mb2_tuning t{};
        check(mb2_context_tuning(context(), &t), "tuning");
        double sweep_s = 0.0;
        check(mb2_estimate_sweep_time(context(), ops.ops.data(), static_cast<uint32_t>(ops.ops.size()), &o, n,
                                      MB2_C128, &sweep_s),
              "time model");
        const double rate = 1.0 / t.pass_s_per_amp;
        double work = std::max(0.0, sweep_s - static_cast<double>(e.passes) * t.pass_s_fixed) * rate +
                      static_cast<double>(amps) / 2.0;  // initialisation writes the state
        uint64_t launches = e.launches;
        if (request.want_statevector) work += static_cast<double>(amps) / 2.0;
        if (request.want_counts) {
            work += 1.5 * static_cast<double>(amps);
            launches += 5;
        }
        if (request.want_expectation) {
            std::vector<uint64_t> xs, zs;
            for (const auto& term : request.observable->terms) {
                xs.push_back(term.first.x_words[0]);
                zs.push_back(term.first.z_words[0]);
            }
            uint64_t words = 0;
            mb2_debug_pauli_groups(xs.data(), zs.data(), static_cast<uint32_t>(terms), n, nullptr, &words);
            std::vector<uint64_t> g(words);
            mb2_debug_pauli_groups(xs.data(), zs.data(), static_cast<uint32_t>(terms), n, g.data(), &words);
            const uint64_t groups = g.empty() ? terms : g[0];
            work += static_cast<double>(groups) * static_cast<double>(amps) / 2.0;
            launches += groups + 1;
        }
        const uint64_t host_bytes = request.want_statevector ? 16 * amps : 0;
        const uint64_t d2h = request.want_statevector ? 16 * amps : 16 * terms;
        CostEstimate est{true, host_bytes, static_cast<uint64_t>(std::llround(work)), "",
                         DeviceCost{device_bytes, e.h2d_bytes, d2h, launches}};
        // Host work in the CPU dense engine's time components, as the
        // reference's CUDA estimate reports it: the passes the host prepares
        // (plan and block build per pass) and, for counts, the per-shot
        // uniforms (the walk itself runs on the device).
        auto& dense = est.time.counts[static_cast<std::size_t>(Engine::Dense)];
        dense[0] = static_cast<double>(e.passes + 1);
        if (request.want_counts) dense[2] = static_cast<double>(request.shots);
        return est;
    }
};

// The engine instance the registration pushes (one per process, stateless).
const SimulationEngine& b200_dense_engine() {
    static const B200DenseEngine engine;
    return engine;
}

int ServerLedger::attach(mb2_server* server) { return mb2_server_set_ledger(server, &charge, &release, this); }

// Called by the server with its lock held, one call at a time.
int ServerLedger::charge(void* user, uint64_t bytes) {
    auto* self = static_cast<ServerLedger*>(user);
    if (self->limit_ != 0 && self->ledger_.live_device_bytes() + bytes > self->limit_) return 0;
    const common::MemoryLedger::Scope scope(self->ledger_);
    self->live_.emplace(bytes, common::MemoryLedger::Charge(bytes, common::MemoryLedger::Space::Device));
    return 1;
}

void ServerLedger::release(void* user, uint64_t bytes) {
    auto* self = static_cast<ServerLedger*>(user);
    const auto it = self->live_.find(bytes);
    if (it != self->live_.end()) self->live_.erase(it);
}

}  // namespace menos::engines::dense_b200
