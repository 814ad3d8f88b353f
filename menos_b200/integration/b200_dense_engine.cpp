// The reference-side binding: menos::SimulationEngine over the mb2 C ABI.
//
// This file belongs in the MENOS tree (src/engines/dense_b200/), compiled
// against MENOS's own headers and linked with libmenos_b200.so; it is the
// drop-in for engines::dense_cuda::CudaDenseEngine
// (src/engines/dense_cuda/cuda_dense_engine.cpp:325-412) behind the same
// (Engine::Dense, Backend::Cuda, Tier::InMemory) triple.  Registration: in
// src/plan/execution_engines.cpp:24-31 push `&kB200Dense` instead of
// `&kCudaDense` when b200_device_available().  Nothing else in MENOS changes:
// planner, KIR, light cone, ledger and front ends call it through the
// interface.  tests/test_integration.py compiles it (-fsyntax-only) against
// the reference headers.
#include <complex>
#include <cstring>
#include <exception>
#include <map>
#include <memory>
#include <string>
#include <type_traits>
#include <variant>
#include <vector>

#include "common/error.h"
#include "common/memory_ledger.h"
#include "engines/dense/cumulative_distribution.h"
#include "ir/noise.h"
#include "mb2.h"
#include "menos/bitstring.h"
#include "menos/simulation_engine.h"

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

// Frees the device state on every exit, unwinding included
// (cuda_dense_engine.cpp:55-57).
struct StateGuard {
    mb2_state* s = nullptr;
    ~StateGuard() { mb2_state_free(s); }
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

}  // namespace

bool b200_device_available() { return context() != nullptr; }

class B200DenseEngine : public SimulationEngine {
public:
    [[nodiscard]] std::string_view name() const override { return "dense_b200"; }
    [[nodiscard]] Engine engine_id() const override { return Engine::Dense; }
    [[nodiscard]] Backend backend() const override { return Backend::Cuda; }
    [[nodiscard]] EngineCapabilities capabilities() const override {
        return EngineCapabilities{/*counts=*/true, /*statevector=*/true, /*expectation=*/true};
    }

    [[nodiscard]] CostEstimate estimate(const EngineEstimateRequest& request) const override {
        if (!b200_device_available()) return CostEstimate{false, 0, 0, "no B200 device is available", {}};
        if (auto reason = ir::first_noise_reason(*request.operations); reason.has_value())
            return CostEstimate{false, 0, 0, *reason, {}};
        if (request.num_qubits > 34) return CostEstimate{false, 0, 0, "more than 34 qubits on one B200", {}};
        Ops ops = to_mb2(*request.operations);
        mb2_sweep_options o{request.fuse_gates ? 1 : 0, 0, 0, 0};
        mb2_sweep_estimate e{};
        if (mb2_estimate_sweep(ops.ops.data(), static_cast<uint32_t>(ops.ops.size()), &o, request.num_qubits, &e) !=
            MB2_OK)
            return CostEstimate{false, 0, 0, "dense_b200: operations rejected", {}};
        uint64_t work = e.work_units;
        const uint64_t amps = uint64_t{1} << request.num_qubits;
        if (request.want_statevector) work += amps;
        if (request.want_counts) work += amps;
        if (request.want_expectation) work += amps * request.observable->terms.size();
        uint64_t free_bytes = 0;
        mb2_device_info(context(), nullptr, nullptr, &free_bytes);
        if (e.device_bytes > free_bytes)
            return CostEstimate{false, 0, 0,
                                "dense_b200 needs " + std::to_string(e.device_bytes) + " device bytes, " +
                                    std::to_string(free_bytes) + " free",
                                {}};
        const uint64_t d2h = request.want_statevector ? 16 * amps
                             : request.want_expectation ? 16 * request.observable->terms.size()
                                                        : 0;
        CostEstimate est{true, request.want_statevector ? 16 * amps : 0, work, "",
                         DeviceCost{e.device_bytes, e.h2d_bytes, d2h, e.launches}};
        return est;
    }

    [[nodiscard]] EngineExecutionResult execute(const EngineExecutionRequest& request) const override {
        common::ensure(b200_device_available(), "B200DenseEngine::execute: no device");
        Ops ops = to_mb2(request.operations);
        uint64_t total = 0, free_bytes = 0;
        check(mb2_device_info(context(), nullptr, &total, &free_bytes), "device_info");
        StateGuard st;
        check(mb2_state_alloc(context(), request.num_qubits, MB2_C128, free_bytes, &st.s), "state");
        check(mb2_init(st.s, request.global_phase), "init");
        mb2_sweep_options o{request.fuse_gates ? 1 : 0, 0, 0, 0};
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
        const uint64_t amps = uint64_t{1} << request.num_qubits;
        result.actual_bytes = 16 * amps;
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
        if (request.want_statevector || (request.want_counts && !request.is_sole_region)) {
            std::vector<std::complex<double>> host(amps);
            common::MemoryLedger::Charge charge(host.size() * sizeof(std::complex<double>));
            check(mb2_copy_out(st.s, host.data(), amps), "copy_out");
            if (request.want_counts && !request.is_sole_region)
                result.counts_sampler = std::make_unique<engines::dense::CumulativeDistribution>(
                    host, request.measure_targets, request.bitstring_width);
            if (request.want_statevector) {
                charge.release();
                result.statevector = std::move(host);
            }
        }
        return result;
    }
};

}  // namespace menos::engines::dense_b200
