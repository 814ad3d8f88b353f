// The reference-side binding of the noisy engines: menos::SimulationEngine
// over the mb2 C ABI for the density-matrix and trajectory engines.
//
// This file belongs in the MENOS tree beside b200_dense_engine.cpp,
// compiled against MENOS's headers and linked with libmenos_b200.so.  The
// reference has CPU implementations only (DensityMatrixEngine,
// src/engines/density_matrix/density_matrix_engine.cpp:356-415;
// TrajectoryEngine, src/engines/trajectory/trajectory_engine.cpp:410-494);
// these register beside them under Backend::Cuda, when
// b200_device_available(), in src/plan/execution_engines.cpp, and the
// planner picks between the backends by its calibrated time model as it does
// for the dense engine.  What they compute is the reference engines'
// arithmetic: rho's bits, the trajectory states, the counts (readout errors
// included), the draws of a Factorized region; traces and term means are
// fixed-order device reductions within 1e-12 of the reference's sequential
// sums.
#include <algorithm>
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
#include "b200_noisy_engines.h"
#include "common/error.h"
#include "common/memory_ledger.h"
#include "common/rng.h"
#include "engines/noise/readout.h"
#include "mb2.h"
#include "menos/bitstring.h"
#include "menos/simulation_engine.h"

namespace menos::engines::dense_b200 {
namespace {

using Complex = std::complex<double>;

void check(int rc, const char* what) {
    if (rc == MB2_OK) return;
    char msg[512] = {0};
    if (b200_context() != nullptr) mb2_last_error(b200_context(), msg, sizeof(msg));
    const std::string text = std::string(what) + ": " + msg;
    if (rc == MB2_ERR_RESOURCE) throw common::ResourceExceeded(text);
    throw common::InternalError(text);
}

// The operations as mb2_op, channels and readout errors included: a
// ChannelOp's Kraus operators consecutive at `matrix` (`reserved` of them),
// a MeasureOp's readout error as its 4 assignment entries.
struct Ops {
    std::vector<mb2_op> ops;
    std::vector<std::vector<double>> storage;
};

Ops to_mb2(std::span<const Operation> operations) {
    Ops out;
    out.ops.reserve(operations.size());
    out.storage.reserve(operations.size());
    auto keep = [&](std::vector<double>&& v) -> const double* {
        out.storage.push_back(std::move(v));
        return out.storage.back().data();
    };
    for (const Operation& operation : operations) {
        mb2_op o{};
        std::visit(
            [&](const auto& op) {
                using T = std::decay_t<decltype(op)>;
                if constexpr (std::is_same_v<T, MeasureOp>) {
                    o.opcode = MB2_MEASURE;
                    o.num_qubits = 1;
                    o.qubits[0] = op.qubit;
                    o.clbit = op.clbit;
                    if (op.readout_error.has_value()) {
                        const auto& a = op.readout_error->assignment;
                        o.matrix = keep(std::vector<double>(a.begin(), a.end()));
                    }
                } else {
                    common::ensure(op.qubits.size() <= MB2_MAX_OP_QUBITS, "noisy b200: operation too wide");
                    o.num_qubits = static_cast<uint32_t>(op.qubits.size());
                    for (size_t j = 0; j < op.qubits.size(); ++j) o.qubits[j] = op.qubits[j];
                    if constexpr (std::is_same_v<T, GateOp>) {
                        o.opcode = static_cast<int32_t>(op.opcode);
                        for (size_t j = 0; j < op.params.size() && j < 3; ++j) o.params[j] = op.params[j];
                    } else if constexpr (std::is_same_v<T, UnitaryOp>) {
                        o.opcode = MB2_UNITARY;
                        std::vector<double> m(2 * op.matrix.size());
                        std::memcpy(m.data(), op.matrix.data(), m.size() * sizeof(double));
                        o.matrix = keep(std::move(m));
                    } else {
                        static_assert(std::is_same_v<T, ChannelOp>);
                        o.opcode = MB2_CHANNEL;
                        std::vector<double> m;
                        for (const auto& k : op.kraus) {
                            const size_t at = m.size();
                            m.resize(at + 2 * k.size());
                            std::memcpy(m.data() + at, k.data(), 2 * k.size() * sizeof(double));
                        }
                        o.reserved = static_cast<uint32_t>(op.kraus.size());
                        o.matrix = keep(std::move(m));
                    }
                }
            },
            operation);
        out.ops.push_back(o);
    }
    return out;
}

std::vector<uint32_t> flat_targets(std::span<const std::pair<QubitId, ClbitId>> targets) {
    std::vector<uint32_t> t;
    for (const auto& [q, c] : targets) {
        t.push_back(q);
        t.push_back(c);
    }
    return t;
}

std::map<BitString, std::uint64_t> histogram(const std::vector<uint64_t>& outcomes,
                                             const std::vector<uint64_t>& counts, uint64_t distinct,
                                             uint32_t width) {
    std::map<BitString, std::uint64_t> hist;
    for (uint64_t i = 0; i < distinct; ++i) {
        BitString key(width);
        for (uint32_t b = 0; b < width && b < 64; ++b)
            if ((outcomes[i] >> b) & 1u) key.set(b, true);
        hist.emplace(std::move(key), counts[i]);
    }
    return hist;
}

uint64_t pow2(uint32_t e) { return uint64_t{1} << e; }

// A density matrix on the device with its Device-space ledger charge.
struct RhoGuard {
    mb2_state* s = nullptr;
    common::MemoryLedger::Charge charge;
    RhoGuard() = default;
    RhoGuard(const RhoGuard&) = delete;
    RhoGuard& operator=(const RhoGuard&) = delete;
    ~RhoGuard() { mb2_state_free(s); }
};

// A Factorized region's outcome distribution with its readout errors, kept
// on the device with rho: the draws of the reference's
// DensityMatrixCountsSampler (density_matrix_engine.cpp:157-179) -- one word
// for the true outcome, then one per readout-errored target (drawn by the
// reference's own apply_readout).  The outcome words are resolved in
// batches: the first call reads ahead from a copy of the caller's Rng,
// skipping each draw's readout words, and resolves the next `batch` outcome
// words in one device walk; each call then checks that the word it takes is
// the one expected (always, in combine_counts) and resolves it alone
// otherwise.
class DeviceRhoSampler final : public RegionCountsSampler {
public:
    DeviceRhoSampler(RhoGuard& rho, uint32_t n, std::span<const std::pair<QubitId, ClbitId>> targets, uint32_t width,
                     std::vector<noise::ReadoutTarget> readouts, uint64_t batch)
        : state_(rho.s),
          charge_(std::move(rho.charge)),
          n_(n),
          targets_(targets.begin(), targets.end()),
          width_(width),
          readouts_(std::move(readouts)),
          batch_(batch == 0 ? 1 : batch) {
        rho.s = nullptr;
    }
    DeviceRhoSampler(const DeviceRhoSampler&) = delete;
    DeviceRhoSampler& operator=(const DeviceRhoSampler&) = delete;
    ~DeviceRhoSampler() override { mb2_state_free(state_); }

    [[nodiscard]] BitString sample_one(common::Rng& rng) const override {
        if (next_ >= words_.size()) {
            common::Rng ahead = rng;
            words_.resize(batch_);
            std::vector<double> u(batch_);
            for (uint64_t i = 0; i < batch_; ++i) {
                words_[i] = ahead.next_word();
                u[i] = common::Rng::word_to_uniform(words_[i]);
                for (size_t r = 0; r < readouts_.size(); ++r) (void)ahead.next_word();
            }
            basis_.assign(batch_, 0);
            check(mb2_dm_sample_basis(state_, n_, u.data(), batch_, basis_.data()), "density-matrix sampler");
            next_ = 0;
        }
        const uint64_t w = rng.next_word();
        uint64_t b = 0;
        if (w == words_[next_]) {
            b = basis_[next_++];
        } else {
            words_.clear();
            next_ = 0;
            const double u = common::Rng::word_to_uniform(w);
            check(mb2_dm_sample_basis(state_, n_, &u, 1, &b), "density-matrix sampler");
        }
        BitString outcome(width_);
        for (const auto& [qubit, clbit] : targets_)
            if ((b >> qubit) & 1u) outcome.set(clbit, true);
        noise::apply_readout(outcome, readouts_, rng);
        return outcome;
    }

private:
    mb2_state* state_;
    common::MemoryLedger::Charge charge_;
    uint32_t n_;
    std::vector<std::pair<QubitId, ClbitId>> targets_;
    uint32_t width_;
    std::vector<noise::ReadoutTarget> readouts_;
    uint64_t batch_;
    mutable std::vector<uint64_t> words_, basis_;
    mutable uint64_t next_ = 0;
};

// The monitor crosses the C boundary as a callback (as in the dense binding).
struct MonitorBridge {
    const ExecutionMonitor* monitor;
    std::exception_ptr error;
};

int on_boundary(void* user, uint64_t crossed) {
    auto* b = static_cast<MonitorBridge*>(user);
    try {
        b->monitor->at_safe_boundary(crossed);
        return 0;
    } catch (...) {
        b->error = std::current_exception();
        return 1;
    }
}

uint64_t operand_count(const Operation& op) {
    return std::visit(
        [](const auto& o) -> uint64_t {
            if constexpr (std::is_same_v<std::decay_t<decltype(o)>, MeasureOp>) return 0;
            else return o.qubits.size();
        },
        op);
}

uint64_t free_device_bytes() {
    uint64_t free_bytes = 0;
    if (b200_context() != nullptr) mb2_device_info(b200_context(), nullptr, nullptr, &free_bytes);
    return free_bytes;
}

class B200DensityMatrixEngine : public SimulationEngine {
public:
    [[nodiscard]] std::string_view name() const override { return "density_matrix_b200"; }
    [[nodiscard]] Engine engine_id() const override { return Engine::DensityMatrix; }
    [[nodiscard]] Backend backend() const override { return Backend::Cuda; }
    [[nodiscard]] EngineCapabilities capabilities() const override {
        return EngineCapabilities{/*counts=*/true, /*statevector=*/false, /*expectation=*/true};
    }

    // Work units as the reference's estimate counts them
    // (density_matrix_engine.cpp:293-350): 4^n to initialise, 2 * 2^(2n+k)
    // per gate, 2^(2n+2k) per channel, 2^n for the diagonal, 2^n per term.
    [[nodiscard]] CostEstimate estimate(const EngineEstimateRequest& request) const override {
        if (request.want_statevector)
            return CostEstimate{false, 0, 0,
                                "the density-matrix engine does not produce a statevector -- a mixed state has none",
                                {}};
        if (!b200_device_available()) return CostEstimate{false, 0, 0, "no B200 device is available", {}};
        const uint32_t n = request.num_qubits;
        if (n < 1 || n > 15) return CostEstimate{false, 0, 0, "density_matrix_b200 holds 1..15 qubits", {}};
        uint64_t work = pow2(2 * n), launches = 1, h2d = 0;
        double passes = 1.0;
        for (const Operation& op : *request.operations) {
            const uint64_t k = operand_count(op);
            if (k == 0) continue;
            if (k > 5) return CostEstimate{false, 0, 0, "density_matrix_b200: an operation on more than 5 qubits", {}};
            if (std::holds_alternative<ChannelOp>(op)) {
                work += pow2(static_cast<uint32_t>(2 * n + 2 * k));
                h2d += 16 * pow2(static_cast<uint32_t>(4 * k));
                passes += 1.0;
            } else {
                work += 2 * pow2(static_cast<uint32_t>(2 * n + k));
                h2d += 32 * pow2(static_cast<uint32_t>(2 * k));
                passes += 2.0;
            }
            ++launches;
        }
        uint64_t d2h = 0, host = 0;
        const uint64_t terms = request.want_expectation ? request.observable->terms.size() : 0;
        if (request.want_counts) {
            work += pow2(n);
            launches += 1;
            d2h += 16 * request.shots;
            host += 32 * request.shots;  // uniforms, basis states, readout words, histogram
        }
        if (request.want_expectation) {
            work += terms * pow2(n);
            launches += 2;
            d2h += 16 * terms;
        }
        const uint64_t device_bytes = 16 * pow2(2 * n) + (uint64_t{1} << 20) + 16 * request.shots + h2d;
        if (device_bytes > free_device_bytes())
            return CostEstimate{false, 0, 0, "density_matrix_b200 needs " + std::to_string(device_bytes) +
                                                 " device bytes", {}};
        CostEstimate est{true, host, work, "", DeviceCost{device_bytes, h2d, d2h, launches}};
        auto& dm = est.time.counts[static_cast<std::size_t>(Engine::DensityMatrix)];
        dm[0] = passes;
        dm[1] = static_cast<double>(work);
        dm[2] = request.want_counts ? static_cast<double>(request.shots) : 0.0;
        return est;
    }

    [[nodiscard]] EngineExecutionResult execute(const EngineExecutionRequest& request) const override {
        common::ensure(b200_device_available(), "B200DensityMatrixEngine::execute: no device");
        common::ensure(!request.want_statevector,
                       "density matrix: a statevector was requested; estimate() refuses that");
        const uint32_t n = request.num_qubits;
        common::ensure(n >= 1 && n <= 15, "density_matrix_b200: 1..15 qubits");
        Ops ops = to_mb2(request.operations);
        const uint64_t rho_bytes = 16 * pow2(2 * n);
        RhoGuard rho;
        // Global phase cancels in rho; budgeted against the device's free
        // memory, refused before allocating, charged to the Device space.
        check(mb2_state_alloc(b200_context(), 2 * n, MB2_C128, free_device_bytes(), &rho.s), "rho");
        rho.charge = common::MemoryLedger::Charge(rho_bytes, common::MemoryLedger::Space::Device);
        check(mb2_init(rho.s, 0.0), "init");
        if (request.monitor == nullptr) {
            check(mb2_dm_apply_program(rho.s, n, ops.ops.data(), static_cast<uint32_t>(ops.ops.size())), "operations");
        } else {
            // The gap between two operations is the reference's safe boundary
            // (density_matrix_engine.cpp:120-152).
            for (size_t i = 0; i < ops.ops.size(); ++i) {
                check(mb2_dm_apply_program(rho.s, n, &ops.ops[i], 1), "operations");
                request.monitor->at_safe_boundary(i + 1);
            }
        }
        EngineExecutionResult result;
        result.actual_bytes = rho_bytes;
        if (request.want_expectation) {
            const auto& terms = request.observable->terms;
            std::vector<uint64_t> xs, zs;
            for (const auto& t : terms) {
                xs.push_back(t.first.x_words[0]);
                zs.push_back(t.first.z_words[0]);
            }
            std::vector<Complex> out(terms.size());
            check(mb2_dm_expectation(rho.s, n, xs.data(), zs.data(), static_cast<uint32_t>(terms.size()),
                                     reinterpret_cast<double*>(out.data())),
                  "traces");
            result.expectation_terms = std::move(out);
        }
        if (request.want_counts) {
            result.actual_bytes += pow2(n) * sizeof(double);
            const std::vector<uint32_t> targets = flat_targets(request.measure_targets);
            if (request.is_sole_region) {
                std::vector<uint64_t> outcomes(std::max<uint64_t>(request.shots, 1)), counts(outcomes.size());
                uint64_t distinct = outcomes.size();
                check(mb2_dm_sample_readout(rho.s, n, ops.ops.data(), static_cast<uint32_t>(ops.ops.size()),
                                            request.shots, request.seed, targets.data(),
                                            static_cast<uint32_t>(request.measure_targets.size()), outcomes.data(),
                                            counts.data(), &distinct),
                      "sample");
                result.counts = histogram(outcomes, counts, request.shots == 0 ? 0 : distinct,
                                          request.bitstring_width);
            } else {
                result.counts_sampler = std::make_unique<DeviceRhoSampler>(
                    rho, n, request.measure_targets, request.bitstring_width,
                    noise::readout_targets(request.operations, request.measure_targets), request.shots);
            }
        }
        return result;
    }
};

class B200TrajectoryEngine : public SimulationEngine {
public:
    [[nodiscard]] std::string_view name() const override { return "trajectory_b200"; }
    [[nodiscard]] Engine engine_id() const override { return Engine::Trajectory; }
    [[nodiscard]] Backend backend() const override { return Backend::Cuda; }
    [[nodiscard]] EngineCapabilities capabilities() const override {
        return EngineCapabilities{/*counts=*/true, /*statevector=*/false, /*expectation=*/true};
    }

    // Work units as the reference counts them (trajectory_engine.cpp:
    // 351-404): per trajectory 2^n to reset, 2^(n+k) per operation, another
    // 2^(n+k) + 2^n per channel, 2^n per term; 2^n per trajectory for counts.
    [[nodiscard]] CostEstimate estimate(const EngineEstimateRequest& request) const override {
        if (request.want_statevector)
            return CostEstimate{false, 0, 0,
                                "the trajectory engine does not produce a statevector -- a noisy job has no single "
                                "final state",
                                {}};
        if (request.trajectories == 0)
            return CostEstimate{false, 0, 0, "the trajectory engine was given no trajectory count", {}};
        if (!b200_device_available()) return CostEstimate{false, 0, 0, "no B200 device is available", {}};
        const uint32_t n = request.num_qubits;
        if (n < 1 || n > 34) return CostEstimate{false, 0, 0, "trajectory_b200 holds 1..34 qubits", {}};
        const uint64_t states = pow2(n);
        uint64_t per = states, launches = 1;
        double passes = 1.0;
        for (const Operation& op : *request.operations) {
            const uint64_t k = operand_count(op);
            if (k == 0) continue;
            const bool channel = std::holds_alternative<ChannelOp>(op);
            if (channel && k > 3)
                return CostEstimate{false, 0, 0, "trajectory_b200: a channel on more than 3 qubits", {}};
            passes += channel ? 2.0 : 1.0;
            per += pow2(static_cast<uint32_t>(n + k));
            if (channel) per += pow2(static_cast<uint32_t>(n + k)) + states;
            launches += channel ? 5 : 1;
        }
        const uint64_t terms = request.want_expectation ? request.observable->terms.size() : 0;
        per += terms * states;
        uint64_t work = request.trajectories * per;
        if (request.want_counts) work += request.trajectories * states;
        const uint64_t device_bytes = 16 * states + (uint64_t{1} << 20);
        if (device_bytes > free_device_bytes())
            return CostEstimate{false, 0, 0, "trajectory_b200 needs " + std::to_string(device_bytes) + " device bytes",
                                {}};
        CostEstimate est{true, 16 * request.shots, work, "",
                         DeviceCost{device_bytes, 0, 16 * (terms + request.shots), request.trajectories * launches}};
        auto& tr = est.time.counts[static_cast<std::size_t>(Engine::Trajectory)];
        tr[0] = static_cast<double>(request.trajectories) * passes;
        tr[1] = static_cast<double>(work);
        tr[2] = static_cast<double>(request.trajectories);
        return est;
    }

    [[nodiscard]] EngineExecutionResult execute(const EngineExecutionRequest& request) const override {
        common::ensure(b200_device_available(), "B200TrajectoryEngine::execute: no device");
        common::ensure(!request.want_statevector, "trajectory: a statevector was requested; estimate() refuses that");
        common::ensure(request.is_sole_region,
                       "trajectory: the engine runs only as a sole region (docs/adr/0017 section 5)");
        const uint64_t trajectories = request.trajectories;
        common::ensure(trajectories >= 1, "trajectory: no trajectory count was given");
        common::ensure(!request.want_counts || request.shots <= trajectories,
                       "trajectory: more shots than trajectories");
        common::ensure(!request.want_expectation || trajectories >= 2,
                       "trajectory: an expectation needs at least 2 trajectories");
        const uint32_t n = request.num_qubits;
        Ops ops = to_mb2(request.operations);
        std::vector<uint64_t> xs, zs;
        std::vector<Complex> coefs;
        if (request.want_expectation) {
            for (const auto& [pauli, coefficient] : request.observable->terms) {
                xs.push_back(pauli.x_words[0]);
                zs.push_back(pauli.z_words[0]);
                coefs.push_back(coefficient);
            }
        }
        const uint32_t num_terms = static_cast<uint32_t>(xs.size());
        const std::vector<uint32_t> targets = flat_targets(request.measure_targets);
        const uint64_t shots = request.want_counts ? request.shots : 0;
        std::vector<Complex> means(std::max<uint32_t>(num_terms, 1));
        double standard_error = 0.0;
        std::vector<uint64_t> outcomes(std::max<uint64_t>(shots, 1)), counts(outcomes.size());
        uint64_t distinct = outcomes.size();
        // The state the run holds on the device, charged to the Device space.
        const common::MemoryLedger::Charge charge(16 * pow2(n), common::MemoryLedger::Space::Device);
        MonitorBridge bridge{request.monitor, nullptr};
        const int rc = mb2_trajectories_monitored(
            b200_context(), n, ops.ops.data(), static_cast<uint32_t>(ops.ops.size()), trajectories, request.seed,
            num_terms ? xs.data() : nullptr, num_terms ? zs.data() : nullptr,
            num_terms ? reinterpret_cast<const double*>(coefs.data()) : nullptr, num_terms,
            reinterpret_cast<double*>(means.data()), &standard_error, shots,
            targets.empty() ? nullptr : targets.data(), static_cast<uint32_t>(request.measure_targets.size()),
            outcomes.data(), counts.data(), &distinct, request.monitor != nullptr ? &on_boundary : nullptr, &bridge);
        if (bridge.error) std::rethrow_exception(bridge.error);
        check(rc, "trajectories");
        EngineExecutionResult result;
        result.statistical = true;
        result.actual_bytes = 16 * pow2(n);
        if (request.want_counts) result.counts = histogram(outcomes, counts, shots == 0 ? 0 : distinct,
                                                           request.bitstring_width);
        if (request.want_expectation) {
            means.resize(num_terms);
            result.expectation_terms = std::move(means);
            result.expectation_standard_error = standard_error;
        }
        return result;
    }
};

}  // namespace

const SimulationEngine& b200_density_matrix_engine() {
    static const B200DensityMatrixEngine engine;
    return engine;
}

const SimulationEngine& b200_trajectory_engine() {
    static const B200TrajectoryEngine engine;
    return engine;
}

}  // namespace menos::engines::dense_b200
