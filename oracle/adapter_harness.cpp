// adapter_harness.cpp -- TEST INFRASTRUCTURE, not product code.
//
// Drives the reference-side binding (menos_b200/integration/
// b200_dense_engine.cpp and b200_noisy_engines.cpp, the
// menos::SimulationEngines the reference would register) and the
// reference's own CPU engines (DenseEngine, src/engines/dense/
// dense_engine.cpp:333-400; DensityMatrixEngine; TrajectoryEngine) through
// one request shape, so
// tests can run the reference's CPU/CUDA differential cases
// (tests/api/cpu_cuda_differential_test.cpp:132-421) against the adapter
// itself.  oracle/Makefile links it with the adapter, the reference's CPU
// engine objects and libmenos_b200.so into oracle/_ref/libmenos_adapter.so.
//
//   ah_execute       one EngineExecutionRequest through either engine, under
//                    an installed MemoryLedger (peaks reported), with an
//                    optional monitor that abandons at a boundary count; a
//                    Factorized region's sampler is drawn from with its own Rng
//   ah_estimate      EngineEstimateRequest through either engine
//   ah_calibration   measure_b200_calibration()
//   ah_serve_with_ledger  the serving loop admitting through the adapter's
//                    ServerLedger (device bytes charged to a MemoryLedger)
#include <chrono>
#include <complex>
#include <cstdint>
#include <cstring>
#include <exception>
#include <span>
#include <string>
#include <vector>

#include "common/error.h"
#include "common/memory_ledger.h"
#include "common/rng.h"
#include "engines/dense/dense_engine.h"
#include "ir/gate_table.h"
#include "menos/bitstring.h"
#include "menos/circuit.h"
#include "menos/observable.h"
#include "menos/simulation_engine.h"
#include "plan/cuda_calibration.h"

#include "../include/mb2.h"

#include "../menos_b200/integration/b200_dense_engine.h"
#include "../menos_b200/integration/b200_noisy_engines.h"
#include "engines/density_matrix/density_matrix_engine.h"
#include "engines/trajectory/trajectory_engine.h"

namespace {

using C = std::complex<double>;

menos::Operation to_operation(const mb2_op& op) {
    if (op.opcode == MB2_MEASURE) {
        menos::MeasureOp m{op.qubits[0], op.clbit};
        if (op.matrix != nullptr)
            m.readout_error = menos::ReadoutError{{op.matrix[0], op.matrix[1], op.matrix[2], op.matrix[3]}};
        return m;
    }
    std::vector<menos::QubitId> qubits(op.qubits, op.qubits + op.num_qubits);
    if (op.opcode == MB2_CHANNEL) {
        const std::size_t entries = std::size_t{1} << (2 * op.num_qubits);
        std::vector<std::vector<C>> kraus(op.reserved, std::vector<C>(entries));
        for (std::size_t t = 0; t < op.reserved; ++t)
            for (std::size_t i = 0; i < entries; ++i)
                kraus[t][i] = C{op.matrix[2 * (t * entries + i)], op.matrix[2 * (t * entries + i) + 1]};
        return menos::ChannelOp{std::move(qubits), std::move(kraus)};
    }
    if (op.opcode == MB2_UNITARY) {
        const std::size_t dim = std::size_t{1} << op.num_qubits;
        std::vector<C> m(dim * dim);
        for (std::size_t i = 0; i < dim * dim; ++i) m[i] = C{op.matrix[2 * i], op.matrix[2 * i + 1]};
        return menos::UnitaryOp{std::move(qubits), std::move(m)};
    }
    const auto opcode = static_cast<menos::Opcode>(op.opcode);
    const int np = menos::ir::gate_info(opcode).num_params;
    return menos::GateOp{opcode, std::move(qubits), std::vector<double>(op.params, op.params + np)};
}

std::uint64_t bits_of(const menos::BitString& b) {
    std::uint64_t v = 0;
    for (std::uint32_t i = 0; i < b.num_bits() && i < 64; ++i)
        if (b.test(i)) v |= std::uint64_t{1} << i;
    return v;
}

// Abandons at the safe boundary whose count reaches `at` (the reference's
// ExecutionMonitor contract: throw to abandon).
class CountingMonitor final : public menos::ExecutionMonitor {
public:
    explicit CountingMonitor(std::int64_t at) : at_(at) {}
    void at_safe_boundary(std::uint64_t crossed) const override {
        ++calls_;
        if (at_ >= 0 && static_cast<std::int64_t>(crossed) >= at_) throw menos::common::InternalError("abandoned");
    }
    mutable std::uint64_t calls_ = 0;

private:
    std::int64_t at_;
};

// 0/1: the reference's CPU DenseEngine / the dense binding; 2/3: the
// reference's DensityMatrixEngine / its binding; 4/5: the reference's
// TrajectoryEngine / its binding.
const menos::SimulationEngine& engine_of(int which) {
    static const menos::engines::dense::DenseEngine cpu;
    static const menos::engines::density_matrix::DensityMatrixEngine dm;
    static const menos::engines::trajectory::TrajectoryEngine traj;
    switch (which) {
        case 0: return cpu;
        case 2: return dm;
        case 3: return menos::engines::dense_b200::b200_density_matrix_engine();
        case 4: return traj;
        case 5: return menos::engines::dense_b200::b200_trajectory_engine();
        default: return menos::engines::dense_b200::b200_dense_engine();
    }
}

void set_error(char* err, std::size_t len, const char* what) {
    if (err == nullptr || len == 0) return;
    std::strncpy(err, what, len - 1);
    err[len - 1] = '\0';
}

}  // namespace

extern "C" {

// The request, as plain C.  abandon_at < 0: no monitor.
typedef struct ah_request {
    std::uint32_t num_qubits;
    std::uint32_t num_ops;
    const mb2_op* ops;
    std::int32_t fuse_gates, want_statevector, want_counts, want_expectation, is_sole_region, reserved;
    std::uint64_t shots, seed;
    const std::uint32_t* targets;  // (qubit, clbit) pairs
    std::uint32_t num_targets, bitstring_width;
    double global_phase;
    std::uint64_t budget_bytes;
    const std::uint64_t* x_masks;
    const std::uint64_t* z_masks;
    std::uint32_t num_terms, reserved2;
    std::int64_t abandon_at;
    std::uint64_t trajectories;   // the trajectory engines' count
    const double* coefs;          // complex coefficient per term (2 doubles), or NULL for 1
} ah_request;

typedef struct ah_result {
    double* statevector;          // 2 * 2^n doubles, or NULL
    std::uint64_t* outcomes;      // sole region: histogram keys (ascending)
    std::uint64_t* counts;
    std::uint64_t capacity;       // of outcomes/counts and of draws
    std::uint64_t num_outcomes;
    double* expectation;          // 2 * num_terms doubles
    std::uint64_t draws;          // Factorized region: draws from counts_sampler with Rng(draw_seed)
    std::uint64_t draw_seed;
    std::uint64_t* drawn;         // the drawn outcomes, in draw order
    std::uint64_t actual_bytes, peak_host, peak_device, monitor_calls;
    std::int32_t has_statevector, has_counts, has_sampler, has_expectation;
    double seconds;               // wall time of execute()
    double standard_error;        // the result's expectation_standard_error, or -1
    std::int32_t statistical, reserved;
} ah_result;

// 0 ok; 1 ResourceExceeded; 2 InternalError (the monitor's abandon included);
// 3 any other exception.
int ah_execute(int which, const ah_request* rq, ah_result* res, char* err, std::size_t errlen) {
    try {
        std::vector<menos::Operation> ops;
        for (std::uint32_t i = 0; i < rq->num_ops; ++i) ops.push_back(to_operation(rq->ops[i]));
        std::vector<std::pair<menos::QubitId, menos::ClbitId>> targets;
        for (std::uint32_t t = 0; t < rq->num_targets; ++t)
            targets.emplace_back(rq->targets[2 * t], rq->targets[2 * t + 1]);
        menos::Observable obs;
        for (std::uint32_t t = 0; t < rq->num_terms; ++t) {
            menos::PauliString p;
            p.num_qubits = rq->num_qubits;
            p.x_words.assign(1, rq->x_masks[t]);
            p.z_words.assign(1, rq->z_masks[t]);
            const C coef = rq->coefs != nullptr ? C{rq->coefs[2 * t], rq->coefs[2 * t + 1]} : C{1.0, 0.0};
            obs.terms.emplace_back(std::move(p), coef);
        }
        CountingMonitor monitor(rq->abandon_at);
        menos::EngineExecutionRequest request{
            .num_qubits = rq->num_qubits,
            .operations = ops,
            .want_statevector = rq->want_statevector != 0,
            .want_counts = rq->want_counts != 0,
            .want_expectation = rq->want_expectation != 0,
            .shots = rq->shots,
            .measure_targets = targets,
            .bitstring_width = rq->bitstring_width,
            .seed = rq->seed,
            .global_phase = rq->global_phase,
            .budget_bytes = rq->budget_bytes,
            .is_sole_region = rq->is_sole_region != 0,
            .observable = rq->want_expectation ? &obs : nullptr,
        };
        request.fuse_gates = rq->fuse_gates != 0;
        request.trajectories = rq->trajectories;
        if (rq->abandon_at >= 0) request.monitor = &monitor;
        menos::common::MemoryLedger ledger;
        {
            menos::common::MemoryLedger::Scope scope(ledger);
            menos::EngineExecutionResult r;
            try {
                const auto t0 = std::chrono::steady_clock::now();
                r = engine_of(which).execute(request);
                res->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            } catch (...) {
                res->monitor_calls = monitor.calls_;
                throw;
            }
            res->monitor_calls = monitor.calls_;
            res->actual_bytes = r.actual_bytes;
            res->has_statevector = r.statevector.has_value();
            if (r.statevector && res->statevector)
                std::memcpy(res->statevector, r.statevector->data(), r.statevector->size() * sizeof(C));
            res->has_counts = r.counts.has_value();
            res->num_outcomes = 0;
            if (r.counts) {
                for (const auto& [key, c] : *r.counts) {
                    if (res->num_outcomes >= res->capacity) break;
                    res->outcomes[res->num_outcomes] = bits_of(key);
                    res->counts[res->num_outcomes] = c;
                    ++res->num_outcomes;
                }
            }
            res->has_sampler = r.counts_sampler != nullptr;
            if (r.counts_sampler && res->drawn) {
                menos::common::Rng rng(res->draw_seed);
                for (std::uint64_t i = 0; i < res->draws && i < res->capacity; ++i)
                    res->drawn[i] = bits_of(r.counts_sampler->sample_one(rng));
            }
            res->statistical = r.statistical ? 1 : 0;
            res->standard_error = r.expectation_standard_error.value_or(-1.0);
            res->has_expectation = r.expectation_terms.has_value();
            if (r.expectation_terms && res->expectation)
                std::memcpy(res->expectation, r.expectation_terms->data(), r.expectation_terms->size() * sizeof(C));
        }
        res->peak_host = ledger.peak_host_bytes();
        res->peak_device = ledger.peak_device_bytes();
        return 0;
    } catch (const menos::common::ResourceExceeded& e) {
        set_error(err, errlen, e.what());
        return 1;
    } catch (const menos::common::InternalError& e) {
        set_error(err, errlen, e.what());
        return 2;
    } catch (const std::exception& e) {
        set_error(err, errlen, e.what());
        return 3;
    }
}

// out: feasible, estimated_peak_bytes, estimated_work_units, device_bytes,
// h2d_bytes, d2h_bytes, kernel_launches, host pass count (time component 0).
int ah_estimate(int which, const ah_request* rq, std::uint64_t* out, char* reason, std::size_t len) {
    try {
        std::vector<menos::Operation> ops;
        for (std::uint32_t i = 0; i < rq->num_ops; ++i) ops.push_back(to_operation(rq->ops[i]));
        menos::Observable obs;
        for (std::uint32_t t = 0; t < rq->num_terms; ++t) {
            menos::PauliString p;
            p.num_qubits = rq->num_qubits;
            p.x_words.assign(1, rq->x_masks[t]);
            p.z_words.assign(1, rq->z_masks[t]);
            obs.terms.emplace_back(std::move(p), C{1.0, 0.0});
        }
        menos::EngineEstimateRequest request{
            .num_qubits = rq->num_qubits,
            .operations = &ops,
            .want_statevector = rq->want_statevector != 0,
            .want_counts = rq->want_counts != 0,
            .want_expectation = rq->want_expectation != 0,
            .observable = rq->want_expectation ? &obs : nullptr,
        };
        request.shots = rq->shots;
        request.bitstring_width = rq->bitstring_width;
        request.is_sole_region = rq->is_sole_region != 0;
        request.fuse_gates = rq->fuse_gates != 0;
        request.trajectories = rq->trajectories;
        const menos::CostEstimate e = engine_of(which).estimate(request);
        out[0] = e.feasible;
        out[1] = e.estimated_peak_bytes;
        out[2] = e.estimated_work_units;
        out[3] = e.device.device_bytes;
        out[4] = e.device.host_to_device_bytes;
        out[5] = e.device.device_to_host_bytes;
        out[6] = e.device.kernel_launches;
        const menos::Engine id = engine_of(which).engine_id();
        out[7] = static_cast<std::uint64_t>(e.time.counts[static_cast<std::size_t>(id)][0]);
        set_error(reason, len, e.infeasible_reason.c_str());
        return 0;
    } catch (const std::exception& e) {
        set_error(reason, len, e.what());
        return 3;
    }
}

// out: present, device_total_bytes, device_available_bytes, h2d B/s, d2h B/s,
// kernel_launch_seconds, execution_seconds, device_work_units_per_second.
int ah_calibration(double* out) {
    const menos::plan::CudaCalibration c = menos::engines::dense_b200::measure_b200_calibration();
    out[0] = c.present ? 1.0 : 0.0;
    out[1] = static_cast<double>(c.device_total_bytes);
    out[2] = static_cast<double>(c.device_available_bytes);
    out[3] = c.host_to_device_bytes_per_second;
    out[4] = c.device_to_host_bytes_per_second;
    out[5] = c.kernel_launch_seconds;
    out[6] = c.execution_seconds;
    out[7] = c.device_work_units_per_second;
    return 0;
}

// The serving loop with its admissions charged to a MemoryLedger through the
// adapter's ServerLedger: `count` requests (brick circuits of qubits[i]
// qubits, depth 8, <Z_0> each) on a server of `slots` slots; the ledger
// refuses beyond `device_limit`.  out: peak device bytes, live device bytes
// after the last completion, completions with status 0, the largest single
// admission's bytes (the server's own count).
int ah_serve_with_ledger(const std::uint32_t* qubits, std::uint32_t count, std::uint32_t slots,
                         std::uint64_t device_limit, std::uint64_t* out) {
    mb2_context* ctx = nullptr;
    if (mb2_context_create(0, &ctx) != MB2_OK) return -1;
    menos::common::MemoryLedger ledger;
    int rc = 0;
    {
        menos::engines::dense_b200::ServerLedger hook(ledger, device_limit);
        mb2_server* srv = nullptr;
        mb2_server_options so{0, slots, 0};
        if (mb2_server_create(ctx, &so, &srv) != MB2_OK) {
            mb2_context_destroy(ctx);
            return -2;
        }
        if (hook.attach(srv) != MB2_OK) rc = -3;
        std::vector<std::vector<mb2_op>> programs(count);
        const std::uint64_t z0 = 1, x0 = 0;
        const double one = 1.0;
        std::uint64_t ok = 0;
        for (std::uint32_t i = 0; i < count && rc == 0; ++i) {
            const std::uint32_t n = qubits[i];
            for (std::uint32_t layer = 0; layer < 8; ++layer) {
                for (std::uint32_t q = 0; q < n; ++q) {
                    mb2_op o{};
                    o.opcode = MB2_U;
                    o.num_qubits = 1;
                    o.qubits[0] = q;
                    o.params[0] = 0.1 * (q + 1) + layer;
                    o.params[1] = 0.2 * q;
                    o.params[2] = 0.3 * layer;
                    programs[i].push_back(o);
                }
                for (std::uint32_t q = layer & 1u; q + 1 < n; q += 2) {
                    mb2_op o{};
                    o.opcode = MB2_CZ;
                    o.num_qubits = 2;
                    o.qubits[0] = q;
                    o.qubits[1] = q + 1;
                    programs[i].push_back(o);
                }
            }
            mb2_request rq{};
            rq.ops = programs[i].data();
            rq.num_ops = static_cast<std::uint32_t>(programs[i].size());
            rq.num_qubits = n;
            rq.fuse_gates = 1;
            rq.output = MB2_OUT_EXPECTATION;
            rq.num_terms = 1;
            rq.x_masks = &x0;
            rq.z_masks = &z0;
            rq.coefs = &one;
            rq.precision = MB2_C128;
            std::uint64_t ticket = 0;
            if (mb2_server_submit(srv, &rq, &ticket) != MB2_OK) rc = -4;
        }
        std::uint32_t got_total = 0;
        for (int spins = 0; got_total < count && rc == 0 && spins < 6000; ++spins) {
            mb2_completion done[16];
            std::uint32_t got = 0;
            const int prc = mb2_server_poll(srv, done, 16, &got, 100);
            if (prc != MB2_OK && prc != MB2_ERR_TIMEOUT) rc = -5;
            for (std::uint32_t k = 0; k < got; ++k) {
                if (done[k].status == MB2_OK) ++ok;
                mb2_server_release(srv, done[k].ticket);
            }
            got_total += got;
        }
        mb2_server_destroy(srv);
        out[0] = ledger.peak_device_bytes();
        out[1] = ledger.live_device_bytes();
        out[2] = ok;
        out[3] = got_total;
    }
    mb2_context_destroy(ctx);
    return rc;
}

}  // extern "C"
