// ref_shim.cpp -- TEST INFRASTRUCTURE, not product code.
//
// A C-ABI wrapper around the reference MENOS CPU dense engine, compiled
// together with the reference's own CPU sources (see oracle/Makefile) into
// oracle/_ref/libmenos_ref.so.  Only tests/, the smoke check and bench.py's
// CPU-baseline leg load it, and only as the checker / timed CPU baseline.
//
// Every function forwards to the reference implementation unchanged:
//   ref_generate_matrix      -> ir::generate_matrix        (src/ir/gate_table.cpp:260)
//   ref_apply_matrix         -> kernels::cpu::apply_matrix (src/kernels/cpu/dense_kernels.cpp:427)
//   ref_apply_matrix_generic -> kernels::cpu::apply_matrix_generic (:465)
//   ref_expectation_of_term  -> kernels::cpu::expectation_of_term  (:562)
//   ref_sample               -> engines::dense::sample     (src/engines/dense/sample.cpp:91)
//   ref_uniforms             -> common::Rng::next_uniform  (src/common/rng.cpp:176)
//   ref_plan_fusion          -> ir::plan_fusion            (src/ir/fuse_gates.cpp:190)
//   ref_fused_block_matrix   -> engines::dense::fused_block_matrix (src/engines/dense/fused_block.cpp:61)
//   ref_run_dense            -> engines::dense::DenseEngine::execute (src/engines/dense/dense_engine.cpp:333)
//   ref_run_plan             -> initialize + engines::dense::apply_blocks with the dense
//                               engine's apply_matrix, for a plan given as ir::FusionPlan's
//                               arrays (src/engines/dense/dense_engine.cpp:100-112)
#include <algorithm>
#include <optional>
#include <chrono>
#include <complex>
#include <cstdint>
#include <cstring>
#include <exception>
#include <span>
#include <string>
#include <vector>

#include "common/rng.h"
#include "engines/dense/apply_matrix.h"
#include "engines/density_matrix/density_matrix_engine.h"
#include "engines/trajectory/trajectory_engine.h"
#include "engines/dense/dense_engine.h"
#ifdef MENOS_REF_CUDA
#include "engines/dense_cuda/cuda_dense_engine.h"
#endif
#include "engines/dense/fused_block.h"
#include "engines/dense/sample.h"
#include "engines/dense_tiered/pass_plan.h"
#include "ir/fuse_gates.h"
#include "ir/gate_table.h"
#include "kernels/cpu/dense_kernel_table.h"
#include "kernels/dense_kernels.h"
#include "menos/bitstring.h"
#include "menos/circuit.h"
#include "menos/observable.h"
#include "menos/simulation_engine.h"

#include "../include/mb2.h"

namespace {

using C = std::complex<double>;
thread_local std::string g_error;

std::span<C> as_span(double* p, std::uint64_t n) {
    return {reinterpret_cast<C*>(p), static_cast<std::size_t>(n)};
}
std::span<const C> as_cspan(const double* p, std::uint64_t n) {
    return {reinterpret_cast<const C*>(p), static_cast<std::size_t>(n)};
}

menos::Operation to_operation(const mb2_op& op) {
    if (op.opcode == MB2_MEASURE) {
        menos::MeasureOp m{op.qubits[0], op.clbit};
        if (op.matrix != nullptr) {
            m.readout_error = menos::ReadoutError{{op.matrix[0], op.matrix[1], op.matrix[2], op.matrix[3]}};
        }
        return m;
    }
    std::vector<menos::QubitId> qubits(op.qubits, op.qubits + op.num_qubits);
    if (op.opcode == MB2_CHANNEL) {
        const std::size_t entries = std::size_t{1} << (2 * op.num_qubits);
        std::vector<std::vector<C>> kraus(op.reserved, std::vector<C>(entries));
        for (std::size_t t = 0; t < op.reserved; ++t) {
            for (std::size_t i = 0; i < entries; ++i) {
                const double* z = op.matrix + 2 * (t * entries + i);
                kraus[t][i] = C{z[0], z[1]};
            }
        }
        return menos::ChannelOp{std::move(qubits), std::move(kraus)};
    }
    if (op.opcode == MB2_UNITARY) {
        const std::size_t dim = std::size_t{1} << op.num_qubits;
        std::vector<C> m(dim * dim);
        for (std::size_t i = 0; i < dim * dim; ++i) {
            m[i] = C{op.matrix[2 * i], op.matrix[2 * i + 1]};
        }
        return menos::UnitaryOp{std::move(qubits), std::move(m)};
    }
    const auto opcode = static_cast<menos::Opcode>(op.opcode);
    const int np = menos::ir::gate_info(opcode).num_params;
    return menos::GateOp{opcode, std::move(qubits), std::vector<double>(op.params, op.params + np)};
}

std::uint64_t bits_of(const menos::BitString& b) {
    std::uint64_t v = 0;
    for (std::uint32_t i = 0; i < b.num_bits() && i < 64; ++i) {
        if (b.test(i)) {
            v |= std::uint64_t{1} << i;
        }
    }
    return v;
}

}  // namespace

extern "C" {

const char* ref_last_error() {
    return g_error.c_str();
}

int ref_generate_matrix(int opcode, const double* params, double* out, std::uint32_t out_len) {
    try {
        const auto op = static_cast<menos::Opcode>(opcode);
        const int np = menos::ir::gate_info(op).num_params;
        const std::vector<C> m = menos::ir::generate_matrix(op, std::span<const double>(params, np));
        if (2 * m.size() > out_len) {
            return -1;
        }
        std::memcpy(out, m.data(), m.size() * sizeof(C));
        return static_cast<int>(m.size());
    } catch (const std::exception& e) {
        g_error = e.what();
        return -1;
    }
}

int ref_apply_matrix(double* state, std::uint64_t n_amps, const double* matrix,
                     const std::uint32_t* operands, std::uint32_t k, std::uint32_t threads) {
    try {
        const std::size_t dim = std::size_t{1} << k;
        menos::kernels::cpu::apply_matrix(as_span(state, n_amps), as_cspan(matrix, dim * dim),
                                          std::span<const std::uint32_t>(operands, k), threads);
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return -1;
    }
}

int ref_apply_matrix_generic(double* state, std::uint64_t n_amps, const double* matrix,
                             const std::uint32_t* operands, std::uint32_t k,
                             std::uint32_t threads) {
    try {
        const std::size_t dim = std::size_t{1} << k;
        menos::kernels::cpu::apply_matrix_generic(as_span(state, n_amps),
                                                  as_cspan(matrix, dim * dim),
                                                  std::span<const std::uint32_t>(operands, k),
                                                  threads);
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return -1;
    }
}

void ref_expectation_of_term(const double* state, std::uint64_t n_amps, std::uint64_t x,
                             std::uint64_t z, double* out) {
    const C v = menos::kernels::cpu::expectation_of_term(as_cspan(state, n_amps), x, z);
    out[0] = v.real();
    out[1] = v.imag();
}

void ref_uniforms(std::uint64_t seed, std::uint64_t n, double* out) {
    menos::common::Rng rng(seed);
    for (std::uint64_t i = 0; i < n; ++i) {
        out[i] = rng.next_uniform();
    }
}

// Returns the number of distinct outcomes (or -1 when cap is too small).
std::int64_t ref_sample(const double* state, std::uint64_t n_amps, std::uint64_t shots,
                        std::uint64_t seed, const std::uint32_t* targets, std::uint32_t n_targets,
                        std::uint32_t width, std::uint64_t* out_outcomes, std::uint64_t* out_counts,
                        std::uint64_t cap) {
    std::vector<std::pair<std::uint32_t, std::uint32_t>> t(n_targets);
    for (std::uint32_t i = 0; i < n_targets; ++i) {
        t[i] = {targets[2 * i], targets[2 * i + 1]};
    }
    const auto counts = menos::engines::dense::sample(as_cspan(state, n_amps), shots, seed, t, width);
    if (counts.size() > cap) {
        return -1;
    }
    std::uint64_t i = 0;
    for (const auto& [key, count] : counts) {
        out_outcomes[i] = bits_of(key);
        out_counts[i] = count;
        ++i;
    }
    return static_cast<std::int64_t>(counts.size());
}

// The fusion plan of ops: returns the block count; order/block_begin/
// block_qubits/qubits_begin are filled when non-null (capacities: ops,
// ops + 1, 64 * ops, ops + 1).
std::int64_t ref_plan_fusion(const mb2_op* ops, std::uint32_t n_ops, std::uint32_t* order,
                             std::uint32_t* block_begin, std::uint32_t* block_qubits,
                             std::uint32_t* qubits_begin) {
    std::vector<menos::Operation> v;
    v.reserve(n_ops);
    for (std::uint32_t i = 0; i < n_ops; ++i) {
        v.push_back(to_operation(ops[i]));
    }
    const menos::ir::FusionPlan plan = menos::ir::plan_fusion(v);
    if (order != nullptr) {
        std::copy(plan.order.begin(), plan.order.end(), order);
        std::copy(plan.block_begin.begin(), plan.block_begin.end(), block_begin);
        std::copy(plan.block_qubits.begin(), plan.block_qubits.end(), block_qubits);
        std::copy(plan.qubits_begin.begin(), plan.qubits_begin.end(), qubits_begin);
    }
    return static_cast<std::int64_t>(plan.block_count());
}

// Block `block`'s fused matrix (row-major, interleaved); returns its
// dimension.
int ref_fused_block_matrix(const mb2_op* ops, std::uint32_t n_ops, std::uint32_t block,
                           double* out, std::uint32_t out_len) {
    std::vector<menos::Operation> v;
    for (std::uint32_t i = 0; i < n_ops; ++i) {
        v.push_back(to_operation(ops[i]));
    }
    const menos::ir::FusionPlan plan = menos::ir::plan_fusion(v);
    const std::vector<C> m = menos::engines::dense::fused_block_matrix(plan, block, v);
    if (2 * m.size() > out_len) {
        return -1;
    }
    std::memcpy(out, m.data(), m.size() * sizeof(C));
    std::size_t dim = 1;
    while (dim * dim < m.size()) {
        dim <<= 1;
    }
    return static_cast<int>(dim);
}

// DenseEngine::execute on ops.  Outputs are filled when their pointers are
// non-null: statevector (2 * 2^n doubles), counts (outcomes/counts with
// capacity *n_outcomes, updated), expectation terms (2 * n_terms doubles).
// seconds_out (optional) receives the wall time of execute() alone.
}  // extern "C"

namespace {

int run_engine(const menos::SimulationEngine& engine, std::uint32_t num_qubits, const mb2_op* ops,
               std::uint32_t n_ops, double global_phase, int fuse_gates, std::uint32_t threads,
               double* statevector, std::uint64_t shots, std::uint64_t seed, const std::uint32_t* targets,
               std::uint32_t n_targets, std::uint32_t width, std::uint64_t* out_outcomes,
               std::uint64_t* out_counts, std::uint64_t* n_outcomes, const std::uint64_t* x_masks,
               const std::uint64_t* z_masks, std::uint32_t n_terms, double* terms_out, double* seconds_out) {
    try {
        std::vector<menos::Operation> v;
        v.reserve(n_ops);
        for (std::uint32_t i = 0; i < n_ops; ++i) {
            v.push_back(to_operation(ops[i]));
        }
        std::vector<std::pair<menos::QubitId, menos::ClbitId>> t(n_targets);
        for (std::uint32_t i = 0; i < n_targets; ++i) {
            t[i] = {targets[2 * i], targets[2 * i + 1]};
        }
        menos::Observable obs;
        for (std::uint32_t i = 0; i < n_terms; ++i) {
            menos::PauliString p{num_qubits, {x_masks[i]}, {z_masks[i]}};
            obs.terms.emplace_back(std::move(p), C{1.0, 0.0});
        }
        menos::EngineExecutionRequest req{};
        req.num_qubits = num_qubits;
        req.operations = v;
        req.want_statevector = statevector != nullptr;
        req.want_counts = out_outcomes != nullptr && shots > 0;
        req.want_expectation = terms_out != nullptr && n_terms > 0;
        req.shots = shots;
        req.measure_targets = t;
        req.bitstring_width = width;
        req.seed = seed;
        req.global_phase = global_phase;
        req.budget_bytes = ~std::uint64_t{0};
        req.is_sole_region = true;
        req.observable = req.want_expectation ? &obs : nullptr;
        req.max_threads = threads == 0 ? menos::common::default_thread_count() : threads;
        req.fuse_gates = fuse_gates != 0;
        const auto t0 = std::chrono::steady_clock::now();
        menos::EngineExecutionResult res = engine.execute(req);
        const auto t1 = std::chrono::steady_clock::now();
        if (seconds_out != nullptr) {
            *seconds_out = std::chrono::duration<double>(t1 - t0).count();
        }
        if (statevector != nullptr) {
            std::memcpy(statevector, res.statevector->data(), res.statevector->size() * sizeof(C));
        }
        if (req.want_counts) {
            std::uint64_t i = 0;
            for (const auto& [key, count] : *res.counts) {
                if (i >= *n_outcomes) {
                    g_error = "outcome capacity exceeded";
                    return -1;
                }
                out_outcomes[i] = bits_of(key);
                out_counts[i] = count;
                ++i;
            }
            *n_outcomes = i;
        }
        if (req.want_expectation) {
            for (std::uint32_t i = 0; i < n_terms; ++i) {
                terms_out[2 * i] = (*res.expectation_terms)[i].real();
                terms_out[2 * i + 1] = (*res.expectation_terms)[i].imag();
            }
        }
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return -1;
    }
}

}  // namespace

extern "C" {

int ref_run_dense(std::uint32_t num_qubits, const mb2_op* ops, std::uint32_t n_ops,
                  double global_phase, int fuse_gates, std::uint32_t threads,
                  double* statevector, std::uint64_t shots, std::uint64_t seed,
                  const std::uint32_t* targets, std::uint32_t n_targets, std::uint32_t width,
                  std::uint64_t* out_outcomes, std::uint64_t* out_counts,
                  std::uint64_t* n_outcomes, const std::uint64_t* x_masks,
                  const std::uint64_t* z_masks, std::uint32_t n_terms, double* terms_out,
                  double* seconds_out) {
    const menos::engines::dense::DenseEngine engine;
    return run_engine(engine, num_qubits, ops, n_ops, global_phase, fuse_gates, threads, statevector, shots, seed,
                      targets, n_targets, width, out_outcomes, out_counts, n_outcomes, x_masks, z_masks, n_terms,
                      terms_out, seconds_out);
}

#ifdef MENOS_REF_CUDA
// CudaDenseEngine::execute (src/engines/dense_cuda/cuda_dense_engine.cpp:
// 325-412) on the same request; arguments as ref_run_dense's.
int ref_run_cuda(std::uint32_t num_qubits, const mb2_op* ops, std::uint32_t n_ops, double global_phase,
                 int fuse_gates, std::uint32_t threads, double* statevector, std::uint64_t shots,
                 std::uint64_t seed, const std::uint32_t* targets, std::uint32_t n_targets, std::uint32_t width,
                 std::uint64_t* out_outcomes, std::uint64_t* out_counts, std::uint64_t* n_outcomes,
                 const std::uint64_t* x_masks, const std::uint64_t* z_masks, std::uint32_t n_terms,
                 double* terms_out, double* seconds_out) {
    if (!menos::engines::dense_cuda::cuda_device_available()) {
        g_error = "no CUDA device";
        return -1;
    }
    const menos::engines::dense_cuda::CudaDenseEngine engine;
    return run_engine(engine, num_qubits, ops, n_ops, global_phase, fuse_gates, threads, statevector, shots, seed,
                      targets, n_targets, width, out_outcomes, out_counts, n_outcomes, x_masks, z_masks, n_terms,
                      terms_out, seconds_out);
}
#endif

// DensityMatrixEngine::execute on ops (src/engines/density_matrix/
// density_matrix_engine.cpp): counts (capacity *n_outcomes, updated) and
// expectation terms (2 * n_terms doubles) when their pointers are non-null;
// seconds_out (optional) the wall time of execute() alone.
int ref_run_dm(std::uint32_t num_qubits, const mb2_op* ops, std::uint32_t n_ops, std::uint32_t threads,
               std::uint64_t shots, std::uint64_t seed, const std::uint32_t* targets, std::uint32_t n_targets,
               std::uint32_t width, std::uint64_t* out_outcomes, std::uint64_t* out_counts,
               std::uint64_t* n_outcomes, const std::uint64_t* x_masks, const std::uint64_t* z_masks,
               std::uint32_t n_terms, double* terms_out, double* seconds_out) {
    try {
        std::vector<menos::Operation> v;
        v.reserve(n_ops);
        for (std::uint32_t i = 0; i < n_ops; ++i) {
            v.push_back(to_operation(ops[i]));
        }
        std::vector<std::pair<menos::QubitId, menos::ClbitId>> t(n_targets);
        for (std::uint32_t i = 0; i < n_targets; ++i) {
            t[i] = {targets[2 * i], targets[2 * i + 1]};
        }
        menos::Observable obs;
        for (std::uint32_t i = 0; i < n_terms; ++i) {
            menos::PauliString p{num_qubits, {x_masks[i]}, {z_masks[i]}};
            obs.terms.emplace_back(std::move(p), C{1.0, 0.0});
        }
        menos::EngineExecutionRequest req{};
        req.num_qubits = num_qubits;
        req.operations = v;
        req.want_statevector = false;
        req.want_counts = out_outcomes != nullptr && shots > 0;
        req.want_expectation = terms_out != nullptr && n_terms > 0;
        req.shots = shots;
        req.measure_targets = t;
        req.bitstring_width = width;
        req.seed = seed;
        req.budget_bytes = ~std::uint64_t{0};
        req.is_sole_region = true;
        req.observable = req.want_expectation ? &obs : nullptr;
        req.max_threads = threads == 0 ? menos::common::default_thread_count() : threads;
        menos::engines::density_matrix::DensityMatrixEngine engine;
        const auto t0 = std::chrono::steady_clock::now();
        menos::EngineExecutionResult res = engine.execute(req);
        const auto t1 = std::chrono::steady_clock::now();
        if (seconds_out != nullptr) {
            *seconds_out = std::chrono::duration<double>(t1 - t0).count();
        }
        if (req.want_counts) {
            std::uint64_t i = 0;
            for (const auto& [key, count] : *res.counts) {
                if (i >= *n_outcomes) {
                    g_error = "outcome capacity exceeded";
                    return -1;
                }
                out_outcomes[i] = bits_of(key);
                out_counts[i] = count;
                ++i;
            }
            *n_outcomes = i;
        }
        if (req.want_expectation) {
            for (std::uint32_t i = 0; i < n_terms; ++i) {
                terms_out[2 * i] = (*res.expectation_terms)[i].real();
                terms_out[2 * i + 1] = (*res.expectation_terms)[i].imag();
            }
        }
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return -1;
    }
}

// TrajectoryEngine::execute on ops (src/engines/trajectory/
// trajectory_engine.cpp:424-494): `trajectories` runs from `seed`; term
// means (2 * n_terms doubles, coefficients `coefs` as complex pairs), the
// standard error, and counts (capacity *n_outcomes, updated) when requested.
int ref_run_trajectories(std::uint32_t num_qubits, const mb2_op* ops, std::uint32_t n_ops,
                         std::uint64_t trajectories, std::uint64_t seed, const std::uint64_t* x_masks,
                         const std::uint64_t* z_masks, const double* coefs, std::uint32_t n_terms, double* terms_out,
                         double* standard_error, std::uint64_t shots, const std::uint32_t* targets,
                         std::uint32_t n_targets, std::uint32_t width, std::uint64_t* out_outcomes,
                         std::uint64_t* out_counts, std::uint64_t* n_outcomes) {
    try {
        std::vector<menos::Operation> v;
        for (std::uint32_t i = 0; i < n_ops; ++i) {
            v.push_back(to_operation(ops[i]));
        }
        std::vector<std::pair<menos::QubitId, menos::ClbitId>> t(n_targets);
        for (std::uint32_t i = 0; i < n_targets; ++i) {
            t[i] = {targets[2 * i], targets[2 * i + 1]};
        }
        menos::Observable obs;
        for (std::uint32_t i = 0; i < n_terms; ++i) {
            menos::PauliString p{num_qubits, {x_masks[i]}, {z_masks[i]}};
            obs.terms.emplace_back(std::move(p), C{coefs[2 * i], coefs[2 * i + 1]});
        }
        menos::EngineExecutionRequest req{};
        req.num_qubits = num_qubits;
        req.operations = v;
        req.want_statevector = false;
        req.want_counts = shots > 0;
        req.want_expectation = n_terms > 0;
        req.shots = shots;
        req.measure_targets = t;
        req.bitstring_width = width;
        req.seed = seed;
        req.budget_bytes = ~std::uint64_t{0};
        req.is_sole_region = true;
        req.observable = req.want_expectation ? &obs : nullptr;
        req.max_threads = 1;
        req.trajectories = trajectories;
        const menos::engines::trajectory::TrajectoryEngine engine;
        menos::EngineExecutionResult res = engine.execute(req);
        if (req.want_expectation) {
            for (std::uint32_t i = 0; i < n_terms; ++i) {
                terms_out[2 * i] = (*res.expectation_terms)[i].real();
                terms_out[2 * i + 1] = (*res.expectation_terms)[i].imag();
            }
            *standard_error = res.expectation_standard_error.value_or(0.0);
        }
        if (req.want_counts) {
            std::uint64_t i = 0;
            for (const auto& [key, count] : *res.counts) {
                if (i >= *n_outcomes) {
                    g_error = "outcome capacity exceeded";
                    return -1;
                }
                out_outcomes[i] = bits_of(key);
                out_counts[i] = count;
                ++i;
            }
            *n_outcomes = i;
        }
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return -1;
    }
}

// The dense engine's fused sweep (apply_fused, src/engines/dense/dense_engine.cpp:
// 100-112) over the plan given as ir::FusionPlan's arrays, from
// initialize(global_phase); the state (2 * 2^n doubles) out.
int ref_run_plan(std::uint32_t num_qubits, const mb2_op* ops, std::uint32_t n_ops, double global_phase,
                 const std::uint32_t* order, const std::uint32_t* block_begin, const std::uint32_t* block_qubits,
                 const std::uint32_t* qubits_begin, std::uint32_t n_blocks, std::uint32_t threads,
                 double* statevector) {
    try {
        std::vector<menos::Operation> v;
        for (std::uint32_t i = 0; i < n_ops; ++i) v.push_back(to_operation(ops[i]));
        menos::ir::FusionPlan plan;
        plan.order.assign(order, order + block_begin[n_blocks]);
        plan.block_begin.assign(block_begin, block_begin + n_blocks + 1);
        plan.qubits_begin.assign(qubits_begin, qubits_begin + n_blocks + 1);
        plan.block_qubits.assign(block_qubits, block_qubits + qubits_begin[n_blocks]);
        auto state = as_span(statevector, std::uint64_t{1} << num_qubits);
        menos::kernels::cpu::initialize(state, global_phase);
        const std::uint32_t t = threads == 0 ? menos::common::default_thread_count() : threads;
        menos::engines::dense::apply_blocks(
            plan, v, nullptr, [&](std::span<const C> matrix, std::span<const menos::QubitId> operands) {
                menos::engines::dense::apply_matrix(state, matrix, operands, t);
            });
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return -1;
    }
}

std::uint32_t ref_default_threads() {
    return menos::common::default_thread_count();
}

// The chunked tier's pass plan over the fusion plan of ops
// (src/engines/dense_tiered/pass_plan.cpp:43-150): build_pass_plan with
// chunk_qubits > 0, else choose_pass_plan (no chunk pair needed).  out:
// [chunk_qubits, window_too_small, passes, then per pass global_mask, first,
// end]; returns the words written, or -1.
std::int64_t ref_pass_plan(std::uint32_t num_qubits, const mb2_op* ops, std::uint32_t n_ops,
                           std::uint32_t chunk_qubits, std::uint32_t window_qubits, std::uint64_t* out,
                           std::uint64_t cap) {
    try {
        std::vector<menos::Operation> v;
        for (std::uint32_t i = 0; i < n_ops; ++i) v.push_back(to_operation(ops[i]));
        const menos::ir::FusionPlan fusion = menos::ir::plan_fusion(v);
        std::optional<menos::engines::dense_tiered::PassPlan> plan;
        if (chunk_qubits > 0) {
            plan = menos::engines::dense_tiered::build_pass_plan(v, num_qubits, chunk_qubits, window_qubits, &fusion);
        } else {
            plan = menos::engines::dense_tiered::choose_pass_plan(v, num_qubits, window_qubits, false, &fusion);
        }
        if (!plan.has_value()) {
            g_error = "no chunk size fits";
            return -1;
        }
        std::vector<std::uint64_t> w{plan->chunk_qubits, plan->window_too_small ? 1u : 0u, plan->passes.size()};
        for (const auto& p : plan->passes) {
            w.push_back(p.global_mask);
            w.push_back(p.first_operation);
            w.push_back(p.end_operation);
        }
        if (w.size() > cap) {
            g_error = "capacity";
            return -1;
        }
        std::copy(w.begin(), w.end(), out);
        return static_cast<std::int64_t>(w.size());
    } catch (const std::exception& e) {
        g_error = e.what();
        return -1;
    }
}

int ref_kernel_isa() {
    return menos::kernels::cpu::active_dense_kernel_isa() == menos::kernels::cpu::KernelIsa::Avx2
               ? 1
               : 0;
}

}  // extern "C"
