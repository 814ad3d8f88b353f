/*
 * mb2.h -- the C ABI of the B200-native dense statevector engine for MENOS.
 *
 * Plain C types only (no CUDA, torch or C++ types cross this boundary), so
 * MENOS's C++ SimulationEngine adapter, a ctypes binding or any other FFI can
 * bind it.  Every function returns an int status (MB2_OK == 0); the message of
 * the most recent failure on a context is read with mb2_last_error().
 *
 * Conventions are the reference's dense-kernel contract
 * (src/kernels/dense_kernels.h:25-58):
 *   - little-endian qubits: bit j of an amplitude index is qubit j;
 *   - operand order: bit j of a gate matrix's row/column index is operand j;
 *   - amplitudes are interleaved (re, im) pairs; complex128 for the plain
 *     path (MB2_C128), complex64 for the precision path (MB2_C64);
 *   - the global phase is part of the state: init writes exp(i*phase)|0..0>;
 *   - Pauli strings use Y = i*X*Z (x/z bit masks, one 64-bit word).
 *
 * The complex64 precision path (MB2_C64 states) runs the same tiled sweep with
 * gate matrices composed in FP64: each phase's gates on its four register
 * qubits compose into one 16x16 complex matrix applied on the tcgen05 tensor
 * cores as a split-precision GEMM (FP16 high and low parts of both operands
 * after a power-of-two scaling of each tile, the products lo*hi, hi*lo and
 * hi*hi, FP32 accumulation), or, per option, gate by gate with FP32 fused
 * multiply-adds; norms, expectations and sampling probabilities accumulate
 * in FP64.
 *
 * The plain complex128 path is bitwise identical to the reference's generic
 * CPU kernel (src/kernels/cpu/dense_kernels.cpp:465-524): every output
 * amplitude is (+0) + sum_in m[out][in]*a[in] in increasing `in`, each
 * product and sum rounded separately (no FMA).
 */
#ifndef MENOS_B200_MB2_ABI_H
#define MENOS_B200_MB2_ABI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
enum {
    MB2_OK = 0,
    MB2_ERR_INVALID = 1,       /* a malformed argument (reference: InternalError from ensure) */
    MB2_ERR_RESOURCE = 2,      /* over budget / out of device memory (reference: ResourceExceeded) */
    MB2_ERR_CUDA = 3,          /* a CUDA runtime failure (reference: ensure_cuda -> InternalError) */
    MB2_ERR_NO_DEVICE = 4,     /* no usable sm_100 device */
    MB2_ERR_TIMEOUT = 5,       /* a bounded wait ran out (serving loop polls) */
    MB2_ERR_UNSUPPORTED = 6,   /* an operation this engine refuses (e.g. a noise channel) */
    MB2_ERR_ABANDONED = 7      /* the execution monitor asked to abandon */
};

/* ---- precisions -------------------------------------------------------- */
enum { MB2_C128 = 0, MB2_C64 = 1 };

/* ---- opcodes: the reference's menos::Opcode order (include/menos/circuit.h:17-41) */
enum {
    MB2_X = 0, MB2_Y, MB2_Z, MB2_H, MB2_S, MB2_SDG, MB2_T, MB2_TDG, MB2_SX, MB2_SXDG,
    MB2_RX, MB2_RY, MB2_RZ, MB2_P, MB2_U, MB2_CX, MB2_CZ, MB2_SWAP, MB2_CP, MB2_RZZ,
    MB2_CCX, MB2_UNITARY, MB2_MEASURE,
    MB2_CHANNEL  /* a noise channel (the reference's ChannelOp, include/menos/circuit.h:85-88):
                    `reserved` Kraus operators of 4^k entries each, consecutive at `matrix`;
                    applied by the density-matrix path only */
};

/* The widest operation carried: the reference caps UnitaryOp at 5 qubits
 * (kMaxUnitaryQubits, include/menos/circuit.h:46); fused blocks reach 6. */
#define MB2_MAX_OP_QUBITS 6

/* One KIR operation, the flat form of the reference's Operation variant
 * (GateOp / UnitaryOp / MeasureOp, include/menos/circuit.h:50-90). */
typedef struct mb2_op {
    int32_t opcode;                      /* MB2_X .. MB2_MEASURE */
    uint32_t num_qubits;                 /* operands used in qubits[] */
    uint32_t qubits[MB2_MAX_OP_QUBITS];  /* operand j = matrix bit j */
    double params[3];                    /* gate parameters (RX/RY/RZ/P/CP/RZZ: 1, U: 3) */
    const double* matrix;                /* MB2_UNITARY: 2*4^k doubles, row-major (re, im);
                                            MB2_MEASURE: NULL, or its readout error as 4 doubles,
                                            P(recorded r | true t) at 2t + r (the reference's
                                            ReadoutError, include/menos/circuit.h:67-77); else NULL */
    uint32_t clbit;                      /* MB2_MEASURE: classical bit written */
    uint32_t reserved;
} mb2_op;

/* Opaque handles. */
typedef struct mb2_context mb2_context;
typedef struct mb2_state mb2_state;

/* ---- context ----------------------------------------------------------- */
/* Replaces: kernels::cuda::device_info()/DevicePool set-up
 * (src/kernels/cuda/device_info.h:14-55, device_pool.h:34-75). */
int mb2_context_create(int device, mb2_context** out);
int mb2_context_destroy(mb2_context* ctx);
/* Copies the last error message of ctx (NUL-terminated, truncated to len). */
int mb2_last_error(const mb2_context* ctx, char* buf, size_t len);
/* Device facts: SM count, total and free bytes. */
int mb2_device_info(mb2_context* ctx, int* sm_count, uint64_t* total_bytes, uint64_t* free_bytes);

/* ---- state ------------------------------------------------------------- */
/* Replaces: DeviceBuffer(num_amplitudes, budget) (src/kernels/cuda/device_buffer.h:25-55);
 * fails with MB2_ERR_RESOURCE before allocating when 2^n amplitudes exceed
 * budget_bytes, as the reference does (device_buffer.cpp:23). */
int mb2_state_alloc(mb2_context* ctx, uint32_t num_qubits, int precision, uint64_t budget_bytes,
                    mb2_state** out);
int mb2_state_free(mb2_state* state);
/* A complex128 state that lives in pinned, mapped HOST memory (for states
 * above the device's memory): every call above works on it unchanged -- the
 * kernels read and write the host buffer over PCIe through its device alias,
 * so results are bitwise those of a device-resident state, and each tiled
 * pass streams the state once (sweeps default to the widest tile, for the
 * fewest passes).  budget_bytes bounds the host buffer (MB2_ERR_RESOURCE
 * before any allocation).  The reference records this tier as measured and
 * not built (include/menos/menos.h:157, Tier::HostOffloaded); its disk tier
 * streams a window of chunks per pass (src/engines/dense_tiered/
 * chunked_executor.cpp).  mb2_state_host_ptr: the host buffer (2 * 2^n
 * doubles), readable once the state's stream is idle (mb2_synchronize). */
int mb2_state_alloc_host(mb2_context* ctx, uint32_t num_qubits, uint64_t budget_bytes, mb2_state** out);
int mb2_state_host_ptr(mb2_state* state, void** out);
/* Replaces: kernels::cuda::initialize (src/kernels/cuda/dense_kernels.cu:273-286). */
int mb2_init(mb2_state* state, double global_phase);
/* Device pointer of the amplitudes (interleaved re/im), for in-process callers. */
int mb2_state_device_ptr(mb2_state* state, void** out);
/* The CUDA stream (cudaStream_t) every call on this state is queued on, for
 * in-process callers that time or order work against it. */
int mb2_state_stream(mb2_state* state, void** out);

/* ---- gate application -------------------------------------------------- */
/* One matrix on one operand list.  Replaces: kernels::cuda::apply_matrix
 * (src/kernels/cuda/dense_kernels.cu:288-328; contract dense_kernels.h:211-225).
 * matrix: 2*4^k doubles, row-major, interleaved.  Asynchronous on the
 * state's stream; the host matrix is staged before return. */
int mb2_apply_matrix(mb2_state* state, const double* matrix, const uint32_t* operands, uint32_t k);
/* The generic kernel, kept as the device oracle of the specialised ones.
 * Replaces: kernels::cuda::apply_matrix_generic (dense_kernels.cu:330-365). */
int mb2_apply_matrix_generic(mb2_state* state, const double* matrix, const uint32_t* operands,
                             uint32_t k);

/* Execution options of a program sweep. */
typedef struct mb2_sweep_options {
    int32_t fuse_gates;      /* 1: the reference's containment fusion (fuse_gates.cpp:190-283) */
    int32_t low_qubits;      /* qubits 0..low-1 held in every tile (contiguous runs); -1 = none, 0 = default 3 */
    int32_t tile_qubits;     /* qubits per multi-gate tile pass; 0 = autotuned */
    int32_t per_gate;        /* 1: one launch per block, no tiling (the reference's sweep shape) */
    int32_t c64_kernel;      /* complex64 states: 0 = automatic (tensor cores for states of more than
                                2^24 amplitudes, which stream from HBM; FP32 SIMT gates below, where
                                the state stays in L2), 1 = FP32 SIMT gates only, 2 = tensor cores
                                (split-FP16 GEMMs of each phase's composed 16x16 matrix) wherever a
                                pass allows */
    int32_t fusion_width;    /* with fuse_gates: 0 = the reference's containment rule; 2..6 = the same
                                plan structure, a gate joining while its block spans at most this
                                many qubits (mb2_fusion_plan gives the plan) */
} mb2_sweep_options;

/* Applies a whole operation list (MeasureOps skipped) as a sequence of
 * multi-gate tiled passes.  Bitwise identical to applying the same blocks
 * one by one with mb2_apply_matrix.  Replaces: apply_blocks / apply_operations
 * in CudaDenseEngine::execute (src/engines/dense_cuda/cuda_dense_engine.cpp:58-87,
 * 337-355).  opts may be NULL (defaults: reference fusion on, autotuned tile). */
int mb2_apply_program(mb2_state* state, const mb2_op* ops, uint32_t num_ops,
                      const mb2_sweep_options* opts);
/* A host-resident state (mb2_state_alloc_host) swept through device
 * windows, the reference's chunked tier on the device's copy engines
 * (src/engines/dense_tiered/pass_plan.h, chunked_executor.cpp): the state is
 * 2^(n-L) chunks of 2^L amplitudes (L = chunk_qubits; 0: chosen as the
 * reference's choose_pass_plan does, pass_plan.cpp:123-150, from 2^24
 * amplitudes up -- below that from 2^min(16, W)); a window of 2^W amplitudes
 * (W = window_qubits, 4..n) holds the 2^g chunks of g <= W - L global qubits;
 * passes are the reference's greedy rule over the fusion plan's blocks
 * (pass_plan.cpp:43-121).  Each window is copied in, swept by the tiled
 * kernels with its blocks' operands remapped, and copied back; two device
 * windows on two streams let one window's copies overlap the other's sweep,
 * and with no barrier between passes (a group's copies in wait only for the
 * copies that last wrote its own chunks back) the copies run on across pass
 * boundaries.  At most 2^24 chunks (L >= n - 24).  Bitwise the
 * device-resident result.  Device memory: two windows (2 * 16 *
 * 2^W bytes, MB2_ERR_RESOURCE when they do not fit).  mb2_sweep_stats:
 * passes = window passes, launches = tile-pass launches.  A block with more
 * than W - L operands at or above L: MB2_ERR_INVALID.  Synchronous. */
int mb2_apply_program_windowed(mb2_state* state, const mb2_op* ops, uint32_t num_ops, const mb2_sweep_options* opts,
                               uint32_t window_qubits, uint32_t chunk_qubits);
/* The window plan mb2_apply_program_windowed runs, on the host: out =
 * [L, W, passes, then per pass its global mask (bit g - L per global qubit
 * g), first block, end block]; *out_words in: capacity, out: words. */
int mb2_window_plan(const mb2_op* ops, uint32_t num_ops, const mb2_sweep_options* opts, uint32_t num_qubits,
                    uint32_t window_qubits, uint32_t chunk_qubits, uint64_t* out, uint64_t* out_words);
/* As mb2_apply_program, calling `boundary(user, blocks_done)` on the host
 * after each pass has completed on the device: the state is then complete
 * and consistent, the reference's safe boundary (ExecutionMonitor::
 * at_safe_boundary, include/menos/simulation_engine.h:94-116).  A nonzero
 * return abandons the sweep: MB2_ERR_ABANDONED, the state as of that pass. */
typedef int (*mb2_boundary_fn)(void* user, uint64_t blocks_done);
int mb2_apply_program_monitored(mb2_state* state, const mb2_op* ops, uint32_t num_ops,
                                const mb2_sweep_options* opts, mb2_boundary_fn boundary, void* user);

/* The fusion plan a sweep with these options applies, in the arrays of the
 * reference's ir::FusionPlan (src/ir/fuse_gates.h:38-76): block b is the ops
 * order[block_begin[b] .. block_begin[b+1]) on the qubits
 * block_qubits[qubits_begin[b] .. qubits_begin[b+1]) (ascending; empty for a
 * MeasureOp barrier).  Handing it to the reference's block sweep
 * (engines::dense::apply_blocks) reproduces this engine's complex128 state
 * bit for bit.  order holds num_ops entries; capacities in, sizes out:
 * *num_blocks (blocks: block_begin and qubits_begin hold one entry more)
 * and *num_block_qubits (entries of block_qubits); MB2_ERR_INVALID with
 * the sizes set when a capacity is short.  Host only. */
int mb2_fusion_plan(const mb2_op* ops, uint32_t num_ops, const mb2_sweep_options* opts, uint32_t* order,
                    uint32_t* block_begin, uint32_t* block_qubits, uint32_t* qubits_begin, uint64_t* num_blocks,
                    uint64_t* num_block_qubits);

/* What a sweep of these ops on a num_qubits state costs the device, without
 * running it: the planner's DeviceCost (include/menos/plan.h:117-122) and the
 * dense work units of DenseEngine::estimate (src/engines/dense/dense_engine.cpp:309-331). */
typedef struct mb2_sweep_estimate {
    uint64_t blocks;
    uint64_t passes;
    uint64_t launches;
    uint64_t device_bytes;     /* state + staging */
    uint64_t h2d_bytes;        /* program upload */
    uint64_t work_units;       /* 2^n + sum over blocks of 2^(n+k) */
    uint64_t fp64_ops_per_amp;
} mb2_sweep_estimate;
int mb2_estimate_sweep(const mb2_op* ops, uint32_t num_ops, const mb2_sweep_options* opts,
                       uint32_t num_qubits, mb2_sweep_estimate* out);

/* Statistics of the last mb2_apply_program on this state. */
typedef struct mb2_sweep_stats {
    uint64_t blocks;         /* blocks applied (after fusion) */
    uint64_t passes;         /* state passes launched */
    uint64_t launches;       /* kernels launched */
    uint64_t fp64_ops_per_amp; /* FP64 instructions per amplitude summed over the sweep (model) */
} mb2_sweep_stats;
int mb2_last_sweep_stats(mb2_state* state, mb2_sweep_stats* out);

/* ---- outputs ----------------------------------------------------------- */
/* <psi|P_t|psi> for each term (coefficient not applied), out[2t] = re,
 * out[2t+1] = im.  Replaces: kernels::cuda::expectation_of_term per term
 * (src/kernels/cuda/dense_kernels.cu:367-409); terms sharing passes.
 * Synchronous. */
int mb2_expectation(mb2_state* state, const uint64_t* x_masks, const uint64_t* z_masks,
                    uint32_t num_terms, double* out);
/* The same reduction for callers that cannot allocate device memory: a
 * serving process whose own allocator has reserved the GPU's memory, or code
 * where a driver allocation must not happen.  It allocates nothing (no
 * cudaMalloc, cudaFree or allocating library call): its scratch -- masks,
 * partial sums, results -- is a file-scope __device__ array of 526,336
 * bytes that every GPU loading this library holds until exit.  The caller
 * passes the state (dev_amps: 2^num_qubits complex128 in device memory), the
 * host masks, the host output (2 doubles per term) and the stream to run on.
 * num_terms above MB2_NOALLOC_MAX_TERMS returns MB2_ERR_RESOURCE and does
 * nothing.  The first call on a device looks the array's device address up
 * (cudaGetSymbolAddress, with that device current); make it before any
 * stream capture.  After a device reset the kept address is stale: the next
 * call sees its first copy refused and looks the address up again.  Calls
 * share the one array: calls that overlap on the GPU (on different streams)
 * race.  A CUDA failure returns MB2_ERR_CUDA with its message kept for the
 * thread, as for launches.  Synchronous.  No counterpart in the
 * reference, which allocates its partial sums per term
 * (src/kernels/cuda/dense_kernels.cu:378-399). */
#define MB2_NOALLOC_MAX_TERMS 64
int mb2_expectation_noalloc(const void* dev_amps, uint32_t num_qubits, const uint64_t* x_masks,
                            const uint64_t* z_masks, uint32_t num_terms, double* out, void* stream);
/* sum |a|^2, accumulated in FP64.  Synchronous. */
int mb2_norm(mb2_state* state, double* out);
/* Renormalises a complex64 state to unit norm (the norm in FP64, the scale
 * applied in FP32); reports the norm before.  complex128 states are only
 * measured, never rescaled (their bits are the reference's).  Synchronous. */
int mb2_normalize(mb2_state* state, double* norm_before);
/* Counts by the reference's sort-then-walk sampler (src/engines/dense/sample.cpp:24-75):
 * seed -> mt19937_64 -> (w>>11)*2^-53 uniforms, sorted, walked against the
 * sequential FP64 cumulative sum of |a|^2 (identical counts).  Outcomes are
 * the measured bits mapped through targets (pairs qubit, clbit; width <= 64),
 * returned in ascending outcome order.  *num_outcomes in: capacity of
 * outcomes/counts, out: distinct outcomes written.  Synchronous. */
int mb2_sample(mb2_state* state, uint64_t shots, uint64_t seed, const uint32_t* targets,
               uint32_t num_targets, uint64_t* outcomes, uint64_t* counts, uint64_t* num_outcomes);
/* For each uniform (any order, each in [0, 1)), the basis state a draw of it
 * lands on: the first index whose sequential FP64 cumulative sum of |a|^2
 * exceeds it, the last index when none does.  The answers of the reference's
 * CumulativeDistribution::sample_one(double) for a region's state
 * (src/engines/dense/cumulative_distribution.cpp:3-124), computed on the
 * device without copying the state back; basis_out[i] belongs to
 * uniforms[i].  Synchronous. */
int mb2_sample_basis(mb2_state* state, const double* uniforms, uint64_t n, uint64_t* basis_out);
/* Copies the amplitudes to host memory (interleaved; 2 doubles or 2 floats
 * per amplitude by precision).  Replaces: DeviceBuffer::copy_to_host
 * (src/kernels/cuda/device_buffer.cpp:60-63).  Synchronous. */
int mb2_copy_out(mb2_state* state, void* host, uint64_t num_amplitudes);
/* Copies amplitudes from host memory into the state. Synchronous. */
int mb2_copy_in(mb2_state* state, const void* host, uint64_t num_amplitudes);
/* Waits for all work queued on the state's stream. */
int mb2_synchronize(mb2_state* state);

/* ---- density matrices (noisy circuits) ---------------------------------- */
/* The reference's density-matrix engine (src/engines/density_matrix/
 * density_matrix_engine.cpp) on the device.  rho for n qubits is a
 * complex128 state of 2n qubits (mb2_state_alloc(ctx, 2n, MB2_C128, ...)),
 * entry (r, c) at index r | c << n; mb2_init(rho, 0.0) sets |0..0><0..0|.
 * mb2_dm_apply_program applies each gate as U on qubits q and conj(U) on
 * q + n, each MB2_CHANNEL as its superoperator (sum over Kraus K of
 * K (x) conj(K), rows r | c << k) on q and q + n, operation by operation:
 * bitwise the reference engine's rho.  mb2_dm_expectation: Tr(P_t rho) per
 * term (within 1e-12 of the reference's sequential sum).  mb2_dm_sample:
 * counts by the reference's sort-then-walk over rho's diagonal (identical
 * counts); outcomes as mb2_sample's.  n <= 15; channels of 1..5 qubits (4- and
 * 5-qubit ones run as 8- and 10-operand blocks from global memory).
 * Readout errors: mb2_dm_sample_readout below. */
int mb2_dm_apply_program(mb2_state* rho, uint32_t num_qubits, const mb2_op* ops, uint32_t num_ops);
int mb2_dm_expectation(mb2_state* rho, uint32_t num_qubits, const uint64_t* x_masks, const uint64_t* z_masks,
                       uint32_t num_terms, double* out);
int mb2_dm_sample(mb2_state* rho, uint32_t num_qubits, uint64_t shots, uint64_t seed, const uint32_t* targets,
                  uint32_t num_targets, uint64_t* outcomes, uint64_t* counts, uint64_t* num_outcomes);
/* mb2_dm_sample with the readout errors of the circuit's measurements: each
 * target's error is that of the last MB2_MEASURE in ops writing its clbit
 * (readout_targets, src/engines/noise/readout.cpp).  Without any, exactly
 * mb2_dm_sample.  With some, the reference's per-shot draws
 * (density_matrix_engine.cpp:378-390): from common::Rng(seed), one word per
 * shot for the true outcome -- the first basis state whose sequential
 * cumulative probability exceeds its uniform, found on the device -- then
 * one word per readout-errored target in target order, the bit flipping
 * when its uniform is below P(recorded != true | true) (apply_readout).
 * Identical counts. */
int mb2_dm_sample_readout(mb2_state* rho, uint32_t num_qubits, const mb2_op* ops, uint32_t num_ops, uint64_t shots,
                          uint64_t seed, const uint32_t* targets, uint32_t num_targets, uint64_t* outcomes,
                          uint64_t* counts, uint64_t* num_outcomes);

/* For each uniform (any order, each in [0, 1)), the basis state whose
 * sequential cumulative probability over rho's diagonal first exceeds it
 * (CumulativeDistribution::sample_one on the diagonal,
 * src/engines/dense/cumulative_distribution.cpp:83-92): the draws of a
 * Factorized region's density-matrix sampler.  Synchronous. */
int mb2_dm_sample_basis(mb2_state* rho, uint32_t num_qubits, const double* uniforms, uint64_t count,
                        uint64_t* basis);

/* The reference's sequential FP64 sum of |a_i|^2 over the state, bit for bit
 * (the exact device chain of mb2_sample), e.g. to renormalise as the
 * reference does (src/engines/trajectory/trajectory_engine.cpp:155-166). */
int mb2_norm_exact(mb2_state* state, double* out);

/* The reference's trajectory engine (src/engines/trajectory/
 * trajectory_engine.cpp:424-494) on the device: `trajectories` pure-state
 * runs of the n-qubit circuit, trajectory t drawing from a common::Rng seeded
 * with SplitMix64 output t + 1 of `seed`.  Gates apply op by op; a channel
 * (MB2_CHANNEL, 1..3 qubits) draws one uniform, picks the first Kraus
 * operator whose cumulative Re Tr(K^dagger K rho_q) exceeds it (rho_q, the
 * reduced density matrix, from the 4^k Pauli expectations on its qubits),
 * applies it and renormalises by the exact sequential norm -- so each
 * trajectory's state is bitwise the reference's whenever its branches are
 * (they are unless a uniform falls within rounding of a branch boundary).
 * Expectation (num_terms > 0; coefs: complex, 2 doubles each): term_means
 * (2 * num_terms doubles, the mean of <P_t> over trajectories) and the
 * standard error of sum_t coef_t <P_t>.  Counts (shots <= trajectories): one
 * draw per trajectory t < shots, after its channel draws, by the exact walk,
 * then one word per readout-errored target (the errors of the MB2_MEASURE
 * ops, as mb2_dm_sample_readout; trajectory_engine.cpp:463-472); outcomes
 * as mb2_sample's. */
int mb2_trajectories(mb2_context* ctx, uint32_t num_qubits, const mb2_op* ops, uint32_t num_ops,
                     uint64_t trajectories, uint64_t seed, const uint64_t* x_masks, const uint64_t* z_masks,
                     const double* coefs, uint32_t num_terms, double* term_means, double* standard_error,
                     uint64_t shots, const uint32_t* targets, uint32_t num_targets, uint64_t* outcomes,
                     uint64_t* counts, uint64_t* num_outcomes);
/* mb2_trajectories with the reference's execution monitor: boundary(user,
 * crossed) is called with the reference's count of safe boundaries crossed
 * (one after every operation of every trajectory, one after each
 * trajectory's outputs; trajectory_engine.cpp:171-181) at the end of each
 * run of gates, each channel and each trajectory; a nonzero return abandons
 * with MB2_ERR_ABANDONED.  A monitor that abandons at count c stops here at
 * the first such point at or past c. */
int mb2_trajectories_monitored(mb2_context* ctx, uint32_t num_qubits, const mb2_op* ops, uint32_t num_ops,
                               uint64_t trajectories, uint64_t seed, const uint64_t* x_masks,
                               const uint64_t* z_masks, const double* coefs, uint32_t num_terms, double* term_means,
                               double* standard_error, uint64_t shots, const uint32_t* targets,
                               uint32_t num_targets, uint64_t* outcomes, uint64_t* counts, uint64_t* num_outcomes,
                               mb2_boundary_fn boundary, void* user);

/* ---- batched parameter sweep ------------------------------------------- */
/* One circuit structure under many parameter bindings, in one device job:
 * every binding's state lives in one buffer (binding b at b * 2^n), the
 * tiled passes run once for all bindings, and <H> = sum_t coef_t <P_t> is
 * returned per binding (out[b], real part).  Binding b's circuit is `ops`
 * with each parameterised gate (RX RY RZ P U CP RZZ), in op order, taking
 * its parameters from params[b * params_per_binding ...] (the ops' own
 * params are ignored; params_per_binding must equal the slots the ops
 * have).  complex128 results per binding are bitwise the state a single run
 * of that binding computes; <H> within the expectation tolerance.  2^n
 * amplitudes per binding with 4 <= n <= 16; at most MB2_BATCH_MAX_TERMS terms.
 * states_out (optional): every binding's final amplitudes, 2 * 2^n doubles
 * each.  Replaces: a run_batch loop of menos::run calls
 * (src/api/batch.cpp:10-27) for a parameter sweep; no direct counterpart. */
#define MB2_BATCH_MAX_TERMS 64
typedef struct mb2_batch_options {
    int32_t precision;   /* MB2_C128, or MB2_C64: complex64 states (FP32 gates, FP64 reductions; states_out promoted) */
    int32_t fuse_gates;  /* 1: the reference's containment fusion per binding; 0: gate by gate */
    int32_t tile_qubits; /* 0: default */
    int32_t reserved;
} mb2_batch_options;
typedef struct mb2_batch_stats {
    uint64_t passes;
    uint64_t blocks;
    uint64_t parametric_blocks;
    uint64_t h2d_bytes;
    uint64_t fp64_ops_per_amp;
} mb2_batch_stats;
int mb2_sweep_batch(mb2_context* ctx, const mb2_op* ops, uint32_t num_ops, uint32_t num_qubits,
                    const double* params, uint32_t params_per_binding, uint32_t num_bindings,
                    const uint64_t* x_masks, const uint64_t* z_masks, const double* coefs,
                    uint32_t num_terms, const mb2_batch_options* opts, double* out,
                    double* states_out, mb2_batch_stats* stats);

/* ---- serving loop (continuous batching) -------------------------------- */
/* A server takes circuit requests as they arrive and runs them on one GPU:
 * `slots` requests at a time, each on its own stream, admitted against a
 * device-memory budget (state + staging); a request that arrives while
 * others run starts as soon as a slot and memory free up.  Results do not
 * depend on what else runs.  New in this engine: the reference runs
 * circuits one after another (src/api/batch.cpp:10-27). */
enum { MB2_OUT_COUNTS = 1, MB2_OUT_EXPECTATION = 2 };
typedef struct mb2_server mb2_server;
typedef struct mb2_server_options {
    uint64_t device_budget_bytes;  /* 0: 90% of the free device memory */
    uint32_t slots;                /* concurrent requests; 0: 16 */
    uint32_t reserved;
} mb2_server_options;
typedef struct mb2_request {
    const mb2_op* ops;
    uint32_t num_ops;
    uint32_t num_qubits;
    double global_phase;
    int32_t fuse_gates;
    int32_t output;                /* MB2_OUT_COUNTS or MB2_OUT_EXPECTATION */
    uint64_t shots, seed;          /* counts */
    const uint32_t* targets;       /* counts: (qubit, clbit) pairs */
    uint32_t num_targets;
    uint32_t num_terms;            /* expectation: <H> = sum_t coefs[t] <P_t> (real part) */
    const uint64_t* x_masks;
    const uint64_t* z_masks;
    const double* coefs;
    int32_t precision;             /* MB2_C128 (0, bitwise the reference) or MB2_C64 (complex64 state) */
    uint32_t reserved;
} mb2_request;
typedef struct mb2_completion {
    uint64_t ticket;
    int32_t status;                /* MB2_OK or the failing call's status */
    uint32_t reserved;
    double value;                  /* expectation requests */
    uint64_t num_outcomes;         /* counts requests */
    const uint64_t* outcomes;      /* ascending; owned by the server until mb2_server_release */
    const uint64_t* counts;
    double queue_seconds;          /* submit -> admission */
    double latency_seconds;        /* submit -> completion */
} mb2_completion;
int mb2_server_create(mb2_context* ctx, const mb2_server_options* opts, mb2_server** out);
/* Copies the request; MB2_ERR_RESOURCE if it could never fit the budget. */
int mb2_server_submit(mb2_server* server, const mb2_request* request, uint64_t* ticket);
/* Up to `capacity` completions; waits at most timeout_ms for the first.
 * MB2_ERR_TIMEOUT when none arrived. */
int mb2_server_poll(mb2_server* server, mb2_completion* out, uint32_t capacity, uint32_t* count,
                    uint32_t timeout_ms);
int mb2_server_release(mb2_server* server, uint64_t ticket);
int mb2_server_stats(mb2_server* server, uint64_t* pending, uint64_t* in_flight, uint64_t* held_bytes,
                     uint64_t* budget_bytes);
/* Drops pending requests, waits for the running ones, frees everything. */
int mb2_server_destroy(mb2_server* server);
/* Admission through the caller's memory ledger (the reference's
 * MemoryLedger, src/common/memory_ledger.h:37-117, Space::Device): a request
 * is admitted when it fits the server's budget AND charge(user, bytes)
 * returns nonzero (the ledger took the bytes: its state and staging, as the
 * server counts them); release(user, bytes) is called when that memory is
 * freed.  Both run on server threads, one call at a time, with the server's
 * lock held (they must not call the server).  A refused request stays
 * pending and is offered again within a few milliseconds.  Set before the
 * first submit; null functions detach the ledger. */
typedef int (*mb2_ledger_charge_fn)(void* user, uint64_t bytes);
typedef void (*mb2_ledger_release_fn)(void* user, uint64_t bytes);
int mb2_server_set_ledger(mb2_server* server, mb2_ledger_charge_fn charge, mb2_ledger_release_fn release,
                          void* user);

/* ---- calibration ------------------------------------------------------- */
/* Measures the device's FP64 multiply/add issue rate (instructions per
 * second) and its device-to-device copy bandwidth (read+write GB/s), for the
 * planner's CUDA time model and the roofline.  Replaces the reference's
 * device microbenchmarks (src/kernels/cuda/device_benchmarks.h:30-67) feeding
 * CudaCalibration (src/plan/cuda_calibration.h:9-48). */
int mb2_probe_rates(mb2_context* ctx, double* fp64_ops_per_s, double* copy_gbs);

/* ---- autotuning and the calibrated time model --------------------------
 * Measures, on the context's device, which tile width runs a synthetic
 * brick sweep fastest (complex128: 10, 11, 12 qubits; complex64: 12, 13) at
 * probe_qubits (0: 24; 16..30) and the costs of the time model, in which a
 * pass takes  fixed + amplitudes * (memory + sum of its blocks' compute):
 * the fixed cost of a pass (timed on a 14-qubit state), the memory cost of a
 * near-empty pass (the state read and written once, at probe_qubits), the
 * compute a dense single-qubit block adds to a pass (a dense k-qubit block
 * counts 2^(k-1) of them) and that of a diagonal block.  The widths become the context's defaults for
 * sweeps with tile_qubits = 0; the costs feed mb2_estimate_sweep_time.
 * Replaces the reference's device microbenchmarks feeding CudaCalibration
 * (src/kernels/cuda/device_benchmarks.h:30-67, src/plan/cuda_calibration.h:9-48),
 * extended to the tile width. */
typedef struct mb2_tuning {
    uint32_t tile_qubits;          /* complex128 */
    uint32_t tile_qubits_c64;      /* complex64 */
    double pass_s_fixed;           /* complex128: seconds per pass (launch) */
    double pass_s_per_amp;         /* complex128 costs, seconds per amplitude */
    double dense1_s_per_amp;
    double diag_s_per_amp;
    double pass_s_fixed_c64;       /* complex64 costs */
    double pass_s_per_amp_c64;
    double dense1_s_per_amp_c64;
    double diag_s_per_amp_c64;
    uint32_t probe_qubits;         /* 0: not measured (the built-in defaults) */
    uint32_t reserved;
} mb2_tuning;
int mb2_autotune(mb2_context* ctx, uint32_t probe_qubits, mb2_tuning* out);
int mb2_context_tuning(mb2_context* ctx, mb2_tuning* out);
/* Seconds a sweep of these ops would take on this context's device: the
 * tile program's passes and blocks weighted by the tuned costs (the planner's
 * calibrated CUDA time model).  Plans only; runs nothing. */
int mb2_estimate_sweep_time(mb2_context* ctx, const mb2_op* ops, uint32_t num_ops, const mb2_sweep_options* opts,
                            uint32_t num_qubits, int32_t precision, double* seconds);

/* Kernels this library has launched since it was loaded, over all contexts
 * and states (probes excluded).  Read before and after a region to count its
 * device launches.  Has no counterpart in the reference. */
int mb2_kernel_launches(uint64_t* out);

/* ---- host-side reference pieces (no device work) ----------------------- */
/* Gate matrix, bitwise ir::generate_matrix (src/ir/gate_table.cpp:260).
 * out: 2*4^k doubles; returns MB2_ERR_INVALID for UNITARY/MEASURE. */
int mb2_gate_matrix(int32_t opcode, const double* params, double* out, uint32_t out_len);

/* ---- diagnostics (no device work) ------------------------------------- */
/* The block schedule mb2_apply_program would run for these ops on a
 * num_qubits state: for each applied block, in application order, its pass
 * index, operand count, operands (6 slots) and matrix (2*4^k doubles,
 * appended to `matrices`).  *num_blocks in: capacity of pass/k/qubits,
 * out: blocks written; *matrix_len in: capacity of matrices (doubles), out:
 * doubles written.  precision: the state's (MB2_C64 schedules reorder
 * commuting blocks into fewer passes; MB2_C128 keeps the plan order).  Lets
 * tests check the tiled schedule on the CPU oracle.  Has no counterpart in
 * the reference (its sweep is in op order). */
int mb2_debug_schedule(const mb2_op* ops, uint32_t num_ops, const mb2_sweep_options* opts,
                       uint32_t num_qubits, uint32_t* pass, uint32_t* k, uint32_t* qubits,
                       double* matrices, uint64_t* num_blocks, uint64_t* matrix_len, int32_t precision);

/* Runs the tiled program mb2_apply_program would plan for these ops on a
 * num_qubits state (precision MB2_C64: the commuting plan and, unless
 * opts->c64_kernel says otherwise, its tensor-core form) on the host, in
 * FP64, instruction by instruction (phase matrices exact): state (2 * 2^n
 * doubles) in and out.  stats (6 words, optional): passes, tensor-core
 * passes, phase matrices, tile qubits, the largest dynamic shared memory
 * (bytes) a tensor-core pass launches with, register layouts the
 * tensor-core passes load.  Lets tests check the plan -- the
 * order of every block, each phase's composed matrix, the placement of
 * elementwise diagonals -- against the oracle on the CPU.  state NULL: the
 * stats only (up to 40 qubits); otherwise at most 28 qubits.  Has no
 * counterpart in the reference. */
int mb2_debug_run_plan(const mb2_op* ops, uint32_t num_ops, const mb2_sweep_options* opts, uint32_t num_qubits,
                       int32_t precision, double* state, uint64_t* stats);

/* The complex64 tensor-core step alone, on the context's device: 256 rows of
 * 16 complex64 amplitudes (rows: 256 * 32 floats, interleaved) times the
 * 16x16 complex matrix (row-major, interleaved doubles) as the tile pass
 * applies a phase -- the rows scaled by a power of two, split-FP16
 * operands, FP32 accumulation, the scale taken out again -- into out
 * (256 * 32 floats): out_row = matrix * in_row.  Lets tests check the
 * tensor-memory and operand layouts in isolation.  Has no counterpart in the
 * reference. */
int mb2_debug_tc_probe(mb2_context* ctx, const float* rows, const double* matrix, float* out);

/* The grouping mb2_expectation uses for these terms on a num_qubits state,
 * as 64-bit words: the group count, then per group c, d, free_mask, nterms,
 * the 2^d span vectors (X-mask bits above c, span[k] = XOR of the basis
 * vectors selected by k), and per term its index, kx (coordinates of its
 * X mask above c) and xl (its low c X bits).  A group's tiles are the cosets
 * of the span: chunk k of the tile at coset index i holds amplitudes
 * ((deposit(i, free_mask) ^ span[k]) << c) | low, low < 2^c.  *out_words in:
 * capacity, out: words needed.  Lets tests check on the CPU that every
 * amplitude pair is visited once.  Has no counterpart in the reference. */
int mb2_debug_pauli_groups(const uint64_t* x_masks, const uint64_t* z_masks, uint32_t num_terms,
                           uint32_t num_qubits, uint64_t* out, uint64_t* out_words);

#ifdef __cplusplus
}
#endif

#endif /* MENOS_B200_MB2_ABI_H */
