// Internal declarations shared by the host C++ and the CUDA translation
// units of the B200 dense engine.  Nothing here crosses the C ABI.
#pragma once

#include <complex>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/mb2.h"

#if defined(__CUDACC__)
#define MB2_HD __host__ __device__
#else
#define MB2_HD
#endif

namespace mb2 {

using Cd = std::complex<double>;

// Shared-memory slot of tile-local index l in the tile kernels.
// complex128 (16-byte slots): the low three bits XOR-folded with every
// higher 3-bit group, so quarter-warps whose eight threads vary three tile
// bits of distinct residue mod 3 hit eight distinct 16-byte bank groups.
MB2_HD inline constexpr uint32_t swz(uint32_t l) {
    const uint32_t h = l >> 3;
    return l ^ ((h ^ (h >> 3) ^ (h >> 6) ^ (h >> 9)) & 7u);
}
// complex64 (8-byte slots): the low four bits XOR-folded with every higher
// 4-bit group.  Both are linear over XOR, so slot addresses compose by XOR.
MB2_HD inline constexpr uint32_t swz8(uint32_t l) { return l ^ (((l >> 4) ^ (l >> 8) ^ (l >> 12)) & 15u); }

// ---- gate table (gate_table.cpp) -------------------------------------------
int gate_num_qubits(int opcode);
int gate_num_params(int opcode);
int gate_matrix(int opcode, const double* params, std::vector<Cd>& m);
Cd initial_phase(double global_phase);

// ---- one block to apply: a matrix on an operand list ----------------------
// Operand j is bit j of the matrix's row/column index (the reference's
// operand-order rule, src/kernels/dense_kernels.h:32-37).
struct Block {
    uint32_t k = 0;
    uint32_t q[MB2_MAX_OP_QUBITS] = {0, 0, 0, 0, 0, 0};
    std::vector<Cd> m;  // (2^k)^2 entries, row-major
    bool diagonal = false;
    uint32_t members = 1;  // gates fused into it
    uint64_t mask() const {
        uint64_t v = 0;
        for (uint32_t j = 0; j < k; ++j) v |= uint64_t{1} << q[j];
        return v;
    }
};

// All off-diagonal entries exactly zero (either sign): the reference's
// is_diagonal (src/kernels/cpu/dense_kernels.cpp:314-324).
bool is_diagonal(const std::vector<Cd>& m, uint32_t dim);

// ---- fusion (fusion.cpp) ----------------------------------------------------
// The operations as blocks: with fuse_gates, the reference's containment plan
// (src/ir/fuse_gates.cpp:190-283), or with width >= 2 the same plan structure
// joining while the block spans at most `width` qubits (fusion.cpp), and the
// reference's block matrices (src/engines/dense/fused_block.cpp:61-99);
// without, one block per gate.  MeasureOps are dropped (they apply nothing).
// plan_out (optional): the plan as ir::FusionPlan's arrays.  Throws
// std::invalid_argument on a malformed op.
struct FusionPlanArrays {
    std::vector<uint32_t> order, block_begin, block_qubits, qubits_begin;
};
std::vector<Block> build_blocks(const mb2_op* ops, uint32_t n_ops, bool fuse_gates, uint32_t width = 0,
                                FusionPlanArrays* plan_out = nullptr);

// The generic kernel on a host vector (the fused-matrix builder's tool):
// bitwise kernels::cpu::apply_matrix_generic.
void host_apply_generic(Cd* state, uint64_t n_amps, const Cd* matrix, const uint32_t* operands,
                        uint32_t k);

// ---- tiled multi-gate passes (tile_plan.cpp) -------------------------------
// One device instruction of a tile pass (32 bytes).
enum TileOp : uint8_t {
    TOP_PHASE = 1,    // load the registers with the mapping in pos[0..kRegQubits) / tperm
    TOP_END = 2,      // write the registers back, barrier
    TOP_G1 = 3,       // 1-qubit dense gate on register slot pos[0]
    TOP_G2 = 4,       // 2-qubit dense gate on register slots (pos[0], pos[1])
    TOP_DIAG = 5,     // diagonal on tile bits pos[0..k-1]
    TOP_SMEM = 6,     // k-qubit dense gate applied from shared memory (own phase)
    TOP_MMA = 7       // tensor-core pass: the phase's composed 16x16 matrix number `aux` (tile_tc.cpp)
};
enum TileKind : uint8_t {
    TK_GEN = 0,   // every entry general
    TK_U3 = 1,    // 1q: entry (0,0) real, the others general
    TK_REAL = 2,  // 1q: every entry real
    TK_MONO = 3,  // 1 nonzero entry per row: a permutation up to per-row factors
    TK_DSMALL = 4, // diagonal, k <= 2: per-entry class in aux (2 bits each: 0 = (1,0), 1 = (-1,0), 2 = general)
    TK_X = 5,      // 1q exact swap of the pair (X)
    TK_SW12 = 6,   // 2q exact exchange of local indices 1 and 2 (SWAP)
    TK_SW13 = 7,   // 2q exact exchange of local indices 1 and 3 (CX, control = operand 0)
    TK_SW23 = 8    // 2q exact exchange of local indices 2 and 3 (CX, control = operand 1)
};
struct TileInstr {
    uint8_t op;
    uint8_t k;
    uint8_t kind;
    uint8_t nthread;   // PHASE: number of thread bits in tperm
    uint8_t pos[8];
    uint32_t data;     // offset (doubles) of the gate's data in the data block
    uint8_t tperm[12];
    uint32_t aux;      // MONO: per-row source slots (2 bits each)
};
static_assert(sizeof(TileInstr) == 32, "TileInstr is 32 bytes");

// Diagonal operands outside a pass's tile: at most kMaxGlobalQubits per
// pass; in instructions, the operand at rank r among them is position
// kGlobalPos0 + r (tile positions are below 16).
constexpr uint32_t kMaxGlobalQubits = 16;
constexpr uint32_t kGlobalPos0 = 16;

struct TilePass {
    uint32_t m = 0;          // tile qubits
    uint64_t smask = 0;      // global qubits in the tile
    uint64_t gmask = 0;      // qubits outside the tile whose bits diagonals read (complex128 plain path)
    uint32_t prog_begin = 0; // first instruction
    uint32_t prog_count = 0;
    uint32_t sdata_begin = 0;  // this pass's staged data (doubles), copied to shared memory
    uint32_t sdata_count = 0;
    uint32_t gates = 0;      // blocks applied in this pass
    // The complex128 kernel's compact stream (tile_encode.cpp).
    uint32_t word_begin = 0;
    uint32_t word_count = 0;
    // Parametric data this pass reads from a binding's record: doubles
    // [param_lo, param_lo + param_len), staged after the pass's data.
    uint32_t param_lo = 0;
    uint32_t param_len = 0;
    bool heavy = false;  // has two-qubit dense/monomial/permutation, kDiagK or kSmem words
    bool mid = false;    // heavy, but only through general dense two-qubit words (kGen2)
    // Tensor-core form (complex64, tile_tc.cpp): the pass's composed phase
    // matrices are tcdata[tc_begin, tc_begin + tc_phases * kTcOperandWords).
    bool tc = false;
    uint32_t tc_begin = 0;
    uint32_t tc_phases = 0;
};

// Compact instruction stream of the complex128 tile kernel, written from the
// TileInstr list by encode_compact (tile_encode.cpp).  A header word holds
//   bits 0-7 the opcode, 8-15 aux, 16-19 a thread tile bit, 20-31 the data
//   offset in 16-byte units from the start of the pass's staged data;
// some opcodes take extra words.  Register-slot operands are part of the
// opcode, so a gate is one jump.  Ordered slot pairs (p0, p1), p0 != p1, are
// numbered p0 * 3 + (p1 < p0 ? p1 : p1 - 1).
namespace cop {
constexpr uint32_t kEnd = 0;     // end of a phase
constexpr uint32_t kU3 = 1;      // + slot
constexpr uint32_t kGen1 = 5;    // + slot
constexpr uint32_t kReal1 = 9;   // + slot
// 13-20 are unused (one-qubit monomials and X are written as kGen1/kReal1).
constexpr uint32_t kGen2 = 21;   // + pair
constexpr uint32_t kMono2 = 33;  // + pair; extra word = source rows (3 bits each)
constexpr uint32_t kSw12 = 45;   // + pair
constexpr uint32_t kSw13 = 57;   // + pair
constexpr uint32_t kSw23 = 69;   // + pair
constexpr uint32_t kDs1R = 81;   // + slot; aux = entry classes
// An operand position (0-31) in a header word: bits 16-19 and bit 31 (the
// staged data offset, bits 20-30, stays below 2048 16-byte units).
constexpr uint32_t kDs1T = 85;   // aux = classes; the operand's position in bits 16-19, 31
constexpr uint32_t kDs2RR = 86;  // + pair; aux = classes
constexpr uint32_t kDs2RT = 98;  // + 2 * slot + (index of the bit-value operand); its position in bits 16-19, 31
// aux = classes; extra word = the two operand positions: low 4 bits at 0-3
// and 4-7, their bit 4 at bits 8 and 9.
constexpr uint32_t kDs2TT = 106;
constexpr uint32_t kDiagK = 107; // aux = k; extra word = tile positions (4 bits each)
constexpr uint32_t kSigns = 108; // aux = monomial count; one word per monomial
// Runs of U3 blocks on consecutive register slots, their matrices
// consecutive in the staged data (one jump for the run).
constexpr uint32_t kU3Run0123 = 109;
constexpr uint32_t kU3Run01 = 110;
constexpr uint32_t kU3Run123 = 111;
constexpr uint32_t kU3Run012 = 112;
// Sign monomials some of whose factors are qubits outside the tile: two
// words per monomial, the register slots (bits 0-15) and the operand bits
// (positions 0-31: tile bits, then the outside qubits from kGlobalPos0).
constexpr uint32_t kSignsW = 113;
// aux = thread bits; bits 16-31 register positions; then the phase record:
// words 1-2 the byte offsets (16 bits each) of the four register bits' slots
// with 16-byte slots, words 3-4 the same with 8-byte slots, words 5-28 a
// table of 48 16-bit entries: entry 16 g + v is the tile bits that thread
// index bits 4g..4g+3 equal to v stand for in this phase.
constexpr uint32_t kPhase = 200;
constexpr uint32_t kPhaseWords = 29;
constexpr uint32_t kSmem = 201;  // aux = k; extra words: tile positions, gdata offset (doubles)
// Tensor-core pass: apply the pass's composed phase matrix number aux (its
// split-FP16 operands staged in shared memory) to the registers' amplitudes.
constexpr uint32_t kMma = 202;
// A sign monomial word: bits 0-15 the register slots j (of 16) whose
// register-bit factors are all 1 (0xffff: no register factor), bits 16-31
// the tile bits of its thread-bit factors.  The amplitudes of slots j in
// threads whose tile bits cover bits 16-31 change sign.
}  // namespace cop

// Shared-memory budget of one pass's staged instructions + data.
constexpr size_t kMaxStagedBytes = 32 * 1024;

// TileInstr.data: for TOP_SMEM an offset into the program's global-only data
// block (gdata); for every other instruction an offset into its pass's
// staged data (sdata, relative to the pass's sdata_begin).
struct TileProgram {
    std::vector<TilePass> passes;
    std::vector<double> gdata;
    std::vector<uint32_t> order;       // block indices in application order
    std::vector<uint32_t> order_pass;  // the pass of each entry of `order`
    std::vector<uint32_t> param_offsets;  // per block: offset in the per-binding record (parametric only)
    uint32_t param_stride = 0;            // doubles per binding record
    std::vector<TileInstr> instrs;
    std::vector<double> data;
    std::vector<uint32_t> words;  // compact stream of every pass (complex128 kernel)
    uint64_t fp64_per_amp = 0;    // modelled FP64 instructions per amplitude
    // Tensor-core passes: per composed phase matrix, its real 32x32 form as
    // FP16 high and low parts in the MMA's shared-memory layout (tile_tc.cpp),
    // and the matrix itself (16x16 complex, FP64) for the host interpreter.
    std::vector<uint32_t> tcdata;
    std::vector<Cd> tcmatrices;
};
// Writes prog.words and each pass's word range and parametric slice.
void encode_compact(TileProgram& prog);

// The complex64 tensor-core form of a planned program (tile_tc.cpp): each
// pass without wide (k > 2), parametric or non-unitary blocks becomes
// phases whose dense gates on the four register qubits compose (in FP64)
// into one 16x16 complex matrix, applied as a split-FP16 tensor-core GEMM,
// with diagonals that involve other tile qubits applied elementwise before
// or after it.  A pass needing more than `max_phases` matrices is split into
// several passes on the same tile.  Rewrites the passes, the staged data and
// the word stream.
// One phase matrix's operand: U's real 32x32 form as FP16 high parts (rows
// 0-31) over FP16 low parts (rows 32-63), 4096 bytes.
constexpr uint32_t kTcOperandWords = 1024;
constexpr double kTcOperandScale = 4096.0;  // U's operand is 2^12 U
void make_tensor_core_program(TileProgram& prog, const std::vector<Block>& blocks, uint32_t max_phases);
// Thread-bit order of a phase whose register bits are reg[0..nreg) (tile
// positions): tperm[0..nthread) lists the other tile positions, the first
// three of distinct residues mod 3 when possible (conflict-free shared-memory
// slots under the tile kernels' XOR-fold swizzle).
void thread_bit_order(uint32_t m, const uint32_t* reg, uint32_t nreg, uint8_t* tperm, uint8_t& nthread);

// Applies a planned program's passes to a host state in FP64, instruction by
// instruction (phase matrices exact, not split): the arithmetic the tile
// kernels carry out, up to their precision, for checking plans on the CPU.
void run_program_on_host(const TileProgram& prog, uint32_t n, Cd* state);

// Register qubits per thread in the tile kernel (16 amplitudes per thread).
constexpr uint32_t kRegQubits = 4;
constexpr uint32_t kMaxTileQubits = 12;
constexpr uint32_t kMinTileQubits = 4;

// Low qubits every tile holds by default (runs of 2^3 amplitudes, 128 bytes).
constexpr uint32_t kDefaultFixedLow = 3;
// Flags of a block in a batched sweep.
constexpr uint8_t kParamBlock = 1;     // its matrix differs between bindings
constexpr uint8_t kParamAllReal = 2;   // ... but every entry is real in every binding
constexpr uint8_t kParamM00Real = 4;   // ... entry (0,0) is real in every binding
// parametric (optional, one flag per block): those blocks' data is not
// staged; each gets an offset in a per-binding record instead
// (param_offsets[block], record length param_stride doubles), and a kind
// that holds for every parameter value.
// commuting: blocks on disjoint qubits may be applied in either order
// (the complex64 path, whose result is not bitwise the reference's), and
// the passes follow a dependency order chosen for few passes and phases.
TileProgram plan_tile_program(const std::vector<Block>& blocks, uint32_t n, uint32_t m,
                              uint32_t fixed_low = kDefaultFixedLow,
                              const std::vector<uint8_t>* parametric = nullptr, bool commuting = false);

// ---- device launches (kernels_*.cu) ----------------------------------------
struct DevCtx;  // forward (engine.cpp)
int launch_init(void* amps, uint64_t n_amps, int precision, double re, double im, void* stream);
int launch_apply_1q(void* amps, uint32_t n, uint32_t q, const double* m8, void* stream);
int launch_apply_2q(void* amps, uint32_t n, uint32_t q0, uint32_t q1, const double* m32, void* stream);
int launch_apply_diag(void* amps, uint32_t n, const uint32_t* q, uint32_t k, const double* dev_diag,
                      void* stream);
int launch_apply_generic(void* amps, uint32_t n, const uint32_t* q, uint32_t k, const double* dev_matrix,
                         void* stream);
// k = 1..10 operands, the matrix transposed (entry (out, in) at in * 2^k +
// out) in device memory; same sums as launch_apply_generic.
int launch_apply_wide(void* amps, uint32_t n, const uint32_t* q, uint32_t k, const double* dev_matrix_t,
                      void* stream);
// A batched sweep: `bindings` states of 2^n amplitudes back to back; the
// data of a parametric instruction for binding b is at pdata + b * pstride
// + instr.data (doubles).
struct BatchLayout {
    uint64_t bindings = 0;
    const double* pdata = nullptr;
    uint32_t pstride = 0;
};
int launch_tile_pass(void* amps, uint32_t n, const TilePass& pass, const uint32_t* dev_words,
                     const double* dev_sdata, const double* dev_gdata, int sm_count, void* stream,
                     const BatchLayout* batch = nullptr);
// One tile-pass launch, as the instances (kernels_tile_*.cu) take it.
struct TileLaunch {
    void* amps = nullptr;
    uint32_t n_all = 0;  // index bits, bindings included
    uint32_t m = 0;
    uint64_t smask = 0;
    uint64_t gmask = 0;
    const uint32_t* words = nullptr;
    uint32_t nwords = 0;
    const double* sdata = nullptr;
    uint32_t nsdata = 0;
    const double* gdata = nullptr;
    uint64_t ntiles = 0;
    const double* pdata = nullptr;
    uint32_t pstride = 0;
    uint32_t param_lo = 0;
    uint32_t param_len = 0;
    uint32_t bshift = 0;
    uint32_t stages = 2;
    int grid = 0;       // set by the instance launcher
    int sm_count = 0;
    bool heavy = false;  // the pass needs the full kernel variant (see TilePass::heavy)
    uint32_t threads = 0;
    size_t smem = 0;
    void* stream = nullptr;
};
// One state's pass in a launch of many (k_tile_pass_jobs): its CTAs are
// [cta_begin, cta_begin + nctas); words and data in device memory.
struct TileJob {
    void* st;  // complex128 amplitudes
    uint64_t smask, gmask, ntiles;
    const uint32_t* words;
    const double* sdata;
    const double* gdata;
    uint32_t n, nwords, nsdata, cta_begin, nctas, pad;
};
// Launches pass jobs[0..njobs) (host array `jobs`, copied to dev_jobs by the
// caller beforehand) with tile width m, the full kernel variant; smem: the
// largest job's dynamic shared memory.
int launch_tile_jobs(const TileJob* dev_jobs, uint32_t njobs, uint32_t total_ctas, uint32_t m, size_t smem,
                     void* stream);
// The small-request batch's other steps (kernels_small.cu), one launch each
// for every state: amplitude 0 of each zeroed state; a Pauli term per
// (state, term) job (out: 2 doubles per job, <psi|P|psi>); the reference's
// exact sampling walk per state (u sorted ascending, basis out).
struct ExpectJob {
    const void* st;
    uint64_t x, z;
    uint32_t n, pad;
};
struct WalkJob {
    const void* st;
    const double* u;
    uint64_t* basis;
    uint64_t shots;
    uint32_t n, pad;
};
// The reference's sorted uniforms for `shots` draws from `seed` (common::Rng,
// src/engines/dense/sample.cpp:36-42), and the outcomes through measure
// targets of a non-decreasing basis list (mb2_sample's histogram).
std::vector<double> sorted_reference_uniforms(uint64_t shots, uint64_t seed);
int counts_of(mb2_context* ctx, uint32_t n, const std::vector<uint64_t>& basis, const uint32_t* targets,
              uint32_t num_targets, uint64_t* outcomes, uint64_t* counts, uint64_t* num_outcomes);
int launch_init_jobs(void* base, const uint64_t* dev_offsets, const double* dev_vals, uint32_t count, void* stream);
int launch_expect_jobs(const ExpectJob* dev_jobs, uint32_t count, double* dev_out, void* stream);
int launch_walk_jobs(const WalkJob* dev_jobs, uint32_t count, void* stream);
constexpr size_t kTileSmemMax = 227 * 1024;  // per block
constexpr size_t kSmemPerSm = 228 * 1024;    // per SM (1 KiB of it reserved per resident block)
int launch_tile_generic(TileLaunch& L);  // any tile width, 64-bit indices
int launch_tile_m11(TileLaunch& L);      // 11-qubit tiles
int launch_tile_m12(TileLaunch& L);      // 12-qubit tiles
// Expectation of num_terms Pauli terms: partials (num_terms * kExpBlocks * 2
// doubles) then the fixed-order finish into out (num_terms * 2 doubles), all
// device pointers.
constexpr uint32_t kExpBlocks = 512;
int launch_expectation(const void* amps, uint32_t n, const uint64_t* dev_x, const uint64_t* dev_z,
                       uint32_t num_terms, double* dev_partials, double* dev_out, void* stream,
                       int precision = MB2_C128);
// Batched sweep (batch.cpp, kernels_batch.cu).
constexpr uint32_t kMaxBatchTerms = MB2_BATCH_MAX_TERMS;

// Exact device sampler (kernels_sample.cu): the chunk size of its scan, the
// scratch its internals need (beyond the sorted uniforms and the per-shot
// basis output), and the launch.  dev_basis[s] receives the basis state of
// the s-th smallest uniform.
constexpr uint32_t kSampleChunk = 4096;
size_t sample_scratch_bytes(uint32_t n, uint64_t shots);
// The reference's sequential FP64 sum of |a_i|^2 over the state, bit for bit
// (the sampler's exact chain; scratch: sample_scratch_bytes(n, 0)); synchronises.
int launch_exact_norm(const void* amps, uint32_t n, void* scratch, double* host_total, void* stream, int precision);
int launch_sample(const void* amps, uint32_t n, const double* dev_uniforms_sorted, uint64_t shots, void* scratch,
                  uint64_t* dev_basis, void* stream, int precision = MB2_C128);
// complex64 precision path (kernels_c64.cu).
constexpr uint32_t kMaxTileQubitsC64 = 13;
// Default complex64 tile: 12 qubits, two CTAs per SM (measured faster per
// circuit than 13-qubit tiles at one CTA per SM, despite more passes).
constexpr uint32_t kDefaultTileQubitsC64 = 12;
int launch_tile_pass_c64(void* amps, uint32_t n, const TilePass& pass, const uint32_t* dev_words,
                         const double* dev_sdata, const double* dev_gdata, int sm_count, void* stream,
                         const BatchLayout* batch = nullptr);
int launch_scale_c64(void* amps, uint64_t n_amps, float s, void* stream);
// The tensor-core complex64 pass (kernels_tc.cu) of a pass in tensor-core
// form (TilePass::tc).  dev_tc: the program's tcdata on the device; dev_err:
// a device word the kernel sets to a nonzero code if a bounded wait on the
// tensor core ran out (the pass's result is then invalid).
constexpr uint32_t kTcMaxPhasesFourCtas = 5;  // 11-qubit tiles, four CTAs per SM
constexpr uint32_t kTcMaxPhasesTwoCtas = 10;  // 12-qubit tiles, two CTAs per SM
constexpr uint32_t kTcMaxPhasesOneCta = 22;   // 13-qubit tiles, one CTA per SM
inline uint32_t tc_max_phases(uint32_t m) {
    return m == 11 ? kTcMaxPhasesFourCtas : (m == 12 ? kTcMaxPhasesTwoCtas : kTcMaxPhasesOneCta);
}
int launch_tile_pass_tc(void* amps, uint32_t n, const TilePass& pass, const uint32_t* dev_words,
                        const double* dev_sdata, const uint32_t* dev_tc, int* dev_err, int sm_count, void* stream);
// Debug probe of the tensor-core step alone: one CTA applies the split-FP16
// operand b (kTcOperandWords words, tile_tc.cpp's layout) to 256 rows of 16
// complex64 amplitudes (in -> out, device pointers).
int launch_tc_probe(const float* in, const uint32_t* b, float* out, int* dev_err, void* stream);
// Writes U (16x16 complex, row-major) as the split-FP16 operand (kTcOperandWords words).
void tc_operands(const Cd* u, uint32_t* out);
int context_device(const mb2_context* ctx);
// The most staging memory a state's calls can hold for a sweep of these ops,
// `shots` counts and `terms` Pauli terms, rounded as the state's grow-only
// staging buffer rounds its size (engine.cpp): what an admission must charge
// beside the state itself.
uint64_t scratch_bound(uint32_t n, const mb2_op* ops, uint32_t num_ops, uint64_t shots, uint32_t terms);
// A complex128 state on a caller-owned stream (engine.cpp).
int state_on_stream(mb2_context* ctx, uint32_t num_qubits, uint64_t budget_bytes, void* stream, mb2_state** out,
                    int precision = MB2_C128);

// Calibration probes (kernels_probe.cu): FP64 instructions per second and
// device-to-device copy GB/s (read + write bytes), on the current device.
int probe_rates(int sm_count, double* fp64_per_s, double* copy_gbs);
// Grouped Pauli terms (pauli_groups.cpp plans, kernels_reduce.cu reduces):
// terms whose X masks above the low c bits span a subspace of dimension d
// share one read of the state, in tiles of 2^(c+d) <= 2^12 amplitudes.
// Partials are written at (term.out * grid + CTA).
constexpr uint32_t kMaxGroupTerms = 16;
constexpr uint32_t kPauliTileQubits = 11;
constexpr uint32_t kPauliMinTileQubits = 10;  // smaller states: one streaming pass per term
constexpr uint32_t kPauliMaxSpan = 8;
struct PauliGroupTerm {
    uint64_t x, z;
    uint32_t kx;   // coordinates of x >> c in the group's basis
    uint32_t xl;   // x's low c bits
    uint32_t out;  // the term's index in the caller's list
    uint32_t pad;
};
struct PauliGroupPlan {
    uint32_t c = 0, d = 0;
    uint64_t free_mask = 0;  // high bits (above c) that index the cosets
    uint32_t span_off = 0, term_off = 0, nterms = 0;
};
struct PauliPlan {
    std::vector<PauliGroupPlan> groups;
    std::vector<uint64_t> spans;  // 2^d per group: span[k] = XOR of basis vectors in k
    std::vector<PauliGroupTerm> terms;
};
PauliPlan plan_pauli_groups(const uint64_t* x, const uint64_t* z, uint32_t num_terms, uint32_t n);
int launch_pauli_group(const void* amps, uint32_t n, uint32_t c, uint32_t d, const uint64_t* dev_span,
                       uint64_t free_mask, const void* dev_terms, uint32_t nterms, double* dev_partials,
                       uint32_t grid, void* stream, int precision);
// One streaming pass per term (partials only), for terms that share no read.
int launch_expectation_partials(const void* amps, uint32_t n, const uint64_t* dev_x, const uint64_t* dev_z,
                                uint32_t num_terms, double* dev_partials, void* stream, int precision);
int launch_expectation_finish(const double* dev_partials, uint32_t blocks, const uint64_t* dev_x,
                              const uint64_t* dev_z, uint32_t num_terms, double* dev_out, void* stream);
// Density matrices (kernels_reduce.cu): rho as a 2n-qubit complex128 vector,
// entry (r, c) at r | c << n.  Tr(P rho) per term (partials as
// launch_expectation's, then the finish); the exact walk of the sorted
// uniforms over rho's diagonal (one thread; n <= 15).
int launch_dm_trace(const void* rho, uint32_t n, const uint64_t* dev_x, const uint64_t* dev_z, uint32_t num_terms,
                    double* dev_partials, double* dev_out, void* stream);
int launch_dm_walk(const void* rho, uint32_t n, const double* dev_uniforms_sorted, uint64_t shots,
                   uint64_t* dev_basis, void* stream);
// MB2_OK after a clean launch, else MB2_ERR_CUDA with the error kept for
// last_cuda_error_string() (which reports and clears it).
int launch_status();
const char* last_cuda_error_string();
// Keeps a failed runtime call's error for last_cuda_error_string() (as
// launch_status does for launches) and returns MB2_ERR_CUDA; MB2_OK for
// cudaSuccess.  The error is passed as an int (a cudaError_t value) so that
// host-only translation units need no CUDA header.
int record_cuda_error(int cuda_error);
// Counts kernels this library launched (process-wide; mb2_kernel_launches).
void note_launches(uint32_t k);

}  // namespace mb2
