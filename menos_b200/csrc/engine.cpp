// The C ABI (include/mb2.h) over the sm_100a kernels: contexts, device
// states, gate application (per block or as multi-gate tiled passes),
// expectation, norm, sampling and copies.
//
// Error conventions follow the reference's CUDA backend
// (src/kernels/cuda/cuda_error.h:23-30, device_buffer.cpp:23,
// device_pool.cpp:73-86): a request over budget fails before anything is
// allocated (MB2_ERR_RESOURCE), an out-of-memory allocation is reported as
// MB2_ERR_RESOURCE with the CUDA error cleared, any other CUDA failure is
// MB2_ERR_CUDA with its message kept on the context.
#include <cuda_runtime.h>

#include <algorithm>
#include <bit>
#include <atomic>
#include <cmath>
#include <cstring>
#include <mutex>
#include <random>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "mb2_internal.h"

struct mb2_context {
    int device = 0;
    int sm_count = 0;
    std::mutex mu;
    std::string last_error;
    // Tile widths and time-model costs (mb2_autotune; built-in defaults
    // measured on B200 until then).
    std::atomic<uint32_t> tile_c128{0}, tile_c64{0};
    mb2_tuning tuning{11, 12, 4e-6, 5.3e-12, 6.0e-13, 3.0e-13, 4e-6, 3.0e-12, 3.5e-13, 2.0e-13, 0, 0};
};

struct mb2_state {
    mb2_context* ctx = nullptr;
    uint32_t n = 0;
    int precision = MB2_C128;
    void* amps = nullptr;
    cudaStream_t stream = nullptr;
    bool owns_stream = true;
    void* scratch = nullptr;  // staging: program, matrices, masks, partials
    size_t scratch_bytes = 0;
    // A host-resident state (mb2_state_alloc_host): the pinned, mapped host
    // buffer, of which `amps` is the device's alias.
    void* host_amps = nullptr;
    mb2_sweep_stats stats{};
};

namespace {

int fail(mb2_context* ctx, int code, const std::string& msg) {
    if (ctx != nullptr) {
        std::lock_guard<std::mutex> lock(ctx->mu);
        ctx->last_error = msg;
    }
    return code;
}

int cuda_fail(mb2_context* ctx, cudaError_t e, const char* what) {
    const std::string msg = std::string(what) + ": " + cudaGetErrorString(e);
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();  // clear the sticky-free allocation error
        return fail(ctx, MB2_ERR_RESOURCE, msg);
    }
    return fail(ctx, MB2_ERR_CUDA, msg);
}

#define MB2_CUDA(ctx, call)                                    \
    do {                                                       \
        const cudaError_t e_ = (call);                         \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #call); \
    } while (0)

size_t amp_bytes(int precision) { return precision == MB2_C64 ? 8 : 16; }

// Grow-only device staging buffer of the state.  Allocations are
// stream-ordered (cudaMallocAsync / cudaFreeAsync on the state's stream):
// work queued before a free finishes before the memory is reused, and no
// call synchronises the device, so states driven from other threads keep
// running.
int ensure_scratch(mb2_state* s, size_t bytes) {
    if (bytes <= s->scratch_bytes) return MB2_OK;
    if (s->scratch != nullptr) MB2_CUDA(s->ctx, cudaFreeAsync(s->scratch, s->stream));
    s->scratch = nullptr;
    s->scratch_bytes = 0;
    size_t want = 1 << 20;
    while (want < bytes) want <<= 1;
    MB2_CUDA(s->ctx, cudaMallocAsync(&s->scratch, want, s->stream));
    s->scratch_bytes = want;
    return MB2_OK;
}

int check_operands(mb2_state* s, const uint32_t* q, uint32_t k) {
    if (k == 0 || k > MB2_MAX_OP_QUBITS) return fail(s->ctx, MB2_ERR_INVALID, "operand count must be 1..6");
    uint64_t seen = 0;
    for (uint32_t j = 0; j < k; ++j) {
        if (q[j] >= s->n) return fail(s->ctx, MB2_ERR_INVALID, "operand out of range");
        if (seen & (uint64_t{1} << q[j])) return fail(s->ctx, MB2_ERR_INVALID, "repeated operand");
        seen |= uint64_t{1} << q[j];
    }
    return MB2_OK;
}

// The reference's walk (src/engines/dense/sample.cpp:55-69), reproduced
// exactly on the device: basis[i] = the first basis state whose sequential
// FP64 cumulative |a|^2 exceeds the sorted uniform u[i] (the last state when
// none does).  Synchronous.
int walk_sorted(mb2_state* s, const std::vector<double>& u, uint64_t* basis) {
    const uint64_t shots = u.size();
    const size_t al_u = (shots * 8 + 255) & ~size_t{255};
    const size_t need = 2 * al_u + mb2::sample_scratch_bytes(s->n, shots);
    if (int e = ensure_scratch(s, need); e != MB2_OK) return e;
    auto* base = static_cast<unsigned char*>(s->scratch);
    auto* dev_u = reinterpret_cast<double*>(base);
    auto* dev_basis = reinterpret_cast<uint64_t*>(base + al_u);
    MB2_CUDA(s->ctx, cudaMemcpyAsync(dev_u, u.data(), shots * 8, cudaMemcpyHostToDevice, s->stream));
    const int rc =
        mb2::launch_sample(s->amps, s->n, dev_u, shots, base + 2 * al_u, dev_basis, s->stream, s->precision);
    if (rc != MB2_OK) return fail(s->ctx, rc, std::string("sample launch: ") + mb2::last_cuda_error_string());
    MB2_CUDA(s->ctx, cudaMemcpyAsync(basis, dev_basis, shots * 8, cudaMemcpyDeviceToHost, s->stream));
    MB2_CUDA(s->ctx, cudaStreamSynchronize(s->stream));
    return MB2_OK;
}

// One block through the per-gate kernels (the reference's apply_matrix
// dispatch, src/kernels/cpu/dense_kernels.cpp:427-463: diagonal, 1q, 2q,
// generic).
int apply_block(mb2_state* s, const mb2::Cd* m, const uint32_t* q, uint32_t k, bool force_generic) {
    const uint32_t dim = 1u << k;
    std::vector<mb2::Cd> mv(m, m + size_t{dim} * dim);
    const double* md = reinterpret_cast<const double*>(mv.data());
    int rc;
    if (!force_generic && mb2::is_diagonal(mv, dim)) {
        std::vector<double> d(2 * dim);
        for (uint32_t i = 0; i < dim; ++i) {
            d[2 * i] = mv[size_t{i} * dim + i].real();
            d[2 * i + 1] = mv[size_t{i} * dim + i].imag();
        }
        rc = mb2::launch_apply_diag(s->amps, s->n, q, k, d.data(), s->stream);
    } else if (!force_generic && k == 1) {
        rc = mb2::launch_apply_1q(s->amps, s->n, q[0], md, s->stream);
    } else if (!force_generic && k == 2) {
        rc = mb2::launch_apply_2q(s->amps, s->n, q[0], q[1], md, s->stream);
    } else {
        const size_t bytes = size_t{dim} * dim * sizeof(mb2::Cd);
        if (int e = ensure_scratch(s, bytes); e != MB2_OK) return e;
        MB2_CUDA(s->ctx, cudaMemcpyAsync(s->scratch, md, bytes, cudaMemcpyHostToDevice, s->stream));
        rc = mb2::launch_apply_generic(s->amps, s->n, q, k, static_cast<const double*>(s->scratch), s->stream);
    }
    if (rc != MB2_OK) return fail(s->ctx, rc, std::string("kernel launch: ") + mb2::last_cuda_error_string());
    s->stats.launches += 1;
    return MB2_OK;
}

// 11-qubit tiles: two (or three) CTAs per SM with double buffering stream
// better than one 12-qubit CTA per SM, and that outweighs the extra passes.
uint32_t default_tile_qubits(uint32_t n) { return std::min<uint32_t>(11, n); }

// The tile width a sweep runs at: the requested (or default) width, raised
// to hold the widest block, within the kernel's limits.
uint32_t tile_width(uint32_t requested, uint32_t n, const std::vector<mb2::Block>& blocks) {
    uint32_t m = requested > 0 ? requested : default_tile_qubits(n);
    for (const mb2::Block& b : blocks) m = std::max(m, b.k);
    m = std::max(m, mb2::kMinTileQubits);
    return std::min(m, mb2::kMaxTileQubits);
}

// A complex64 sweep's tile width and kernel.  Automatic: the tensor-core
// pass for states of more than 2^24 amplitudes (which stream from HBM, where
// it is the faster one) at 11-qubit tiles up to 28 qubits and 12 above; the
// FP32 SIMT pass below, at the context's complex64 tile width.
struct C64Choice {
    uint32_t m;
    bool tc;
};
C64Choice c64_choice(const mb2_sweep_options& o, uint32_t n, uint32_t default_tile,
                     const std::vector<mb2::Block>& blocks) {
    const bool want_tc = o.c64_kernel == 2 || (o.c64_kernel == 0 && n > 24);
    uint32_t m = o.tile_qubits > 0 ? static_cast<uint32_t>(o.tile_qubits)
                                   : (want_tc && o.c64_kernel == 0 ? (n <= 28 ? 11u : 12u) : default_tile);
    m = std::min(std::min(m, mb2::kMaxTileQubitsC64), n);
    for (const mb2::Block& b : blocks) m = std::max(m, b.k);
    m = std::max(m, mb2::kMinTileQubits);
    return {m, want_tc && m >= 11 && m <= 13};
}

}  // namespace

namespace mb2 {
uint64_t scratch_bound(uint32_t n, const mb2_op* ops, uint32_t num_ops, uint64_t shots, uint32_t terms) {
    auto up = [](uint64_t v) { return (v + 255) & ~uint64_t{255}; };
    // The sweep's upload (mb2_apply_program_monitored): per block at most a
    // phase record, a few gate words and pass padding (144 bytes) and its
    // matrix (16 * 4^k, staged or global-only); blocks never outnumber ops.
    uint64_t program = 4 * 256;
    for (uint32_t i = 0; i < num_ops; ++i)
        if (ops[i].opcode != MB2_MEASURE) program += 144 + (16ull << (2 * ops[i].num_qubits));
    // The sampler (walk_sorted): uniforms, per-shot basis, the walk's scratch.
    const uint64_t sample = shots == 0 ? 0 : 2 * up(8 * shots) + sample_scratch_bytes(n, shots);
    // The expectation (mb2_expectation): masks, partials, results, the
    // groups' span vectors (at most 2^kPauliMaxSpan per group) and terms.
    const uint64_t t = terms;
    const uint64_t expect = terms == 0 ? 0
                                       : 2 * up(8 * t) + up(16 * kExpBlocks * t + 16 * t) +
                                             up(8 * t << kPauliMaxSpan) + sizeof(PauliGroupTerm) * t;
    const uint64_t need = std::max({program, sample, expect});
    uint64_t rounded = uint64_t{1} << 20;  // ensure_scratch's power-of-two growth
    while (rounded < need) rounded <<= 1;
    return rounded;
}

int context_device(const mb2_context* ctx) { return ctx == nullptr ? 0 : ctx->device; }

// A state whose work is queued on a stream the caller owns (the serving
// loop's worker streams); freed with mb2_state_free, which leaves the
// stream alone.
int state_on_stream(mb2_context* ctx, uint32_t num_qubits, uint64_t budget_bytes, void* stream, mb2_state** out,
                    int precision) {
    if (ctx == nullptr || out == nullptr || stream == nullptr) return MB2_ERR_INVALID;
    *out = nullptr;
    if (num_qubits < 1 || num_qubits > 40) return fail(ctx, MB2_ERR_INVALID, "num_qubits must be 1..40");
    if (precision == MB2_C64 && num_qubits < mb2::kMinTileQubits)
        return fail(ctx, MB2_ERR_UNSUPPORTED, "complex64 states need >= 4 qubits");
    const uint64_t bytes = (uint64_t{1} << num_qubits) * amp_bytes(precision);
    if (bytes > budget_bytes) return fail(ctx, MB2_ERR_RESOURCE, "state over budget");
    auto* s = new mb2_state;
    s->ctx = ctx;
    s->n = num_qubits;
    s->precision = precision;
    s->stream = static_cast<cudaStream_t>(stream);
    s->owns_stream = false;
    const cudaError_t e = cudaMallocAsync(&s->amps, bytes, s->stream);
    if (e != cudaSuccess) {
        delete s;
        return cuda_fail(ctx, e, "cudaMallocAsync(state)");
    }
    *out = s;
    return MB2_OK;
}
}  // namespace mb2

namespace mb2 {
namespace {
std::atomic<uint64_t> g_kernel_launches{0};
}
void note_launches(uint32_t k) { g_kernel_launches.fetch_add(k, std::memory_order_relaxed); }
}  // namespace mb2

extern "C" {

int mb2_context_create(int device, mb2_context** out) {
    if (out == nullptr) return MB2_ERR_INVALID;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count <= device || device < 0) {
        cudaGetLastError();
        return MB2_ERR_NO_DEVICE;
    }
    cudaDeviceProp prop{};
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return MB2_ERR_NO_DEVICE;
    if (prop.major < 10) return MB2_ERR_NO_DEVICE;  // sm_100a kernels only
    if (cudaSetDevice(device) != cudaSuccess) return MB2_ERR_NO_DEVICE;
    // Freed states stay in the device's stream-ordered pool for reuse.
    cudaMemPool_t pool = nullptr;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t keep = ~uint64_t{0};
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    auto* ctx = new mb2_context;
    ctx->device = device;
    ctx->sm_count = prop.multiProcessorCount;
    *out = ctx;
    return MB2_OK;
}

int mb2_context_destroy(mb2_context* ctx) {
    delete ctx;
    return MB2_OK;
}

int mb2_last_error(const mb2_context* ctx, char* buf, size_t len) {
    if (ctx == nullptr || buf == nullptr || len == 0) return MB2_ERR_INVALID;
    auto* c = const_cast<mb2_context*>(ctx);
    std::lock_guard<std::mutex> lock(c->mu);
    const size_t n = std::min(len - 1, c->last_error.size());
    std::memcpy(buf, c->last_error.data(), n);
    buf[n] = '\0';
    return MB2_OK;
}

int mb2_device_info(mb2_context* ctx, int* sm_count, uint64_t* total_bytes, uint64_t* free_bytes) {
    if (ctx == nullptr) return MB2_ERR_INVALID;
    MB2_CUDA(ctx, cudaSetDevice(ctx->device));
    size_t fr = 0, tot = 0;
    MB2_CUDA(ctx, cudaMemGetInfo(&fr, &tot));
    if (sm_count) *sm_count = ctx->sm_count;
    if (total_bytes) *total_bytes = tot;
    if (free_bytes) *free_bytes = fr;
    return MB2_OK;
}

int mb2_kernel_launches(uint64_t* out) {
    if (out == nullptr) return MB2_ERR_INVALID;
    *out = mb2::g_kernel_launches.load(std::memory_order_relaxed);
    return MB2_OK;
}

int mb2_probe_rates(mb2_context* ctx, double* fp64_ops_per_s, double* copy_gbs) {
    if (ctx == nullptr || fp64_ops_per_s == nullptr || copy_gbs == nullptr) return MB2_ERR_INVALID;
    MB2_CUDA(ctx, cudaSetDevice(ctx->device));
    const int rc = mb2::probe_rates(ctx->sm_count, fp64_ops_per_s, copy_gbs);
    if (rc != MB2_OK) return fail(ctx, rc, "probe_rates failed");
    return MB2_OK;
}

int mb2_state_alloc(mb2_context* ctx, uint32_t num_qubits, int precision, uint64_t budget_bytes, mb2_state** out) {
    if (ctx == nullptr || out == nullptr) return MB2_ERR_INVALID;
    *out = nullptr;
    if (precision != MB2_C128 && precision != MB2_C64) return fail(ctx, MB2_ERR_INVALID, "unknown precision");
    if (num_qubits < 1 || num_qubits > 40) return fail(ctx, MB2_ERR_INVALID, "num_qubits must be 1..40");
    const uint64_t bytes = (uint64_t{1} << num_qubits) * amp_bytes(precision);
    if (bytes > budget_bytes)
        return fail(ctx, MB2_ERR_RESOURCE,
                    "state needs " + std::to_string(bytes) + " bytes, budget is " + std::to_string(budget_bytes));
    MB2_CUDA(ctx, cudaSetDevice(ctx->device));
    auto* s = new mb2_state;
    s->ctx = ctx;
    s->n = num_qubits;
    s->precision = precision;
    cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete s;
        return cuda_fail(ctx, e, "cudaStreamCreate");
    }
    e = cudaMallocAsync(&s->amps, bytes, s->stream);
    if (e != cudaSuccess) {
        cudaStreamDestroy(s->stream);
        delete s;
        return cuda_fail(ctx, e, "cudaMallocAsync(state)");
    }
    *out = s;
    return MB2_OK;
}

int mb2_state_alloc_host(mb2_context* ctx, uint32_t num_qubits, uint64_t budget_bytes, mb2_state** out) {
    if (ctx == nullptr || out == nullptr) return MB2_ERR_INVALID;
    *out = nullptr;
    if (num_qubits < 1 || num_qubits > 40) return fail(ctx, MB2_ERR_INVALID, "num_qubits must be 1..40");
    const uint64_t bytes = (uint64_t{1} << num_qubits) * amp_bytes(MB2_C128);
    if (bytes > budget_bytes)
        return fail(ctx, MB2_ERR_RESOURCE,
                    "host state needs " + std::to_string(bytes) + " bytes, budget is " + std::to_string(budget_bytes));
    MB2_CUDA(ctx, cudaSetDevice(ctx->device));
    void* host = nullptr;
    cudaError_t e = cudaHostAlloc(&host, bytes, cudaHostAllocMapped | cudaHostAllocPortable);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(ctx, MB2_ERR_RESOURCE, "cudaHostAlloc of " + std::to_string(bytes) + " bytes failed");
    }
    void* dev = nullptr;
    e = cudaHostGetDevicePointer(&dev, host, 0);
    if (e != cudaSuccess) {
        cudaFreeHost(host);
        return cuda_fail(ctx, e, "cudaHostGetDevicePointer");
    }
    auto* s = new mb2_state;
    s->ctx = ctx;
    s->n = num_qubits;
    s->precision = MB2_C128;
    e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        cudaFreeHost(host);
        delete s;
        return cuda_fail(ctx, e, "cudaStreamCreate");
    }
    s->amps = dev;
    s->host_amps = host;
    *out = s;
    return MB2_OK;
}

int mb2_state_host_ptr(mb2_state* s, void** out) {
    if (s == nullptr || out == nullptr) return MB2_ERR_INVALID;
    *out = s->host_amps;
    return MB2_OK;
}

int mb2_state_free(mb2_state* s) {
    if (s == nullptr) return MB2_OK;
    if (s->scratch) cudaFreeAsync(s->scratch, s->stream);
    if (s->host_amps == nullptr) cudaFreeAsync(s->amps, s->stream);
    cudaStreamSynchronize(s->stream);
    if (s->host_amps != nullptr) cudaFreeHost(s->host_amps);
    if (s->owns_stream) cudaStreamDestroy(s->stream);
    delete s;
    return MB2_OK;
}

int mb2_state_device_ptr(mb2_state* s, void** out) {
    if (s == nullptr || out == nullptr) return MB2_ERR_INVALID;
    *out = s->amps;
    return MB2_OK;
}

int mb2_state_stream(mb2_state* s, void** out) {
    if (s == nullptr || out == nullptr) return MB2_ERR_INVALID;
    *out = s->stream;
    return MB2_OK;
}

int mb2_init(mb2_state* s, double global_phase) {
    if (s == nullptr) return MB2_ERR_INVALID;
    const mb2::Cd ph = mb2::initial_phase(global_phase);
    const int rc = mb2::launch_init(s->amps, uint64_t{1} << s->n, s->precision, ph.real(), ph.imag(), s->stream);
    if (rc != MB2_OK) return fail(s->ctx, rc, std::string("init: ") + mb2::last_cuda_error_string());
    return MB2_OK;
}

int mb2_apply_matrix(mb2_state* s, const double* matrix, const uint32_t* operands, uint32_t k) {
    if (s == nullptr || matrix == nullptr || operands == nullptr) return MB2_ERR_INVALID;
    if (s->precision != MB2_C128) return fail(s->ctx, MB2_ERR_UNSUPPORTED, "mb2_apply_matrix: complex128 states only");
    if (int e = check_operands(s, operands, k); e != MB2_OK) return e;
    return apply_block(s, reinterpret_cast<const mb2::Cd*>(matrix), operands, k, false);
}

int mb2_apply_matrix_generic(mb2_state* s, const double* matrix, const uint32_t* operands, uint32_t k) {
    if (s == nullptr || matrix == nullptr || operands == nullptr) return MB2_ERR_INVALID;
    if (s->precision != MB2_C128) return fail(s->ctx, MB2_ERR_UNSUPPORTED, "complex128 states only");
    if (int e = check_operands(s, operands, k); e != MB2_OK) return e;
    return apply_block(s, reinterpret_cast<const mb2::Cd*>(matrix), operands, k, true);
}

int mb2_apply_program_monitored(mb2_state* s, const mb2_op* ops, uint32_t num_ops, const mb2_sweep_options* opts,
                                mb2_boundary_fn boundary, void* user) {
    if (s == nullptr || (ops == nullptr && num_ops != 0)) return MB2_ERR_INVALID;
    mb2_sweep_options o{1, 0, 0, 0, 0, 0};
    if (opts != nullptr) o = *opts;
    for (uint32_t i = 0; i < num_ops; ++i) {
        if (ops[i].opcode == MB2_MEASURE) continue;
        if (ops[i].num_qubits == 0 || ops[i].num_qubits > MB2_MAX_OP_QUBITS)
            return fail(s->ctx, MB2_ERR_INVALID, "operation " + std::to_string(i) + ": operand count");
        if (int e = check_operands(s, ops[i].qubits, ops[i].num_qubits); e != MB2_OK) return e;
    }
    std::vector<mb2::Block> blocks;
    try {
        blocks = mb2::build_blocks(ops, num_ops, o.fuse_gates != 0, static_cast<uint32_t>(o.fusion_width));
    } catch (const std::exception& e) {
        return fail(s->ctx, MB2_ERR_INVALID, e.what());
    }
    s->stats = mb2_sweep_stats{};
    s->stats.blocks = blocks.size();
    if (blocks.empty()) return MB2_OK;
    const bool c64 = s->precision == MB2_C64;
    // The widest tile (fewest passes) unless asked otherwise for a
    // host-resident state, which streams over PCIe once per pass, and for a
    // small one (up to 16 qubits: a 12-qubit tile holds a whole 12-qubit
    // state), whose passes are a few CTAs each and cost their launches.
    const uint32_t dflt = s->host_amps != nullptr || s->n <= 16 ? mb2::kMaxTileQubits : s->ctx->tile_c128.load();
    uint32_t m = tile_width(o.tile_qubits > 0 ? static_cast<uint32_t>(o.tile_qubits) : dflt, s->n, blocks);
    bool tc = false;
    if (c64) {
        // 8-byte amplitudes: up to 13-qubit tiles fit the same shared memory.
        if (s->n < mb2::kMinTileQubits) return fail(s->ctx, MB2_ERR_UNSUPPORTED, "complex64 states need >= 4 qubits");
        const uint32_t tile64 = s->ctx->tile_c64.load() ? s->ctx->tile_c64.load() : mb2::kDefaultTileQubitsC64;
        const C64Choice ch = c64_choice(o, s->n, tile64, blocks);
        m = ch.m;
        tc = ch.tc;
    }
    if (!c64 && (o.per_gate != 0 || s->n < mb2::kMinTileQubits)) {
        for (const mb2::Block& b : blocks) {
            if (int e = apply_block(s, b.m.data(), b.q, b.k, false); e != MB2_OK) return e;
            s->stats.passes += 1;
            if (boundary != nullptr) {
                MB2_CUDA(s->ctx, cudaStreamSynchronize(s->stream));
                if (boundary(user, s->stats.passes) != 0) return fail(s->ctx, MB2_ERR_ABANDONED, "sweep abandoned");
            }
        }
        return MB2_OK;
    }
    mb2::TileProgram prog;
    try {
        const uint32_t low = o.low_qubits < 0 ? 0u : (o.low_qubits == 0 ? mb2::kDefaultFixedLow
                                                                         : static_cast<uint32_t>(o.low_qubits));
        // complex64 results are not bitwise the reference's: commuting
        // blocks may be reordered into fewer passes.
        prog = mb2::plan_tile_program(blocks, s->n, m, low, nullptr, c64);
        if (tc) mb2::make_tensor_core_program(prog, blocks, mb2::tc_max_phases(m));
    } catch (const std::exception& e) {
        return fail(s->ctx, MB2_ERR_INVALID, e.what());
    }
    // One upload: the compact word stream, staged data, global-only data,
    // the tensor-core phase matrices and their error word (256-byte aligned
    // parts).
    const size_t ibytes = prog.words.size() * sizeof(uint32_t);
    const size_t dbytes = prog.data.size() * sizeof(double);
    const size_t gbytes = prog.gdata.size() * sizeof(double);
    const size_t tbytes = prog.tcdata.size() * sizeof(uint32_t);
    const size_t doff = (ibytes + 255) & ~size_t{255};
    const size_t goff = (doff + dbytes + 255) & ~size_t{255};
    const size_t toff = (goff + gbytes + 255) & ~size_t{255};
    const size_t eoff = (toff + tbytes + 255) & ~size_t{255};
    if (int e = ensure_scratch(s, eoff + 256); e != MB2_OK) return e;
    std::vector<unsigned char> host(eoff + sizeof(int), 0);
    std::memcpy(host.data(), prog.words.data(), ibytes);
    if (dbytes) std::memcpy(host.data() + doff, prog.data.data(), dbytes);
    if (gbytes) std::memcpy(host.data() + goff, prog.gdata.data(), gbytes);
    if (tbytes) std::memcpy(host.data() + toff, prog.tcdata.data(), tbytes);
    MB2_CUDA(s->ctx, cudaMemcpyAsync(s->scratch, host.data(), host.size(), cudaMemcpyHostToDevice, s->stream));
    auto* base = static_cast<unsigned char*>(s->scratch);
    const auto* dev_words = reinterpret_cast<const uint32_t*>(base);
    const auto* dev_sdata = reinterpret_cast<const double*>(base + doff);
    const auto* dev_gdata = reinterpret_cast<const double*>(base + goff);
    const auto* dev_tc = reinterpret_cast<const uint32_t*>(base + toff);
    auto* dev_err = reinterpret_cast<int*>(base + eoff);
    s->stats.fp64_ops_per_amp = prog.fp64_per_amp;
    uint64_t done = 0;
    bool any_tc = false;
    // A bounded wait on the tensor core that ran out leaves a nonzero code
    // in the error word; read it whenever the sweep synchronises.
    auto check_tc = [&]() -> int {
        if (!any_tc) return MB2_OK;
        int err = 0;
        MB2_CUDA(s->ctx, cudaMemcpyAsync(&err, dev_err, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
        MB2_CUDA(s->ctx, cudaStreamSynchronize(s->stream));
        if (err != 0) return fail(s->ctx, MB2_ERR_CUDA, "tensor-core pass: a bounded wait ran out");
        return MB2_OK;
    };
    for (const mb2::TilePass& pass : prog.passes) {
        int rc;
        if (pass.tc) {
            any_tc = true;
            rc = mb2::launch_tile_pass_tc(s->amps, s->n, pass, dev_words, dev_sdata, dev_tc, dev_err,
                                          s->ctx->sm_count, s->stream);
        } else if (c64) {
            rc = mb2::launch_tile_pass_c64(s->amps, s->n, pass, dev_words, dev_sdata, dev_gdata, s->ctx->sm_count,
                                           s->stream);
        } else {
            rc = mb2::launch_tile_pass(s->amps, s->n, pass, dev_words, dev_sdata, dev_gdata, s->ctx->sm_count,
                                       s->stream);
        }
        if (rc != MB2_OK) return fail(s->ctx, rc, std::string("tile pass launch: ") + mb2::last_cuda_error_string());
        s->stats.passes += 1;
        s->stats.launches += 1;
        done += pass.gates;
        if (boundary != nullptr) {
            MB2_CUDA(s->ctx, cudaStreamSynchronize(s->stream));
            if (int e = check_tc(); e != MB2_OK) return e;
            if (boundary(user, done) != 0) return fail(s->ctx, MB2_ERR_ABANDONED, "sweep abandoned");
        }
    }
    return check_tc();
}

int mb2_apply_program(mb2_state* s, const mb2_op* ops, uint32_t num_ops, const mb2_sweep_options* opts) {
    return mb2_apply_program_monitored(s, ops, num_ops, opts, nullptr, nullptr);
}

}  // extern "C"

// ---- host-resident states streamed through device windows -------------------
// The reference's chunked tier (src/engines/dense_tiered/pass_plan.h): a state
// of n qubits is 2^(n-L) chunks of 2^L amplitudes (local qubits 0..L-1,
// global qubits L..n-1); a window of 2^W amplitudes holds the 2^g chunks of
// any g <= W - L global qubits G, whose slot bits L..L+g-1 stand for G in
// increasing order, so a block on local qubits and qubits of G runs on the
// window with its operands remapped, and multiplies every amplitude by the
// same entries in the same order as on the whole state.
namespace {

struct WindowPass {
    uint64_t global_mask;  // bit g - L for each global qubit g in G
    size_t first, end;     // blocks [first, end)
};
struct WindowPlan {
    uint32_t chunk_qubits = 0, window_qubits = 0;
    std::vector<WindowPass> passes;
    bool too_small = false;
};

// The greedy rule of build_pass_plan (pass_plan.cpp:43-121) over the fusion
// plan's blocks: a pass opens with the first block's global operands as G
// and absorbs each following block while G stays within W - L qubits.
WindowPlan window_plan(const std::vector<mb2::Block>& blocks, uint32_t L, uint32_t W) {
    WindowPlan p;
    p.chunk_qubits = L;
    p.window_qubits = W;
    const int wg = static_cast<int>(W - L);
    bool open = false;
    uint64_t group = 0;
    size_t first = 0;
    for (size_t i = 0; i < blocks.size(); ++i) {
        uint64_t mask = 0;
        for (uint32_t j = 0; j < blocks[i].k; ++j)
            if (blocks[i].q[j] >= L) mask |= uint64_t{1} << (blocks[i].q[j] - L);
        if (std::popcount(mask) > wg) p.too_small = true;
        if (!open) {
            open = true;
            group = mask;
            continue;
        }
        const uint64_t merged = group | mask;
        if (std::popcount(merged) <= wg) {
            group = merged;
        } else {
            p.passes.push_back(WindowPass{group, first, i});
            first = i;
            group = mask;
        }
    }
    if (open) p.passes.push_back(WindowPass{group, first, blocks.size()});
    return p;
}

// Smallest chunk the automatic choice takes: 2^16 amplitudes (1 MiB a copy).
constexpr uint32_t kMinWindowChunkQubits = 16;

// The chunk size as choose_pass_plan picks it (pass_plan.cpp:123-150): the
// fewest passes, the larger chunk on a tie, among chunks from 2^24
// amplitudes up to the window, smaller ones only when none of those fits the
// blocks -- except that for a window of at most 2^24 the search starts
// below at 2^min(16, W) rather than at one amplitude (a device copy of less
// than 1 MiB costs more in calls than it saves in passes), and no chunk is
// below the tile kernels' 2^4.  W >= 4.
WindowPlan choose_window_plan(const std::vector<mb2::Block>& blocks, uint32_t W) {
    const uint32_t lowest = W > 24 ? 24u : std::min(W, kMinWindowChunkQubits);
    WindowPlan best;
    best.too_small = true;
    for (uint32_t L = W;; --L) {
        if (L < lowest && !best.too_small) break;
        WindowPlan p = window_plan(blocks, L, W);
        if (!p.too_small && (best.too_small || p.passes.size() < best.passes.size())) best = std::move(p);
        if (L <= mb2::kMinTileQubits) break;
    }
    return best;
}

uint64_t pdep_host(uint64_t v, uint64_t mask) {
    uint64_t r = 0;
    for (uint64_t m = mask; m != 0; m &= m - 1) {
        if (v & 1u) r |= m & (~m + 1);
        v >>= 1;
    }
    return r;
}

// The blocks of a fusion plan, validated against n qubits.
int window_blocks(mb2_context* ctx, uint32_t n, const mb2_op* ops, uint32_t num_ops, const mb2_sweep_options* opts,
                  std::vector<mb2::Block>& blocks) {
    mb2_sweep_options o{1, 0, 0, 0, 0, 0};
    if (opts != nullptr) o = *opts;
    for (uint32_t i = 0; i < num_ops; ++i) {
        if (ops[i].opcode == MB2_MEASURE) continue;
        if (ops[i].num_qubits == 0 || ops[i].num_qubits > MB2_MAX_OP_QUBITS)
            return fail(ctx, MB2_ERR_INVALID, "operation " + std::to_string(i) + ": operand count");
        for (uint32_t j = 0; j < ops[i].num_qubits; ++j)
            if (ops[i].qubits[j] >= n) return fail(ctx, MB2_ERR_INVALID, "operation " + std::to_string(i) + ": operand out of range");
    }
    try {
        blocks = mb2::build_blocks(ops, num_ops, o.fuse_gates != 0, static_cast<uint32_t>(o.fusion_width));
    } catch (const std::exception& e) {
        return fail(ctx, MB2_ERR_INVALID, e.what());
    }
    return MB2_OK;
}

int plan_windows(mb2_context* ctx, const std::vector<mb2::Block>& blocks, uint32_t n, uint32_t W, uint32_t L,
                 WindowPlan& plan) {
    if (W < mb2::kMinTileQubits || W > n) return fail(ctx, MB2_ERR_INVALID, "the window holds 4..n qubits");
    if (L != 0 && (L < mb2::kMinTileQubits || L > W))
        return fail(ctx, MB2_ERR_INVALID, "a chunk holds 4..window qubits (0: chosen)");
    plan = L != 0 ? window_plan(blocks, L, W) : choose_window_plan(blocks, W);
    if (plan.too_small)
        return fail(ctx, MB2_ERR_INVALID, "a block has more operands above the chunk than the window holds");
    return MB2_OK;
}

}  // namespace

extern "C" {

int mb2_window_plan(const mb2_op* ops, uint32_t num_ops, const mb2_sweep_options* opts, uint32_t num_qubits,
                    uint32_t window_qubits, uint32_t chunk_qubits, uint64_t* out, uint64_t* out_words) {
    if ((ops == nullptr && num_ops != 0) || out_words == nullptr || num_qubits < 1 || num_qubits > 40)
        return MB2_ERR_INVALID;
    std::vector<mb2::Block> blocks;
    if (int e = window_blocks(nullptr, num_qubits, ops, num_ops, opts, blocks); e != MB2_OK) return e;
    WindowPlan plan;
    if (int e = plan_windows(nullptr, blocks, num_qubits, window_qubits, chunk_qubits, plan); e != MB2_OK) return e;
    std::vector<uint64_t> w{plan.chunk_qubits, plan.window_qubits, plan.passes.size()};
    for (const WindowPass& p : plan.passes) {
        w.push_back(p.global_mask);
        w.push_back(p.first);
        w.push_back(p.end);
    }
    const uint64_t cap = *out_words;
    *out_words = w.size();
    if (out == nullptr || cap < w.size()) return MB2_ERR_INVALID;
    std::copy(w.begin(), w.end(), out);
    return MB2_OK;
}

int mb2_apply_program_windowed(mb2_state* s, const mb2_op* ops, uint32_t num_ops, const mb2_sweep_options* opts,
                               uint32_t window_qubits, uint32_t chunk_qubits) {
    if (s == nullptr || (ops == nullptr && num_ops != 0)) return MB2_ERR_INVALID;
    mb2_context* ctx = s->ctx;
    if (s->host_amps == nullptr) return fail(ctx, MB2_ERR_INVALID, "windowed sweeps take a host-resident state");
    if (s->precision != MB2_C128) return fail(ctx, MB2_ERR_UNSUPPORTED, "windowed sweeps: complex128 states only");
    const uint32_t n = s->n;
    std::vector<mb2::Block> blocks;
    if (int e = window_blocks(ctx, n, ops, num_ops, opts, blocks); e != MB2_OK) return e;
    s->stats = mb2_sweep_stats{};
    s->stats.blocks = blocks.size();
    if (blocks.empty()) return MB2_OK;
    WindowPlan plan;
    if (int e = plan_windows(ctx, blocks, n, window_qubits, chunk_qubits, plan); e != MB2_OK) return e;
    const uint32_t L = plan.chunk_qubits, W = plan.window_qubits;
    // Chunk bookkeeping is one entry per chunk: at most 2^24 of them.
    if (n - L > 24) return fail(ctx, MB2_ERR_INVALID, "chunks of at least 2^(n - 24) amplitudes");
    MB2_CUDA(ctx, cudaSetDevice(ctx->device));
    // Whatever the state's own stream wrote (initialisation, earlier calls
    // through the mapped alias) lands before the copies read the host buffer.
    MB2_CUDA(ctx, cudaStreamSynchronize(s->stream));
    // Two windows, each with its stream: a window's copies in, sweep and
    // copies out are ordered on its stream, and the two streams overlap, so
    // one window's copies run while the other is swept.  Groups alternate
    // between them across passes.
    const size_t win_bytes = (size_t{1} << W) * 16;
    size_t free_bytes = 0, total_bytes = 0;
    MB2_CUDA(ctx, cudaMemGetInfo(&free_bytes, &total_bytes));
    if (2 * win_bytes + (size_t{64} << 20) > free_bytes)
        return fail(ctx, MB2_ERR_RESOURCE, "two windows of " + std::to_string(win_bytes) + " bytes do not fit the device");
    struct Res {
        cudaStream_t st[2] = {nullptr, nullptr};
        void* win[2] = {nullptr, nullptr};
        void* prog = nullptr;
        std::vector<cudaEvent_t> events;
        ~Res() {
            for (cudaStream_t t : st)
                if (t != nullptr) cudaStreamSynchronize(t);
            for (cudaEvent_t e : events) cudaEventDestroy(e);
            for (void* p : win)
                if (p != nullptr) cudaFree(p);
            if (prog != nullptr) cudaFree(prog);
            for (cudaStream_t t : st)
                if (t != nullptr) cudaStreamDestroy(t);
        }
    } r;
    for (int b = 0; b < 2; ++b) {
        MB2_CUDA(ctx, cudaStreamCreateWithFlags(&r.st[b], cudaStreamNonBlocking));
        MB2_CUDA(ctx, cudaMalloc(&r.win[b], win_bytes));
    }
    // Every pass's tiled program, planned on its window qubits (local qubits
    // stay, global qubit L + b becomes L + its rank among G) and uploaded once.
    struct PassProg {
        mb2::TileProgram prog;
        uint32_t n_eff = 0;
        size_t off = 0, doff = 0, goff = 0;
    };
    std::vector<PassProg> progs(plan.passes.size());
    size_t total = 0;
    for (size_t pi = 0; pi < plan.passes.size(); ++pi) {
        const WindowPass& wp = plan.passes[pi];
        const uint32_t n_eff = L + static_cast<uint32_t>(std::popcount(wp.global_mask));
        std::vector<mb2::Block> local(blocks.begin() + static_cast<std::ptrdiff_t>(wp.first),
                                      blocks.begin() + static_cast<std::ptrdiff_t>(wp.end));
        for (mb2::Block& b : local)
            for (uint32_t j = 0; j < b.k; ++j)
                if (b.q[j] >= L) {
                    const uint32_t bit = b.q[j] - L;
                    b.q[j] = L + static_cast<uint32_t>(std::popcount(wp.global_mask & ((uint64_t{1} << bit) - 1)));
                }
        const uint32_t dflt = n_eff <= 16 ? mb2::kMaxTileQubits : ctx->tile_c128.load();
        const uint32_t m = std::min(tile_width(dflt, n_eff, local), n_eff);
        PassProg& pp = progs[pi];
        try {
            pp.prog = mb2::plan_tile_program(local, n_eff, m);
        } catch (const std::exception& e) {
            return fail(ctx, MB2_ERR_INVALID, e.what());
        }
        pp.n_eff = n_eff;
        pp.off = total;
        pp.doff = total + ((pp.prog.words.size() * sizeof(uint32_t) + 255) & ~size_t{255});
        pp.goff = pp.doff + ((pp.prog.data.size() * sizeof(double) + 255) & ~size_t{255});
        total = pp.goff + ((pp.prog.gdata.size() * sizeof(double) + 255) & ~size_t{255}) + 256;
    }
    {
        std::vector<unsigned char> staged(total, 0);
        for (const PassProg& pp : progs) {
            std::memcpy(staged.data() + pp.off, pp.prog.words.data(), pp.prog.words.size() * sizeof(uint32_t));
            if (!pp.prog.data.empty())
                std::memcpy(staged.data() + pp.doff, pp.prog.data.data(), pp.prog.data.size() * sizeof(double));
            if (!pp.prog.gdata.empty())
                std::memcpy(staged.data() + pp.goff, pp.prog.gdata.data(), pp.prog.gdata.size() * sizeof(double));
        }
        MB2_CUDA(ctx, cudaMalloc(&r.prog, total));
        MB2_CUDA(ctx, cudaMemcpy(r.prog, staged.data(), total, cudaMemcpyHostToDevice));
    }
    auto* pbase = static_cast<unsigned char*>(r.prog);
    auto* host = static_cast<unsigned char*>(s->host_amps);
    const uint64_t global_bits = n - L;
    const uint64_t all_globals = global_bits >= 64 ? ~uint64_t{0} : (uint64_t{1} << global_bits) - 1;
    // No barrier between passes: each chunk remembers the event recorded
    // after the copy that last wrote it back, and a group's copies in wait on
    // the events of the chunks it reads (which are the chunks it writes), so
    // a group starts as soon as its own chunks are home and the two copy
    // directions stay busy across pass boundaries.
    std::vector<cudaEvent_t> last_writer(size_t{1} << global_bits, nullptr);
    uint64_t turn = 0;  // alternates the windows across groups and passes
    std::vector<cudaEvent_t> waits;
    for (size_t pi = 0; pi < plan.passes.size(); ++pi) {
        const WindowPass& wp = plan.passes[pi];
        const PassProg& pp = progs[pi];
        const uint32_t g = static_cast<uint32_t>(std::popcount(wp.global_mask));
        const auto* dev_words = reinterpret_cast<const uint32_t*>(pbase + pp.off);
        const auto* dev_sdata = reinterpret_cast<const double*>(pbase + pp.doff);
        const auto* dev_gdata = reinterpret_cast<const double*>(pbase + pp.goff);
        // Chunks whose slots follow each other and whose host addresses do too
        // (the lowest global qubits, when G holds them) move in one copy.
        const uint32_t run = static_cast<uint32_t>(std::countr_one(wp.global_mask));
        const size_t copy_bytes = (size_t{1} << (L + run)) * 16;
        const uint64_t other = all_globals & ~wp.global_mask;
        const uint64_t groups = uint64_t{1} << (global_bits - g);
        for (uint64_t grp = 0; grp < groups; ++grp, ++turn) {
            const int b = static_cast<int>(turn & 1u);
            cudaStream_t st = r.st[b];
            auto* win = static_cast<unsigned char*>(r.win[b]);
            const uint64_t base_chunk = pdep_host(grp, other);
            waits.clear();
            for (uint64_t slot = 0; slot < (uint64_t{1} << g); ++slot) {
                const cudaEvent_t e = last_writer[base_chunk | pdep_host(slot, wp.global_mask)];
                if (e != nullptr && std::find(waits.begin(), waits.end(), e) == waits.end()) waits.push_back(e);
            }
            for (cudaEvent_t e : waits) MB2_CUDA(ctx, cudaStreamWaitEvent(st, e, 0));
            for (uint64_t slot = 0; slot < (uint64_t{1} << g); slot += uint64_t{1} << run) {
                const uint64_t chunk = base_chunk | pdep_host(slot, wp.global_mask);
                MB2_CUDA(ctx, cudaMemcpyAsync(win + ((slot << L) * 16), host + ((chunk << L) * 16), copy_bytes,
                                              cudaMemcpyHostToDevice, st));
            }
            for (const mb2::TilePass& pass : pp.prog.passes) {
                const int rc = mb2::launch_tile_pass(win, pp.n_eff, pass, dev_words, dev_sdata, dev_gdata,
                                                     ctx->sm_count, st);
                if (rc != MB2_OK) return fail(ctx, rc, std::string("tile pass launch: ") + mb2::last_cuda_error_string());
                s->stats.launches += 1;
            }
            for (uint64_t slot = 0; slot < (uint64_t{1} << g); slot += uint64_t{1} << run) {
                const uint64_t chunk = base_chunk | pdep_host(slot, wp.global_mask);
                MB2_CUDA(ctx, cudaMemcpyAsync(host + ((chunk << L) * 16), win + ((slot << L) * 16), copy_bytes,
                                              cudaMemcpyDeviceToHost, st));
            }
            cudaEvent_t done = nullptr;
            MB2_CUDA(ctx, cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
            r.events.push_back(done);
            MB2_CUDA(ctx, cudaEventRecord(done, st));
            for (uint64_t slot = 0; slot < (uint64_t{1} << g); ++slot)
                last_writer[base_chunk | pdep_host(slot, wp.global_mask)] = done;
        }
        s->stats.passes += 1;
    }
    MB2_CUDA(ctx, cudaStreamSynchronize(r.st[0]));
    MB2_CUDA(ctx, cudaStreamSynchronize(r.st[1]));
    return MB2_OK;
}

int mb2_fusion_plan(const mb2_op* ops, uint32_t num_ops, const mb2_sweep_options* opts, uint32_t* order,
                    uint32_t* block_begin, uint32_t* block_qubits, uint32_t* qubits_begin, uint64_t* num_blocks,
                    uint64_t* num_block_qubits) {
    if ((ops == nullptr && num_ops != 0) || num_blocks == nullptr || num_block_qubits == nullptr)
        return MB2_ERR_INVALID;
    mb2_sweep_options o{1, 0, 0, 0, 0, 0};
    if (opts != nullptr) o = *opts;
    mb2::FusionPlanArrays plan;
    try {
        mb2::build_blocks(ops, num_ops, true, static_cast<uint32_t>(o.fusion_width), &plan);
    } catch (const std::exception&) {
        return MB2_ERR_INVALID;
    }
    const uint64_t blocks = plan.block_begin.size() - 1;
    const uint64_t cap_b = *num_blocks, cap_q = *num_block_qubits;
    *num_blocks = blocks;
    *num_block_qubits = plan.block_qubits.size();
    if (order == nullptr || block_begin == nullptr || qubits_begin == nullptr ||
        (block_qubits == nullptr && !plan.block_qubits.empty()) || cap_b < blocks || cap_q < plan.block_qubits.size())
        return MB2_ERR_INVALID;
    std::copy(plan.order.begin(), plan.order.end(), order);
    std::copy(plan.block_begin.begin(), plan.block_begin.end(), block_begin);
    std::copy(plan.block_qubits.begin(), plan.block_qubits.end(), block_qubits);
    std::copy(plan.qubits_begin.begin(), plan.qubits_begin.end(), qubits_begin);
    return MB2_OK;
}

int mb2_estimate_sweep(const mb2_op* ops, uint32_t num_ops, const mb2_sweep_options* opts, uint32_t num_qubits,
                       mb2_sweep_estimate* out) {
    if (out == nullptr || (ops == nullptr && num_ops != 0) || num_qubits < 1 || num_qubits > 40) return MB2_ERR_INVALID;
    mb2_sweep_options o{1, 0, 0, 0, 0, 0};
    if (opts != nullptr) o = *opts;
    *out = mb2_sweep_estimate{};
    try {
        const std::vector<mb2::Block> blocks = mb2::build_blocks(ops, num_ops, o.fuse_gates != 0, static_cast<uint32_t>(o.fusion_width));
        out->blocks = blocks.size();
        out->work_units = uint64_t{1} << num_qubits;
        for (const mb2::Block& b : blocks) out->work_units += uint64_t{1} << (num_qubits + b.k);
        out->device_bytes = (uint64_t{1} << num_qubits) * 16;
        if (o.per_gate != 0 || num_qubits < mb2::kMinTileQubits || blocks.empty()) {
            out->passes = blocks.size();
            out->launches = blocks.size() + 1;
            for (const mb2::Block& b : blocks) out->h2d_bytes += 16ull << (2 * b.k);
        } else {
            const uint32_t m = tile_width(o.tile_qubits > 0 ? static_cast<uint32_t>(o.tile_qubits) : 0, num_qubits,
                                          blocks);
            const mb2::TileProgram prog = mb2::plan_tile_program(blocks, num_qubits, m);
            out->passes = prog.passes.size();
            out->launches = prog.passes.size() + 1;
            out->h2d_bytes = prog.words.size() * sizeof(uint32_t) + (prog.data.size() + prog.gdata.size()) * sizeof(double);
            out->fp64_ops_per_amp = prog.fp64_per_amp;
        }
        out->device_bytes += out->h2d_bytes;
    } catch (const std::exception&) {
        return MB2_ERR_INVALID;
    }
    return MB2_OK;
}

int mb2_last_sweep_stats(mb2_state* s, mb2_sweep_stats* out) {
    if (s == nullptr || out == nullptr) return MB2_ERR_INVALID;
    *out = s->stats;
    return MB2_OK;
}

int mb2_expectation(mb2_state* s, const uint64_t* x_masks, const uint64_t* z_masks, uint32_t num_terms, double* out) {
    if (s == nullptr || (num_terms != 0 && (x_masks == nullptr || z_masks == nullptr || out == nullptr)))
        return MB2_ERR_INVALID;
    if (num_terms == 0) return MB2_OK;
    const uint64_t lim = (s->n >= 64) ? ~uint64_t{0} : ((uint64_t{1} << s->n) - 1);
    for (uint32_t t = 0; t < num_terms; ++t)
        if ((x_masks[t] | z_masks[t]) & ~lim) return fail(s->ctx, MB2_ERR_INVALID, "Pauli mask beyond the state's qubits");
    // Terms are grouped so that each group reads the state once (one launch
    // per group); the fixed-order finish then adds every term's partials.
    const mb2::PauliPlan plan = mb2::plan_pauli_groups(x_masks, z_masks, num_terms, s->n);
    const size_t mask_bytes = size_t{num_terms} * 8;
    const size_t part_bytes = size_t{num_terms} * mb2::kExpBlocks * 16;
    const size_t out_bytes = size_t{num_terms} * 16;
    const size_t span_bytes = plan.spans.size() * 8;
    const size_t term_bytes = plan.terms.size() * sizeof(mb2::PauliGroupTerm);
    auto up = [](size_t v) { return (v + 255) & ~size_t{255}; };
    const size_t off_z = up(mask_bytes);
    const size_t off_p = off_z + up(mask_bytes);
    const size_t off_o = off_p + part_bytes;
    const size_t off_s = up(off_o + out_bytes);
    const size_t off_t = off_s + up(span_bytes);
    if (int e = ensure_scratch(s, off_t + term_bytes); e != MB2_OK) return e;
    auto* base = static_cast<unsigned char*>(s->scratch);
    std::vector<unsigned char> host(off_t + term_bytes - off_s);
    std::memcpy(host.data(), plan.spans.data(), span_bytes);
    std::memcpy(host.data() + (off_t - off_s), plan.terms.data(), term_bytes);
    MB2_CUDA(s->ctx, cudaMemcpyAsync(base, x_masks, mask_bytes, cudaMemcpyHostToDevice, s->stream));
    MB2_CUDA(s->ctx, cudaMemcpyAsync(base + off_z, z_masks, mask_bytes, cudaMemcpyHostToDevice, s->stream));
    MB2_CUDA(s->ctx, cudaMemcpyAsync(base + off_s, host.data(), host.size(), cudaMemcpyHostToDevice, s->stream));
    auto* partials = reinterpret_cast<double*>(base + off_p);
    for (const mb2::PauliGroupPlan& g : plan.groups) {
        if (g.nterms == 1 || g.c + g.d < mb2::kPauliMinTileQubits) {
            // Nothing to share (or a state too small for the grouped tiles):
            // one streaming read per term, its partials in place.
            for (uint32_t i = 0; i < g.nterms; ++i) {
                const uint32_t t = plan.terms[g.term_off + i].out;
                const int rc = mb2::launch_expectation_partials(
                    s->amps, s->n, reinterpret_cast<const uint64_t*>(base) + t,
                    reinterpret_cast<const uint64_t*>(base + off_z) + t, 1,
                    partials + 2 * static_cast<size_t>(t) * mb2::kExpBlocks, s->stream, s->precision);
                if (rc != MB2_OK)
                    return fail(s->ctx, rc, std::string("expectation launch: ") + mb2::last_cuda_error_string());
            }
            continue;
        }
        const int rc = mb2::launch_pauli_group(
            s->amps, s->n, g.c, g.d, reinterpret_cast<const uint64_t*>(base + off_s) + g.span_off, g.free_mask,
            base + off_t + size_t{g.term_off} * sizeof(mb2::PauliGroupTerm), g.nterms, partials, mb2::kExpBlocks,
            s->stream, s->precision);
        if (rc != MB2_OK) return fail(s->ctx, rc, std::string("expectation launch: ") + mb2::last_cuda_error_string());
    }
    const int rc = mb2::launch_expectation_finish(partials, mb2::kExpBlocks, reinterpret_cast<const uint64_t*>(base),
                                                  reinterpret_cast<const uint64_t*>(base + off_z), num_terms,
                                                  reinterpret_cast<double*>(base + off_o), s->stream);
    if (rc != MB2_OK) return fail(s->ctx, rc, std::string("expectation launch: ") + mb2::last_cuda_error_string());
    MB2_CUDA(s->ctx, cudaMemcpyAsync(out, base + off_o, out_bytes, cudaMemcpyDeviceToHost, s->stream));
    MB2_CUDA(s->ctx, cudaStreamSynchronize(s->stream));
    return MB2_OK;
}

int mb2_normalize(mb2_state* s, double* norm_before) {
    if (s == nullptr) return MB2_ERR_INVALID;
    double nrm = 0.0;
    if (int e = mb2_norm(s, &nrm); e != MB2_OK) return e;
    if (norm_before != nullptr) *norm_before = nrm;
    if (!(nrm > 0.0)) return fail(s->ctx, MB2_ERR_INVALID, "cannot normalise a zero state");
    if (s->precision != MB2_C64) return MB2_OK;  // complex128 states are left exactly as computed
    const double scale = 1.0 / std::sqrt(nrm);
    const int rc = mb2::launch_scale_c64(s->amps, uint64_t{1} << s->n, static_cast<float>(scale), s->stream);
    if (rc != MB2_OK) return fail(s->ctx, rc, "normalise launch");
    return MB2_OK;
}

int mb2_norm(mb2_state* s, double* out) {
    if (s == nullptr || out == nullptr) return MB2_ERR_INVALID;
    const uint64_t zero = 0;
    double v[2];
    if (int e = mb2_expectation(s, &zero, &zero, 1, v); e != MB2_OK) return e;
    *out = v[0];
    return MB2_OK;
}

}  // extern "C"

namespace {

// Uniforms exactly as common::Rng (src/common/rng.cpp:176-186), sorted
// (src/engines/dense/sample.cpp:37-42).  u = k * 2^-53 with k the top 53
// bits of a word, so sorting the integers k sorts the uniforms: one
// counting pass on the top 12 bits, then the buckets (about shots / 4096
// keys each, uniform) sorted independently on a few host threads.
std::vector<double> sorted_uniforms(uint64_t shots, uint64_t seed) {
    std::vector<double> u(shots);
    {
        std::vector<uint64_t> key(shots), sorted(shots);
        std::mt19937_64 eng(seed);
        for (uint64_t i = 0; i < shots; ++i) key[i] = eng() >> 11;
        constexpr uint32_t kBits = 12, kBuckets = 1u << kBits;
        std::vector<uint64_t> start(kBuckets + 1, 0);
        for (uint64_t i = 0; i < shots; ++i) ++start[(key[i] >> (53 - kBits)) + 1];
        for (uint32_t b = 0; b < kBuckets; ++b) start[b + 1] += start[b];
        {
            std::vector<uint64_t> pos(start.begin(), start.end() - 1);
            for (uint64_t i = 0; i < shots; ++i) sorted[pos[key[i] >> (53 - kBits)]++] = key[i];
        }
        const uint32_t nthreads = shots < (1u << 16) ? 1u : std::max(1u, std::min(8u, std::thread::hardware_concurrency()));
        auto sort_range = [&](uint32_t w) {
            for (uint32_t b = w; b < kBuckets; b += nthreads) {
                std::sort(sorted.begin() + static_cast<long>(start[b]), sorted.begin() + static_cast<long>(start[b + 1]));
                for (uint64_t i = start[b]; i < start[b + 1]; ++i)
                    u[i] = static_cast<double>(sorted[i]) * (1.0 / 9007199254740992.0);
            }
        };
        std::vector<std::thread> pool;
        for (uint32_t w = 1; w < nthreads; ++w) pool.emplace_back(sort_range, w);
        sort_range(0);
        for (auto& th : pool) th.join();
    }
    return u;
}

// The walk's basis states (non-decreasing) as counts of the measured
// outcomes, ascending: mb2_sample's output.
int histogram(mb2_context* ctx, uint32_t n, const std::vector<uint64_t>& basis, const uint32_t* targets,
              uint32_t num_targets, uint64_t* outcomes, uint64_t* counts, uint64_t* num_outcomes) {
    const uint64_t shots = basis.size();
    // Outcomes through the measure targets, ascending, with counts.  The walk
    // gives non-decreasing basis indices (sorted uniforms against the
    // cumulative sum), so runs are counted first; the distinct outcomes are
    // sorted only when the target map does not keep their order.
    // Outcome of a basis index: one table per byte of the index (the OR of
    // the target bits that byte carries), or the index itself when every
    // qubit is read into the clbit of its own number.
    bool identity = num_targets == n;
    std::vector<uint64_t> table(8 * 256, 0);
    for (uint32_t t = 0; t < num_targets; ++t) {
        const uint32_t q = targets[2 * t], c = targets[2 * t + 1];
        if (q != c) identity = false;
        for (uint32_t v = 0; v < 256; ++v)
            if ((v >> (q & 7u)) & 1u) table[(q >> 3) * 256 + v] |= uint64_t{1} << c;
    }
    if (identity) {
        uint64_t seen = 0;
        for (uint32_t t = 0; t < num_targets; ++t) seen |= uint64_t{1} << targets[2 * t];
        identity = seen == ((n >= 64) ? ~uint64_t{0} : ((uint64_t{1} << n) - 1));
    }
    const uint32_t nbytes = (n + 7) / 8;
    auto outcome_of = [&](uint64_t b) {
        if (identity) return b;
        uint64_t o = 0;
        for (uint32_t k = 0; k < nbytes; ++k) o |= table[k * 256 + ((b >> (8 * k)) & 255u)];
        return o;
    };
    std::vector<std::pair<uint64_t, uint64_t>> oc;
    oc.reserve(std::min<uint64_t>(shots, uint64_t{1} << std::min<uint32_t>(n, 30)));
    for (uint64_t i = 0; i < shots;) {
        uint64_t j = i + 1;
        while (j < shots && basis[j] == basis[i]) ++j;
        oc.emplace_back(outcome_of(basis[i]), j - i);
        i = j;
    }
    bool ordered = true;
    for (size_t i = 1; i < oc.size() && ordered; ++i) ordered = oc[i - 1].first < oc[i].first;
    if (!ordered) std::sort(oc.begin(), oc.end());
    uint64_t d = 0;
    for (const auto& [o, c] : oc) {
        if (d > 0 && outcomes[d - 1] == o) {
            counts[d - 1] += c;
            continue;
        }
        if (d >= *num_outcomes) return fail(ctx, MB2_ERR_INVALID, "outcome capacity too small");
        outcomes[d] = o;
        counts[d] = c;
        ++d;
    }
    *num_outcomes = d;
    return MB2_OK;
}

}  // namespace

namespace mb2 {
std::vector<double> sorted_reference_uniforms(uint64_t shots, uint64_t seed) { return sorted_uniforms(shots, seed); }
int counts_of(mb2_context* ctx, uint32_t n, const std::vector<uint64_t>& basis, const uint32_t* targets,
              uint32_t num_targets, uint64_t* outcomes, uint64_t* counts, uint64_t* num_outcomes) {
    return histogram(ctx, n, basis, targets, num_targets, outcomes, counts, num_outcomes);
}
}  // namespace mb2

extern "C" {

int mb2_sample(mb2_state* s, uint64_t shots, uint64_t seed, const uint32_t* targets, uint32_t num_targets,
               uint64_t* outcomes, uint64_t* counts, uint64_t* num_outcomes) {
    if (s == nullptr || num_outcomes == nullptr) return MB2_ERR_INVALID;
    for (uint32_t t = 0; t < num_targets; ++t)
        if (targets[2 * t] >= s->n || targets[2 * t + 1] >= 64)
            return fail(s->ctx, MB2_ERR_INVALID, "measure target out of range");
    if (shots == 0) {
        *num_outcomes = 0;
        return MB2_OK;
    }
    const std::vector<double> u = sorted_uniforms(shots, seed);
    std::vector<uint64_t> basis(shots);
    if (int e = walk_sorted(s, u, basis.data()); e != MB2_OK) return e;
    return histogram(s->ctx, s->n, basis, targets, num_targets, outcomes, counts, num_outcomes);
}

int mb2_sample_basis(mb2_state* s, const double* uniforms, uint64_t n, uint64_t* basis_out) {
    if (s == nullptr || (n != 0 && (uniforms == nullptr || basis_out == nullptr))) return MB2_ERR_INVALID;
    if (n == 0) return MB2_OK;
    for (uint64_t i = 0; i < n; ++i)
        if (!(uniforms[i] >= 0.0 && uniforms[i] < 1.0))
            return fail(s->ctx, MB2_ERR_INVALID, "uniforms must lie in [0, 1)");
    // Draw order -> ascending order (ties keep draw order), one walk, back.
    std::vector<uint64_t> order(n);
    for (uint64_t i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](uint64_t a, uint64_t b) { return uniforms[a] < uniforms[b]; });
    std::vector<double> u(n);
    for (uint64_t i = 0; i < n; ++i) u[i] = uniforms[order[i]];
    std::vector<uint64_t> basis(n);
    if (int e = walk_sorted(s, u, basis.data()); e != MB2_OK) return e;
    for (uint64_t i = 0; i < n; ++i) basis_out[order[i]] = basis[i];
    return MB2_OK;
}

// ---- density matrices ------------------------------------------------------
// The reference's density-matrix engine (src/engines/density_matrix/
// density_matrix_engine.cpp): rho as a 2n-qubit vector, entry (r, c) at
// r | c << n.

}  // extern "C"

namespace {

// A channel's superoperator on (q, q + n): S[(r | c << k), (r2 | c2 << k)] =
// sum over the Kraus operators K, in order, of K[r][r2] conj(K[c][c2]) --
// the reference's construction and summation order (superoperator(),
// density_matrix_engine.cpp), so its bits are the reference's.
std::vector<mb2::Cd> superoperator(const std::vector<std::vector<mb2::Cd>>& kraus, uint32_t k) {
    const size_t dim = size_t{1} << k, sdim = dim * dim;
    std::vector<mb2::Cd> sop(sdim * sdim, mb2::Cd{0.0, 0.0});
    for (const std::vector<mb2::Cd>& op : kraus)
        for (size_t r = 0; r < dim; ++r)
            for (size_t c = 0; c < dim; ++c) {
                const size_t row = r | (c << k);
                for (size_t r2 = 0; r2 < dim; ++r2)
                    for (size_t c2 = 0; c2 < dim; ++c2)
                        sop[row * sdim + (r2 | (c2 << k))] += op[r * dim + r2] * std::conj(op[c * dim + c2]);
            }
    return sop;
}

int check_rho(mb2_state* rho, uint32_t n) {
    if (rho == nullptr) return MB2_ERR_INVALID;
    if (n < 1 || n > 15 || rho->n != 2 * n || rho->precision != MB2_C128)
        return fail(rho->ctx, MB2_ERR_INVALID, "a density matrix of n qubits is a complex128 state of 2n qubits, n <= 15");
    return MB2_OK;
}

}  // namespace

extern "C" {

int mb2_dm_apply_program(mb2_state* rho, uint32_t n, const mb2_op* ops, uint32_t num_ops) {
    if (int e = check_rho(rho, n); e != MB2_OK) return e;
    if (ops == nullptr && num_ops != 0) return MB2_ERR_INVALID;
    // Each operation as 2n-qubit blocks, applied one by one in order (the
    // reference fuses nothing here): a gate U on q and conj(U) on q + n; a
    // channel's superoperator on q and q + n.  Runs of blocks of up to six
    // operands go through the sweep; a 4- or 5-qubit channel's 8- or
    // 10-operand superoperator through the wide generic kernel.
    std::vector<mb2_op> out;
    std::vector<std::vector<double>> keep;
    auto block = [&](const std::vector<mb2::Cd>& m, const uint32_t* q, uint32_t k) {
        mb2_op o{};
        o.opcode = MB2_UNITARY;
        o.num_qubits = k;
        std::copy(q, q + k, o.qubits);
        keep.emplace_back(2 * m.size());
        std::memcpy(keep.back().data(), m.data(), m.size() * sizeof(mb2::Cd));
        out.push_back(o);
    };
    auto flush = [&]() -> int {
        if (out.empty()) return MB2_OK;
        for (size_t i = 0; i < out.size(); ++i) out[i].matrix = keep[i].data();
        mb2_sweep_options o{0, 0, 0, 0, 0, 0};
        const int rc = mb2_apply_program(rho, out.data(), static_cast<uint32_t>(out.size()), &o);
        out.clear();
        keep.clear();
        return rc;
    };
    try {
        for (uint32_t i = 0; i < num_ops; ++i) {
            const mb2_op& op = ops[i];
            if (op.opcode == MB2_MEASURE) continue;
            const uint32_t k = op.num_qubits;
            const bool channel = op.opcode == MB2_CHANNEL;
            if (k == 0 || k > (channel ? 5u : static_cast<uint32_t>(MB2_MAX_OP_QUBITS)))
                return fail(rho->ctx, MB2_ERR_INVALID, "operation " + std::to_string(i) + ": operand count");
            uint32_t both[10];
            uint64_t seen = 0;
            for (uint32_t j = 0; j < k; ++j) {
                if (op.qubits[j] >= n) return fail(rho->ctx, MB2_ERR_INVALID, "operand out of range");
                if (seen >> op.qubits[j] & 1u) return fail(rho->ctx, MB2_ERR_INVALID, "repeated operand");
                seen |= uint64_t{1} << op.qubits[j];
                both[j] = op.qubits[j];
                both[k + j] = op.qubits[j] + n;
            }
            const uint32_t dim = 1u << k;
            if (channel) {
                if (op.matrix == nullptr || op.reserved == 0)
                    return fail(rho->ctx, MB2_ERR_INVALID, "operation " + std::to_string(i) + ": channel without Kraus operators");
                std::vector<std::vector<mb2::Cd>> kraus(op.reserved, std::vector<mb2::Cd>(size_t{dim} * dim));
                for (uint32_t t = 0; t < op.reserved; ++t)
                    for (size_t e = 0; e < size_t{dim} * dim; ++e) {
                        const double* z = op.matrix + 2 * (size_t{t} * dim * dim + e);
                        kraus[t][e] = mb2::Cd{z[0], z[1]};
                    }
                const std::vector<mb2::Cd> sop = superoperator(kraus, k);
                if (2 * k <= MB2_MAX_OP_QUBITS) {
                    block(sop, both, 2 * k);
                    continue;
                }
                if (int rc = flush(); rc != MB2_OK) return rc;
                const size_t sd = size_t{dim} * dim;
                std::vector<mb2::Cd> mt(sd * sd);
                for (size_t r = 0; r < sd; ++r)
                    for (size_t c = 0; c < sd; ++c) mt[c * sd + r] = sop[r * sd + c];
                if (int e = ensure_scratch(rho, mt.size() * sizeof(mb2::Cd)); e != MB2_OK) return e;
                MB2_CUDA(rho->ctx, cudaMemcpyAsync(rho->scratch, mt.data(), mt.size() * sizeof(mb2::Cd),
                                                   cudaMemcpyHostToDevice, rho->stream));
                const int rc = mb2::launch_apply_wide(rho->amps, 2 * n, both, 2 * k,
                                                      static_cast<const double*>(rho->scratch), rho->stream);
                if (rc != MB2_OK) return fail(rho->ctx, rc, std::string("wide apply: ") + mb2::last_cuda_error_string());
                // The host copy of the matrix must outlive the transfer.
                MB2_CUDA(rho->ctx, cudaStreamSynchronize(rho->stream));
                continue;
            }
            std::vector<mb2::Cd> m;
            if (op.opcode == MB2_UNITARY) {
                if (op.matrix == nullptr) return fail(rho->ctx, MB2_ERR_INVALID, "unitary without a matrix");
                m.resize(size_t{dim} * dim);
                for (size_t e = 0; e < m.size(); ++e) m[e] = mb2::Cd{op.matrix[2 * e], op.matrix[2 * e + 1]};
            } else if (mb2::gate_matrix(op.opcode, op.params, m) != static_cast<int>(dim)) {
                return fail(rho->ctx, MB2_ERR_INVALID, "operation " + std::to_string(i) + ": unknown gate");
            }
            std::vector<mb2::Cd> mc(m.size());
            for (size_t e = 0; e < m.size(); ++e) mc[e] = std::conj(m[e]);
            block(m, both, k);
            block(mc, both + k, k);
        }
    } catch (const std::exception& e) {
        return fail(rho->ctx, MB2_ERR_INVALID, e.what());
    }
    return flush();
}

int mb2_dm_expectation(mb2_state* rho, uint32_t n, const uint64_t* x_masks, const uint64_t* z_masks,
                       uint32_t num_terms, double* out) {
    if (int e = check_rho(rho, n); e != MB2_OK) return e;
    if (num_terms == 0) return MB2_OK;
    if (x_masks == nullptr || z_masks == nullptr || out == nullptr) return MB2_ERR_INVALID;
    const uint64_t lim = (uint64_t{1} << n) - 1;
    for (uint32_t t = 0; t < num_terms; ++t)
        if ((x_masks[t] | z_masks[t]) & ~lim) return fail(rho->ctx, MB2_ERR_INVALID, "Pauli mask beyond the qubits");
    auto up = [](size_t v) { return (v + 255) & ~size_t{255}; };
    const size_t mb = size_t{num_terms} * 8;
    const size_t off_z = up(mb), off_p = off_z + up(mb), off_o = off_p + size_t{num_terms} * mb2::kExpBlocks * 16;
    if (int e = ensure_scratch(rho, off_o + size_t{num_terms} * 16); e != MB2_OK) return e;
    auto* base = static_cast<unsigned char*>(rho->scratch);
    MB2_CUDA(rho->ctx, cudaMemcpyAsync(base, x_masks, mb, cudaMemcpyHostToDevice, rho->stream));
    MB2_CUDA(rho->ctx, cudaMemcpyAsync(base + off_z, z_masks, mb, cudaMemcpyHostToDevice, rho->stream));
    const int rc = mb2::launch_dm_trace(rho->amps, n, reinterpret_cast<const uint64_t*>(base),
                                        reinterpret_cast<const uint64_t*>(base + off_z), num_terms,
                                        reinterpret_cast<double*>(base + off_p), reinterpret_cast<double*>(base + off_o),
                                        rho->stream);
    if (rc != MB2_OK) return fail(rho->ctx, rc, std::string("trace launch: ") + mb2::last_cuda_error_string());
    MB2_CUDA(rho->ctx, cudaMemcpyAsync(out, base + off_o, size_t{num_terms} * 16, cudaMemcpyDeviceToHost, rho->stream));
    MB2_CUDA(rho->ctx, cudaStreamSynchronize(rho->stream));
    return MB2_OK;
}

int mb2_dm_sample(mb2_state* rho, uint32_t n, uint64_t shots, uint64_t seed, const uint32_t* targets,
                  uint32_t num_targets, uint64_t* outcomes, uint64_t* counts, uint64_t* num_outcomes) {
    if (int e = check_rho(rho, n); e != MB2_OK) return e;
    if (num_outcomes == nullptr) return MB2_ERR_INVALID;
    for (uint32_t t = 0; t < num_targets; ++t)
        if (targets[2 * t] >= n || targets[2 * t + 1] >= 64)
            return fail(rho->ctx, MB2_ERR_INVALID, "measure target out of range");
    if (shots == 0) {
        *num_outcomes = 0;
        return MB2_OK;
    }
    const std::vector<double> u = sorted_uniforms(shots, seed);
    const size_t al_u = (shots * 8 + 255) & ~size_t{255};
    if (int e = ensure_scratch(rho, 2 * al_u); e != MB2_OK) return e;
    auto* base = static_cast<unsigned char*>(rho->scratch);
    MB2_CUDA(rho->ctx, cudaMemcpyAsync(base, u.data(), shots * 8, cudaMemcpyHostToDevice, rho->stream));
    const int rc = mb2::launch_dm_walk(rho->amps, n, reinterpret_cast<const double*>(base), shots,
                                       reinterpret_cast<uint64_t*>(base + al_u), rho->stream);
    if (rc != MB2_OK) return fail(rho->ctx, rc, std::string("walk launch: ") + mb2::last_cuda_error_string());
    std::vector<uint64_t> basis(shots);
    MB2_CUDA(rho->ctx, cudaMemcpyAsync(basis.data(), base + al_u, shots * 8, cudaMemcpyDeviceToHost, rho->stream));
    MB2_CUDA(rho->ctx, cudaStreamSynchronize(rho->stream));
    return histogram(rho->ctx, n, basis, targets, num_targets, outcomes, counts, num_outcomes);
}

int mb2_norm_exact(mb2_state* s, double* out) {
    if (s == nullptr || out == nullptr) return MB2_ERR_INVALID;
    if (int e = ensure_scratch(s, mb2::sample_scratch_bytes(s->n, 0)); e != MB2_OK) return e;
    const int rc = mb2::launch_exact_norm(s->amps, s->n, s->scratch, out, s->stream, s->precision);
    if (rc != MB2_OK) return fail(s->ctx, rc, std::string("exact norm: ") + mb2::last_cuda_error_string());
    return MB2_OK;
}

// ---- trajectories ----------------------------------------------------------
// The reference's trajectory engine (src/engines/trajectory/
// trajectory_engine.cpp:205-241,424-494) on the device.

}  // extern "C"

namespace {

// SplitMix64 output t + 1 of the stream seeded with base_seed: the
// trajectory's seed (trajectory_engine.cpp:319-323, src/common/splitmix64.h).
uint64_t trajectory_seed(uint64_t base_seed, uint64_t t) {
    uint64_t z = base_seed + t * 0x9E3779B97F4A7C15ULL + 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

double word_to_uniform(uint64_t w) { return static_cast<double>(w >> 11) * 0x1.0p-53; }

// A measure target's readout error (the reference's ReadoutTarget,
// src/engines/noise/readout.h): its clbit and P(recorded r | true t) at 2t + r.
struct Readout {
    uint32_t clbit;
    double a[4];
};

// readout_targets (src/engines/noise/readout.cpp): per measure target, in
// target order, the readout error of the last MB2_MEASURE writing its clbit,
// when that measurement has one.
std::vector<Readout> readout_targets(const mb2_op* ops, uint32_t num_ops, const uint32_t* targets,
                                     uint32_t num_targets) {
    std::vector<Readout> out;
    for (uint32_t t = 0; t < num_targets; ++t) {
        const uint32_t clbit = targets[2 * t + 1];
        const double* err = nullptr;
        for (uint32_t i = 0; i < num_ops; ++i)
            if (ops[i].opcode == MB2_MEASURE && ops[i].clbit == clbit) err = ops[i].matrix;
        if (err != nullptr) out.push_back(Readout{clbit, {err[0], err[1], err[2], err[3]}});
    }
    return out;
}

bool readouts_valid(const std::vector<Readout>& rs) {
    for (const Readout& r : rs)
        for (double v : r.a)
            if (!(v >= 0.0 && v <= 1.0)) return false;
    return true;
}

// apply_readout: one uniform per readout-errored target, in order; the bit
// flips when the uniform is below P(recorded != true | true).
void apply_readout(uint64_t& outcome, const std::vector<Readout>& rs, std::mt19937_64& rng) {
    for (const Readout& r : rs) {
        const bool truth = ((outcome >> r.clbit) & 1u) != 0;
        const double flip = truth ? r.a[2] : r.a[1];
        if (word_to_uniform(rng()) < flip) outcome ^= uint64_t{1} << r.clbit;
    }
}

// The outcome word of a basis index: bit clbit set when the target's qubit is.
uint64_t outcome_word(uint64_t basis, const uint32_t* targets, uint32_t num_targets) {
    uint64_t o = 0;
    for (uint32_t t = 0; t < num_targets; ++t)
        if ((basis >> targets[2 * t]) & 1u) o |= uint64_t{1} << targets[2 * t + 1];
    return o;
}

// Ascending distinct outcomes with their counts.
int histogram_words(mb2_context* ctx, std::vector<uint64_t> words, uint64_t* outcomes, uint64_t* counts,
                    uint64_t* num_outcomes) {
    std::sort(words.begin(), words.end());
    uint64_t d = 0;
    for (size_t i = 0; i < words.size();) {
        size_t j = i + 1;
        while (j < words.size() && words[j] == words[i]) ++j;
        if (d >= *num_outcomes) return fail(ctx, MB2_ERR_INVALID, "outcome capacity too small");
        outcomes[d] = words[i];
        counts[d] = j - i;
        ++d;
        i = j;
    }
    *num_outcomes = d;
    return MB2_OK;
}

struct TrajChannel {
    std::vector<uint32_t> qubits;
    std::vector<std::vector<mb2::Cd>> kraus;     // each dim x dim, row-major
    std::vector<std::vector<mb2::Cd>> products;  // K^dagger K, as the reference forms them
    std::vector<uint64_t> xs, zs;                // the 4^k Pauli strings on the channel's qubits
};

// K^dagger K (kraus_products, trajectory_engine.cpp:50-69).
std::vector<mb2::Cd> kraus_product(const std::vector<mb2::Cd>& k, size_t dim) {
    std::vector<mb2::Cd> m(dim * dim, mb2::Cd{0.0, 0.0});
    for (size_t a = 0; a < dim; ++a)
        for (size_t b = 0; b < dim; ++b) {
            mb2::Cd sum{0.0, 0.0};
            for (size_t r = 0; r < dim; ++r) sum += std::conj(k[r * dim + a]) * k[r * dim + b];
            m[a * dim + b] = sum;
        }
    return m;
}

}  // namespace

extern "C" {

int mb2_trajectories(mb2_context* ctx, uint32_t n, const mb2_op* ops, uint32_t num_ops, uint64_t trajectories,
                     uint64_t seed, const uint64_t* x_masks, const uint64_t* z_masks, const double* coefs,
                     uint32_t num_terms, double* term_means, double* standard_error, uint64_t shots,
                     const uint32_t* targets, uint32_t num_targets, uint64_t* outcomes, uint64_t* counts,
                     uint64_t* num_outcomes) {
    return mb2_trajectories_monitored(ctx, n, ops, num_ops, trajectories, seed, x_masks, z_masks, coefs, num_terms,
                                      term_means, standard_error, shots, targets, num_targets, outcomes, counts,
                                      num_outcomes, nullptr, nullptr);
}

int mb2_trajectories_monitored(mb2_context* ctx, uint32_t n, const mb2_op* ops, uint32_t num_ops,
                               uint64_t trajectories, uint64_t seed, const uint64_t* x_masks,
                               const uint64_t* z_masks, const double* coefs, uint32_t num_terms, double* term_means,
                               double* standard_error, uint64_t shots, const uint32_t* targets,
                               uint32_t num_targets, uint64_t* outcomes, uint64_t* counts, uint64_t* num_outcomes,
                               mb2_boundary_fn boundary, void* user) {
    if (ctx == nullptr || n < 1 || n > 34 || (ops == nullptr && num_ops != 0) || trajectories == 0)
        return MB2_ERR_INVALID;
    const bool want_exp = num_terms != 0;
    const bool want_counts = shots != 0;
    if (want_exp && (x_masks == nullptr || z_masks == nullptr || coefs == nullptr || term_means == nullptr))
        return MB2_ERR_INVALID;
    if (want_exp && trajectories < 2) return fail(ctx, MB2_ERR_INVALID, "an expectation needs at least 2 trajectories");
    if (want_counts && (shots > trajectories || num_outcomes == nullptr || outcomes == nullptr || counts == nullptr))
        return fail(ctx, MB2_ERR_INVALID, "more shots than trajectories");
    for (uint32_t t = 0; t < num_targets; ++t)
        if (targets[2 * t] >= n || targets[2 * t + 1] >= 64) return fail(ctx, MB2_ERR_INVALID, "measure target out of range");
    // Segments: runs of gates (applied op by op, as the reference's
    // apply_matrix per operation) and channels.
    std::vector<std::vector<mb2_op>> gate_runs;
    std::vector<TrajChannel> channels;
    std::vector<std::pair<int, size_t>> steps;  // (0: gate run, 1: channel), index
    std::vector<uint64_t> step_end;             // operations done once the step is (measurements included)
    try {
        for (uint32_t i = 0; i < num_ops; ++i) {
            const mb2_op& op = ops[i];
            if (op.opcode == MB2_MEASURE) continue;
            if (op.opcode != MB2_CHANNEL) {
                if (steps.empty() || steps.back().first != 0) {
                    steps.emplace_back(0, gate_runs.size());
                    step_end.push_back(0);
                    gate_runs.emplace_back();
                }
                gate_runs.back().push_back(op);
                step_end.back() = i + 1;
                continue;
            }
            const uint32_t k = op.num_qubits;
            if (k == 0 || k > 3 || op.matrix == nullptr || op.reserved == 0)
                return fail(ctx, MB2_ERR_INVALID, "operation " + std::to_string(i) + ": channel of 1..3 qubits with Kraus operators");
            const size_t dim = size_t{1} << k;
            TrajChannel ch;
            ch.qubits.assign(op.qubits, op.qubits + k);
            for (uint32_t q : ch.qubits)
                if (q >= n) return fail(ctx, MB2_ERR_INVALID, "operand out of range");
            for (uint32_t t = 0; t < op.reserved; ++t) {
                std::vector<mb2::Cd> km(dim * dim);
                for (size_t e = 0; e < dim * dim; ++e)
                    km[e] = mb2::Cd{op.matrix[2 * (t * dim * dim + e)], op.matrix[2 * (t * dim * dim + e) + 1]};
                ch.products.push_back(kraus_product(km, dim));
                ch.kraus.push_back(std::move(km));
            }
            for (uint64_t lx = 0; lx < dim; ++lx)
                for (uint64_t lz = 0; lz < dim; ++lz) {
                    uint64_t gx = 0, gz = 0;
                    for (uint32_t j = 0; j < k; ++j) {
                        if ((lx >> j) & 1u) gx |= uint64_t{1} << ch.qubits[j];
                        if ((lz >> j) & 1u) gz |= uint64_t{1} << ch.qubits[j];
                    }
                    ch.xs.push_back(gx);
                    ch.zs.push_back(gz);
                }
            steps.emplace_back(1, channels.size());
            step_end.push_back(i + 1);
            channels.push_back(std::move(ch));
        }
    } catch (const std::exception& e) {
        return fail(ctx, MB2_ERR_INVALID, e.what());
    }
    const std::vector<Readout> readouts =
        want_counts ? readout_targets(ops, num_ops, targets, num_targets) : std::vector<Readout>{};
    if (!readouts_valid(readouts)) return fail(ctx, MB2_ERR_INVALID, "readout error entries must lie in [0, 1]");
    mb2_state* st = nullptr;
    if (int e = mb2_state_alloc(ctx, n, MB2_C128, ~uint64_t{0}, &st); e != MB2_OK) return e;
    struct Free {
        mb2_state* s;
        ~Free() { mb2_state_free(s); }
    } guard{st};
    const mb2_sweep_options one_by_one{0, 0, 0, 0, 0, 0};
    std::vector<mb2::Cd> term_sums(num_terms, mb2::Cd{0.0, 0.0});
    std::vector<double> vals(2 * std::max<uint32_t>(num_terms, 1));
    uint64_t count = 0;  // Welford (trajectory_engine.cpp:244-265)
    mb2::Cd mean{0.0, 0.0};
    double ssd = 0.0;
    std::vector<uint64_t> shot_words;
    // The reference's safe boundaries (trajectory_engine.cpp:171-181,216,
    // 473): one after every operation of every trajectory and one after each
    // trajectory's outputs, counted across trajectories; the monitor is asked
    // at the end of each step here, with the count the reference has there.
    const uint64_t per_trajectory = uint64_t{num_ops} + 1;
    auto cross = [&](uint64_t crossed) {
        return boundary == nullptr || boundary(user, crossed) == 0;
    };
    for (uint64_t t = 0; t < trajectories; ++t) {
        std::mt19937_64 rng(trajectory_seed(seed, t));
        if (int e = mb2_init(st, 0.0); e != MB2_OK) return e;  // |0..0>, no global phase
        for (size_t si = 0; si < steps.size(); ++si) {
            if (si > 0 && !cross(t * per_trajectory + step_end[si - 1]))
                return fail(ctx, MB2_ERR_ABANDONED, "abandoned at a safe boundary");
            const auto& [kind, idx] = steps[si];
            if (kind == 0) {
                const std::vector<mb2_op>& run = gate_runs[idx];
                if (int e = mb2_apply_program(st, run.data(), static_cast<uint32_t>(run.size()), &one_by_one); e != MB2_OK)
                    return e;
                continue;
            }
            const TrajChannel& ch = channels[idx];
            const uint32_t k = static_cast<uint32_t>(ch.qubits.size());
            const size_t dim = size_t{1} << k;
            // rho_q from its Pauli expectations: rho = 2^-k sum_P <P> P,
            // P = i^{|x&z|} X^x Z^z in the channel's local basis.
            std::vector<double> pv(2 * ch.xs.size());
            if (int e = mb2_expectation(st, ch.xs.data(), ch.zs.data(), static_cast<uint32_t>(ch.xs.size()), pv.data());
                e != MB2_OK)
                return e;
            std::vector<mb2::Cd> rho(dim * dim, mb2::Cd{0.0, 0.0});
            const mb2::Cd ipow[4] = {{1.0, 0.0}, {0.0, 1.0}, {-1.0, 0.0}, {0.0, -1.0}};
            size_t pi = 0;
            for (uint64_t lx = 0; lx < dim; ++lx)
                for (uint64_t lz = 0; lz < dim; ++lz, ++pi) {
                    const mb2::Cd v{pv[2 * pi], pv[2 * pi + 1]};
                    const mb2::Cd ph = ipow[std::popcount(lx & lz) & 3];
                    for (uint64_t c = 0; c < dim; ++c) {
                        const double sgn = (std::popcount(c & lz) & 1) ? -1.0 : 1.0;
                        rho[(c ^ lx) * dim + c] += v * ph * sgn;
                    }
                }
            for (mb2::Cd& r : rho) r /= static_cast<double>(dim);
            // The branch: the first with cumulative p_i = Re Tr(M_i rho) above
            // u, else the last with p_i > 0 (choose_branch, :123-152).
            const double u = word_to_uniform(rng());
            double cumulative = 0.0;
            int64_t branch = -1, last_positive = -1;
            for (size_t b = 0; b < ch.products.size() && branch < 0; ++b) {
                double p = 0.0;
                for (size_t a = 0; a < dim; ++a)
                    for (size_t c = 0; c < dim; ++c) p += (ch.products[b][a * dim + c] * rho[c * dim + a]).real();
                if (p > 0.0) {
                    last_positive = static_cast<int64_t>(b);
                    cumulative += p;
                    if (u < cumulative) branch = static_cast<int64_t>(b);
                }
            }
            if (branch < 0) branch = last_positive;
            if (branch < 0) return fail(ctx, MB2_ERR_INVALID, "every Kraus branch has probability 0");
            const std::vector<mb2::Cd>& km = ch.kraus[static_cast<size_t>(branch)];
            if (int e = mb2_apply_matrix(st, reinterpret_cast<const double*>(km.data()), ch.qubits.data(), k); e != MB2_OK)
                return e;
            // psi /= ||psi|| with the reference's sequential norm (renormalize, :155-166).
            double norm_sq = 0.0;
            if (int e = mb2_norm_exact(st, &norm_sq); e != MB2_OK) return e;
            if (!(norm_sq > 0.0)) return fail(ctx, MB2_ERR_INVALID, "a chosen Kraus branch annihilated the state");
            const double scale = 1.0 / std::sqrt(norm_sq);
            const double sm[8] = {scale, 0.0, 0.0, 0.0, 0.0, 0.0, scale, 0.0};
            const uint32_t q0 = 0;
            if (int e = mb2_apply_matrix(st, sm, &q0, 1); e != MB2_OK) return e;
        }
        if (want_exp) {
            if (int e = mb2_expectation(st, x_masks, z_masks, num_terms, vals.data()); e != MB2_OK) return e;
            mb2::Cd x{0.0, 0.0};
            for (uint32_t i = 0; i < num_terms; ++i) {
                const mb2::Cd v{vals[2 * i], vals[2 * i + 1]};
                term_sums[i] += v;
                x += mb2::Cd{coefs[2 * i], coefs[2 * i + 1]} * v;
            }
            ++count;
            const mb2::Cd delta = x - mean;
            mean += delta / static_cast<double>(count);
            ssd += (std::conj(delta) * (x - mean)).real();
        }
        if (want_counts && t < shots) {
            // One word for the shot, then one per readout-errored target
            // (trajectory_engine.cpp:465-471).
            const double u = word_to_uniform(rng());
            uint64_t b = 0;
            if (int e = mb2_sample_basis(st, &u, 1, &b); e != MB2_OK) return e;
            uint64_t o = outcome_word(b, targets, num_targets);
            apply_readout(o, readouts, rng);
            shot_words.push_back(o);
        }
        if ((!steps.empty() && !cross(t * per_trajectory + num_ops)) || !cross((t + 1) * per_trajectory))
            return fail(ctx, MB2_ERR_ABANDONED, "abandoned at a safe boundary");
    }
    if (want_exp) {
        for (uint32_t i = 0; i < num_terms; ++i) {
            term_sums[i] /= static_cast<double>(trajectories);
            term_means[2 * i] = term_sums[i].real();
            term_means[2 * i + 1] = term_sums[i].imag();
        }
        if (standard_error != nullptr) {
            const double cnt = static_cast<double>(count);
            *standard_error = std::sqrt(ssd / (cnt - 1.0) / cnt);
        }
    }
    if (want_counts) return histogram_words(ctx, std::move(shot_words), outcomes, counts, num_outcomes);
    return MB2_OK;
}

int mb2_dm_sample_basis(mb2_state* rho, uint32_t n, const double* uniforms, uint64_t count, uint64_t* basis) {
    if (int e = check_rho(rho, n); e != MB2_OK) return e;
    if (count == 0) return MB2_OK;
    if (uniforms == nullptr || basis == nullptr) return MB2_ERR_INVALID;
    std::vector<std::pair<double, uint64_t>> draw(count);
    for (uint64_t i = 0; i < count; ++i) {
        if (!(uniforms[i] >= 0.0 && uniforms[i] < 1.0)) return fail(rho->ctx, MB2_ERR_INVALID, "a uniform outside [0, 1)");
        draw[i] = {uniforms[i], i};
    }
    std::sort(draw.begin(), draw.end());
    std::vector<double> u(count);
    for (uint64_t i = 0; i < count; ++i) u[i] = draw[i].first;
    const size_t al_u = (count * 8 + 255) & ~size_t{255};
    if (int e = ensure_scratch(rho, 2 * al_u); e != MB2_OK) return e;
    auto* base = static_cast<unsigned char*>(rho->scratch);
    MB2_CUDA(rho->ctx, cudaMemcpyAsync(base, u.data(), count * 8, cudaMemcpyHostToDevice, rho->stream));
    const int rc = mb2::launch_dm_walk(rho->amps, n, reinterpret_cast<const double*>(base), count,
                                       reinterpret_cast<uint64_t*>(base + al_u), rho->stream);
    if (rc != MB2_OK) return fail(rho->ctx, rc, std::string("walk launch: ") + mb2::last_cuda_error_string());
    std::vector<uint64_t> sorted(count);
    MB2_CUDA(rho->ctx, cudaMemcpyAsync(sorted.data(), base + al_u, count * 8, cudaMemcpyDeviceToHost, rho->stream));
    MB2_CUDA(rho->ctx, cudaStreamSynchronize(rho->stream));
    for (uint64_t i = 0; i < count; ++i) basis[draw[i].second] = sorted[i];
    return MB2_OK;
}

int mb2_dm_sample_readout(mb2_state* rho, uint32_t n, const mb2_op* ops, uint32_t num_ops, uint64_t shots,
                          uint64_t seed, const uint32_t* targets, uint32_t num_targets, uint64_t* outcomes,
                          uint64_t* counts, uint64_t* num_outcomes) {
    if (int e = check_rho(rho, n); e != MB2_OK) return e;
    if (num_outcomes == nullptr || (ops == nullptr && num_ops != 0) || (targets == nullptr && num_targets != 0))
        return MB2_ERR_INVALID;
    for (uint32_t t = 0; t < num_targets; ++t)
        if (targets[2 * t] >= n || targets[2 * t + 1] >= 64)
            return fail(rho->ctx, MB2_ERR_INVALID, "measure target out of range");
    const std::vector<Readout> rs = readout_targets(ops, num_ops, targets, num_targets);
    if (rs.empty()) return mb2_dm_sample(rho, n, shots, seed, targets, num_targets, outcomes, counts, num_outcomes);
    if (!readouts_valid(rs)) return fail(rho->ctx, MB2_ERR_INVALID, "readout error entries must lie in [0, 1]");
    if (shots == 0) {
        *num_outcomes = 0;
        return MB2_OK;
    }
    if (outcomes == nullptr || counts == nullptr) return MB2_ERR_INVALID;
    // Per shot, from one generator: the outcome's word, then one word per
    // readout-errored target (density_matrix_engine.cpp:378-390).
    const size_t R = rs.size();
    std::mt19937_64 rng(seed);
    std::vector<std::pair<double, uint64_t>> draw(shots);  // (uniform, shot)
    std::vector<uint64_t> flip_words(shots * R);
    for (uint64_t i = 0; i < shots; ++i) {
        draw[i] = {word_to_uniform(rng()), i};
        for (size_t r = 0; r < R; ++r) flip_words[i * R + r] = rng();
    }
    // Each shot's basis state is the first whose sequential cumulative
    // probability exceeds its uniform (CumulativeDistribution::sample_one):
    // the device walk takes the uniforms sorted.
    std::sort(draw.begin(), draw.end());
    std::vector<double> u(shots);
    for (uint64_t i = 0; i < shots; ++i) u[i] = draw[i].first;
    const size_t al_u = (shots * 8 + 255) & ~size_t{255};
    if (int e = ensure_scratch(rho, 2 * al_u); e != MB2_OK) return e;
    auto* base = static_cast<unsigned char*>(rho->scratch);
    MB2_CUDA(rho->ctx, cudaMemcpyAsync(base, u.data(), shots * 8, cudaMemcpyHostToDevice, rho->stream));
    const int rc = mb2::launch_dm_walk(rho->amps, n, reinterpret_cast<const double*>(base), shots,
                                       reinterpret_cast<uint64_t*>(base + al_u), rho->stream);
    if (rc != MB2_OK) return fail(rho->ctx, rc, std::string("walk launch: ") + mb2::last_cuda_error_string());
    std::vector<uint64_t> basis(shots);
    MB2_CUDA(rho->ctx, cudaMemcpyAsync(basis.data(), base + al_u, shots * 8, cudaMemcpyDeviceToHost, rho->stream));
    MB2_CUDA(rho->ctx, cudaStreamSynchronize(rho->stream));
    std::vector<uint64_t> words(shots);
    for (uint64_t i = 0; i < shots; ++i) {
        const uint64_t shot = draw[i].second;
        uint64_t o = outcome_word(basis[i], targets, num_targets);
        for (size_t r = 0; r < R; ++r) {
            const bool truth = ((o >> rs[r].clbit) & 1u) != 0;
            if (word_to_uniform(flip_words[shot * R + r]) < (truth ? rs[r].a[2] : rs[r].a[1]))
                o ^= uint64_t{1} << rs[r].clbit;
        }
        words[i] = o;
    }
    return histogram_words(rho->ctx, std::move(words), outcomes, counts, num_outcomes);
}

int mb2_copy_out(mb2_state* s, void* host, uint64_t num_amplitudes) {
    if (s == nullptr || host == nullptr) return MB2_ERR_INVALID;
    if (num_amplitudes > (uint64_t{1} << s->n)) return fail(s->ctx, MB2_ERR_INVALID, "copy beyond the state");
    MB2_CUDA(s->ctx, cudaMemcpyAsync(host, s->amps, num_amplitudes * amp_bytes(s->precision),
                                     s->host_amps != nullptr ? cudaMemcpyDefault : cudaMemcpyDeviceToHost,
                                     s->stream));
    MB2_CUDA(s->ctx, cudaStreamSynchronize(s->stream));
    return MB2_OK;
}

int mb2_copy_in(mb2_state* s, const void* host, uint64_t num_amplitudes) {
    if (s == nullptr || host == nullptr) return MB2_ERR_INVALID;
    if (num_amplitudes > (uint64_t{1} << s->n)) return fail(s->ctx, MB2_ERR_INVALID, "copy beyond the state");
    MB2_CUDA(s->ctx, cudaMemcpyAsync(s->amps, host, num_amplitudes * amp_bytes(s->precision),
                                     s->host_amps != nullptr ? cudaMemcpyDefault : cudaMemcpyHostToDevice,
                                     s->stream));
    MB2_CUDA(s->ctx, cudaStreamSynchronize(s->stream));
    return MB2_OK;
}

int mb2_synchronize(mb2_state* s) {
    if (s == nullptr) return MB2_ERR_INVALID;
    MB2_CUDA(s->ctx, cudaStreamSynchronize(s->stream));
    return MB2_OK;
}

int mb2_debug_run_plan(const mb2_op* ops, uint32_t num_ops, const mb2_sweep_options* opts, uint32_t num_qubits,
                       int32_t precision, double* state, uint64_t* stats) {
    if ((ops == nullptr && num_ops != 0) || num_qubits < 1 || num_qubits > 40 || (state != nullptr && num_qubits > 28) ||
        (precision != MB2_C128 && precision != MB2_C64))
        return MB2_ERR_INVALID;
    mb2_sweep_options o{1, 0, 0, 0, 0, 0};
    if (opts != nullptr) o = *opts;
    try {
        const std::vector<mb2::Block> blocks = mb2::build_blocks(ops, num_ops, o.fuse_gates != 0, static_cast<uint32_t>(o.fusion_width));
        if (blocks.empty()) return MB2_OK;
        const bool c64 = precision == MB2_C64;
        uint32_t m = tile_width(o.tile_qubits > 0 ? static_cast<uint32_t>(o.tile_qubits) : 0, num_qubits, blocks);
        bool tc = false;
        if (c64) {
            if (num_qubits < mb2::kMinTileQubits) return MB2_ERR_UNSUPPORTED;
            const C64Choice ch = c64_choice(o, num_qubits, mb2::kDefaultTileQubitsC64, blocks);
            m = ch.m;
            tc = ch.tc;
        }
        m = std::min(std::max(m, mb2::kMinTileQubits), num_qubits);
        const uint32_t low = o.low_qubits < 0 ? 0u : (o.low_qubits == 0 ? mb2::kDefaultFixedLow
                                                                         : static_cast<uint32_t>(o.low_qubits));
        mb2::TileProgram prog = mb2::plan_tile_program(blocks, num_qubits, m, low, nullptr, c64);
        if (tc) mb2::make_tensor_core_program(prog, blocks, mb2::tc_max_phases(m));
        if (state != nullptr) mb2::run_program_on_host(prog, num_qubits, reinterpret_cast<mb2::Cd*>(state));
        if (stats != nullptr) {
            uint64_t tcp = 0, smem = 0, layouts = 0;
            for (const mb2::TilePass& p : prog.passes) {
                if (!p.tc) continue;
                tcp += 1;
                for (uint32_t i = 0; i < p.prog_count; ++i) layouts += prog.instrs[p.prog_begin + i].op == mb2::TOP_PHASE;
                smem = std::max<uint64_t>(smem, 2 * (8ull << p.m) + uint64_t{p.tc_phases} * mb2::kTcOperandWords * 4 +
                                                    4ull * p.word_count + 4ull * p.sdata_count);
            }
            stats[0] = prog.passes.size();
            stats[1] = tcp;
            stats[2] = prog.tcmatrices.size() / 256;
            stats[3] = m;
            stats[4] = smem;
            stats[5] = layouts;
        }
    } catch (const std::exception&) {
        return MB2_ERR_INVALID;
    }
    return MB2_OK;
}

int mb2_debug_tc_probe(mb2_context* ctx, const float* rows, const double* matrix, float* out) {
    if (ctx == nullptr || rows == nullptr || matrix == nullptr || out == nullptr) return MB2_ERR_INVALID;
    MB2_CUDA(ctx, cudaSetDevice(ctx->device));
    std::vector<uint32_t> b(mb2::kTcOperandWords);
    mb2::tc_operands(reinterpret_cast<const mb2::Cd*>(matrix), b.data());
    constexpr size_t kRowBytes = 256 * 32 * sizeof(float);
    const size_t bytes = 2 * kRowBytes + b.size() * sizeof(uint32_t) + 256;
    cudaStream_t stream = nullptr;
    MB2_CUDA(ctx, cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    unsigned char* dev = nullptr;
    cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(&dev), bytes, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(dev, 0, bytes, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dev, rows, kRowBytes, cudaMemcpyHostToDevice, stream);
    auto* dev_b = reinterpret_cast<uint32_t*>(dev + 2 * kRowBytes);
    int* dev_err = reinterpret_cast<int*>(dev + 2 * kRowBytes + b.size() * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMemcpyAsync(dev_b, b.data(), b.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, stream);
    int rc = MB2_OK;
    if (e == cudaSuccess) {
        rc = mb2::launch_tc_probe(reinterpret_cast<const float*>(dev), dev_b, reinterpret_cast<float*>(dev + kRowBytes),
                                  dev_err, stream);
        if (rc != MB2_OK) rc = fail(ctx, rc, std::string("tc probe launch: ") + mb2::last_cuda_error_string());
    }
    int err = 0;
    if (e == cudaSuccess && rc == MB2_OK) e = cudaMemcpyAsync(out, dev + kRowBytes, kRowBytes, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess && rc == MB2_OK) e = cudaMemcpyAsync(&err, dev_err, sizeof(int), cudaMemcpyDeviceToHost, stream);
    if (dev != nullptr) cudaFreeAsync(dev, stream);
    const cudaError_t se = cudaStreamSynchronize(stream);
    cudaStreamDestroy(stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "tc probe");
    if (se != cudaSuccess) return cuda_fail(ctx, se, "tc probe");
    if (rc != MB2_OK) return rc;
    if (err != 0) return fail(ctx, MB2_ERR_CUDA, "tc probe: a bounded wait ran out");
    return MB2_OK;
}

int mb2_debug_schedule(const mb2_op* ops, uint32_t num_ops, const mb2_sweep_options* opts, uint32_t num_qubits,
                       uint32_t* pass, uint32_t* k, uint32_t* qubits, double* matrices, uint64_t* num_blocks,
                       uint64_t* matrix_len, int32_t precision) {
    if (num_blocks == nullptr || matrix_len == nullptr || (ops == nullptr && num_ops != 0)) return MB2_ERR_INVALID;
    if (precision != MB2_C128 && precision != MB2_C64) return MB2_ERR_INVALID;
    const bool c64 = precision == MB2_C64;
    if (num_qubits < 1 || num_qubits > 40) return MB2_ERR_INVALID;
    mb2_sweep_options o{1, 0, 0, 0, 0, 0};
    if (opts != nullptr) o = *opts;
    std::vector<mb2::Block> blocks;
    std::vector<uint32_t> order, order_pass;
    try {
        blocks = mb2::build_blocks(ops, num_ops, o.fuse_gates != 0, static_cast<uint32_t>(o.fusion_width));
        uint32_t m = tile_width(o.tile_qubits > 0 ? static_cast<uint32_t>(o.tile_qubits) : 0, num_qubits, blocks);
        if (c64) {
            m = o.tile_qubits > 0 ? std::min<uint32_t>(static_cast<uint32_t>(o.tile_qubits), mb2::kMaxTileQubitsC64)
                                  : std::min<uint32_t>(mb2::kDefaultTileQubitsC64, num_qubits);
            for (const mb2::Block& b : blocks) m = std::max(m, b.k);
            m = std::max(m, mb2::kMinTileQubits);
        }
        if ((!c64 && o.per_gate != 0) || num_qubits < mb2::kMinTileQubits || blocks.empty()) {
            for (uint32_t i = 0; i < blocks.size(); ++i) {
                order.push_back(i);
                order_pass.push_back(i);
            }
        } else {
            const uint32_t low = o.low_qubits < 0 ? 0u : (o.low_qubits == 0 ? mb2::kDefaultFixedLow
                                                                             : static_cast<uint32_t>(o.low_qubits));
            const mb2::TileProgram prog = mb2::plan_tile_program(blocks, num_qubits, m, low, nullptr, c64);
            order = prog.order;
            order_pass = prog.order_pass;
        }
    } catch (const std::exception&) {
        return MB2_ERR_INVALID;
    }
    if (order.size() > *num_blocks) return MB2_ERR_INVALID;
    uint64_t mlen = 0;
    for (size_t i = 0; i < order.size(); ++i) {
        const mb2::Block& b = blocks[order[i]];
        const uint64_t need = 2ull << (2 * b.k);
        if (mlen + need > *matrix_len) return MB2_ERR_INVALID;
        pass[i] = order_pass[i];
        k[i] = b.k;
        for (uint32_t j = 0; j < 6; ++j) qubits[6 * i + j] = j < b.k ? b.q[j] : 0;
        std::memcpy(matrices + mlen, b.m.data(), need * sizeof(double));
        mlen += need;
    }
    *num_blocks = order.size();
    *matrix_len = mlen;
    return MB2_OK;
}

// ---- autotuning -----------------------------------------------------------
namespace {

// Synthetic probe circuits (angles from a fixed LCG; their values do not
// change the work).
struct ProbeOps {
    std::vector<mb2_op> ops;
    uint64_t seed = 0x9E3779B97F4A7C15ull;
    double angle() {
        seed = seed * 6364136223846793005ull + 1442695040888963407ull;
        return static_cast<double>(seed >> 11) * (6.283185307179586 / 9007199254740992.0);
    }
    void gate(int32_t opcode, std::initializer_list<uint32_t> qs, int np) {
        mb2_op o{};
        o.opcode = opcode;
        o.num_qubits = static_cast<uint32_t>(qs.size());
        uint32_t i = 0;
        for (uint32_t q : qs) o.qubits[i++] = q;
        for (int p = 0; p < np; ++p) o.params[p] = angle();
        ops.push_back(o);
    }
};

std::vector<mb2_op> probe_brick(uint32_t n, uint32_t layers) {
    ProbeOps p;
    for (uint32_t l = 0; l < layers; ++l) {
        for (uint32_t q = 0; q < n; ++q) p.gate(MB2_U, {q}, 3);
        for (uint32_t q = l % 2; q + 1 < n; q += 2) p.gate(MB2_CZ, {q, q + 1}, 0);
    }
    return p.ops;
}

int time_sweep(mb2_state* st, const std::vector<mb2_op>& ops, uint32_t tile, double* ms, int32_t fuse = 1) {
    mb2_sweep_options o{fuse, 0, static_cast<int32_t>(tile), 0, 0, 0};
    if (int e = mb2_init(st, 0.0); e != MB2_OK) return e;
    if (int e = mb2_apply_program(st, ops.data(), static_cast<uint32_t>(ops.size()), &o); e != MB2_OK) return e;
    cudaEvent_t a = nullptr, b = nullptr;
    if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) return MB2_ERR_CUDA;
    double best = 1e30;
    int rc = MB2_OK;
    for (int rep = 0; rep < 3 && rc == MB2_OK; ++rep) {
        rc = mb2_init(st, 0.0);
        if (rc != MB2_OK) break;
        cudaEventRecord(a, st->stream);
        rc = mb2_apply_program(st, ops.data(), static_cast<uint32_t>(ops.size()), &o);
        cudaEventRecord(b, st->stream);
        if (cudaEventSynchronize(b) != cudaSuccess) rc = MB2_ERR_CUDA;
        float t = 0.f;
        cudaEventElapsedTime(&t, a, b);
        best = std::min(best, static_cast<double>(t));
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    *ms = best;
    return rc;
}

// The time model's costs at one precision and tile width.  A pass takes
//   fixed + amps * (memory + sum over its blocks of compute),
// the fixed cost from a pass over a 14-qubit state, memory from a
// near-empty pass at n qubits, compute from one pass each of many unfused
// blocks, less its memory time: a dense one-qubit block and a two-qubit
// diagonal block.
// The state whose pass times the per-pass fixed cost (launch, ramp, tail).
constexpr uint32_t kFixedCostQubits = 14;

int measure_costs(mb2_state* st, mb2_state* small, uint32_t m, double* fixed, double* pass, double* dense1,
                  double* diag) {
    const uint32_t n = st->n;
    ProbeOps e, es, u, d;
    e.gate(MB2_Z, {n - 1}, 0);
    es.gate(MB2_Z, {small->n - 1}, 0);
    for (int rep = 0; rep < 3; ++rep)
        for (uint32_t q = 0; q < m; ++q) u.gate(MB2_U, {q}, 3);
    for (int rep = 0; rep < 6; ++rep)
        for (uint32_t q = 0; q + 1 < m; ++q) d.gate(MB2_CP, {q, q + 1}, 1);
    double te = 0, tes = 0, tu = 0, td = 0;
    if (int rc = time_sweep(st, e.ops, m, &te); rc != MB2_OK) return rc;
    if (int rc = time_sweep(small, es.ops, m, &tes); rc != MB2_OK) return rc;
    if (int rc = time_sweep(st, u.ops, m, &tu, 0); rc != MB2_OK) return rc;
    if (int rc = time_sweep(st, d.ops, m, &td, 0); rc != MB2_OK) return rc;
    const double amps = static_cast<double>(uint64_t{1} << n);
    // The small state's pass is all fixed cost (its bytes take well under a
    // microsecond); te = f + A p.
    const double f = tes * 1e-3;
    *fixed = f;
    *pass = std::max(0.0, te * 1e-3 - f) / amps;
    // The probes' blocks each fit one pass: what they add to its memory time
    // is their compute, per amplitude and block.
    *dense1 = std::max(0.0, (tu * 1e-3 - f) / amps - *pass) / static_cast<double>(u.ops.size());
    *diag = std::max(0.0, (td * 1e-3 - f) / amps - *pass) / static_cast<double>(d.ops.size());
    return MB2_OK;
}

// Seconds for one pass of blocks [b0, b1) over 2^n amplitudes: the fixed
// cost, the memory time and the blocks' compute, added -- a pass with dense
// blocks is bound by FP64 latency at the resident warps, so its loads and
// stores overlap its arithmetic only in part (measured: a 28-qubit brick pass
// of 8 U3s takes about its DRAM time plus its FP64 time at the measured rate).
double pass_seconds(const mb2_tuning& t, bool c64, const std::vector<mb2::Block>& blocks, size_t b0, size_t b1,
                    uint32_t n) {
    const double mem = c64 ? t.pass_s_per_amp_c64 : t.pass_s_per_amp;
    const double dense1 = c64 ? t.dense1_s_per_amp_c64 : t.dense1_s_per_amp;
    const double diag = c64 ? t.diag_s_per_amp_c64 : t.diag_s_per_amp;
    double compute = 0.0;
    for (size_t i = b0; i < b1; ++i)  // a dense k-qubit block sums 2^k terms per amplitude
        compute += blocks[i].diagonal ? diag : dense1 * static_cast<double>(uint64_t{1} << (blocks[i].k - 1));
    return (c64 ? t.pass_s_fixed_c64 : t.pass_s_fixed) + (mem + compute) * static_cast<double>(uint64_t{1} << n);
}

}  // namespace

int mb2_autotune(mb2_context* ctx, uint32_t probe_qubits, mb2_tuning* out) {
    if (ctx == nullptr) return MB2_ERR_INVALID;
    const uint32_t n = probe_qubits == 0 ? 24u : probe_qubits;
    if (n < 16 || n > 30) return fail(ctx, MB2_ERR_INVALID, "probe_qubits must be 16..30");
    mb2_tuning t = ctx->tuning;
    const std::vector<mb2_op> brick = probe_brick(n, 8);
    for (int prec : {MB2_C128, MB2_C64}) {
        mb2_state* st = nullptr;
        mb2_state* small = nullptr;
        if (int rc = mb2_state_alloc(ctx, n, prec, ~uint64_t{0}, &st); rc != MB2_OK) return rc;
        if (int rc = mb2_state_alloc(ctx, kFixedCostQubits, prec, ~uint64_t{0}, &small); rc != MB2_OK) {
            mb2_state_free(st);
            return rc;
        }
        const std::vector<uint32_t> widths = prec == MB2_C128 ? std::vector<uint32_t>{10, 11, 12}
                                                              : std::vector<uint32_t>{12, 13};
        uint32_t best_m = widths[0];
        double best_ms = 1e30;
        int rc = MB2_OK;
        for (uint32_t m : widths) {
            double ms = 0;
            rc = time_sweep(st, brick, m, &ms);
            if (rc != MB2_OK) break;
            if (ms < best_ms) {
                best_ms = ms;
                best_m = m;
            }
        }
        if (rc == MB2_OK) {
            if (prec == MB2_C128) {
                t.tile_qubits = best_m;
                rc = measure_costs(st, small, best_m, &t.pass_s_fixed, &t.pass_s_per_amp, &t.dense1_s_per_amp,
                                   &t.diag_s_per_amp);
            } else {
                t.tile_qubits_c64 = best_m;
                rc = measure_costs(st, small, best_m, &t.pass_s_fixed_c64, &t.pass_s_per_amp_c64,
                                   &t.dense1_s_per_amp_c64, &t.diag_s_per_amp_c64);
            }
        }
        mb2_state_free(small);
        mb2_state_free(st);
        if (rc != MB2_OK) return rc;
    }
    t.probe_qubits = n;
    {
        std::lock_guard<std::mutex> lock(ctx->mu);
        ctx->tuning = t;
    }
    ctx->tile_c128.store(t.tile_qubits);
    ctx->tile_c64.store(t.tile_qubits_c64);
    if (out != nullptr) *out = t;
    return MB2_OK;
}

int mb2_context_tuning(mb2_context* ctx, mb2_tuning* out) {
    if (ctx == nullptr || out == nullptr) return MB2_ERR_INVALID;
    std::lock_guard<std::mutex> lock(ctx->mu);
    *out = ctx->tuning;
    return MB2_OK;
}

int mb2_estimate_sweep_time(mb2_context* ctx, const mb2_op* ops, uint32_t num_ops, const mb2_sweep_options* opts,
                            uint32_t num_qubits, int32_t precision, double* seconds) {
    if (ctx == nullptr || seconds == nullptr || (ops == nullptr && num_ops != 0) || num_qubits < 1 ||
        num_qubits > 40 || (precision != MB2_C128 && precision != MB2_C64))
        return MB2_ERR_INVALID;
    mb2_sweep_options o{1, 0, 0, 0, 0, 0};
    if (opts != nullptr) o = *opts;
    mb2_tuning t;
    {
        std::lock_guard<std::mutex> lock(ctx->mu);
        t = ctx->tuning;
    }
    const bool c64 = precision == MB2_C64;
    try {
        const std::vector<mb2::Block> blocks = mb2::build_blocks(ops, num_ops, o.fuse_gates != 0, static_cast<uint32_t>(o.fusion_width));
        double total = 0.0;
        if (o.per_gate != 0 || num_qubits < mb2::kMinTileQubits || blocks.empty()) {
            for (size_t i = 0; i < blocks.size(); ++i) total += pass_seconds(t, c64, blocks, i, i + 1, num_qubits);
        } else {
            const uint32_t req = o.tile_qubits > 0 ? static_cast<uint32_t>(o.tile_qubits)
                                                   : (c64 ? t.tile_qubits_c64 : t.tile_qubits);
            uint32_t m = c64 ? std::min<uint32_t>(std::max<uint32_t>(req, mb2::kMinTileQubits), mb2::kMaxTileQubitsC64)
                             : tile_width(req, num_qubits, blocks);
            for (const mb2::Block& b : blocks) m = std::max(m, b.k);
            m = std::min(m, num_qubits);
            // Pass i applies the next `gates` blocks of the program's order.
            const mb2::TileProgram prog = mb2::plan_tile_program(blocks, num_qubits, m, mb2::kDefaultFixedLow,
                                                                 nullptr, c64);
            std::vector<mb2::Block> ordered;
            ordered.reserve(prog.order.size());
            for (uint32_t i : prog.order) ordered.push_back(blocks[i]);
            size_t b0 = 0;
            for (const mb2::TilePass& p : prog.passes) {
                const size_t b1 = std::min(ordered.size(), b0 + p.gates);
                total += pass_seconds(t, c64, ordered, b0, b1, num_qubits);
                b0 = b1;
            }
        }
        *seconds = total;
    } catch (const std::exception& e) {
        return fail(ctx, MB2_ERR_INVALID, e.what());
    }
    return MB2_OK;
}

}  // extern "C"
