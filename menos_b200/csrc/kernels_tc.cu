// The complex64 tile pass on the tensor cores (sm_100a tcgen05).
//
// Same tiled sweep as kernels_c64.cu -- persistent CTAs, a tile of 2^m
// amplitudes staged in shared memory with cp.async, one thread per row of 16
// register amplitudes, phases that choose the four register qubits -- but a
// phase's dense gates are applied as one composed 16x16 complex matrix U on
// the tensor cores (tile_tc.cpp builds the program):
//
//   a tile is scaled once, at its first phase, by the power of two that puts
//   its norm in [2^13, 2^14) (unitary gates on tile qubits keep every
//   amplitude below the norm), and unscaled when it is stored; each thread
//   splits its row (32 floats, interleaved re/im) into FP16 high and low
//   parts and stores both into tensor memory (TMEM lane =
//   row within a 128-row block, two FP16 values per 32-bit column); one
//   thread issues, per 128-row block, six tcgen05.mma kind::f16 (N = 32,
//   two K-steps of 16 each) with A from tensor memory and B = 2^12 U's
//   operand in shared memory (FP16 high parts over low parts):
//   A_lo x B_hi, A_hi x B_lo, then A_hi x B_hi, all accumulated into one
//   block of 32 FP32 columns; tcgen05.commit signals an mbarrier that every
//   thread waits on; each thread then reads its row back (one tcgen05.ld),
//   takes out the 2^12 and applies the phase's elementwise diagonals on
//   registers.
//
// Every wait on the tensor core is bounded: a wait that runs out sets the
// caller's error word, the CTA stops issuing work, frees its tensor memory
// and returns.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "c64_ops.cuh"
#include "device_math.cuh"
#include "mb2_internal.h"

namespace mb2 {
namespace {
using dev::pdep64;
using namespace c64;

// ---- tcgen05 and mbarrier primitives ----------------------------------------
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
// One warp allocates `cols` TMEM columns (a power of two >= 32) and writes
// their base address to *dst.
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t cols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_addr(dst)), "r"(cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t cols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(cols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }
// Generic-proxy writes to shared memory made visible to the tensor core.
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n"
        ".reg .pred p;\n"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        "selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded: false when the phase did not complete within the limit.
constexpr uint32_t kSpinLimit = 1u << 22;
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    for (uint32_t i = 0; i < kSpinLimit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
// The mbarrier completes a phase when every tcgen05.mma this thread issued
// before has completed.
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(smem_addr(bar))
                 : "memory");
}
// D (TMEM) [+]= A (TMEM) * B (shared memory, descriptor), kind::f16.
__device__ __forceinline__ void mma_f16(uint32_t d, uint32_t a, uint64_t bdesc, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n"
        ".reg .pred p;\n"
        "setp.ne.b32 p, %4, 0;\n"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n"
        "}\n" ::"r"(d),
        "r"(a), "l"(bdesc), "r"(idesc), "r"(acc)
        : "memory");
}

#define MB2_R8(i) "r"(v[i]), "r"(v[i + 1]), "r"(v[i + 2]), "r"(v[i + 3]), "r"(v[i + 4]), "r"(v[i + 5]), "r"(v[i + 6]), "r"(v[i + 7])
#define MB2_W8(i) "=r"(v[i]), "=r"(v[i + 1]), "=r"(v[i + 2]), "=r"(v[i + 3]), "=r"(v[i + 4]), "=r"(v[i + 5]), "=r"(v[i + 6]), "=r"(v[i + 7])
// Consecutive 32-bit columns of this thread's lane (warp w reaches lanes
// 32 (w % 4) .. + 31; taddr carries the lane in bits 16-31).
__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t (&v)[16]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16};\n" ::"r"(taddr),
        MB2_R8(0), MB2_R8(8)
        : "memory");
}
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
        : MB2_W8(0), MB2_W8(8), MB2_W8(16), MB2_W8(24)
        : "r"(taddr)
        : "memory");
}
#undef MB2_R8
#undef MB2_W8
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;\n" ::: "memory"); }
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory"); }

__device__ __forceinline__ uint32_t half2_bits(__half2 h) { return *reinterpret_cast<uint32_t*>(&h); }

// tcgen05.mma kind::f16 instruction descriptor: D FP32 (bits 4-5 = 1),
// A and B FP16 (bits 7-9, 10-12 = 0), both K-major, N >> 3 at bit 17,
// M >> 4 at bit 24; M = 128 rows, N = 32 (U's 32 real output rows: their
// high parts at the operand's start, their low parts 2048 bytes on).
constexpr uint32_t kIdescN32 = (1u << 4) | ((32u >> 3) << 17) | ((128u >> 4) << 24);
constexpr uint32_t kLowPartBytes = 2048;  // 4 row groups of 512 bytes

// Packed FP32 pairs (sm_100a f32x2): one instruction for both parts.
__device__ __forceinline__ float2 sub_f32x2(float2 a, float2 b) {
    uint64_t r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(*reinterpret_cast<uint64_t*>(&a)), "l"(*reinterpret_cast<uint64_t*>(&b)));
    return *reinterpret_cast<float2*>(&r);
}
__device__ __forceinline__ float2 mul_f32x2(float2 a, float2 b) {
    uint64_t r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(*reinterpret_cast<uint64_t*>(&a)), "l"(*reinterpret_cast<uint64_t*>(&b)));
    return *reinterpret_cast<float2*>(&r);
}
// Shared-memory descriptor of B: start address >> 4 (bits 0-13), leading
// (K) byte offset 128 >> 4 (bits 16-29), stride (N) byte offset 512 >> 4
// (bits 32-45), descriptor version 1 (bits 46-47), no swizzle (bits 61-63 = 0).
__device__ __forceinline__ uint64_t b_desc(uint32_t saddr) {
    return static_cast<uint64_t>((saddr >> 4) & 0x3fffu) | (uint64_t{128u >> 4} << 16) |
           (uint64_t{512u >> 4} << 32) | (uint64_t{1} << 46);
}

// The block state of the tensor-core step: TMEM base, mbarrier, its phase
// parity, the CTA's abort flag and the caller's error word.
struct TcCtx {
    uint32_t tmem;
    uint64_t* bar;
    uint32_t parity;
    volatile int* abort;
    int* err;
};

// The power-of-two scale of a tile: 2^e puts the norm of the CTA's rows
// in [2^13, 2^14), so every amplitude -- at most the norm, which the pass's
// unitary gates on tile qubits preserve -- stays in FP16's range through all
// phases (e <= 126 keeps 2^-e a normal float; a zero tile keeps e = 0).
// Every thread of the CTA calls it; red: shared scratch of one float per warp.
__device__ __forceinline__ int tile_scale_exp(const float2 (&a)[kNA], float* red) {
    float ss = 0.0f;
#pragma unroll
    for (int j = 0; j < kNA; ++j) ss = fmaf(a[j].x, a[j].x, fmaf(a[j].y, a[j].y, ss));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) ss += __shfl_xor_sync(0xffffffffu, ss, o);
    if ((threadIdx.x & 31u) == 0) red[threadIdx.x >> 5] = ss;
    __syncthreads();
    float tot = 0.0f;
    for (uint32_t w = 0; w < (blockDim.x >> 5); ++w) tot += red[w];
    __syncthreads();  // red is free again
    const int ex = static_cast<int>((__float_as_uint(sqrtf(tot)) >> 23) & 0xffu);
    return ex == 0 ? 0 : max(-126, min(140 - ex, 126));
}
__device__ __forceinline__ float pow2f(int e) { return __uint_as_float(static_cast<uint32_t>(127 + e) << 23); }

// a <- U a for this thread's row, U's operand (kTcOperandWords words, the
// layout of tile_tc.cpp) at shared address b; the row is already scaled
// into FP16's range (tile_scale_exp).  ROWS threads, ROWS / 128 row blocks;
// TMEM columns: [0, 16 NB) high parts, [16 NB, 32 NB) low parts,
// [32 NB, 64 NB) the products (32 per block).  All threads of the CTA call
// it; thread 0 issues the MMAs, every thread waits for them on the mbarrier.
template <int ROWS>
__device__ __forceinline__ void tc_apply(float2 (&a)[kNA], uint32_t b, TcCtx& c) {
    constexpr uint32_t NB = ROWS / 128;
    const uint32_t tid = threadIdx.x;
    const uint32_t blk = tid >> 7;
    const uint32_t lane = (tid & 0x60u) << 16;  // this warp's lane quarter
    {
        uint32_t hi[16], lo[16];
#pragma unroll
        for (int j = 0; j < kNA; ++j) {
            const __half2 h = __floats2half2_rn(a[j].x, a[j].y);
            hi[j] = half2_bits(h);
            lo[j] = half2_bits(__float22half2_rn(sub_f32x2(a[j], __half22float2(h))));
        }
        tmem_st16(c.tmem + lane + 16 * blk, hi);
        tmem_st16(c.tmem + lane + 16 * NB + 16 * blk, lo);
    }
    tmem_wait_st();
    tc_fence_before();
    __syncthreads();
    const bool abort = *c.abort != 0;
    if (!abort && tid == 0) {
        tc_fence_after();
        const uint64_t bh0 = b_desc(b), bh1 = b_desc(b + 256);
        const uint64_t bl0 = b_desc(b + kLowPartBytes), bl1 = b_desc(b + kLowPartBytes + 256);
#pragma unroll
        for (uint32_t k = 0; k < NB; ++k) {
            const uint32_t ah = c.tmem + 16 * k, al = c.tmem + 16 * NB + 16 * k, d = c.tmem + 32 * NB + 32 * k;
            // The small products first, the high-by-high product last.
            mma_f16(d, al, bh0, kIdescN32, 0);
            mma_f16(d, al + 8, bh1, kIdescN32, 1);
            mma_f16(d, ah, bl0, kIdescN32, 1);
            mma_f16(d, ah + 8, bl1, kIdescN32, 1);
            mma_f16(d, ah, bh0, kIdescN32, 1);
            mma_f16(d, ah + 8, bh1, kIdescN32, 1);
        }
        mma_commit(c.bar);
    }
    // Every thread waits on the MMAs' mbarrier itself (no CTA barrier): its
    // phase completes when the products are in tensor memory.
    if (!abort) {
        if (!mbar_wait(c.bar, c.parity)) {
            *c.abort = 1;
            atomicExch(c.err, 1);
        }
        c.parity ^= 1u;
    }
    tc_fence_after();
    uint32_t v[32];
    tmem_ld32(c.tmem + lane + 32 * NB + 32 * blk, v);
    tmem_wait_ld();
    constexpr float kUnscale = static_cast<float>(1.0 / kTcOperandScale);
#pragma unroll
    for (int j = 0; j < kNA; ++j)
        a[j] = mul_f32x2(make_float2(__uint_as_float(v[2 * j]), __uint_as_float(v[2 * j + 1])),
                         make_float2(kUnscale, kUnscale));
}

// Sets up TMEM (warp 0), the mbarrier and the abort flag; the caller's
// shared words hold them.
template <uint32_t COLS>
__device__ __forceinline__ TcCtx tc_setup(uint32_t* s_tmem, uint64_t* s_bar, int* s_abort, int* err) {
    if (threadIdx.x < 32) tmem_alloc(s_tmem, COLS);
    if (threadIdx.x == 0) {
        mbar_init(s_bar, 1);
        *s_abort = 0;
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    return TcCtx{*s_tmem, s_bar, 0u, s_abort, err};
}
template <uint32_t COLS>
__device__ __forceinline__ void tc_teardown(const TcCtx& c) {
    tc_fence_before();
    __syncthreads();
    if (threadIdx.x < 32) {
        tc_fence_after();
        tmem_dealloc(c.tmem, COLS);
    }
}

// ---- probe: the tensor-core step alone, on 256 rows -------------------------
__global__ void __launch_bounds__(256, 1) k_tc_probe(const float2* __restrict__ in, const uint32_t* __restrict__ b,
                                                     float2* __restrict__ out, int* err) {
    __shared__ __align__(128) uint32_t sb[kTcOperandWords];
    __shared__ uint32_t s_tmem;
    __shared__ __align__(8) uint64_t s_bar;
    __shared__ int s_abort;
    for (uint32_t i = threadIdx.x; i < kTcOperandWords / 4; i += blockDim.x)
        reinterpret_cast<uint4*>(sb)[i] = reinterpret_cast<const uint4*>(b)[i];
    fence_async_smem();
    TcCtx c = tc_setup<256>(&s_tmem, &s_bar, &s_abort, err);
    __shared__ float s_red[8];
    float2 a[kNA];
#pragma unroll
    for (int j = 0; j < kNA; ++j) a[j] = in[threadIdx.x * kNA + j];
    const int e = tile_scale_exp(a, s_red);
    const float scale = pow2f(e), unscale = pow2f(-e);
#pragma unroll
    for (int j = 0; j < kNA; ++j) a[j] = make_float2(a[j].x * scale, a[j].y * scale);
    tc_apply<256>(a, smem_addr(sb), c);
#pragma unroll
    for (int j = 0; j < kNA; ++j) out[threadIdx.x * kNA + j] = make_float2(a[j].x * unscale, a[j].y * unscale);
    tc_teardown<256>(c);
}

// ---- the pass ----------------------------------------------------------------
// MT: tile qubits (11: 128 threads, four CTAs per SM; 12: 256 threads, two;
// 13: 512 threads, one);
// IDX: the amplitude index type.  Dynamic shared memory: `stages` tile
// buffers, the pass's phase matrices, its words, its diagonal data (FP32).
template <int MT, int MINB, typename IDX>
__global__ void __launch_bounds__(1 << (MT - 4), MINB)
    k_tile_pass_tc(float2* __restrict__ st, uint32_t n, uint64_t smask, const uint32_t* __restrict__ words,
                   uint32_t nwords, const double* __restrict__ sdata, uint32_t nsdata,
                   const uint32_t* __restrict__ tcm, uint32_t nphases, uint64_t ntiles, uint32_t stages, int* err) {
    constexpr uint32_t kRows = 1u << (MT - 4);
    constexpr uint32_t kCols = kRows == 128 ? 128 : (kRows == 256 ? 256 : 512);
    extern __shared__ __align__(128) float2 smem_f[];
    __shared__ uint32_t s_tmem;
    __shared__ __align__(8) uint64_t s_bar;
    __shared__ int s_abort;
    __shared__ float s_red[kRows / 32];
    const uint32_t tid = threadIdx.x;
    constexpr uint32_t m = MT;
    constexpr uint32_t tbits = m - kRegQubits;
    constexpr uint32_t tile_amps = 1u << m;
    uint32_t* sb = reinterpret_cast<uint32_t*>(smem_f + stages * tile_amps);
    uint32_t* sw = sb + nphases * kTcOperandWords;
    float* sd = reinterpret_cast<float*>(sw + nwords);
    for (uint32_t i = tid; i < nphases * (kTcOperandWords / 4); i += kRows)
        reinterpret_cast<uint4*>(sb)[i] = __ldg(reinterpret_cast<const uint4*>(tcm) + i);
    for (uint32_t i = tid; i < nwords / 4; i += kRows)
        reinterpret_cast<uint4*>(sw)[i] = __ldg(reinterpret_cast<const uint4*>(words) + i);
    for (uint32_t i = tid; i < nsdata; i += kRows) sd[i] = static_cast<float>(__ldg(sdata + i));
    fence_async_smem();
    TcCtx c = tc_setup<kCols>(&s_tmem, &s_bar, &s_abort, err);
    const uint32_t sb_addr = smem_addr(sb);

    IDX off_lo = 0, hib0 = 0, hib1 = 0, hib2 = 0, hib3 = 0;
    {
        uint32_t b = 0;
        for (uint32_t p = 0; p < n; ++p) {
            if (!((smask >> p) & 1u)) continue;
            if (b < tbits) {
                off_lo |= static_cast<IDX>((tid >> b) & 1u) << p;
            } else {
                const IDX v = IDX{1} << p;
                const uint32_t r = b - tbits;
                if (r == 0) hib0 = v;
                else if (r == 1) hib1 = v;
                else if (r == 2) hib2 = v;
                else hib3 = v;
            }
            ++b;
        }
    }
    const uint64_t nmask64 = ((n >= 64) ? ~uint64_t{0} : ((uint64_t{1} << n) - 1)) & ~smask;
    const IDX nmask = static_cast<IDX>(nmask64);
    const IDX step = static_cast<IDX>(pdep64(gridDim.x, nmask64));
    auto advance = [&](IDX b) -> IDX { return ((b | ~nmask) + step) & nmask; };
    const uint32_t s_tid = swz8(tid);
    auto reg_off = [&](int j) -> IDX {
        return ((j & 1) ? hib0 : IDX{0}) + ((j & 2) ? hib1 : IDX{0}) + ((j & 4) ? hib2 : IDX{0}) +
               ((j & 8) ? hib3 : IDX{0});
    };
    auto slot = [&](int j) -> uint32_t { return s_tid ^ swz8(static_cast<uint32_t>(j) << tbits); };
    auto prefetch = [&](IDX base, float2* buf) {
        const IDX b0 = base + off_lo;
#pragma unroll
        for (int j = 0; j < kNA; ++j) cp_async8(buf + slot(j), st + (b0 + reg_off(j)));
        cp_async_commit();
    };
    uint64_t tp = blockIdx.x;
    IDX pbase = static_cast<IDX>(pdep64(blockIdx.x, nmask64));
    IDX cbase = pbase;
    for (uint32_t sg = 0; sg + 1 < stages; ++sg) {
        if (tp < ntiles) prefetch(pbase, smem_f + sg * tile_amps);
        else cp_async_commit();
        tp += gridDim.x;
        pbase = advance(pbase);
    }
    uint32_t cur = 0, nxt = stages - 1;
    for (uint64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        float2* tile = smem_f + cur * tile_amps;
        if (tp < ntiles) prefetch(pbase, smem_f + nxt * tile_amps);
        else cp_async_commit();
        tp += gridDim.x;
        pbase = advance(pbase);
        cur = cur + 1 == stages ? 0u : cur + 1;
        nxt = nxt + 1 == stages ? 0u : nxt + 1;
        if (stages == 3) cp_async_wait<2>();
        else cp_async_wait<1>();
        __syncthreads();

        float2 a[kNA];
        uint32_t pc = 0;
        // The tile's scale, set at its first phase; the tile is stored unscaled.
        float unscale = 1.0f;
        bool first = true;
        while (pc < nwords) {
            const uint32_t w0 = sw[pc];
            if ((w0 & 0xffu) != cop::kPhase) break;  // padding after the last phase
            // The phase record (cop::kPhase), 8-byte slot offsets.
            const uint32_t* rec = sw + pc;
            pc += cop::kPhaseWords;
            const uint16_t* et = reinterpret_cast<const uint16_t*>(rec + 5);
            uint32_t tb = static_cast<uint32_t>(et[tid & 15u]) | static_cast<uint32_t>(et[16 + ((tid >> 4) & 15u)]);
            if (MT > 12) tb |= static_cast<uint32_t>(et[32 + ((tid >> 8) & 15u)]);
            uint32_t rb[kR];
#pragma unroll
            for (int b = 0; b < kR; ++b) rb[b] = 1u << ((w0 >> (16 + 4 * b)) & 15u);
            const uint32_t z0 = swz8(tb) << 3, z1 = rec[3] & 0xffffu, z2 = rec[3] >> 16, z3 = rec[4] & 0xffffu,
                           z4 = rec[4] >> 16;
            char* const tile_b = reinterpret_cast<char*>(tile);
            auto at = [&](int j) -> float2& {
                return *reinterpret_cast<float2*>(tile_b + (z0 ^ ((j & 1) ? z1 : 0u) ^ ((j & 2) ? z2 : 0u) ^
                                                             ((j & 4) ? z3 : 0u) ^ ((j & 8) ? z4 : 0u)));
            };
#pragma unroll
            for (int j = 0; j < kNA; ++j) a[j] = at(j);
            if (first) {
                first = false;
                const int e = tile_scale_exp(a, s_red);
                const float scale = pow2f(e);
                unscale = pow2f(-e);
#pragma unroll
                for (int j = 0; j < kNA; ++j) a[j] = make_float2(a[j].x * scale, a[j].y * scale);
            }
            for (;;) {
                const uint32_t w = sw[pc++];
                const uint32_t op = w & 0xffu;
                if (op == cop::kEnd) break;
                if (op == cop::kMma) {
                    tc_apply<kRows>(a, sb_addr + ((w >> 8) & 0xffu) * (kTcOperandWords * 4), c);
                    continue;
                }
                const uint32_t aux = (w >> 8) & 0xffu;
                const float* md = sd + ((w >> 20) << 1);
                const uint32_t tv = (tb >> ((w >> 16) & 15u)) & 1u;
                switch (op) {
                    case cop::kDs1R + 0: diag_regs<0, -1>(a, md, 1, aux, 0u, 0u); break;
                    case cop::kDs1R + 1: diag_regs<1, -1>(a, md, 1, aux, 0u, 0u); break;
                    case cop::kDs1R + 2: diag_regs<2, -1>(a, md, 1, aux, 0u, 0u); break;
                    case cop::kDs1R + 3: diag_regs<3, -1>(a, md, 1, aux, 0u, 0u); break;
                    case cop::kDs2RR + 0: diag_regs<0, 1>(a, md, 2, aux, 0u, 0u); break;
                    case cop::kDs2RR + 1: diag_regs<0, 2>(a, md, 2, aux, 0u, 0u); break;
                    case cop::kDs2RR + 2: diag_regs<0, 3>(a, md, 2, aux, 0u, 0u); break;
                    case cop::kDs2RR + 3: diag_regs<1, 0>(a, md, 2, aux, 0u, 0u); break;
                    case cop::kDs2RR + 4: diag_regs<1, 2>(a, md, 2, aux, 0u, 0u); break;
                    case cop::kDs2RR + 5: diag_regs<1, 3>(a, md, 2, aux, 0u, 0u); break;
                    case cop::kDs2RR + 6: diag_regs<2, 0>(a, md, 2, aux, 0u, 0u); break;
                    case cop::kDs2RR + 7: diag_regs<2, 1>(a, md, 2, aux, 0u, 0u); break;
                    case cop::kDs2RR + 8: diag_regs<2, 3>(a, md, 2, aux, 0u, 0u); break;
                    case cop::kDs2RR + 9: diag_regs<3, 0>(a, md, 2, aux, 0u, 0u); break;
                    case cop::kDs2RR + 10: diag_regs<3, 1>(a, md, 2, aux, 0u, 0u); break;
                    case cop::kDs2RR + 11: diag_regs<3, 2>(a, md, 2, aux, 0u, 0u); break;
                    case cop::kDs1T: diag_regs<-1, -1>(a, md, 1, aux, tv, 0u); break;
                    // kDs2RT + 2s + w: register slot s and a thread bit as operand w.
                    case cop::kDs2RT + 0: diag_regs<-1, 0>(a, md, 2, aux, tv, 0u); break;
                    case cop::kDs2RT + 1: diag_regs<0, -1>(a, md, 2, aux, 0u, tv); break;
                    case cop::kDs2RT + 2: diag_regs<-1, 1>(a, md, 2, aux, tv, 0u); break;
                    case cop::kDs2RT + 3: diag_regs<1, -1>(a, md, 2, aux, 0u, tv); break;
                    case cop::kDs2RT + 4: diag_regs<-1, 2>(a, md, 2, aux, tv, 0u); break;
                    case cop::kDs2RT + 5: diag_regs<2, -1>(a, md, 2, aux, 0u, tv); break;
                    case cop::kDs2RT + 6: diag_regs<-1, 3>(a, md, 2, aux, tv, 0u); break;
                    case cop::kDs2RT + 7: diag_regs<3, -1>(a, md, 2, aux, 0u, tv); break;
                    case cop::kDs2TT: {
                        const uint32_t cc = sw[pc++];
                        diag_regs<-1, -1>(a, md, 2, aux, (tb >> (cc & 15u)) & 1u, (tb >> ((cc >> 4) & 15u)) & 1u);
                    } break;
                    case cop::kSigns: {
                        uint32_t M = 0;
                        for (uint32_t i = 0; i < aux; ++i) {
                            const uint32_t mono = sw[pc++];
                            const uint32_t tm = mono >> 16;
                            M ^= (tb & tm) == tm ? (mono & 0xffffu) : 0u;
                        }
#pragma unroll
                        for (int j = 0; j < kNA; ++j) a[j] = fneg_if(a[j], (M >> j) & 1u);
                    } break;
                    default: {  // cop::kDiagK: entry per amplitude
                        const uint32_t pos = sw[pc++];
                        uint32_t et2 = 0, e0 = 0, e1 = 0, e2 = 0, e3 = 0;
                        for (uint32_t b = 0; b < aux; ++b) {
                            const uint32_t bit = 1u << ((pos >> (4 * b)) & 15u);
                            et2 |= ((tb & bit) ? 1u : 0u) << b;
                            if (bit == rb[0]) e0 = 1u << b;
                            if (bit == rb[1]) e1 = 1u << b;
                            if (bit == rb[2]) e2 = 1u << b;
                            if (bit == rb[3]) e3 = 1u << b;
                        }
#pragma unroll
                        for (int j = 0; j < kNA; ++j) {
                            const uint32_t e = et2 | ((j & 1) ? e0 : 0u) | ((j & 2) ? e1 : 0u) | ((j & 4) ? e2 : 0u) |
                                               ((j & 8) ? e3 : 0u);
                            a[j] = cmulf(entry(md, e), a[j]);
                        }
                    } break;
                }
            }
#pragma unroll
            for (int j = 0; j < kNA; ++j) at(j) = a[j];
            __syncthreads();
        }
        const IDX b0 = cbase + off_lo;
#pragma unroll
        for (int j = 0; j < kNA; ++j) {
            const float2 v = tile[slot(j)];
            st[b0 + reg_off(j)] = make_float2(v.x * unscale, v.y * unscale);
        }
        cbase = advance(cbase);
        __syncthreads();
        if (*c.abort) break;
    }
    cp_async_wait<0>();
    tc_teardown<kCols>(c);
}

template <int MT, int MINB, typename IDX>
int launch_tc_instance(const TileLaunch& L, const uint32_t* tcm, uint32_t nphases, int* err) {
    static const size_t dyn_max = [] {
        cudaFuncAttributes fa{};
        if (cudaFuncGetAttributes(&fa, k_tile_pass_tc<MT, MINB, IDX>) != cudaSuccess) return size_t{0};
        const size_t v = kTileSmemMax - fa.sharedSizeBytes;
        if (cudaFuncSetAttribute(k_tile_pass_tc<MT, MINB, IDX>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(v)) != cudaSuccess)
            return size_t{0};
        return v;
    }();
    if (dyn_max == 0) return launch_status();
    if (L.smem > dyn_max) return MB2_ERR_INVALID;
    k_tile_pass_tc<MT, MINB, IDX><<<L.grid, 1u << (MT - 4), L.smem, static_cast<cudaStream_t>(L.stream)>>>(
        static_cast<float2*>(L.amps), L.n_all, L.smask, L.words, L.nwords, L.sdata, L.nsdata, tcm, nphases, L.ntiles,
        L.stages, err);
    return launch_status();
}

}  // namespace

int launch_tile_pass_tc(void* amps, uint32_t n, const TilePass& pass, const uint32_t* dev_words,
                        const double* dev_sdata, const uint32_t* dev_tc, int* dev_err, int sm_count, void* stream) {
    if (!pass.tc || pass.m < 11 || pass.m > 13 || (pass.word_count & 3u) != 0 || pass.gmask != 0)
        return MB2_ERR_INVALID;
    TileLaunch L;
    L.amps = amps;
    L.m = pass.m;
    L.smask = pass.smask;
    L.words = dev_words + pass.word_begin;
    L.nwords = pass.word_count;
    L.sdata = dev_sdata + pass.sdata_begin;
    L.nsdata = pass.sdata_count;
    L.stream = stream;
    L.stages = 2;
    L.smem = L.stages * (size_t{1} << pass.m) * sizeof(float2) + size_t{pass.tc_phases} * kTcOperandWords * 4 +
             size_t{pass.word_count} * 4 + size_t{pass.sdata_count} * 4;
    L.ntiles = (uint64_t{1} << n) >> pass.m;
    L.n_all = n;
    // Resident CTAs per SM: tensor memory (128, 256 or 512 columns per CTA)
    // and shared memory allow four, two or one.
    const uint32_t per_sm = pass.m == 11 ? 4u : (pass.m == 12 ? 2u : 1u);
    const uint64_t cap = static_cast<uint64_t>(sm_count) * per_sm;
    L.grid = static_cast<int>(L.ntiles < cap ? L.ntiles : cap);
    const uint32_t* tcm = dev_tc + pass.tc_begin;
    const bool i32 = n <= 32;
    int rc;
    if (pass.m == 11) rc = i32 ? launch_tc_instance<11, 4, uint32_t>(L, tcm, pass.tc_phases, dev_err)
                               : launch_tc_instance<11, 4, uint64_t>(L, tcm, pass.tc_phases, dev_err);
    else if (pass.m == 12) rc = i32 ? launch_tc_instance<12, 2, uint32_t>(L, tcm, pass.tc_phases, dev_err)
                                    : launch_tc_instance<12, 2, uint64_t>(L, tcm, pass.tc_phases, dev_err);
    else rc = i32 ? launch_tc_instance<13, 1, uint32_t>(L, tcm, pass.tc_phases, dev_err)
                  : launch_tc_instance<13, 1, uint64_t>(L, tcm, pass.tc_phases, dev_err);
    note_launches(1);
    return rc;
}

int launch_tc_probe(const float* in, const uint32_t* b, float* out, int* dev_err, void* stream) {
    k_tc_probe<<<1, 256, 0, static_cast<cudaStream_t>(stream)>>>(reinterpret_cast<const float2*>(in), b,
                                                                 reinterpret_cast<float2*>(out), dev_err);
    note_launches(1);
    return launch_status();
}

}  // namespace mb2
