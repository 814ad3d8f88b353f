// The complex64 precision path's tile pass: the same tiled multi-gate sweep
// as the complex128 kernel (same planner, same compact instruction stream)
// on a state of (float, float) amplitudes, with FP32 fused multiply-adds.
//
// Gate matrices are composed in FP64 on the host and rounded to FP32 once
// per gate; every amplitude update is an FMA chain (one rounding per term
// instead of two), so the state's error against the FP64 oracle grows with
// depth at roughly one FP32 rounding per gate.  Expectations, norms and the
// sampler's probabilities are accumulated in FP64 from these amplitudes
// (kernels_reduce.cu, kernels_sample.cu).
#include <cuda_runtime.h>

#include <cstdint>

#include "c64_ops.cuh"
#include "device_math.cuh"
#include "mb2_internal.h"

namespace mb2 {
namespace {
using dev::pdep64;

using namespace c64;

// Tile slots are swizzled by swz8 (mb2_internal.h).

// A dense 2x2 on register slot P.  KIND: 0 general, 1 entry (0,0) real
// (U3), 2 every entry real; the known-zero imaginary parts are skipped.
template <int P, int KIND = 0>
__device__ __forceinline__ void g1(float2 (&a)[kNA], const float* md) {
    const Cf m00 = entry(md, 0), m01 = entry(md, 1), m10 = entry(md, 2), m11 = entry(md, 3);
#pragma unroll
    for (int j = 0; j < kNA; ++j) {
        if (j & (1 << P)) continue;
        const float2 x = a[j], y = a[j | (1 << P)];
        if constexpr (KIND == 2) {
            a[j] = make_float2(fmaf(m01.r, y.x, m00.r * x.x), fmaf(m01.r, y.y, m00.r * x.y));
            a[j | (1 << P)] = make_float2(fmaf(m11.r, y.x, m10.r * x.x), fmaf(m11.r, y.y, m10.r * x.y));
        } else if constexpr (KIND == 1) {
            a[j] = cfma(m01, y, make_float2(m00.r * x.x, m00.r * x.y));
            a[j | (1 << P)] = cfma(m11, y, cmulf(m10, x));
        } else {
            a[j] = cfma(m01, y, cmulf(m00, x));
            a[j | (1 << P)] = cfma(m11, y, cmulf(m10, x));
        }
    }
}

template <int P0, int P1>
__device__ __forceinline__ void g2(float2 (&a)[kNA], const float* md) {
    if constexpr (P0 == P1) {
        return;
    } else {
        Cf m[16];
#pragma unroll
        for (int e = 0; e < 16; ++e) m[e] = entry(md, e);
#pragma unroll
        for (int j = 0; j < kNA; ++j) {
            if (j & ((1 << P0) | (1 << P1))) continue;
            const int idx[4] = {j, j | (1 << P0), j | (1 << P1), j | (1 << P0) | (1 << P1)};
            const float2 in[4] = {a[idx[0]], a[idx[1]], a[idx[2]], a[idx[3]]};
#pragma unroll
            for (int o = 0; o < 4; ++o) {
                float2 acc = cmulf(m[4 * o], in[0]);
#pragma unroll
                for (int i = 1; i < 4; ++i) acc = cfma(m[4 * o + i], in[i], acc);
                a[idx[o]] = acc;
            }
        }
    }
}

template <int P0, int P1, int KIND>
__device__ __forceinline__ void perm2(float2 (&a)[kNA]) {
    if constexpr (P0 == P1) {
        return;
    } else {
        constexpr int lo = KIND == TK_SW23 ? 2 : 1;
        constexpr int hi = KIND == TK_SW12 ? 2 : 3;
#pragma unroll
        for (int j = 0; j < kNA; ++j) {
            if (j & ((1 << P0) | (1 << P1))) continue;
            const int il = j | ((lo & 1) ? (1 << P0) : 0) | ((lo & 2) ? (1 << P1) : 0);
            const int ih = j | ((hi & 1) ? (1 << P0) : 0) | ((hi & 2) ? (1 << P1) : 0);
            const float2 t = a[il];
            a[il] = a[ih];
            a[ih] = t;
        }
    }
}


// One pass: the complex128 kernel's structure (persistent CTAs, tiles
// `stages - 1` ahead in flight, masked-add tile bases, the pass's words and
// data staged in shared memory, a batch's parametric slice per tile) with
// FP32 gates.  MT > 0 fixes the tile width; IDX is the index type.
// V: 0 the lean variant without register-moving and rare heavy
// instructions (as the complex128 kernel's), for passes without them;
// 1 adds general dense two-qubit blocks (ansatz layers) and nothing else;
// 2 the full set.
template <int MAXT, int MINB, int MT, typename IDX, int V>
__global__ void __launch_bounds__(MAXT, MINB)
    k_tile_pass_c64(float2* __restrict__ st, uint32_t n, uint32_t m_rt, uint64_t smask,
                    const uint32_t* __restrict__ words, uint32_t nwords, const double* __restrict__ sdata,
                    uint32_t nsdata, const double* __restrict__ gdata, uint64_t ntiles,
                    const double* __restrict__ pdata, uint32_t pstride, uint32_t param_lo, uint32_t param_len,
                    uint32_t bshift, uint32_t stages) {
    extern __shared__ float2 smem_f[];
    const uint32_t m = MT > 0 ? static_cast<uint32_t>(MT) : m_rt;
    const uint32_t tid = threadIdx.x;
    const uint32_t tbits = m - kRegQubits;
    const uint32_t tile_amps = 1u << m;
    uint32_t* sw = reinterpret_cast<uint32_t*>(smem_f + stages * tile_amps);
    // The pass's data is staged as FP32 (each FP64-composed entry rounded once).
    float* sd = reinterpret_cast<float*>(sw + nwords);
    for (uint32_t i = tid; i < nwords / 4; i += blockDim.x)
        reinterpret_cast<uint4*>(sw)[i] = __ldg(reinterpret_cast<const uint4*>(words) + i);
    for (uint32_t i = tid; i < nsdata; i += blockDim.x) sd[i] = static_cast<float>(__ldg(sdata + i));
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
        if (param_len != 0) {  // a batched sweep: this tile's binding is t >> bshift
            const double* src = pdata + (t >> bshift) * pstride + param_lo;
            float* dst = sd + nsdata;
            for (uint32_t i = tid; i < param_len; i += blockDim.x) dst[i] = static_cast<float>(__ldg(src + i));
        }
        if (stages == 3) cp_async_wait<2>();
        else cp_async_wait<1>();
        __syncthreads();

        float2 a[kNA];
        uint32_t pc = 0;
        while (pc < nwords) {
            const uint32_t w0 = sw[pc];
            const uint32_t op0 = w0 & 0xffu;
            if (op0 == cop::kPhase) {
                // The phase record (cop::kPhase), 8-byte slot offsets.
                const uint32_t* rec = sw + pc;
                pc += cop::kPhaseWords;
                const uint16_t* et = reinterpret_cast<const uint16_t*>(rec + 5);
                uint32_t tb = static_cast<uint32_t>(et[tid & 15u]) | static_cast<uint32_t>(et[16 + ((tid >> 4) & 15u)]);
                if (MT == 0 || MT > 12) tb |= static_cast<uint32_t>(et[32 + ((tid >> 8) & 15u)]);
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
                for (;;) {
                    const uint32_t w = sw[pc++];
                    const uint32_t op = w & 0xffu;
                    if (op == cop::kEnd) break;
                    const uint32_t aux = (w >> 8) & 0xffu;
                    const float* md = sd + ((w >> 20) << 1);
                    const uint32_t tv = (tb >> ((w >> 16) & 15u)) & 1u;
                    switch (op) {
#define MB2_CASE4(BASE, ...) \
    case BASE + 0: { constexpr int P = 0; __VA_ARGS__; } break; \
    case BASE + 1: { constexpr int P = 1; __VA_ARGS__; } break; \
    case BASE + 2: { constexpr int P = 2; __VA_ARGS__; } break; \
    case BASE + 3: { constexpr int P = 3; __VA_ARGS__; } break;
#define MB2_CASE12(BASE, ...) \
    case BASE + 0: { constexpr int P0 = 0, P1 = 1; __VA_ARGS__; } break; \
    case BASE + 1: { constexpr int P0 = 0, P1 = 2; __VA_ARGS__; } break; \
    case BASE + 2: { constexpr int P0 = 0, P1 = 3; __VA_ARGS__; } break; \
    case BASE + 3: { constexpr int P0 = 1, P1 = 0; __VA_ARGS__; } break; \
    case BASE + 4: { constexpr int P0 = 1, P1 = 2; __VA_ARGS__; } break; \
    case BASE + 5: { constexpr int P0 = 1, P1 = 3; __VA_ARGS__; } break; \
    case BASE + 6: { constexpr int P0 = 2, P1 = 0; __VA_ARGS__; } break; \
    case BASE + 7: { constexpr int P0 = 2, P1 = 1; __VA_ARGS__; } break; \
    case BASE + 8: { constexpr int P0 = 2, P1 = 3; __VA_ARGS__; } break; \
    case BASE + 9: { constexpr int P0 = 3, P1 = 0; __VA_ARGS__; } break; \
    case BASE + 10: { constexpr int P0 = 3, P1 = 1; __VA_ARGS__; } break; \
    case BASE + 11: { constexpr int P0 = 3, P1 = 2; __VA_ARGS__; } break;
                        // Every dense 1q kind is the general 2x2 in FP32.
                        MB2_CASE4(cop::kU3, (g1<P, 1>(a, md)))
                        MB2_CASE4(cop::kGen1, (g1<P>(a, md)))
                        MB2_CASE4(cop::kReal1, (g1<P, 2>(a, md)))
                        case cop::kU3Run0123:
                            g1<0, 1>(a, md);
                            g1<1, 1>(a, md + 8);
                            g1<2, 1>(a, md + 16);
                            g1<3, 1>(a, md + 24);
                            break;
                        case cop::kU3Run01:
                            g1<0, 1>(a, md);
                            g1<1, 1>(a, md + 8);
                            break;
                        case cop::kU3Run123:
                            g1<1, 1>(a, md);
                            g1<2, 1>(a, md + 8);
                            g1<3, 1>(a, md + 16);
                            break;
                        case cop::kU3Run012:
                            g1<0, 1>(a, md);
                            g1<1, 1>(a, md + 8);
                            g1<2, 1>(a, md + 16);
                            break;
                        MB2_CASE12(cop::kGen2, if constexpr (V >= 1) g2<P0, P1>(a, md))
                        MB2_CASE12(cop::kMono2, if constexpr (V == 2) { ++pc; g2<P0, P1>(a, md); })
                        MB2_CASE12(cop::kSw12, if constexpr (V == 2) perm2<P0, P1, TK_SW12>(a))
                        MB2_CASE12(cop::kSw13, if constexpr (V == 2) perm2<P0, P1, TK_SW13>(a))
                        MB2_CASE12(cop::kSw23, if constexpr (V == 2) perm2<P0, P1, TK_SW23>(a))
                        MB2_CASE4(cop::kDs1R, (diag_regs<P, -1>(a, md, 1, aux, 0u, 0u)))
                        MB2_CASE12(cop::kDs2RR, (diag_regs<P0, P1>(a, md, 2, aux, 0u, 0u)))
#undef MB2_CASE4
#undef MB2_CASE12
                        case cop::kDs1T: diag_regs<-1, -1>(a, md, 1, aux, tv, 0u); break;
                        // kDs2RT + 2s + w: register slot s and a thread bit as operand w
                        // (w = 0: operand 0 is the thread bit, operand 1 the register).
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
                            for (int j = 0; j < kNA; ++j) {
                                const uint32_t msk = (M << (31 - j)) & 0x80000000u;
                                a[j] = make_float2(__uint_as_float(__float_as_uint(a[j].x) ^ msk),
                                                   __uint_as_float(__float_as_uint(a[j].y) ^ msk));
                            }
                        } break;
                        default: {  // cop::kDiagK: entry per amplitude
                            if constexpr (V != 2) break;
                            const uint32_t pos = sw[pc++];
                            uint32_t et = 0, e0 = 0, e1 = 0, e2 = 0, e3 = 0;
                            for (uint32_t b = 0; b < aux; ++b) {
                                const uint32_t bit = 1u << ((pos >> (4 * b)) & 15u);
                                et |= ((tb & bit) ? 1u : 0u) << b;
                                if (bit == rb[0]) e0 = 1u << b;
                                if (bit == rb[1]) e1 = 1u << b;
                                if (bit == rb[2]) e2 = 1u << b;
                                if (bit == rb[3]) e3 = 1u << b;
                            }
#pragma unroll
                            for (int j = 0; j < kNA; ++j) {
                                const uint32_t e = et | ((j & 1) ? e0 : 0u) | ((j & 2) ? e1 : 0u) |
                                                   ((j & 4) ? e2 : 0u) | ((j & 8) ? e3 : 0u);
                                a[j] = cmulf(entry(md, e), a[j]);
                            }
                        } break;
                    }
                }
#pragma unroll
                for (int j = 0; j < kNA; ++j) at(j) = a[j];
                __syncthreads();
            } else if (V == 2 && op0 == cop::kSmem) {
                const uint32_t k = (w0 >> 8) & 0xffu, dim = 1u << k;
                const uint32_t pos = sw[pc + 1];
                const double* md = gdata + sw[pc + 2];
                pc += 3;
                auto qpos = [&](uint32_t b) -> uint32_t { return (pos >> (4 * b)) & 15u; };
                uint32_t opm = 0;
                for (uint32_t b = 0; b < k; ++b) opm |= 1u << qpos(b);
#pragma unroll
                for (int j = 0; j < kNA; ++j) {
                    const uint32_t l = tid | (static_cast<uint32_t>(j) << tbits);
                    uint32_t out = 0;
                    for (uint32_t b = 0; b < k; ++b) out |= ((l >> qpos(b)) & 1u) << b;
                    const uint32_t gbase = l & ~opm;
                    float2 acc = make_float2(0.f, 0.f);
                    for (uint32_t in = 0; in < dim; ++in) {
                        uint32_t li = gbase;
                        for (uint32_t b = 0; b < k; ++b)
                            if ((in >> b) & 1u) li |= 1u << qpos(b);
                        acc = cfma(entry(md, out * dim + in), tile[swz8(li)], acc);
                    }
                    a[j] = acc;
                }
                __syncthreads();
#pragma unroll
                for (int j = 0; j < kNA; ++j) tile[slot(j)] = a[j];
                __syncthreads();
            } else {
                break;  // padding after the last instruction
            }
        }
        const IDX b0 = cbase + off_lo;
#pragma unroll
        for (int j = 0; j < kNA; ++j) st[b0 + reg_off(j)] = tile[slot(j)];
        cbase = advance(cbase);
        __syncthreads();
    }
}

template <int MAXT, int MINB, int MT, typename IDX, int V>
int launch_c64_instance(const TileLaunch& L) {
    // The dynamic limit is what the static shared memory leaves of the
    // per-block maximum; it is raised once, by whichever thread launches
    // first (the serving loop's workers launch concurrently: the static's
    // initialisation is thread-safe and every thread sees it complete).
    static const size_t dyn_max = [] {
        cudaFuncAttributes fa{};
        if (cudaFuncGetAttributes(&fa, k_tile_pass_c64<MAXT, MINB, MT, IDX, V>) != cudaSuccess) return size_t{0};
        const size_t v = kTileSmemMax - fa.sharedSizeBytes;
        if (cudaFuncSetAttribute(k_tile_pass_c64<MAXT, MINB, MT, IDX, V>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(v)) != cudaSuccess)
            return size_t{0};
        return v;
    }();
    if (dyn_max == 0) return launch_status();
    if (L.smem > dyn_max) return MB2_ERR_INVALID;
    k_tile_pass_c64<MAXT, MINB, MT, IDX, V><<<L.grid, L.threads, L.smem, static_cast<cudaStream_t>(L.stream)>>>(
        static_cast<float2*>(L.amps), L.n_all, L.m, L.smask, L.words, L.nwords, L.sdata, L.nsdata, L.gdata, L.ntiles,
        L.pdata, L.pstride, L.param_lo, L.param_len, L.bshift, L.stages);
    return launch_status();
}

// Scales every amplitude by s (FP32 product of an FP64-computed factor).
__global__ void k_scale_c64(float2* st, uint64_t n_amps, float s) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n_amps; i += stride) {
        const float2 a = st[i];
        st[i] = make_float2(a.x * s, a.y * s);
    }
}

}  // namespace

int launch_tile_pass_c64(void* amps, uint32_t n, const TilePass& pass, const uint32_t* dev_words,
                         const double* dev_sdata, const double* dev_gdata, int sm_count, void* stream,
                         const BatchLayout* batch) {
    if (pass.m > kMaxTileQubitsC64 || pass.m < kMinTileQubits) return MB2_ERR_INVALID;
    if ((pass.word_count & 3u) != 0 || (pass.param_len != 0 && batch == nullptr)) return MB2_ERR_INVALID;
    if (pass.gmask != 0) return MB2_ERR_INVALID;  // the complex64 kernels read operands inside the tile only
    TileLaunch L;
    L.amps = amps;
    L.m = pass.m;
    L.smask = pass.smask;
    L.words = dev_words + pass.word_begin;
    L.nwords = pass.word_count;
    L.sdata = dev_sdata + pass.sdata_begin;
    L.nsdata = pass.sdata_count;
    L.gdata = dev_gdata;
    L.pdata = batch ? batch->pdata : nullptr;
    L.pstride = batch ? batch->pstride : 0u;
    L.param_lo = pass.param_lo;
    L.param_len = pass.param_len;
    L.bshift = n - pass.m;
    L.stream = stream;
    L.threads = 1u << (pass.m - kRegQubits);
    // 13-qubit tiles (64 KiB): one CTA per SM with three buffers; smaller
    // tiles (12 by default, its own instances): two CTAs per SM with two
    // buffers each.
    L.stages = pass.m == kMaxTileQubitsC64 ? 3u : 2u;
    L.smem = L.stages * (size_t{1} << pass.m) * sizeof(float2) + size_t{pass.word_count} * 4 +
             (size_t{pass.sdata_count} + pass.param_len) * sizeof(float);
    L.ntiles = (uint64_t{1} << n) >> pass.m;
    L.n_all = n;
    if (batch != nullptr) {
        L.ntiles *= batch->bindings;
        while ((uint64_t{1} << (L.n_all - n)) < batch->bindings) ++L.n_all;
    }
    const uint64_t cap = static_cast<uint64_t>(sm_count) * (pass.m == kMaxTileQubitsC64 ? 1u : 2u);
    L.grid = static_cast<int>(L.ntiles < cap ? L.ntiles : cap);
    int rc;
    // Variant: lean, lean + dense two-qubit blocks, or full (TilePass::heavy/mid).
    const int v = !pass.heavy ? 0 : pass.mid ? 1 : 2;
    const bool i32 = L.n_all <= 32;
    if (pass.m == kMaxTileQubitsC64) {
        if (v == 0)
            rc = i32 ? launch_c64_instance<512, 1, 13, uint32_t, 0>(L) : launch_c64_instance<512, 1, 13, uint64_t, 0>(L);
        else if (v == 1)
            rc = i32 ? launch_c64_instance<512, 1, 13, uint32_t, 1>(L) : launch_c64_instance<512, 1, 13, uint64_t, 1>(L);
        else
            rc = i32 ? launch_c64_instance<512, 1, 13, uint32_t, 2>(L) : launch_c64_instance<512, 1, 13, uint64_t, 2>(L);
    } else if (pass.m == 12) {
        if (v == 0)
            rc = i32 ? launch_c64_instance<256, 2, 12, uint32_t, 0>(L) : launch_c64_instance<256, 2, 12, uint64_t, 0>(L);
        else if (v == 1)
            rc = i32 ? launch_c64_instance<256, 2, 12, uint32_t, 1>(L) : launch_c64_instance<256, 2, 12, uint64_t, 1>(L);
        else
            rc = i32 ? launch_c64_instance<256, 2, 12, uint32_t, 2>(L) : launch_c64_instance<256, 2, 12, uint64_t, 2>(L);
    } else {
        rc = launch_c64_instance<512, 1, 0, uint64_t, 2>(L);
    }
    note_launches(1);
    return rc;
}

int launch_scale_c64(void* amps, uint64_t n_amps, float s, void* stream) {
    const uint64_t blocks = (n_amps + 255) / 256;
    k_scale_c64<<<static_cast<unsigned>(blocks < 148ull * 16 ? blocks : 148ull * 16), 256, 0,
                  static_cast<cudaStream_t>(stream)>>>(static_cast<float2*>(amps), n_amps, s);
    note_launches(1);
    return launch_status();
}

}  // namespace mb2
