// The complex64 precision path's tile pass: the same tiled multi-gate sweep
// as the complex128 kernel (same planner, same instruction stream) on a
// state of (float, float) amplitudes, with FP32 fused multiply-adds.
//
// Gate matrices are composed in FP64 on the host and rounded to FP32 once
// per gate; every amplitude update is an FMA chain (one rounding per term
// instead of two), so the state's error against the FP64 oracle grows with
// depth at roughly one FP32 rounding per gate.  Expectations, norms and the
// sampler's probabilities are accumulated in FP64 from these amplitudes
// (kernels_reduce.cu, kernels_sample.cu).
#include <cuda_runtime.h>

#include <cstdint>

#include "mb2_internal.h"

namespace mb2 {
namespace {

constexpr int kR = static_cast<int>(kRegQubits);
constexpr int kNA = 1 << kR;
static_assert(kR == 4, "written for 4 register qubits");

__host__ __device__ constexpr int lowbit_index(int j) { return (j & 1) ? 0 : (j & 2) ? 1 : (j & 4) ? 2 : 3; }

// 8-byte slots: the low four bits XOR-folded with every higher 4-bit group
// (XOR-linear, so slot addresses compose by XOR).
__device__ __forceinline__ uint32_t swz8(uint32_t l) {
    const uint32_t h = l >> 4;
    return l ^ ((h ^ (h >> 4) ^ (h >> 8)) & 15u);
}

struct DI {
    uint64_t w0, w1, w2, w3;
    __device__ __forceinline__ uint32_t op() const { return static_cast<uint32_t>(w0 & 0xffu); }
    __device__ __forceinline__ uint32_t k() const { return static_cast<uint32_t>((w0 >> 8) & 0xffu); }
    __device__ __forceinline__ uint32_t kind() const { return static_cast<uint32_t>((w0 >> 16) & 0xffu); }
    __device__ __forceinline__ uint32_t nthread() const { return static_cast<uint32_t>((w0 >> 24) & 0xffu); }
    __device__ __forceinline__ uint32_t pos(uint32_t b) const {
        return static_cast<uint32_t>((b < 4 ? (w0 >> (32 + 8 * b)) : (w1 >> (8 * (b - 4)))) & 0xffu);
    }
    __device__ __forceinline__ uint32_t data() const { return static_cast<uint32_t>(w1 >> 32); }
    __device__ __forceinline__ uint32_t tperm(uint32_t i) const {
        return static_cast<uint32_t>((i < 8 ? (w2 >> (8 * i)) : (w3 >> (8 * (i - 8)))) & 0xffu);
    }
    __device__ __forceinline__ uint32_t aux() const { return static_cast<uint32_t>(w3 >> 32); }
};

__device__ __forceinline__ DI load_instr(const TileInstr* p) {
    const ulonglong2* s = reinterpret_cast<const ulonglong2*>(p);
    const ulonglong2 a = s[0], b = s[1];
    return DI{a.x, a.y, b.x, b.y};
}

__device__ __forceinline__ uint64_t pdep64(uint64_t v, uint64_t mask) {
    uint64_t r = 0;
    while (mask != 0) {
        const uint64_t low = mask & (~mask + 1);
        if (v & 1) r |= low;
        v >>= 1;
        mask ^= low;
    }
    return r;
}

struct Cf {
    float r, i;
};
__device__ __forceinline__ Cf entry(const double* md, uint32_t e) {
    const double2 d = reinterpret_cast<const double2*>(md)[e];
    return Cf{static_cast<float>(d.x), static_cast<float>(d.y)};
}
// acc + m * x, as two FMA chains.
__device__ __forceinline__ float2 cfma(Cf m, float2 x, float2 acc) {
    return make_float2(fmaf(m.r, x.x, fmaf(-m.i, x.y, acc.x)), fmaf(m.r, x.y, fmaf(m.i, x.x, acc.y)));
}
__device__ __forceinline__ float2 cmulf(Cf m, float2 x) { return cfma(m, x, make_float2(0.f, 0.f)); }

template <int P>
__device__ __forceinline__ void g1(float2 (&a)[kNA], const double* md) {
    const Cf m00 = entry(md, 0), m01 = entry(md, 1), m10 = entry(md, 2), m11 = entry(md, 3);
#pragma unroll
    for (int j = 0; j < kNA; ++j) {
        if (j & (1 << P)) continue;
        const float2 x = a[j], y = a[j | (1 << P)];
        a[j] = cfma(m01, y, cmulf(m00, x));
        a[j | (1 << P)] = cfma(m11, y, cmulf(m10, x));
    }
}

template <int P0, int P1>
__device__ __forceinline__ void g2(float2 (&a)[kNA], const double* md) {
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

template <int P>
__device__ __forceinline__ void perm1(float2 (&a)[kNA]) {
#pragma unroll
    for (int j = 0; j < kNA; ++j) {
        if (j & (1 << P)) continue;
        const float2 t = a[j];
        a[j] = a[j | (1 << P)];
        a[j | (1 << P)] = t;
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

#define MB2_PAIR_SWITCH(p0, p1, CALL)                 \
    switch ((p0) * 4 + (p1)) {                        \
        case 1: CALL(0, 1); break;                    \
        case 2: CALL(0, 2); break;                    \
        case 3: CALL(0, 3); break;                    \
        case 4: CALL(1, 0); break;                    \
        case 6: CALL(1, 2); break;                    \
        case 7: CALL(1, 3); break;                    \
        case 8: CALL(2, 0); break;                    \
        case 9: CALL(2, 1); break;                    \
        case 11: CALL(2, 3); break;                   \
        case 12: CALL(3, 0); break;                   \
        case 13: CALL(3, 1); break;                   \
        case 14: CALL(3, 2); break;                   \
        default: break;                               \
    }

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const uint32_t s = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

__global__ void __launch_bounds__(512, 1)
    k_tile_pass_c64(float2* __restrict__ st, uint32_t n, uint32_t m, uint64_t smask, const TileInstr* __restrict__ prog,
                    uint32_t nprog, const double* __restrict__ sdata, uint32_t nsdata, const double* __restrict__ gdata,
                    uint64_t ntiles, uint32_t stages) {
    extern __shared__ float2 smem_tiles_f[];
    const uint32_t tid = threadIdx.x;
    const uint32_t tbits = m - kRegQubits;
    const uint32_t tile_amps = 1u << m;
    TileInstr* sprog = reinterpret_cast<TileInstr*>(smem_tiles_f + stages * tile_amps);
    double* sd = reinterpret_cast<double*>(sprog + nprog);
    for (uint32_t i = tid; i < nprog * 2; i += blockDim.x)
        reinterpret_cast<ulonglong2*>(sprog)[i] = __ldg(reinterpret_cast<const ulonglong2*>(prog) + i);
    for (uint32_t i = tid; i < nsdata; i += blockDim.x) sd[i] = __ldg(sdata + i);
    uint64_t off_lo = 0, hib[kR] = {0, 0, 0, 0};
    {
        uint32_t b = 0;
        for (uint32_t p = 0; p < n; ++p) {
            if (!((smask >> p) & 1u)) continue;
            if (b < tbits) {
                off_lo |= static_cast<uint64_t>((tid >> b) & 1u) << p;
            } else {
#pragma unroll
                for (int r = 0; r < kR; ++r)
                    if (static_cast<uint32_t>(r) == b - tbits) hib[r] = uint64_t{1} << p;
            }
            ++b;
        }
    }
    const uint64_t nmask = ((n >= 64) ? ~uint64_t{0} : ((uint64_t{1} << n) - 1)) & ~smask;
    // Canonical slots: tid | j << tbits, by XOR-linearity from four constants.
    uint32_t cadr[kNA];
    cadr[0] = swz8(tid);
#pragma unroll
    for (int j = 1; j < kNA; ++j) cadr[j] = cadr[j & (j - 1)] ^ swz8(1u << (tbits + lowbit_index(j)));
    auto reg_off = [&](int j) -> uint64_t {
        return ((j & 1) ? hib[0] : 0) | ((j & 2) ? hib[1] : 0) | ((j & 4) ? hib[2] : 0) | ((j & 8) ? hib[3] : 0);
    };
    auto prefetch = [&](uint64_t t, float2* buf) {
        const uint64_t base = pdep64(t, nmask) | off_lo;
#pragma unroll
        for (int j = 0; j < kNA; ++j) cp_async8(buf + cadr[j], st + (base | reg_off(j)));
        cp_async_commit();
    };

    const uint64_t t0 = blockIdx.x;
    for (uint32_t sg = 0; sg + 1 < stages; ++sg) {
        const uint64_t tp = t0 + static_cast<uint64_t>(sg) * gridDim.x;
        if (tp < ntiles) prefetch(tp, smem_tiles_f + sg * tile_amps);
        else cp_async_commit();
    }
    uint64_t t = t0;
    for (uint32_t it = 0; t < ntiles; t += gridDim.x, ++it) {
        float2* tile = smem_tiles_f + (it % stages) * tile_amps;
        const uint64_t tn = t + static_cast<uint64_t>(stages - 1) * gridDim.x;
        if (tn < ntiles) prefetch(tn, smem_tiles_f + ((it + stages - 1) % stages) * tile_amps);
        else cp_async_commit();
        if (stages == 3) cp_async_wait<2>();
        else cp_async_wait<1>();
        __syncthreads();

        float2 a[kNA];
        uint32_t pc = 0;
        while (pc < nprog) {
            const DI I = load_instr(sprog + pc);
            ++pc;
            if (I.op() == TOP_PHASE) {
                uint32_t tb = 0;
                for (uint32_t i = 0; i < I.nthread(); ++i) tb |= ((tid >> i) & 1u) << I.tperm(i);
                uint32_t rb[kR];
#pragma unroll
                for (int b = 0; b < kR; ++b) rb[b] = 1u << I.pos(b);
                uint32_t adr[kNA];
                adr[0] = swz8(tb);
#pragma unroll
                for (int j = 1; j < kNA; ++j) adr[j] = adr[j & (j - 1)] ^ swz8(rb[lowbit_index(j)]);
#pragma unroll
                for (int j = 0; j < kNA; ++j) a[j] = tile[adr[j]];
                for (;;) {
                    const DI G = load_instr(sprog + pc);
                    ++pc;
                    if (G.op() == TOP_END) break;
                    const double* md = sd + G.data();
                    if (G.op() == TOP_G1) {
                        if (G.kind() == TK_X) {
                            switch (G.pos(0)) {
                                case 0: perm1<0>(a); break;
                                case 1: perm1<1>(a); break;
                                case 2: perm1<2>(a); break;
                                default: perm1<3>(a); break;
                            }
                        } else {
                            switch (G.pos(0)) {
                                case 0: g1<0>(a, md); break;
                                case 1: g1<1>(a, md); break;
                                case 2: g1<2>(a, md); break;
                                default: g1<3>(a, md); break;
                            }
                        }
                    } else if (G.op() == TOP_G2) {
                        const int p0 = static_cast<int>(G.pos(0)), p1 = static_cast<int>(G.pos(1));
                        switch (G.kind()) {
#define MB2_P12(x, y) perm2<x, y, TK_SW12>(a)
#define MB2_P13(x, y) perm2<x, y, TK_SW13>(a)
#define MB2_P23(x, y) perm2<x, y, TK_SW23>(a)
#define MB2_G2(x, y) g2<x, y>(a, md)
                            case TK_SW12: MB2_PAIR_SWITCH(p0, p1, MB2_P12); break;
                            case TK_SW13: MB2_PAIR_SWITCH(p0, p1, MB2_P13); break;
                            case TK_SW23: MB2_PAIR_SWITCH(p0, p1, MB2_P23); break;
                            default: MB2_PAIR_SWITCH(p0, p1, MB2_G2); break;
#undef MB2_P12
#undef MB2_P13
#undef MB2_P23
#undef MB2_G2
                        }
                    } else {  // TOP_DIAG: entry per amplitude (k <= 6)
                        const uint32_t k = G.k();
                        uint32_t et = 0, e0 = 0, e1 = 0, e2 = 0, e3 = 0;
                        for (uint32_t b = 0; b < k; ++b) {
                            const uint32_t bit = 1u << G.pos(b);
                            et |= ((tb & bit) ? 1u : 0u) << b;
                            if (bit == rb[0]) e0 = 1u << b;
                            if (bit == rb[1]) e1 = 1u << b;
                            if (bit == rb[2]) e2 = 1u << b;
                            if (bit == rb[3]) e3 = 1u << b;
                        }
#pragma unroll
                        for (int j = 0; j < kNA; ++j) {
                            const uint32_t e = et | ((j & 1) ? e0 : 0u) | ((j & 2) ? e1 : 0u) | ((j & 4) ? e2 : 0u) |
                                               ((j & 8) ? e3 : 0u);
                            a[j] = cmulf(entry(md, e), a[j]);
                        }
                    }
                }
#pragma unroll
                for (int j = 0; j < kNA; ++j) tile[adr[j]] = a[j];
                __syncthreads();
            } else if (I.op() == TOP_SMEM) {
                const uint32_t k = I.k(), dim = 1u << k;
                uint32_t opm = 0;
                for (uint32_t b = 0; b < k; ++b) opm |= 1u << I.pos(b);
                const double* md = gdata + I.data();
#pragma unroll
                for (int j = 0; j < kNA; ++j) {
                    const uint32_t l = tid | (static_cast<uint32_t>(j) << tbits);
                    uint32_t out = 0;
                    for (uint32_t b = 0; b < k; ++b) out |= ((l >> I.pos(b)) & 1u) << b;
                    const uint32_t gbase = l & ~opm;
                    float2 acc = make_float2(0.f, 0.f);
                    for (uint32_t in = 0; in < dim; ++in) {
                        uint32_t li = gbase;
                        for (uint32_t b = 0; b < k; ++b)
                            if ((in >> b) & 1u) li |= 1u << I.pos(b);
                        acc = cfma(entry(md, out * dim + in), tile[swz8(li)], acc);
                    }
                    a[j] = acc;
                }
                __syncthreads();
#pragma unroll
                for (int j = 0; j < kNA; ++j) tile[cadr[j]] = a[j];
                __syncthreads();
            }
        }
        const uint64_t base = pdep64(t, nmask) | off_lo;
#pragma unroll
        for (int j = 0; j < kNA; ++j) st[base | reg_off(j)] = tile[cadr[j]];
        __syncthreads();
    }
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

int launch_tile_pass_c64(void* amps, uint32_t n, const TilePass& pass, const TileInstr* dev_instrs,
                         const double* dev_sdata, const double* dev_gdata, int sm_count, void* stream) {
    static bool attr_set = false;
    if (!attr_set) {
        cudaFuncSetAttribute(k_tile_pass_c64, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(3 * (size_t{1} << kMaxTileQubitsC64) * sizeof(float2) + kMaxStagedBytes));
        attr_set = true;
    }
    if (pass.m > kMaxTileQubitsC64 || pass.m < kMinTileQubits) return MB2_ERR_INVALID;
    const size_t staged = size_t{pass.prog_count} * sizeof(TileInstr) + size_t{pass.sdata_count} * sizeof(double);
    if (staged > kMaxStagedBytes) return MB2_ERR_INVALID;
    const uint32_t threads = 1u << (pass.m - kRegQubits);
    const uint32_t stages = pass.m == kMaxTileQubitsC64 ? 3u : 2u;
    const size_t smem = stages * (size_t{1} << pass.m) * sizeof(float2) + staged;
    const uint64_t ntiles = (uint64_t{1} << n) >> pass.m;
    const uint64_t cap = static_cast<uint64_t>(sm_count) * (pass.m <= 12 ? 2u : 1u);
    const int grid = static_cast<int>(ntiles < cap ? ntiles : cap);
    k_tile_pass_c64<<<grid, threads, smem, static_cast<cudaStream_t>(stream)>>>(
        static_cast<float2*>(amps), n, pass.m, pass.smask, dev_instrs + pass.prog_begin, pass.prog_count,
        dev_sdata + pass.sdata_begin, pass.sdata_count, dev_gdata, ntiles, stages);
    note_launches(1);
    return launch_status();
}

int launch_scale_c64(void* amps, uint64_t n_amps, float s, void* stream) {
    const uint64_t blocks = (n_amps + 255) / 256;
    k_scale_c64<<<static_cast<unsigned>(blocks < 148ull * 16 ? blocks : 148ull * 16), 256, 0,
                  static_cast<cudaStream_t>(stream)>>>(static_cast<float2*>(amps), n_amps, s);
    note_launches(1);
    return launch_status();
}

}  // namespace mb2
