// Device helpers of the complex64 tile kernels (kernels_c64.cu, the SIMT
// FP32 pass; kernels_tc.cu, the tensor-core pass): complex FP32 arithmetic on
// matrices composed in FP64, diagonal gates on a thread's 16 register
// amplitudes, and cp.async staging.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "mb2_internal.h"

namespace mb2 {
namespace c64 {

constexpr int kR = static_cast<int>(kRegQubits);
constexpr int kNA = 1 << kR;
static_assert(kR == 4, "written for 4 register qubits");

struct Cf {
    float r, i;
};
// Entry e of a matrix staged as FP32 pairs (rounded once from the FP64
// composition when the pass's data is staged), or read from FP64 data.
__device__ __forceinline__ Cf entry(const float* md, uint32_t e) {
    const float2 d = reinterpret_cast<const float2*>(md)[e];
    return Cf{d.x, d.y};
}
__device__ __forceinline__ Cf entry(const double* md, uint32_t e) {
    const double2 d = reinterpret_cast<const double2*>(md)[e];
    return Cf{static_cast<float>(d.x), static_cast<float>(d.y)};
}
// acc + m * x, as two FMA chains.
__device__ __forceinline__ float2 cfma(Cf m, float2 x, float2 acc) {
    return make_float2(fmaf(m.r, x.x, fmaf(-m.i, x.y, acc.x)), fmaf(m.r, x.y, fmaf(m.i, x.x, acc.y)));
}
__device__ __forceinline__ float2 cmulf(Cf m, float2 x) { return cfma(m, x, make_float2(0.f, 0.f)); }
__device__ __forceinline__ float2 fneg_if(float2 v, uint32_t flip) {
    const uint32_t msk = flip << 31;
    return make_float2(__uint_as_float(__float_as_uint(v.x) ^ msk), __uint_as_float(__float_as_uint(v.y) ^ msk));
}

// A diagonal of k <= 2 operands: operand b is register slot P_b (P < 0: a
// thread bit of value v_b).  Entry e multiplies the amplitudes whose operand
// bits spell e; class 0 entries (exactly 1) are skipped.
template <int P0, int P1>
__device__ __forceinline__ void diag_regs(float2 (&a)[kNA], const float* md, uint32_t k, uint32_t cls, uint32_t v0,
                                          uint32_t v1) {
#pragma unroll
    for (uint32_t e = 0; e < 4; ++e) {
        if (e >= (1u << k)) break;
        if (P0 < 0 && (e & 1u) != v0) continue;
        if (P1 < 0 && k > 1 && ((e >> 1) & 1u) != v1) continue;
        const uint32_t c = (cls >> (2 * e)) & 3u;
        if (c == 0u) continue;
        if (c == 1u) {  // -1: sign flips only
#pragma unroll
            for (int j = 0; j < kNA; ++j) {
                if (P0 >= 0 && ((j >> (P0 < 0 ? 0 : P0)) & 1) != static_cast<int>(e & 1u)) continue;
                if (P1 >= 0 && ((j >> (P1 < 0 ? 0 : P1)) & 1) != static_cast<int>((e >> 1) & 1u)) continue;
                a[j] = fneg_if(a[j], 1u);
            }
            continue;
        }
        const Cf d = entry(md, e);
#pragma unroll
        for (int j = 0; j < kNA; ++j) {
            if (P0 >= 0 && ((j >> (P0 < 0 ? 0 : P0)) & 1) != static_cast<int>(e & 1u)) continue;
            if (P1 >= 0 && ((j >> (P1 < 0 ? 0 : P1)) & 1) != static_cast<int>((e >> 1) & 1u)) continue;
            a[j] = cmulf(d, a[j]);
        }
    }
}

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const uint32_t s = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

}  // namespace c64
}  // namespace mb2
