// Device arithmetic shared by the complex128 kernels: complex products and
// sums with every multiply and add rounded on its own (__dmul_rn /
// __dadd_rn / __dsub_rn, never contracted), signed-zero canonicalisation
// and the bit-deposit used to enumerate tiles.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace mb2 {
namespace dev {

__device__ __forceinline__ double2 cmul(double mr, double mi, double2 x) {
    return make_double2(__dsub_rn(__dmul_rn(mr, x.x), __dmul_rn(mi, x.y)),
                        __dadd_rn(__dmul_rn(mr, x.y), __dmul_rn(mi, x.x)));
}
__device__ __forceinline__ double2 cmul_re(double mr, double2 x) {
    return make_double2(__dmul_rn(mr, x.x), __dmul_rn(mr, x.y));
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) {
    return make_double2(__dadd_rn(a.x, b.x), __dadd_rn(a.y, b.y));
}
// -0.0 -> +0.0, everything else unchanged (integer compares on the two
// 32-bit halves, no FP64 issue).
__device__ __forceinline__ double canon1(double v) {
    const int hi = __double2hiint(v), lo = __double2loint(v);
    return __hiloint2double((lo == 0 && hi == static_cast<int>(0x80000000u)) ? 0 : hi, lo);
}
__device__ __forceinline__ double2 canon(double2 v) { return make_double2(canon1(v.x), canon1(v.y)); }
// v negated when flip is 1: the sign bits flipped with an integer XOR (no
// FP64 issue, and exact for every value).
__device__ __forceinline__ double2 cneg_if(double2 v, uint32_t flip) {
    const uint32_t msk = flip << 31;
    int hx = __double2hiint(v.x), hy = __double2hiint(v.y);
    asm("xor.b32 %0, %0, %1;" : "+r"(hx) : "r"(msk));
    asm("xor.b32 %0, %0, %1;" : "+r"(hy) : "r"(msk));
    return make_double2(__hiloint2double(hx, __double2loint(v.x)), __hiloint2double(hy, __double2loint(v.y)));
}
__device__ __forceinline__ double2 cneg(double2 v) { return cneg_if(v, 1u); }
// Negates both parts when msk (0 or 0x80000000) is set.
__device__ __forceinline__ double2 cneg_mask(double2 v, uint32_t msk) {
    return make_double2(__hiloint2double(__double2hiint(v.x) ^ static_cast<int>(msk), __double2loint(v.x)),
                        __hiloint2double(__double2hiint(v.y) ^ static_cast<int>(msk), __double2loint(v.y)));
}
// d * a for one diagonal / monomial entry, exact up to a zero's sign:
// (1, 0) -> a, (-1, 0) -> -a, else the full product.
__device__ __forceinline__ double2 scale_entry(double dr, double di, double2 a) {
    if (di == 0.0) {
        if (dr == 1.0) return a;
        if (dr == -1.0) return cneg(a);
    }
    return cmul(dr, di, a);
}

__device__ __forceinline__ uint64_t insert_zero(uint64_t i, uint32_t pos) {
    const uint64_t low = (uint64_t{1} << pos) - 1;
    return ((i & ~low) << 1) | (i & low);
}

// Scatters the low bits of v onto the set bits of mask (ascending).
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

}  // namespace dev
}  // namespace mb2
