// The multi-gate tile pass of the plain complex128 path: the kernel template
// and its launcher, instantiated in kernels_tile_*.cu (one file per tile
// width, so the instances compile in parallel).
//
// Bitwise contract: as the per-gate kernels (kernels_apply.cu); every
// amplitude sees the blocks of the pass in plan order, each applied with the
// reference kernel's operation order.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "device_math.cuh"
#include "mb2_internal.h"

namespace mb2 {
namespace tile {
using namespace dev;

// ---------------------------------------------------------------- tile pass
// Tile slots are swizzled by swz (mb2_internal.h).

constexpr int kR = static_cast<int>(kRegQubits);  // register qubits per thread
constexpr int kNA = 1 << kR;                         // amplitudes per thread
static_assert(kR == 4, "the register-slot dispatch below is written for 4 register qubits");

// Index of the lowest set bit of a (compile-time) register index j > 0.
__host__ __device__ constexpr int lowbit_index(int j) { return (j & 1) ? 0 : (j & 2) ? 1 : (j & 4) ? 2 : 3; }

template <int P, int KIND>
__device__ __forceinline__ void g1(double2 (&a)[kNA], const double* md, uint32_t aux) {
    const double2 e0 = reinterpret_cast<const double2*>(md)[0], e1 = reinterpret_cast<const double2*>(md)[1];
    const double2 e2 = reinterpret_cast<const double2*>(md)[2], e3 = reinterpret_cast<const double2*>(md)[3];
    const double m00r = e0.x, m00i = e0.y, m01r = e1.x, m01i = e1.y;
    const double m10r = e2.x, m10i = e2.y, m11r = e3.x, m11i = e3.y;
#pragma unroll
    for (int j = 0; j < kNA; ++j) {
        if (j & (1 << P)) continue;
        const double2 x = a[j];
        const double2 y = a[j | (1 << P)];
        double2 o0, o1;
        if (KIND == TK_GEN) {
            o0 = cadd(cmul(m00r, m00i, x), cmul(m01r, m01i, y));
            o1 = cadd(cmul(m10r, m10i, x), cmul(m11r, m11i, y));
        } else if (KIND == TK_U3) {
            o0 = cadd(cmul_re(m00r, x), cmul(m01r, m01i, y));
            o1 = cadd(cmul(m10r, m10i, x), cmul(m11r, m11i, y));
        } else if (KIND == TK_REAL) {
            o0 = cadd(cmul_re(m00r, x), cmul_re(m01r, y));
            o1 = cadd(cmul_re(m10r, x), cmul_re(m11r, y));
        } else {  // TK_MONO: row r takes entry (r, src_r) of column src_r, or is zero
            const uint32_t s0 = aux & 7u, s1 = (aux >> 3) & 7u;
            o0 = s0 == 7u ? make_double2(0.0, 0.0)
                          : scale_entry(s0 ? m01r : m00r, s0 ? m01i : m00i, s0 ? y : x);
            o1 = s1 == 7u ? make_double2(0.0, 0.0)
                          : scale_entry(s1 ? m11r : m10r, s1 ? m11i : m10i, s1 ? y : x);
        }
        a[j] = o0;
        a[j | (1 << P)] = o1;
    }
}

template <int P0, int P1, int KIND>
__device__ __forceinline__ void g2(double2 (&a)[kNA], const double* md, uint32_t aux) {
    if constexpr (P0 == P1) {
        return;
    } else {
#pragma unroll
        for (int j = 0; j < kNA; ++j) {
            if (j & ((1 << P0) | (1 << P1))) continue;
            const int idx[4] = {j, j | (1 << P0), j | (1 << P1), j | (1 << P0) | (1 << P1)};
            const double2 in[4] = {a[idx[0]], a[idx[1]], a[idx[2]], a[idx[3]]};
            double2 out[4];
#pragma unroll
            for (int o = 0; o < 4; ++o) {
                if (KIND == TK_MONO) {
                    const uint32_t s = (aux >> (3 * o)) & 7u;
                    if (s == 7u) {
                        out[o] = make_double2(0.0, 0.0);
                    } else {
                        const double2 src = s == 0 ? in[0] : s == 1 ? in[1] : s == 2 ? in[2] : in[3];
                        out[o] = scale_entry(md[8 * o + 2 * s], md[8 * o + 2 * s + 1], src);
                    }
                } else {
                    // Row o is read from shared memory where it is used: the
                    // empty asm with a memory clobber keeps the compiler from
                    // holding all 32 entries in registers across the groups,
                    // which would set the register count of the whole kernel.
                    asm volatile("" ::: "memory");
                    double2 acc = cmul(md[8 * o], md[8 * o + 1], in[0]);
#pragma unroll
                    for (int i = 1; i < 4; ++i) acc = cadd(acc, cmul(md[8 * o + 2 * i], md[8 * o + 2 * i + 1], in[i]));
                    out[o] = acc;
                }
            }
#pragma unroll
            for (int o = 0; o < 4; ++o) a[idx[o]] = out[o];
        }
    }
}

// A diagonal block of k <= 2 qubits in registers.  Each operand is either
// a register slot (its bit over j is known at compile time in the templates
// below) or a thread bit (one value for all 16 amplitudes).  The entry of
// amplitude j is e = bit0 | bit1 << 1; its class (aux, 2 bits per entry:
// 0 copy, 1 negate, 2 multiply) is resolved once per gate or per thread, and
// each class runs its own loop, so an amplitude costs nothing (copy), two
// integer ops (negate) or one complex product (multiply).
struct Diag4 {
    double2 d[4];
    uint32_t aux;
};

// The entries of a k <= 2 diagonal (k = 1: entries 2 and 3 repeat 0 and 1,
// which only the k = 1 paths' selectors never reach) with its classes.
__device__ __forceinline__ Diag4 load_diag(const double* md, uint32_t k, uint32_t aux) {
    Diag4 D;
    D.aux = aux;
    D.d[0] = reinterpret_cast<const double2*>(md)[0];
    D.d[1] = reinterpret_cast<const double2*>(md)[1];
    D.d[2] = k > 1 ? reinterpret_cast<const double2*>(md)[2] : D.d[0];
    D.d[3] = k > 1 ? reinterpret_cast<const double2*>(md)[3] : D.d[1];
    return D;
}

__device__ __forceinline__ double2 diag_entry(const Diag4& D, uint32_t e) {
    return (e & 2u) ? ((e & 1u) ? D.d[3] : D.d[2]) : ((e & 1u) ? D.d[1] : D.d[0]);
}

// Applies entry class `cls` with entry d to the amplitudes j whose selector
// bits (j >> P0 & 1, j >> P1 & 1) equal (b0, b1); P < 0 means "no condition".
template <int P0, int P1>
__device__ __forceinline__ void diag_set(double2 (&a)[kNA], uint32_t cls, double2 d, int b0, int b1) {
    if (cls == 1u) {
#pragma unroll
        for (int j = 0; j < kNA; ++j) {
            if (P0 >= 0 && ((j >> (P0 < 0 ? 0 : P0)) & 1) != b0) continue;
            if (P1 >= 0 && ((j >> (P1 < 0 ? 0 : P1)) & 1) != b1) continue;
            a[j] = cneg(a[j]);
        }
    } else if (cls == 2u) {
#pragma unroll
        for (int j = 0; j < kNA; ++j) {
            if (P0 >= 0 && ((j >> (P0 < 0 ? 0 : P0)) & 1) != b0) continue;
            if (P1 >= 0 && ((j >> (P1 < 0 ? 0 : P1)) & 1) != b1) continue;
            a[j] = cmul(d.x, d.y, a[j]);
        }
    }
}

// Both operands in register slots (P1 < 0: one operand).
template <int P0, int P1>
__device__ __forceinline__ void diag_rr(double2 (&a)[kNA], const Diag4& D) {
#pragma unroll
    for (int e = 0; e < (P1 >= 0 ? 4 : 2); ++e)
        diag_set<P0, P1>(a, (D.aux >> (2 * e)) & 3u, D.d[e], e & 1, (e >> 1) & 1);
}

// One operand in register slot P (bit `shift` of e), the other a thread bit tv.
template <int P>
__device__ __forceinline__ void diag_rt(double2 (&a)[kNA], const Diag4& D, uint32_t shift, uint32_t tv) {
#pragma unroll
    for (int b = 0; b < 2; ++b) {
        const uint32_t e = (static_cast<uint32_t>(b) << shift) | (tv << (1u - shift));
        diag_set<P, -1>(a, (D.aux >> (2 * e)) & 3u, diag_entry(D, e), b, 0);
    }
}

// A dense two-qubit block in registers, compiled only into the FULL variant.
template <int P0, int P1, bool FULL>
__device__ __forceinline__ void gen2_if(double2 (&a)[kNA], const double* md) {
    if constexpr (FULL) g2<P0, P1, TK_GEN>(a, md, 0u);
}

// Exact permutations (every nonzero entry (1,0)): register moves only.
// TK_X: 1q swap; TK_SW12 / TK_SW13 / TK_SW23: 2q, exchange local indices
// (1,2) (SWAP), (1,3) (CX, control = operand 0), (2,3) (CX, control = operand 1).
template <int P0, int P1, int KIND>
__device__ __forceinline__ void perm2(double2 (&a)[kNA]) {
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
            const double2 t = a[il];
            a[il] = a[ih];
            a[ih] = t;
        }
    }
}

// cp.async of one 16-byte amplitude, global -> shared (L2 only, no L1).
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const uint32_t s = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// The instructions of one pass applied to one tile held in shared memory
// (canonical layout on entry and exit).  `sync` is the barrier of the
// threads that share the tile; parametric data sits pshift doubles past the
// staged data's end.  FULL = false compiles out every instruction that moves
// amplitudes between registers or selects them at run time (permutations,
// monomial rows) and the rare heavy ones (dense two-qubit blocks, wide
// diagonals, shared-memory blocks): measured per U3, their presence in the
// same switch costs ~60-85 extra register moves on every gate path (the
// allocator's layout at the merge).  The launcher picks the lean variant for
// passes without them (the encoder writes single-qubit X and monomial gates
// as general 2x2 products, exact up to zero signs).
template <int MT, bool FULL, typename SYNC>
__device__ __forceinline__ void compute_tile(double2* __restrict__ tile, const uint32_t* __restrict__ sw,
                                             uint32_t nwords, const double* __restrict__ sd, uint32_t nsdata,
                                             uint32_t pshift, const double* __restrict__ gdata, uint32_t tid,
                                             uint32_t m, uint32_t gbits, SYNC sync) {
    const uint32_t tbits = m - kRegQubits;
    const uint32_t s_tid = swz(tid);
    auto slot = [&](int j) -> uint32_t { return s_tid ^ swz(static_cast<uint32_t>(j) << tbits); };
    double2 a[kNA];
    uint32_t pc = 0;
    while (pc < nwords) {
        const uint32_t w0 = sw[pc];
        const uint32_t op0 = w0 & 0xffu;
        if (op0 == cop::kPhase) {
            // The phase record (cop::kPhase): this thread's tile bits from
            // the nibble table, the register bits' slot byte offsets as words.
            const uint32_t* rec = sw + pc;
            pc += cop::kPhaseWords;
            const uint16_t* et = reinterpret_cast<const uint16_t*>(rec + 5);
            uint32_t tb = static_cast<uint32_t>(et[tid & 15u]) | static_cast<uint32_t>(et[16 + ((tid >> 4) & 15u)]);
            if (MT == 0 || MT > 12) tb |= static_cast<uint32_t>(et[32 + ((tid >> 8) & 15u)]);
            uint32_t rb[kR];
#pragma unroll
            for (int b = 0; b < kR; ++b) rb[b] = 1u << ((w0 >> (16 + 4 * b)) & 15u);
            // swz is linear over XOR, so slot j's byte offset is swz(tb)'s
            // XOR the register bits' of j (recomputed for the write-back
            // rather than held in 16 registers through the gates).
            const uint32_t z0 = swz(tb) << 4, z1 = rec[1] & 0xffffu, z2 = rec[1] >> 16, z3 = rec[2] & 0xffffu,
                           z4 = rec[2] >> 16;
            // Operand bit values from here on: the tile bits, and from
            // position kGlobalPos0 the tile's bits of the qubits outside it.
            tb |= gbits;
            char* const tile_b = reinterpret_cast<char*>(tile);
            auto at = [&](int j) -> double2& {
                return *reinterpret_cast<double2*>(
                    tile_b + (z0 ^ ((j & 1) ? z1 : 0u) ^ ((j & 2) ? z2 : 0u) ^ ((j & 4) ? z3 : 0u) ^ ((j & 8) ? z4 : 0u)));
            };
#pragma unroll
            for (int j = 0; j < kNA; ++j) a[j] = at(j);
            for (;;) {
                const uint32_t w = sw[pc++];
                const uint32_t op = w & 0xffu;
                if (op == cop::kEnd) break;
                const uint32_t aux = (w >> 8) & 0xffu;
                const uint32_t off = ((w >> 20) & 0x7ffu) << 1;
                const double* md = sd + off + (off >= nsdata ? pshift : 0u);
                // The bit-value operand's value (position: bits 16-19, 31).
                const uint32_t tv = (tb >> (((w >> 16) & 15u) | ((w >> 27) & 16u))) & 1u;
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
                    MB2_CASE4(cop::kU3, (g1<P, TK_U3>(a, md, 0u)))
                    MB2_CASE4(cop::kGen1, (g1<P, TK_GEN>(a, md, 0u)))
                    MB2_CASE4(cop::kReal1, (g1<P, TK_REAL>(a, md, 0u)))
                    MB2_CASE12(cop::kGen2, (gen2_if<P0, P1, FULL>(a, md)))
                    MB2_CASE12(cop::kMono2, if constexpr (FULL) g2<P0, P1, TK_MONO>(a, md, sw[pc++]))
                    MB2_CASE12(cop::kSw12, if constexpr (FULL) perm2<P0, P1, TK_SW12>(a))
                    MB2_CASE12(cop::kSw13, if constexpr (FULL) perm2<P0, P1, TK_SW13>(a))
                    MB2_CASE12(cop::kSw23, if constexpr (FULL) perm2<P0, P1, TK_SW23>(a))
                    case cop::kU3Run0123:
                        g1<0, TK_U3>(a, md, 0u);
                        g1<1, TK_U3>(a, md + 8, 0u);
                        g1<2, TK_U3>(a, md + 16, 0u);
                        g1<3, TK_U3>(a, md + 24, 0u);
                        break;
                    case cop::kU3Run01:
                        g1<0, TK_U3>(a, md, 0u);
                        g1<1, TK_U3>(a, md + 8, 0u);
                        break;
                    case cop::kU3Run123:
                        g1<1, TK_U3>(a, md, 0u);
                        g1<2, TK_U3>(a, md + 8, 0u);
                        g1<3, TK_U3>(a, md + 16, 0u);
                        break;
                    case cop::kU3Run012:
                        g1<0, TK_U3>(a, md, 0u);
                        g1<1, TK_U3>(a, md + 8, 0u);
                        g1<2, TK_U3>(a, md + 16, 0u);
                        break;
                    MB2_CASE4(cop::kDs1R, (diag_rr<P, -1>(a, load_diag(md, 1, aux))))
                    MB2_CASE12(cop::kDs2RR, (diag_rr<P0, P1>(a, load_diag(md, 2, aux))))
#undef MB2_CASE4
#undef MB2_CASE12
                    case cop::kDs1T: {
                        const Diag4 D = load_diag(md, 1, aux);
                        diag_set<-1, -1>(a, (aux >> (2 * tv)) & 3u, diag_entry(D, tv), 0, 0);
                    } break;
                    // One register operand (slot s) and one thread bit (operand index wi).
                    case cop::kDs2RT + 0: diag_rt<0>(a, load_diag(md, 2, aux), 1u, tv); break;
                    case cop::kDs2RT + 1: diag_rt<0>(a, load_diag(md, 2, aux), 0u, tv); break;
                    case cop::kDs2RT + 2: diag_rt<1>(a, load_diag(md, 2, aux), 1u, tv); break;
                    case cop::kDs2RT + 3: diag_rt<1>(a, load_diag(md, 2, aux), 0u, tv); break;
                    case cop::kDs2RT + 4: diag_rt<2>(a, load_diag(md, 2, aux), 1u, tv); break;
                    case cop::kDs2RT + 5: diag_rt<2>(a, load_diag(md, 2, aux), 0u, tv); break;
                    case cop::kDs2RT + 6: diag_rt<3>(a, load_diag(md, 2, aux), 1u, tv); break;
                    case cop::kDs2RT + 7: diag_rt<3>(a, load_diag(md, 2, aux), 0u, tv); break;
                    case cop::kDs2TT: {
                        const uint32_t cc = sw[pc++];
                        const uint32_t e = ((tb >> ((cc & 15u) | ((cc >> 4) & 16u))) & 1u) |
                                           (((tb >> (((cc >> 4) & 15u) | ((cc >> 5) & 16u))) & 1u) << 1);
                        const Diag4 D = load_diag(md, 2, aux);
                        diag_set<-1, -1>(a, (aux >> (2 * e)) & 3u, diag_entry(D, e), 0, 0);
                    } break;
                    case cop::kSigns: {
                        // XOR of the monomials' masks over the 16 register slots j.
                        uint32_t M = 0;
                        for (uint32_t i = 0; i < aux; ++i) {
                            const uint32_t mono = sw[pc++];
                            const uint32_t tm = mono >> 16;
                            M ^= (tb & tm) == tm ? (mono & 0xffffu) : 0u;
                        }
#pragma unroll
                        for (int j = 0; j < kNA; ++j) a[j] = cneg_mask(a[j], (M << (31 - j)) & 0x80000000u);
                    } break;
                    case cop::kSignsW: {
                        uint32_t M = 0;
                        for (uint32_t i = 0; i < aux; ++i) {
                            const uint32_t slots = sw[pc], bits = sw[pc + 1];
                            pc += 2;
                            M ^= (tb & bits) == bits ? slots : 0u;
                        }
#pragma unroll
                        for (int j = 0; j < kNA; ++j) a[j] = cneg_mask(a[j], (M << (31 - j)) & 0x80000000u);
                    } break;
                    default: {  // cop::kDiagK: any k, entry index per amplitude
                        if constexpr (!FULL) break;
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
                            a[j] = scale_entry(md[2 * e], md[2 * e + 1], a[j]);
                        }
                    } break;
                }
            }
#pragma unroll
            for (int j = 0; j < kNA; ++j) at(j) = a[j];
            sync();
        } else if (FULL && op0 == cop::kSmem) {
            // A dense k-qubit block (k >= 3) on the whole tile in shared memory.
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
                double2 acc = make_double2(0.0, 0.0);
                for (uint32_t in = 0; in < dim; ++in) {
                    uint32_t li = gbase;
                    for (uint32_t b = 0; b < k; ++b)
                        if ((in >> b) & 1u) li |= 1u << qpos(b);
                    const double2 p = cmul(__ldg(md + 2 * (out * dim + in)), __ldg(md + 2 * (out * dim + in) + 1),
                                           tile[swz(li)]);
                    acc = (in == 0) ? p : cadd(acc, p);
                }
                a[j] = acc;
            }
            sync();
#pragma unroll
            for (int j = 0; j < kNA; ++j) tile[slot(j)] = a[j];
            sync();
        } else {
            break;  // padding after the last instruction
        }
    }
}

// One pass of the tiled sweep.  blockDim.x == 2^(m-4) <= 256; each thread
// owns 16 amplitudes.  Persistent CTAs take tiles round-robin; the tiles
// `stages - 1` ahead are gathered into shared-memory buffers with cp.async
// while the current one is computed, so HBM traffic overlaps the FP64 work.
// The pass's instructions and small-matrix data are staged in shared memory
// once per CTA.
//
// MT > 0 fixes the tile width at compile time (shared-memory slots of the
// canonical mapping become constants); IDX is the amplitude-index type,
// 32-bit when the state (all bindings included) has at most 2^32
// amplitudes.  A tile's base index is its number deposited on the bits
// outside the tile (nmask); moving gridDim.x tiles on is the masked add
// ((base | ~nmask) + step) & nmask, step = deposit(gridDim.x).
// The pass over this CTA's share of the tiles: tiles cta, cta + nctas, ...
template <int MT, typename IDX, bool FULL>
__device__ __forceinline__ void tile_pass_body(double2* __restrict__ st, uint32_t n, uint32_t m_rt, uint64_t smask,
                                               uint64_t gmask, const uint32_t* __restrict__ words, uint32_t nwords,
                                               const double* __restrict__ sdata, uint32_t nsdata,
                                               const double* __restrict__ gdata, uint64_t ntiles,
                                               const double* __restrict__ pdata, uint32_t pstride, uint32_t param_lo,
                                               uint32_t param_len, uint32_t bshift, uint32_t stages, uint32_t cta,
                                               uint32_t nctas) {
    extern __shared__ double2 smem_tiles[];
    const uint32_t m = MT > 0 ? static_cast<uint32_t>(MT) : m_rt;
    const uint32_t tid = threadIdx.x;
    const uint32_t tbits = m - kRegQubits;
    const uint32_t tile_amps = 1u << m;
    // Shared memory: tile buffers, the pass's words (a multiple of four),
    // its staged data, then the parametric slice of the current tile's binding.
    uint32_t* sw = reinterpret_cast<uint32_t*>(smem_tiles + stages * tile_amps);
    double* sd = reinterpret_cast<double*>(sw + nwords);
    for (uint32_t i = tid; i < nwords / 4; i += blockDim.x)
        reinterpret_cast<uint4*>(sw)[i] = __ldg(reinterpret_cast<const uint4*>(words) + i);
    for (uint32_t i = tid; i < nsdata; i += blockDim.x) sd[i] = __ldg(sdata + i);
    // Canonical (load/store) mapping: thread bits = tile bits 0..tbits-1,
    // register bits = tile bits tbits..m-1.
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
    const IDX step = static_cast<IDX>(pdep64(nctas, nmask64));
    auto advance = [&](IDX b) -> IDX { return ((b | ~nmask) + step) & nmask; };
    // Amplitude (tid, j) of the canonical mapping: global index base +
    // off_lo + the register bits of j (disjoint bit sets, so + is |);
    // shared-memory slot swz(tid) ^ swz(j << tbits) (swz is XOR-linear).
    const uint32_t s_tid = swz(tid);
    auto reg_off = [&](int j) -> IDX {
        return ((j & 1) ? hib0 : IDX{0}) + ((j & 2) ? hib1 : IDX{0}) + ((j & 4) ? hib2 : IDX{0}) +
               ((j & 8) ? hib3 : IDX{0});
    };
    auto slot = [&](int j) -> uint32_t { return s_tid ^ swz(static_cast<uint32_t>(j) << tbits); };
    auto prefetch = [&](IDX base, double2* buf) {
        const IDX b0 = base + off_lo;
#pragma unroll
        for (int j = 0; j < kNA; ++j) cp_async16(buf + slot(j), st + (b0 + reg_off(j)));
        cp_async_commit();
    };

    // `stages` tile buffers: the tiles `stages - 1` ahead are in flight
    // while this one is computed (one commit group per tile, empty groups
    // past the end keep the count uniform).
    uint64_t tp = cta;  // next tile to prefetch
    IDX pbase = static_cast<IDX>(pdep64(cta, nmask64));
    IDX cbase = pbase;  // base of the tile being computed
    for (uint32_t sg = 0; sg + 1 < stages; ++sg) {
        if (tp < ntiles) prefetch(pbase, smem_tiles + sg * tile_amps);
        else cp_async_commit();
        tp += nctas;
        pbase = advance(pbase);
    }
    uint32_t cur = 0, nxt = stages - 1;  // buffer of this tile, of the next prefetch
    for (uint64_t t = cta; t < ntiles; t += nctas) {
        double2* tile = smem_tiles + cur * tile_amps;
        if (tp < ntiles) prefetch(pbase, smem_tiles + nxt * tile_amps);
        else cp_async_commit();
        tp += nctas;
        pbase = advance(pbase);
        cur = cur + 1 == stages ? 0u : cur + 1;
        nxt = nxt + 1 == stages ? 0u : nxt + 1;
        if (param_len != 0) {  // a batched sweep: this tile's binding is t >> bshift
            const double2* src = reinterpret_cast<const double2*>(pdata + (t >> bshift) * pstride + param_lo);
            double2* dst = reinterpret_cast<double2*>(sd + nsdata);
            for (uint32_t i = tid; i < param_len / 2; i += blockDim.x) dst[i] = __ldg(src + i);
        }
        if (stages == 3) cp_async_wait<2>();
        else cp_async_wait<1>();
        __syncthreads();

        // The tile's bits of the qubits outside it that diagonals read, at
        // positions kGlobalPos0 + rank.
        uint32_t gbits = 0;
        {
            uint32_t r = kGlobalPos0;
            for (uint64_t g = gmask; g != 0; g &= g - 1, ++r)
                gbits |= static_cast<uint32_t>((static_cast<uint64_t>(cbase) >> (__ffsll(static_cast<long long>(g)) - 1)) & 1u) << r;
        }
        compute_tile<MT, FULL>(tile, sw, nwords, sd, nsdata, 0u, gdata, tid, m, gbits, [] { __syncthreads(); });

        // Store: canonical mapping, -0.0 normalised.
        const IDX b0 = cbase + off_lo;
#pragma unroll
        for (int j = 0; j < kNA; ++j) st[b0 + reg_off(j)] = canon(tile[slot(j)]);
        cbase = advance(cbase);
        __syncthreads();  // the buffer is the target of a later prefetch
    }
}

template <int MAXT, int MINB, int MT, typename IDX, bool FULL>
__global__ void __launch_bounds__(MAXT, MINB)
    k_tile_pass(double2* __restrict__ st, uint32_t n, uint32_t m_rt, uint64_t smask, uint64_t gmask,
                const uint32_t* __restrict__ words, uint32_t nwords, const double* __restrict__ sdata,
                uint32_t nsdata, const double* __restrict__ gdata, uint64_t ntiles, const double* __restrict__ pdata,
                uint32_t pstride, uint32_t param_lo, uint32_t param_len, uint32_t bshift, uint32_t stages) {
    tile_pass_body<MT, IDX, FULL>(st, n, m_rt, smask, gmask, words, nwords, sdata, nsdata, gdata, ntiles, pdata,
                                  pstride, param_lo, param_len, bshift, stages, blockIdx.x, gridDim.x);
}

// Many states' passes in one launch (small states, one tile width): CTAs
// [jobs[j].cta_begin, jobs[j + 1].cta_begin) run job j's pass over its state.
template <int MAXT, int MT, bool FULL>
__global__ void __launch_bounds__(MAXT, 1) k_tile_pass_jobs(const TileJob* __restrict__ jobs, uint32_t njobs,
                                                           uint32_t m_rt) {
    uint32_t lo = 0, hi = njobs;  // the last job whose cta_begin <= blockIdx.x
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (jobs[mid].cta_begin <= blockIdx.x) lo = mid;
        else hi = mid;
    }
    const TileJob& J = jobs[lo];
    tile_pass_body<MT, uint64_t, FULL>(static_cast<double2*>(J.st), J.n, m_rt, J.smask, J.gmask, J.words, J.nwords, J.sdata, J.nsdata,
                                       J.gdata, J.ntiles, nullptr, 0, 0, 0, 0, 2, blockIdx.x - J.cta_begin,
                                       J.nctas);
}

// Launches one instance; the shared-memory limit is raised once per instance.
template <int MAXT, int MINB, int MT, typename IDX, bool FULL>
int launch_instance(const TileLaunch& L) {
    // The dynamic limit is what the static shared memory leaves of the
    // per-block maximum; it is raised once, by whichever thread launches
    // first (the serving loop's workers launch concurrently: the static's
    // initialisation is thread-safe and every thread sees it complete).
    static const size_t dyn_max = [] {
        cudaFuncAttributes fa{};
        if (cudaFuncGetAttributes(&fa, k_tile_pass<MAXT, MINB, MT, IDX, FULL>) != cudaSuccess) return size_t{0};
        const size_t v = kTileSmemMax - fa.sharedSizeBytes;
        if (cudaFuncSetAttribute(k_tile_pass<MAXT, MINB, MT, IDX, FULL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(v)) != cudaSuccess)
            return size_t{0};
        return v;
    }();
    if (dyn_max == 0) return launch_status();
    if (L.smem > dyn_max) return MB2_ERR_INVALID;
    k_tile_pass<MAXT, MINB, MT, IDX, FULL><<<L.grid, L.threads, L.smem, static_cast<cudaStream_t>(L.stream)>>>(
        static_cast<double2*>(L.amps), L.n_all, L.m, L.smask, L.gmask, L.words, L.nwords, L.sdata, L.nsdata, L.gdata,
        L.ntiles, L.pdata, L.pstride, L.param_lo, L.param_len, L.bshift, L.stages);
    return launch_status();
}

}  // namespace tile
}  // namespace mb2
