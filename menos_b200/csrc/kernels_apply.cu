// sm_100a gate kernels of the plain complex128 path.
//
// Bitwise contract (the reference's generic kernel,
// src/kernels/cpu/dense_kernels.cpp:465-524): each output amplitude is
//     (+0) + m[out][0]*a[0] + m[out][1]*a[1] + ...   (increasing `in`)
// with the product (mr*ar - mi*ai, mr*ai + mi*ar), every multiply and add
// rounded on its own (built with -fmad=false and written with __dmul_rn /
// __dadd_rn / __dsub_rn, which are never contracted).  Two rewrites keep the
// result identical and save FP64 issue slots:
//   * the leading "(+0) +" only turns a -0.0 into +0.0, and the sign of a
//     zero never changes a later non-zero sum, so it is dropped inside the
//     arithmetic and applied once, as canon(), where an amplitude is stored;
//   * a product term whose matrix entry is exactly zero (either sign) is a
//     signed zero and changes nothing but a zero's sign, so it is skipped;
//     an entry with zero imaginary part contributes (mr*ar, mr*ai).
// Both hold for finite amplitudes, the reference kernels' own precondition
// (src/kernels/dense_kernels.h:105-124).
#include <cuda_runtime.h>

#include <cstdint>

#include "mb2_internal.h"

namespace mb2 {
namespace {

// ---------------------------------------------------------------- arithmetic
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
// -0.0 -> +0.0, everything else unchanged (integer compare, no FP64 issue).
__device__ __forceinline__ double canon1(double v) {
    const long long b = __double_as_longlong(v);
    return __longlong_as_double(b == static_cast<long long>(0x8000000000000000ULL) ? 0LL : b);
}
__device__ __forceinline__ double2 canon(double2 v) { return make_double2(canon1(v.x), canon1(v.y)); }
__device__ __forceinline__ double2 cneg(double2 v) {
    return make_double2(__longlong_as_double(__double_as_longlong(v.x) ^ static_cast<long long>(0x8000000000000000ULL)),
                        __longlong_as_double(__double_as_longlong(v.y) ^ static_cast<long long>(0x8000000000000000ULL)));
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

// ---------------------------------------------------------------- init
__global__ void k_init_c128(double2* st, uint64_t n_amps, double re, double im) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n_amps; i += stride)
        st[i] = (i == 0) ? make_double2(re, im) : make_double2(0.0, 0.0);
}
__global__ void k_init_c64(float2* st, uint64_t n_amps, float re, float im) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n_amps; i += stride)
        st[i] = (i == 0) ? make_float2(re, im) : make_float2(0.0f, 0.0f);
}

// ---------------------------------------------------------------- per-gate kernels
struct M8 {
    double v[8];
};
struct M32 {
    double v[32];
};
struct D128 {
    double v[128];
};

// One pair (i0, i0 | 2^q) per thread iteration: the reference's 1-qubit
// contract (dense_kernels.cpp:227-273).
__global__ void __launch_bounds__(256) k_apply_1q(double2* __restrict__ st, uint64_t npairs, uint32_t q, M8 m) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    const uint64_t bit = uint64_t{1} << q;
    for (uint64_t p = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; p < npairs; p += stride) {
        const uint64_t i0 = insert_zero(p, q);
        const double2 a0 = st[i0];
        const double2 a1 = st[i0 | bit];
        st[i0] = canon(cadd(cmul(m.v[0], m.v[1], a0), cmul(m.v[2], m.v[3], a1)));
        st[i0 | bit] = canon(cadd(cmul(m.v[4], m.v[5], a0), cmul(m.v[6], m.v[7], a1)));
    }
}

// One group of four per thread iteration; local bit j = operand j
// (dense_kernels.cpp:275-297).
__global__ void __launch_bounds__(256) k_apply_2q(double2* __restrict__ st, uint64_t ngroups, uint32_t q0,
                                                  uint32_t q1, M32 m) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    const uint32_t lo = q0 < q1 ? q0 : q1;
    const uint32_t hi = q0 < q1 ? q1 : q0;
    const uint64_t b0 = uint64_t{1} << q0, b1 = uint64_t{1} << q1;
    for (uint64_t g = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < ngroups; g += stride) {
        const uint64_t base = insert_zero(insert_zero(g, lo), hi);
        const uint64_t idx[4] = {base, base | b0, base | b1, base | b0 | b1};
        double2 a[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) a[i] = st[idx[i]];
#pragma unroll
        for (int o = 0; o < 4; ++o) {
            double2 s = cmul(m.v[8 * o], m.v[8 * o + 1], a[0]);
#pragma unroll
            for (int i = 1; i < 4; ++i) s = cadd(s, cmul(m.v[8 * o + 2 * i], m.v[8 * o + 2 * i + 1], a[i]));
            st[idx[o]] = canon(s);
        }
    }
}

// Diagonal matrices: each amplitude times its entry (dense_kernels.cpp:299-363).
__global__ void __launch_bounds__(256) k_apply_diag(double2* __restrict__ st, uint64_t n_amps, uint32_t k,
                                                    uint32_t q0, uint32_t q1, uint32_t q2, uint32_t q3,
                                                    uint32_t q4, uint32_t q5, D128 d) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    const uint32_t q[6] = {q0, q1, q2, q3, q4, q5};
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n_amps; i += stride) {
        uint32_t e = 0;
        for (uint32_t j = 0; j < k; ++j) e |= static_cast<uint32_t>((i >> q[j]) & 1u) << j;
        st[i] = canon(scale_entry(d.v[2 * e], d.v[2 * e + 1], st[i]));
    }
}

// The generic k-operand kernel (dense_kernels.cpp:465-524), cooperative per
// CTA: a batch of groups is gathered into shared memory, each thread then
// forms whole outputs (sum over `in` in increasing order) and stores them.
// Dynamic shared memory: the matrix (dim^2) then the batch (kGenBatch amps).
constexpr uint32_t kGenBatch = 1024;
__global__ void __launch_bounds__(256) k_apply_generic(double2* __restrict__ st, uint32_t n, uint32_t k,
                                                       uint32_t q0, uint32_t q1, uint32_t q2, uint32_t q3,
                                                       uint32_t q4, uint32_t q5,
                                                       const double2* __restrict__ matrix) {
    extern __shared__ double2 smem[];
    const uint32_t dim = 1u << k;
    double2* mat = smem;
    double2* buf = smem + dim * dim;
    const uint32_t q[6] = {q0, q1, q2, q3, q4, q5};
    uint64_t opmask = 0;
    for (uint32_t j = 0; j < k; ++j) opmask |= uint64_t{1} << q[j];
    const uint64_t rest = ((n >= 64) ? ~uint64_t{0} : ((uint64_t{1} << n) - 1)) & ~opmask;
    for (uint32_t i = threadIdx.x; i < dim * dim; i += blockDim.x) mat[i] = matrix[i];
    const uint64_t ngroups = (uint64_t{1} << n) >> k;
    const uint32_t per_batch = kGenBatch >> k;  // groups per batch (k <= 6 -> >= 16)
    const uint64_t nbatches = (ngroups + per_batch - 1) / per_batch;
    for (uint64_t bt = blockIdx.x; bt < nbatches; bt += gridDim.x) {
        __syncthreads();
        // gather
        for (uint32_t s = threadIdx.x; s < kGenBatch; s += blockDim.x) {
            const uint64_t g = bt * per_batch + (s >> k);
            if (g >= ngroups) continue;
            const uint32_t local = s & (dim - 1);
            uint64_t idx = pdep64(g, rest);
            for (uint32_t j = 0; j < k; ++j)
                if ((local >> j) & 1u) idx |= uint64_t{1} << q[j];
            buf[s] = st[idx];
        }
        __syncthreads();
        for (uint32_t s = threadIdx.x; s < kGenBatch; s += blockDim.x) {
            const uint64_t g = bt * per_batch + (s >> k);
            if (g >= ngroups) continue;
            const uint32_t out = s & (dim - 1);
            const double2* grp = buf + (s & ~(dim - 1));
            double2 acc = cmul(mat[out * dim].x, mat[out * dim].y, grp[0]);
            for (uint32_t in = 1; in < dim; ++in) acc = cadd(acc, cmul(mat[out * dim + in].x, mat[out * dim + in].y, grp[in]));
            uint64_t idx = pdep64(g, rest);
            for (uint32_t j = 0; j < k; ++j)
                if ((out >> j) & 1u) idx |= uint64_t{1} << q[j];
            st[idx] = canon(acc);
        }
    }
}

// ---------------------------------------------------------------- tile pass
// Shared-memory slot of tile-local index l: the low three bits XOR-folded
// with every higher 3-bit group, so quarter-warps whose eight threads vary
// three tile bits of distinct residue mod 3 hit eight distinct 16-byte bank
// groups.
__device__ __forceinline__ uint32_t swz(uint32_t l) {
    const uint32_t h = l >> 3;
    return l ^ ((h ^ (h >> 3) ^ (h >> 6) ^ (h >> 9)) & 7u);
}

// A TileInstr read as four 64-bit words (fields extracted by shifts, so no
// field is ever indexed dynamically in local memory).  Layout: bytes 0-3 op,
// k, kind, nthread; 4-11 pos[8]; 12-15 data; 16-27 tperm[12]; 28-31 aux.
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

// Reads one instruction from the pass program staged in shared memory
// (a plain load: the program is not in the global address space).
__device__ __forceinline__ DI load_instr(const TileInstr* p) {
    const ulonglong2* s = reinterpret_cast<const ulonglong2*>(p);
    const ulonglong2 a = s[0], b = s[1];
    return DI{a.x, a.y, b.x, b.y};
}

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

template <int KIND>
__device__ __forceinline__ void dispatch_g1(int p, double2 (&a)[kNA], const double* md, uint32_t aux) {
    switch (p) {
        case 0: g1<0, KIND>(a, md, aux); break;
        case 1: g1<1, KIND>(a, md, aux); break;
        case 2: g1<2, KIND>(a, md, aux); break;
        default: g1<3, KIND>(a, md, aux); break;
    }
}

template <int P0, int KIND>
__device__ __forceinline__ void dispatch_g2b(int p1, double2 (&a)[kNA], const double* md, uint32_t aux) {
    switch (p1) {
        case 0: g2<P0, 0, KIND>(a, md, aux); break;
        case 1: g2<P0, 1, KIND>(a, md, aux); break;
        case 2: g2<P0, 2, KIND>(a, md, aux); break;
        default: g2<P0, 3, KIND>(a, md, aux); break;
    }
}

template <int KIND>
__device__ __forceinline__ void dispatch_g2(int p0, int p1, double2 (&a)[kNA], const double* md, uint32_t aux) {
    switch (p0) {
        case 0: dispatch_g2b<0, KIND>(p1, a, md, aux); break;
        case 1: dispatch_g2b<1, KIND>(p1, a, md, aux); break;
        case 2: dispatch_g2b<2, KIND>(p1, a, md, aux); break;
        default: dispatch_g2b<3, KIND>(p1, a, md, aux); break;
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

__device__ __forceinline__ void diag_small(double2 (&a)[kNA], const double* md, uint32_t k, uint32_t aux, int s0,
                                           int s1, uint32_t t0, uint32_t t1) {
    // s0/s1: register slot of operand 0/1, or -1 for a thread bit of value t0/t1.
    Diag4 D;
    D.aux = aux;
    D.d[0] = reinterpret_cast<const double2*>(md)[0];
    D.d[1] = reinterpret_cast<const double2*>(md)[1];
    D.d[2] = k > 1 ? reinterpret_cast<const double2*>(md)[2] : D.d[0];
    D.d[3] = k > 1 ? reinterpret_cast<const double2*>(md)[3] : D.d[1];
    if (k == 1) {
        if (s0 < 0) {
            diag_set<-1, -1>(a, (aux >> (2 * t0)) & 3u, diag_entry(D, t0), 0, 0);
            return;
        }
        switch (s0) {
            case 0: diag_rr<0, -1>(a, D); break;
            case 1: diag_rr<1, -1>(a, D); break;
            case 2: diag_rr<2, -1>(a, D); break;
            default: diag_rr<3, -1>(a, D); break;
        }
        return;
    }
    if (s0 >= 0 && s1 >= 0) {
        switch (s0 * 4 + s1) {
            case 1: diag_rr<0, 1>(a, D); break;
            case 2: diag_rr<0, 2>(a, D); break;
            case 3: diag_rr<0, 3>(a, D); break;
            case 4: diag_rr<1, 0>(a, D); break;
            case 6: diag_rr<1, 2>(a, D); break;
            case 7: diag_rr<1, 3>(a, D); break;
            case 8: diag_rr<2, 0>(a, D); break;
            case 9: diag_rr<2, 1>(a, D); break;
            case 11: diag_rr<2, 3>(a, D); break;
            case 12: diag_rr<3, 0>(a, D); break;
            case 13: diag_rr<3, 1>(a, D); break;
            case 14: diag_rr<3, 2>(a, D); break;
            default: break;
        }
        return;
    }
    if (s0 < 0 && s1 < 0) {
        const uint32_t e = t0 | (t1 << 1);
        diag_set<-1, -1>(a, (aux >> (2 * e)) & 3u, diag_entry(D, e), 0, 0);
        return;
    }
    const int s = s0 >= 0 ? s0 : s1;
    const uint32_t shift = s0 >= 0 ? 0u : 1u;
    const uint32_t tv = s0 >= 0 ? t1 : t0;
    switch (s) {
        case 0: diag_rt<0>(a, D, shift, tv); break;
        case 1: diag_rt<1>(a, D, shift, tv); break;
        case 2: diag_rt<2>(a, D, shift, tv); break;
        default: diag_rt<3>(a, D, shift, tv); break;
    }
}

// Exact permutations (every nonzero entry (1,0)): register moves only.
// TK_X: 1q swap; TK_SW12 / TK_SW13 / TK_SW23: 2q, exchange local indices
// (1,2) (SWAP), (1,3) (CX, control = operand 0), (2,3) (CX, control = operand 1).
template <int P>
__device__ __forceinline__ void perm1(double2 (&a)[kNA]) {
#pragma unroll
    for (int j = 0; j < kNA; ++j) {
        if (j & (1 << P)) continue;
        const double2 t = a[j];
        a[j] = a[j | (1 << P)];
        a[j | (1 << P)] = t;
    }
}

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

template <int KIND>
__device__ __forceinline__ void dispatch_perm2(int p0, int p1, double2 (&a)[kNA]) {
    switch (p0 * 4 + p1) {
        case 1: perm2<0, 1, KIND>(a); break;
        case 2: perm2<0, 2, KIND>(a); break;
        case 3: perm2<0, 3, KIND>(a); break;
        case 4: perm2<1, 0, KIND>(a); break;
        case 6: perm2<1, 2, KIND>(a); break;
        case 7: perm2<1, 3, KIND>(a); break;
        case 8: perm2<2, 0, KIND>(a); break;
        case 9: perm2<2, 1, KIND>(a); break;
        case 11: perm2<2, 3, KIND>(a); break;
        case 12: perm2<3, 0, KIND>(a); break;
        case 13: perm2<3, 1, KIND>(a); break;
        case 14: perm2<3, 2, KIND>(a); break;
        default: break;
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

// One pass of the tiled sweep.  blockDim.x == 2^(m-4) <= 256; each thread
// owns 16 amplitudes.  Persistent CTAs take tiles round-robin; the next
// tile is gathered into the second shared-memory buffer with cp.async while
// the current one is computed, so HBM traffic overlaps the FP64 work.  The
// pass's instructions and small-matrix data are staged in shared memory once
// per CTA.
template <int MAXT, int MINB>
__global__ void __launch_bounds__(MAXT, MINB)
    k_tile_pass(double2* __restrict__ st, uint32_t n, uint32_t m, uint64_t smask, const TileInstr* __restrict__ prog,
                uint32_t nprog, const double* __restrict__ sdata, uint32_t nsdata, const double* __restrict__ gdata,
                uint64_t ntiles, const double* __restrict__ pdata, uint32_t pstride, uint32_t bshift,
                uint32_t stages) {
    extern __shared__ double2 smem_tiles[];
    const uint32_t tid = threadIdx.x;
    const uint32_t tbits = m - kRegQubits;
    const uint32_t tile_amps = 1u << m;
    TileInstr* sprog = reinterpret_cast<TileInstr*>(smem_tiles + stages * tile_amps);
    double* sd = reinterpret_cast<double*>(sprog + nprog);
    for (uint32_t i = tid; i < nprog * 2; i += blockDim.x)
        reinterpret_cast<ulonglong2*>(sprog)[i] = __ldg(reinterpret_cast<const ulonglong2*>(prog) + i);
    for (uint32_t i = tid; i < nsdata; i += blockDim.x) sd[i] = __ldg(sdata + i);
    // Canonical (load/store) mapping: thread bits = tile bits 0..tbits-1,
    // register bits = tile bits tbits..m-1.
    uint64_t off_lo = 0, hib0 = 0, hib1 = 0, hib2 = 0, hib3 = 0;
    {
        uint32_t b = 0;
        for (uint32_t p = 0; p < n; ++p) {
            if (!((smask >> p) & 1u)) continue;
            if (b < tbits) {
                off_lo |= static_cast<uint64_t>((tid >> b) & 1u) << p;
            } else {
                const uint64_t v = uint64_t{1} << p;
                const uint32_t r = b - tbits;
                if (r == 0) hib0 = v;
                else if (r == 1) hib1 = v;
                else if (r == 2) hib2 = v;
                else hib3 = v;
            }
            ++b;
        }
    }
    const uint64_t nmask = ((n >= 64) ? ~uint64_t{0} : ((uint64_t{1} << n) - 1)) & ~smask;
    auto reg_off = [&](int j) -> uint64_t {
        return ((j & 1) ? hib0 : 0) | ((j & 2) ? hib1 : 0) | ((j & 4) ? hib2 : 0) | ((j & 8) ? hib3 : 0);
    };
    auto prefetch = [&](uint64_t t, double2* buf) {
        const uint64_t base = pdep64(t, nmask) | off_lo;
#pragma unroll
        for (int j = 0; j < kNA; ++j)
            cp_async16(buf + swz(tid | (static_cast<uint32_t>(j) << tbits)), st + (base | reg_off(j)));
        cp_async_commit();
    };

    // `stages` tile buffers: the tiles `stages - 1` ahead are in flight
    // while this one is computed (one commit group per tile, empty groups
    // past the end keep the count uniform).
    const uint64_t t0 = blockIdx.x;
    for (uint32_t sg = 0; sg + 1 < stages; ++sg) {
        const uint64_t tp = t0 + static_cast<uint64_t>(sg) * gridDim.x;
        if (tp < ntiles) prefetch(tp, smem_tiles + sg * tile_amps);
        else cp_async_commit();
    }
    uint64_t t = t0;
    for (uint32_t it = 0; t < ntiles; t += gridDim.x, ++it) {
        double2* tile = smem_tiles + (it % stages) * tile_amps;
        const uint64_t tn = t + static_cast<uint64_t>(stages - 1) * gridDim.x;
        if (tn < ntiles) prefetch(tn, smem_tiles + ((it + stages - 1) % stages) * tile_amps);
        else cp_async_commit();
        if (stages == 3) cp_async_wait<2>();
        else cp_async_wait<1>();
        __syncthreads();

        double2 a[kNA];
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
                // swz is linear over XOR, so slot j's address is swz(tb) XOR the
                // swizzled register bits of j.
                uint32_t adr[kNA];
                adr[0] = swz(tb);
#pragma unroll
                for (int j = 1; j < kNA; ++j) adr[j] = adr[j & (j - 1)] ^ swz(rb[lowbit_index(j)]);
#pragma unroll
                for (int j = 0; j < kNA; ++j) a[j] = tile[adr[j]];
                // The next instruction is read while this one executes (every
                // group ends with TOP_END, so the read stays in the program).
                DI G = load_instr(sprog + pc);
                ++pc;
                for (; G.op() != TOP_END; ++pc) {
                    const DI Gn = load_instr(sprog + pc);
                    // Parametric blocks (a batched sweep) read the matrix of
                    // this tile's binding: binding = tile >> bshift.
                    const double* md = G.nthread() ? pdata + (t >> bshift) * pstride + G.data() : sd + G.data();
                    if (G.op() == TOP_G1) {
                        switch (G.kind()) {
                            case TK_GEN: dispatch_g1<TK_GEN>(G.pos(0), a, md, G.aux()); break;
                            case TK_U3: dispatch_g1<TK_U3>(G.pos(0), a, md, G.aux()); break;
                            case TK_REAL: dispatch_g1<TK_REAL>(G.pos(0), a, md, G.aux()); break;
                            case TK_X:
                                switch (G.pos(0)) {
                                    case 0: perm1<0>(a); break;
                                    case 1: perm1<1>(a); break;
                                    case 2: perm1<2>(a); break;
                                    default: perm1<3>(a); break;
                                }
                                break;
                            default: dispatch_g1<TK_MONO>(G.pos(0), a, md, G.aux()); break;
                        }
                    } else if (G.op() == TOP_G2) {
                        switch (G.kind()) {
                            case TK_SW12: dispatch_perm2<TK_SW12>(G.pos(0), G.pos(1), a); break;
                            case TK_SW13: dispatch_perm2<TK_SW13>(G.pos(0), G.pos(1), a); break;
                            case TK_SW23: dispatch_perm2<TK_SW23>(G.pos(0), G.pos(1), a); break;
                            case TK_MONO: dispatch_g2<TK_MONO>(G.pos(0), G.pos(1), a, md, G.aux()); break;
                            default: dispatch_g2<TK_GEN>(G.pos(0), G.pos(1), a, md, G.aux()); break;
                        }
                    } else if (G.kind() == TK_DSMALL) {
                        // Operand sources decided on the host: 0x80 | slot, or a thread bit.
                        const uint32_t c0 = G.pos(4), c1 = G.pos(5);
                        const int s0 = (c0 & 0x80u) ? static_cast<int>(c0 & 3u) : -1;
                        const int s1 = (c1 & 0x80u) ? static_cast<int>(c1 & 3u) : -1;
                        const uint32_t t0 = (c0 & 0x80u) ? 0u : (tb >> c0) & 1u;
                        const uint32_t t1 = (c1 & 0x80u) ? 0u : (tb >> c1) & 1u;
                        diag_small(a, md, G.k(), G.aux(), s0, s1, t0, t1);
                    } else {  // TOP_DIAG, any k: entry index per amplitude
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
                            a[j] = scale_entry(md[2 * e], md[2 * e + 1], a[j]);
                        }
                    }
                    G = Gn;
                }
#pragma unroll
                for (int j = 0; j < kNA; ++j) tile[adr[j]] = a[j];
                __syncthreads();
            } else if (I.op() == TOP_SMEM) {
                // A dense k-qubit block (k >= 3) on the whole tile in shared memory.
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
                    double2 acc = make_double2(0.0, 0.0);
                    for (uint32_t in = 0; in < dim; ++in) {
                        uint32_t li = gbase;
                        for (uint32_t b = 0; b < k; ++b)
                            if ((in >> b) & 1u) li |= 1u << I.pos(b);
                        const double2 p = cmul(__ldg(md + 2 * (out * dim + in)), __ldg(md + 2 * (out * dim + in) + 1),
                                               tile[swz(li)]);
                        acc = (in == 0) ? p : cadd(acc, p);
                    }
                    a[j] = acc;
                }
                __syncthreads();
#pragma unroll
                for (int j = 0; j < kNA; ++j) tile[swz(tid | (static_cast<uint32_t>(j) << tbits))] = a[j];
                __syncthreads();
            }
        }

        // Store: canonical mapping, -0.0 normalised.
        const uint64_t base = pdep64(t, nmask) | off_lo;
#pragma unroll
        for (int j = 0; j < kNA; ++j)
            st[base | reg_off(j)] = canon(tile[swz(tid | (static_cast<uint32_t>(j) << tbits))]);
        __syncthreads();  // the buffer is the target of the prefetch two tiles on
    }
}

// Shared memory an SM gives its resident CTAs (228 KiB less the 1 KiB the
// system reserves per CTA is accounted per CTA by the callers).
constexpr size_t kSmemPerSm = 228 * 1024;

int grid_for(uint64_t work, int threads) {
    const uint64_t blocks = (work + threads - 1) / threads;
    return static_cast<int>(blocks < 148ull * 16 ? (blocks == 0 ? 1 : blocks) : 148ull * 16);
}

int status_of(cudaError_t e) { return e == cudaSuccess ? MB2_OK : MB2_ERR_CUDA; }

}  // namespace

int launch_init(void* amps, uint64_t n_amps, int precision, double re, double im, void* stream) {
    const auto s = static_cast<cudaStream_t>(stream);
    if (precision == MB2_C64)
        k_init_c64<<<grid_for(n_amps, 256), 256, 0, s>>>(static_cast<float2*>(amps), n_amps, static_cast<float>(re),
                                                        static_cast<float>(im));
    else
        k_init_c128<<<grid_for(n_amps, 256), 256, 0, s>>>(static_cast<double2*>(amps), n_amps, re, im);
    note_launches(1);
    return status_of(cudaGetLastError());
}

int launch_apply_1q(void* amps, uint32_t n, uint32_t q, const double* m8, void* stream) {
    M8 m;
    for (int i = 0; i < 8; ++i) m.v[i] = m8[i];
    const uint64_t npairs = (uint64_t{1} << n) >> 1;
    k_apply_1q<<<grid_for(npairs, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(static_cast<double2*>(amps),
                                                                                    npairs, q, m);
    note_launches(1);
    return status_of(cudaGetLastError());
}

int launch_apply_2q(void* amps, uint32_t n, uint32_t q0, uint32_t q1, const double* m32, void* stream) {
    M32 m;
    for (int i = 0; i < 32; ++i) m.v[i] = m32[i];
    const uint64_t ng = (uint64_t{1} << n) >> 2;
    k_apply_2q<<<grid_for(ng, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(static_cast<double2*>(amps), ng, q0,
                                                                                q1, m);
    note_launches(1);
    return status_of(cudaGetLastError());
}

int launch_apply_diag(void* amps, uint32_t n, const uint32_t* q, uint32_t k, const double* diag, void* stream) {
    D128 d;
    const uint32_t dim = 1u << k;
    for (uint32_t i = 0; i < 2 * dim; ++i) d.v[i] = diag[i];
    uint32_t qq[6] = {0, 0, 0, 0, 0, 0};
    for (uint32_t j = 0; j < k; ++j) qq[j] = q[j];
    const uint64_t na = uint64_t{1} << n;
    k_apply_diag<<<grid_for(na, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<double2*>(amps), na, k, qq[0], qq[1], qq[2], qq[3], qq[4], qq[5], d);
    note_launches(1);
    return status_of(cudaGetLastError());
}

int launch_apply_generic(void* amps, uint32_t n, const uint32_t* q, uint32_t k, const double* dev_matrix,
                         void* stream) {
    uint32_t qq[6] = {0, 0, 0, 0, 0, 0};
    for (uint32_t j = 0; j < k; ++j) qq[j] = q[j];
    const uint32_t dim = 1u << k;
    const size_t smem = (size_t{dim} * dim + kGenBatch) * sizeof(double2);
    static bool attr_set = false;
    if (!attr_set) {
        cudaFuncSetAttribute(k_apply_generic, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
        attr_set = true;
    }
    const uint64_t ngroups = (uint64_t{1} << n) >> k;
    const uint64_t nb = (ngroups + (kGenBatch >> k) - 1) / (kGenBatch >> k);
    const int grid = static_cast<int>(nb < 148ull * 4 ? nb : 148ull * 4);
    k_apply_generic<<<grid, 256, smem, static_cast<cudaStream_t>(stream)>>>(
        static_cast<double2*>(amps), n, k, qq[0], qq[1], qq[2], qq[3], qq[4], qq[5],
        reinterpret_cast<const double2*>(dev_matrix));
    note_launches(1);
    return status_of(cudaGetLastError());
}

int launch_tile_pass(void* amps, uint32_t n, const TilePass& pass, const TileInstr* dev_instrs,
                     const double* dev_sdata, const double* dev_gdata, int sm_count, void* stream,
                     const BatchLayout* batch, uint32_t ctas_per_sm, uint32_t buffers) {
    static bool attr_set = false;
    if (!attr_set) {
        const int most = static_cast<int>(3 * (size_t{1} << kMaxTileQubits) * sizeof(double2) + kMaxStagedBytes);
        cudaFuncSetAttribute(k_tile_pass<256, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, most);
        cudaFuncSetAttribute(k_tile_pass<128, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, most);
        cudaFuncSetAttribute(k_tile_pass<128, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, most);
        attr_set = true;
    }
    if (pass.m > kMaxTileQubits || pass.m < kMinTileQubits) return MB2_ERR_INVALID;
    const size_t staged = size_t{pass.prog_count} * sizeof(TileInstr) + size_t{pass.sdata_count} * sizeof(double);
    if (staged > kMaxStagedBytes) return MB2_ERR_INVALID;
    const uint32_t threads = 1u << (pass.m - kRegQubits);
    // 12-qubit tiles: one CTA per SM; smaller tiles: two CTAs per SM, or
    // three (168 registers a thread) when ctas_per_sm asks for it and the
    // shared memory allows.  Each CTA keeps `stages` tile buffers (tiles
    // stages - 1 ahead in flight): three where they fit beside the other
    // CTAs of the SM, else two.
    const uint32_t want_per_sm = pass.m == kMaxTileQubits ? 1u : (ctas_per_sm >= 3 ? 3u : 2u);
    const size_t tile_bytes = (size_t{1} << pass.m) * sizeof(double2);
    uint32_t stages = buffers == 2 ? 2u : 3u;
    if (stages == 3 && want_per_sm * (3 * tile_bytes + staged + 1024) > kSmemPerSm) stages = 2;
    const size_t smem = stages * tile_bytes + staged;
    auto kern = pass.m == kMaxTileQubits ? k_tile_pass<256, 1> : k_tile_pass<128, 2>;
    uint32_t per_sm = pass.m == kMaxTileQubits ? 1u : 2u;
    if (want_per_sm >= 3) {
        int resident = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, k_tile_pass<128, 3>, static_cast<int>(threads), smem);
        if (resident >= 3) {
            kern = k_tile_pass<128, 3>;
            per_sm = 3;
        }
    }
    // A batch adds the bindings above the n qubits: ntiles counts every
    // binding's tiles, and n grows to the bits the binding index occupies.
    uint64_t ntiles = (uint64_t{1} << n) >> pass.m;
    uint32_t n_all = n;
    if (batch != nullptr) {
        ntiles *= batch->bindings;
        while ((uint64_t{1} << (n_all - n)) < batch->bindings) ++n_all;
    }
    const uint64_t cap = static_cast<uint64_t>(sm_count) * per_sm;
    const int grid = static_cast<int>(ntiles < cap ? ntiles : cap);
    kern<<<grid, threads, smem, static_cast<cudaStream_t>(stream)>>>(
        static_cast<double2*>(amps), n_all, pass.m, pass.smask, dev_instrs + pass.prog_begin, pass.prog_count,
        dev_sdata + pass.sdata_begin, pass.sdata_count, dev_gdata, ntiles, batch ? batch->pdata : nullptr,
        batch ? batch->pstride : 0u, n - pass.m, stages);
    note_launches(1);
    return status_of(cudaGetLastError());
}

const char* last_cuda_error_string() { return cudaGetErrorString(cudaGetLastError()); }

}  // namespace mb2
