// Pauli-string expectation and norm reductions (FP64), fixed-order.
//
// <psi|P|psi> = i^popcount(x&z) * sum_m conj(psi[m]) psi[m^x] (-1)^popcount(z & (m^x))
// (src/kernels/cpu/dense_kernels.cpp:544-569).  The pair (m, m^x) is visited
// once, from the member whose bit h (the highest bit of x) is clear:
//     t = conj(a_m) a_m'                 (m' = m ^ x)
//     contribution = t s(m') + conj(t) s(m)
// so each amplitude is read once per term.  Partial sums land in a fixed
// number of blocks and are added in block order by one thread per term, so
// the value does not depend on the GPU's SM count or on what else runs.
// Like the reference's CUDA reduction (dense_kernels.h:237-246) it is not
// bitwise the CPU's sequential sum; the parity tests bound the difference.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <mutex>

#include "mb2_internal.h"

namespace mb2 {
namespace {

__device__ __forceinline__ uint64_t insert_zero(uint64_t i, uint32_t pos) {
    const uint64_t low = (uint64_t{1} << pos) - 1;
    return ((i & ~low) << 1) | (i & low);
}

constexpr int kThreads = 256;

__device__ __forceinline__ void block_reduce2(double& re, double& im) {
    __shared__ double sre[kThreads / 32], sim[kThreads / 32];
    for (int o = 16; o > 0; o >>= 1) {
        re += __shfl_down_sync(0xffffffffu, re, o);
        im += __shfl_down_sync(0xffffffffu, im, o);
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) {
        sre[w] = re;
        sim[w] = im;
    }
    __syncthreads();
    if (w == 0) {
        re = l < kThreads / 32 ? sre[l] : 0.0;
        im = l < kThreads / 32 ? sim[l] : 0.0;
        for (int o = 4; o > 0; o >>= 1) {
            re += __shfl_down_sync(0xffffffffu, re, o);
            im += __shfl_down_sync(0xffffffffu, im, o);
        }
    }
}

__device__ __forceinline__ double2 as_d2(double2 a) { return a; }
__device__ __forceinline__ double2 as_d2(float2 a) { return make_double2(a.x, a.y); }

// A: double2 (complex128 state) or float2 (complex64 state, promoted to FP64).
template <typename A>
__global__ void __launch_bounds__(kThreads)
    k_expectation(const A* __restrict__ st, uint32_t n, const uint64_t* __restrict__ xs,
                  const uint64_t* __restrict__ zs, double* __restrict__ partials) {
    const uint32_t term = blockIdx.y;
    const uint64_t x = xs[term], z = zs[term];
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    const uint64_t first = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    double re = 0.0, im = 0.0;
    if (x == 0) {
        const uint64_t na = uint64_t{1} << n;
        for (uint64_t m = first; m < na; m += stride) {
            const double2 a = as_d2(st[m]);
            const double p = __dadd_rn(__dmul_rn(a.x, a.x), __dmul_rn(a.y, a.y));
            re = (__popcll(z & m) & 1) ? __dsub_rn(re, p) : __dadd_rn(re, p);
        }
    } else {
        const uint32_t h = 63 - __clzll(static_cast<long long>(x));
        const uint64_t np = (uint64_t{1} << n) >> 1;
        for (uint64_t c = first; c < np; c += stride) {
            const uint64_t m = insert_zero(c, h);
            const uint64_t m2 = m ^ x;
            const double2 a = as_d2(st[m]), b = as_d2(st[m2]);
            // t = conj(a) * b
            const double tr = __dadd_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y));
            const double ti = __dsub_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x));
            const bool neg2 = __popcll(z & m2) & 1;  // sign of the (m, m') term
            const bool neg1 = __popcll(z & m) & 1;   // sign of the (m', m) term, conj(t)
            re = neg2 ? __dsub_rn(re, tr) : __dadd_rn(re, tr);
            im = neg2 ? __dsub_rn(im, ti) : __dadd_rn(im, ti);
            re = neg1 ? __dsub_rn(re, tr) : __dadd_rn(re, tr);
            im = neg1 ? __dadd_rn(im, ti) : __dsub_rn(im, ti);
        }
    }
    block_reduce2(re, im);
    if (threadIdx.x == 0) {
        double* p = partials + 2 * (static_cast<uint64_t>(term) * gridDim.x + blockIdx.x);
        p[0] = re;
        p[1] = im;
    }
}

// One thread per term: the partials in block order, then i^popcount(x&z).
__global__ void k_expectation_finish(const double* __restrict__ partials, uint32_t blocks,
                                     const uint64_t* __restrict__ xs, const uint64_t* __restrict__ zs,
                                     uint32_t num_terms, double* __restrict__ out) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= num_terms) return;
    double re = 0.0, im = 0.0;
    const double* p = partials + 2 * static_cast<uint64_t>(t) * blocks;
    for (uint32_t b = 0; b < blocks; ++b) {
        re = __dadd_rn(re, p[2 * b]);
        im = __dadd_rn(im, p[2 * b + 1]);
    }
    const int ph = __popcll(xs[t] & zs[t]) & 3;
    double orr = re, oi = im;
    if (ph == 1) {
        orr = -im;
        oi = re;
    } else if (ph == 2) {
        orr = -re;
        oi = -im;
    } else if (ph == 3) {
        orr = im;
        oi = -re;
    }
    out[2 * t] = orr;
    out[2 * t + 1] = oi;
}

// ---- grouped terms: one state read per group --------------------------------
// A group's terms have X masks whose bits above c lie in a subspace V of
// dimension d.  A tile is a coset of V: 2^d chunks of 2^c contiguous
// amplitudes (chunk k's high bits are rep ^ span[k]), so for every term the
// partner m ^ x of each amplitude m is in the same tile, at tile index
// L ^ dl with dl = (kx << c) | xl.
//
// With s(m) = (-1)^popcount(z & m) and s(m ^ x) = s(m) (-1)^popcount(z & x),
// the pair's share t s(m') + conj(t) s(m), t = conj(a_m) a_m', is
// 2 s(m) Re t when popcount(z & x) is even and -2i s(m) Im t when it is odd,
// so one real accumulator per term suffices; seen from the other member the
// same pair gives the same s(m) Re t (or s(m) Im t), so a pair may equally be
// visited once with weight 2 or from both members with weight 1.
//
// Thread r of the CTA owns tile amplitudes L = r | i << 8 (i < 2^(c+d-8),
// four or eight), read into registers once per tile; per term it visits its
// own amplitudes and reads only the partners from shared memory.  When dl
// has a bit b >= 8 the visiting member is the one with bit b clear (half of
// every thread's amplitudes, weight 2); otherwise every member visits
// (weight 1).  s(m) is linear over XOR in the tile index apart from the
// coset representative: s = parity(z_hi & rep) ^ sigma(r) ^ sigma(i << 8),
// with sigma(L) = parity(z_lo & L) ^ parity(z_hi & span[L >> c]); the
// thread's sigma(r) of every term is a register bit mask, sigma(i << 8) a
// per-term byte.  Each term runs a body compiled for its (own count,
// visiting bit, mode): its products are independent and summed as a
// balanced tree before one add into the thread's accumulator of the term
// (in shared memory, so the term loop needs no unrolling).
// Partial sums go to fixed slots (term, CTA) and are added in CTA order by
// the finish kernel.
using GroupTerm = PauliGroupTerm;
constexpr uint32_t kChunkWords = (1u << kPauliMaxSpan) / 32;
constexpr uint32_t kOwnShift = 8;  // log2(kThreads): tile bits of the thread index
constexpr uint32_t kMaxOwn = 1u << (kPauliTileQubits - kOwnShift);
static_assert(kThreads == (1 << kOwnShift), "one thread per low tile index");
static_assert(kPauliMinTileQubits >= kOwnShift + 1, "every thread owns at least two amplitudes");

// cp.async of one amplitude (16 or 8 bytes), global -> shared.
__device__ __forceinline__ void cp_async_amp(double2* smem, const double2* gmem) {
    const uint32_t sa = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_amp(float2* smem, const float2* gmem) {
    const uint32_t sa = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}

// Per-group tables in shared memory: the span, the parity of z_hi & span[k]
// per chunk k, per term its partner offset, body, sigma(i << 8) bits and
// high z bits, and every thread's accumulator of every term.
struct GroupShared {
    uint64_t sspan[1u << kPauliMaxSpan];
    uint32_t cpar[kMaxGroupTerms][kChunkWords];  // parity of z_hi & span[k], bit k
    uint32_t tdl[kMaxGroupTerms], tzl[kMaxGroupTerms], tmode[kMaxGroupTerms];
    uint32_t tcode[kMaxGroupTerms];  // the term's body (term_body)
    uint32_t tsigi[kMaxGroupTerms];  // bit i: sigma(i << 8)
    uint32_t tweight[kMaxGroupTerms];  // 2: each pair visited once; 1: from both members
    uint64_t tzh[kMaxGroupTerms];
    double acc[kMaxGroupTerms][kThreads];
    double red[kThreads / 32];
};

// sigma(L): the sign parity of tile index L without the coset's part.
__device__ __forceinline__ uint32_t group_sigma(const GroupShared& g, uint32_t t, uint32_t L, uint32_t c) {
    const uint32_t k = L >> c;
    return ((g.cpar[t][k >> 5] >> (k & 31u)) ^ static_cast<uint32_t>(__popc(g.tzl[t] & L))) & 1u;
}

// Term bodies: (own amplitudes, selector bit, mode).  Code = base of the
// own count (0 for four, 7 for eight) + 0 for a Z string, else
// 1 + 2 * (selector bit + 1) + (mode - 1), the selector bit -1 meaning every
// member visits.
__host__ __device__ constexpr uint32_t body_code(uint32_t own, int selb, uint32_t mode) {
    return (own == 8 ? 7u : 0u) + (mode == 0 ? 0u : 1u + 2u * static_cast<uint32_t>(selb + 1) + (mode - 1));
}

// Fills the tables and clears the accumulators; returns this thread's
// sigma(r) of every term (bit t).
__device__ __forceinline__ uint32_t group_setup(GroupShared& g, uint32_t c, uint32_t d,
                                                const uint64_t* __restrict__ span,
                                                const GroupTerm* __restrict__ terms, uint32_t nterms) {
    const uint32_t nchunks = 1u << d;
    const uint32_t own = 1u << (c + d - kOwnShift);
    for (uint32_t i = threadIdx.x; i < nchunks; i += kThreads) g.sspan[i] = span[i];
    for (uint32_t t = threadIdx.x; t < nterms; t += kThreads) {
        const GroupTerm T = terms[t];
        const uint32_t dl = (T.kx << c) | T.xl;
        g.tdl[t] = dl;
        g.tzl[t] = static_cast<uint32_t>(T.z & ((uint64_t{1} << c) - 1));
        g.tzh[t] = T.z >> c;
        // 0: a Z string (x = 0); 1: real pair sum; 2: imaginary pair sum
        const uint32_t mode = T.x == 0 ? 0u : ((__popcll(T.x & T.z) & 1) ? 2u : 1u);
        g.tmode[t] = mode;
        // The visiting member of a pair: the one whose highest bit of dl
        // among the register index bits is clear; none there: both visit.
        const uint32_t hi = dl >> kOwnShift;
        const int selb = hi == 0 ? -1 : 31 - __clz(hi);
        g.tcode[t] = body_code(own, mode == 0 ? -1 : selb, mode);
        g.tweight[t] = (mode != 0 && selb >= 0) ? 2u : 1u;
    }
    for (uint32_t i = threadIdx.x; i < kMaxGroupTerms * kThreads; i += kThreads) (&g.acc[0][0])[i] = 0.0;
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < kMaxGroupTerms * kChunkWords; i += kThreads) {
        const uint32_t t = i / kChunkWords, w = i % kChunkWords;
        uint32_t bits = 0;
        if (t < nterms)
            for (uint32_t b = 0; b < 32 && w * 32 + b < nchunks; ++b)
                bits |= static_cast<uint32_t>(__popcll(g.tzh[t] & g.sspan[w * 32 + b]) & 1) << b;
        g.cpar[t][w] = bits;
    }
    __syncthreads();
    for (uint32_t t = threadIdx.x; t < nterms; t += kThreads) {
        uint32_t bits = 0;
        for (uint32_t i = 0; i < own; ++i) bits |= group_sigma(g, t, i << kOwnShift, c) << i;
        g.tsigi[t] = bits;
    }
    uint32_t sig = 0;
    for (uint32_t t = 0; t < nterms; ++t) sig |= group_sigma(g, t, threadIdx.x, c) << t;
    __syncthreads();
    return sig;
}

// v with its sign flipped when f is 1 (an integer XOR: exact).
__device__ __forceinline__ double flip_if(double v, uint32_t f) {
    return __hiloint2double(__double2hiint(v) ^ static_cast<int>(f << 31), __double2loint(v));
}

// One term's share of this thread's own amplitudes in one tile, as a
// balanced sum in a fixed order: OWN own amplitudes, SELB the register bit
// that marks the non-visiting member (-1: all visit), MODE 0 (|a|^2),
// 1 (Re conj(a) b) or 2 (Im conj(a) b); sg bit i: the sign of own
// amplitude i.  Every branch is resolved at compile time.
template <int OWN, int SELB, int MODE, typename A>
__device__ __forceinline__ double term_body(const double2 (&a)[kMaxOwn], const A* __restrict__ cur, uint32_t r,
                                            uint32_t dl, uint32_t sg) {
    constexpr int NV = SELB < 0 ? OWN : OWN / 2;
    constexpr int SB = SELB < 0 ? 0 : SELB;
    double v[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        // The k-th visiting own amplitude: k with a zero inserted at SELB.
        const int i = SELB < 0 ? k : (((k >> SB) << (SB + 1)) | (k & ((1 << SB) - 1)));
        double x;
        if constexpr (MODE == 0) {
            x = __dadd_rn(__dmul_rn(a[i].x, a[i].x), __dmul_rn(a[i].y, a[i].y));
        } else {
            const double2 b = as_d2(cur[(r | (static_cast<uint32_t>(i) << kOwnShift)) ^ dl]);
            x = MODE == 1 ? __dadd_rn(__dmul_rn(a[i].x, b.x), __dmul_rn(a[i].y, b.y))
                          : __dsub_rn(__dmul_rn(a[i].x, b.y), __dmul_rn(a[i].y, b.x));
        }
        v[k] = flip_if(x, (sg >> i) & 1u);
    }
#pragma unroll
    for (int w = 1; w < NV; w <<= 1)
#pragma unroll
        for (int j = 0; j + w < NV; j += 2 * w) v[j] = __dadd_rn(v[j], v[j + w]);
    return v[0];
}

// Adds one gathered coset tile (representative rep) to every term's
// accumulator.  sig: this thread's sigma(r) bits (group_setup).
template <typename A>
__device__ __forceinline__ void group_tile(GroupShared& g, const A* __restrict__ cur, uint64_t rep,
                                           uint32_t tile_amps, uint32_t nterms, uint32_t sig) {
    const uint32_t r = threadIdx.x;
    const uint32_t own = tile_amps >> kOwnShift;
    double2 a[kMaxOwn];
#pragma unroll
    for (uint32_t i = 0; i < kMaxOwn; ++i)
        a[i] = i < own ? as_d2(cur[r | (i << kOwnShift)]) : make_double2(0.0, 0.0);
    for (uint32_t t = 0; t < nterms; ++t) {
        // Bit i: the sign of own amplitude i.
        const uint32_t s0 = (static_cast<uint32_t>(__popcll(g.tzh[t] & rep)) ^ (sig >> t)) & 1u;
        const uint32_t sg = g.tsigi[t] ^ (0u - s0);
        const uint32_t dl = g.tdl[t];
        double v = 0.0;
        switch (g.tcode[t]) {
            case body_code(4, -1, 0): v = term_body<4, -1, 0>(a, cur, r, dl, sg); break;
            case body_code(4, -1, 1): v = term_body<4, -1, 1>(a, cur, r, dl, sg); break;
            case body_code(4, -1, 2): v = term_body<4, -1, 2>(a, cur, r, dl, sg); break;
            case body_code(4, 0, 1): v = term_body<4, 0, 1>(a, cur, r, dl, sg); break;
            case body_code(4, 0, 2): v = term_body<4, 0, 2>(a, cur, r, dl, sg); break;
            case body_code(4, 1, 1): v = term_body<4, 1, 1>(a, cur, r, dl, sg); break;
            case body_code(4, 1, 2): v = term_body<4, 1, 2>(a, cur, r, dl, sg); break;
            case body_code(8, -1, 0): v = term_body<8, -1, 0>(a, cur, r, dl, sg); break;
            case body_code(8, -1, 1): v = term_body<8, -1, 1>(a, cur, r, dl, sg); break;
            case body_code(8, -1, 2): v = term_body<8, -1, 2>(a, cur, r, dl, sg); break;
            case body_code(8, 0, 1): v = term_body<8, 0, 1>(a, cur, r, dl, sg); break;
            case body_code(8, 0, 2): v = term_body<8, 0, 2>(a, cur, r, dl, sg); break;
            case body_code(8, 1, 1): v = term_body<8, 1, 1>(a, cur, r, dl, sg); break;
            case body_code(8, 1, 2): v = term_body<8, 1, 2>(a, cur, r, dl, sg); break;
            case body_code(8, 2, 1): v = term_body<8, 2, 1>(a, cur, r, dl, sg); break;
            case body_code(8, 2, 2): v = term_body<8, 2, 2>(a, cur, r, dl, sg); break;
            default: break;
        }
        g.acc[t][r] = __dadd_rn(g.acc[t][r], v);
    }
}

// Per term: this CTA's sum in a fixed order (lanes, then warps), written to
// slot_of(t) as (re, im) of the pair sum before the i^popcount(x & z)
// factor, with the term's visit weight; the accumulators are cleared.
template <typename SLOT>
__device__ __forceinline__ void group_write(GroupShared& g, const GroupTerm* __restrict__ terms, uint32_t nterms,
                                            SLOT slot_of) {
    for (uint32_t t = 0; t < nterms; ++t) {
        double r = g.acc[t][threadIdx.x];
        g.acc[t][threadIdx.x] = 0.0;
        for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
        __syncthreads();
        if ((threadIdx.x & 31) == 0) g.red[threadIdx.x >> 5] = r;
        __syncthreads();
        if (threadIdx.x == 0) {
            double sum = 0.0;
            for (int w = 0; w < kThreads / 32; ++w) sum += g.red[w];
            double* p = slot_of(terms[t].out);
            const uint32_t mode = g.tmode[t];
            const double w = static_cast<double>(g.tweight[t]);
            p[0] = mode == 0 ? sum : mode == 1 ? w * sum : 0.0;
            p[1] = mode == 2 ? -w * sum : 0.0;
        }
    }
}

// Coset representative: the coset number deposited on the free (non-pivot)
// high bits.
__device__ __forceinline__ uint64_t deposit_bits(uint64_t v, uint64_t mask) {
    uint64_t r = 0;
    while (mask != 0) {
        const uint64_t low = mask & (~mask + 1);
        if (v & 1) r |= low;
        v >>= 1;
        mask ^= low;
    }
    return r;
}

template <typename A>
__device__ __forceinline__ void group_gather(const A* __restrict__ st, uint64_t rep, A* buf, const GroupShared& g,
                                             uint32_t c, uint32_t tile_amps) {
    const uint32_t lowmask = (1u << c) - 1;
    for (uint32_t L = threadIdx.x; L < tile_amps; L += kThreads) {
        const uint64_t m = ((rep ^ g.sspan[L >> c]) << c) | (L & lowmask);
        cp_async_amp(buf + L, st + m);
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}

// Cosets are processed with two shared-memory buffers: the next coset's
// amplitudes are gathered with cp.async while this one is reduced.
template <typename A>
__global__ void __launch_bounds__(kThreads, 2)
    k_pauli_group(const A* __restrict__ st, uint32_t c, uint32_t d, const uint64_t* __restrict__ span,
                  uint64_t free_mask, const GroupTerm* __restrict__ terms, uint32_t nterms, uint64_t ncosets,
                  double* __restrict__ partials) {
    extern __shared__ __align__(16) unsigned char gsm[];
    __shared__ GroupShared g;
    const uint32_t tile_amps = 1u << (c + d);
    A* buf0 = reinterpret_cast<A*>(gsm);
    A* buf1 = buf0 + tile_amps;
    const uint32_t sig = group_setup(g, c, d, span, terms, nterms);
    // Moving gridDim.x cosets on is a masked add on the free bits.
    const uint64_t rstep = deposit_bits(gridDim.x, free_mask);
    auto advance = [&](uint64_t r) { return ((r | ~free_mask) + rstep) & free_mask; };
    uint64_t rep = deposit_bits(blockIdx.x, free_mask);
    if (blockIdx.x < ncosets) group_gather(st, rep, buf0, g, c, tile_amps);
    A* cur = buf0;
    A* nxt = buf1;
    for (uint64_t cs = blockIdx.x; cs < ncosets; cs += gridDim.x) {
        const uint64_t rep_next = advance(rep);
        if (cs + gridDim.x < ncosets) group_gather(st, rep_next, nxt, g, c, tile_amps);
        else asm volatile("cp.async.commit_group;\n" ::: "memory");
        asm volatile("cp.async.wait_group 1;\n" ::: "memory");
        __syncthreads();
        group_tile(g, cur, rep, tile_amps, nterms, sig);
        __syncthreads();  // this buffer is the target of the gather after next
        rep = rep_next;
        A* tmp = cur;
        cur = nxt;
        nxt = tmp;
    }
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    group_write(g, terms, nterms, [&](uint32_t out) {
        return partials + 2 * (static_cast<uint64_t>(out) * gridDim.x + blockIdx.x);
    });
}

// The same grouped reduction over a batch of states (binding b's 2^n
// amplitudes at b * 2^n).  `per` CTAs share a binding: CTA slot s takes the
// binding's cosets s, s + per, ...; bindings are taken gridDim.x / per
// apart.  Partial (term, binding, slot) lands at
// partials[2 * ((term * bindings + b) * per + s)], so a binding's value
// depends only on its own state and on `per`.
template <typename A>
__global__ void __launch_bounds__(kThreads, 2)
    k_pauli_group_batch(const A* __restrict__ st, uint32_t n, uint32_t c, uint32_t d,
                        const uint64_t* __restrict__ span, uint64_t free_mask, const GroupTerm* __restrict__ terms,
                        uint32_t nterms, uint64_t bindings, uint32_t per, double* __restrict__ partials) {
    extern __shared__ __align__(16) unsigned char gsm[];
    __shared__ GroupShared g;
    const uint32_t tile_amps = 1u << (c + d);
    A* buf0 = reinterpret_cast<A*>(gsm);
    A* buf1 = buf0 + tile_amps;
    const uint32_t sig = group_setup(g, c, d, span, terms, nterms);
    const uint64_t ncosets = uint64_t{1} << (n - c - d);
    const uint32_t slot = blockIdx.x % per;
    const uint64_t b0 = blockIdx.x / per, bstep = gridDim.x / per;
    if (b0 >= bindings) return;  // (uniform over the CTA)
    // This CTA's cosets in each binding, and its work items in order:
    // item f = (binding b0 + (f / mine) * bstep, coset slot + (f % mine) * per).
    const uint64_t mine = ncosets > slot ? (ncosets - slot + per - 1) / per : 0;
    const uint64_t nb = (bindings - b0 + bstep - 1) / bstep;
    auto write = [&](uint64_t b) {
        group_write(g, terms, nterms, [&](uint32_t out) {
            return partials + 2 * ((static_cast<uint64_t>(out) * bindings + b) * per + slot);
        });
    };
    if (mine == 0) {  // more slots than cosets: this slot's partials are zero
        for (uint64_t i = 0; i < nb; ++i) write(b0 + i * bstep);
        return;
    }
    const uint64_t items = nb * mine;
    auto item = [&](uint64_t f, uint64_t& b, uint64_t& rep) {
        b = b0 + (f / mine) * bstep;
        rep = deposit_bits(slot + (f % mine) * per, free_mask);
    };
    uint64_t b = 0, rep = 0;
    item(0, b, rep);
    group_gather(st + (b << n), rep, buf0, g, c, tile_amps);
    A* cur = buf0;
    A* nxt = buf1;
    for (uint64_t f = 0; f < items; ++f) {
        uint64_t bn = 0, repn = 0;
        if (f + 1 < items) {
            item(f + 1, bn, repn);
            group_gather(st + (bn << n), repn, nxt, g, c, tile_amps);
        } else {
            asm volatile("cp.async.commit_group;\n" ::: "memory");
        }
        asm volatile("cp.async.wait_group 1;\n" ::: "memory");
        __syncthreads();
        group_tile(g, cur, rep, tile_amps, nterms, sig);
        __syncthreads();  // this buffer is the target of the gather after next
        if ((f + 1) % mine == 0) write(b);
        b = bn;
        rep = repn;
        A* tmp = cur;
        cur = nxt;
        nxt = tmp;
    }
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// <H> per binding: sum over terms in term order of coef * Re(i^popcount(x&z)
// * (sum over the binding's slots, in slot order, of the partials)).
__global__ void k_batch_group_finish(const double* __restrict__ partials, uint64_t bindings, uint32_t per,
                                     const uint64_t* __restrict__ xs, const uint64_t* __restrict__ zs,
                                     const double* __restrict__ coefs, uint32_t num_terms, double* __restrict__ out) {
    for (uint64_t b = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; b < bindings;
         b += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        double total = 0.0;
        for (uint32_t t = 0; t < num_terms; ++t) {
            const double* p = partials + 2 * ((static_cast<uint64_t>(t) * bindings + b) * per);
            double re = 0.0, im = 0.0;
            for (uint32_t s = 0; s < per; ++s) {
                re += p[2 * s];
                im += p[2 * s + 1];
            }
            const int ph = __popcll(xs[t] & zs[t]) & 3;
            total += coefs[t] * (ph == 0 ? re : ph == 1 ? -im : ph == 2 ? -re : im);
        }
        out[b] = total;
    }
}

}  // namespace

int launch_pauli_group(const void* amps, uint32_t n, uint32_t c, uint32_t d, const uint64_t* dev_span,
                       uint64_t free_mask, const void* dev_terms, uint32_t nterms, double* dev_partials,
                       uint32_t grid, void* stream, int precision) {
    if (nterms == 0) return MB2_OK;
    if (nterms > kMaxGroupTerms || c + d > kPauliTileQubits || d > kPauliMaxSpan) return MB2_ERR_INVALID;
    const auto s = static_cast<cudaStream_t>(stream);
    const uint64_t ncosets = uint64_t{1} << (n - c - d);
    // Two buffers of 2^(c+d) amplitudes; each thread takes two amplitudes (or
    // two pairs) per step, so a tile holds at least 4 * kThreads of them.
    if (c + d < kPauliMinTileQubits) return MB2_ERR_INVALID;
    const size_t smem = 2 * (size_t{1} << (c + d)) * (precision == MB2_C64 ? sizeof(float2) : sizeof(double2));
    static const bool attr = [] {  // once, thread-safe (concurrent callers wait for it)
        return cudaFuncSetAttribute(k_pauli_group<double2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    128 * 1024) == cudaSuccess &&
               cudaFuncSetAttribute(k_pauli_group<float2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    128 * 1024) == cudaSuccess;
    }();
    if (!attr) return launch_status();
    const auto* terms = static_cast<const GroupTerm*>(dev_terms);
    if (precision == MB2_C64)
        k_pauli_group<float2><<<grid, kThreads, smem, s>>>(static_cast<const float2*>(amps), c, d, dev_span,
                                                           free_mask, terms, nterms, ncosets, dev_partials);
    else
        k_pauli_group<double2><<<grid, kThreads, smem, s>>>(static_cast<const double2*>(amps), c, d, dev_span,
                                                            free_mask, terms, nterms, ncosets, dev_partials);
    note_launches(1);
    return launch_status();
}

int launch_pauli_group_batch(const void* amps, uint32_t n, uint32_t c, uint32_t d, const uint64_t* dev_span,
                             uint64_t free_mask, const void* dev_terms, uint32_t nterms, uint64_t bindings,
                             uint32_t per, double* dev_partials, int sm_count, void* stream, int precision) {
    if (nterms == 0) return MB2_OK;
    if (nterms > kMaxGroupTerms || c + d > kPauliTileQubits || d > kPauliMaxSpan || c + d > n || per == 0 ||
        c + d < kPauliMinTileQubits)
        return MB2_ERR_INVALID;
    const size_t smem = 2 * (size_t{1} << (c + d)) * (precision == MB2_C64 ? sizeof(float2) : sizeof(double2));
    static const bool attr = [] {  // once, thread-safe
        return cudaFuncSetAttribute(k_pauli_group_batch<double2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    128 * 1024) == cudaSuccess &&
               cudaFuncSetAttribute(k_pauli_group_batch<float2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    128 * 1024) == cudaSuccess;
    }();
    if (!attr) return launch_status();
    // Two CTAs per SM, a multiple of `per`, no more binding lanes than bindings.
    uint64_t lanes = std::max<uint64_t>(1, (2ull * static_cast<uint64_t>(sm_count)) / per);
    lanes = std::min<uint64_t>(lanes, bindings);
    const unsigned grid = static_cast<unsigned>(lanes * per);
    const auto s = static_cast<cudaStream_t>(stream);
    const auto* terms = static_cast<const GroupTerm*>(dev_terms);
    if (precision == MB2_C64)
        k_pauli_group_batch<float2><<<grid, kThreads, smem, s>>>(static_cast<const float2*>(amps), n, c, d, dev_span,
                                                                 free_mask, terms, nterms, bindings, per, dev_partials);
    else
        k_pauli_group_batch<double2><<<grid, kThreads, smem, s>>>(static_cast<const double2*>(amps), n, c, d,
                                                                  dev_span, free_mask, terms, nterms, bindings, per,
                                                                  dev_partials);
    note_launches(1);
    return launch_status();
}

int launch_batch_group_finish(const double* dev_partials, uint64_t bindings, uint32_t per, const uint64_t* dev_x,
                              const uint64_t* dev_z, const double* dev_coefs, uint32_t num_terms, double* dev_out,
                              void* stream) {
    const uint64_t blocks = (bindings + 127) / 128;
    k_batch_group_finish<<<static_cast<unsigned>(blocks < 1024 ? blocks : 1024), 128, 0,
                           static_cast<cudaStream_t>(stream)>>>(dev_partials, bindings, per, dev_x, dev_z, dev_coefs,
                                                                num_terms, dev_out);
    note_launches(1);
    return launch_status();
}

// ---- density matrices ---------------------------------------------------
// rho as a 2n-qubit vector, entry (r, c) at r | c << n.  Tr(P rho) partials:
// the sum over c of (-1)^popcount(c & z) rho[c | (c ^ x) << n] (the
// reference's trace_with_pauli, src/engines/density_matrix/
// density_matrix_engine.cpp); k_expectation_finish adds the partials in
// block order and applies i^popcount(x & z).
__global__ void __launch_bounds__(kThreads)
    k_dm_trace(const double2* __restrict__ rho, uint32_t n, const uint64_t* __restrict__ xs,
               const uint64_t* __restrict__ zs, double* __restrict__ partials) {
    const uint32_t term = blockIdx.y;
    const uint64_t x = xs[term], z = zs[term];
    const uint64_t dim = uint64_t{1} << n;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    double re = 0.0, im = 0.0;
    for (uint64_t c = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; c < dim; c += stride) {
        const double2 e = rho[c | ((c ^ x) << n)];
        if (__popcll(c & z) & 1) {
            re = __dsub_rn(re, e.x);
            im = __dsub_rn(im, e.y);
        } else {
            re = __dadd_rn(re, e.x);
            im = __dadd_rn(im, e.y);
        }
    }
    block_reduce2(re, im);
    if (threadIdx.x == 0) {
        double* p = partials + 2 * (static_cast<uint64_t>(term) * gridDim.x + blockIdx.x);
        p[0] = re;
        p[1] = im;
    }
}

// The reference's sort-then-walk over rho's diagonal, strictly in order
// (src/engines/dense/sample.cpp:55-69 over probabilities Re rho[x | x << n]):
// one thread, for the density matrices this path holds (n <= 15).
__global__ void k_dm_walk(const double2* __restrict__ rho, uint32_t n, const double* __restrict__ u, uint64_t shots,
                          uint64_t* __restrict__ basis) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    const uint64_t dim = uint64_t{1} << n;
    double cumulative = 0.0;
    uint64_t s = 0;
    for (uint64_t b = 0; b < dim && s < shots; ++b) {
        cumulative = __dadd_rn(cumulative, rho[b * (dim + 1)].x);
        while (s < shots && u[s] < cumulative) basis[s++] = b;
    }
    for (; s < shots; ++s) basis[s] = dim - 1;
}

int launch_expectation_finish(const double* dev_partials, uint32_t blocks, const uint64_t* dev_x,
                              const uint64_t* dev_z, uint32_t num_terms, double* dev_out, void* stream) {
    k_expectation_finish<<<(num_terms + 127) / 128, 128, 0, static_cast<cudaStream_t>(stream)>>>(
        dev_partials, blocks, dev_x, dev_z, num_terms, dev_out);
    note_launches(1);
    return launch_status();
}

int launch_dm_trace(const void* rho, uint32_t n, const uint64_t* dev_x, const uint64_t* dev_z, uint32_t num_terms,
                    double* dev_partials, double* dev_out, void* stream) {
    if (num_terms == 0) return MB2_OK;
    const auto s = static_cast<cudaStream_t>(stream);
    k_dm_trace<<<dim3(kExpBlocks, num_terms), kThreads, 0, s>>>(static_cast<const double2*>(rho), n, dev_x, dev_z,
                                                               dev_partials);
    note_launches(1);
    if (int rc = launch_status(); rc != MB2_OK) return rc;
    return launch_expectation_finish(dev_partials, kExpBlocks, dev_x, dev_z, num_terms, dev_out, stream);
}

int launch_dm_walk(const void* rho, uint32_t n, const double* dev_uniforms_sorted, uint64_t shots,
                   uint64_t* dev_basis, void* stream) {
    k_dm_walk<<<1, 32, 0, static_cast<cudaStream_t>(stream)>>>(static_cast<const double2*>(rho), n,
                                                              dev_uniforms_sorted, shots, dev_basis);
    note_launches(1);
    return launch_status();
}

int launch_expectation_partials(const void* amps, uint32_t n, const uint64_t* dev_x, const uint64_t* dev_z,
                                uint32_t num_terms, double* dev_partials, void* stream, int precision) {
    if (num_terms == 0) return MB2_OK;
    const auto s = static_cast<cudaStream_t>(stream);
    const dim3 grid(kExpBlocks, num_terms);
    if (precision == MB2_C64)
        k_expectation<float2><<<grid, kThreads, 0, s>>>(static_cast<const float2*>(amps), n, dev_x, dev_z, dev_partials);
    else
        k_expectation<double2><<<grid, kThreads, 0, s>>>(static_cast<const double2*>(amps), n, dev_x, dev_z,
                                                         dev_partials);
    note_launches(1);
    return launch_status();
}

int launch_expectation(const void* amps, uint32_t n, const uint64_t* dev_x, const uint64_t* dev_z,
                       uint32_t num_terms, double* dev_partials, double* dev_out, void* stream, int precision) {
    if (num_terms == 0) return MB2_OK;
    const auto s = static_cast<cudaStream_t>(stream);
    const dim3 grid(kExpBlocks, num_terms);
    if (precision == MB2_C64)
        k_expectation<float2><<<grid, kThreads, 0, s>>>(static_cast<const float2*>(amps), n, dev_x, dev_z, dev_partials);
    else
        k_expectation<double2><<<grid, kThreads, 0, s>>>(static_cast<const double2*>(amps), n, dev_x, dev_z,
                                                         dev_partials);
    k_expectation_finish<<<(num_terms + 127) / 128, 128, 0, s>>>(dev_partials, kExpBlocks, dev_x, dev_z, num_terms,
                                                                  dev_out);
    note_launches(2);
    return launch_status();
}

}  // namespace mb2

// ---------------------------------------------------------------------------
// The expectation reduction for callers that cannot allocate device memory.
//
// Some callers of this library must not call cudaMalloc: a serving process
// whose own pool allocator has reserved the GPU's memory up front (a
// cudaMalloc from here would fail or fragment that pool), or code running
// where allocation is not allowed at all (a latency-critical loop that must
// not stall on the driver's allocator).  mb2_expectation_noalloc gives them
// the Pauli-expectation reduction with every byte of scratch it needs --
// the Pauli masks, the per-block partial sums and the finished terms -- in
// the file-scope array below, a fixed 526,336 bytes that every GPU which
// loads this library holds until the process exits.
// ---------------------------------------------------------------------------
namespace mb2 {
namespace {

constexpr uint32_t kNoAllocTerms = MB2_NOALLOC_MAX_TERMS;
constexpr size_t kNoAllocMasks = kNoAllocTerms * sizeof(uint64_t);                 // x, then z
constexpr size_t kNoAllocPartials = size_t{kNoAllocTerms} * kExpBlocks * 2 * sizeof(double);
constexpr size_t kNoAllocOut = kNoAllocTerms * 2 * sizeof(double);
constexpr size_t kNoAllocBytes = 2 * kNoAllocMasks + kNoAllocPartials + kNoAllocOut;
static_assert(kNoAllocBytes == 526336, "the documented size");

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
unsigned char* g_noalloc_ptr[kMaxDevices] = {};

// The device address of g_noalloc_scratch on the current device.  In host
// code the symbol names a host-side stand-in, not device memory, so the
// address is looked up once per device (with that device current) and kept;
// `refresh` looks it up again (after a device reset the module is loaded
// anew and the kept address is stale).
int noalloc_scratch(unsigned char** out, bool refresh = false) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        cudaGetLastError();
        return MB2_ERR_NO_DEVICE;
    }
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (g_noalloc_ptr[dev] == nullptr || refresh) {
        void* p = nullptr;
        if (const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch); e != cudaSuccess)
            return record_cuda_error(e);
        g_noalloc_ptr[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_noalloc_ptr[dev];
    return MB2_OK;
}

}  // namespace

}  // namespace mb2

extern "C" int mb2_expectation_noalloc(const void* dev_amps, uint32_t num_qubits, const uint64_t* x_masks,
                                       const uint64_t* z_masks, uint32_t num_terms, double* out, void* stream) {
    using namespace mb2;
    if (num_terms == 0) return MB2_OK;
    if (num_terms > kNoAllocTerms) return MB2_ERR_RESOURCE;
    if (dev_amps == nullptr || x_masks == nullptr || z_masks == nullptr || out == nullptr || num_qubits < 1 ||
        num_qubits > 40)
        return MB2_ERR_INVALID;
    const uint64_t lim = (uint64_t{1} << num_qubits) - 1;
    for (uint32_t t = 0; t < num_terms; ++t)
        if ((x_masks[t] | z_masks[t]) & ~lim) return MB2_ERR_INVALID;
    unsigned char* base = nullptr;
    if (int rc = noalloc_scratch(&base); rc != MB2_OK) return rc;
    auto* dx = reinterpret_cast<uint64_t*>(base);
    auto* dz = reinterpret_cast<uint64_t*>(base + kNoAllocMasks);
    auto* partials = reinterpret_cast<double*>(base + 2 * kNoAllocMasks);
    auto* dout = reinterpret_cast<double*>(base + 2 * kNoAllocMasks + kNoAllocPartials);
    const auto s = static_cast<cudaStream_t>(stream);
    const size_t mb = size_t{num_terms} * sizeof(uint64_t);
    cudaError_t e = cudaMemcpyAsync(dx, x_masks, mb, cudaMemcpyHostToDevice, s);
    if (e == cudaErrorInvalidValue) {
        // A kept address from before a device reset: look it up again, once.
        cudaGetLastError();
        if (int rc = noalloc_scratch(&base, true); rc != MB2_OK) return rc;
        dx = reinterpret_cast<uint64_t*>(base);
        dz = reinterpret_cast<uint64_t*>(base + kNoAllocMasks);
        partials = reinterpret_cast<double*>(base + 2 * kNoAllocMasks);
        dout = reinterpret_cast<double*>(base + 2 * kNoAllocMasks + kNoAllocPartials);
        e = cudaMemcpyAsync(dx, x_masks, mb, cudaMemcpyHostToDevice, s);
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(dz, z_masks, mb, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return record_cuda_error(e);
    // Every partial and every output slot is written before it is read, so
    // nothing left in the array by an earlier call needs clearing.
    if (launch_expectation(dev_amps, num_qubits, dx, dz, num_terms, partials, dout, stream) != MB2_OK)
        return MB2_ERR_CUDA;
    e = cudaMemcpyAsync(out, dout, size_t{num_terms} * 2 * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return record_cuda_error(e);
}

