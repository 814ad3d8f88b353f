/*
 * oracle.c -- TEST INFRASTRUCTURE: the CPU oracle of the dense statevector
 * path, a plain-C restatement of the reference MENOS CPU algorithm.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load this library, and only as the checker.  The product (menos_b200/)
 * never links or calls it.
 *
 * Pinned against: the reference itself compiled here (oracle/_ref, see
 * oracle/Makefile) on every function below, and the reference's golden
 * counts (tests/engines/dense/sample_test.cpp:85-97: seed 42, 20 shots on
 * |+> -> {0: 9, 1: 11}); fixtures in tests/golden/.
 *
 * Arithmetic rules followed exactly (build with -ffp-contract=off):
 *   complex product  (a.r*b.r - a.i*b.i, a.r*b.i + a.i*b.r)   [std::complex operator*]
 *   every gate output (+0) + sum_in m[out][in]*a[in], increasing in
 *                     (src/kernels/cpu/dense_kernels.cpp:513-520)
 */
#define _GNU_SOURCE
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------
 * mt19937_64 (Matsumoto & Nishimura 2004; the parameters the C++ standard
 * fixes for std::mt19937_64) and the reference's word -> uniform map
 * (src/common/rng.cpp:184-186: (w >> 11) * 2^-53).
 * ---------------------------------------------------------------------- */
typedef struct {
    uint64_t mt[312];
    int idx;
} orc_mt64;

static void mt_seed(orc_mt64* s, uint64_t seed) {
    s->mt[0] = seed;
    for (int i = 1; i < 312; ++i) {
        s->mt[i] = 6364136223846793005ULL * (s->mt[i - 1] ^ (s->mt[i - 1] >> 62)) + (uint64_t)i;
    }
    s->idx = 312;
}

static uint64_t mt_next(orc_mt64* s) {
    if (s->idx >= 312) {
        for (int i = 0; i < 312; ++i) {
            const uint64_t y = (s->mt[i] & 0xFFFFFFFF80000000ULL) | (s->mt[(i + 1) % 312] & 0x7FFFFFFFULL);
            uint64_t v = s->mt[(i + 156) % 312] ^ (y >> 1);
            if (y & 1ULL) v ^= 0xB5026F5AA96619E9ULL;
            s->mt[i] = v;
        }
        s->idx = 0;
    }
    uint64_t x = s->mt[s->idx++];
    x ^= (x >> 29) & 0x5555555555555555ULL;
    x ^= (x << 17) & 0x71D67FFFEDA60000ULL;
    x ^= (x << 37) & 0xFFF7EEE000000000ULL;
    x ^= x >> 43;
    return x;
}

static double word_to_uniform(uint64_t w) {
    return (double)(w >> 11) * (1.0 / 9007199254740992.0);
}

void orc_uniforms(uint64_t seed, uint64_t n, double* out) {
    orc_mt64 s;
    mt_seed(&s, seed);
    for (uint64_t i = 0; i < n; ++i) out[i] = word_to_uniform(mt_next(&s));
}

void orc_words(uint64_t seed, uint64_t n, uint64_t* out) {
    orc_mt64 s;
    mt_seed(&s, seed);
    for (uint64_t i = 0; i < n; ++i) out[i] = mt_next(&s);
}

/* ------------------------------------------------------------------------
 * Gate matrices: src/ir/gate_table.cpp:17-206, term by term.  std::exp of a
 * std::complex<double> is glibc's cexp; `1.0i * t` is (0.0*t, 1.0*t) and
 * `-1.0i * t` is (-0.0*t, -1.0*t); complex * real scales both parts.
 * ---------------------------------------------------------------------- */
static void put(double* out, int i, double re, double im) {
    out[2 * i] = re;
    out[2 * i + 1] = im;
}

static double complex iexp(double coef_re, double coef_im, double t) {
    /* std::exp(complex(coef_re, coef_im) * t) */
    return cexp(CMPLX(coef_re * t, coef_im * t));
}

/* Returns the matrix dimension (2, 4 or 8), 0 for an unknown opcode. */
int orc_gate_matrix(int opcode, const double* p, double* out) {
    memset(out, 0, sizeof(double) * 2 * 64);
    switch (opcode) {
        case 0: /* X */ put(out, 1, 1.0, 0.0); put(out, 2, 1.0, 0.0); return 2;
        case 1: /* Y: {0, -1.0i, 1.0i, 0} */ put(out, 1, -0.0, -1.0); put(out, 2, 0.0, 1.0); return 2;
        case 2: /* Z */ put(out, 0, 1.0, 0.0); put(out, 3, -1.0, 0.0); return 2;
        case 3: { /* H */
            const double s = 1.0 / sqrt(2.0);
            put(out, 0, s, 0.0); put(out, 1, s, 0.0); put(out, 2, s, 0.0); put(out, 3, -s, 0.0);
            return 2;
        }
        case 4: /* S */ put(out, 0, 1.0, 0.0); put(out, 3, 0.0, 1.0); return 2;
        case 5: /* Sdg: -1.0i */ put(out, 0, 1.0, 0.0); put(out, 3, -0.0, -1.0); return 2;
        case 6: { /* T */
            const double complex e = iexp(0.0, 1.0, M_PI / 4.0);
            put(out, 0, 1.0, 0.0); put(out, 3, creal(e), cimag(e));
            return 2;
        }
        case 7: { /* Tdg */
            const double complex e = iexp(-0.0, -1.0, M_PI / 4.0);
            put(out, 0, 1.0, 0.0); put(out, 3, creal(e), cimag(e));
            return 2;
        }
        case 8: /* SX: 0.5*(1+1i), 0.5*(1-1i) */
            put(out, 0, 0.5, 0.5); put(out, 1, 0.5, -0.5); put(out, 2, 0.5, -0.5); put(out, 3, 0.5, 0.5);
            return 2;
        case 9: /* SXdg */
            put(out, 0, 0.5, -0.5); put(out, 1, 0.5, 0.5); put(out, 2, 0.5, 0.5); put(out, 3, 0.5, -0.5);
            return 2;
        case 10: { /* RX: {c, -1.0i*s, -1.0i*s, c} */
            const double c = cos(p[0] / 2.0), s = sin(p[0] / 2.0);
            put(out, 0, c, 0.0); put(out, 1, -0.0 * s, -1.0 * s);
            put(out, 2, -0.0 * s, -1.0 * s); put(out, 3, c, 0.0);
            return 2;
        }
        case 11: { /* RY: {c, -s, s, c} */
            const double c = cos(p[0] / 2.0), s = sin(p[0] / 2.0);
            put(out, 0, c, 0.0); put(out, 1, -s, 0.0); put(out, 2, s, 0.0); put(out, 3, c, 0.0);
            return 2;
        }
        case 12: { /* RZ: {exp(-1.0i*(t/2)), 0, 0, exp(1.0i*(t/2))} */
            const double complex a = iexp(-0.0, -1.0, p[0] / 2.0);
            const double complex b = iexp(0.0, 1.0, p[0] / 2.0);
            put(out, 0, creal(a), cimag(a)); put(out, 3, creal(b), cimag(b));
            return 2;
        }
        case 13: { /* P */
            const double complex b = iexp(0.0, 1.0, p[0]);
            put(out, 0, 1.0, 0.0); put(out, 3, creal(b), cimag(b));
            return 2;
        }
        case 14: { /* U(theta, phi, lambda) */
            const double c = cos(p[0] / 2.0), s = sin(p[0] / 2.0);
            const double complex el = iexp(0.0, 1.0, p[2]);
            const double complex ep = iexp(0.0, 1.0, p[1]);
            const double complex epl = iexp(0.0, 1.0, p[1] + p[2]);
            put(out, 0, c, 0.0);
            put(out, 1, (-creal(el)) * s, (-cimag(el)) * s);
            put(out, 2, creal(ep) * s, cimag(ep) * s);
            put(out, 3, creal(epl) * c, cimag(epl) * c);
            return 2;
        }
        case 15: /* CX (control bit 0, target bit 1) */
            put(out, 0, 1.0, 0.0); put(out, 7, 1.0, 0.0); put(out, 10, 1.0, 0.0); put(out, 13, 1.0, 0.0);
            return 4;
        case 16: /* CZ */
            put(out, 0, 1.0, 0.0); put(out, 5, 1.0, 0.0); put(out, 10, 1.0, 0.0); put(out, 15, -1.0, 0.0);
            return 4;
        case 17: /* SWAP */
            put(out, 0, 1.0, 0.0); put(out, 6, 1.0, 0.0); put(out, 9, 1.0, 0.0); put(out, 15, 1.0, 0.0);
            return 4;
        case 18: { /* CP */
            const double complex b = iexp(0.0, 1.0, p[0]);
            put(out, 0, 1.0, 0.0); put(out, 5, 1.0, 0.0); put(out, 10, 1.0, 0.0);
            put(out, 15, creal(b), cimag(b));
            return 4;
        }
        case 19: { /* RZZ: same = exp(-0.5i*t), diff = exp(0.5i*t) */
            const double complex same = iexp(-0.0, -0.5, p[0]);
            const double complex diff = iexp(0.0, 0.5, p[0]);
            put(out, 0, creal(same), cimag(same)); put(out, 5, creal(diff), cimag(diff));
            put(out, 10, creal(diff), cimag(diff)); put(out, 15, creal(same), cimag(same));
            return 4;
        }
        case 20: /* CCX */
            for (int i = 0; i < 8; ++i) put(out, i * 8 + i, 1.0, 0.0);
            put(out, 3 * 8 + 3, 0.0, 0.0); put(out, 7 * 8 + 7, 0.0, 0.0);
            put(out, 3 * 8 + 7, 1.0, 0.0); put(out, 7 * 8 + 3, 1.0, 0.0);
            return 8;
        default:
            return 0;
    }
}

int orc_gate_num_params(int opcode) {
    switch (opcode) {
        case 10: case 11: case 12: case 13: case 18: case 19: return 1;
        case 14: return 3;
        default: return 0;
    }
}

int orc_gate_num_qubits(int opcode) {
    if (opcode <= 14) return 1;
    if (opcode <= 19) return 2;
    if (opcode == 20) return 3;
    return 0;
}

/* ------------------------------------------------------------------------
 * The generic kernel: src/kernels/cpu/dense_kernels.cpp:465-524.
 * state: 2*n_amps doubles (interleaved); matrix: 2*4^k doubles row-major.
 * ---------------------------------------------------------------------- */
void orc_apply_generic(double* state, uint64_t n_amps, const double* matrix,
                       const uint32_t* operands, uint32_t k) {
    const uint64_t dim = 1ULL << k;
    int n = 0;
    while ((1ULL << n) < n_amps) ++n;
    uint64_t mask = 0;
    for (uint32_t j = 0; j < k; ++j) mask |= 1ULL << operands[j];
    const uint64_t n_outer = n_amps >> k;
    uint64_t idx[64];
    double g[128];
    for (uint64_t compact = 0; compact < n_outer; ++compact) {
        uint64_t base = 0;
        int src = 0;
        for (int p = 0; p < n; ++p) {
            if ((mask >> p) & 1ULL) continue;
            base |= ((compact >> src) & 1ULL) << p;
            ++src;
        }
        for (uint64_t local = 0; local < dim; ++local) {
            uint64_t i = base;
            for (uint32_t j = 0; j < k; ++j)
                if ((local >> j) & 1ULL) i |= 1ULL << operands[j];
            idx[local] = i;
            g[2 * local] = state[2 * i];
            g[2 * local + 1] = state[2 * i + 1];
        }
        for (uint64_t out = 0; out < dim; ++out) {
            double sr = 0.0, si = 0.0;
            for (uint64_t in = 0; in < dim; ++in) {
                const double mr = matrix[2 * (out * dim + in)], mi = matrix[2 * (out * dim + in) + 1];
                const double ar = g[2 * in], ai = g[2 * in + 1];
                const double pr = mr * ar - mi * ai;
                const double pi = mr * ai + mi * ar;
                sr = sr + pr;
                si = si + pi;
            }
            state[2 * idx[out]] = sr;
            state[2 * idx[out] + 1] = si;
        }
    }
}

/* initialize: src/kernels/cpu/dense_kernels.cpp:21-27. */
void orc_initialize(double* state, uint64_t n_amps, double global_phase) {
    const double complex ph = cexp(CMPLX(0.0, global_phase)); /* std::exp(complex{0.0, phase}) */
    memset(state, 0, sizeof(double) * 2 * n_amps);
    state[0] = creal(ph);
    state[1] = cimag(ph);
}

/* ------------------------------------------------------------------------
 * Expectation of one Pauli term: src/kernels/cpu/dense_kernels.cpp:544-569,
 * sequential in index order, times i^popcount(x & z).
 * ---------------------------------------------------------------------- */
void orc_expectation(const double* state, uint64_t n_amps, uint64_t x, uint64_t z, double* out) {
    double sr = 0.0, si = 0.0;
    for (uint64_t j = 0; j < n_amps; ++j) {
        const uint64_t k = j ^ x;
        const int neg = __builtin_popcountll(z & k) & 1;
        const double ar = state[2 * j], ai = -state[2 * j + 1]; /* conj */
        const double br = state[2 * k], bi = state[2 * k + 1];
        double tr = ar * br - ai * bi;
        double ti = ar * bi + ai * br;
        if (neg) {
            tr = -tr;
            ti = -ti;
        }
        sr = sr + tr;
        si = si + ti;
    }
    const int ph = __builtin_popcountll(x & z) & 3;
    /* i^ph * (sr, si) with std::complex operator*: (a.r*b.r - a.i*b.i, a.r*b.i + a.i*b.r) */
    static const double pr[4] = {1.0, 0.0, -1.0, 0.0};
    static const double pi[4] = {0.0, 1.0, 0.0, -1.0};
    out[0] = pr[ph] * sr - pi[ph] * si;
    out[1] = pr[ph] * si + pi[ph] * sr;
}

/* ------------------------------------------------------------------------
 * Sampling: src/engines/dense/sample.cpp:24-75.  Uniforms from mt19937_64,
 * sorted; one walk `cumulative += re*re + im*im` (std::norm, two roundings);
 * shots past the last cumulative go to the last basis state.  Outcomes are
 * the measured qubits mapped to clbits (targets = (qubit, clbit) pairs),
 * reported in ascending outcome order with their counts.
 * ---------------------------------------------------------------------- */
static int cmp_double(const void* a, const void* b) {
    const double x = *(const double*)a, y = *(const double*)b;
    return (x > y) - (x < y);
}

static int cmp_u64pair(const void* a, const void* b) {
    const uint64_t x = ((const uint64_t*)a)[0], y = ((const uint64_t*)b)[0];
    return (x > y) - (x < y);
}

static uint64_t outcome_of(uint64_t basis, const uint32_t* targets, uint32_t n_targets) {
    uint64_t o = 0;
    for (uint32_t t = 0; t < n_targets; ++t)
        if ((basis >> targets[2 * t]) & 1ULL) o |= 1ULL << targets[2 * t + 1];
    return o;
}

/* Per-shot basis indices in sorted-uniform order (the walk itself). */
void orc_sample_basis(const double* state, uint64_t n_amps, uint64_t shots, uint64_t seed,
                      uint64_t* basis_out) {
    double* u = (double*)malloc(sizeof(double) * (shots ? shots : 1));
    orc_uniforms(seed, shots, u);
    qsort(u, shots, sizeof(double), cmp_double);
    double cumulative = 0.0;
    uint64_t s = 0;
    for (uint64_t b = 0; b < n_amps && s < shots; ++b) {
        const double re = state[2 * b], im = state[2 * b + 1];
        const double p = re * re + im * im;
        cumulative += p;
        while (s < shots && u[s] < cumulative) basis_out[s++] = b;
    }
    while (s < shots) basis_out[s++] = n_amps - 1;
    free(u);
}

/* Returns the number of distinct outcomes, or -1 if cap is too small. */
int64_t orc_sample(const double* state, uint64_t n_amps, uint64_t shots, uint64_t seed,
                   const uint32_t* targets, uint32_t n_targets, uint64_t* outcomes,
                   uint64_t* counts, uint64_t cap) {
    if (shots == 0) return 0;
    uint64_t* basis = (uint64_t*)malloc(sizeof(uint64_t) * shots);
    orc_sample_basis(state, n_amps, shots, seed, basis);
    uint64_t* pairs = (uint64_t*)malloc(sizeof(uint64_t) * 2 * shots);
    for (uint64_t s = 0; s < shots; ++s) {
        pairs[2 * s] = outcome_of(basis[s], targets, n_targets);
        pairs[2 * s + 1] = 1;
    }
    qsort(pairs, shots, 2 * sizeof(uint64_t), cmp_u64pair);
    int64_t d = 0;
    for (uint64_t s = 0; s < shots; ++s) {
        if (d > 0 && outcomes[d - 1] == pairs[2 * s]) {
            counts[d - 1] += 1;
            continue;
        }
        if ((uint64_t)d >= cap) {
            d = -1;
            break;
        }
        outcomes[d] = pairs[2 * s];
        counts[d] = 1;
        ++d;
    }
    free(pairs);
    free(basis);
    return d;
}

/* ------------------------------------------------------------------------
 * Operations and the containment fusion plan: src/ir/fuse_gates.cpp:135-283.
 * Ops are passed as parallel arrays: opcode, nq, qubits (6 per op), params
 * (3 per op), matrices (for UNITARY, 2*4^k doubles each, concatenated in op
 * order).  Opcode 21 = UNITARY, 22 = MEASURE.
 * ---------------------------------------------------------------------- */
typedef struct {
    int opcode;
    uint32_t nq;
    uint32_t q[6];
    double p[3];
    const double* m;
} orc_op;

static int op_is_diagonal(const orc_op* op) {
    /* ir::is_diagonal_operation (src/ir/fuse_diagonal.cpp:16-44,180-193): a
     * named gate by its opcode (Z S Sdg T Tdg RZ P CZ CP RZZ), a UnitaryOp by
     * its matrix (every off-diagonal entry exactly zero). */
    if (op->opcode != 21) {
        switch (op->opcode) {
            case 2: case 4: case 5: case 6: case 7: case 12: case 13: case 16: case 18: case 19: return 1;
            default: return 0;
        }
    }
    const double* m = op->m;
    const uint32_t dim = 1u << op->nq;
    for (uint32_t r = 0; r < dim; ++r)
        for (uint32_t c = 0; c < dim; ++c)
            if (r != c && (m[2 * (r * dim + c)] != 0.0 || m[2 * (r * dim + c) + 1] != 0.0)) return 0;
    return 1;
}

static int may_join(uint64_t block, int block_diag, uint64_t gate, int gate_diag) {
    if (block == gate) return 1;
    if ((block & gate) == block) return !gate_diag || block_diag;
    if ((block & gate) == gate) return !block_diag || gate_diag;
    return 0;
}

static void unpack_ops(uint32_t n_ops, const int32_t* opcode, const uint32_t* nq, const uint32_t* qubits,
                       const double* params, const double* matrices, orc_op* ops) {
    const double* mp = matrices;
    for (uint32_t i = 0; i < n_ops; ++i) {
        ops[i].opcode = opcode[i];
        ops[i].nq = nq[i];
        for (int j = 0; j < 6; ++j) ops[i].q[j] = qubits[6 * i + j];
        for (int j = 0; j < 3; ++j) ops[i].p[j] = params[3 * i + j];
        ops[i].m = NULL;
        if (opcode[i] == 21) {
            ops[i].m = mp;
            mp += 2 * (1u << nq[i]) * (1u << nq[i]);
        }
    }
}

/* Fills block_of[i] for every op; returns the block count.  block_mask and
 * block_diag are per block (capacity n_ops). */
static uint32_t plan_blocks(uint32_t n_ops, const orc_op* ops, uint32_t* block_of, uint64_t* block_mask,
                            unsigned char* block_diag) {
    const uint32_t none = 0xFFFFFFFFu;
    uint32_t newest[64];
    for (int q = 0; q < 64; ++q) newest[q] = none;
    uint32_t blocks = 0;
    for (uint32_t i = 0; i < n_ops; ++i) {
        if (ops[i].opcode == 22) {
            block_of[i] = blocks;
            block_mask[blocks] = 0;
            block_diag[blocks] = 0;
            ++blocks;
            for (int q = 0; q < 64; ++q) newest[q] = none;
            continue;
        }
        uint64_t mask = 0;
        for (uint32_t j = 0; j < ops[i].nq; ++j) mask |= 1ULL << ops[i].q[j];
        const int diag = op_is_diagonal(&ops[i]);
        uint32_t dep = none;
        for (uint64_t rest = mask; rest; rest &= rest - 1) {
            const uint32_t b = newest[__builtin_ctzll(rest)];
            if (b != none && (dep == none || b > dep)) dep = b;
        }
        uint32_t b;
        if (dep != none && may_join(block_mask[dep], block_diag[dep], mask, diag)) {
            b = dep;
            block_mask[b] |= mask;
            block_diag[b] = (unsigned char)(block_diag[b] && diag);
        } else {
            b = blocks++;
            block_mask[b] = mask;
            block_diag[b] = (unsigned char)diag;
        }
        block_of[i] = b;
        for (uint64_t rest = mask; rest; rest &= rest - 1) newest[__builtin_ctzll(rest)] = b;
    }
    return blocks;
}

/* Builds the block's matrix as fused_block_matrix does
 * (src/engines/dense/fused_block.cpp:61-99): the generic kernel on each
 * identity column, member gates in order on local operands, then a
 * transpose.  Returns k. */
static uint32_t fused_matrix(uint64_t block_mask, uint32_t n_members, const uint32_t* members,
                             const orc_op* ops, double* out) {
    uint32_t bq[64];
    uint32_t k = 0;
    for (uint64_t rest = block_mask; rest; rest &= rest - 1) bq[k++] = (uint32_t)__builtin_ctzll(rest);
    const uint64_t dim = 1ULL << k;
    memset(out, 0, sizeof(double) * 2 * dim * dim);
    for (uint64_t c = 0; c < dim; ++c) out[2 * (c * dim + c)] = 1.0;
    double gm[2 * 64 * 64];
    for (uint32_t mi = 0; mi < n_members; ++mi) {
        const orc_op* op = &ops[members[mi]];
        const double* m;
        if (op->opcode == 21) {
            m = op->m;
        } else {
            orc_gate_matrix(op->opcode, op->p, gm);
            m = gm;
        }
        uint32_t local[6];
        for (uint32_t j = 0; j < op->nq; ++j) {
            for (uint32_t t = 0; t < k; ++t)
                if (bq[t] == op->q[j]) local[j] = t;
        }
        for (uint64_t c = 0; c < dim; ++c) orc_apply_generic(out + 2 * c * dim, dim, m, local, op->nq);
    }
    for (uint64_t r = 0; r < dim; ++r)
        for (uint64_t c = r + 1; c < dim; ++c) {
            double t0 = out[2 * (r * dim + c)], t1 = out[2 * (r * dim + c) + 1];
            out[2 * (r * dim + c)] = out[2 * (c * dim + r)];
            out[2 * (r * dim + c) + 1] = out[2 * (c * dim + r) + 1];
            out[2 * (c * dim + r)] = t0;
            out[2 * (c * dim + r) + 1] = t1;
        }
    return k;
}

/* The containment plan as CSR arrays (the FusionPlan fields).  Returns the
 * block count.  Capacities: order n_ops, block_begin n_ops+1,
 * block_qubits 64*n_ops, qubits_begin n_ops+1. */
int64_t orc_plan_fusion(uint32_t n_ops, const int32_t* opcode, const uint32_t* nq, const uint32_t* qubits,
                        const double* params, const double* matrices, uint32_t* order,
                        uint32_t* block_begin, uint32_t* block_qubits, uint32_t* qubits_begin) {
    orc_op* ops = (orc_op*)malloc(sizeof(orc_op) * (n_ops ? n_ops : 1));
    unpack_ops(n_ops, opcode, nq, qubits, params, matrices, ops);
    uint32_t* block_of = (uint32_t*)malloc(sizeof(uint32_t) * (n_ops ? n_ops : 1));
    uint64_t* block_mask = (uint64_t*)malloc(sizeof(uint64_t) * (n_ops ? n_ops : 1));
    unsigned char* block_diag = (unsigned char*)malloc(n_ops ? n_ops : 1);
    const uint32_t blocks = plan_blocks(n_ops, ops, block_of, block_mask, block_diag);
    for (uint32_t b = 0; b <= blocks; ++b) block_begin[b] = 0;
    for (uint32_t i = 0; i < n_ops; ++i) block_begin[block_of[i] + 1]++;
    for (uint32_t b = 0; b < blocks; ++b) block_begin[b + 1] += block_begin[b];
    uint32_t* fill = (uint32_t*)malloc(sizeof(uint32_t) * (blocks ? blocks : 1));
    for (uint32_t b = 0; b < blocks; ++b) fill[b] = block_begin[b];
    for (uint32_t i = 0; i < n_ops; ++i) order[fill[block_of[i]]++] = i;
    qubits_begin[0] = 0;
    for (uint32_t b = 0; b < blocks; ++b) {
        uint32_t at = qubits_begin[b];
        for (uint64_t rest = block_mask[b]; rest; rest &= rest - 1) block_qubits[at++] = (uint32_t)__builtin_ctzll(rest);
        qubits_begin[b + 1] = at;
    }
    free(fill);
    free(block_diag);
    free(block_mask);
    free(block_of);
    free(ops);
    return blocks;
}

/* ------------------------------------------------------------------------
 * DenseEngine::execute restated (src/engines/dense/dense_engine.cpp:333-400):
 * init, then every block (fuse_gates) or every op in order, then the
 * outputs.  Returns 0, or -1 on a malformed op.
 * ---------------------------------------------------------------------- */
int orc_run(uint32_t num_qubits, uint32_t n_ops, const int32_t* opcode, const uint32_t* nq,
            const uint32_t* qubits, const double* params, const double* matrices, double global_phase,
            int fuse_gates, double* state /* 2 * 2^n, output */) {
    const uint64_t n_amps = 1ULL << num_qubits;
    orc_op* ops = (orc_op*)malloc(sizeof(orc_op) * (n_ops ? n_ops : 1));
    unpack_ops(n_ops, opcode, nq, qubits, params, matrices, ops);
    orc_initialize(state, n_amps, global_phase);
    double* m = (double*)malloc(sizeof(double) * 2 * 64 * 64);
    if (!fuse_gates) {
        for (uint32_t i = 0; i < n_ops; ++i) {
            if (ops[i].opcode == 22) continue;
            const double* mat = ops[i].m;
            if (ops[i].opcode != 21) {
                orc_gate_matrix(ops[i].opcode, ops[i].p, m);
                mat = m;
            }
            orc_apply_generic(state, n_amps, mat, ops[i].q, ops[i].nq);
        }
    } else {
        uint32_t* block_of = (uint32_t*)malloc(sizeof(uint32_t) * (n_ops ? n_ops : 1));
        uint64_t* block_mask = (uint64_t*)malloc(sizeof(uint64_t) * (n_ops ? n_ops : 1));
        unsigned char* block_diag = (unsigned char*)malloc(n_ops ? n_ops : 1);
        uint32_t* members = (uint32_t*)malloc(sizeof(uint32_t) * (n_ops ? n_ops : 1));
        const uint32_t blocks = plan_blocks(n_ops, ops, block_of, block_mask, block_diag);
        for (uint32_t b = 0; b < blocks; ++b) {
            uint32_t cnt = 0;
            for (uint32_t i = 0; i < n_ops; ++i)
                if (block_of[i] == b) members[cnt++] = i;
            if (cnt == 0 || block_mask[b] == 0) continue; /* barrier */
            if (cnt == 1) {
                const orc_op* op = &ops[members[0]];
                const double* mat = op->m;
                if (op->opcode != 21) {
                    orc_gate_matrix(op->opcode, op->p, m);
                    mat = m;
                }
                orc_apply_generic(state, n_amps, mat, op->q, op->nq);
            } else {
                uint32_t bq[64];
                uint32_t k = 0;
                for (uint64_t rest = block_mask[b]; rest; rest &= rest - 1) bq[k++] = (uint32_t)__builtin_ctzll(rest);
                fused_matrix(block_mask[b], cnt, members, ops, m);
                orc_apply_generic(state, n_amps, m, bq, k);
            }
        }
        free(members);
        free(block_diag);
        free(block_mask);
        free(block_of);
    }
    free(m);
    free(ops);
    return 0;
}

/* One fused block's matrix for the plan of the given ops (for pinning
 * against the reference's fused_block_matrix).  Returns its dimension. */
int orc_fused_block_matrix(uint32_t n_ops, const int32_t* opcode, const uint32_t* nq, const uint32_t* qubits,
                           const double* params, const double* matrices, uint32_t block, double* out) {
    orc_op* ops = (orc_op*)malloc(sizeof(orc_op) * (n_ops ? n_ops : 1));
    unpack_ops(n_ops, opcode, nq, qubits, params, matrices, ops);
    uint32_t* block_of = (uint32_t*)malloc(sizeof(uint32_t) * (n_ops ? n_ops : 1));
    uint64_t* block_mask = (uint64_t*)malloc(sizeof(uint64_t) * (n_ops ? n_ops : 1));
    unsigned char* block_diag = (unsigned char*)malloc(n_ops ? n_ops : 1);
    uint32_t* members = (uint32_t*)malloc(sizeof(uint32_t) * (n_ops ? n_ops : 1));
    plan_blocks(n_ops, ops, block_of, block_mask, block_diag);
    uint32_t cnt = 0;
    for (uint32_t i = 0; i < n_ops; ++i)
        if (block_of[i] == block) members[cnt++] = i;
    const uint32_t k = fused_matrix(block_mask[block], cnt, members, ops, out);
    free(members);
    free(block_diag);
    free(block_mask);
    free(block_of);
    free(ops);
    return (int)(1u << k);
}
