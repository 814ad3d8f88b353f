// The tensor-core form of the complex64 tile program.
//
// The planner (tile_plan.cpp) gives each pass phases: a phase holds four
// tile qubits in every thread's registers (16 amplitudes per thread) and
// applies the dense one- and two-qubit blocks on them, with diagonal blocks
// on any tile qubits in between.  Here each phase becomes, per thread row of
// 16 amplitudes,
//
//     pre-diagonals,  a <- U a,  post-diagonals
//
// where U is the product (composed in FP64) of the phase's dense blocks and
// of its diagonals on register qubits only.  A diagonal that also involves a
// thread qubit cannot enter U (it differs between rows); it is applied
// elementwise before U when none of its register qubits has been touched by
// a dense block of U yet (it then commutes with everything in U before it),
// else after U, and its register qubits are then closed to further dense
// blocks: a later dense block on one of them starts a new product on the
// same registers (no data movement in between).
//
// a <- U a over the tile's 2^(m-4) rows is a GEMM: rows x (16 complex)
// times U^T, as real operands rows x 32 and 32 x 32 (interleaved re/im).
// The kernel (kernels_tc.cu) runs it on tcgen05 tensor cores with FP16
// operands and FP32 accumulation, each operand split into an FP16 high part
// and an FP16 low part (x = hi + lo to 22 bits; the amplitudes are scaled by
// a power of two first, so their magnitudes sit in FP16's range) and the
// products hi*hi + hi*lo + lo*hi summed; the tile is scaled by a power of
// two once per pass, which needs every block of a tensor-core pass to be
// unitary (it keeps the tile's norm), and U by 2^12 (kTcOperandScale: the
// low part of an entry as small as 2^-14 is still an FP16 normal), undone
// when the product is read back.  This file writes U's operand:
// 64 rows of 32 FP16 values -- rows 0-31 the high parts of U's real form
// (row = output re/im, column = input re/im), rows 32-63 the low parts --
// K-major, no swizzle, in 8-row x 16-byte core matrices: element (n, k) at
// byte (n / 8) * 512 + (k / 8) * 128 + (n % 8) * 16 + (k % 8) * 2, i.e.
// leading (K) byte offset 128 and stride (N) byte offset 512.
#include <algorithm>
#include <bit>
#include <cmath>
#include <cstring>
#include <stdexcept>

#include "mb2_internal.h"

namespace mb2 {
namespace {

constexpr uint32_t kDim = 1u << kRegQubits;  // 16

// IEEE binary16, round to nearest even (subnormals included; |x| must stay
// below 65520).
uint16_t to_half(double x) {
    const uint16_t sign = std::signbit(x) ? 0x8000u : 0u;
    const double a = std::fabs(x);
    if (a == 0.0) return sign;
    int e = 0;
    std::frexp(a, &e);  // a = m 2^e, m in [0.5, 1)
    int biased = e + 14;
    if (biased < 1) return sign | static_cast<uint16_t>(std::nearbyint(std::ldexp(a, 24)));  // k 2^-24
    double sig = std::nearbyint(std::ldexp(a, 11 - e));  // [1024, 2048]
    if (sig == 2048.0) {
        sig = 1024.0;
        ++biased;
    }
    return sign | static_cast<uint16_t>(biased << 10) | static_cast<uint16_t>(static_cast<uint32_t>(sig) - 1024u);
}
double from_half(uint16_t h) {
    const double sign = (h & 0x8000u) ? -1.0 : 1.0;
    const int biased = (h >> 10) & 31;
    const double frac = h & 1023u;
    if (biased == 0) return sign * std::ldexp(frac, -24);
    return sign * std::ldexp(1024.0 + frac, biased - 25);
}

// U <- G U for a dense gate g (dim 2^k, row-major, operand t = register slot sl[t]).
void left_dense(std::vector<Cd>& u, const Cd* g, const uint32_t* sl, uint32_t k) {
    const uint32_t gd = 1u << k;
    uint32_t opm = 0;
    for (uint32_t t = 0; t < k; ++t) opm |= 1u << sl[t];
    std::vector<Cd> in(gd), out(gd);
    for (uint32_t c = 0; c < kDim; ++c) {
        for (uint32_t base = 0; base < kDim; ++base) {
            if (base & opm) continue;
            for (uint32_t e = 0; e < gd; ++e) {
                uint32_t r = base;
                for (uint32_t t = 0; t < k; ++t)
                    if ((e >> t) & 1u) r |= 1u << sl[t];
                in[e] = u[r * kDim + c];
            }
            for (uint32_t o = 0; o < gd; ++o) {
                Cd acc = 0.0;
                for (uint32_t e = 0; e < gd; ++e) acc += g[o * gd + e] * in[e];
                out[o] = acc;
            }
            for (uint32_t o = 0; o < gd; ++o) {
                uint32_t r = base;
                for (uint32_t t = 0; t < k; ++t)
                    if ((o >> t) & 1u) r |= 1u << sl[t];
                u[r * kDim + c] = out[o];
            }
        }
    }
}

// U <- D U for a diagonal d (entries 2^k) on register slots sl.
void left_diag(std::vector<Cd>& u, const Cd* d, const uint32_t* sl, uint32_t k) {
    for (uint32_t r = 0; r < kDim; ++r) {
        uint32_t e = 0;
        for (uint32_t t = 0; t < k; ++t) e |= ((r >> sl[t]) & 1u) << t;
        for (uint32_t c = 0; c < kDim; ++c) u[r * kDim + c] *= d[e];
    }
}

bool is_unitary(const Block& b) {
    const uint32_t dim = 1u << b.k;
    for (uint32_t r = 0; r < dim; ++r)
        for (uint32_t c = 0; c < dim; ++c) {
            Cd dot = 0.0;
            for (uint32_t i = 0; i < dim; ++i) dot += std::conj(b.m[i * dim + r]) * b.m[i * dim + c];
            if (std::abs(dot - (r == c ? Cd(1.0, 0.0) : Cd(0.0, 0.0))) > 1e-10) return false;
        }
    return true;
}

}  // namespace

void tc_operands(const Cd* u, uint32_t* out) {
    auto* h = reinterpret_cast<uint16_t*>(out);  // little-endian: element k even in a word's low half
    for (uint32_t n = 0; n < 32; ++n) {
        for (uint32_t k = 0; k < 32; ++k) {
            // Real form of U: out_re = Re U in_re - Im U in_im, out_im = Im U in_re + Re U in_im,
            // scaled by kTcOperandScale so that the low parts of small entries stay FP16 normals.
            const Cd z = u[(n >> 1) * kDim + (k >> 1)];
            const uint32_t cn = n & 1u, ck = k & 1u;
            const double v = (cn == ck ? z.real() : (cn == 0 ? -z.imag() : z.imag())) * kTcOperandScale;
            const uint16_t hi = to_half(v);
            const uint16_t lo = to_half(v - from_half(hi));
            auto at = [&](uint32_t row) { return (row / 8) * 256 + (k / 8) * 64 + (row % 8) * 8 + (k % 8); };
            h[at(n)] = hi;
            h[at(n + 32)] = lo;
        }
    }
}

namespace {

// One tensor-core phase of a pass: its register positions and, as indices
// into the pass's member list, the diagonals applied before the product,
// the blocks composed into it and the diagonals applied after it.
struct TcPhase {
    uint32_t reg[kRegQubits];
    std::vector<uint32_t> pre, prod, post;
};

// Plans a pass's members (blocks on tile positions, in a dependency order)
// as tensor-core phases.  Each phase takes the register set that lets the
// most dense blocks enter its product (the qubits of the earliest waiting
// dense block first, then grown one qubit at a time), keeping the previous
// set when it does as well (no data movement); then it takes every ready
// block the rules allow -- a dense block or a diagonal on register qubits
// none of which is closed joins the product; a diagonal on none of the
// product's qubits goes before it; any other diagonal goes after it and
// closes its register qubits -- until nothing more is ready.
std::vector<TcPhase> plan_tc_phases(const std::vector<Block>& blocks, const std::vector<uint32_t>& members,
                                    const std::vector<uint32_t>& lp, uint32_t m) {
    const uint32_t nm = static_cast<uint32_t>(members.size());
    std::vector<uint32_t> lmask(nm, 0);
    std::vector<std::vector<uint32_t>> lists(m);
    for (uint32_t i = 0; i < nm; ++i) {
        const Block& b = blocks[members[i]];
        for (uint32_t t = 0; t < b.k; ++t) {
            lmask[i] |= 1u << lp[b.q[t]];
            lists[lp[b.q[t]]].push_back(i);
        }
    }
    std::vector<uint32_t> head(m, 0);
    auto ready = [&](const std::vector<uint32_t>& h, uint32_t i) {
        for (uint32_t p = 0; p < m; ++p)
            if (((lmask[i] >> p) & 1u) && (h[p] >= lists[p].size() || lists[p][h[p]] != i)) return false;
        return true;
    };
    // Takes every block phase `rmask` allows from heads h; returns the dense
    // blocks taken (and the lists when `out`).
    auto take = [&](uint32_t rmask, std::vector<uint32_t>& h, TcPhase* out) {
        uint32_t touched = 0, frozen = 0, dense = 0, total = 0;
        for (bool progress = true; progress;) {
            progress = false;
            for (uint32_t p = 0; p < m; ++p) {
                if (h[p] >= lists[p].size()) continue;
                const uint32_t i = lists[p][h[p]];
                if (!ready(h, i)) continue;
                const Block& b = blocks[members[i]];
                const uint32_t qm = lmask[i];
                const bool in_reg = (qm & ~rmask) == 0 && (qm & frozen) == 0;
                std::vector<uint32_t>* dst = nullptr;
                if (!b.diagonal) {
                    if (!in_reg) continue;
                    dst = out ? &out->prod : nullptr;
                    touched |= qm;
                    ++dense;
                } else if (in_reg) {
                    dst = out ? &out->prod : nullptr;
                    touched |= qm;
                } else if ((qm & rmask & (touched | frozen)) == 0) {
                    dst = out ? &out->pre : nullptr;
                } else {
                    dst = out ? &out->post : nullptr;
                    frozen |= qm & rmask;
                }
                if (dst) dst->push_back(i);
                ++total;
                for (uint32_t q = 0; q < m; ++q)
                    if ((qm >> q) & 1u) ++h[q];
                progress = true;
            }
        }
        return (uint64_t{dense} << 32) | total;
    };
    std::vector<TcPhase> phases;
    uint32_t done = 0, cur = 0;  // cur: the previous phase's register mask
    std::vector<uint32_t> sim;
    while (done < nm) {
        // The earliest waiting dense block seeds the register set.
        uint32_t seed = 0;
        for (uint32_t i = 0; i < nm && seed == 0; ++i) {
            bool waiting = false;
            for (uint32_t p = 0; p < m && !waiting; ++p)
                if (((lmask[i] >> p) & 1u) && head[p] < lists[p].size()) {
                    for (uint32_t k = head[p]; k < lists[p].size(); ++k)
                        if (lists[p][k] == i) waiting = true;
                }
            if (waiting && !blocks[members[i]].diagonal) seed = lmask[i];
        }
        uint32_t rmask = seed;
        while (static_cast<uint32_t>(std::popcount(rmask)) < kRegQubits) {
            uint64_t best_score = 0;
            uint32_t best = m;
            for (uint32_t x = 0; x < m; ++x) {
                if ((rmask >> x) & 1u) continue;
                sim = head;
                const uint64_t sc = take(rmask | (1u << x), sim, nullptr);
                if (best == m || sc > best_score) {
                    best_score = sc;
                    best = x;
                }
            }
            rmask |= 1u << best;
        }
        if (cur != 0 && rmask != cur) {
            sim = head;
            const uint64_t keep = take(cur, sim, nullptr);
            sim = head;
            if ((keep >> 32) >= (take(rmask, sim, nullptr) >> 32)) rmask = cur;
        }
        TcPhase ph;
        uint32_t r = 0;
        for (uint32_t p = 0; p < m; ++p)
            if ((rmask >> p) & 1u) ph.reg[r++] = p;
        const uint64_t got = take(rmask, head, &ph);
        if (static_cast<uint32_t>(got) == 0) throw std::logic_error("tensor-core phase planning made no progress");
        done += static_cast<uint32_t>(got);
        cur = rmask;
        phases.push_back(std::move(ph));
    }
    return phases;
}

}  // namespace

void make_tensor_core_program(TileProgram& prog, const std::vector<Block>& blocks, uint32_t max_phases) {
    if (max_phases == 0) throw std::invalid_argument("max_phases must be positive");
    std::vector<std::vector<uint32_t>> members(prog.passes.size());
    for (size_t i = 0; i < prog.order.size(); ++i) members[prog.order_pass[i]].push_back(prog.order[i]);
    std::vector<TilePass> passes;
    std::vector<TileInstr> instrs;
    std::vector<double> data;
    std::vector<uint32_t>& tcdata = prog.tcdata;
    tcdata.clear();
    prog.tcmatrices.clear();
    for (size_t pi = 0; pi < prog.passes.size(); ++pi) {
        const TilePass& src = prog.passes[pi];
        const std::vector<uint32_t>& mem = members[pi];
        // Convertible: no wide dense or parametric blocks, and every block
        // unitary (to 1e-10): the pass then preserves each tile's norm, which
        // the kernel's FP16 scaling relies on.
        bool convertible = src.param_len == 0 && !mem.empty();
        for (uint32_t i : mem) {
            const Block& b = blocks[i];
            if (!b.diagonal && b.k > 2) convertible = false;
            if (convertible && !is_unitary(b)) convertible = false;
        }
        if (!convertible) {  // kept as it is, for the FP32 SIMT kernel
            const TileInstr* ins = prog.instrs.data() + src.prog_begin;
            const double* sdata = prog.data.data() + src.sdata_begin;
            TilePass p = src;
            p.prog_begin = static_cast<uint32_t>(instrs.size());
            p.sdata_begin = static_cast<uint32_t>(data.size());
            instrs.insert(instrs.end(), ins, ins + src.prog_count);
            data.insert(data.end(), sdata, sdata + src.sdata_count);
            passes.push_back(p);
            continue;
        }
        std::vector<uint32_t> lp(64, 0);
        {
            uint32_t b = 0;
            for (uint32_t q = 0; q < 64; ++q)
                if ((src.smask >> q) & 1u) lp[q] = b++;
        }
        const std::vector<TcPhase> phases = plan_tc_phases(blocks, mem, lp, src.m);
        TilePass cur;
        uint32_t blocks_in = 0;
        auto open_pass = [&]() {
            cur = TilePass{};
            cur.m = src.m;
            cur.smask = src.smask;
            cur.gmask = src.gmask;
            cur.tc = true;
            cur.prog_begin = static_cast<uint32_t>(instrs.size());
            cur.sdata_begin = static_cast<uint32_t>(data.size());
            cur.tc_begin = static_cast<uint32_t>(tcdata.size());
            blocks_in = 0;
        };
        auto close_pass = [&]() {
            cur.gates = blocks_in;
            cur.prog_count = static_cast<uint32_t>(instrs.size()) - cur.prog_begin;
            cur.sdata_count = static_cast<uint32_t>(data.size()) - cur.sdata_begin;
            passes.push_back(cur);
        };
        uint32_t reg[kRegQubits];
        auto emit_phase = [&](const uint32_t* r) {
            TileInstr ph{};
            ph.op = TOP_PHASE;
            for (uint32_t t = 0; t < kRegQubits; ++t) {
                reg[t] = r[t];
                ph.pos[t] = static_cast<uint8_t>(r[t]);
            }
            thread_bit_order(src.m, reg, kRegQubits, ph.tperm, ph.nthread);
            instrs.push_back(ph);
        };
        auto end_phase = [&]() {
            TileInstr e{};
            e.op = TOP_END;
            instrs.push_back(e);
        };
        auto slot_of = [&](uint32_t p) -> int {
            for (uint32_t t = 0; t < kRegQubits; ++t)
                if (reg[t] == p) return static_cast<int>(t);
            return -1;
        };
        // A diagonal block as an elementwise instruction in the open phase.
        auto emit_diag = [&](const Block& b) {
            const uint32_t dim = 1u << b.k;
            TileInstr g{};
            g.op = TOP_DIAG;
            g.k = static_cast<uint8_t>(b.k);
            for (uint32_t t = 0; t < b.k; ++t) g.pos[t] = static_cast<uint8_t>(lp[b.q[t]]);
            g.data = static_cast<uint32_t>(data.size()) - cur.sdata_begin;
            for (uint32_t e = 0; e < dim; ++e) {
                data.push_back(b.m[e * dim + e].real());
                data.push_back(b.m[e * dim + e].imag());
            }
            if (b.k <= 2) {
                g.kind = TK_DSMALL;
                for (uint32_t e = 0; e < dim; ++e) {
                    const Cd d = b.m[e * dim + e];
                    const uint32_t cls = d == Cd(1.0, 0.0) ? 0u : (d == Cd(-1.0, 0.0) ? 1u : 2u);
                    g.aux |= cls << (2 * e);
                }
                for (uint32_t t = 0; t < b.k; ++t) {
                    const int sl = slot_of(g.pos[t]);
                    g.pos[4 + t] = static_cast<uint8_t>(sl >= 0 ? (0x80u | static_cast<uint32_t>(sl)) : g.pos[t]);
                }
            } else {
                g.kind = TK_GEN;
            }
            instrs.push_back(g);
        };
        open_pass();
        bool open = false;
        for (size_t k = 0; k < phases.size(); ++k) {
            const TcPhase& ph = phases[k];
            const bool same = open && std::equal(ph.reg, ph.reg + kRegQubits, reg);
            if (!same) {
                if (open) end_phase();
                emit_phase(ph.reg);
                open = true;
            }
            for (uint32_t i : ph.pre) emit_diag(blocks[mem[i]]);
            if (!ph.prod.empty()) {
                std::vector<Cd> u(kDim * kDim, Cd(0.0, 0.0));
                for (uint32_t d = 0; d < kDim; ++d) u[d * kDim + d] = 1.0;
                for (uint32_t i : ph.prod) {
                    const Block& b = blocks[mem[i]];
                    uint32_t sl[8];
                    for (uint32_t t = 0; t < b.k; ++t) sl[t] = static_cast<uint32_t>(slot_of(lp[b.q[t]]));
                    if (b.diagonal) {
                        const uint32_t dim = 1u << b.k;
                        std::vector<Cd> dg(dim);
                        for (uint32_t e = 0; e < dim; ++e) dg[e] = b.m[e * dim + e];
                        left_diag(u, dg.data(), sl, b.k);
                    } else {
                        left_dense(u, b.m.data(), sl, b.k);
                    }
                }
                if (cur.tc_phases == max_phases) {
                    // Split: the pass goes on in a new pass on the same tile.
                    end_phase();
                    close_pass();
                    open_pass();
                    emit_phase(ph.reg);
                }
                TileInstr mma{};
                mma.op = TOP_MMA;
                mma.aux = cur.tc_phases++;
                instrs.push_back(mma);
                const size_t at = tcdata.size();
                tcdata.resize(at + kTcOperandWords);
                tc_operands(u.data(), tcdata.data() + at);
                prog.tcmatrices.insert(prog.tcmatrices.end(), u.begin(), u.end());
            }
            for (uint32_t i : ph.post) emit_diag(blocks[mem[i]]);
            blocks_in += static_cast<uint32_t>(ph.pre.size() + ph.prod.size() + ph.post.size());
        }
        if (open) end_phase();
        close_pass();
    }
    prog.passes = std::move(passes);
    prog.instrs = std::move(instrs);
    prog.data = std::move(data);
    encode_compact(prog);
}

void run_program_on_host(const TileProgram& prog, uint32_t n, Cd* state) {
    const uint64_t amps = uint64_t{1} << n;
    for (const TilePass& pass : prog.passes) {
        if (pass.param_len != 0) throw std::invalid_argument("parametric passes are not interpreted");
        // Tile position p -> the p-th qubit of the pass's tile.
        std::vector<uint32_t> qubit;
        for (uint32_t q = 0; q < n; ++q)
            if ((pass.smask >> q) & 1u) qubit.push_back(q);
        // A diagonal's operand position: a tile position, or kGlobalPos0 +
        // rank among the outside qubits it reads.
        std::vector<uint32_t> outside;
        for (uint32_t q = 0; q < n; ++q)
            if ((pass.gmask >> q) & 1u) outside.push_back(q);
        auto qubit_at = [&](uint32_t p) { return p >= kGlobalPos0 ? outside.at(p - kGlobalPos0) : qubit.at(p); };
        const TileInstr* ins = prog.instrs.data() + pass.prog_begin;
        const double* sdata = prog.data.data() + pass.sdata_begin;
        uint32_t reg[kRegQubits] = {0, 1, 2, 3};
        for (uint32_t i = 0; i < pass.prog_count; ++i) {
            const TileInstr& g = ins[i];
            uint32_t ops[8];
            switch (g.op) {
                case TOP_PHASE:
                    for (uint32_t s = 0; s < kRegQubits; ++s) reg[s] = g.pos[s];
                    break;
                case TOP_END:
                    break;
                case TOP_MMA: {
                    for (uint32_t s = 0; s < kRegQubits; ++s) ops[s] = qubit[reg[s]];
                    const Cd* u = prog.tcmatrices.data() + size_t{pass.tc_begin / kTcOperandWords + g.aux} * kDim * kDim;
                    host_apply_generic(state, amps, u, ops, kRegQubits);
                    break;
                }
                case TOP_G1:
                case TOP_G2: {
                    for (uint32_t t = 0; t < g.k; ++t) ops[t] = qubit[reg[g.pos[t]]];
                    host_apply_generic(state, amps, reinterpret_cast<const Cd*>(sdata + g.data), ops, g.k);
                    break;
                }
                case TOP_DIAG: {
                    const uint32_t dim = 1u << g.k;
                    std::vector<Cd> m(size_t{dim} * dim, Cd(0.0, 0.0));
                    for (uint32_t e = 0; e < dim; ++e) m[e * dim + e] = Cd(sdata[g.data + 2 * e], sdata[g.data + 2 * e + 1]);
                    for (uint32_t t = 0; t < g.k; ++t) ops[t] = qubit_at(g.pos[t]);
                    host_apply_generic(state, amps, m.data(), ops, g.k);
                    break;
                }
                case TOP_SMEM: {
                    for (uint32_t t = 0; t < g.k; ++t) ops[t] = qubit[g.pos[t]];
                    host_apply_generic(state, amps, reinterpret_cast<const Cd*>(prog.gdata.data() + g.data), ops, g.k);
                    break;
                }
                default:
                    throw std::logic_error("unknown tile instruction");
            }
        }
    }
}

}  // namespace mb2
