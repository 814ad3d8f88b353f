// Encoder of the complex128 tile kernel's compact instruction stream (the
// format is described with the opcodes in mb2_internal.h).
//
// Besides the one-to-one translation of the planned instructions, one rewrite
// is made: a run of consecutive diagonal blocks whose entries are all +1 or
// -1 becomes one sign instruction.  Such a block only flips the sign of the
// amplitudes where a boolean function of its operand bits is 1; written in
// algebraic normal form that function is an XOR of AND-monomials, and the
// blocks of a run compose by XOR-ing their monomials (pairs cancel).
// Negation is exact and sign flips commute, so the state is the one the
// blocks give one by one (up to the sign of zero results, which the store
// normalises, as for every specialisation of the per-gate arithmetic).
#include <algorithm>
#include <cstdint>
#include <map>
#include <stdexcept>
#include <vector>

#include "mb2_internal.h"

namespace mb2 {
namespace {

uint32_t pair_index(uint32_t p0, uint32_t p1) { return p0 * 3 + (p1 < p0 ? p1 : p1 - 1); }

// op, aux, an operand position (0-31: bits 16-19 and 31) and the staged data
// offset in 16-byte units (bits 20-30).
uint32_t header(uint32_t op, uint32_t aux, uint32_t tbit, uint32_t off_doubles) {
    if (off_doubles & 1u) throw std::logic_error("staged data offset is not 16-byte aligned");
    const uint32_t off = off_doubles / 2;
    if (off >= 2048u || aux > 255u || tbit > 31u)
        throw std::invalid_argument("pass data beyond the compact stream's reach");
    return op | (aux << 8) | ((tbit & 15u) << 16) | (off << 20) | ((tbit >> 4) << 31);
}

bool is_param(const TileInstr& g) {
    return g.op != TOP_PHASE && g.op != TOP_END && g.op != TOP_MMA && g.nthread != 0;
}

// Doubles of a parametric instruction's per-binding record.
uint32_t param_doubles(const TileInstr& g) {
    const uint32_t dim = 1u << g.k;
    return g.op == TOP_DIAG ? 2 * dim : 2 * dim * dim;
}

// Rewrites runs of U3 words on slots 0-1-2-3, 0-1, 1-2-3 or 0-1-2 whose
// matrices are consecutive (8 doubles apart) into one run word, in the
// words from `begin` on.
void fuse_u3_runs(std::vector<uint32_t>& w, size_t begin) {
    std::vector<uint32_t> out(w.begin(), w.begin() + static_cast<long>(begin));
    size_t i = begin;
    auto is_u3 = [&](size_t k, uint32_t slot) { return k < w.size() && (w[k] & 0xffu) == cop::kU3 + slot; };
    auto off = [&](size_t k) { return (w[k] >> 20) & 0x7ffu; };
    auto chain = [&](size_t k, uint32_t first, uint32_t len) {
        for (uint32_t t = 0; t < len; ++t) {
            if (!is_u3(k + t, first + t)) return false;
            if (t > 0 && off(k + t) != off(k) + 4 * t) return false;
        }
        return true;
    };
    while (i < w.size()) {
        const uint32_t op = w[i] & 0xffu;
        // Skip over multi-word instructions unchanged.
        uint32_t len = 1;
        if (op == cop::kPhase) len = cop::kPhaseWords;
        else if (op == cop::kSmem) len = 3;
        else if ((op >= cop::kMono2 && op < cop::kSw12) || op == cop::kDs2TT || op == cop::kDiagK) len = 2;
        else if (op == cop::kSigns) len = 1 + ((w[i] >> 8) & 0xffu);
        else if (op == cop::kSignsW) len = 1 + 2 * ((w[i] >> 8) & 0xffu);
        if (op == cop::kU3 && chain(i, 0, 4)) {
            out.push_back((w[i] & ~0xffu) | cop::kU3Run0123);
            i += 4;
        } else if (op == cop::kU3 && chain(i, 0, 3)) {
            out.push_back((w[i] & ~0xffu) | cop::kU3Run012);
            i += 3;
        } else if (op == cop::kU3 && chain(i, 0, 2)) {
            out.push_back((w[i] & ~0xffu) | cop::kU3Run01);
            i += 2;
        } else if (op == cop::kU3 + 1 && chain(i, 1, 3)) {
            out.push_back((w[i] & ~0xffu) | cop::kU3Run123);
            i += 3;
        } else {
            out.insert(out.end(), w.begin() + static_cast<long>(i), w.begin() + static_cast<long>(i + len));
            i += len;
        }
    }
    w.swap(out);
}

}  // namespace

void encode_compact(TileProgram& prog) {
    prog.words.clear();
    for (TilePass& pass : prog.passes) {
        pass.word_begin = static_cast<uint32_t>(prog.words.size());
        const TileInstr* ins = prog.instrs.data() + pass.prog_begin;
        const double* sdata = prog.data.data() + pass.sdata_begin;
        // The parametric slice this pass reads.
        uint32_t lo = UINT32_MAX, hi = 0;
        for (uint32_t i = 0; i < pass.prog_count; ++i)
            if (is_param(ins[i])) {
                lo = std::min(lo, ins[i].data);
                hi = std::max(hi, ins[i].data + param_doubles(ins[i]));
            }
        pass.param_lo = lo == UINT32_MAX ? 0u : lo;
        pass.param_len = lo == UINT32_MAX ? 0u : hi - lo;
        auto data_off = [&](const TileInstr& g) {
            return is_param(g) ? pass.sdata_count + (g.data - pass.param_lo) : g.data;
        };
        auto& w = prog.words;
        bool heavy = false, heavy_other = false;  // other: beyond general dense 2q
        uint32_t reg[kRegQubits] = {0, 1, 2, 3};
        // A diagonal of at most two operands by entry class.
        auto emit_dsmall = [&](const TileInstr& g, uint32_t off) {
            const uint32_t c0 = g.pos[4], c1 = g.pos[5];
            const bool r0 = (c0 & 0x80u) != 0, r1 = (c1 & 0x80u) != 0;
            const uint32_t cls = g.aux & 255u;
            if (g.k == 1) {
                if (r0) w.push_back(header(cop::kDs1R + (c0 & 3u), cls, 0, off));
                else w.push_back(header(cop::kDs1T, cls, c0, off));
            } else if (r0 && r1) {
                w.push_back(header(cop::kDs2RR + pair_index(c0 & 3u, c1 & 3u), cls, 0, off));
            } else if (r0) {
                w.push_back(header(cop::kDs2RT + 2 * (c0 & 3u) + 1, cls, c1, off));
            } else if (r1) {
                w.push_back(header(cop::kDs2RT + 2 * (c1 & 3u), cls, c0, off));
            } else {
                w.push_back(header(cop::kDs2TT, cls, 0, off));
                w.push_back((c0 & 15u) | ((c1 & 15u) << 4) | ((c0 >> 4) << 8) | ((c1 >> 4) << 9));
            }
        };
        // Pending sign monomials (register slots | operand bits << 16),
        // toggled so pairs cancel, and the +-1 diagonals they come from.
        std::map<uint64_t, bool> signs;
        std::vector<const TileInstr*> sign_run;
        auto flush_signs = [&]() {
            if (sign_run.size() == 1 && sign_run[0]->kind == TK_DSMALL) {
                // A lone +-1 diagonal of at most two operands keeps its
                // entry-class instruction: it negates only the amplitudes it
                // selects, where a sign instruction passes over all 16.
                const TileInstr& g = *sign_run[0];
                signs.clear();
                sign_run.clear();
                emit_dsmall(g, data_off(g));
                return;
            }
            sign_run.clear();
            std::vector<uint64_t> live;
            bool wide = false;  // a factor outside the tile: two words per monomial
            for (const auto& [mono, on] : signs)
                if (on) {
                    live.push_back(mono);
                    wide = wide || (mono >> 32) != 0;
                }
            signs.clear();
            for (size_t i = 0; i < live.size(); i += 255) {
                const uint32_t cnt = static_cast<uint32_t>(std::min<size_t>(255, live.size() - i));
                w.push_back(header(wide ? cop::kSignsW : cop::kSigns, cnt, 0, 0));
                for (size_t t = i; t < i + cnt; ++t) {
                    if (wide) {
                        w.push_back(static_cast<uint32_t>(live[t] & 0xffffu));
                        w.push_back(static_cast<uint32_t>(live[t] >> 16));
                    } else {
                        w.push_back(static_cast<uint32_t>(live[t]));
                    }
                }
            }
        };
        // Register slot of tile position p in the current phase, -1 for a thread bit.
        auto slot_of = [&](uint32_t p) -> int {
            for (uint32_t s = 0; s < kRegQubits; ++s)
                if (reg[s] == p) return static_cast<int>(s);
            return -1;
        };
        // Adds the sign function of a +-1 diagonal (neg[e]: entry e is -1)
        // on tile positions pos[0..k-1].
        auto add_signs = [&](uint32_t k, const uint32_t* pos, const std::vector<uint8_t>& neg) {
            const uint32_t dim = 1u << k;
            std::vector<uint8_t> c(neg);
            for (uint32_t i = 0; i < k; ++i)
                for (uint32_t s = 0; s < dim; ++s)
                    if (s & (1u << i)) c[s] ^= c[s ^ (1u << i)];
            // Register slot s's bit over the 16 slots j: 0xAAAA, 0xCCCC, 0xF0F0, 0xFF00.
            constexpr uint32_t kSlotBits[kRegQubits] = {0xAAAAu, 0xCCCCu, 0xF0F0u, 0xFF00u};
            for (uint32_t s = 0; s < dim; ++s) {
                if (!c[s]) continue;
                uint64_t slots = 0xffffu, tbits = 0;
                for (uint32_t t = 0; t < k; ++t) {
                    if (!(s & (1u << t))) continue;
                    const int r = slot_of(pos[t]);
                    if (r >= 0) slots &= kSlotBits[r];
                    else tbits |= uint64_t{1} << pos[t];
                }
                const uint64_t mono = slots | (tbits << 16);
                signs[mono] = !signs[mono];
            }
        };
        for (uint32_t i = 0; i < pass.prog_count; ++i) {
            const TileInstr& g = ins[i];
            if (g.op == TOP_DIAG && !is_param(g)) {
                const uint32_t dim = 1u << g.k;
                std::vector<uint8_t> neg(dim, 0);
                bool pm1 = true;
                for (uint32_t e = 0; e < dim && pm1; ++e) {
                    const double re = sdata[g.data + 2 * e], im = sdata[g.data + 2 * e + 1];
                    if (im != 0.0 || (re != 1.0 && re != -1.0)) pm1 = false;
                    neg[e] = re == -1.0;
                }
                if (pm1) {
                    uint32_t pos[8];
                    for (uint32_t t = 0; t < g.k; ++t) pos[t] = g.pos[t];
                    add_signs(g.k, pos, neg);
                    sign_run.push_back(&g);
                    continue;
                }
            }
            flush_signs();
            const uint32_t off =
                (g.op == TOP_PHASE || g.op == TOP_END || g.op == TOP_SMEM || g.op == TOP_MMA) ? 0u : data_off(g);
            switch (g.op) {
                case TOP_PHASE: {
                    uint32_t packed = 0;
                    for (uint32_t s = 0; s < kRegQubits; ++s) {
                        reg[s] = g.pos[s];
                        packed |= static_cast<uint32_t>(g.pos[s]) << (4 * s);
                    }
                    w.push_back(cop::kPhase | (static_cast<uint32_t>(g.nthread) << 8) | (packed << 16));
                    // Slot byte offsets of the register bits (16-byte slots:
                    // tiles of at most 12 qubits; 8-byte slots: at most 13).
                    uint32_t z16[kRegQubits], z8[kRegQubits];
                    for (uint32_t s = 0; s < kRegQubits; ++s) {
                        z16[s] = (swz(1u << g.pos[s]) << 4) & 0xffffu;
                        z8[s] = (swz8(1u << g.pos[s]) << 3) & 0xffffu;
                    }
                    w.push_back(z16[0] | (z16[1] << 16));
                    w.push_back(z16[2] | (z16[3] << 16));
                    w.push_back(z8[0] | (z8[1] << 16));
                    w.push_back(z8[2] | (z8[3] << 16));
                    // Tile bits of each nibble of the thread index.
                    uint32_t et[48] = {};
                    for (uint32_t gi = 0; gi < 3; ++gi)
                        for (uint32_t v = 0; v < 16; ++v)
                            for (uint32_t t = 0; t < 4; ++t) {
                                const uint32_t i = 4 * gi + t;
                                if (i < g.nthread && ((v >> t) & 1u)) et[16 * gi + v] |= 1u << g.tperm[i];
                            }
                    for (uint32_t k = 0; k < 24; ++k) w.push_back(et[2 * k] | (et[2 * k + 1] << 16));
                    break;
                }
                case TOP_END:
                    w.push_back(cop::kEnd);
                    break;
                case TOP_MMA:
                    if (g.aux > 255u) throw std::invalid_argument("too many phase matrices in a pass");
                    w.push_back(cop::kMma | (g.aux << 8));
                    break;
                case TOP_SMEM: {
                    heavy = heavy_other = true;
                    uint32_t packed = 0;
                    for (uint32_t t = 0; t < g.k; ++t) packed |= static_cast<uint32_t>(g.pos[t]) << (4 * t);
                    w.push_back(cop::kSmem | (static_cast<uint32_t>(g.k) << 8));
                    w.push_back(packed);
                    w.push_back(g.data);
                    break;
                }
                case TOP_G1: {
                    // X and monomial rows as general 2x2 products: the zero
                    // entry's product only moves a zero's sign, so the result
                    // is the same, and the kernel's lean variant keeps no
                    // register-moving instructions.
                    const uint32_t p = g.pos[0];
                    switch (g.kind) {
                        case TK_U3: w.push_back(header(cop::kU3 + p, 0, 0, off)); break;
                        case TK_REAL: w.push_back(header(cop::kReal1 + p, 0, 0, off)); break;
                        case TK_X:
                            w.push_back(header(cop::kReal1 + p, 0, 0, off));
                            prog.fp64_per_amp += 6;
                            break;
                        case TK_MONO:
                            w.push_back(header(cop::kGen1 + p, 0, 0, off));
                            prog.fp64_per_amp += 8;
                            break;
                        default: w.push_back(header(cop::kGen1 + p, 0, 0, off)); break;
                    }
                    break;
                }
                case TOP_G2: {
                    heavy = true;  // permutations and monomials move registers: full variant
                    const uint32_t pr = pair_index(g.pos[0], g.pos[1]);
                    if (g.kind != TK_GEN) heavy_other = true;
                    switch (g.kind) {
                        case TK_SW12: w.push_back(header(cop::kSw12 + pr, 0, 0, 0)); break;
                        case TK_SW13: w.push_back(header(cop::kSw13 + pr, 0, 0, 0)); break;
                        case TK_SW23: w.push_back(header(cop::kSw23 + pr, 0, 0, 0)); break;
                        case TK_MONO:
                            w.push_back(header(cop::kMono2 + pr, 0, 0, off));
                            w.push_back(g.aux);
                            break;
                        default: w.push_back(header(cop::kGen2 + pr, 0, 0, off)); break;
                    }
                    break;
                }
                case TOP_DIAG: {
                    if (g.kind == TK_DSMALL) {
                        emit_dsmall(g, off);
                    } else {
                        heavy = heavy_other = true;
                        uint32_t packed = 0;
                        for (uint32_t t = 0; t < g.k; ++t) packed |= static_cast<uint32_t>(g.pos[t]) << (4 * t);
                        w.push_back(header(cop::kDiagK, g.k, 0, off));
                        w.push_back(packed);
                    }
                    break;
                }
                default:
                    throw std::logic_error("unknown tile instruction");
            }
        }
        flush_signs();
        fuse_u3_runs(w, pass.word_begin);
        pass.heavy = heavy;
        pass.mid = heavy && !heavy_other;
        while (w.size() & 3u) w.push_back(cop::kEnd);  // 16-byte multiple: the staged data follows
        pass.word_count = static_cast<uint32_t>(w.size()) - pass.word_begin;
    }
}

}  // namespace mb2
