// Host planner of the multi-gate tiled sweep.
//
// A pass loads every tile of 2^m amplitudes -- the amplitudes that share
// their bits outside a set S of m qubits -- into shared memory once, applies
// a run of blocks whose operands lie in S, and writes the tile back once.
// A pass applies a run of consecutive blocks, in their order, and per
// amplitude the arithmetic of every block is exactly the per-gate kernel's,
// so the state after the sweep is bitwise the one the reference's
// block-by-block sweep gives
// (src/engines/dense/fused_block.h:60-101, src/engines/dense/dense_engine.cpp:65-112).
//
// Inside a pass each thread holds 16 amplitudes in registers (4 "register
// qubits"); a PHASE instruction picks which 4 tile qubits those are, and the
// blocks of the phase act on registers only.  Diagonal blocks need no pairing
// and run in any phase.  Blocks wider than 2 dense qubits run from shared
// memory (TOP_SMEM).
#include <algorithm>
#include <bit>
#include <cmath>
#include <initializer_list>
#include <stdexcept>

#include "mb2_internal.h"

namespace mb2 {
namespace {

// A pass's instruction words and small-matrix data are staged in shared
// memory (kMaxStagedBytes); a block costs at most a phase record, three
// more words (gate, extra word, end) and its staged entries.
constexpr size_t kMaxBlocksPerPass = 300;

size_t staged_bytes(const Block& b) {
    const size_t dim = size_t{1} << b.k;
    const size_t entries = b.diagonal ? dim : (b.k <= 2 ? dim * dim : 0);
    return (cop::kPhaseWords + 3) * sizeof(uint32_t) + entries * 2 * sizeof(double);
}


uint32_t local_pos(uint64_t smask, uint32_t q) {
    return static_cast<uint32_t>(std::popcount(smask & ((uint64_t{1} << q) - 1)));
}

bool is_real(const Cd& c) { return c.imag() == 0.0; }
bool is_zero(const Cd& c) { return c.real() == 0.0 && c.imag() == 0.0; }

// Row r's single nonzero column, -1 for an all-zero row, -2 if the row has more.
int mono_src(const std::vector<Cd>& m, uint32_t dim, uint32_t r) {
    int src = -1;
    for (uint32_t c = 0; c < dim; ++c) {
        if (!is_zero(m[r * dim + c])) {
            if (src != -1) return -2;
            src = static_cast<int>(c);
        }
    }
    return src;
}

struct PassSel {
    uint64_t smask;
    uint64_t gmask = 0;           // qubits outside the tile that diagonals of the pass read
    std::vector<uint32_t> gates;  // block indices in application order
};

// A diagonal block's operands need not lie in the tile: an amplitude's entry
// depends only on its operand bits, and a qubit outside the tile has one
// value over the whole tile, which the kernel reads off the tile's base
// index.  That holds for the instructions that take an operand as a bit
// value -- diagonals of at most two operands and +-1 diagonals (sign
// monomials) -- not for the wide entry-index diagonal (kDiagK).
bool diagonal_any_operand(const Block& b, bool parametric) {
    if (!b.diagonal) return false;
    if (b.k <= 2) return true;
    if (parametric) return false;
    const uint32_t dim = 1u << b.k;
    for (uint32_t e = 0; e < dim; ++e) {
        const Cd& d = b.m[size_t{e} * dim + e];
        if (d.imag() != 0.0 || (d.real() != 1.0 && d.real() != -1.0)) return false;
    }
    return true;
}

// A diagonal operand's instruction position: its tile position, or
// kGlobalPos0 + its rank among the pass's outside qubits.
uint32_t operand_pos(uint64_t smask, uint64_t gmask, uint32_t q) {
    if ((smask >> q) & 1u) return local_pos(smask, q);
    if (!((gmask >> q) & 1u)) throw std::logic_error("diagonal operand neither in the tile nor global");
    return kGlobalPos0 + static_cast<uint32_t>(std::popcount(gmask & ((uint64_t{1} << q) - 1)));
}

// Passes are maximal runs of CONSECUTIVE blocks whose operands fit one
// tile -- diagonals read up to kMaxGlobalQubits qubits outside it.  Blocks
// are never reordered, not even commuting ones: two gates on disjoint qubits
// applied in the other order give the same state only up to rounding, and
// the plain path is bitwise the reference's sweep, which applies the blocks
// in plan order.
std::vector<PassSel> select_passes(const std::vector<Block>& blocks, uint32_t n, uint32_t m, uint32_t fixed_low,
                                   const std::vector<uint8_t>* parametric) {
    std::vector<PassSel> passes;
    uint32_t widest = 1;
    for (const Block& b : blocks) widest = std::max(widest, b.k);
    const uint32_t mt = std::min(m, n);
    if (widest > mt) throw std::invalid_argument("a block is wider than the tile");
    // Low qubits kept in every tile so that tiles gather contiguous runs,
    // leaving room for the widest block.
    const uint32_t fixed = std::min(fixed_low, mt - widest);
    // Qubits outside the tile that the diagonals read, once the tile is
    // padded to mt qubits with them first.
    auto outside = [&](uint64_t s, uint64_t d) {
        return std::popcount(d & ~s) - (static_cast<int>(mt) - std::popcount(s));
    };
    size_t i = 0;
    while (i < blocks.size()) {
        uint64_t smask = 0, dmask = 0;  // the tile's qubits so far; the diagonals' operands
        for (uint32_t q = 0; q < fixed; ++q) smask |= uint64_t{1} << q;
        PassSel sel;
        size_t staged = 0;
        while (i < blocks.size() && sel.gates.size() < kMaxBlocksPerPass) {
            const bool param = parametric != nullptr && ((*parametric)[i] & kParamBlock) != 0;
            uint64_t s2 = smask, d2 = dmask;
            if (diagonal_any_operand(blocks[i], param)) d2 |= blocks[i].mask();
            else s2 |= blocks[i].mask();
            if (static_cast<uint32_t>(std::popcount(s2)) > mt) break;
            if (outside(s2, d2) > static_cast<int>(kMaxGlobalQubits)) break;
            if (staged + staged_bytes(blocks[i]) > kMaxStagedBytes && !sel.gates.empty()) break;
            staged += staged_bytes(blocks[i]);
            smask = s2;
            dmask = d2;
            sel.gates.push_back(static_cast<uint32_t>(i));
            ++i;
        }
        // Pad the tile to exactly mt qubits: first with the diagonals'
        // operands the global limit leaves out, then with the lowest unused
        // qubits (longer contiguous runs per tile).
        for (uint64_t rest = dmask & ~smask; std::popcount(rest) > static_cast<int>(kMaxGlobalQubits);
             rest &= rest - 1)
            smask |= rest & (~rest + 1);
        for (uint32_t q = 0; q < n && static_cast<uint32_t>(std::popcount(smask)) < mt; ++q)
            smask |= uint64_t{1} << q;
        sel.smask = smask;
        sel.gmask = dmask & ~smask;
        passes.push_back(std::move(sel));
    }
    return passes;
}

uint32_t push_matrix(std::vector<double>& data, const std::vector<Cd>& m) {
    const uint32_t off = static_cast<uint32_t>(data.size());
    for (const Cd& c : m) {
        data.push_back(c.real());
        data.push_back(c.imag());
    }
    return off;
}

}  // namespace

// Thread-bit order for a phase whose register bits are `reg` (tile-local
// positions): the first three thread bits get distinct residues mod 3 when
// possible, so that the eight threads of a quarter warp hit eight distinct
// 16-byte bank groups under the kernel's XOR-fold swizzle.
void thread_bit_order(uint32_t m, const uint32_t* reg, uint32_t nreg, uint8_t* tperm, uint8_t& nthread) {
    std::vector<uint32_t> free_pos;
    for (uint32_t p = 0; p < m; ++p)
        if (std::find(reg, reg + nreg, p) == reg + nreg) free_pos.push_back(p);
    std::vector<uint32_t> order;
    for (uint32_t res = 0; res < 3; ++res) {
        for (uint32_t p : free_pos)
            if (p % 3 == res && std::find(order.begin(), order.end(), p) == order.end()) {
                order.push_back(p);
                break;
            }
    }
    if (order.size() < 3) order.clear();
    for (uint32_t p : free_pos)
        if (std::find(order.begin(), order.end(), p) == order.end()) order.push_back(p);
    nthread = static_cast<uint8_t>(order.size());
    for (size_t i = 0; i < order.size(); ++i) tperm[i] = static_cast<uint8_t>(order[i]);
}

// Passes over a topological order of the blocks' dependencies (two blocks
// depend when they share a qubit; blocks on disjoint qubits commute), for
// the paths that are not bitwise the reference's sweep (complex64).  Each
// pass picks its tile greedily: the qubits of the earliest unapplied block,
// the fixed low qubits, then one qubit at a time the one that lets the most
// blocks run (ties: the one most blocked blocks wait for).  Inside the pass
// the blocks are ordered phase by phase: every ready block that a register
// set of four qubits (or no register at all: diagonals) can take, then the
// next set from the ready dense blocks, so the kernel changes phase rarely.
std::vector<PassSel> select_passes_commuting(const std::vector<Block>& blocks, uint32_t n, uint32_t m,
                                             uint32_t fixed_low) {
    std::vector<PassSel> passes;
    uint32_t widest = 1;
    for (const Block& b : blocks) widest = std::max(widest, b.k);
    const uint32_t mt = std::min(m, n);
    if (widest > mt) throw std::invalid_argument("a block is wider than the tile");
    const uint32_t fixed = std::min(fixed_low, mt - widest);
    const uint32_t nb = static_cast<uint32_t>(blocks.size());
    std::vector<std::vector<uint32_t>> lists(n);
    for (uint32_t i = 0; i < nb; ++i)
        for (uint32_t t = 0; t < blocks[i].k; ++t) lists[blocks[i].q[t]].push_back(i);
    std::vector<uint32_t> head(n, 0);
    auto at_head = [&](const std::vector<uint32_t>& h, uint32_t i) {
        for (uint32_t t = 0; t < blocks[i].k; ++t) {
            const uint32_t y = blocks[i].q[t];
            if (h[y] >= lists[y].size() || lists[y][h[y]] != i) return false;
        }
        return true;
    };
    // Blocks that can run inside tile s from heads h, in a dependency order
    // (h advances past them); stops at the pass limits when `limit`.
    std::vector<uint32_t> work;
    auto closure = [&](uint64_t s, std::vector<uint32_t>& h, std::vector<uint32_t>* out, bool limit) {
        uint32_t count = 0;
        size_t staged = 0;
        work.clear();
        for (uint32_t x = 0; x < n; ++x)
            if ((s >> x) & 1u) work.push_back(x);
        while (!work.empty()) {
            const uint32_t x = work.back();
            work.pop_back();
            if (h[x] >= lists[x].size()) continue;
            const uint32_t i = lists[x][h[x]];
            if ((blocks[i].mask() & ~s) != 0 || !at_head(h, i)) continue;
            if (limit && (count >= kMaxBlocksPerPass ||
                          (count > 0 && staged + staged_bytes(blocks[i]) > kMaxStagedBytes)))
                break;
            staged += staged_bytes(blocks[i]);
            ++count;
            if (out) out->push_back(i);
            for (uint32_t t = 0; t < blocks[i].k; ++t) {
                ++h[blocks[i].q[t]];
                work.push_back(blocks[i].q[t]);
            }
        }
        return count;
    };
    uint32_t applied = 0, first = 0;
    std::vector<uint8_t> done(nb, 0);
    std::vector<uint32_t> h;
    while (applied < nb) {
        while (done[first]) ++first;
        uint64_t s = blocks[first].mask();
        for (uint32_t q = 0; q < fixed; ++q) s |= uint64_t{1} << q;
        while (static_cast<uint32_t>(std::popcount(s)) < mt) {
            uint64_t best_score = 0;
            uint32_t best = n;
            for (uint32_t x = 0; x < n; ++x) {
                if ((s >> x) & 1u) continue;
                h = head;
                const uint64_t runs = closure(s | (uint64_t{1} << x), h, nullptr, false);
                // Blocked blocks at the tile's heads that wait for x.
                uint32_t waits = 0;
                for (uint32_t y = 0; y < n; ++y)
                    if (((s >> y) & 1u) && head[y] < lists[y].size() &&
                        ((blocks[lists[y][head[y]]].mask() >> x) & 1u))
                        ++waits;
                const uint64_t score = (runs << 16) | waits;
                if (best == n || score > best_score) {
                    best_score = score;
                    best = x;
                }
            }
            s |= uint64_t{1} << best;
        }
        std::vector<uint32_t> members;
        h = head;
        closure(s, h, &members, true);
        if (members.empty()) throw std::logic_error("tile selection made no progress");
        // Phase-by-phase order of the members.
        PassSel sel;
        sel.smask = s;
        std::vector<uint8_t> in_pass(nb, 0);
        for (uint32_t i : members) in_pass[i] = 1;
        std::vector<uint32_t> ph = head, sim;
        std::vector<uint8_t> sim_in;
        // Runs every member that register set `regs` can take (diagonals and
        // wide blocks need none), from heads hh, in waves: the ready dense
        // blocks, then the ready diagonals (so that the diagonals of one
        // layer are consecutive and merge), and so on; returns the dense
        // ones run.
        auto run = [&](uint64_t regs, std::vector<uint32_t>& hh, std::vector<uint8_t>& in, std::vector<uint32_t>* out) {
            uint32_t dense = 0;
            for (bool any = true; any;) {
                any = false;
                for (const bool diag : {false, true}) {
                    work.clear();
                    for (uint32_t x = 0; x < n; ++x)
                        if ((s >> x) & 1u) work.push_back(x);
                    while (!work.empty()) {
                        const uint32_t x = work.back();
                        work.pop_back();
                        if (hh[x] >= lists[x].size()) continue;
                        const uint32_t i = lists[x][hh[x]];
                        const Block& b = blocks[i];
                        if (!in[i] || b.diagonal != diag || !at_head(hh, i) ||
                            !(b.diagonal || b.k > 2 || (b.mask() & ~regs) == 0))
                            continue;
                        in[i] = 0;
                        any = true;
                        if (!b.diagonal && b.k <= 2) ++dense;
                        if (out) out->push_back(i);
                        for (uint32_t t = 0; t < b.k; ++t) {
                            ++hh[b.q[t]];
                            work.push_back(b.q[t]);
                        }
                    }
                }
            }
            return dense;
        };
        size_t left = members.size();
        uint64_t regs = 0;
        for (;;) {
            const size_t before = sel.gates.size();
            run(regs, ph, in_pass, &sel.gates);
            left -= sel.gates.size() - before;
            if (left == 0) break;
            // Next register set: grown one qubit at a time by the qubit that
            // lets the most dense blocks run (ties: the one most ready dense
            // blocks use, then the lowest).
            uint64_t cand = 0;
            for (uint32_t i : members)
                if (in_pass[i] && !blocks[i].diagonal && blocks[i].k <= 2) cand |= blocks[i].mask();
            regs = 0;
            for (uint32_t r = 0; r < kRegQubits && (cand & ~regs) != 0; ++r) {
                uint64_t best_score = 0;
                uint32_t best = n;
                for (uint32_t x = 0; x < n; ++x) {
                    if (!((cand >> x) & 1u) || ((regs >> x) & 1u)) continue;
                    sim = ph;
                    sim_in = in_pass;
                    const uint64_t runs = run(regs | (uint64_t{1} << x), sim, sim_in, nullptr);
                    uint32_t uses = 0;
                    for (uint32_t i : members)
                        if (in_pass[i] && !blocks[i].diagonal && blocks[i].k <= 2 && ((blocks[i].mask() >> x) & 1u) &&
                            at_head(ph, i))
                            ++uses;
                    const uint64_t score = (runs << 16) | uses;
                    if (best == n || score > best_score) {
                        best_score = score;
                        best = x;
                    }
                }
                regs |= uint64_t{1} << best;
            }
            if (regs == 0) throw std::logic_error("phase ordering made no progress");
        }
        for (uint32_t i : sel.gates) done[i] = 1;
        applied += static_cast<uint32_t>(sel.gates.size());
        head = ph;
        passes.push_back(std::move(sel));
    }
    return passes;
}

TileProgram plan_tile_program(const std::vector<Block>& blocks, uint32_t n, uint32_t m, uint32_t fixed_low,
                              const std::vector<uint8_t>* parametric, bool commuting) {
    if (m < kMinTileQubits || m > kMaxTileQubitsC64) throw std::invalid_argument("tile width out of range");
    TileProgram prog;
    const uint32_t mt = std::min(m, n);
    if (mt < kRegQubits) throw std::invalid_argument("state too small for the tile kernel");
    const std::vector<PassSel> sels =
        commuting ? select_passes_commuting(blocks, n, mt, fixed_low)
                  : select_passes(blocks, n, mt, fixed_low, parametric);
    prog.param_offsets.assign(blocks.size(), 0);
    auto param_flags = [&](uint32_t bi) -> uint8_t { return parametric ? (*parametric)[bi] : uint8_t{0}; };
    // A parametric block's data goes to the per-binding record.
    auto push_param = [&](uint32_t bi, uint32_t doubles) {
        const uint32_t off = prog.param_stride;
        prog.param_offsets[bi] = off;
        prog.param_stride += (doubles + 1) & ~1u;  // keep 16-byte alignment
        return off;
    };
    for (const PassSel& sel : sels) {
        TilePass pass;
        pass.m = mt;
        pass.smask = sel.smask;
        pass.gmask = sel.gmask;
        pass.prog_begin = static_cast<uint32_t>(prog.instrs.size());
        pass.sdata_begin = static_cast<uint32_t>(prog.data.size());
        pass.gates = static_cast<uint32_t>(sel.gates.size());
        auto push_staged = [&](const std::vector<Cd>& m) {
            return push_matrix(prog.data, m) - pass.sdata_begin;
        };

        bool open = false;
        uint32_t reg[kRegQubits];
        for (uint32_t r = 0; r < kRegQubits; ++r) reg[r] = r;
        auto in_reg = [&](uint32_t p) -> int {
            for (uint32_t s = 0; s < kRegQubits; ++s)
                if (reg[s] == p) return static_cast<int>(s);
            return -1;
        };
        auto close_phase = [&]() {
            if (open) {
                TileInstr e{};
                e.op = TOP_END;
                prog.instrs.push_back(e);
                open = false;
            }
        };
        // Opens a phase whose registers hold `first` (in order), filled from
        // the dense 1q/2q blocks that follow position `from` in this pass.
        auto open_phase = [&](const std::vector<uint32_t>& first, size_t from) {
            close_phase();
            std::vector<uint32_t> r(first);
            for (size_t j = from; j < sel.gates.size() && r.size() < kRegQubits; ++j) {
                const Block& b = blocks[sel.gates[j]];
                if (b.diagonal || b.k > 2) continue;
                bool fits = true;
                uint32_t extra = 0;
                for (uint32_t t = 0; t < b.k; ++t)
                    if (std::find(r.begin(), r.end(), local_pos(sel.smask, b.q[t])) == r.end()) ++extra;
                if (r.size() + extra > kRegQubits) fits = false;
                if (!fits) continue;
                for (uint32_t t = 0; t < b.k; ++t) {
                    const uint32_t p = local_pos(sel.smask, b.q[t]);
                    if (std::find(r.begin(), r.end(), p) == r.end()) r.push_back(p);
                }
            }
            for (uint32_t p = 0; p < mt && r.size() < kRegQubits; ++p)
                if (std::find(r.begin(), r.end(), p) == r.end()) r.push_back(p);
            for (uint32_t s = 0; s < kRegQubits; ++s) reg[s] = r[s];
            TileInstr ph{};
            ph.op = TOP_PHASE;
            for (uint32_t s = 0; s < kRegQubits; ++s) ph.pos[s] = static_cast<uint8_t>(reg[s]);
            thread_bit_order(mt, reg, kRegQubits, ph.tperm, ph.nthread);
            prog.instrs.push_back(ph);
            open = true;
        };

        // A small diagonal's operand sources, decided here once: pos[4 + b]
        // = 0x80 | register slot, or the operand's tile bit (a thread bit).
        auto encode_sources = [&](TileInstr& g, uint32_t k) {
            for (uint32_t t = 0; t < k; ++t) {
                const int slot = in_reg(g.pos[t]);
                g.pos[4 + t] = static_cast<uint8_t>(slot >= 0 ? (0x80u | static_cast<uint32_t>(slot)) : g.pos[t]);
            }
        };
        for (size_t j = 0; j < sel.gates.size(); ++j) {
            const Block& b = blocks[sel.gates[j]];
            const uint32_t dim = 1u << b.k;
            prog.order.push_back(sel.gates[j]);
            prog.order_pass.push_back(static_cast<uint32_t>(prog.passes.size()));
            TileInstr g{};
            g.k = static_cast<uint8_t>(b.k);
            if (b.diagonal) {
                if (!open) open_phase({}, j + 1);
                g.op = TOP_DIAG;
                for (uint32_t t = 0; t < b.k; ++t)
                    g.pos[t] = static_cast<uint8_t>(operand_pos(sel.smask, sel.gmask, b.q[t]));
                std::vector<Cd> d(dim);
                for (uint32_t i = 0; i < dim; ++i) d[i] = b.m[i * dim + i];
                if (param_flags(sel.gates[j]) & kParamBlock) {
                    g.nthread = 1;
                    g.data = push_param(sel.gates[j], 2 * dim);
                    g.kind = b.k <= 2 ? TK_DSMALL : TK_GEN;
                    if (b.k <= 2) {
                        for (uint32_t i = 0; i < dim; ++i) g.aux |= 2u << (2 * i);  // every entry multiplies
                        encode_sources(g, b.k);
                    }
                    prog.fp64_per_amp += 6;
                    prog.instrs.push_back(g);
                    continue;
                }
                g.data = push_staged(d);
                if (b.k <= 2) {
                    // Entry classes: (1,0) copies, (-1,0) negates, the rest multiply.
                    g.kind = TK_DSMALL;
                    uint32_t gen = 0;
                    for (uint32_t i = 0; i < dim; ++i) {
                        uint32_t cls = 2;
                        if (d[i].imag() == 0.0 && d[i].real() == 1.0) cls = 0;
                        else if (d[i].imag() == 0.0 && d[i].real() == -1.0) cls = 1;
                        if (cls == 2) ++gen;
                        g.aux |= cls << (2 * i);
                    }
                    prog.fp64_per_amp += (6 * gen + dim - 1) / dim;
                    encode_sources(g, b.k);
                } else {
                    g.kind = TK_GEN;
                    prog.fp64_per_amp += 6;
                }
                prog.instrs.push_back(g);
                continue;
            }
            if (b.k <= 2) {
                int slot[2] = {-1, -1};
                bool have = open;
                for (uint32_t t = 0; t < b.k && have; ++t) {
                    slot[t] = in_reg(local_pos(sel.smask, b.q[t]));
                    if (slot[t] < 0) have = false;
                }
                if (!have) {
                    std::vector<uint32_t> first;
                    for (uint32_t t = 0; t < b.k; ++t) first.push_back(local_pos(sel.smask, b.q[t]));
                    open_phase(first, j + 1);
                    for (uint32_t t = 0; t < b.k; ++t) slot[t] = in_reg(local_pos(sel.smask, b.q[t]));
                }
                g.op = b.k == 1 ? TOP_G1 : TOP_G2;
                g.pos[0] = static_cast<uint8_t>(slot[0]);
                if (b.k == 2) g.pos[1] = static_cast<uint8_t>(slot[1]);
                // Specialisations, each exact up to the sign of zero results
                // (normalised at the store): monomial rows, real entries.
                const uint8_t pf = param_flags(sel.gates[j]);
                bool mono = (pf & kParamBlock) == 0;
                uint32_t aux = 0;
                for (uint32_t r = 0; r < dim && mono; ++r) {
                    const int s = mono_src(b.m, dim, r);
                    if (s == -2) {
                        mono = false;
                        break;
                    }
                    aux |= static_cast<uint32_t>(s < 0 ? 7 : s) << (3 * r);
                }
                if (mono) {
                    g.kind = TK_MONO;
                    g.aux = aux;
                    // Exact permutations run as register moves.
                    bool ones = true;
                    for (uint32_t r = 0; r < dim; ++r) {
                        const uint32_t src = (aux >> (3 * r)) & 7u;
                        if (src == 7u || b.m[r * dim + src] != Cd(1.0, 0.0) || std::signbit(b.m[r * dim + src].imag()))
                            ones = false;
                    }
                    auto is_perm = [&](std::initializer_list<uint32_t> srcs) {
                        uint32_t r = 0;
                        for (uint32_t v : srcs)
                            if (((aux >> (3 * r++)) & 7u) != v) return false;
                        return true;
                    };
                    if (ones && b.k == 1 && is_perm({1, 0})) g.kind = TK_X;
                    else if (ones && b.k == 2 && is_perm({0, 2, 1, 3})) g.kind = TK_SW12;
                    else if (ones && b.k == 2 && is_perm({0, 3, 2, 1})) g.kind = TK_SW13;
                    else if (ones && b.k == 2 && is_perm({0, 1, 3, 2})) g.kind = TK_SW23;
                    prog.fp64_per_amp += (g.kind == TK_MONO) ? 6 : 0;
                } else if (b.k == 1) {
                    bool all_real = is_real(b.m[0]) && is_real(b.m[1]) && is_real(b.m[2]) && is_real(b.m[3]);
                    bool m00_real = is_real(b.m[0]);
                    if (pf & kParamBlock) {  // what holds for every binding
                        all_real = (pf & kParamAllReal) != 0;
                        m00_real = (pf & kParamM00Real) != 0;
                    }
                    if (all_real) {
                        g.kind = TK_REAL;
                        prog.fp64_per_amp += 6;
                    } else if (m00_real) {
                        g.kind = TK_U3;
                        prog.fp64_per_amp += 12;
                    } else {
                        g.kind = TK_GEN;
                        prog.fp64_per_amp += 14;
                    }
                } else {
                    g.kind = TK_GEN;
                    prog.fp64_per_amp += 30;
                }
                if (pf & kParamBlock) {
                    g.nthread = 1;
                    g.data = push_param(sel.gates[j], 2 * dim * dim);
                } else {
                    g.data = push_staged(b.m);
                }
                prog.instrs.push_back(g);
                continue;
            }
            // Wider dense block: from shared memory, as a phase of its own.
            close_phase();
            g.op = TOP_SMEM;
            for (uint32_t t = 0; t < b.k; ++t) g.pos[t] = static_cast<uint8_t>(local_pos(sel.smask, b.q[t]));
            if (param_flags(sel.gates[j]) & kParamBlock)
                throw std::invalid_argument("parametric blocks wider than 2 qubits are not batched");
            g.data = push_matrix(prog.gdata, b.m);
            prog.instrs.push_back(g);
            prog.fp64_per_amp += 8ull * dim - 2;
        }
        close_phase();
        pass.prog_count = static_cast<uint32_t>(prog.instrs.size()) - pass.prog_begin;
        pass.sdata_count = static_cast<uint32_t>(prog.data.size()) - pass.sdata_begin;
        prog.passes.push_back(pass);
    }
    encode_compact(prog);
    return prog;
}

}  // namespace mb2
