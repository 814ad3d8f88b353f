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
// The kernel (kernels_tc.cu) runs it on tcgen05 tensor cores in TF32 with
// FP32 accumulation, splitting both operands into a TF32 high part and a
// TF32 low part (x = hi + lo to ~22 bits) and summing hi*hi + hi*lo + lo*hi.
// This file writes U's split operands in the shared-memory layout the MMA
// reads: K-major, no swizzle, 8x16-byte core matrices -- element (n, k) at
// byte (n / 8) * 1024 + (k / 4) * 128 + (n % 8) * 16 + (k % 4) * 4, i.e.
// leading (K) byte offset 128 and stride (N) byte offset 1024.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>

#include "mb2_internal.h"

namespace mb2 {
namespace {

constexpr uint32_t kDim = 1u << kRegQubits;  // 16

// Round to TF32 (10 explicit mantissa bits), nearest-even.
float to_tf32(double x) {
    float f = static_cast<float>(x);
    uint32_t u;
    std::memcpy(&u, &f, 4);
    if ((u & 0x7f800000u) != 0x7f800000u) {
        u += 0x0fffu + ((u >> 13) & 1u);
        u &= 0xffffe000u;
    }
    std::memcpy(&f, &u, 4);
    return f;
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

}  // namespace

void tc_operands(const Cd* u, float* out) {
    float* hi = out;
    float* lo = out + kTcMatrixFloats / 2;
    for (uint32_t n = 0; n < 32; ++n) {
        for (uint32_t k = 0; k < 32; ++k) {
            // Real form of U: out_re = Re U in_re - Im U in_im, out_im = Im U in_re + Re U in_im.
            const Cd z = u[(n >> 1) * kDim + (k >> 1)];
            const uint32_t cn = n & 1u, ck = k & 1u;
            const double v = cn == ck ? z.real() : (cn == 0 ? -z.imag() : z.imag());
            const uint32_t at = (n / 8) * 256 + (k / 4) * 32 + (n % 8) * 4 + (k % 4);
            hi[at] = to_tf32(v);
            lo[at] = to_tf32(v - static_cast<double>(hi[at]));
        }
    }
}

void make_tensor_core_program(TileProgram& prog, uint32_t max_phases) {
    if (max_phases == 0) throw std::invalid_argument("max_phases must be positive");
    std::vector<TilePass> passes;
    std::vector<TileInstr> instrs;
    std::vector<double> data;
    std::vector<float>& tcdata = prog.tcdata;
    tcdata.clear();
    prog.tcmatrices.clear();
    for (const TilePass& src : prog.passes) {
        const TileInstr* ins = prog.instrs.data() + src.prog_begin;
        const double* sdata = prog.data.data() + src.sdata_begin;
        bool convertible = src.param_len == 0;
        for (uint32_t i = 0; i < src.prog_count && convertible; ++i)
            if (ins[i].op == TOP_SMEM || (ins[i].op != TOP_PHASE && ins[i].op != TOP_END && ins[i].nthread != 0))
                convertible = false;
        if (!convertible) {  // kept as it is, for the FP32 SIMT kernel
            TilePass p = src;
            p.prog_begin = static_cast<uint32_t>(instrs.size());
            p.sdata_begin = static_cast<uint32_t>(data.size());
            instrs.insert(instrs.end(), ins, ins + src.prog_count);
            data.insert(data.end(), sdata, sdata + src.sdata_count);
            passes.push_back(p);
            continue;
        }
        TilePass cur;
        const TileInstr* phase_instr = nullptr;  // the open phase's PHASE instruction
        // Blocks read so far; a split pass reports the blocks it read.
        uint32_t blocks_read = 0, blocks_at_open = 0;
        auto open_pass = [&]() {
            cur = TilePass{};
            cur.m = src.m;
            cur.smask = src.smask;
            blocks_at_open = blocks_read;
            cur.tc = true;
            cur.prog_begin = static_cast<uint32_t>(instrs.size());
            cur.sdata_begin = static_cast<uint32_t>(data.size());
            cur.tc_begin = static_cast<uint32_t>(tcdata.size());
        };
        auto close_pass = [&]() {
            cur.gates = blocks_read - blocks_at_open;
            cur.prog_count = static_cast<uint32_t>(instrs.size()) - cur.prog_begin;
            cur.sdata_count = static_cast<uint32_t>(data.size()) - cur.sdata_begin;
            passes.push_back(cur);
        };
        // A diagonal instruction copied with its entries restaged.
        auto push_diag = [&](const TileInstr& g) {
            TileInstr d = g;
            d.data = static_cast<uint32_t>(data.size()) - cur.sdata_begin;
            const uint32_t n = 2u << g.k;
            data.insert(data.end(), sdata + g.data, sdata + g.data + n);
            instrs.push_back(d);
        };
        std::vector<Cd> u;
        bool have_u = false;
        uint32_t touched = 0, frozen = 0;  // register slots
        std::vector<const TileInstr*> pre, post;
        auto reset = [&]() {
            u.assign(kDim * kDim, Cd(0.0, 0.0));
            for (uint32_t i = 0; i < kDim; ++i) u[i * kDim + i] = 1.0;
            have_u = false;
            touched = frozen = 0;
            pre.clear();
            post.clear();
        };
        // Emits the open product: pre-diagonals, the matrix, post-diagonals.
        auto flush = [&]() {
            for (const TileInstr* g : pre) push_diag(*g);
            if (have_u) {
                if (cur.tc_phases == max_phases) {
                    // Split: this phase goes on in a new pass on the same tile.
                    TileInstr e{};
                    e.op = TOP_END;
                    instrs.push_back(e);
                    close_pass();
                    open_pass();
                    instrs.push_back(*phase_instr);
                }
                TileInstr mma{};
                mma.op = TOP_MMA;
                mma.aux = cur.tc_phases++;
                instrs.push_back(mma);
                const size_t at = tcdata.size();
                tcdata.resize(at + kTcMatrixFloats);
                tc_operands(u.data(), tcdata.data() + at);
                prog.tcmatrices.insert(prog.tcmatrices.end(), u.begin(), u.end());
            }
            for (const TileInstr* g : post) push_diag(*g);
            reset();
        };
        open_pass();
        reset();
        uint32_t reg[kRegQubits] = {0, 1, 2, 3};
        auto slot_of = [&](uint32_t p) -> int {
            for (uint32_t s = 0; s < kRegQubits; ++s)
                if (reg[s] == p) return static_cast<int>(s);
            return -1;
        };
        for (uint32_t i = 0; i < src.prog_count; ++i) {
            const TileInstr& g = ins[i];
            switch (g.op) {
                case TOP_PHASE:
                    flush();
                    phase_instr = &g;
                    for (uint32_t s = 0; s < kRegQubits; ++s) reg[s] = g.pos[s];
                    instrs.push_back(g);
                    break;
                case TOP_END:
                    flush();
                    instrs.push_back(g);
                    break;
                case TOP_G1:
                case TOP_G2: {
                    ++blocks_read;
                    uint32_t sl[2] = {g.pos[0], g.pos[1]}, msk = 0;
                    for (uint32_t t = 0; t < g.k; ++t) msk |= 1u << sl[t];
                    if (msk & frozen) flush();
                    const Cd* gm = reinterpret_cast<const Cd*>(sdata + g.data);
                    left_dense(u, gm, sl, g.k);
                    have_u = true;
                    touched |= msk;
                    break;
                }
                case TOP_DIAG: {
                    ++blocks_read;
                    uint32_t sl[8], msk = 0;
                    bool all_reg = true;
                    for (uint32_t t = 0; t < g.k; ++t) {
                        const int s = slot_of(g.pos[t]);
                        if (s < 0) {
                            all_reg = false;
                        } else {
                            sl[t] = static_cast<uint32_t>(s);
                            msk |= 1u << s;
                        }
                    }
                    if (all_reg && (msk & frozen) == 0) {
                        std::vector<Cd> d(1u << g.k);
                        for (uint32_t e = 0; e < d.size(); ++e) d[e] = Cd(sdata[g.data + 2 * e], sdata[g.data + 2 * e + 1]);
                        left_diag(u, d.data(), sl, g.k);
                        have_u = true;
                        touched |= msk;
                    } else if ((msk & (touched | frozen)) == 0) {
                        pre.push_back(&g);
                    } else {
                        post.push_back(&g);
                        frozen |= msk;
                    }
                    break;
                }
                default:
                    throw std::logic_error("unexpected instruction in a tensor-core pass");
            }
        }
        flush();
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
                    const Cd* u = prog.tcmatrices.data() + size_t{pass.tc_begin / kTcMatrixFloats + g.aux} * kDim * kDim;
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
                    for (uint32_t t = 0; t < g.k; ++t) ops[t] = qubit[g.pos[t]];
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
