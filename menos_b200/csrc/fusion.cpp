// Operations -> blocks.  The reference's gate-fusion plan by containment
// (src/ir/fuse_gates.cpp:109-147 shape/may_join, :190-283 plan_fusion) and
// its fused block matrices (src/engines/dense/fused_block.cpp:61-99), so the
// blocks this engine applies are the same matrices on the same operands as
// the reference CPU and CUDA engines apply: results stay bitwise identical
// with fusion on.
//
// Wider fusion (width k >= 2) keeps the plan's structure -- a gate joins the
// newest open block that shares a qubit with it, blocks run in the order they
// opened, a MeasureOp closes every block -- and only changes the join rule:
// the gate joins when the block and the gate together span at most k qubits.
// The structure is what makes any join rule sound: every block opened after
// the one the gate joins is on qubits disjoint from the gate's, so it
// commutes with it.  The plan (FusionPlan's arrays) can be handed to the
// reference's own block sweep (engines::dense::apply_blocks), which then
// computes the same bits.
#include <algorithm>
#include <array>
#include <stdexcept>
#include <string>

#include "mb2_internal.h"

namespace mb2 {

bool is_diagonal(const std::vector<Cd>& m, uint32_t dim) {
    for (uint32_t r = 0; r < dim; ++r)
        for (uint32_t c = 0; c < dim; ++c)
            if (r != c && (m[r * dim + c].real() != 0.0 || m[r * dim + c].imag() != 0.0)) return false;
    return true;
}

void host_apply_generic(Cd* state, uint64_t n_amps, const Cd* matrix, const uint32_t* operands,
                        uint32_t k) {
    // kernels::cpu::apply_matrix_generic (src/kernels/cpu/dense_kernels.cpp:465-524):
    // out = (+0) + sum_in m[out][in] * a[in], increasing in; std::complex
    // operator* and += with no contraction (this file is built -ffp-contract=off).
    const uint64_t dim = uint64_t{1} << k;
    int n = 0;
    while ((uint64_t{1} << n) < n_amps) ++n;
    uint64_t mask = 0;
    for (uint32_t j = 0; j < k; ++j) mask |= uint64_t{1} << operands[j];
    const uint64_t n_outer = n_amps >> k;
    std::vector<uint64_t> idx(dim);
    std::vector<Cd> g(dim);
    for (uint64_t compact = 0; compact < n_outer; ++compact) {
        uint64_t base = 0;
        int src = 0;
        for (int p = 0; p < n; ++p) {
            if ((mask >> p) & 1u) continue;
            base |= ((compact >> src) & uint64_t{1}) << p;
            ++src;
        }
        for (uint64_t local = 0; local < dim; ++local) {
            uint64_t i = base;
            for (uint32_t j = 0; j < k; ++j)
                if ((local >> j) & 1u) i |= uint64_t{1} << operands[j];
            idx[local] = i;
            g[local] = state[i];
        }
        for (uint64_t out = 0; out < dim; ++out) {
            Cd sum{0.0, 0.0};
            for (uint64_t in = 0; in < dim; ++in) sum += matrix[out * dim + in] * g[in];
            state[idx[out]] = sum;
        }
    }
}

namespace {

// ir::is_diagonal_operation (src/ir/fuse_diagonal.cpp:16-32, 180-193): a named
// gate by its opcode, a UnitaryOp by its matrix.
bool diagonal_opcode(int opcode) {
    switch (opcode) {
        case MB2_Z: case MB2_S: case MB2_SDG: case MB2_T: case MB2_TDG: case MB2_RZ: case MB2_P:
        case MB2_CZ: case MB2_CP: case MB2_RZZ:
            return true;
        default:
            return false;
    }
}

struct OpView {
    bool is_gate = false;
    uint32_t k = 0;
    const uint32_t* q = nullptr;
    std::vector<Cd> m;  // the op's own matrix
    bool fusion_diagonal = false;
    uint64_t mask = 0;
};

OpView view_of(const mb2_op& op, uint32_t index) {
    OpView v;
    if (op.opcode == MB2_MEASURE) return v;
    if (op.opcode == MB2_CHANNEL)
        throw std::invalid_argument("operation " + std::to_string(index) +
                                    ": a noise channel needs the density-matrix path (mb2_dm_apply_program)");
    if (op.opcode < 0 || op.opcode > MB2_UNITARY)
        throw std::invalid_argument("operation " + std::to_string(index) + ": unknown opcode");
    if (op.opcode == MB2_UNITARY) {
        if (op.num_qubits < 1 || op.num_qubits > MB2_MAX_OP_QUBITS || op.matrix == nullptr)
            throw std::invalid_argument("operation " + std::to_string(index) + ": bad unitary");
        const uint32_t dim = 1u << op.num_qubits;
        v.m.resize(size_t{dim} * dim);
        for (size_t i = 0; i < v.m.size(); ++i) v.m[i] = Cd{op.matrix[2 * i], op.matrix[2 * i + 1]};
        v.fusion_diagonal = is_diagonal(v.m, dim);
    } else {
        if (op.num_qubits != static_cast<uint32_t>(gate_num_qubits(op.opcode)))
            throw std::invalid_argument("operation " + std::to_string(index) + ": operand count");
        gate_matrix(op.opcode, op.params, v.m);
        v.fusion_diagonal = diagonal_opcode(op.opcode);
    }
    v.is_gate = true;
    v.k = op.num_qubits;
    v.q = op.qubits;
    for (uint32_t j = 0; j < v.k; ++j) {
        if (op.qubits[j] >= 64) throw std::invalid_argument("operation " + std::to_string(index) + ": operand >= 64");
        if (v.mask & (uint64_t{1} << op.qubits[j]))
            throw std::invalid_argument("operation " + std::to_string(index) + ": repeated operand");
        v.mask |= uint64_t{1} << op.qubits[j];
    }
    return v;
}

// may_join (src/ir/fuse_gates.cpp:135-147).
bool may_join(uint64_t block, bool block_diagonal, uint64_t gate, bool gate_diagonal) {
    if (block == gate) return true;
    if ((block & gate) == block) return !gate_diagonal || block_diagonal;
    if ((block & gate) == gate) return !block_diagonal || gate_diagonal;
    return false;
}

}  // namespace

std::vector<Block> build_blocks(const mb2_op* ops, uint32_t n_ops, bool fuse_gates, uint32_t width,
                                FusionPlanArrays* plan_out) {
    if (width == 1 || width > MB2_MAX_OP_QUBITS) throw std::invalid_argument("fusion width must be 0 or 2..6");
    std::vector<OpView> views;
    views.reserve(n_ops);
    for (uint32_t i = 0; i < n_ops; ++i) views.push_back(view_of(ops[i], i));

    auto own_block = [](const OpView& v) {
        Block b;
        b.k = v.k;
        std::copy(v.q, v.q + v.k, b.q);
        b.m = v.m;
        b.diagonal = is_diagonal(b.m, 1u << b.k);
        return b;
    };

    std::vector<Block> out;
    if (!fuse_gates) {
        for (const OpView& v : views)
            if (v.is_gate) out.push_back(own_block(v));
        return out;
    }

    // plan_fusion: each gate joins the newest open block sharing a qubit
    // when may_join allows; a MeasureOp is a barrier that closes every block.
    constexpr uint32_t kNone = 0xFFFFFFFFu;
    std::vector<uint32_t> block_of(n_ops, kNone);
    std::vector<uint64_t> block_mask;
    std::vector<unsigned char> block_diag;
    std::array<uint32_t, 64> newest;
    newest.fill(kNone);
    for (uint32_t i = 0; i < n_ops; ++i) {
        const OpView& v = views[i];
        if (!v.is_gate) {
            block_of[i] = static_cast<uint32_t>(block_mask.size());
            block_mask.push_back(0);
            block_diag.push_back(0);
            newest.fill(kNone);
            continue;
        }
        uint32_t dep = kNone;
        for (uint64_t rest = v.mask; rest != 0; rest &= rest - 1) {
            const uint32_t b = newest[__builtin_ctzll(rest)];
            if (b != kNone && (dep == kNone || b > dep)) dep = b;
        }
        uint32_t b;
        const bool join = dep != kNone && (width == 0 ? may_join(block_mask[dep], block_diag[dep] != 0, v.mask,
                                                                  v.fusion_diagonal)
                                                       : __builtin_popcountll(block_mask[dep] | v.mask) <=
                                                             static_cast<int>(width));
        if (join) {
            b = dep;
            block_mask[b] |= v.mask;
            block_diag[b] = static_cast<unsigned char>(block_diag[b] != 0 && v.fusion_diagonal);
        } else {
            b = static_cast<uint32_t>(block_mask.size());
            block_mask.push_back(v.mask);
            block_diag.push_back(v.fusion_diagonal ? 1 : 0);
        }
        block_of[i] = b;
        for (uint64_t rest = v.mask; rest != 0; rest &= rest - 1) newest[__builtin_ctzll(rest)] = b;
    }

    // Members of each block in op order (a stable counting sort, as the plan's order).
    const uint32_t blocks = static_cast<uint32_t>(block_mask.size());
    std::vector<std::vector<uint32_t>> members(blocks);
    for (uint32_t i = 0; i < n_ops; ++i) members[block_of[i]].push_back(i);
    if (plan_out != nullptr) {
        *plan_out = FusionPlanArrays{};
        plan_out->block_begin.push_back(0);
        plan_out->qubits_begin.push_back(0);
        for (uint32_t b = 0; b < blocks; ++b) {
            plan_out->order.insert(plan_out->order.end(), members[b].begin(), members[b].end());
            plan_out->block_begin.push_back(static_cast<uint32_t>(plan_out->order.size()));
            for (uint64_t rest = block_mask[b]; rest != 0; rest &= rest - 1)
                plan_out->block_qubits.push_back(static_cast<uint32_t>(__builtin_ctzll(rest)));
            plan_out->qubits_begin.push_back(static_cast<uint32_t>(plan_out->block_qubits.size()));
        }
    }

    for (uint32_t b = 0; b < blocks; ++b) {
        if (block_mask[b] == 0) continue;  // barrier
        if (members[b].size() == 1) {
            // The gate's own operand order, not the block's ascending list.
            out.push_back(own_block(views[members[b][0]]));
            continue;
        }
        // fused_block_matrix: the generic kernel on each basis column, member
        // gates in order on local (ascending block) operands, then transposed.
        Block blk;
        uint32_t bq[64];
        uint32_t k = 0;
        for (uint64_t rest = block_mask[b]; rest != 0; rest &= rest - 1)
            bq[k++] = static_cast<uint32_t>(__builtin_ctzll(rest));
        if (k > MB2_MAX_OP_QUBITS) throw std::invalid_argument("fused block wider than 6 qubits");
        const uint32_t dim = 1u << k;
        std::vector<Cd> cols(size_t{dim} * dim, Cd{0.0, 0.0});
        for (uint32_t c = 0; c < dim; ++c) cols[size_t{c} * dim + c] = Cd{1.0, 0.0};
        for (const uint32_t index : members[b]) {
            const OpView& v = views[index];
            uint32_t local[MB2_MAX_OP_QUBITS];
            for (uint32_t j = 0; j < v.k; ++j)
                local[j] = static_cast<uint32_t>(std::find(bq, bq + k, v.q[j]) - bq);
            for (uint32_t c = 0; c < dim; ++c)
                host_apply_generic(cols.data() + size_t{c} * dim, dim, v.m.data(), local, v.k);
        }
        for (uint32_t r = 0; r < dim; ++r)
            for (uint32_t c = r + 1; c < dim; ++c) std::swap(cols[size_t{r} * dim + c], cols[size_t{c} * dim + r]);
        blk.k = k;
        std::copy(bq, bq + k, blk.q);
        blk.m = std::move(cols);
        blk.diagonal = is_diagonal(blk.m, dim);
        blk.members = static_cast<uint32_t>(members[b].size());
        out.push_back(std::move(blk));
    }
    return out;
}

}  // namespace mb2
