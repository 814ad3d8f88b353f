// Batched parameter sweep (mb2_sweep_batch): one circuit structure under many
// parameter bindings in one device job.
//
// Each binding's blocks are built on the host exactly as a single run builds
// them (gate matrices from the same libm calls, the same fusion plan and
// fused matrices), so every binding's state is bitwise the state the
// reference computes for that binding alone.  All bindings share one tile
// program; blocks whose matrices differ between bindings read their entries
// from a per-binding record selected by the tile's binding index.  The
// expectation is the grouped Pauli reduction over every binding's state
// (kernels_reduce.cu); states under 11 qubits take one 8-CTA cluster per
// binding (kernels_batch.cu).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "mb2_internal.h"

namespace mb2 {
int launch_batch_init(void* amps, uint32_t n, uint64_t bindings, double re, double im, void* stream,
                      int precision);
int launch_batch_expect(const void* amps, uint32_t n, uint64_t bindings, const uint64_t* dev_x,
                        const uint64_t* dev_z, const double* dev_coefs, uint32_t num_terms, double* dev_out,
                        void* stream, int precision);
int launch_pauli_group_batch(const void* amps, uint32_t n, uint32_t c, uint32_t d, const uint64_t* dev_span,
                             uint64_t free_mask, const void* dev_terms, uint32_t nterms, uint64_t bindings,
                             uint32_t per, double* dev_partials, int sm_count, void* stream, int precision);
int launch_batch_group_finish(const double* dev_partials, uint64_t bindings, uint32_t per, const uint64_t* dev_x,
                              const uint64_t* dev_z, const double* dev_coefs, uint32_t num_terms, double* dev_out,
                              void* stream);
}  // namespace mb2

namespace {

// The blocks of binding b: ops with their parameters taken, in op order,
// from params.
std::vector<mb2::Block> binding_blocks(const mb2_op* ops, uint32_t num_ops, const double* params, bool fuse) {
    std::vector<mb2_op> mine(ops, ops + num_ops);
    uint32_t k = 0;
    for (mb2_op& o : mine) {
        if (o.opcode == MB2_MEASURE || o.opcode == MB2_UNITARY) continue;
        const int np = mb2::gate_num_params(o.opcode);
        for (int p = 0; p < np; ++p) o.params[p] = params[k++];
    }
    return mb2::build_blocks(mine.data(), num_ops, fuse);
}

uint32_t param_slots(const mb2_op* ops, uint32_t num_ops) {
    uint32_t k = 0;
    for (uint32_t i = 0; i < num_ops; ++i)
        if (ops[i].opcode != MB2_MEASURE && ops[i].opcode != MB2_UNITARY) k += mb2::gate_num_params(ops[i].opcode);
    return k;
}

struct Runner {
    int device;
    cudaStream_t stream = nullptr;
    void* state = nullptr;
    void* work = nullptr;
    ~Runner() {
        if (stream) cudaStreamSynchronize(stream);
        if (state) cudaFree(state);
        if (work) cudaFree(work);
        if (stream) cudaStreamDestroy(stream);
    }
};

}  // namespace

extern "C" int mb2_sweep_batch(mb2_context* ctx, const mb2_op* ops, uint32_t num_ops, uint32_t num_qubits,
                               const double* params, uint32_t params_per_binding, uint32_t num_bindings,
                               const uint64_t* x_masks, const uint64_t* z_masks, const double* coefs,
                               uint32_t num_terms, const mb2_batch_options* opts, double* out,
                               double* states_out, mb2_batch_stats* stats) {
    if (ctx == nullptr || out == nullptr || (ops == nullptr && num_ops != 0)) return MB2_ERR_INVALID;
    if (num_bindings == 0) return MB2_OK;
    if (num_qubits < mb2::kMinTileQubits || num_qubits > 16) return MB2_ERR_INVALID;
    if (num_terms > mb2::kMaxBatchTerms || (num_terms > 0 && (!x_masks || !z_masks || !coefs))) return MB2_ERR_INVALID;
    if (param_slots(ops, num_ops) != params_per_binding || (params_per_binding > 0 && params == nullptr))
        return MB2_ERR_INVALID;
    for (uint32_t i = 0; i < num_ops; ++i) {
        if (ops[i].opcode == MB2_MEASURE) continue;
        if (ops[i].num_qubits == 0 || ops[i].num_qubits > MB2_MAX_OP_QUBITS) return MB2_ERR_INVALID;
        for (uint32_t j = 0; j < ops[i].num_qubits; ++j)
            if (ops[i].qubits[j] >= num_qubits) return MB2_ERR_INVALID;
    }
    const uint64_t lim = (uint64_t{1} << num_qubits) - 1;
    for (uint32_t t = 0; t < num_terms; ++t)
        if ((x_masks[t] | z_masks[t]) & ~lim) return MB2_ERR_INVALID;
    mb2_batch_options o{MB2_C128, 0, 0, 0};
    if (opts != nullptr) o = *opts;
    if (o.precision != MB2_C128 && o.precision != MB2_C64) return MB2_ERR_INVALID;
    const bool c64 = o.precision == MB2_C64;
    const bool fuse = o.fuse_gates != 0;

    // ---- host: the shared block structure and, per block, whether it is
    // parametric and what holds for every binding (threads over bindings).
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const unsigned nt = std::min<unsigned>(hw, num_bindings);
    auto parallel = [&](auto&& body) {  // body(worker) for workers 0..nt-1; false on any exception
        std::vector<std::thread> pool;
        std::vector<std::string> errors(nt);
        for (unsigned w = 0; w < nt; ++w)
            pool.emplace_back([&, w]() {
                try {
                    body(w);
                } catch (const std::exception& e) {
                    errors[w] = e.what();
                }
            });
        for (auto& th : pool) th.join();
        for (const auto& e : errors)
            if (!e.empty()) return false;
        return true;
    };
    std::vector<mb2::Block> shape;
    std::vector<std::vector<mb2::Block>> per;  // every binding's blocks (fused batches only)
    // Unfused: block i is gate op i; only gates with parameters can differ,
    // and their matrices are built per binding from the gate table.
    std::vector<uint32_t> gate_op, gate_pofs;
    try {
        shape = binding_blocks(ops, num_ops, params, fuse);
    } catch (const std::exception&) {
        return MB2_ERR_INVALID;
    }
    const size_t nb = shape.size();
    std::vector<uint8_t> flags(nb, 0);
    if (!fuse) {
        uint32_t k = 0;
        for (uint32_t i = 0; i < num_ops; ++i) {
            if (ops[i].opcode == MB2_MEASURE) continue;
            gate_op.push_back(i);
            gate_pofs.push_back(k);
            if (ops[i].opcode != MB2_UNITARY) k += static_cast<uint32_t>(mb2::gate_num_params(ops[i].opcode));
        }
        if (gate_op.size() != nb) return MB2_ERR_INVALID;
        // Per worker: differs / all_real / m00_real / all_diag per block.
        std::vector<std::vector<uint8_t>> acc(nt, std::vector<uint8_t>(4 * nb, 0));
        const bool ok = parallel([&](unsigned w) {
            std::vector<mb2::Cd> m;
            auto& f = acc[w];
            for (size_t i = 0; i < nb; ++i) f[4 * i + 1] = f[4 * i + 2] = f[4 * i + 3] = 1;
            for (uint32_t b = w; b < num_bindings; b += nt) {
                const double* pb = params + size_t{b} * params_per_binding;
                for (size_t i = 0; i < nb; ++i) {
                    const mb2_op& o = ops[gate_op[i]];
                    const int np = o.opcode == MB2_UNITARY ? 0 : mb2::gate_num_params(o.opcode);
                    if (np == 0) continue;
                    if (mb2::gate_matrix(o.opcode, pb + gate_pofs[i], m) == 0)
                        throw std::invalid_argument("gate matrix");
                    const uint32_t dim = 1u << shape[i].k;
                    if (std::memcmp(m.data(), shape[i].m.data(), m.size() * sizeof(mb2::Cd)) != 0) f[4 * i] = 1;
                    for (const mb2::Cd& c : m) f[4 * i + 1] &= c.imag() == 0.0 ? 1 : 0;
                    f[4 * i + 2] &= m[0].imag() == 0.0 ? 1 : 0;
                    for (uint32_t r = 0; r < dim; ++r)
                        for (uint32_t c = 0; c < dim; ++c)
                            if (r != c && (m[r * dim + c].real() != 0.0 || m[r * dim + c].imag() != 0.0)) f[4 * i + 3] = 0;
                }
            }
        });
        if (!ok) return MB2_ERR_INVALID;
        for (size_t i = 0; i < nb; ++i) {
            bool differs = false, all_real = true, m00_real = true, all_diag = true;
            for (unsigned w = 0; w < nt; ++w) {
                differs = differs || acc[w][4 * i];
                all_real = all_real && acc[w][4 * i + 1];
                m00_real = m00_real && acc[w][4 * i + 2];
                all_diag = all_diag && acc[w][4 * i + 3];
            }
            // A block that is diagonal for some bindings only (an angle of 0)
            // runs through the dense path for every binding.  For such a
            // binding each output is d*a plus products with exactly-zero
            // entries: the diagonal kernel's value except possibly for the
            // sign of a zero result, and every stored zero is canonical (+0)
            // on both paths, so the state's bits are the same.
            shape[i].diagonal = shape[i].diagonal && all_diag;
            if (differs) {
                flags[i] = mb2::kParamBlock | (all_real ? mb2::kParamAllReal : 0) | (m00_real ? mb2::kParamM00Real : 0);
                if (!shape[i].diagonal && shape[i].k > 2) return MB2_ERR_UNSUPPORTED;
            }
        }
    } else {
        per.resize(num_bindings);
        const bool ok = parallel([&](unsigned w) {
            for (uint32_t b = w; b < num_bindings; b += nt)
                per[b] = binding_blocks(ops, num_ops, params + size_t{b} * params_per_binding, fuse);
        });
        if (!ok) return MB2_ERR_INVALID;
        for (uint32_t b = 1; b < num_bindings; ++b) {  // one structure for every binding
            if (per[b].size() != nb) return MB2_ERR_INVALID;
            for (size_t i = 0; i < nb; ++i)
                if (per[b][i].k != shape[i].k || per[b][i].mask() != shape[i].mask()) return MB2_ERR_INVALID;
        }
        for (size_t i = 0; i < nb; ++i) {
            bool differs = false, all_real = true, m00_real = true, all_diag = true;
            for (uint32_t b = 0; b < num_bindings; ++b) {
                const auto& m = per[b][i].m;
                if (std::memcmp(m.data(), shape[i].m.data(), m.size() * sizeof(mb2::Cd)) != 0) differs = true;
                for (const mb2::Cd& c : m) all_real = all_real && c.imag() == 0.0;
                m00_real = m00_real && m[0].imag() == 0.0;
                all_diag = all_diag && per[b][i].diagonal;
            }
            shape[i].diagonal = all_diag;
            if (differs) {
                flags[i] = mb2::kParamBlock | (all_real ? mb2::kParamAllReal : 0) | (m00_real ? mb2::kParamM00Real : 0);
                if (!all_diag && shape[i].k > 2) return MB2_ERR_UNSUPPORTED;  // parametric wide dense blocks
            }
        }
    }
    const uint32_t mmax = c64 ? mb2::kMaxTileQubitsC64 : mb2::kMaxTileQubits;
    uint32_t m = o.tile_qubits > 0 ? static_cast<uint32_t>(o.tile_qubits) : (c64 ? mb2::kMaxTileQubitsC64 : 11u);
    for (const auto& b : shape) m = std::max(m, b.k);
    m = std::min(std::max(m, mb2::kMinTileQubits), std::min(mmax, num_qubits));
    mb2::TileProgram prog;
    try {
        prog = mb2::plan_tile_program(shape, num_qubits, m, mb2::kDefaultFixedLow, &flags, c64);
    } catch (const std::exception&) {
        return MB2_ERR_INVALID;
    }
    // Per-binding records of the parametric blocks, in the kernel's layout.
    const size_t stride = prog.param_stride;
    std::vector<double> pdata(std::max<size_t>(1, stride * num_bindings), 0.0);
    auto write_record = [&](uint32_t b, size_t i, const std::vector<mb2::Cd>& m, uint32_t k) {
        const uint32_t dim = 1u << k;
        double* dst = pdata.data() + size_t{b} * stride + prog.param_offsets[i];
        if (shape[i].diagonal) {
            for (uint32_t e = 0; e < dim; ++e) {
                dst[2 * e] = m[size_t{e} * dim + e].real();
                dst[2 * e + 1] = m[size_t{e} * dim + e].imag();
            }
        } else {
            std::memcpy(dst, m.data(), size_t{dim} * dim * sizeof(mb2::Cd));
        }
    };
    const bool filled = parallel([&](unsigned w) {
        std::vector<mb2::Cd> m;
        for (uint32_t b = w; b < num_bindings; b += nt)
            for (size_t i = 0; i < nb; ++i) {
                if (!(flags[i] & mb2::kParamBlock)) continue;
                if (fuse) {
                    write_record(b, i, per[b][i].m, per[b][i].k);
                } else {
                    const mb2_op& o = ops[gate_op[i]];
                    if (mb2::gate_matrix(o.opcode, params + size_t{b} * params_per_binding + gate_pofs[i], m) == 0)
                        throw std::invalid_argument("gate matrix");
                    write_record(b, i, m, shape[i].k);
                }
            }
    });
    if (!filled) return MB2_ERR_INVALID;

    // ---- device
    Runner r{0};
    // Everything below runs on the context's device, whichever device the
    // calling thread had selected.
    const int dev = mb2::context_device(ctx);
    if (cudaSetDevice(dev) != cudaSuccess) return MB2_ERR_CUDA;
    if (cudaStreamCreateWithFlags(&r.stream, cudaStreamNonBlocking) != cudaSuccess) return MB2_ERR_CUDA;
    const size_t state_bytes = (size_t{num_bindings} << num_qubits) * (c64 ? 8 : sizeof(mb2::Cd));
    auto al = [](size_t v) { return (v + 255) & ~size_t{255}; };
    const size_t ib = prog.words.size() * sizeof(uint32_t), sb = prog.data.size() * 8,
                 gb = prog.gdata.size() * 8, pb = pdata.size() * 8, tb = size_t{num_terms} * 8;
    // <H> per binding: with at least kPauliTileQubits qubits, the grouped
    // reduction (terms sharing a GF(2) span read each state once, `per`
    // CTAs per binding); smaller states: one 8-CTA cluster per binding.
    mb2::PauliPlan pplan;
    bool grouped = num_terms > 0 && num_qubits >= mb2::kPauliTileQubits;
    if (grouped) {
        pplan = mb2::plan_pauli_groups(x_masks, z_masks, num_terms, num_qubits);
        for (const mb2::PauliGroupPlan& g : pplan.groups)
            if (g.c + g.d < mb2::kPauliMinTileQubits) grouped = false;
    }
    const uint32_t gper = std::min<uint32_t>(4u, 1u << std::min<uint32_t>(2u, num_qubits - mb2::kPauliTileQubits));
    const size_t spb = grouped ? pplan.spans.size() * 8 : 0,
                 trb = grouped ? pplan.terms.size() * sizeof(mb2::PauliGroupTerm) : 0,
                 prb = grouped ? size_t{num_terms} * num_bindings * gper * 16 : 0;
    const size_t o_s = al(ib), o_g = o_s + al(sb), o_p = o_g + al(gb), o_x = o_p + al(pb), o_z = o_x + al(tb),
                 o_c = o_z + al(tb), o_sp = o_c + al(tb), o_tr = o_sp + al(spb), o_o = o_tr + al(trb),
                 o_pr = o_o + al(size_t{num_bindings} * 8), total = o_pr + al(prb);
    if (cudaMalloc(&r.state, state_bytes) != cudaSuccess || cudaMalloc(&r.work, total) != cudaSuccess) {
        cudaGetLastError();
        return MB2_ERR_RESOURCE;
    }
    auto* w = static_cast<unsigned char*>(r.work);
    std::vector<unsigned char> host(o_o, 0);
    std::memcpy(host.data(), prog.words.data(), ib);
    if (sb) std::memcpy(host.data() + o_s, prog.data.data(), sb);
    if (gb) std::memcpy(host.data() + o_g, prog.gdata.data(), gb);
    std::memcpy(host.data() + o_p, pdata.data(), pb);
    if (tb) {
        std::memcpy(host.data() + o_x, x_masks, tb);
        std::memcpy(host.data() + o_z, z_masks, tb);
        std::memcpy(host.data() + o_c, coefs, tb);
    }
    if (spb) std::memcpy(host.data() + o_sp, pplan.spans.data(), spb);
    if (trb) std::memcpy(host.data() + o_tr, pplan.terms.data(), trb);
    if (cudaMemcpyAsync(w, host.data(), host.size(), cudaMemcpyHostToDevice, r.stream) != cudaSuccess)
        return MB2_ERR_CUDA;
    const mb2::Cd ph = mb2::initial_phase(0.0);
    if (mb2::launch_batch_init(r.state, num_qubits, num_bindings, ph.real(), ph.imag(), r.stream, o.precision) !=
        MB2_OK)
        return MB2_ERR_CUDA;
    int sm = 148;
    cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, dev);
    mb2::BatchLayout layout;
    layout.bindings = num_bindings;
    layout.pdata = reinterpret_cast<const double*>(w + o_p);
    layout.pstride = static_cast<uint32_t>(stride);
    for (const mb2::TilePass& pass : prog.passes) {
        const auto* dw = reinterpret_cast<const uint32_t*>(w);
        const auto* ds = reinterpret_cast<const double*>(w + o_s);
        const auto* dg = reinterpret_cast<const double*>(w + o_g);
        const int rc = c64 ? mb2::launch_tile_pass_c64(r.state, num_qubits, pass, dw, ds, dg, sm, r.stream, &layout)
                           : mb2::launch_tile_pass(r.state, num_qubits, pass, dw, ds, dg, sm, r.stream, &layout);
        if (rc != MB2_OK) return MB2_ERR_CUDA;
    }
    if (num_terms > 0) {
        const auto* dx = reinterpret_cast<const uint64_t*>(w + o_x);
        const auto* dz = reinterpret_cast<const uint64_t*>(w + o_z);
        const auto* dc = reinterpret_cast<const double*>(w + o_c);
        auto* dout = reinterpret_cast<double*>(w + o_o);
        if (grouped) {
            auto* parts = reinterpret_cast<double*>(w + o_pr);
            for (const mb2::PauliGroupPlan& g : pplan.groups)
                if (mb2::launch_pauli_group_batch(
                        r.state, num_qubits, g.c, g.d, reinterpret_cast<const uint64_t*>(w + o_sp) + g.span_off,
                        g.free_mask, w + o_tr + size_t{g.term_off} * sizeof(mb2::PauliGroupTerm), g.nterms,
                        num_bindings, gper, parts, sm, r.stream, o.precision) != MB2_OK)
                    return MB2_ERR_CUDA;
            if (mb2::launch_batch_group_finish(parts, num_bindings, gper, dx, dz, dc, num_terms, dout, r.stream) !=
                MB2_OK)
                return MB2_ERR_CUDA;
        } else if (mb2::launch_batch_expect(r.state, num_qubits, num_bindings, dx, dz, dc, num_terms, dout, r.stream,
                                            o.precision) != MB2_OK) {
            return MB2_ERR_CUDA;
        }
        if (cudaMemcpyAsync(out, w + o_o, size_t{num_bindings} * 8, cudaMemcpyDeviceToHost, r.stream) != cudaSuccess)
            return MB2_ERR_CUDA;
    } else {
        std::fill(out, out + num_bindings, 0.0);
    }
    // States out as complex128 (a complex64 batch's amplitudes promoted).
    std::vector<float> lo;
    if (states_out != nullptr) {
        void* dst = states_out;
        if (c64) {
            lo.resize(state_bytes / sizeof(float));
            dst = lo.data();
        }
        if (cudaMemcpyAsync(dst, r.state, state_bytes, cudaMemcpyDeviceToHost, r.stream) != cudaSuccess)
            return MB2_ERR_CUDA;
    }
    if (cudaStreamSynchronize(r.stream) != cudaSuccess) return MB2_ERR_CUDA;
    if (states_out != nullptr && c64)
        for (size_t i = 0; i < lo.size(); ++i) states_out[i] = static_cast<double>(lo[i]);
    if (stats != nullptr) {
        stats->passes = prog.passes.size();
        stats->blocks = nb;
        stats->parametric_blocks = static_cast<uint64_t>(std::count_if(flags.begin(), flags.end(), [](uint8_t f) {
            return (f & mb2::kParamBlock) != 0;
        }));
        stats->h2d_bytes = host.size();
        stats->fp64_ops_per_amp = prog.fp64_per_amp;
    }
    return MB2_OK;
}
