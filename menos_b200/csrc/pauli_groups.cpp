// Grouping of Pauli terms for the expectation reduction.
//
// <psi|P|psi> for P = (x, z) pairs amplitude m with m ^ x.  Terms whose X
// masks, above the low c bits, lie in one GF(2) subspace V of dimension d
// can share one read of the state: a tile is a coset of V (2^d chunks of
// 2^c contiguous amplitudes), and every term's partner of every amplitude of
// the tile is in the tile.  Tiles hold at most 2^12 amplitudes (c + d <= 12).
// Groups are formed first-fit in term order; each group then takes the
// largest c with c + rank(x >> c) <= 12, so chunks are as long as possible.
// The same grouping for the same term list every time: the reduction order,
// and so the value, does not depend on anything else.
#include <algorithm>
#include <cstdint>
#include <vector>

#include "mb2_internal.h"

namespace mb2 {
namespace {

// GF(2) basis in reduced echelon form: vec[i] has bit piv[i] set and no other
// basis vector has that bit, so a vector of the span has coordinate i equal
// to its bit piv[i].
struct Gf2Basis {
    std::vector<uint64_t> vec;
    std::vector<uint32_t> piv;
    uint64_t reduce(uint64_t v) const {
        for (size_t i = 0; i < vec.size(); ++i)
            if ((v >> piv[i]) & 1u) v ^= vec[i];
        return v;
    }
    bool add(uint64_t v) {
        v = reduce(v);
        if (v == 0) return false;
        const uint32_t p = 63u - static_cast<uint32_t>(__builtin_clzll(v));
        for (uint64_t& b : vec)
            if ((b >> p) & 1u) b ^= v;
        vec.push_back(v);
        piv.push_back(p);
        return true;
    }
    uint32_t coords(uint64_t v) const {
        uint32_t k = 0;
        for (size_t i = 0; i < vec.size(); ++i) k |= static_cast<uint32_t>((v >> piv[i]) & 1u) << i;
        return k;
    }
};

uint32_t rank_above(const std::vector<uint64_t>& xs, uint32_t c) {
    Gf2Basis b;
    for (uint64_t x : xs) b.add(x >> c);
    return static_cast<uint32_t>(b.vec.size());
}

}  // namespace

PauliPlan plan_pauli_groups(const uint64_t* x, const uint64_t* z, uint32_t num_terms, uint32_t n) {
    const uint32_t tile = std::min<uint32_t>(kPauliTileQubits, n);
    const uint32_t cmin = std::min<uint32_t>(3, n);
    const uint32_t dmax = std::min<uint32_t>(kPauliMaxSpan, tile - cmin);
    struct Open {
        Gf2Basis basis;
        std::vector<uint32_t> members;
    };
    std::vector<Open> open;
    for (uint32_t t = 0; t < num_terms; ++t) {
        const uint64_t xh = x[t] >> cmin;
        bool placed = false;
        for (Open& g : open) {
            if (g.members.size() >= kMaxGroupTerms) continue;
            if (g.basis.reduce(xh) != 0 && g.basis.vec.size() >= dmax) continue;
            g.basis.add(xh);
            g.members.push_back(t);
            placed = true;
            break;
        }
        if (!placed) {
            Open g;
            g.basis.add(xh);
            g.members.push_back(t);
            open.push_back(std::move(g));
        }
    }
    PauliPlan plan;
    for (const Open& g : open) {
        std::vector<uint64_t> xs;
        for (uint32_t t : g.members) xs.push_back(x[t]);
        uint32_t c = cmin;
        for (uint32_t cc = tile; cc > cmin; --cc)
            if (cc + rank_above(xs, cc) <= tile) {
                c = cc;
                break;
            }
        Gf2Basis b;
        for (uint64_t v : xs) b.add(v >> c);
        PauliGroupPlan gp;
        gp.c = c;
        gp.d = static_cast<uint32_t>(b.vec.size());
        uint64_t pivots = 0;
        for (uint32_t p : b.piv) pivots |= uint64_t{1} << p;
        const uint64_t high = (n - c >= 64) ? ~uint64_t{0} : ((uint64_t{1} << (n - c)) - 1);
        gp.free_mask = high & ~pivots;
        gp.span_off = static_cast<uint32_t>(plan.spans.size());
        for (uint32_t k = 0; k < (1u << gp.d); ++k) {
            uint64_t v = 0;
            for (uint32_t i = 0; i < gp.d; ++i)
                if ((k >> i) & 1u) v ^= b.vec[i];
            plan.spans.push_back(v);
        }
        gp.term_off = static_cast<uint32_t>(plan.terms.size());
        gp.nterms = static_cast<uint32_t>(g.members.size());
        for (uint32_t t : g.members) {
            PauliGroupTerm pt{};
            pt.x = x[t];
            pt.z = z[t];
            pt.kx = b.coords(x[t] >> c);
            pt.xl = static_cast<uint32_t>(x[t] & ((uint64_t{1} << c) - 1));
            pt.out = t;
            plan.terms.push_back(pt);
        }
        plan.groups.push_back(gp);
    }
    return plan;
}

}  // namespace mb2

extern "C" int mb2_debug_pauli_groups(const uint64_t* x_masks, const uint64_t* z_masks, uint32_t num_terms,
                                      uint32_t num_qubits, uint64_t* out, uint64_t* out_words) {
    if (out_words == nullptr || (num_terms != 0 && (x_masks == nullptr || z_masks == nullptr)) || num_qubits == 0 ||
        num_qubits > 63)
        return MB2_ERR_INVALID;
    const mb2::PauliPlan plan = mb2::plan_pauli_groups(x_masks, z_masks, num_terms, num_qubits);
    std::vector<uint64_t> w;
    w.push_back(plan.groups.size());
    for (const mb2::PauliGroupPlan& g : plan.groups) {
        w.push_back(g.c);
        w.push_back(g.d);
        w.push_back(g.free_mask);
        w.push_back(g.nterms);
        for (uint32_t k = 0; k < (1u << g.d); ++k) w.push_back(plan.spans[g.span_off + k]);
        for (uint32_t i = 0; i < g.nterms; ++i) {
            const mb2::PauliGroupTerm& t = plan.terms[g.term_off + i];
            w.push_back(t.out);
            w.push_back(t.kx);
            w.push_back(t.xl);
        }
    }
    const uint64_t cap = *out_words;
    *out_words = w.size();
    if (out == nullptr || cap < w.size()) return MB2_ERR_INVALID;
    std::copy(w.begin(), w.end(), out);
    return MB2_OK;
}
