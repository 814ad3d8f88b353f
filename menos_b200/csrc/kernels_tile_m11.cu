// Tile-pass instances for 11-qubit tiles (128 threads a CTA): the lean
// variant for passes of single-qubit dense blocks, diagonals and sign runs,
// the full one for the rest.  The lean 32-bit-index variant runs three CTAs
// per SM (168 registers): its passes are bound by FP64 dependency latency,
// and the third CTA's warps hide more of it (28-qubit brick+QFT sweep 6.5 %
// faster than with two); the others keep two.
#include "tile_pass.cuh"

namespace mb2 {

int launch_tile_m11(TileLaunch& L) {
    // Three resident CTAs need their shared memory to fit too (1 KiB of each
    // SM's is reserved per resident block); otherwise the grid is sized for two.
    const bool three = !L.heavy && L.n_all <= 32 && 3 * (L.smem + 1024) <= kSmemPerSm;
    const uint64_t cap = static_cast<uint64_t>(L.sm_count) * (three ? 3u : 2u);
    L.grid = static_cast<int>(L.ntiles < cap ? L.ntiles : cap);
    if (!L.heavy)
        return L.n_all <= 32 ? tile::launch_instance<128, 3, 11, uint32_t, false>(L)
                             : tile::launch_instance<128, 2, 11, uint64_t, false>(L);
    return L.n_all <= 32 ? tile::launch_instance<128, 2, 11, uint32_t, true>(L)
                         : tile::launch_instance<128, 2, 11, uint64_t, true>(L);
}

}  // namespace mb2
