// Tile-pass instances for 11-qubit tiles (128 threads a CTA).  Passes without
// the heavy instructions run the lean variant, three CTAs per SM where the
// shared memory allows; the others run the full variant, two CTAs per SM.
#include "tile_pass.cuh"

namespace mb2 {

int launch_tile_m11(TileLaunch& L) {
    const bool lean = !L.heavy && 3 * (L.smem + 1024) <= kSmemPerSm;
    const uint64_t cap = static_cast<uint64_t>(L.sm_count) * (lean ? 3u : 2u);
    L.grid = static_cast<int>(L.ntiles < cap ? L.ntiles : cap);
    if (lean)
        return L.n_all <= 32 ? tile::launch_instance<128, 3, 11, uint32_t, false>(L)
                             : tile::launch_instance<128, 3, 11, uint64_t, false>(L);
    return L.n_all <= 32 ? tile::launch_instance<128, 2, 11, uint32_t, true>(L)
                         : tile::launch_instance<128, 2, 11, uint64_t, true>(L);
}

}  // namespace mb2
