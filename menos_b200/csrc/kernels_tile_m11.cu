// Tile-pass instances for 11-qubit tiles (128 threads a CTA, two CTAs per
// SM): the lean variant for passes of single-qubit dense blocks, diagonals and
// sign runs, the full one for the rest.
#include "tile_pass.cuh"

namespace mb2 {

int launch_tile_m11(TileLaunch& L) {
    const uint64_t cap = static_cast<uint64_t>(L.sm_count) * 2u;
    L.grid = static_cast<int>(L.ntiles < cap ? L.ntiles : cap);
    if (!L.heavy)
        return L.n_all <= 32 ? tile::launch_instance<128, 2, 11, uint32_t, false>(L)
                             : tile::launch_instance<128, 2, 11, uint64_t, false>(L);
    return L.n_all <= 32 ? tile::launch_instance<128, 2, 11, uint32_t, true>(L)
                         : tile::launch_instance<128, 2, 11, uint64_t, true>(L);
}

}  // namespace mb2
