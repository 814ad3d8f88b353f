// Tile-pass instances for 12-qubit tiles (256 threads, one CTA per SM), lean
// and full variants as for 11-qubit tiles.
#include "tile_pass.cuh"

namespace mb2 {

int launch_tile_m12(TileLaunch& L) {
    const uint64_t cap = static_cast<uint64_t>(L.sm_count);
    L.grid = static_cast<int>(L.ntiles < cap ? L.ntiles : cap);
    if (!L.heavy)
        return L.n_all <= 32 ? tile::launch_instance<256, 1, 12, uint32_t, false>(L)
                             : tile::launch_instance<256, 1, 12, uint64_t, false>(L);
    return L.n_all <= 32 ? tile::launch_instance<256, 1, 12, uint32_t, true>(L)
                         : tile::launch_instance<256, 1, 12, uint64_t, true>(L);
}

}  // namespace mb2
