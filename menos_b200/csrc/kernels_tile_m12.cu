// Tile-pass instances for 12-qubit tiles (256 threads, one CTA per SM).
#include "tile_pass.cuh"

namespace mb2 {

int launch_tile_m12(const TileLaunch& L) {
    return L.n_all <= 32 ? tile::launch_instance<256, 1, 12, uint32_t>(L)
                         : tile::launch_instance<256, 1, 12, uint64_t>(L);
}

}  // namespace mb2
