// Tile-pass instances for 11-qubit tiles (128 threads, two CTAs per SM).
#include "tile_pass.cuh"

namespace mb2 {

int launch_tile_m11(const TileLaunch& L) {
    return L.n_all <= 32 ? tile::launch_instance<128, 2, 11, uint32_t>(L)
                         : tile::launch_instance<128, 2, 11, uint64_t>(L);
}

}  // namespace mb2
