// Tile-pass instances for 11-qubit tiles: the ping-pong kernel (two groups
// of 128 threads per CTA, one CTA per SM).
#include "tile_pass.cuh"

namespace mb2 {

int launch_tile_m11(const TileLaunch& L) {
    return L.n_all <= 32 ? tile::launch_pingpong<11, uint32_t>(L) : tile::launch_pingpong<11, uint64_t>(L);
}

}  // namespace mb2
