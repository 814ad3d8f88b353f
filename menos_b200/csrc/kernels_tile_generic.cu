// Tile-pass instance for any tile width (runtime m, 64-bit amplitude indices).
#include "tile_pass.cuh"

namespace mb2 {

int launch_tile_generic(const TileLaunch& L) { return tile::launch_instance<256, 1, 0, uint64_t>(L); }

}  // namespace mb2
