// Tile-pass instance for any tile width (runtime m, 64-bit amplitude indices).
#include "tile_pass.cuh"

namespace mb2 {

int launch_tile_generic(TileLaunch& L) {
    const uint64_t cap = static_cast<uint64_t>(L.sm_count) * 2u;
    L.grid = static_cast<int>(L.ntiles < cap ? L.ntiles : cap);
    return tile::launch_instance<256, 1, 0, uint64_t, true>(L);
}

}  // namespace mb2
