// The tile pass over many small states in one launch (k_tile_pass_jobs):
// runtime tile width, full variant, 64-bit indices; one CTA per tile.
#include "tile_pass.cuh"

namespace mb2 {

int launch_tile_jobs(const TileJob* dev_jobs, uint32_t njobs, uint32_t total_ctas, uint32_t m, size_t smem,
                     void* stream) {
    if (njobs == 0 || total_ctas == 0) return MB2_OK;
    if (m < kMinTileQubits || m > kMaxTileQubits) return MB2_ERR_INVALID;
    static const size_t dyn_max = [] {
        cudaFuncAttributes fa{};
        if (cudaFuncGetAttributes(&fa, tile::k_tile_pass_jobs<256, 0, true>) != cudaSuccess) return size_t{0};
        const size_t v = kTileSmemMax - fa.sharedSizeBytes;
        if (cudaFuncSetAttribute(tile::k_tile_pass_jobs<256, 0, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(v)) != cudaSuccess)
            return size_t{0};
        return v;
    }();
    if (dyn_max == 0) return launch_status();
    if (smem > dyn_max) return MB2_ERR_INVALID;
    tile::k_tile_pass_jobs<256, 0, true><<<total_ctas, 1u << (m - kRegQubits), smem,
                                           static_cast<cudaStream_t>(stream)>>>(dev_jobs, njobs, m);
    note_launches(1);
    return launch_status();
}

}  // namespace mb2
