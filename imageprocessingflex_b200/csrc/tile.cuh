// tile.cuh -- border-resolving tile loader shared by the generic kernels.
//
// A tile is RY rows x SW flat samples of the source, starting at flat sample
// gq0 of row gy0 (both may be negative or run past the image).  Each sample is
// resolved by the border rule at load time: rows through border_index on y,
// samples through border_sample on the interleaved row (channel preserved),
// and Constant positions take `bv`.  This is the reference's padded-row
// construction (filter.hpp:51-63, 179-180) done once per tile in shared
// memory instead of once per output.
#pragma once

#include "common.cuh"

namespace ipfc {

template <typename Tin, typename Tacc>
__device__ __forceinline__ void load_tile(Tacc* tile, int RY, int SW, const void* src, long long spitch, int W, int H,
                                          int C, int gq0, int gy0, int border, Tacc bv) {
    const int rowlen = W * C;
    const bool inside_x = gq0 >= 0 && gq0 + SW <= rowlen;
    // warps take rows, lanes take samples (any block shape of whole warps)
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    const int lane = tid & 31, nrow = (blockDim.x * blockDim.y) >> 5;
    for (int r = tid >> 5; r < RY; r += nrow) {
        const int sy = border_index(gy0 + r, H, border);
        Tacc* dst = tile + (size_t)r * SW;
        if (sy < 0) {
            for (int s = lane; s < SW; s += 32) dst[s] = bv;
            continue;
        }
        const Tin* srow = row_ptr<Tin>(src, spitch, sy);
        if (inside_x) {
            for (int s = lane; s < SW; s += 32) dst[s] = static_cast<Tacc>(srow[gq0 + s]);
        } else {
            for (int s = lane; s < SW; s += 32) {
                const int g = gq0 + s;
                const int idx = ((unsigned)g < (unsigned)rowlen) ? g : border_sample(g, W, C, border);
                dst[s] = idx < 0 ? bv : static_cast<Tacc>(srow[idx]);
            }
        }
    }
}

}  // namespace ipfc
