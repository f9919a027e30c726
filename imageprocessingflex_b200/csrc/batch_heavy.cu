// batch_heavy.cu -- the separable group launches with 15 to 25 taps (and
// the heavy class's persistent kernel, which no queue tile uses now).
#include "batch_kernel.cuh"

namespace ipfc {

cudaError_t batch_launch_heavy(const BatchItem* items, const BatchTile* tiles, int ntiles, unsigned* counter, int grid,
                               size_t smem, cudaStream_t s) {
    return batch_launch_class<1>(items, tiles, ntiles, counter, grid, smem, s);
}

cudaError_t batch_occupancy_heavy(size_t smem, int* occ) { return batch_occupancy_class<1>(smem, occ); }

// Separable group launches with 15 to 25 taps.
bool batch_sep_group_heavy(int k, int c, const SepGroup& g, int n, int max_tiles, cudaStream_t s, cudaError_t* e) {
    return batch_sep_group_case<15>(k, c, g, n, max_tiles, s, e) ||
           batch_sep_group_case<17>(k, c, g, n, max_tiles, s, e) ||
           batch_sep_group_case<19>(k, c, g, n, max_tiles, s, e) ||
           batch_sep_group_case<21>(k, c, g, n, max_tiles, s, e) ||
           batch_sep_group_case<23>(k, c, g, n, max_tiles, s, e) ||
           batch_sep_group_case<25>(k, c, g, n, max_tiles, s, e);
}

}  // namespace ipfc
