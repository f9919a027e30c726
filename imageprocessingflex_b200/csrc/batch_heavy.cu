// batch_heavy.cu -- the heavy-class persistent batch kernel (separable
// K 15..25).
#include "batch_kernel.cuh"

namespace ipfc {

cudaError_t batch_launch_heavy(const BatchItem* items, const BatchTile* tiles, int ntiles, unsigned* counter, int grid,
                               size_t smem, cudaStream_t s) {
    return batch_launch_class<1>(items, tiles, ntiles, counter, grid, smem, s);
}

cudaError_t batch_occupancy_heavy(size_t smem, int* occ) { return batch_occupancy_class<1>(smem, occ); }

}  // namespace ipfc
