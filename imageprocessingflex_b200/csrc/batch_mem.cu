// batch_mem.cu -- the memory-bound-class persistent batch kernel (3x3 and
// 5x5 uint8 median, uint8 morphology).
#include "batch_kernel.cuh"

namespace ipfc {

cudaError_t batch_launch_mem(const BatchItem* items, const BatchTile* tiles, int ntiles, unsigned* counter, int grid,
                             size_t smem, cudaStream_t s) {
    return batch_launch_class<kBatchMem>(items, tiles, ntiles, counter, grid, smem, s);
}

cudaError_t batch_occupancy_mem(size_t smem, int* occ) { return batch_occupancy_class<kBatchMem>(smem, occ); }

}  // namespace ipfc
