// batch_plan.h -- host side of a batch plan, shared by the batch API
// (batch.cu) and the request server (serve.cu).
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "batch.cuh"

namespace ipfc {

struct TuneVal {
    int a;  // separable: rows per tile; median / morphology: tile width (samples)
    int b;  // median / morphology: tile height (rows)
};

// One image and its op, with the image's size.
struct HostItem {
    BatchItem it;
    int W = 0, H = 0;
};

// Items with their tile parameters applied, and the tile list grouped by
// class (light, heavy, memory-bound), each class ordered by estimated cost
// per tile.
// One launch of separable items with the same taps and channels (at most
// kSepGroupItems): indices into HostPlan::items, and the largest tile count.
struct SepGroupLaunch {
    int K = 0, C = 0, cls = 0;
    int max_tiles = 0;
    double cost = 0;  // estimated work (sum of its tiles' costs)
    std::vector<int> items;
};

struct HostPlan {
    std::vector<BatchItem> items;
    std::vector<BatchTile> tiles;  // queue tiles (median, morphology)
    int ntiles[kBatchClasses] = {};
    int tile_off[kBatchClasses] = {};
    size_t smem[kBatchClasses] = {};
    double cost[kBatchClasses] = {};
    std::vector<SepGroupLaunch> groups;  // separable items, heavy groups first
    int sep_tiles[kBatchClasses] = {};  // tiles in the groups, by class
};

void build_host_plan(const std::vector<HostItem>& items, const std::vector<TuneVal>& vals, HostPlan* p);

// Persistent grid of each class: resident CTAs on all SMs, at most one per
// tile.
cudaError_t plan_grids(const HostPlan& p, int grid[kBatchClasses]);

// Enqueues the plan whose items and tiles are in device memory: resets the
// class counters, then issues the separable group launches and the queue
// kernels, on s0 in order, or, when nside side streams, fork and join are
// given, spread over s0 and the side streams as parallel graph branches.
cudaError_t launch_plan(const BatchItem* d_items, const BatchTile* d_tiles, unsigned* d_counter, const HostPlan& p,
                        const int grid[kBatchClasses], cudaStream_t s0, const cudaStream_t* side, int nside,
                        cudaEvent_t fork, cudaEvent_t join);

// Tile parameters for an item: the autotuner's entry for its key on the
// current device, else the built-in default.  Never tunes.
TuneVal tuned_or_default(int kind, int k, int c, int W, int H);

}  // namespace ipfc
