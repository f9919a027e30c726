// batch.cuh -- the persistent batch kernel: many uneven uint8 images, one
// launch per register class, tiles pulled from a queue.
//
// A batch is a list of items (one image and one op each: a separable filter
// such as gaussianBlur, a k x k median, or an erosion / dilation by an
// all-ones element).  The host cuts every item into tiles -- the same tiles
// the per-image kernels run as one CTA each -- and writes two device arrays:
// the items' argument blocks and the tile list, ordered so that the most
// expensive tiles come first.  Each CTA of the persistent kernel then loops:
// take the next tile index from a global counter, copy the tile's item into
// shared memory when it changes, and run the tile body (sep_fast_tile,
// median_u8_tile / median_tile, morph_u8_tile).  The tile bodies are the per-image kernels'
// own code, so a batched image is computed exactly as the per-image call
// computes it.
//
// Register classes: the tile bodies differ a lot in registers and shared
// memory, and a kernel is launched with the largest need of everything it
// can run.  Light tiles (separable K <= 13, median k >= 7) run two CTAs per
// SM; heavy tiles (separable K 15..25) one; memory-bound tiles (3x3 and 5x5
// median, morphology) at least four, with 64 registers a thread, so that
// many tiles' loads are in flight and their CTAs fit beside a heavy one.
// The median and morphology classes are persistent kernels with their own
// queues; separable tiles run as group launches (below) with the class's
// CTAs per SM.
#pragma once

#include "median.cuh"
#include "median_u8.cuh"
#include "morph.cuh"
#include "morph_u8.cuh"
#include "sep_fast.cuh"

namespace ipfc {

enum BatchKind { kBatchSep = 0, kBatchMedian = 1, kBatchMorph = 2 };

constexpr int kBatchClasses = 3;
constexpr int kBatchLight = 0, kBatchHeavy = 1, kBatchMem = 2;
constexpr int kBatchLightMaxTaps = 13;
constexpr int kBatchMaxTaps = 25;

struct BatchTile {
    int item;  // index into the item array
    int x;     // separable: strip; median / morphology: tile column
    int y;     // separable: row chunk; median / morphology: tile row
    int pad;
};

struct __align__(16) BatchItem {
    int kind;  // BatchKind
    int K;     // separable taps (both axes); median ksize
    int C;     // channels
    int tx;    // median / morphology tile width (flat samples)
    int ty;    // median / morphology tile height (rows)
    int pad[3];
    union {
        SepFastArgs sep;
        MedianArgs med;
        MorphCore morph;
    } u;
};

// Separable items run as group launches, not from the queues: the argument
// blocks of up to kSepGroupItems items with the same tap count and channels
// are the kernel's parameter block, blockIdx.y selects the item and
// blockIdx.x the tile.  Because the item index comes from blockIdx, the
// compiler reads the taps and scalars as uniform constant-bank operands, as in
// the per-image kernel; from the queue's shared-memory copy of the item every
// use was a load, and a batched tile ran about 1.6x slower than the same tile
// per image.
constexpr int kSepGroupItems = 40;  // 40 x 712 B of parameters, within the 32 KB limit
struct SepGroup {
    SepFastArgs it[kSepGroupItems];
};
// The whole group is one kernel's parameter block, whose limit is 32764 bytes.
static_assert(sizeof(SepGroup) <= 32764, "a separable group must fit in the kernel parameters");

// Launches a group of n separable uint8 items with K taps and C channels:
// max_tiles x n CTAs (CTAs past an item's own tiles return at once).
cudaError_t batch_sep_group_launch(int K, int C, const SepGroup& g, int n, int max_tiles, cudaStream_t s);

// Launches the class-`cls` persistent kernel: `grid` CTAs of kFastThreads
// threads with `smem` bytes of dynamic shared memory walk tiles[0, ntiles)
// through *counter (which must start at 0).
cudaError_t batch_launch(int cls, const BatchItem* items, const BatchTile* tiles, int ntiles, unsigned* counter,
                         int grid, size_t smem, cudaStream_t s);

// Resident CTAs per SM of the class-`cls` kernel at `smem` bytes.
cudaError_t batch_occupancy(int cls, size_t smem, int* ctas_per_sm);

// Strip width (pixels) and shared memory (bytes) of a separable uint8 tile.
int batch_sep_px(int K, int C);
size_t batch_sep_smem(int K, int C);

}  // namespace ipfc
