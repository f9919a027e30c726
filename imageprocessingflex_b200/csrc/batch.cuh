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
// Each class is its own persistent kernel with its own queue.
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
