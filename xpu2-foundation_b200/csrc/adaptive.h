// The adaptive pass chain on the device (adaptive.cu; internal to libx2).
//
// Between two passes of an adaptive frame the chain turns the film into the next pass's work: every pixel's error,
// then either the region trees (MoonRay's rule, regions.cuh) or the next cellular generation of the 8x8 tiles, then
// each tile's mask of pixels to sample with each such pixel's first sample index, then the pass's active tiles as
// chunks. A frame queued whole (x2_render_adaptive) runs it inside one CUDA graph; the trees are grown there by a
// conditional while node, a level of every region's nodes an iteration.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/x2.h"
#include "regions.cuh"

namespace x2 {

// The trees of all regions in one node pool, structure of arrays. Nodes are allocated a level at a time, so the nodes
// of the level being decided are the pool's range [level[0], level[1]) and the next level's come after them.
struct TreePool {
    float *x0, *y0, *x1, *y1;  // a node's bounds
    int32_t* child;            // its first child (the second follows it), -1 for a leaf
    uint8_t* fate;             // rg::kOpen or rg::kConverged (a split node keeps kOpen and has children)
    uint32_t* region;          // its region
    uint32_t capacity;         // nodes the pool holds (the regions' bounds, added)
    // count: nodes allocated; level: [begin, end) of the level under decision.
    uint32_t *count, *level;
};

// Per region: its pixel box (x0, y0, x1, y1), its summed-area table's offset, its node bound and nodes so far, and
// two flags the pass sets: every pixel ready (both halves sampled) and some node left open (not converged).
struct RegionState {
    const int32_t* box;
    const unsigned long long* satOffset;
    const uint32_t* bound;
    uint32_t* nodes;
    uint32_t* ready;
    uint32_t* open;
    uint32_t count;
    // The rows and columns of all regions, one thread each: region r's rows start at rowStart[r] (columns likewise).
    const uint32_t* rowStart;
    const uint32_t* colStart;
    uint32_t rows, cols;
    rg::RegionGrid grid;
};

struct AdaptiveArgs {
    uint32_t width, height, tilesX, tiles;
    float target;
    RegionState regions;
    TreePool pool;
    double* sat;
    float* errors;
    const uint64_t* inImage;
    uint64_t* reach;     // a pass's union of open leaves over each tile (before filling to bounds)
    uint64_t* tileMask;  // each tile's pixels to sample in the pass
    uint32_t* planned;   // each pixel's samples planned so far
    uint32_t* base;      // each pixel's first sample index in the pass
    uint32_t* stop;      // set once nothing is left to refine
    // A frame queued on the device whole: once *stop is set its chain steps do nothing. Its pass's active tiles as
    // chunks, their masks, their count (live), the passes launched and the samples planned.
    uint32_t queued;
    x2_chunk* chunks;
    uint64_t* chunkMasks;
    uint32_t* live;
    uint32_t* passes;
    unsigned long long* samples;
    uint32_t* blockTiles;  // the compaction's active tiles a block of kCompactBlock tiles
    // Cellular generations in place of the trees (alive null: trees): the generation the pass samples (a byte a tile)
    // and its live tiles' count; each tile's error ratio of the last generation.
    const uint8_t* alive;
    uint32_t* liveTiles;
    float* ratio;
};

constexpr int kCompactBlock = 256;

// Each pixel's error (regions.cuh pixelError) from the film.
__global__ void chainPixelErrors(AdaptiveArgs a, const double* sums, const double* odd, const uint32_t* counts);
// Trees: the roots (one thread a region), the summed-area tables (a thread a region row, then a thread a region
// column), a level of every region's nodes (the pool's level range; with a loop handle, the next level's range and
// whether to go on), the open leaves' reach over the tiles (a warp a node) and each tile's mask.
__global__ void treeRoots(AdaptiveArgs a);
__global__ void tableRows(AdaptiveArgs a);
__global__ void tableColumns(AdaptiveArgs a);
__global__ void treeLevel(AdaptiveArgs a);
__global__ void treeNextLevel(AdaptiveArgs a, cudaGraphConditionalHandle loop);
__global__ void leafReach(AdaptiveArgs a);
// Each tile's mask for a pass of `size` samples a pixel (every pixel of the image in a uniform pass), its pixels'
// first sample indices and planned counts. In a non-uniform pass with nothing left to refine (every region converged;
// cellular: no live tile) it sets the stop word instead.
__global__ void tileMasks(AdaptiveArgs a, uint32_t uniform, uint32_t size);
// Cellular: each tile's error ratio, then the next generation (`aliveIn` to `aliveOut`, live tiles counted).
constexpr float kSurvive = 0.5f, kBirth = 0.75f;
constexpr int kSurviveNeighbours = 3, kBirthNeighbours = 5;
__global__ void tileRatios(AdaptiveArgs a);
__global__ void nextGeneration(AdaptiveArgs a, const uint8_t* aliveIn, uint8_t* aliveOut);
// The pass's active tiles, in tile order, as chunks of `size` samples with their masks: active tiles counted a block,
// then written (each block's offset the counts of the blocks before it); a pass with none sets the stop word.
__global__ void compactCount(AdaptiveArgs a);
__global__ void compactWrite(AdaptiveArgs a, uint32_t size);

}  // namespace x2
