// The adaptive pass chain's kernels (adaptive.cu; internal to libx2).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/x2.h"
#include "adaptive.cuh"

namespace x2 {

// A frame's adaptive state on the device: the film's pixel errors, the region trees (their bounds, node arrays and
// summed-area tables), each tile's pixels in the image and its mask for the pass, each pixel's planned sample count
// and its first sample index in the pass, and the chain's stop word (1: every region converged).
struct AdaptiveArgs {
    uint32_t width, height, tilesX, tiles, regionCount;
    float target;
    ad::Layout layout;
    const ad::IBox* regions;
    const uint32_t* nodeOffset;
    const uint32_t* nodeCapacity;
    const unsigned long long* satOffset;
    double* sat;
    ad::Node* nodes;
    uint32_t* regionDone;
    float* errors;
    const uint64_t* inImage;
    uint64_t* tileMask;
    uint32_t* planned;
    uint32_t* base;
    uint32_t* stop;
    // A frame queued on the device whole (x2_render_adaptive): once the stop word is set its chain steps do nothing
    // (0: a step the host runs, x2_adaptive_step). Its pass's active tiles as chunks, their masks and their count,
    // and the frame's tallies: passes launched and samples planned.
    uint32_t queued;
    x2_chunk* chunks;
    uint64_t* chunkMasks;
    uint32_t* live;
    uint32_t* passes;
    unsigned long long* samples;
    // Cellular generations in place of the trees (null: trees): the generation a pass samples (a byte a tile, 1 live)
    // and its live tiles' count.
    const uint8_t* alive;
    uint32_t* liveTiles;
};

// Every pixel's error from the film (FP64 sums and odd sums, 4 a pixel; counts).
__global__ void adErrors(AdaptiveArgs a, const double* sums, const double* odd, const uint32_t* counts);
// Each region's tree rebuilt from the errors, one block a region (regionDone: 1 converged, 0 not).
__global__ void adTrees(AdaptiveArgs a);
// The next cellular generation (the reference's adaptive::Cellular::update, async_adaptive.h:147-232) from the pixel
// errors: each tile's error is the node error of its pixels' summed errors over its pixel count (unknown while a pixel
// has no error), over the target; a live tile stays alive at a ratio of 1, or of Survive with SurviveNeighbours live
// neighbours, a dead one comes back at 1, or at Birth with BirthNeighbours; tiles outside the image never live. One
// thread a tile; `aliveIn` the last generation, `aliveOut` the next, its live tiles counted into a.liveTiles.
constexpr float kSurvive = 0.5f, kBirth = 0.75f;
constexpr int kSurviveNeighbours = 3, kBirthNeighbours = 5;
__global__ void adCellular(AdaptiveArgs a, const uint8_t* aliveIn, uint8_t* aliveOut);
// Each tile's mask for a pass of `size` samples a pixel (every pixel in the image in a uniform pass), its pixels'
// first sample indices and planned counts; a non-uniform pass whose regions have all converged (cellular: whose
// generation has no live tile) sets the stop word. With cellular generations a live tile samples all its pixels.
__global__ void adMasks(AdaptiveArgs a, uint32_t uniform, uint32_t size);
// One block of kCompactThreads: a queued frame's pass's active tiles, in tile order, as chunks of `size` samples with
// their masks, and their count; a pass with none sets the stop word (nothing can change after it).
constexpr int kCompactThreads = 1024;
__global__ void adCompact(AdaptiveArgs a, uint32_t size);

}  // namespace x2
