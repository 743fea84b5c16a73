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
};

// Every pixel's error from the film (FP64 sums and odd sums, 4 a pixel; counts).
__global__ void adErrors(AdaptiveArgs a, const double* sums, const double* odd, const uint32_t* counts);
// Each region's tree rebuilt from the errors, one block a region (regionDone: 1 converged, 0 not).
__global__ void adTrees(AdaptiveArgs a);
// Each tile's mask for a pass of `size` samples a pixel (every pixel in the image in a uniform pass), its pixels'
// first sample indices and planned counts; a non-uniform pass whose regions have all converged sets the stop word.
__global__ void adMasks(AdaptiveArgs a, uint32_t uniform, uint32_t size);
// One block of kCompactThreads: a queued frame's pass's active tiles, in tile order, as chunks of `size` samples with
// their masks, and their count; a pass with none sets the stop word (nothing can change after it).
constexpr int kCompactThreads = 1024;
__global__ void adCompact(AdaptiveArgs a, uint32_t size);

}  // namespace x2
