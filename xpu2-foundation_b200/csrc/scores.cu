// Important parts first (row f1's scoring): each work-grid cell's score from the picture so far — the mean, over the
// cell's sampled pixels, of the differences of each pixel's tone from its left and upper neighbours' (where those are
// sampled), a tone being light / (1 + light) of the pixel's luma; -1 for a cell none of whose pixels has a sample.
// The reference scores its cells this way on the host (xpu2/interactive/async_render.h:1581-1611 cellScores) from its
// preview picture (async_cpu.h:1359-1379 HostFilm::preview: each pixel's film sum over its count, as a float). Here
// one thread a cell walks its pixels in the reference's order (rows, then columns), so the sums round alike.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <vector>

#include "../../include/x2.h"

namespace x2 {
namespace {

__device__ __forceinline__ float previewTone(const double* sums, const uint32_t* counts, size_t i) {
    const uint32_t n = counts[i];
    float rgb[3];
    for (int c = 0; c < 3; ++c) rgb[c] = n ? float(sums[4 * i + c] / double(n)) : 0.0f;
    const float l = __fadd_rn(__fadd_rn(__fmul_rn(0.2126f, rgb[0]), __fmul_rn(0.7152f, rgb[1])), __fmul_rn(0.0722f, rgb[2]));
    return isfinite(l) && l > 0 ? l / (1 + l) : 0.0f;
}

__global__ void cellScores(const double* sums, const uint32_t* counts, uint32_t width, uint32_t height, uint32_t cellSize, uint32_t cellsX,
                           uint32_t cellCount, float* scores) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cellCount) return;
    const uint32_t x0 = (c % cellsX) * cellSize, y0 = (c / cellsX) * cellSize;
    const uint32_t x1 = min(width, x0 + cellSize), y1 = min(height, y0 + cellSize);
    double sum = 0;
    uint32_t n = 0;
    for (uint32_t y = y0; y < y1; ++y)
        for (uint32_t x = x0; x < x1; ++x) {
            const size_t i = size_t(y) * width + x;
            if (!counts[i]) continue;
            const float t = previewTone(sums, counts, i);
            double d = 0;
            if (x > 0 && counts[i - 1]) d += fabsf(t - previewTone(sums, counts, i - 1));
            if (y > 0 && counts[i - width]) d += fabsf(t - previewTone(sums, counts, i - width));
            sum += d;
            ++n;
        }
    scores[c] = n ? float(sum / n) : -1.0f;
}

}  // namespace
}  // namespace x2

extern "C" int x2_workgrid_score_film(x2_scene* scene, x2_workgrid* grid, float* scores) {
    uint32_t width = 0, height = 0;
    x2_workgrid_options o;
    double* sums = nullptr;
    uint32_t* counts = nullptr;
    if (!scene || !grid || x2_workgrid_info(grid, &width, &height, nullptr, &o) != X2_OK ||
        x2_film_device(scene, &sums, nullptr, &counts) != X2_OK || !sums || !counts)
        return X2_EINVAL;
    if (x2_wait(scene, 600000, nullptr) != X2_OK) return X2_ECUDA;
    const uint32_t cellsX = (width + o.cell_size - 1) / o.cell_size, cellCount = x2_workgrid_cells(grid);
    float* dScores = nullptr;
    if (cudaMalloc(&dScores, sizeof(float) * cellCount) != cudaSuccess) return X2_ENOMEM;
    x2::cellScores<<<(cellCount + 127) / 128, 128>>>(sums, counts, width, height, o.cell_size, cellsX, cellCount, dScores);
    std::vector<float> host(cellCount);
    const cudaError_t e = cudaMemcpy(host.data(), dScores, sizeof(float) * cellCount, cudaMemcpyDeviceToHost);
    cudaFree(dScores);
    if (e != cudaSuccess) return X2_ECUDA;
    if (scores)
        for (uint32_t i = 0; i < cellCount; ++i) scores[i] = host[i];
    return x2_workgrid_set_scores(grid, host.data(), cellCount);
}
