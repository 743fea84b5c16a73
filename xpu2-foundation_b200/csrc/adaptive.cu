// The adaptive pass chain on the device (row f2 of the path's scope): between a frame's passes, every pixel's error
// from the film, the region trees rebuilt from the errors, and the next pass's tile masks with each active pixel's
// first sample index — the reference's GPU chain (xpu2/interactive/async_adaptive.cu: chainErrors, chainTrees,
// chainMasks) with the arithmetic of adaptive.cuh, which the host's trees share, so the masks equal the reference's
// host trees' for the same film.
#include "adaptive.h"

namespace x2 {

// A queued frame's chain does nothing once the stop word is set.
__device__ __forceinline__ bool halted(const AdaptiveArgs& a) { return a.queued && *(volatile const uint32_t*)a.stop; }

__global__ void adErrors(AdaptiveArgs a, const double* sums, const double* odd, const uint32_t* counts) {
    if (halted(a)) return;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.width * a.height) return;
    a.errors[i] = ad::pixelError(sums + 4ull * i, odd + 4ull * i, counts[i]);
}

// One block a region: the summed-area table of its errors (each row's running sums, then each column's, the sums in
// the host's order), then its nodes a level at a time, each decided as the host's recursion decides it. A region with a
// pixel not ready keeps its root alone, unconverged.
__global__ void adTrees(AdaptiveArgs a) {
    if (halted(a)) return;
    const uint32_t r = blockIdx.x;
    const ad::IBox root = a.regions[r];
    const int w = root.x1 - root.x0, h = root.y1 - root.y0, w1 = w + 1;
    double* sat = a.sat + a.satOffset[r];
    ad::Node* nodes = a.nodes + a.nodeOffset[r];
    __shared__ int notReady, unconverged, count;
    if (threadIdx.x == 0) {
        notReady = unconverged = 0;
        count = 1;
        nodes[0] = ad::Node{{float(root.x0), float(root.y0), float(root.x1), float(root.y1)}, -1, 0};
    }
    __syncthreads();
    for (int x = threadIdx.x; x <= w; x += blockDim.x) sat[x] = 0.0;
    for (int y = threadIdx.x; y < h; y += blockDim.x) {
        const float* e = a.errors + size_t(root.y0 + y) * a.width + root.x0;
        double* out = sat + size_t(y + 1) * w1;
        double run = 0.0;
        out[0] = 0.0;
        bool missing = false;
        for (int x = 0; x < w; ++x) {
            const float v = e[x];
            missing = missing || v < 0;
            run += v;
            out[x + 1] = run;
        }
        if (missing) notReady = 1;
    }
    __syncthreads();
    if (notReady) {
        if (threadIdx.x == 0) a.regionDone[r] = 0;
        return;
    }
    for (int x = threadIdx.x + 1; x <= w; x += blockDim.x)
        for (int y = 1; y <= h; ++y) sat[size_t(y) * w1 + x] += sat[size_t(y - 1) * w1 + x];
    __syncthreads();
    const ad::Sat s{sat, root.x0, root.y0, w1};
    const int capacity = int(a.nodeCapacity[r]);
    int begin = 0, end = 1;
    while (begin < end) {
        for (int i = begin + int(threadIdx.x); i < end; i += blockDim.x) {
            ad::FBox left, right;
            const int fate = ad::decide(s, root, nodes[i].b, a.target, left, right);
            if (fate == ad::kConverged) {
                nodes[i].complete = 1;
            } else if (fate == ad::kSplit) {
                const int c = atomicAdd(&count, 2);
                if (c + 2 <= capacity) {
                    nodes[c] = ad::Node{left, -1, 0};
                    nodes[c + 1] = ad::Node{right, -1, 0};
                    nodes[i].children = c;
                } else {
                    unconverged = 1;  // past the tree's bound (never, by the bound's construction)
                }
            } else {
                unconverged = 1;
            }
        }
        __syncthreads();
        begin = end;
        end = count < capacity ? count : capacity;
        __syncthreads();
    }
    if (threadIdx.x == 0) a.regionDone[r] = unconverged ? 0 : 1;
}

__global__ void adMasks(AdaptiveArgs a, uint32_t uniform, uint32_t size) {
    if (halted(a)) return;
    if (!uniform) {
        bool converged = true;
        if (a.alive) converged = *a.liveTiles == 0;
        else
            for (uint32_t r = 0; r < a.regionCount; ++r) converged = converged && a.regionDone[r] != 0;
        if (converged) {
            if (blockIdx.x == 0 && threadIdx.x == 0) *a.stop = 1;
            return;
        }
    }
    const uint32_t tile = blockIdx.x * blockDim.x + threadIdx.x;
    if (tile >= a.tiles) return;
    uint64_t mask = a.inImage[tile];
    if (!uniform && a.alive) {
        if (!a.alive[tile]) mask = 0;
    } else if (!uniform) {
        const int tx = int(tile % a.tilesX) * 8, ty = int(tile / a.tilesX) * 8;
        mask &= ad::tileSamples(a.nodes + a.nodeOffset[a.layout.regionOf(tx, ty)], tx, ty);
    }
    a.tileMask[tile] = mask;
    for (uint32_t p = 0; p < 64; ++p)
        if (mask >> p & 1) {
            const uint32_t x = (tile % a.tilesX) * 8 + p % 8, y = (tile / a.tilesX) * 8 + p / 8;
            const uint32_t pixel = y * a.width + x;
            a.base[pixel] = a.planned[pixel];
            a.planned[pixel] += size;
        }
}

__global__ void adCellular(AdaptiveArgs a, const uint8_t* aliveIn, uint8_t* aliveOut) {
    if (halted(a)) return;
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.tiles) return;
    const int tilesX = int(a.tilesX), tilesY = int(a.tiles / a.tilesX), tx = int(t) % tilesX, ty = int(t) / tilesX;
    const int width = int(a.width), height = int(a.height);
    double sum = 0.0;
    int n = 0;
    bool unknown = false;
    for (int y = ty * 8; y < ad::imin(height, ty * 8 + 8); ++y)
        for (int x = tx * 8; x < ad::imin(width, tx * 8 + 8); ++x) {
            const float e = a.errors[size_t(y) * size_t(width) + size_t(x)];
            if (e < 0) unknown = true;
            else sum += e;
            ++n;
        }
    const float error = unknown ? -1.0f : ad::nodeError(float(sum), float(n));
    const float ratio = error < 0 ? 3.4e38f : error / a.target;
    int k = 0;
    for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
            const int x = tx + dx, y = ty + dy;
            if ((dx || dy) && x >= 0 && y >= 0 && x < tilesX && y < tilesY && aliveIn[size_t(y) * tilesX + x]) ++k;
        }
    bool next = aliveIn[t] ? (ratio >= 1.0f || (ratio >= kSurvive && k >= kSurviveNeighbours))
                           : (ratio >= 1.0f || (ratio >= kBirth && k >= kBirthNeighbours));
    if (!a.inImage[t]) next = false;
    aliveOut[t] = next ? 1 : 0;
    if (next) atomicAdd(a.liveTiles, 1u);
}

__global__ void adCompact(AdaptiveArgs a, uint32_t size) {
    __shared__ uint32_t scan[kCompactThreads];
    const uint32_t tid = threadIdx.x;
    if (halted(a)) {
        if (tid == 0) *a.live = 0;
        return;
    }
    const uint32_t per = (a.tiles + kCompactThreads - 1) / kCompactThreads, first = tid * per;
    const uint32_t last = first + per < a.tiles ? first + per : a.tiles;
    uint32_t mine = 0;
    unsigned long long pixels = 0;
    for (uint32_t t = first; t < last; ++t) {
        const uint64_t m = a.tileMask[t];
        if (m) {
            ++mine;
            pixels += __popcll(m);
        }
    }
    scan[tid] = mine;
    __syncthreads();
    for (uint32_t offset = 1; offset < kCompactThreads; offset <<= 1) {
        const uint32_t v = tid >= offset ? scan[tid - offset] : 0u;
        __syncthreads();
        scan[tid] += v;
        __syncthreads();
    }
    uint32_t at = scan[tid] - mine;
    for (uint32_t t = first; t < last; ++t) {
        const uint64_t m = a.tileMask[t];
        if (m) {
            a.chunks[at] = x2_chunk{t, 0, size, 0};
            a.chunkMasks[at] = m;
            ++at;
        }
    }
    if (pixels) atomicAdd(a.samples, pixels * size);
    if (tid == kCompactThreads - 1) {
        const uint32_t total = scan[tid];
        *a.live = total;
        if (total) ++*a.passes;
        else *a.stop = 1;
    }
}

}  // namespace x2
