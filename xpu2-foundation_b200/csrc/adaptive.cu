// The adaptive pass chain on the device (row f2 of the path's scope): from the film between two passes to the next
// pass's chunks, with the rules of the reference's adaptive frame (xpu2/interactive/async_adaptive.cu,
// async_adaptive.h Regions and Cellular; the arithmetic in regions.cuh), so that the masks equal the reference's host
// trees and generations bit for bit on the same film.
//
// The trees of all regions grow together, a level at a time: the pool's level range holds every region's nodes of
// that depth, one thread decides each (converge, split or stay open), and a split takes two slots at the pool's end,
// which form the next level. A tile's mask is then gathered the other way round from the reference's tree walk: each
// open leaf ORs the pixels it covers into the tiles whose region it belongs to, and each tile fills its union to the
// rectangle it spans.
#include "adaptive.h"

namespace x2 {

namespace {

// A frame queued whole does nothing once its stop word is set.
__device__ __forceinline__ bool halted(const AdaptiveArgs& a) { return a.queued && *(volatile const uint32_t*)a.stop; }

// The region of a row or column index over all regions (at most 16 regions: a linear search).
__device__ __forceinline__ uint32_t owner(const uint32_t* start, uint32_t count, uint32_t i) {
    uint32_t r = 0;
    while (r + 1 < count && start[r + 1] <= i) ++r;
    return r;
}

__device__ __forceinline__ rg::SummedErrors tableOf(const AdaptiveArgs& a, uint32_t r) {
    const int32_t* b = a.regions.box + 4 * r;
    return rg::SummedErrors{a.sat + a.regions.satOffset[r], b[0], b[1], b[2] - b[0] + 1};
}

}  // namespace

__global__ void chainPixelErrors(AdaptiveArgs a, const double* sums, const double* odd, const uint32_t* counts) {
    if (halted(a)) return;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < a.width * a.height) a.errors[i] = rg::pixelError(sums + 4ull * i, odd + 4ull * i, counts[i]);
}

__global__ void treeRoots(AdaptiveArgs a) {
    if (halted(a)) return;
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < a.regions.count) {
        const int32_t* b = a.regions.box + 4 * r;
        a.pool.x0[r] = float(b[0]);
        a.pool.y0[r] = float(b[1]);
        a.pool.x1[r] = float(b[2]);
        a.pool.y1[r] = float(b[3]);
        a.pool.child[r] = -1;
        a.pool.fate[r] = rg::kOpen;
        a.pool.region[r] = r;
        a.regions.nodes[r] = 1;
        a.regions.ready[r] = 1;
        a.regions.open[r] = 0;
    }
    if (r == 0) {
        *a.pool.count = a.regions.count;
        a.pool.level[0] = 0;
        a.pool.level[1] = a.regions.count;
    }
}

// Row y of region r: its running error sums left to right (in double, as the table keeps them) into table row y + 1;
// the thread of row 0 also clears table row 0. A pixel without both halves marks its region not ready.
__global__ void tableRows(AdaptiveArgs a) {
    if (halted(a)) return;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.regions.rows) return;
    const uint32_t r = owner(a.regions.rowStart, a.regions.count, i);
    const int32_t* b = a.regions.box + 4 * r;
    const int y = int(i - a.regions.rowStart[r]), w = b[2] - b[0];
    double* table = a.sat + a.regions.satOffset[r];
    double* out = table + size_t(y + 1) * size_t(w + 1);
    if (y == 0)
        for (int x = 0; x <= w; ++x) table[x] = 0.0;
    const float* e = a.errors + size_t(b[1] + y) * a.width + size_t(b[0]);
    bool missing = false;
    double run = 0.0;
    out[0] = 0.0;
    for (int x = 0; x < w; ++x) {
        missing |= e[x] < 0.0f;
        run += double(e[x]);
        out[x + 1] = run;
    }
    if (missing) a.regions.ready[r] = 0;
}

// Column x (1..w) of region r's table: the row sums added downwards.
__global__ void tableColumns(AdaptiveArgs a) {
    if (halted(a)) return;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.regions.cols) return;
    const uint32_t r = owner(a.regions.colStart, a.regions.count, i);
    const int32_t* b = a.regions.box + 4 * r;
    const int x = int(i - a.regions.colStart[r]) + 1, w1 = b[2] - b[0] + 1, h = b[3] - b[1];
    double* col = a.sat + a.regions.satOffset[r] + x;
    double run = col[w1];
    for (int y = 2; y <= h; ++y) {
        run += col[size_t(y) * size_t(w1)];
        col[size_t(y) * size_t(w1)] = run;
    }
}

// One level of every region's nodes. A region not ready keeps its root, open. A split allocates its two children
// within its region's bound (past it the node stays open: never, by the bound's construction) at the pool's end.
__global__ void treeLevel(AdaptiveArgs a) {
    if (halted(a)) return;
    const uint32_t begin = a.pool.level[0], end = a.pool.level[1];
    const unsigned full = 0xffffffffu;
    // A warp takes 32 consecutive nodes a round (blockDim.x is a multiple of 32).
    for (uint32_t base = begin + ((blockIdx.x * blockDim.x + threadIdx.x) & ~31u); base < end; base += gridDim.x * blockDim.x) {
        const uint32_t i = base + (threadIdx.x & 31u);
        bool split = false;
        float cut = 0.0f;
        bool alongX = false;
        uint32_t r = 0;
        if (i < end) {
            r = a.pool.region[i];
            if (!a.regions.ready[r]) {
                a.regions.open[r] = 1;
            } else {
                const int32_t* b = a.regions.box + 4 * r;
                const rg::Fate f = rg::nodeFate(tableOf(a, r), b[0], b[1], b[2], b[3], a.pool.x0[i], a.pool.y0[i], a.pool.x1[i], a.pool.y1[i],
                                                a.target, &cut, &alongX);
                if (f == rg::kConverged) a.pool.fate[i] = rg::kConverged;
                else if (f == rg::kOpen) a.regions.open[r] = 1;
                else if (atomicAdd(a.regions.nodes + r, 2u) + 2u <= a.regions.bound[r]) split = true;
                else a.regions.open[r] = 1;
            }
        }
        // The warp's splits take consecutive slot pairs with one atomic.
        const unsigned want = __ballot_sync(full, split);
        uint32_t first = 0;
        if (want && (threadIdx.x & 31u) == 0) first = atomicAdd(a.pool.count, 2u * __popc(want));
        first = __shfl_sync(full, first, 0);
        if (split) {
            const uint32_t c = first + 2u * __popc(want & ((1u << (threadIdx.x & 31u)) - 1u));
            if (c + 1 < a.pool.capacity) {
                const float x0 = a.pool.x0[i], y0 = a.pool.y0[i], x1 = a.pool.x1[i], y1 = a.pool.y1[i];
                for (uint32_t k = 0; k < 2; ++k) {
                    a.pool.x0[c + k] = alongX && k ? cut : x0;
                    a.pool.x1[c + k] = alongX && !k ? cut : x1;
                    a.pool.y0[c + k] = !alongX && k ? cut : y0;
                    a.pool.y1[c + k] = !alongX && !k ? cut : y1;
                    a.pool.child[c + k] = -1;
                    a.pool.fate[c + k] = rg::kOpen;
                    a.pool.region[c + k] = r;
                }
                a.pool.child[i] = int32_t(c);
            } else {
                a.regions.open[r] = 1;
            }
        }
    }
}

// The next level: the nodes the last one allocated. With a loop handle, go on while there are any.
__global__ void treeNextLevel(AdaptiveArgs a, cudaGraphConditionalHandle loop) {
    if (threadIdx.x != 0) return;
    const uint32_t next = min(*(volatile uint32_t*)a.pool.count, a.pool.capacity);
    a.pool.level[0] = a.pool.level[1];
    a.pool.level[1] = next;
    cudaGraphSetConditional(loop, !halted(a) && a.pool.level[0] < next ? 1u : 0u);
}

// One warp a node: an open leaf ORs the pixels it covers into each tile that intersects it and reads its region's tree
// (the region of the tile's top-left pixel).
__global__ void leafReach(AdaptiveArgs a) {
    if (halted(a)) return;
    const uint32_t warps = gridDim.x * blockDim.x / 32u, lane = threadIdx.x & 31u;
    const uint32_t n = min(*a.pool.count, a.pool.capacity);
    for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) / 32u; i < n; i += warps) {
        if (a.pool.child[i] >= 0 || a.pool.fate[i] == rg::kConverged) continue;
        const float x0 = a.pool.x0[i], y0 = a.pool.y0[i], x1 = a.pool.x1[i], y1 = a.pool.y1[i];
        const uint32_t r = a.pool.region[i];
        const int px0 = int(floorf(x0)), py0 = int(floorf(y0)), px1 = int(ceilf(x1)), py1 = int(ceilf(y1));
        const int tx0 = px0 / 8, ty0 = py0 / 8, tx1 = (px1 + 7) / 8, ty1 = (py1 + 7) / 8;
        const int across = tx1 - tx0, tilesHere = across * (ty1 - ty0);
        for (int k = int(lane); k < tilesHere; k += 32) {
            const int tx = tx0 + k % across, ty = ty0 + k / across;
            const float fx0 = float(tx * 8), fy0 = float(ty * 8), fx1 = float(tx * 8 + 8), fy1 = float(ty * 8 + 8);
            // The leaf's overlap with the tile, as the reference's walk tests it (a touching edge is no overlap).
            if (!(fminf(x1, fx1) > fmaxf(x0, fx0)) || !(fminf(y1, fy1) > fmaxf(y0, fy0))) continue;
            if (uint32_t(a.regions.grid.regionOfTile(tx * 8, ty * 8)) != r) continue;
            const int cx0 = max(px0, tx * 8) - tx * 8, cx1 = min(px1, tx * 8 + 8) - tx * 8;
            const int cy0 = max(py0, ty * 8) - ty * 8, cy1 = min(py1, ty * 8 + 8) - ty * 8;
            const uint64_t row = (0xffull >> (8 - (cx1 - cx0))) << cx0;
            uint64_t bits = 0;
            for (int y = cy0; y < cy1; ++y) bits |= row << (8 * y);
            if (bits) atomicOr(reinterpret_cast<unsigned long long*>(a.reach) + (size_t(ty) * a.tilesX + size_t(tx)), (unsigned long long)bits);
        }
    }
}

__global__ void tileMasks(AdaptiveArgs a, uint32_t uniform, uint32_t size) {
    if (halted(a)) return;
    if (!uniform) {
        bool left;
        if (a.alive) {
            left = *a.liveTiles != 0;
        } else {
            left = false;
            for (uint32_t r = 0; r < a.regions.count; ++r) left = left || a.regions.open[r] != 0;
        }
        if (!left) {
            if (blockIdx.x == 0 && threadIdx.x == 0) *a.stop = 1;
            return;
        }
    }
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.tiles) return;
    uint64_t m = a.inImage[t];
    if (!uniform) m = a.alive ? (a.alive[t] ? m : 0ull) : (m & rg::fillToBounds(a.reach[t]));
    a.tileMask[t] = m;
    const uint32_t x0 = (t % a.tilesX) * 8, y0 = (t / a.tilesX) * 8;
    for (uint64_t rest = m; rest; rest &= rest - 1) {
        const uint32_t p = uint32_t(__ffsll((long long)rest) - 1);
        const uint32_t pixel = (y0 + p / 8) * a.width + x0 + p % 8;
        a.base[pixel] = a.planned[pixel];
        a.planned[pixel] += size;
    }
}

// A tile's error over the target: its pixels' errors added row by row (in double), as a node's error over the tile's
// pixel count; a tile with a pixel not ready has the largest ratio.
__global__ void tileRatios(AdaptiveArgs a) {
    if (halted(a)) return;
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.tiles) return;
    const uint32_t x0 = (t % a.tilesX) * 8, y0 = (t / a.tilesX) * 8;
    const uint32_t x1 = min(x0 + 8, a.width), y1 = min(y0 + 8, a.height);
    double sum = 0.0;
    bool ready = true;
    for (uint32_t y = y0; y < y1; ++y) {
        const float* row = a.errors + size_t(y) * a.width;
        for (uint32_t x = x0; x < x1; ++x) {
            if (row[x] < 0.0f) ready = false;
            else sum += double(row[x]);
        }
    }
    a.ratio[t] = ready ? rg::nodeError(float(sum), float((x1 - x0) * (y1 - y0))) / a.target : 3.4e38f;
}

// The generation rule: a live tile stays at a ratio of 1, or of kSurvive with kSurviveNeighbours live neighbours of
// its eight; a dead one returns at 1, or at kBirth with kBirthNeighbours; a tile outside the image never lives.
__global__ void nextGeneration(AdaptiveArgs a, const uint8_t* aliveIn, uint8_t* aliveOut) {
    if (halted(a)) return;
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    bool lives = false;
    if (t < a.tiles) {
        const int tilesX = int(a.tilesX), tilesY = int(a.tiles / a.tilesX), tx = int(t) % tilesX, ty = int(t) / tilesX;
        int around = 0;
        for (int y = max(ty - 1, 0); y <= min(ty + 1, tilesY - 1); ++y)
            for (int x = max(tx - 1, 0); x <= min(tx + 1, tilesX - 1); ++x)
                around += (x != tx || y != ty) && aliveIn[size_t(y) * tilesX + x] ? 1 : 0;
        const float q = a.ratio[t];
        const bool was = aliveIn[t] != 0;
        lives = a.inImage[t] && (q >= 1.0f || (was ? q >= kSurvive && around >= kSurviveNeighbours : q >= kBirth && around >= kBirthNeighbours));
        aliveOut[t] = lives ? 1 : 0;
    }
    const unsigned ballot = __ballot_sync(0xffffffffu, lives);
    if ((threadIdx.x & 31u) == 0 && ballot) atomicAdd(a.liveTiles, uint32_t(__popc(ballot)));
}

__global__ void compactCount(AdaptiveArgs a) {
    if (halted(a)) return;
    __shared__ uint32_t warpTiles[kCompactBlock / 32];
    const uint32_t t = blockIdx.x * kCompactBlock + threadIdx.x;
    const bool active = t < a.tiles && a.tileMask[t] != 0;
    const unsigned ballot = __ballot_sync(0xffffffffu, active);
    if ((threadIdx.x & 31u) == 0) warpTiles[threadIdx.x / 32] = __popc(ballot);
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t n = 0;
        for (int w = 0; w < kCompactBlock / 32; ++w) n += warpTiles[w];
        a.blockTiles[blockIdx.x] = n;
    }
}

__global__ void compactWrite(AdaptiveArgs a, uint32_t size) {
    __shared__ uint32_t warpTiles[kCompactBlock / 32];
    __shared__ uint32_t blockFirst, total;
    if (halted(a)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) *a.live = 0;
        return;
    }
    // This block's first chunk: the active tiles of the blocks before it (thread 0 adds them), and the pass's total.
    if (threadIdx.x == 0) {
        uint32_t before = 0, all = 0;
        for (uint32_t b = 0; b < gridDim.x; ++b) {
            if (b == blockIdx.x) before = all;
            all += a.blockTiles[b];
        }
        blockFirst = before;
        total = all;
    }
    const uint32_t t = blockIdx.x * kCompactBlock + threadIdx.x;
    const uint64_t m = t < a.tiles ? a.tileMask[t] : 0ull;
    const unsigned ballot = __ballot_sync(0xffffffffu, m != 0);
    if ((threadIdx.x & 31u) == 0) warpTiles[threadIdx.x / 32] = __popc(ballot);
    __syncthreads();
    uint32_t at = blockFirst + __popc(ballot & ((1u << (threadIdx.x & 31u)) - 1u));
    for (uint32_t w = 0; w < threadIdx.x / 32; ++w) at += warpTiles[w];
    if (m) {
        a.chunks[at] = x2_chunk{t, 0, size, 0};
        a.chunkMasks[at] = m;
    }
    // The pass's samples (its active pixels times its size), a warp's at a time.
    unsigned long long pixels = __popcll(m);
    for (int off = 16; off; off >>= 1) pixels += __shfl_down_sync(0xffffffffu, pixels, off);
    if ((threadIdx.x & 31u) == 0 && pixels) atomicAdd(a.samples, pixels * size);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *a.live = total;
        if (total) ++*a.passes;
        else *a.stop = 1;
    }
}

}  // namespace x2
