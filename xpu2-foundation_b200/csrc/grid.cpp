// The work grid (row f1 of the path's scope): the image cut into square cells, each holding its unstarted chunks in
// a queue that one writer appends to and any number of claimants take from (one atomic cursor, so a chunk is claimed
// exactly once); a uniform frame's sample ranges, in the progressive order (1, 1, 2, then the chunk size) behind a
// frontier; cell owners, scores and the rights of passage; and the cellular choice of where a worker goes next — the
// reference's Grid (xpu2/interactive/async_grid.h:96-430). The GPU broker on top (x2_workgrid_take, x2_render_workgrid)
// forms each wavefront launch from the shares of the GPU's cellular workers, as the reference's feeder forms a GPU
// launch (async_render.h:600-605, 780-797).
#include <algorithm>
#include <atomic>
#include <chrono>
#include <climits>
#include <cstring>
#include <memory>
#include <new>
#include <vector>

#include "../../include/x2.h"

namespace {

constexpr uint32_t kTile = 8;

// A cell's chunk queue. Chunks live in fixed blocks that never move once written; the writer publishes a count after
// writing, and a claim never passes the published count or the caller's limit.
class CellQueue {
   public:
    static constexpr uint32_t kBlock = 4096, kMaxBlocks = 2048;
    CellQueue() : blocks_(new std::atomic<x2_chunk*>[kMaxBlocks]) {
        for (uint32_t i = 0; i < kMaxBlocks; ++i) blocks_[i].store(nullptr, std::memory_order_relaxed);
    }
    ~CellQueue() {
        for (uint32_t i = 0; i < kMaxBlocks; ++i) delete[] blocks_[i].load(std::memory_order_relaxed);
    }
    CellQueue(const CellQueue&) = delete;
    CellQueue& operator=(const CellQueue&) = delete;

    // The single writer: false when the queue would exceed its capacity (nothing is written then).
    bool append(const x2_chunk* chunks, uint32_t n) {
        uint32_t at = published_.load(std::memory_order_relaxed);
        if (uint64_t(at) + n > uint64_t(kBlock) * kMaxBlocks) return false;
        for (uint32_t i = 0; i < n; ++i, ++at) {
            std::atomic<x2_chunk*>& slot = blocks_[at / kBlock];
            x2_chunk* block = slot.load(std::memory_order_relaxed);
            if (!block) {
                block = new x2_chunk[kBlock];
                slot.store(block, std::memory_order_relaxed);
            }
            block[at % kBlock] = chunks[i];
        }
        published_.store(at, std::memory_order_release);
        return true;
    }
    uint32_t published() const { return published_.load(std::memory_order_acquire); }
    uint32_t taken() const { return next_.load(std::memory_order_acquire); }
    uint32_t remaining() const {
        const uint32_t end = published(), t = taken();
        return t >= end ? 0 : end - t;
    }
    // Up to n chunks from the cursor, none at or past position `limit`.
    uint32_t claim(uint32_t n, x2_chunk* out, uint32_t limit) {
        const uint32_t end = std::min(published(), limit);
        uint32_t start = next_.load(std::memory_order_relaxed), stop = 0;
        do {
            if (start >= end) return 0;
            stop = start + std::min(n, end - start);
        } while (!next_.compare_exchange_weak(start, stop, std::memory_order_acq_rel, std::memory_order_relaxed));
        for (uint32_t i = start; i < stop; ++i) out[i - start] = blocks_[i / kBlock].load(std::memory_order_relaxed)[i % kBlock];
        return stop - start;
    }

   private:
    std::unique_ptr<std::atomic<x2_chunk*>[]> blocks_;
    alignas(64) std::atomic<uint32_t> published_{0};
    alignas(64) std::atomic<uint32_t> next_{0};
};

struct Cell {
    uint32_t x = 0, y = 0;
    uint32_t owner = X2_DEVICE_CPU;
    CellQueue queue;
    std::atomic<uint64_t> samples[2] = {};  // rendered by each device
    uint32_t tiles = 0;                     // its tiles with pixels in the frame: one sample range's chunks
    float gpu = 0.5f;                       // the GPU's suitability for it (a probability)
    std::atomic<float> score{0.0f};         // what is in it, once the picture is scored
    std::atomic<bool> important{false};
};

struct Range {
    uint32_t first, count;
};

long long nowNs() {
    return std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// The tie-break among equally good cells, a hash of (cell, worker salt) so workers spread out. Its constants are the
// reference's (async_grid.h hash), so both grids break ties alike.
uint32_t spread(uint32_t a, uint32_t b) {
    uint32_t h = a * 0x9e3779b1u ^ (b + 0x7f4a7c15u + (a << 6) + (a >> 2));
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    return h;
}

}  // namespace

struct x2_workgrid {
    uint32_t width = 0, height = 0, spp = 0, cellsX = 0, cellsY = 0;
    int32_t view[4] = {0, 0, INT_MAX, INT_MAX};
    x2_workgrid_options options{};
    std::unique_ptr<Cell[]> cells;
    uint32_t cellCount = 0;
    std::atomic<uint64_t> total{0};
    std::atomic<bool> closed{false};
    std::vector<Range> ranges;  // a uniform frame's sample ranges (none: cells filled by append)
    std::atomic<uint32_t> frontier[2] = {};
    std::atomic<bool> scored{false};
    // The coordinator's measurements for the rights of passage.
    std::atomic<double> gpuItems{0.0}, cpuWorker{0.0}, window{0.01};
    std::atomic<uint32_t> cpuWorkers{1};
    std::atomic<long long> gpuClaim{0};
    // The GPU broker: its cellular workers' cells (seeded at its first launch) and the chunks it took from cells the
    // CPU owns.
    std::vector<uint32_t> gpuCells;
    uint64_t stolen = 0;

    uint32_t tilesX() const { return (width + kTile - 1) / kTile; }
    uint32_t tilePixels(uint32_t tile) const {
        const int x = int((tile % tilesX()) * kTile), y = int((tile / tilesX()) * kTile);
        const int x0 = std::max(x, view[0]), y0 = std::max(y, view[1]);
        const int x1 = std::min({x + int(kTile), int(width), view[2]}), y1 = std::min({y + int(kTile), int(height), view[3]});
        return x1 > x0 && y1 > y0 ? uint32_t(x1 - x0) * uint32_t(y1 - y0) : 0u;
    }
    bool important(uint32_t i) const { return cells[i].important.load(std::memory_order_relaxed); }
    bool isScored() const { return scored.load(std::memory_order_acquire); }
    // A cell its owner works first: all of them until the picture is scored, then the important ones.
    bool reserved(uint32_t i) const { return !isScored() || important(i); }
    bool isClosed() const { return closed.load(std::memory_order_acquire); }
    uint32_t remaining(uint32_t i) const { return isClosed() ? 0u : cells[i].queue.remaining(); }
    uint32_t frontierOf(uint32_t device) const { return frontier[device].load(std::memory_order_acquire); }

    // The queue positions of a cell a device may claim up to: every chunk of the ranges up to its frontier, and one
    // range more in an important cell.
    uint32_t limit(uint32_t i, uint32_t device) const {
        if (ranges.empty()) return ~0u;
        const uint64_t lead = isScored() && important(i) ? 1 : 0;
        const uint64_t upTo = std::min<uint64_t>(uint64_t(frontierOf(device)) + lead + 1, ranges.size());
        return uint32_t(std::min<uint64_t>(upTo * cells[i].tiles, ~0u));
    }
    uint32_t claimable(uint32_t i, uint32_t device) const {
        if (isClosed()) return 0;
        const CellQueue& q = cells[i].queue;
        const uint32_t end = std::min(q.published(), limit(i, device)), t = q.taken();
        return t >= end ? 0 : end - t;
    }
    // Each device's frontier: the least range still to hand out among its own reserved cells and the open ones (among
    // every cell when none is left there), at most the range count.
    void refreshFrontiers() {
        if (ranges.empty()) return;
        uint32_t least[3] = {~0u, ~0u, ~0u};  // the CPU's, the GPU's, every cell's
        for (uint32_t i = 0; i < cellCount; ++i) {
            const Cell& c = cells[i];
            if (!c.tiles || !c.queue.remaining()) continue;
            const uint32_t range = c.queue.taken() / c.tiles;
            const bool open = !reserved(i);
            for (uint32_t d = 0; d < 2; ++d)
                if (open || c.owner == d) least[d] = std::min(least[d], range);
            least[2] = std::min(least[2], range);
        }
        for (uint32_t d = 0; d < 2; ++d)
            frontier[d].store(std::min<uint32_t>(least[d] != ~0u ? least[d] : least[2], uint32_t(ranges.size())), std::memory_order_release);
    }
    uint32_t claim(uint32_t i, uint32_t n, x2_chunk* out, uint32_t device) {
        if (isClosed()) return 0;
        const uint32_t got = cells[i].queue.claim(n, out, limit(i, device));
        if (got && !ranges.empty()) refreshFrontiers();
        return got;
    }
    uint64_t reservedChunks(uint32_t device) const {
        uint64_t n = 0;
        for (uint32_t i = 0; i < cellCount; ++i)
            if (cells[i].owner == device && reserved(i)) n += remaining(i);
        return n;
    }
    // Whether a device may work in a cell the other has reserved: yes before anything is measured; the CPU when the
    // GPU has not claimed for a while, or when one CPU chunk ends well before the GPU would finish its reserved work;
    // the GPU when the CPU's reserved work outlasts a few of its launches, in a cell suited to it.
    bool passage(uint32_t device, uint32_t i) const {
        const double g = gpuItems.load(std::memory_order_relaxed), c = cpuWorker.load(std::memory_order_relaxed);
        if (g <= 0 || c <= 0) return true;
        const double chunk = double(options.samples_per_chunk) * kTile * kTile, w = window.load(std::memory_order_relaxed);
        if (device == X2_DEVICE_CPU) {
            const long long last = gpuClaim.load(std::memory_order_relaxed);
            if (last && double(nowNs() - last) * 1e-9 > std::max(4 * w, 0.05)) return true;
            return chunk / c < 0.5 * double(reservedChunks(X2_DEVICE_GPU)) * chunk / g;
        }
        if (cells[i].gpu < 0.2f) return false;
        const uint32_t workers = std::max(1u, cpuWorkers.load(std::memory_order_relaxed));
        return double(reservedChunks(X2_DEVICE_CPU)) * chunk / (c * workers) > 4 * w;
    }
    template <class F>
    void neighbours(uint32_t i, F f) const {
        const int x = int(i % cellsX), y = int(i / cellsX);
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx) {
                const int nx = x + dx, ny = y + dy;
                if ((dx || dy) && nx >= 0 && ny >= 0 && nx < int(cellsX) && ny < int(cellsY)) f(uint32_t(ny) * cellsX + uint32_t(nx));
            }
    }
    // Where a worker of a device goes next (~0u: nowhere now). It finishes its cell; then, tier by tier — its device's
    // reserved cells (the most unclaimed work first), the open ones (the highest score first), the other device's
    // reserved ones by a right of passage — a neighbour of its cell before the best cell anywhere.
    uint32_t choose(uint32_t device, uint32_t current, uint32_t salt) const {
        auto tier = [&](uint32_t i) { return !reserved(i) ? 1 : cells[i].owner == device ? 0 : 2; };
        int cpuPassage = -1;  // the CPU's right of passage does not depend on the cell: worked out once
        auto passes = [&](uint32_t i) {
            if (device == X2_DEVICE_GPU) return passage(device, i);
            if (cpuPassage < 0) cpuPassage = passage(device, i) ? 1 : 0;
            return cpuPassage == 1;
        };
        if (current < cellCount && claimable(current, device) && (tier(current) != 2 || passes(current))) return current;
        for (int t = 0; t < 3; ++t) {
            uint32_t best = ~0u;
            float bestKey = 0;
            auto consider = [&](uint32_t i) {
                if (tier(i) != t) return;
                const uint32_t work = claimable(i, device);
                if (!work || (t == 2 && !passes(i))) return;
                const float key = t == 1 ? cells[i].score.load(std::memory_order_relaxed) + 1e-9f * float(work) : float(work);
                if (best == ~0u || key > bestKey || (key == bestKey && spread(i, salt) > spread(best, salt))) {
                    best = i;
                    bestKey = key;
                }
            };
            if (current < cellCount) {
                neighbours(current, consider);
                if (best != ~0u) return best;
            }
            for (uint32_t i = 0; i < cellCount; ++i) consider(i);
            if (best != ~0u) return best;
        }
        return ~0u;
    }
    // The starting cell of worker w of n on a device: its cells spread evenly over them.
    uint32_t seed(uint32_t device, uint32_t worker, uint32_t workers) const {
        std::vector<uint32_t> own;
        for (uint32_t i = 0; i < cellCount; ++i)
            if (cells[i].owner == device) own.push_back(i);
        if (own.empty()) return choose(device, ~0u, worker);
        return own[(size_t(worker) * own.size()) / std::max(1u, workers)];
    }
};

extern "C" {

void x2_workgrid_options_defaults(x2_workgrid_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->cell_size = 64;
    o->samples_per_chunk = 4;
    o->mode = X2_WORKGRID_BOTH;
    o->progressive = 1;
    o->gpu_workers = 32;
}

int x2_workgrid_create(uint32_t width, uint32_t height, uint32_t spp, const x2_workgrid_options* options, const uint32_t* owners, uint32_t ownerCount,
                   uint32_t empty, const int32_t* viewport, x2_workgrid** out) {
    if (!out) return X2_EINVAL;
    *out = nullptr;
    x2_workgrid_options o;
    if (options) o = *options;
    else x2_workgrid_options_defaults(&o);
    if (!width || !height || !spp || !o.cell_size || o.cell_size % kTile || !o.samples_per_chunk || o.mode < X2_WORKGRID_CPU ||
        o.mode > X2_WORKGRID_BOTH)
        return X2_EINVAL;
    x2_workgrid* g = new (std::nothrow) x2_workgrid();
    if (!g) return X2_ENOMEM;
    g->width = width;
    g->height = height;
    g->spp = spp;
    g->options = o;
    if (viewport) std::memcpy(g->view, viewport, sizeof(g->view));
    g->cellsX = (width + o.cell_size - 1) / o.cell_size;
    g->cellsY = (height + o.cell_size - 1) / o.cell_size;
    g->cellCount = g->cellsX * g->cellsY;
    g->cells.reset(new (std::nothrow) Cell[g->cellCount]);
    if (!g->cells) {
        delete g;
        return X2_ENOMEM;
    }
    if (owners && ownerCount != g->cellCount) owners = nullptr;
    if (!empty) {
        const uint32_t from = o.sample_count ? o.sample_first : 0u, to = o.sample_count ? std::min(spp, o.sample_first + o.sample_count) : spp;
        for (uint32_t first = from; first < to;) {
            const uint32_t done = first - from;
            const uint32_t size = !o.progressive ? o.samples_per_chunk : done < 2 ? 1u : done < 4 ? 2u : o.samples_per_chunk;
            g->ranges.push_back({first, std::min(size, to - first)});
            first += g->ranges.back().count;
        }
    }
    const uint32_t tilesX = (width + kTile - 1) / kTile, tilesY = (height + kTile - 1) / kTile, perCell = o.cell_size / kTile;
    std::vector<x2_chunk> chunks;
    for (uint32_t cy = 0; cy < g->cellsY; ++cy)
        for (uint32_t cx = 0; cx < g->cellsX; ++cx) {
            const uint32_t index = cy * g->cellsX + cx;
            Cell& c = g->cells[index];
            c.x = cx;
            c.y = cy;
            c.owner = o.mode == X2_WORKGRID_CPU   ? uint32_t(X2_DEVICE_CPU)
                      : o.mode == X2_WORKGRID_GPU ? uint32_t(X2_DEVICE_GPU)
                      : owners                ? (owners[index] ? uint32_t(X2_DEVICE_GPU) : uint32_t(X2_DEVICE_CPU))
                                              : ((cx + cy) % 2 == 0 ? uint32_t(X2_DEVICE_GPU) : uint32_t(X2_DEVICE_CPU));
            if (empty) continue;
            // The cell's chunks by sample range, then by tile (row-major within the cell).
            chunks.clear();
            for (const Range& r : g->ranges)
                for (uint32_t ty = cy * perCell; ty < std::min(tilesY, (cy + 1) * perCell); ++ty)
                    for (uint32_t tx = cx * perCell; tx < std::min(tilesX, (cx + 1) * perCell); ++tx)
                        if (g->tilePixels(ty * tilesX + tx)) chunks.push_back(x2_chunk{ty * tilesX + tx, r.first, r.count, index});
            c.tiles = g->ranges.empty() ? 0 : uint32_t(chunks.size() / g->ranges.size());
            if (!c.queue.append(chunks.data(), uint32_t(chunks.size()))) {
                delete g;
                return X2_EINVAL;
            }
            g->total += chunks.size();
        }
    g->refreshFrontiers();
    *out = g;
    return X2_OK;
}

void x2_workgrid_free(x2_workgrid* g) { delete g; }

int x2_workgrid_info(const x2_workgrid* g, uint32_t* width, uint32_t* height, uint32_t* spp, x2_workgrid_options* options) {
    if (!g) return X2_EINVAL;
    if (width) *width = g->width;
    if (height) *height = g->height;
    if (spp) *spp = g->spp;
    if (options) *options = g->options;
    return X2_OK;
}

uint32_t x2_workgrid_cells(const x2_workgrid* g) { return g ? g->cellCount : 0; }
uint64_t x2_workgrid_total(const x2_workgrid* g) { return g ? g->total.load() : 0; }

uint32_t x2_workgrid_ranges(const x2_workgrid* g, uint32_t* ranges, uint32_t capacity) {
    if (!g) return 0;
    for (uint32_t k = 0; ranges && k < g->ranges.size() && k < capacity; ++k) {
        ranges[2 * k] = g->ranges[k].first;
        ranges[2 * k + 1] = g->ranges[k].count;
    }
    return uint32_t(g->ranges.size());
}

int x2_workgrid_cell(const x2_workgrid* g, uint32_t cell, uint32_t* owner, uint32_t* tiles, uint32_t* published, uint32_t* taken) {
    if (!g || cell >= g->cellCount) return X2_EINVAL;
    const Cell& c = g->cells[cell];
    if (owner) *owner = c.owner;
    if (tiles) *tiles = c.tiles;
    if (published) *published = c.queue.published();
    if (taken) *taken = c.queue.taken();
    return X2_OK;
}

int x2_workgrid_append(x2_workgrid* g, uint32_t cell, const x2_chunk* chunks, uint32_t n) {
    if (!g || cell >= g->cellCount || (n && !chunks)) return X2_EINVAL;
    if (!g->cells[cell].queue.append(chunks, n)) return X2_EINVAL;
    g->total += n;
    return X2_OK;
}

uint32_t x2_workgrid_claim(x2_workgrid* g, uint32_t cell, uint32_t n, x2_chunk* out, uint32_t device) {
    if (!g || cell >= g->cellCount || !out || device > X2_DEVICE_GPU) return 0;
    return g->claim(cell, n, out, device);
}

uint32_t x2_workgrid_claimable(const x2_workgrid* g, uint32_t cell, uint32_t device) {
    if (!g || cell >= g->cellCount || device > X2_DEVICE_GPU) return 0;
    return g->claimable(cell, device);
}

uint32_t x2_workgrid_remaining(const x2_workgrid* g, uint32_t cell) {
    if (!g || cell >= g->cellCount) return 0;
    return g->remaining(cell);
}

uint32_t x2_workgrid_empty(const x2_workgrid* g) {
    if (!g) return 1;
    for (uint32_t i = 0; i < g->cellCount; ++i)
        if (g->remaining(i)) return 0;
    return 1;
}

uint32_t x2_workgrid_frontier(const x2_workgrid* g, uint32_t device) { return g && device <= X2_DEVICE_GPU ? g->frontierOf(device) : 0; }

uint32_t x2_workgrid_choose(const x2_workgrid* g, uint32_t device, uint32_t current, uint32_t salt) {
    return g && device <= X2_DEVICE_GPU ? g->choose(device, current, salt) : ~0u;
}

uint32_t x2_workgrid_seed(const x2_workgrid* g, uint32_t device, uint32_t worker, uint32_t workers) {
    return g && device <= X2_DEVICE_GPU ? g->seed(device, worker, workers) : ~0u;
}

// Important parts first: each cell's score (below zero: not known). The cells above the mean of the known scores are
// important; the picture counts as scored from then on.
int x2_workgrid_set_scores(x2_workgrid* g, const float* scores, uint32_t n) {
    if (!g || !scores) return X2_EINVAL;
    if (n != g->cellCount) return X2_OK;
    double sum = 0;
    uint32_t known = 0;
    for (uint32_t i = 0; i < n; ++i)
        if (scores[i] >= 0) {
            sum += scores[i];
            ++known;
        }
    if (!known) return X2_OK;
    const float mean = float(sum / known);
    for (uint32_t i = 0; i < n; ++i) {
        g->cells[i].score.store(std::max(scores[i], 0.0f), std::memory_order_relaxed);
        g->cells[i].important.store(scores[i] > mean, std::memory_order_relaxed);
    }
    g->scored.store(true, std::memory_order_release);
    g->refreshFrontiers();
    return X2_OK;
}

int x2_workgrid_set_suitability(x2_workgrid* g, const float* gpu, uint32_t n) {
    if (!g || !gpu) return X2_EINVAL;
    if (n == g->cellCount)
        for (uint32_t i = 0; i < n; ++i) g->cells[i].gpu = gpu[i];
    return X2_OK;
}

int x2_workgrid_set_rates(x2_workgrid* g, double gpuItems, double cpuWorker, uint32_t cpuWorkers, double window) {
    if (!g) return X2_EINVAL;
    g->gpuItems.store(gpuItems, std::memory_order_relaxed);
    g->cpuWorker.store(cpuWorker, std::memory_order_relaxed);
    g->cpuWorkers.store(cpuWorkers, std::memory_order_relaxed);
    g->window.store(window, std::memory_order_relaxed);
    return X2_OK;
}

int x2_workgrid_rendered(x2_workgrid* g, uint32_t cell, uint32_t device, uint64_t samples) {
    if (!g || cell >= g->cellCount || device > X2_DEVICE_GPU) return X2_EINVAL;
    g->cells[cell].samples[device].fetch_add(samples, std::memory_order_relaxed);
    return X2_OK;
}

void x2_workgrid_close(x2_workgrid* g) {
    if (g) g->closed.store(true, std::memory_order_release);
}

// The GPU broker's next launch: up to `want` chunks, split into equal shares for the GPU's cellular workers, each
// taking its share from its cell and moving by the cellular rules (at most 8 moves) where that cell has nothing more
// it may take now.
uint32_t x2_workgrid_take(x2_workgrid* g, uint32_t want, x2_chunk* out) {
    if (!g || !out || !want) return 0;
    if (g->gpuCells.empty()) {
        g->gpuCells.assign(std::max(1u, g->options.gpu_workers), ~0u);
        for (uint32_t w = 0; w < g->gpuCells.size(); ++w) g->gpuCells[w] = g->seed(X2_DEVICE_GPU, w, uint32_t(g->gpuCells.size()));
    }
    const uint32_t workers = uint32_t(g->gpuCells.size()), share = (want + workers - 1) / workers;
    uint32_t got = 0;
    for (uint32_t w = 0; w < workers && got < want; ++w)
        for (uint32_t need = std::min(share, want - got), moves = 0; need && moves < 8; ++moves) {
            const uint32_t cell = g->choose(X2_DEVICE_GPU, g->gpuCells[w], w);
            if (cell == ~0u) break;
            g->gpuCells[w] = cell;
            const uint32_t n = g->claim(cell, need, out + got, X2_DEVICE_GPU);
            if (n && g->cells[cell].owner != X2_DEVICE_GPU) g->stolen += n;
            got += n;
            need -= n;
        }
    if (got) g->gpuClaim.store(nowNs(), std::memory_order_relaxed);
    return got;
}

uint64_t x2_workgrid_stolen(const x2_workgrid* g) { return g ? g->stolen : 0; }

// Cell ownership across the frames of one grid size (the reference's Ownership, async_grid.h:432-480): each finished
// frame records every cell's GPU share of its samples in an 8-frame window; from the ninth frame on, a cell whose
// other device took more than 0.6 of the window's samples flips, at most min(8, max(1, cells / 10)) a frame, the
// furthest ahead first (ties by cell index), a cell at most once in 16 frames; a cell flipping back within 32 frames
// freezes every flip for 64 frames instead.
struct x2_workgrid_ownership {
    static constexpr uint32_t kWindow = 8;
    std::vector<uint32_t> owners;
    std::vector<float> history;
    std::vector<long long> lastFlip;
    long long frame = 0, frozenUntil = 0;
};

int x2_workgrid_ownership_create(x2_workgrid_ownership** out) {
    if (!out) return X2_EINVAL;
    *out = new (std::nothrow) x2_workgrid_ownership();
    return *out ? X2_OK : X2_ENOMEM;
}

void x2_workgrid_ownership_free(x2_workgrid_ownership* o) { delete o; }

uint32_t x2_workgrid_ownership_owners(const x2_workgrid_ownership* o, uint32_t cells, uint32_t* owners) {
    if (!o || o->owners.size() != cells || !cells) return 0;
    if (owners) std::copy(o->owners.begin(), o->owners.end(), owners);
    return 1;
}

int x2_workgrid_ownership_finished(x2_workgrid_ownership* o, const x2_workgrid* g) {
    if (!o || !g) return X2_EINVAL;
    constexpr uint32_t W = x2_workgrid_ownership::kWindow;
    const uint32_t n = g->cellCount;
    if (o->owners.size() != n) {
        o->owners.resize(n);
        o->history.assign(size_t(n) * W, 0.0f);
        o->lastFlip.assign(n, -1000000);
        for (uint32_t i = 0; i < n; ++i) o->owners[i] = g->cells[i].owner;
    }
    for (uint32_t i = 0; i < n; ++i) {
        const double cpu = double(g->cells[i].samples[0].load()), gpu = double(g->cells[i].samples[1].load());
        o->history[size_t(i) * W + size_t(o->frame % W)] = cpu + gpu > 0 ? float(gpu / (cpu + gpu)) : 0.5f;
    }
    ++o->frame;
    if (o->frame < o->frozenUntil || o->frame < W) return X2_OK;
    std::vector<std::pair<float, uint32_t>> flips;  // (the other device's share, cell)
    for (uint32_t i = 0; i < n; ++i) {
        if (o->frame - o->lastFlip[i] < 16) continue;
        float gpuShare = 0;
        for (uint32_t k = 0; k < W; ++k) gpuShare += o->history[size_t(i) * W + k];
        gpuShare /= W;
        const float other = o->owners[i] == X2_DEVICE_CPU ? gpuShare : 1 - gpuShare;
        if (other > 0.6f) flips.push_back({other, i});
    }
    std::stable_sort(flips.begin(), flips.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
    const size_t limit = std::min<size_t>(8, std::max<size_t>(1, n / 10));
    for (size_t k = 0; k < flips.size() && k < limit; ++k) {
        const uint32_t i = flips[k].second;
        if (o->frame - o->lastFlip[i] < 32) {
            o->frozenUntil = o->frame + 64;
            return X2_OK;
        }
        o->owners[i] = o->owners[i] == X2_DEVICE_CPU ? uint32_t(X2_DEVICE_GPU) : uint32_t(X2_DEVICE_CPU);
        o->lastFlip[i] = o->frame;
    }
    return X2_OK;
}

}  // extern "C"
