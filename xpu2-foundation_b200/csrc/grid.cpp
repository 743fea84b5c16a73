// The work grid and its broker (row f1 of the path's scope), for a GPU-only renderer.
//
// What it must do, from the reference (xpu2/interactive/async_grid.h:96-430 Grid with GridOptions::mode 1, and the
// feeder's GPU claims, async_render.h:600-605, 780-797): hand the lane the same chunks, in the same order, as the
// reference's grid hands its GPU lane. The rules that fix that order are the reference's and are kept: the sample
// ranges of a uniform frame (progressive 1, 1, 2, then the chunk size), a cell's chunks by range then tile, the
// frontier (the least range still unclaimed among cells with work left) with an important cell's one-range lead, the
// cellular choice (finish the cell; the reserved cells by their unclaimed work, then the open ones by score; a
// neighbour before the best anywhere; ties by a hash of cell and worker), the even spread of starting cells, and the
// feeder's equal shares with at most 8 moves a worker.
//
// How it is built here:
//  - A uniform frame's chunks are never stored. A cell keeps the list of its tiles with pixels in the viewport
//    (one array for all cells, indexed by an offset table), and its queue position k is the chunk (tile k mod n,
//    range k div n) computed on demand; only chunks appended later (an adaptive frame's passes) are stored, in
//    pages that never move once written.
//  - Each cell's state is two counters: chunks published and chunks taken. A claim is a compare-and-swap on the
//    taken counter bounded by the published count and the frontier's limit, so every chunk goes out exactly once.
//  - There is one device. The reference's CPU lane (cell owners, rights of passage, rates, suitability, ownership
//    across frames) has no part here: every cell is the GPU's, so a cell is "reserved" (worked first, by its
//    unclaimed work) until scores arrive and afterwards only when important; the rest are "open" (by score).
#include <algorithm>
#include <atomic>
#include <cstring>
#include <memory>
#include <new>
#include <vector>

#include "../../include/x2.h"

namespace {

constexpr uint32_t kTileSize = 8;
constexpr uint32_t kNone = ~0u;
constexpr uint32_t kPageChunks = 2048, kMaxPages = 4096;  // appended chunks a cell: up to 8M

// The tie-break hash of the cellular choice (the reference's constants; its value decides which of equally good cells
// a worker takes, so workers spread out the same way).
inline uint32_t spreadHash(uint32_t cell, uint32_t salt) {
    uint32_t h = cell * 0x9e3779b1u ^ (salt + 0x7f4a7c15u + (cell << 6) + (cell >> 2));
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    return h;
}

// Appended chunks of one cell: pages of kPageChunks allocated as the writer reaches them. A reader only reads
// positions below the published count it loaded with acquire order, all written (and their pages set) before it.
struct AppendedPages {
    std::unique_ptr<std::atomic<x2_chunk*>[]> page;
    AppendedPages() : page(new std::atomic<x2_chunk*>[kMaxPages]) {
        for (uint32_t i = 0; i < kMaxPages; ++i) page[i].store(nullptr, std::memory_order_relaxed);
    }
    ~AppendedPages() {
        for (uint32_t i = 0; i < kMaxPages; ++i) delete[] page[i].load(std::memory_order_relaxed);
    }
    const x2_chunk& at(uint32_t k) const { return page[k / kPageChunks].load(std::memory_order_relaxed)[k % kPageChunks]; }
    bool put(uint32_t k, const x2_chunk& c) {
        if (k / kPageChunks >= kMaxPages) return false;
        std::atomic<x2_chunk*>& slot = page[k / kPageChunks];
        x2_chunk* p = slot.load(std::memory_order_relaxed);
        if (!p) {
            p = new (std::nothrow) x2_chunk[kPageChunks];
            if (!p) return false;
            slot.store(p, std::memory_order_relaxed);
        }
        p[k % kPageChunks] = c;
        return true;
    }
};

}  // namespace

struct x2_workgrid {
    uint32_t width = 0, height = 0, spp = 0;
    x2_workgrid_options options{};
    int32_t view[4] = {0, 0, 0x7fffffff, 0x7fffffff};
    uint32_t tilesX = 0, tilesY = 0, cellsX = 0, cellsY = 0, tilesPerCell = 0;
    std::vector<uint32_t> rangeFirst, rangeCount;  // a uniform frame's sample ranges (none: an empty grid)

    // Per cell. tileOffset[c]..tileOffset[c+1]: the cell's tiles in tileList, row-major within the cell.
    std::vector<uint32_t> tileOffset, tileList;
    std::unique_ptr<std::atomic<uint32_t>[]> published, taken;
    std::vector<std::unique_ptr<AppendedPages>> appended;
    std::unique_ptr<std::atomic<float>[]> score;
    std::unique_ptr<std::atomic<uint8_t>[]> important;

    std::atomic<uint64_t> total{0};
    std::atomic<bool> closed{false}, scored{false};
    std::atomic<uint32_t> frontierRange{0};
    std::vector<uint32_t> workerCell;  // the broker's workers' cells (seeded at its first take)

    uint32_t cellCount() const { return cellsX * cellsY; }
    uint32_t tiles(uint32_t c) const { return tileOffset[c + 1] - tileOffset[c]; }
    uint32_t uniformChunks(uint32_t c) const { return uint32_t(rangeFirst.size()) * tiles(c); }

    // Pixels of a tile inside the image and the viewport.
    uint32_t tileArea(uint32_t tile) const {
        const int x = int((tile % tilesX) * kTileSize), y = int((tile / tilesX) * kTileSize);
        const int x0 = std::max(x, view[0]), y0 = std::max(y, view[1]);
        const int x1 = std::min(std::min(x + int(kTileSize), int(width)), view[2]);
        const int y1 = std::min(std::min(y + int(kTileSize), int(height)), view[3]);
        return x1 > x0 && y1 > y0 ? uint32_t(x1 - x0) * uint32_t(y1 - y0) : 0u;
    }
    // Queue position k of cell c.
    x2_chunk chunkAt(uint32_t c, uint32_t k) const {
        const uint32_t u = uniformChunks(c);
        if (k >= u) return appended[c]->at(k - u);
        const uint32_t n = tiles(c), r = k / n;
        return x2_chunk{tileList[tileOffset[c] + k % n], rangeFirst[r], rangeCount[r], c};
    }
    uint32_t left(uint32_t c) const {
        const uint32_t p = published[c].load(std::memory_order_acquire), t = taken[c].load(std::memory_order_acquire);
        return t < p ? p - t : 0u;
    }
    bool reserved(uint32_t c) const { return !scored.load(std::memory_order_acquire) || important[c].load(std::memory_order_relaxed); }
    // The queue position a claim in cell c may not reach: the frontier's range plus one (two for an important cell),
    // in chunks; no bound for an empty grid's appended passes.
    uint32_t bound(uint32_t c) const {
        const uint64_t ranges = rangeFirst.size();
        if (!ranges) return kNone;
        const uint64_t lead = scored.load(std::memory_order_acquire) && important[c].load(std::memory_order_relaxed) ? 2 : 1;
        const uint64_t upTo = std::min<uint64_t>(uint64_t(frontierRange.load(std::memory_order_acquire)) + lead, ranges);
        return uint32_t(std::min<uint64_t>(upTo * tiles(c), kNone));
    }
    uint32_t open(uint32_t c) const {
        if (closed.load(std::memory_order_acquire)) return 0;
        const uint32_t end = std::min(published[c].load(std::memory_order_acquire), bound(c));
        const uint32_t t = taken[c].load(std::memory_order_acquire);
        return t < end ? end - t : 0u;
    }
    // The frontier: the least range any cell with tiles and work left still has to hand out (the number of ranges when
    // none has).
    void advanceFrontier() {
        const uint32_t ranges = uint32_t(rangeFirst.size());
        if (!ranges) return;
        uint32_t least = ranges;
        for (uint32_t c = 0; c < cellCount(); ++c) {
            const uint32_t n = tiles(c);
            if (n && left(c)) least = std::min(least, taken[c].load(std::memory_order_acquire) / n);
        }
        frontierRange.store(least, std::memory_order_release);
    }
    uint32_t claim(uint32_t c, uint32_t n, x2_chunk* out) {
        if (closed.load(std::memory_order_acquire) || !n) return 0;
        const uint32_t end = std::min(published[c].load(std::memory_order_acquire), bound(c));
        uint32_t from = taken[c].load(std::memory_order_relaxed), to = 0;
        do {
            if (from >= end) return 0;
            to = from + std::min(n, end - from);
        } while (!taken[c].compare_exchange_weak(from, to, std::memory_order_acq_rel, std::memory_order_relaxed));
        for (uint32_t k = from; k < to; ++k) out[k - from] = chunkAt(c, k);
        if (!rangeFirst.empty()) advanceFrontier();
        return to - from;
    }
    // Where a worker in cell `current` goes next (the cellular rules), kNone when nothing may be taken now.
    uint32_t choose(uint32_t current, uint32_t salt) const {
        const uint32_t cells = cellCount();
        if (current < cells && open(current)) return current;
        // Two tiers: reserved cells ranked by their open work, then the open ones by score (work breaking near-ties).
        for (int tier = 0; tier < 2; ++tier) {
            uint32_t best = kNone;
            float bestKey = 0.0f;
            auto rank = [&](uint32_t c) {
                if ((reserved(c) ? 0 : 1) != tier) return;
                const uint32_t work = open(c);
                if (!work) return;
                const float key = tier ? score[c].load(std::memory_order_relaxed) + 1e-9f * float(work) : float(work);
                const bool better = best == kNone || key > bestKey || (key == bestKey && spreadHash(c, salt) > spreadHash(best, salt));
                if (better) best = c, bestKey = key;
            };
            if (current < cells) {
                const int cx = int(current % cellsX), cy = int(current / cellsX);
                for (int y = cy - 1; y <= cy + 1; ++y)
                    for (int x = cx - 1; x <= cx + 1; ++x)
                        if ((x != cx || y != cy) && x >= 0 && y >= 0 && x < int(cellsX) && y < int(cellsY)) rank(uint32_t(y) * cellsX + uint32_t(x));
                if (best != kNone) return best;
            }
            for (uint32_t c = 0; c < cells; ++c) rank(c);
            if (best != kNone) return best;
        }
        return kNone;
    }
};

extern "C" {

void x2_workgrid_options_defaults(x2_workgrid_options* o) {
    if (!o) return;
    *o = x2_workgrid_options{};
    o->cell_size = 64;
    o->samples_per_chunk = 4;
    o->progressive = 1;
    o->workers = 32;
}

int x2_workgrid_create(uint32_t width, uint32_t height, uint32_t spp, const x2_workgrid_options* options, uint32_t empty,
                       const int32_t* viewport, x2_workgrid** out) {
    if (!out) return X2_EINVAL;
    *out = nullptr;
    x2_workgrid_options o;
    x2_workgrid_options_defaults(&o);
    if (options) o = *options;
    if (!width || !height || !spp || !o.cell_size || o.cell_size % kTileSize || !o.samples_per_chunk) return X2_EINVAL;
    std::unique_ptr<x2_workgrid> g(new (std::nothrow) x2_workgrid);
    if (!g) return X2_ENOMEM;
    g->width = width;
    g->height = height;
    g->spp = spp;
    g->options = o;
    if (viewport) std::memcpy(g->view, viewport, sizeof g->view);
    g->tilesX = (width + kTileSize - 1) / kTileSize;
    g->tilesY = (height + kTileSize - 1) / kTileSize;
    g->tilesPerCell = o.cell_size / kTileSize;
    g->cellsX = (width + o.cell_size - 1) / o.cell_size;
    g->cellsY = (height + o.cell_size - 1) / o.cell_size;
    const uint32_t cells = g->cellCount();
    if (!empty) {
        // The share's sample indices, cut into ranges: 1, 1, 2, then the chunk size (progressive), or the chunk size.
        const uint32_t begin = o.sample_count ? o.sample_first : 0u;
        const uint32_t end = o.sample_count ? std::min<uint64_t>(spp, uint64_t(o.sample_first) + o.sample_count) : spp;
        for (uint32_t first = begin; first < end;) {
            const uint32_t into = first - begin;
            const uint32_t size = !o.progressive ? o.samples_per_chunk : into < 2 ? 1u : into < 4 ? 2u : o.samples_per_chunk;
            const uint32_t count = std::min(size, end - first);
            g->rangeFirst.push_back(first);
            g->rangeCount.push_back(count);
            first += count;
        }
    }
    g->tileOffset.assign(cells + 1, 0);
    for (uint32_t cy = 0; cy < g->cellsY; ++cy)
        for (uint32_t cx = 0; cx < g->cellsX; ++cx) {
            const uint32_t c = cy * g->cellsX + cx;
            const uint32_t ty1 = std::min(g->tilesY, (cy + 1) * g->tilesPerCell), tx1 = std::min(g->tilesX, (cx + 1) * g->tilesPerCell);
            for (uint32_t ty = cy * g->tilesPerCell; ty < ty1; ++ty)
                for (uint32_t tx = cx * g->tilesPerCell; tx < tx1; ++tx)
                    if (g->tileArea(ty * g->tilesX + tx)) g->tileList.push_back(ty * g->tilesX + tx);
            g->tileOffset[c + 1] = uint32_t(g->tileList.size());
        }
    g->published.reset(new std::atomic<uint32_t>[cells]);
    g->taken.reset(new std::atomic<uint32_t>[cells]);
    g->score.reset(new std::atomic<float>[cells]);
    g->important.reset(new std::atomic<uint8_t>[cells]);
    g->appended.resize(cells);
    uint64_t total = 0;
    for (uint32_t c = 0; c < cells; ++c) {
        const uint64_t u = uint64_t(g->rangeFirst.size()) * g->tiles(c);
        if (u > kNone / 2) return X2_EINVAL;
        g->published[c].store(uint32_t(u), std::memory_order_relaxed);
        g->taken[c].store(0, std::memory_order_relaxed);
        g->score[c].store(0.0f, std::memory_order_relaxed);
        g->important[c].store(0, std::memory_order_relaxed);
        total += u;
    }
    g->total.store(total, std::memory_order_relaxed);
    g->advanceFrontier();
    *out = g.release();
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

uint32_t x2_workgrid_cells(const x2_workgrid* g) { return g ? g->cellCount() : 0; }
uint64_t x2_workgrid_total(const x2_workgrid* g) { return g ? g->total.load(std::memory_order_acquire) : 0; }

uint32_t x2_workgrid_ranges(const x2_workgrid* g, uint32_t* ranges, uint32_t capacity) {
    if (!g) return 0;
    const uint32_t n = uint32_t(g->rangeFirst.size());
    for (uint32_t i = 0; ranges && i < std::min(n, capacity); ++i) {
        ranges[2 * i] = g->rangeFirst[i];
        ranges[2 * i + 1] = g->rangeCount[i];
    }
    return n;
}

int x2_workgrid_cell(const x2_workgrid* g, uint32_t c, uint32_t* tiles, uint32_t* published, uint32_t* taken) {
    if (!g || c >= g->cellCount()) return X2_EINVAL;
    if (tiles) *tiles = g->tiles(c);
    if (published) *published = g->published[c].load(std::memory_order_acquire);
    if (taken) *taken = g->taken[c].load(std::memory_order_acquire);
    return X2_OK;
}

int x2_workgrid_append(x2_workgrid* g, uint32_t c, const x2_chunk* chunks, uint32_t n) {
    if (!g || c >= g->cellCount() || (n && !chunks)) return X2_EINVAL;
    if (!g->appended[c]) g->appended[c].reset(new (std::nothrow) AppendedPages);
    if (!g->appended[c]) return X2_ENOMEM;
    const uint32_t at = g->published[c].load(std::memory_order_relaxed), u = g->uniformChunks(c);
    if (uint64_t(at - u) + n > uint64_t(kPageChunks) * kMaxPages) return X2_ENOMEM;
    for (uint32_t i = 0; i < n; ++i)
        if (!g->appended[c]->put(at - u + i, chunks[i])) return X2_ENOMEM;
    g->published[c].store(at + n, std::memory_order_release);
    g->total.fetch_add(n, std::memory_order_acq_rel);
    return X2_OK;
}

uint32_t x2_workgrid_claim(x2_workgrid* g, uint32_t c, uint32_t n, x2_chunk* out) {
    if (!g || c >= g->cellCount() || !out) return 0;
    return g->claim(c, n, out);
}

uint32_t x2_workgrid_claimable(const x2_workgrid* g, uint32_t c) { return g && c < g->cellCount() ? g->open(c) : 0; }

uint32_t x2_workgrid_remaining(const x2_workgrid* g, uint32_t c) {
    if (!g || c >= g->cellCount() || g->closed.load(std::memory_order_acquire)) return 0;
    return g->left(c);
}

uint32_t x2_workgrid_empty(const x2_workgrid* g) {
    if (!g) return 1;
    for (uint32_t c = 0; c < g->cellCount(); ++c)
        if (x2_workgrid_remaining(g, c)) return 0;
    return 1;
}

uint32_t x2_workgrid_frontier(const x2_workgrid* g) { return g ? g->frontierRange.load(std::memory_order_acquire) : 0; }

uint32_t x2_workgrid_choose(const x2_workgrid* g, uint32_t current, uint32_t salt) { return g ? g->choose(current, salt) : kNone; }

uint32_t x2_workgrid_seed(const x2_workgrid* g, uint32_t worker, uint32_t workers) {
    if (!g || !g->cellCount()) return kNone;
    // Every cell is the device's own: worker w of n starts at cell floor(w * cells / n).
    return uint32_t((uint64_t(worker) * g->cellCount()) / std::max(1u, workers));
}

int x2_workgrid_set_scores(x2_workgrid* g, const float* scores, uint32_t n) {
    if (!g || (n && !scores)) return X2_EINVAL;
    if (n != g->cellCount()) return X2_OK;  // scores of another grid: ignored
    // The cells above the mean of the known scores (those not below zero) are important.
    double sum = 0.0;
    uint32_t known = 0;
    for (uint32_t c = 0; c < n; ++c)
        if (scores[c] >= 0.0f) sum += scores[c], ++known;
    if (!known) return X2_OK;
    const float mean = float(sum / known);
    for (uint32_t c = 0; c < n; ++c) {
        g->score[c].store(std::max(scores[c], 0.0f), std::memory_order_relaxed);
        g->important[c].store(scores[c] > mean ? 1 : 0, std::memory_order_relaxed);
    }
    g->scored.store(true, std::memory_order_release);
    g->advanceFrontier();
    return X2_OK;
}

void x2_workgrid_close(x2_workgrid* g) {
    if (g) g->closed.store(true, std::memory_order_release);
}

// The broker's next launch: `want` split into equal shares for its workers; each takes its share from its cell and,
// where that cell has nothing more it may take now, moves by the cellular rules (at most 8 moves a worker).
uint32_t x2_workgrid_take(x2_workgrid* g, uint32_t want, x2_chunk* out) {
    if (!g || !out || !want) return 0;
    if (g->workerCell.empty()) {
        const uint32_t n = std::max(1u, g->options.workers);
        for (uint32_t w = 0; w < n; ++w) g->workerCell.push_back(x2_workgrid_seed(g, w, n));
    }
    const uint32_t workers = uint32_t(g->workerCell.size()), share = (want + workers - 1) / workers;
    uint32_t got = 0;
    for (uint32_t w = 0; w < workers && got < want; ++w) {
        uint32_t need = std::min(share, want - got);
        for (uint32_t move = 0; need && move < 8; ++move) {
            const uint32_t c = g->choose(g->workerCell[w], w);
            if (c == kNone) break;
            g->workerCell[w] = c;
            const uint32_t n = g->claim(c, need, out + got);
            got += n;
            need -= n;
        }
    }
    return got;
}

}  // extern "C"
