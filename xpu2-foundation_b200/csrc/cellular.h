// Cellular generations on the host, for frames by sampling generations under a sample budget (row f2): the
// reference makes these generations on the host between passes (xpu2/interactive/async_adaptive.h:147-232 Cellular,
// async_render.h:1318-1410 the budget's samples left and the pass's tiles), and a budget's target needs every tile's
// state at once. The generation rule is the device's (adaptive.cu adCellular); the budget's target is the error the
// samples still to spend would bring every tile to, found by halving the interval in log space.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <numeric>
#include <vector>

#include "adaptive.cuh"

namespace x2 {

// A budget for the next generation: each pixel's planned samples, the samples still to spend, the most a pixel may
// have, and the error no tile need go below (0: none).
struct SampleBudget {
    const std::vector<uint32_t>* planned;
    double remaining;
    uint32_t most;
    float floor;
};

class CellularGenerations {
   public:
    static constexpr float kSurvive = 0.5f, kBirth = 0.75f;
    static constexpr int kSurviveNeighbours = 3, kBirthNeighbours = 5;

    CellularGenerations(int width, int height, float target, const std::vector<uint64_t>& inImage)
        : width_(width), height_(height), tilesX_((width + 7) / 8), tilesY_((height + 7) / 8), target_(target) {
        const size_t n = size_t(tilesX_) * tilesY_;
        alive_.assign(n, 1);
        next_.assign(n, 0);
        dead_.assign(n, 0);
        ratio_.assign(n, 0.0f);
        error_.assign(n, 0.0f);
        pixels_.assign(n, 0.0);
        most_.assign(n, 0.0);
        for (size_t t = 0; t < n && t < inImage.size(); ++t)
            if (!inImage[t]) dead_[t] = 1, alive_[t] = 0;
    }

    // The next generation from per-pixel errors (width a row); its live tiles' count.
    size_t update(const float* errors, const SampleBudget* budget) {
        for (int ty = 0; ty < tilesY_; ++ty)
            for (int tx = 0; tx < tilesX_; ++tx) {
                const size_t t = size_t(ty) * tilesX_ + tx;
                double sum = 0, most = 0, rendered = 0;
                int n = 0;
                bool unknown = false;
                for (int y = ty * 8; y < std::min(height_, ty * 8 + 8); ++y)
                    for (int x = tx * 8; x < std::min(width_, tx * 8 + 8); ++x) {
                        const size_t i = size_t(y) * size_t(width_) + size_t(x);
                        const float e = errors[i];
                        if (e < 0) unknown = true;
                        else sum += e;
                        ++n;
                        if (budget) {
                            const double s = (*budget->planned)[i];
                            most = std::max(most, s);
                            rendered += s > 0 ? 1 : 0;
                        }
                    }
                error_[t] = unknown ? -1.0f : ad::nodeError(float(sum), float(n));
                pixels_[t] = rendered;
                most_[t] = most;
            }
        const float target = budget ? std::max(budgetTarget(*budget), budget->floor) : target_;
        for (size_t t = 0; t < ratio_.size(); ++t) ratio_[t] = error_[t] < 0 ? 3.4e38f : error_[t] / target;
        size_t live = 0;
        for (int ty = 0; ty < tilesY_; ++ty)
            for (int tx = 0; tx < tilesX_; ++tx) {
                const size_t t = size_t(ty) * tilesX_ + tx;
                int k = 0;
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dx = -1; dx <= 1; ++dx) {
                        const int x = tx + dx, y = ty + dy;
                        if ((dx || dy) && x >= 0 && y >= 0 && x < tilesX_ && y < tilesY_ && alive_[size_t(y) * tilesX_ + x]) ++k;
                    }
                const float r = ratio_[t];
                bool next = alive_[t] ? (r >= 1.0f || (r >= kSurvive && k >= kSurviveNeighbours)) : (r >= 1.0f || (r >= kBirth && k >= kBirthNeighbours));
                if (dead_[t]) next = false;
                next_[t] = next ? 1 : 0;
                live += next ? 1 : 0;
            }
        alive_.swap(next_);
        return live;
    }
    bool alive(size_t tile) const { return alive_[tile] != 0; }
    float ratio(size_t tile) const { return ratio_[tile]; }

   private:
    // The error the samples still to spend would bring every tile to: the target whose cost — each tile's rendered
    // pixels times the samples that take its error down to it, n (error / target)^2 less the n it has, both capped at
    // the most a pixel may have — is the samples left. The cost falls as the target rises: 48 halvings in log space
    // between a thousandth of the least tile error and the largest.
    float budgetTarget(const SampleBudget& b) {
        double lo = 3.4e38, hi = 0;
        for (size_t t = 0; t < error_.size(); ++t)
            if (!dead_[t] && error_[t] > 0 && most_[t] > 0) lo = std::min(lo, double(error_[t])), hi = std::max(hi, double(error_[t]));
        if (b.remaining <= 0 || hi <= 0) return 3.4e38f;
        auto cost = [&](double target) {
            double c = 0;
            for (size_t t = 0; t < error_.size(); ++t) {
                if (dead_[t] || error_[t] <= 0 || most_[t] <= 0) continue;
                const double n = most_[t], r = double(error_[t]) / target;
                c += pixels_[t] * (std::min(std::max(n * r * r, n), double(b.most)) - std::min(n, double(b.most)));
            }
            return c;
        };
        double low = lo * 1e-3, high = hi;
        if (cost(low) <= b.remaining) return float(low);
        for (int i = 0; i < 48; ++i) {
            const double middle = std::sqrt(low * high);
            (cost(middle) > b.remaining ? low : high) = middle;
        }
        return float(high);
    }

    int width_, height_, tilesX_, tilesY_;
    float target_;
    std::vector<char> alive_, next_, dead_;
    std::vector<float> ratio_, error_;
    std::vector<double> pixels_, most_;
};

// A budget pass's tiles when its live tiles want more samples than are left: the live tiles furthest above the target
// first (ties by tile order), as long as each fits in what is left; the rest dropped (1).
inline std::vector<char> dropForBudget(const CellularGenerations& cells, const std::vector<uint64_t>& inImage, uint32_t size, double left) {
    std::vector<uint32_t> live;
    double wanted = 0;
    for (uint32_t t = 0; t < inImage.size(); ++t)
        if (inImage[t] && cells.alive(t)) {
            live.push_back(t);
            wanted += double(__builtin_popcountll(inImage[t])) * size;
        }
    if (wanted <= left) return {};
    std::stable_sort(live.begin(), live.end(), [&](uint32_t a, uint32_t b) { return cells.ratio(a) > cells.ratio(b); });
    std::vector<char> dropped(inImage.size(), 1);
    double taken = 0;
    for (uint32_t t : live) {
        const double cost = double(__builtin_popcountll(inImage[t])) * size;
        if (taken + cost > left) break;
        taken += cost;
        dropped[t] = 0;
    }
    return dropped;
}

}  // namespace x2
