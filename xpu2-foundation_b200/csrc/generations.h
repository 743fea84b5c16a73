// Cellular generations under a sample budget, made on the host between passes (x2_render_adaptive_budget).
//
// The rules are the reference's (xpu2/interactive/async_adaptive.h Cellular with a Budget; async_render.h's adaptive
// frame with budgetBySamples): each 8x8 tile is a cell whose ratio is its node error over the generation's target;
// a live tile survives at a ratio of 1, or of 0.5 with 3 live neighbours of its eight, a dead one is born at 1, or at
// 0.75 with 5; tiles outside the image never live. Under a budget the target is the error that the samples still to
// spend would bring every tile to: the root of cost(target) = remaining, where a tile of p rendered pixels of n
// samples costs p (min(max(n (e / target)^2, n), most) - min(n, most)), found by halving the interval in log space
// 48 times, no lower than the floor. A pass whose live tiles want more than what is left takes the tiles furthest
// above the target first (ties by tile order) while each fits.
//
// Here the image's statistics are gathered in one sweep over its pixel rows into per-tile accumulators (a tile's
// pixels still added in row-major order, as the reference adds them), and the budget's cost is evaluated over a
// compact list of the tiles that take part in it.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "regions.cuh"

namespace x2 {

class TileGenerations {
   public:
    TileGenerations(uint32_t width, uint32_t height, float floor, const std::vector<uint64_t>& inImage)
        : width_(width), height_(height), tilesX_((width + 7) / 8), tilesY_((height + 7) / 8), floor_(floor), inImage_(inImage) {
        const size_t n = size_t(tilesX_) * tilesY_;
        alive_.resize(n);
        for (size_t t = 0; t < n; ++t) alive_[t] = inImage_[t] ? 1 : 0;
        ratio_.assign(n, 0.0f);
    }

    bool alive(uint32_t t) const { return alive_[t] != 0; }
    float ratio(uint32_t t) const { return ratio_[t]; }

    // The next generation from the pixels' errors and their planned samples, `remaining` samples of the budget still
    // to spend and `most` samples a pixel at most. Returns its live tiles.
    uint32_t advance(const float* errors, const std::vector<uint32_t>& samples, double remaining, uint32_t most) {
        const size_t n = alive_.size();
        std::vector<double> sum(n, 0.0), rendered(n, 0.0), deepest(n, 0.0);
        std::vector<uint32_t> pixels(n, 0);
        std::vector<uint8_t> unknown(n, 0);
        for (uint32_t y = 0; y < height_; ++y)
            for (uint32_t x = 0; x < width_; ++x) {
                const size_t t = size_t(y / 8) * tilesX_ + x / 8, i = size_t(y) * width_ + x;
                const float e = errors[i];
                if (e < 0.0f) unknown[t] = 1;
                else sum[t] += e;
                ++pixels[t];
                const double s = samples[i];
                deepest[t] = std::max(deepest[t], s);
                rendered[t] += s > 0 ? 1.0 : 0.0;
            }
        std::vector<float> error(n);
        for (size_t t = 0; t < n; ++t) error[t] = unknown[t] ? -1.0f : rg::nodeError(float(sum[t]), float(pixels[t]));
        const float target = std::max(budgetTarget(error, rendered, deepest, remaining, most), floor_);
        for (size_t t = 0; t < n; ++t) ratio_[t] = error[t] < 0.0f ? 3.4e38f : error[t] / target;
        std::vector<uint8_t> next(n, 0);
        uint32_t live = 0;
        for (int ty = 0; ty < int(tilesY_); ++ty)
            for (int tx = 0; tx < int(tilesX_); ++tx) {
                const size_t t = size_t(ty) * tilesX_ + tx;
                int around = 0;
                for (int y = std::max(ty - 1, 0); y <= std::min(ty + 1, int(tilesY_) - 1); ++y)
                    for (int x = std::max(tx - 1, 0); x <= std::min(tx + 1, int(tilesX_) - 1); ++x)
                        around += (x != tx || y != ty) && alive_[size_t(y) * tilesX_ + x] ? 1 : 0;
                const float q = ratio_[t];
                const bool lives = inImage_[t] && (q >= 1.0f || (alive_[t] ? q >= 0.5f && around >= 3 : q >= 0.75f && around >= 5));
                next[t] = lives ? 1 : 0;
                live += lives ? 1u : 0u;
            }
        alive_.swap(next);
        return live;
    }

    // A pass of `size` samples a pixel under `left` samples of budget: the live tiles it takes (all of them when they
    // fit, else those furthest above the target while each fits).
    std::vector<uint8_t> chosen(uint32_t size, double left) const {
        std::vector<uint32_t> live;
        double wanted = 0.0;
        for (uint32_t t = 0; t < alive_.size(); ++t)
            if (inImage_[t] && alive_[t]) {
                live.push_back(t);
                wanted += double(__builtin_popcountll(inImage_[t])) * size;
            }
        std::vector<uint8_t> take(alive_.size(), 0);
        if (wanted <= left) {
            for (uint32_t t : live) take[t] = 1;
            return take;
        }
        std::stable_sort(live.begin(), live.end(), [&](uint32_t a, uint32_t b) { return ratio_[a] > ratio_[b]; });
        double used = 0.0;
        for (uint32_t t : live) {
            const double cost = double(__builtin_popcountll(inImage_[t])) * size;
            if (used + cost > left) break;
            used += cost;
            take[t] = 1;
        }
        return take;
    }

   private:
    // The target whose cost is the samples left (a huge target when nothing is left to spend or refine).
    float budgetTarget(const std::vector<float>& error, const std::vector<double>& rendered, const std::vector<double>& deepest, double remaining,
                       uint32_t most) const {
        std::vector<double> e, p, n;  // the tiles that take part: in the image, refinable, sampled
        double least = 3.4e38, largest = 0.0;
        for (size_t t = 0; t < error.size(); ++t)
            if (inImage_[t] && error[t] > 0.0f && deepest[t] > 0.0) {
                e.push_back(error[t]);
                p.push_back(rendered[t]);
                n.push_back(deepest[t]);
                least = std::min(least, double(error[t]));
                largest = std::max(largest, double(error[t]));
            }
        if (remaining <= 0.0 || largest <= 0.0) return 3.4e38f;
        const double cap = double(most);
        auto cost = [&](double target) {
            double c = 0.0;
            for (size_t k = 0; k < e.size(); ++k) {
                const double q = e[k] / target;
                c += p[k] * (std::min(std::max(n[k] * q * q, n[k]), cap) - std::min(n[k], cap));
            }
            return c;
        };
        double below = least * 1e-3, above = largest;  // cost(above) is 0
        if (cost(below) <= remaining) return float(below);
        for (int i = 0; i < 48; ++i) {
            const double mid = std::sqrt(below * above);
            if (cost(mid) > remaining) below = mid;
            else above = mid;
        }
        return float(above);
    }

    uint32_t width_, height_, tilesX_, tilesY_;
    float floor_;
    std::vector<uint64_t> inImage_;
    std::vector<uint8_t> alive_;
    std::vector<float> ratio_;
};

}  // namespace x2
