// Adaptive sampling's arithmetic, shared by the host and the device so both reach the same decisions from the same
// errors (row f2 of the path's scope).
//
// The rules are those of the reference's adaptive frame (xpu2/interactive/async_integrator.h:3088-3125 pixelError;
// async_adaptive_core.h; async_adaptive.h Regions and Cellular), which follow MoonRay's adaptive region trees:
//   Portions of this file restate arithmetic of MoonRay (rndr/adaptive/AdaptiveRegionTree, ActivePixelMask and the
//   pixel error estimate), Copyright 2023-2024 DreamWorks Animation LLC, licensed under the Apache License, Version
//   2.0 (http://www.apache.org/licenses/LICENSE-2.0): the pixel error, the node error with its fixed image area, the
//   split position rule and its constants, the error-halving split point and the filled tile mask.
// A tile mask computed here must equal the reference's bit for bit, so every value is rounded where the reference
// rounds it: products and sums that a compiler could fuse are made with mulR/addR, and the library is built without
// contraction as well.
#pragma once
#include <math.h>

#include <cstdint>

#if defined(__CUDACC__)
#define X2_RG __host__ __device__ __forceinline__
#else
#define X2_RG inline
#endif

namespace x2 {
namespace rg {

X2_RG float mulR(float a, float b) {
#if defined(__CUDA_ARCH__)
    return __fmul_rn(a, b);
#else
    return a * b;
#endif
}
X2_RG float addR(float a, float b) {
#if defined(__CUDA_ARCH__)
    return __fadd_rn(a, b);
#else
    return a + b;
#endif
}

// Constants of the tree rules.
constexpr float kMinSide = 1.27201964951407f;  // the smallest node side: the square root of the golden ratio
constexpr float kMaxSide = 16.0f;              // a converged node is shorter than this
constexpr float kSplitFactor = 256.0f;         // a node splits only below this many times the target
constexpr float kImageArea = ((815.0f - 0.0f) * (1943.0f - -24.0f)) / 4.0f;  // the image area every node is judged by
constexpr float kNotReady = -1.0f;             // a pixel's error before both its half images have a sample

// The luma of an rgb triple, in the rounding order the error estimate uses.
X2_RG float luma3(float r, float g, float b) { return addR(addR(mulR(0.299f, r), mulR(0.587f, g)), mulR(0.114f, b)); }

// A pixel's error from its FP64 film: sums (rgba), odd-index sums and its sample count. The two half images (odd and
// even sample indices) differ by |t n_odd - o n| / (n_odd n_even) a channel; the error is that difference's luma over
// the square root of the pixel's mean luma, plus alpha's difference; kNotReady until both halves have a sample.
X2_RG float pixelError(const double* sum, const double* odd, uint32_t count) {
    const float n = float(count);
    const float nOdd = float(count / 2);
    const float nEven = n - nOdd;
    if (!(nOdd > 0) || !(nEven > 0)) return kNotReady;
    const float halves = mulR(nOdd, nEven);
    float diff[4], mean[3];
    for (int k = 0; k < 4; ++k) {
        const float t = float(sum[k]), o = float(odd[k]);
        if (t != t || o != o) return 0.0f;  // a NaN in the film
        diff[k] = fabsf(addR(mulR(t, nOdd), -mulR(o, n)) / halves);
        if (k < 3) mean[k] = t / n;
    }
    const float meanLuma = luma3(mean[0], mean[1], mean[2]);
    if (meanLuma <= 0) return diff[3];
    return addR(luma3(diff[0], diff[1], diff[2]) / sqrtf(meanLuma), diff[3]);
}

// A node's error: its summed pixel error over the root of its area times the fixed image area.
X2_RG float nodeError(float summed, float area) { return summed / sqrtf(mulR(area, kImageArea)); }

// The most nodes a region of w x h pixels can grow: twice the number of smallest squares it holds, less one.
X2_RG int regionNodeBound(int w, int h) {
    if (w <= 0 || h <= 0) return 0;
    return 2 * int(ceilf(mulR(float(w) / kMinSide, float(h) / kMinSide))) - 1;
}

// Where a node of side `side` splits, as a fraction of its side, given the fraction `at` that halves its error: at
// least kMinSide from either end, or no split (a negative value) when the node is too short for that.
X2_RG float splitFraction(float at, float side) {
    const bool fromFar = !(at <= 0.5f);
    const float near = fromFar ? 1.0f - at : at;
    float f;
    if (mulR(side, near) >= kMinSide) f = near;
    else if (side >= kMinSide * 2) f = kMinSide / side;
    else return -1.0f;
    return fromFar ? 1.0f - f : f;
}

// A region's summed-area table of pixel errors: (w + 1) x (h + 1) doubles, row 0 and column 0 zero, for the region
// whose corner is (x0, y0). box() sums the pixels of [ax, bx) x [ay, by) in image coordinates.
struct SummedErrors {
    const double* table;
    int x0, y0, stride;
    X2_RG double at(int x, int y) const { return table[size_t(y - y0) * size_t(stride) + size_t(x - x0)]; }
    X2_RG double box(int ax, int ay, int bx, int by) const { return at(bx, by) - at(ax, by) - at(bx, ay) + at(ax, ay); }
};

// A node under decision, its pixel span clipped to the region, along its longer side.
struct Span {
    int ax, ay, bx, by;  // pixels [ax, bx) x [ay, by)
    bool alongX;         // the longer side is x
    int cells;           // pixel columns (alongX) or rows across the span
    // The error of the span's first k + 1 columns (rows), in float, as the marginals are kept.
    X2_RG float upTo(const SummedErrors& s, int k) const {
        return alongX ? float(s.box(ax, ay, ax + k + 1, by)) : float(s.box(ax, ay, bx, ay + k + 1));
    }
};

// The fraction of a span that halves its error: the first column whose running error passes half the total (by
// bisection over the running errors, which never decrease), then linear between it and the one before.
X2_RG float halvingFraction(const SummedErrors& s, const Span& sp) {
    const int n = sp.cells;
    const float total = n > 0 ? sp.upTo(s, n - 1) : 0.0f;
    const float half = mulR(total, 0.5f);
    int k = n / 2;
    if (total != 0.0f) {
        int lo = 0, hi = n;  // the first k in [lo, hi) with upTo(k) > half
        while (lo < hi) {
            const int mid = (lo + hi) / 2;
            if (sp.upTo(s, mid) > half) hi = mid;
            else lo = mid + 1;
        }
        k = lo;
    }
    k = k < 1 ? 1 : k;
    k = k > n - 1 ? n - 1 : k;
    const float below = sp.upTo(s, k - 1), above = sp.upTo(s, k);
    const float step = above - below;
    return addR(float(k), step > 0 ? (half - below) / step : 0.5f) / float(n);
}

enum Fate : uint8_t { kOpen = 0, kConverged = 1, kSplit = 2 };

// The fate of a node [x0, x1) x [y0, y1) of a region [rx0, rx1) x [ry0, ry1): converged (its error below the target
// and shorter than kMaxSide), split at the point halving its error along its longer side (its error below
// kSplitFactor times the target and long enough; the cut in *cut, along x when *alongX), or left open.
X2_RG Fate nodeFate(const SummedErrors& s, int rx0, int ry0, int rx1, int ry1, float x0, float y0, float x1, float y1, float target,
                    float* cut, bool* alongX) {
    const float w = x1 - x0, h = y1 - y0;
    Span sp;
    sp.alongX = w > h;
    const float side = sp.alongX ? w : h;
    const int fx0 = int(floorf(x0)), fy0 = int(floorf(y0)), cx1 = int(ceilf(x1)), cy1 = int(ceilf(y1));
    sp.ax = fx0 > rx0 ? fx0 : rx0;
    sp.ay = fy0 > ry0 ? fy0 : ry0;
    sp.bx = cx1 < rx1 ? cx1 : rx1;
    sp.by = cy1 < ry1 ? cy1 : ry1;
    sp.cells = sp.alongX ? sp.bx - sp.ax : sp.by - sp.ay;
    const float summed = sp.cells > 0 ? sp.upTo(s, sp.cells - 1) : 0.0f;
    const float err = nodeError(summed, mulR(w, h));
    if (err < target && side < kMaxSide) return kConverged;
    if (!(err < mulR(target, kSplitFactor)) || !(side > kMinSide * 2)) return kOpen;
    const float f = splitFraction(halvingFraction(s, sp), side);
    if (f == -1.0f) return kOpen;
    *alongX = sp.alongX;
    *cut = sp.alongX ? addR(x0, mulR(f, w)) : addR(y0, mulR(f, h));
    return kSplit;
}

// A 64-bit tile mask (bit y * 8 + x) filled to the rectangle its set bits span.
X2_RG uint64_t fillToBounds(uint64_t m) {
    if (!m) return 0;
    uint32_t rows = 0, cols = 0;
    for (int y = 0; y < 8; ++y) {
        const uint32_t row = uint32_t(m >> (8 * y)) & 0xffu;
        cols |= row;
        if (row) rows |= 1u << y;
    }
    auto low = [](uint32_t v) { int i = 0; while (!(v >> i & 1u)) ++i; return i; };
    auto high = [](uint32_t v) { int i = 7; while (!(v >> i & 1u)) --i; return i; };
    const int c0 = low(cols), c1 = high(cols), r0 = low(rows), r1 = high(rows);
    const uint64_t rowBits = ((0xffull << c0) & (0xffull >> (7 - c1))) & 0xffull;
    uint64_t out = 0;
    for (int y = r0; y <= r1; ++y) out |= rowBits << (8 * y);
    return out;
}

// The overlapping regions' layout: up to 4 x 4 regions of whole 8-pixel tiles, each widened by an 8-pixel overlap and
// clamped to the image. A tile reads the tree of the region its top-left pixel lies in.
struct RegionGrid {
    int across = 1, regionW = 0, regionH = 0;
    X2_RG int regionOfTile(int px, int py) const {
        const int rx = px / regionW, ry = py / regionH;
        return (ry < across - 1 ? ry : across - 1) * across + (rx < across - 1 ? rx : across - 1);
    }
};
inline RegionGrid regionGrid(int width, int height) {
    constexpr int kTile = 8, kOverlap = 8, kMostAcross = 4, kLeast = kTile + kOverlap;
    RegionGrid g;
    if (kLeast >= width || kLeast >= height) {
        g.regionW = width;
        g.regionH = height;
        return g;
    }
    const int fit = width / kLeast < height / kLeast ? width / kLeast : height / kLeast;
    g.across = fit < kMostAcross ? (fit > 1 ? fit : 1) : kMostAcross;
    auto tiles = [](int n) { return (n + kTile - 1) / kTile * kTile; };
    g.regionW = tiles(1 + (width - 1) / g.across);
    g.regionH = tiles(1 + (height - 1) / g.across);
    return g;
}
// Region i's pixel box [x0, x1) x [y0, y1).
inline void regionBox(const RegionGrid& g, int i, int width, int height, int box[4]) {
    constexpr int kOverlap = 8;
    const int rx = i % g.across, ry = i / g.across;
    const int x0 = rx * g.regionW - kOverlap, y0 = ry * g.regionH - kOverlap;
    const int x1 = (rx + 1) * g.regionW + kOverlap, y1 = (ry + 1) * g.regionH + kOverlap;
    box[0] = x0 > 0 ? x0 : 0;
    box[1] = y0 > 0 ? y0 : 0;
    box[2] = x1 < width ? x1 : width;
    box[3] = y1 < height ? y1 : height;
}

}  // namespace rg
}  // namespace x2
