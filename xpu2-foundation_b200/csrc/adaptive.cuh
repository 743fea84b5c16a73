// Adaptive sampling's arithmetic (row f2 of the path's scope): each pixel's error from the film, the region trees
// that split the image where the error is, and each 8x8 tile's mask of pixels still to sample — the reference's
// adaptive frame (xpu2/interactive/async_integrator.h:3088-3125 pixelError; async_adaptive_core.h, async_adaptive.h:
// Tree, Regions, schedule), which follows MoonRay's adaptive region trees (after Dammertz et al., "A hierarchical
// automatic stopping condition for Monte Carlo global illumination"). Host and device share these functions so both
// make the same trees from the same errors; products and sums the compiler could fuse into one FMA are written with
// mulR / addR (the library is built with -fmad=false as well).
#pragma once
#include <cstdint>
#include <math.h>

#if defined(__CUDACC__)
#define X2_AD __host__ __device__ __forceinline__
#else
#define X2_AD inline
#endif

namespace x2 {
namespace ad {

X2_AD float mulR(float a, float b) {
#if defined(__CUDA_ARCH__)
    return __fmul_rn(a, b);
#else
    return a * b;
#endif
}
X2_AD float addR(float a, float b) {
#if defined(__CUDA_ARCH__)
    return __fadd_rn(a, b);
#else
    return a + b;
#endif
}

constexpr float kNotReady = -1.0f;  // a pixel without samples in both halves yet

// A pixel's error: the luma of the difference between its even- and odd-index half images over the square root of
// its luma, plus the alpha difference (MoonRay's estimatePixelErrorInternal).
X2_AD float pixelError(const double* total, const double* odd, uint32_t samples) {
    const float n = float(samples), nOdd = float(samples / 2), nEven = n - nOdd;
    if (nOdd <= 0 || nEven <= 0) return kNotReady;
    float d[4], m[3];
    for (int c = 0; c < 4; ++c) {
        const float t = float(total[c]), o = float(odd[c]);
        if (t != t || o != o) return 0.0f;
        d[c] = fabsf(addR(mulR(t, nOdd), -mulR(o, n)) / mulR(nOdd, nEven));
        if (c < 3) m[c] = t / n;
    }
    const float dl = addR(addR(mulR(0.299f, d[0]), mulR(0.587f, d[1])), mulR(0.114f, d[2]));
    const float ml = addR(addR(mulR(0.299f, m[0]), mulR(0.587f, m[1])), mulR(0.114f, m[2]));
    if (ml <= 0) return d[3];
    return addR(dl / sqrtf(ml), d[3]);
}

struct IBox {
    int x0, y0, x1, y1;
};
struct FBox {
    float x0, y0, x1, y1;
};
// A tree node: its bounds, its first child (-1: a leaf; the second follows it), and whether it has converged.
struct Node {
    FBox b;
    int children;
    int complete;
};

constexpr float kMinNode = 1.27201964951407f;  // sqrt of the golden ratio: the smallest node side
constexpr float kMaxNode = 16.0f;              // a node longer than this never converges whole
constexpr float kSplitFactor = 256.0f;         // a node splits while its error is under this many targets
constexpr float kNoSplit = -1.0f;

X2_AD int imin(int a, int b) { return b < a ? b : a; }
X2_AD int imax(int a, int b) { return a < b ? b : a; }
X2_AD float fmin2(float a, float b) { return b < a ? b : a; }
X2_AD float fmax2(float a, float b) { return a < b ? b : a; }
X2_AD IBox outward(const FBox& b) { return {int(floorf(b.x0)), int(floorf(b.y0)), int(ceilf(b.x1)), int(ceilf(b.y1))}; }

// The most nodes a region's tree can have.
X2_AD int nodeBound(const IBox& b) {
    const int w = b.x1 - b.x0, h = b.y1 - b.y0;
    if (w <= 0 || h <= 0) return 0;
    return 2 * int(ceilf(mulR(float(w) / kMinNode, float(h) / kMinNode))) - 1;
}
// A node's error: its summed pixel error over the square root of its area times a fixed image area (so regions of
// any image are weighed alike).
X2_AD float nodeError(float error, float area) {
    constexpr float imageArea = ((815.0f - 0.0f) * (1943.0f - -24.0f)) / 4.0f;
    return error / sqrtf(mulR(area, imageArea));
}
X2_AD float splitAt(float location, float length) {
    if (mulR(length, location) >= kMinNode) return location;
    if (length >= kMinNode * 2) return kMinNode / length;
    return kNoSplit;
}
X2_AD float splitLocation(float location, float length) {
    if (location <= 0.5f) return splitAt(location, length);
    const float h = splitAt(1.0f - location, length);
    return h == kNoSplit ? kNoSplit : 1.0f - h;
}

// A region's summed-area table of pixel errors ((w + 1) x (h + 1) doubles, first row and column zero), corner x0, y0.
struct Sat {
    const double* s;
    int x0, y0, w1;
    X2_AD double at(int x, int y) const { return s[size_t(y - y0) * size_t(w1) + size_t(x - x0)]; }
    X2_AD double rect(int ax, int ay, int bx, int by) const { return at(bx, by) - at(ax, by) - at(bx, ay) + at(ax, ay); }
};
// Running sums of a node's error along its split axis: entry i covers its first i + 1 columns (rows if vertical).
struct Runs {
    const Sat& sat;
    IBox ib;
    bool horizontal;
    int n;
    X2_AD float operator()(int i) const {
        return horizontal ? float(sat.rect(ib.x0, ib.y0, ib.x0 + i + 1, ib.y1)) : float(sat.rect(ib.x0, ib.y0, ib.x1, ib.y0 + i + 1));
    }
    X2_AD float total() const { return n > 0 ? (*this)(n - 1) : 0.f; }
};
// Where along a node its error is halved: the first run above half (bisection), interpolated within its step.
X2_AD float halfway(const Runs& r) {
    const float total = r.total(), half = mulR(total, 0.5f);
    int i = r.n / 2;
    if (total != 0.f) {
        int lo = 0, hi = r.n;
        while (lo < hi) {
            const int mid = (lo + hi) / 2;
            if (r(mid) > half) hi = mid;
            else lo = mid + 1;
        }
        i = lo;
    }
    i = imin(imax(i, 1), r.n - 1);
    const float below = r(i - 1), above = r(i), step = above - below;
    const float frac = step > 0 ? (half - below) / step : 0.5f;
    return addR(float(i), frac) / float(r.n);
}

enum : int { kUnconverged = 0, kConverged = 1, kSplit = 2 };

// What becomes of node bounds b of the tree rooted at root: it converged, it splits at the halfway point of its error
// along its longer side into left and right, or it stays an unconverged leaf.
X2_AD int decide(const Sat& sat, const IBox& root, const FBox& b, float target, FBox& left, FBox& right) {
    const float w = b.x1 - b.x0, h = b.y1 - b.y0;
    const bool horizontal = w > h;
    const float length = horizontal ? w : h;
    IBox ib = outward(b);
    ib = {imax(ib.x0, root.x0), imax(ib.y0, root.y0), imin(ib.x1, root.x1), imin(ib.y1, root.y1)};
    const Runs runs{sat, ib, horizontal, horizontal ? ib.x1 - ib.x0 : ib.y1 - ib.y0};
    const float error = nodeError(runs.total(), mulR(w, h));
    if (error < target && length < kMaxNode) return kConverged;
    if (error < mulR(target, kSplitFactor) && length > kMinNode * 2) {
        const float at = splitLocation(halfway(runs), length);
        if (at == kNoSplit) return kUnconverged;
        left = right = b;
        if (horizontal) left.x1 = right.x0 = addR(b.x0, mulR(at, w));
        else left.y1 = right.y0 = addR(b.y0, mulR(at, h));
        return kSplit;
    }
    return kUnconverged;
}

// Every pixel within the rows and columns the active ones span.
X2_AD uint64_t fillRect(uint64_t m) {
    if (!m) return 0;
    int r0 = 8, r1 = -1, c0 = 8, c1 = -1;
    for (int b = 0; b < 64; ++b)
        if (m >> b & 1) {
            r0 = imin(r0, b / 8);
            r1 = imax(r1, b / 8);
            c0 = imin(c0, b % 8);
            c1 = imax(c1, b % 8);
        }
    uint64_t out = 0;
    for (int y = r0; y <= r1; ++y)
        for (int x = c0; x <= c1; ++x) out |= uint64_t(1) << (y * 8 + x);
    return out;
}

// The pixels of the 8x8 tile at (tx, ty) the tree still samples (bit y * 8 + x), filled to their bounding rectangle;
// a tree deeper than the walk's stack samples the whole tile.
X2_AD uint64_t tileSamples(const Node* nodes, int tx, int ty) {
    const FBox tile{float(tx), float(ty), float(tx + 8), float(ty + 8)};
    constexpr int kDepth = 128;
    int stack[kDepth], top = 0;
    stack[top++] = 0;
    uint64_t mask = 0;
    while (top) {
        const Node n = nodes[stack[--top]];
        if (n.complete) continue;
        const FBox i{fmax2(n.b.x0, tile.x0), fmax2(n.b.y0, tile.y0), fmin2(n.b.x1, tile.x1), fmin2(n.b.y1, tile.y1)};
        if (i.x1 <= i.x0 || i.y1 <= i.y0) continue;
        if (n.children >= 0) {
            if (top + 2 > kDepth) return ~uint64_t(0);
            stack[top++] = n.children;
            stack[top++] = n.children + 1;
            continue;
        }
        const IBox r = outward(i);
        for (int y = imax(r.y0, ty); y < imin(r.y1, ty + 8); ++y)
            for (int x = imax(r.x0, tx); x < imin(r.x1, tx + 8); ++x) mask |= uint64_t(1) << ((y - ty) * 8 + (x - tx));
    }
    return fillRect(mask);
}

// The overlapping regions' layout: up to 4 x 4 regions of whole 8-pixel tiles, each widened by 8 pixels; a tile reads
// the tree of the region its corner lies in.
struct Layout {
    int perDim = 1, regionW = 0, regionH = 0;
    X2_AD int regionOf(int tx, int ty) const { return imin(ty / regionH, perDim - 1) * perDim + imin(tx / regionW, perDim - 1); }
};

}  // namespace ad
}  // namespace x2
