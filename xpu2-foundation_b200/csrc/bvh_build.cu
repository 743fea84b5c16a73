// On-device BVH build: Morton codes -> radix sort -> LBVH hierarchy (Karras 2012, "Maximizing Parallelism in the
// Construction of BVHs, Octrees, and k-d Trees") -> bottom-up bounds -> collapse to compressed 8-wide nodes
// (Ylitie et al. 2017), one level of wide nodes a launch. Build time is reported apart from render time.
#include "bvh.cuh"
#include "engine.h"

#include <cub/device/device_radix_sort.cuh>
#include <cuda_runtime.h>

#include <cfloat>
#include <cstdio>
#include <vector>

namespace x2 {

namespace {

constexpr int kBlock = 256;

struct Aabb {
    float lo[3], hi[3];
};

__device__ __forceinline__ unsigned floatToOrdered(float f) {
    const unsigned u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float orderedToFloat(unsigned u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

__global__ void triBounds(const float* __restrict__ v, const uint32_t* __restrict__ t, uint32_t n, Aabb* __restrict__ leaf,
                          unsigned* __restrict__ sceneBox) {
    __shared__ unsigned box[6];
    if (threadIdx.x < 6) box[threadIdx.x] = threadIdx.x < 3 ? 0xffffffffu : 0u;
    __syncthreads();
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        Aabb b;
        for (int k = 0; k < 3; ++k) {
            const float a = v[3 * t[3 * i] + k], c = v[3 * t[3 * i + 1] + k], d = v[3 * t[3 * i + 2] + k];
            b.lo[k] = fminf(a, fminf(c, d));
            b.hi[k] = fmaxf(a, fmaxf(c, d));
            const float centre = 0.5f * (b.lo[k] + b.hi[k]);
            atomicMin(&box[k], floatToOrdered(centre));
            atomicMax(&box[3 + k], floatToOrdered(centre));
        }
        leaf[i] = b;
    }
    __syncthreads();
    if (threadIdx.x < 3) atomicMin(&sceneBox[threadIdx.x], box[threadIdx.x]);
    else if (threadIdx.x < 6) atomicMax(&sceneBox[threadIdx.x], box[threadIdx.x]);
}

__device__ __forceinline__ uint64_t spread21(uint64_t x) {
    x &= 0x1fffffull;
    x = (x | x << 32) & 0x1f00000000ffffull;
    x = (x | x << 16) & 0x1f0000ff0000ffull;
    x = (x | x << 8) & 0x100f00f00f00f00full;
    x = (x | x << 4) & 0x10c30c30c30c30c3ull;
    x = (x | x << 2) & 0x1249249249249249ull;
    return x;
}

__global__ void mortonCodes(const Aabb* __restrict__ leaf, uint32_t n, const unsigned* __restrict__ sceneBox, uint64_t* __restrict__ keys,
                            uint32_t* __restrict__ values) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint64_t code = 0;
    for (int k = 0; k < 3; ++k) {
        const float lo = orderedToFloat(sceneBox[k]), hi = orderedToFloat(sceneBox[3 + k]);
        const float centre = 0.5f * (leaf[i].lo[k] + leaf[i].hi[k]);
        const float extent = hi - lo;
        float u = extent > 0.0f ? (centre - lo) / extent : 0.5f;
        u = fminf(fmaxf(u, 0.0f), 1.0f);
        const uint64_t q = uint64_t(fminf(u * 2097152.0f, 2097151.0f));
        code |= spread21(q) << (2 - k);
    }
    keys[i] = code;
    values[i] = i;
}

// Karras's delta: the common prefix of keys i and j, ties broken by the index.
__device__ __forceinline__ int delta(const uint64_t* keys, uint32_t n, int i, int j) {
    if (j < 0 || j >= int(n)) return -1;
    const uint64_t a = keys[i], b = keys[j];
    if (a == b) return 64 + __clz(uint32_t(i ^ j));
    return __clzll(a ^ b);
}

// Binary nodes: internal 0..n-2, leaves n-1+0 .. n-1+n-1 (index n-1+k is sorted leaf k).
__global__ void karras(const uint64_t* __restrict__ keys, uint32_t n, uint32_t* __restrict__ left, uint32_t* __restrict__ right,
                       uint32_t* __restrict__ parent) {
    const int i = int(blockIdx.x * blockDim.x + threadIdx.x);
    if (i >= int(n) - 1) return;
    const int d = (delta(keys, n, i, i + 1) - delta(keys, n, i, i - 1)) >= 0 ? 1 : -1;
    const int dmin = delta(keys, n, i, i - d);
    int lmax = 2;
    while (delta(keys, n, i, i + lmax * d) > dmin) lmax <<= 1;
    int l = 0;
    for (int t = lmax >> 1; t >= 1; t >>= 1)
        if (delta(keys, n, i, i + (l + t) * d) > dmin) l += t;
    const int j = i + l * d;
    const int dnode = delta(keys, n, i, j);
    int s = 0;
    int t = (l + 1) >> 1;
    for (;;) {
        if (delta(keys, n, i, i + (s + t) * d) > dnode) s += t;
        if (t == 1) break;
        t = (t + 1) >> 1;
    }
    const int gamma = i + s * d + min(d, 0);
    const int lo = min(i, j), hi = max(i, j);
    const uint32_t lc = lo == gamma ? uint32_t(n - 1 + gamma) : uint32_t(gamma);
    const uint32_t rc = hi == gamma + 1 ? uint32_t(n - 1 + gamma + 1) : uint32_t(gamma + 1);
    left[i] = lc;
    right[i] = rc;
    parent[lc] = uint32_t(i);
    parent[rc] = uint32_t(i);
}

// Bottom-up bounds and triangle counts: the second child to arrive at a node merges it.
__global__ void refit(uint32_t n, const uint32_t* __restrict__ order, const Aabb* __restrict__ triBox, const uint32_t* __restrict__ left,
                      const uint32_t* __restrict__ right, const uint32_t* __restrict__ parent, Aabb* box, uint32_t* count,
                      unsigned* flags) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    uint32_t node = n - 1 + k;
    box[node] = triBox[order[k]];
    count[node] = 1;
    if (n == 1) return;
    __threadfence();
    node = parent[node];
    for (;;) {
        if (atomicAdd(&flags[node], 1u) == 0u) return;  // the first arrival leaves the merge to the second
        __threadfence();
        const uint32_t a = left[node], b = right[node];
        const volatile float* pa = reinterpret_cast<const volatile float*>(&box[a]);
        const volatile float* pb = reinterpret_cast<const volatile float*>(&box[b]);
        Aabb m;
        for (int c = 0; c < 3; ++c) {
            m.lo[c] = fminf(pa[c], pb[c]);
            m.hi[c] = fmaxf(pa[3 + c], pb[3 + c]);
        }
        box[node] = m;
        count[node] = *(volatile uint32_t*)&count[a] + *(volatile uint32_t*)&count[b];
        __threadfence();
        if (node == 0) return;
        node = parent[node];
    }
}

__device__ __forceinline__ float area(const Aabb& b) {
    const float x = b.hi[0] - b.lo[0], y = b.hi[1] - b.lo[1], z = b.hi[2] - b.lo[2];
    return x * y + y * z + z * x;
}

__device__ __forceinline__ bool isLeafNode(uint32_t b, uint32_t n) { return b >= n - 1; }

__device__ __forceinline__ Aabb loadBox(const Aabb* box, uint32_t i) {
    const float* p = reinterpret_cast<const float*>(box + i);
    Aabb b;
    for (int k = 0; k < 3; ++k) {
        b.lo[k] = __ldcg(p + k);
        b.hi[k] = __ldcg(p + 3 + k);
    }
    return b;
}

__device__ __forceinline__ void grow(Aabb& a, const Aabb& b) {
    for (int k = 0; k < 3; ++k) {
        a.lo[k] = fminf(a.lo[k], b.lo[k]);
        a.hi[k] = fmaxf(a.hi[k], b.hi[k]);
    }
}

// Treelet restructuring (Karras and Aila 2013, "Fast Parallel Construction of High-Quality Bounding Volume
// Hierarchies"): bottom up, as refit, each internal node of at least kTreelet triangles is the root of a treelet of
// kTreelet subtrees (grown by opening the largest-area subtree), rearranged into the binary tree over them of least
// surface-area cost (Ci per internal node's area, Ct per triangle's leaf area), found by dynamic programming over the
// 2^kTreelet - 1 subsets. The treelet keeps its root and reuses its internal nodes; subtrees below it are final.
// Reads of nodes other threads wrote go through L2 (__ldcg), after the arrival counter that orders them.
constexpr int kTreelet = 7;
constexpr float kCi = 1.2f, kCt = 1.0f;
constexpr int kRestructurePasses = 3;

__device__ void optimiseTreelet(uint32_t root, uint32_t n, uint32_t* left, uint32_t* right, uint32_t* parent, Aabb* box, uint32_t* count,
                                float* cost) {
    uint32_t L[kTreelet], I[kTreelet - 1];
    float La[kTreelet];
    int nl = 2, ni = 1;
    I[0] = root;
    L[0] = __ldcg(left + root);
    L[1] = __ldcg(right + root);
    La[0] = area(loadBox(box, L[0]));
    La[1] = area(loadBox(box, L[1]));
    while (nl < kTreelet) {
        int j = -1;
        float best = -1.0f;
        for (int i = 0; i < nl; ++i)
            if (!isLeafNode(L[i], n) && La[i] > best) {
                best = La[i];
                j = i;
            }
        if (j < 0) break;
        const uint32_t x = L[j];
        I[ni++] = x;
        L[j] = __ldcg(left + x);
        L[nl] = __ldcg(right + x);
        La[j] = area(loadBox(box, L[j]));
        La[nl] = area(loadBox(box, L[nl]));
        ++nl;
    }
    Aabb lb[kTreelet];
    float lc[kTreelet];
    uint32_t lcount[kTreelet];
    for (int i = 0; i < nl; ++i) {
        lb[i] = loadBox(box, L[i]);
        lc[i] = __ldcg(cost + L[i]);
        lcount[i] = __ldcg(count + L[i]);
    }
    const uint32_t all = (1u << nl) - 1u;
    float c[1 << kTreelet], sa[1 << kTreelet];
    uint8_t part[1 << kTreelet];
    for (uint32_t S = 1; S <= all; ++S) {
        Aabb b = lb[__ffs(S) - 1];
        for (uint32_t m = S & (S - 1); m; m &= m - 1) grow(b, lb[__ffs(m) - 1]);
        sa[S] = area(b);
        if (!(S & (S - 1))) {
            c[S] = lc[__ffs(S) - 1];
            part[S] = 0;
            continue;
        }
        const uint32_t lowest = S & (0u - S);
        float best = FLT_MAX;
        uint32_t bp = lowest;
        for (uint32_t P = (S - 1) & S; P; P = (P - 1) & S) {
            if (!(P & lowest)) continue;
            const float v = c[P] + c[S ^ P];
            if (v < best) {
                best = v;
                bp = P;
            }
        }
        c[S] = kCi * sa[S] + best;
        part[S] = uint8_t(bp);
    }
    // Rebuild top down: each subset of two or more subtrees takes the next internal node of the treelet.
    uint32_t stackS[kTreelet], stackN[kTreelet];
    int sp = 0, next = 1;
    stackS[sp] = all;
    stackN[sp++] = root;
    while (sp) {
        --sp;
        const uint32_t S = stackS[sp], nd = stackN[sp];
        const uint32_t P = part[S], Q = S ^ P;
        uint32_t child[2];
        const uint32_t sub[2] = {P, Q};
        for (int h = 0; h < 2; ++h) {
            if (!(sub[h] & (sub[h] - 1))) {
                child[h] = L[__ffs(sub[h]) - 1];
            } else {
                child[h] = I[next++];
                stackS[sp] = sub[h];
                stackN[sp++] = child[h];
            }
            parent[child[h]] = nd;
        }
        left[nd] = child[0];
        right[nd] = child[1];
        Aabb b = lb[__ffs(S) - 1];
        uint32_t cnt = 0;
        for (uint32_t m = S; m; m &= m - 1) {
            grow(b, lb[__ffs(m) - 1]);
            cnt += lcount[__ffs(m) - 1];
        }
        box[nd] = b;
        count[nd] = cnt;
        cost[nd] = c[S];
    }
}

__global__ void restructure(uint32_t n, uint32_t* left, uint32_t* right, uint32_t* parent, Aabb* box, uint32_t* count, float* cost,
                            unsigned* flags) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    uint32_t node = n - 1 + k;
    cost[node] = kCt * area(box[node]);
    if (n == 1) return;
    __threadfence();
    node = __ldcg(parent + node);
    for (;;) {
        if (atomicAdd(&flags[node], 1u) == 0u) return;  // the first arrival leaves the node to the second
        __threadfence();
        const uint32_t l = __ldcg(left + node), r = __ldcg(right + node);
        const uint32_t cnt = __ldcg(count + l) + __ldcg(count + r);
        if (cnt >= uint32_t(kTreelet)) {
            optimiseTreelet(node, n, left, right, parent, box, count, cost);
        } else {
            Aabb b = loadBox(box, l);
            grow(b, loadBox(box, r));
            box[node] = b;
            count[node] = cnt;
            cost[node] = kCi * area(b) + __ldcg(cost + l) + __ldcg(cost + r);
        }
        __threadfence();
        if (node == 0) return;
        node = __ldcg(parent + node);
    }
}

struct CollapseArgs {
    uint32_t n;
    const uint32_t* left;
    const uint32_t* right;
    const Aabb* box;
    const uint32_t* count;
    const uint32_t* order;      // sorted leaf k -> scene triangle
    const float* vertices;
    const uint32_t* triangles;
    Node8* nodes;
    TriRec* tris;
    uint32_t* nodeCounter;
    uint32_t* triCounter;
    const uint2* queueIn;       // (binary node, wide node)
    uint2* queueOut;
    uint32_t* queueOutCount;
    uint32_t queueInCount;
    uint32_t* overflow;
};


// One wide node from binary node `b`: open the largest-area internal node until eight children; binary subtrees of
// at most three triangles become leaves; order the slots by direction octant; quantise the child boxes.
// The leaf-order triangles with each vertex's coordinates rotated: (y, z, x) for rays whose dominant axis is x, and
// (z, x, y) for y (traverse.cuh triTestRotated); the scene index stays in v0.w.
__global__ void rotateTriangles(const TriRec* __restrict__ tris, uint32_t n, TriRec* __restrict__ yzx, TriRec* __restrict__ zxy) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const TriRec t = tris[i];
    const float4 v[3] = {t.v0, t.v1, t.v2};
    float4 a[3], b[3];
    for (int k = 0; k < 3; ++k) {
        a[k] = make_float4(v[k].y, v[k].z, v[k].x, v[k].w);
        b[k] = make_float4(v[k].z, v[k].x, v[k].y, v[k].w);
    }
    yzx[i] = TriRec{a[0], a[1], a[2]};
    zxy[i] = TriRec{b[0], b[1], b[2]};
}

__global__ void countLeafTriangles(const TriRec* __restrict__ tris, uint32_t n, unsigned* seen) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t id = __float_as_uint(tris[i].v0.w);
    if (id < n) atomicAdd(seen + id, 1u);
}

__global__ void checkLeafTriangles(const unsigned* __restrict__ seen, uint32_t n, uint32_t* bad) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && seen[i] != 1u) atomicAdd(bad, 1u);
}

__global__ void collapse(CollapseArgs a) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= a.queueInCount) return;
    const uint2 item = a.queueIn[q];
    const uint32_t n = a.n;
    uint32_t c[8];
    int nc = 0;
    if (isLeafNode(item.x, n)) {
        c[nc++] = item.x;
    } else {
        c[nc++] = a.left[item.x];
        c[nc++] = a.right[item.x];
    }
    while (nc < 8) {
        // Subtrees of more than three triangles first (each would otherwise become a node of its own); then the small
        // ones, whose triangles stay in this node either way but get tighter boxes.
        int best = -1;
        float bestArea = -1.0f;
        bool bestBig = false;
        for (int i = 0; i < nc; ++i) {
            if (isLeafNode(c[i], n)) continue;
            const bool big = a.count[c[i]] > 3;
            const float s = area(a.box[c[i]]);
            if ((big && !bestBig) || (big == bestBig && s > bestArea)) {
                bestArea = s;
                best = i;
                bestBig = big;
            }
        }
        if (best < 0) break;
        const uint32_t b = c[best];
        c[best] = a.left[b];
        c[nc++] = a.right[b];
    }
    // Node bounds and the octant ordering of the slots.
    Aabb nb;
    for (int k = 0; k < 3; ++k) {
        nb.lo[k] = FLT_MAX;
        nb.hi[k] = -FLT_MAX;
    }
    float cen[8][3];
    for (int i = 0; i < nc; ++i) {
        const Aabb& b = a.box[c[i]];
        for (int k = 0; k < 3; ++k) {
            nb.lo[k] = fminf(nb.lo[k], b.lo[k]);
            nb.hi[k] = fmaxf(nb.hi[k], b.hi[k]);
            cen[i][k] = 0.5f * (b.lo[k] + b.hi[k]);
        }
    }
    const float pc[3] = {0.5f * (nb.lo[0] + nb.hi[0]), 0.5f * (nb.lo[1] + nb.hi[1]), 0.5f * (nb.lo[2] + nb.hi[2])};
    int slotOf[8];
    bool takenSlot[8] = {false, false, false, false, false, false, false, false};
    bool placed[8] = {false, false, false, false, false, false, false, false};
    for (int round = 0; round < nc; ++round) {
        float bestScore = -FLT_MAX;
        int bc = -1, bs = -1;
        for (int i = 0; i < nc; ++i) {
            if (placed[i]) continue;
            for (int s = 0; s < 8; ++s) {
                if (takenSlot[s]) continue;
                // Slot s lies toward (s&1 ? -x : +x, s&2 ? -y : +y, s&4 ? -z : +z) of the node's centre.
                const float score = ((s & 1) ? pc[0] - cen[i][0] : cen[i][0] - pc[0]) + ((s & 2) ? pc[1] - cen[i][1] : cen[i][1] - pc[1]) +
                                    ((s & 4) ? pc[2] - cen[i][2] : cen[i][2] - pc[2]);
                if (score > bestScore) {
                    bestScore = score;
                    bc = i;
                    bs = s;
                }
            }
        }
        placed[bc] = true;
        takenSlot[bs] = true;
        slotOf[bc] = bs;
    }
    // Which children are wide nodes, which leaves (and their triangles).
    int internalCount = 0, triTotal = 0;
    bool internal[8];
    int triCount[8];
    for (int i = 0; i < nc; ++i) {
        const uint32_t cnt = a.count[c[i]];
        internal[i] = !isLeafNode(c[i], n) && cnt > 3;
        triCount[i] = internal[i] ? 0 : int(cnt);
        internalCount += internal[i] ? 1 : 0;
        triTotal += triCount[i];
    }
    const uint32_t childBase = internalCount ? atomicAdd(a.nodeCounter, uint32_t(internalCount)) : 0u;
    const uint32_t triBase = triTotal ? atomicAdd(a.triCounter, uint32_t(triTotal)) : 0u;
    const uint32_t outBase = internalCount ? atomicAdd(a.queueOutCount, uint32_t(internalCount)) : 0u;
    Node8 node;
    node.px = nb.lo[0];
    node.py = nb.lo[1];
    node.pz = nb.lo[2];
    uint8_t e[3];
    float scale[3];
    for (int k = 0; k < 3; ++k) {
        const float extent = __fsub_ru(nb.hi[k], nb.lo[k]);
        int ex = extent > 0.0f ? int(ceilf(log2f(extent / 255.0f))) : -126;
        // Make sure 255 * 2^ex covers the extent whatever log2f's rounding did.
        while (ldexpf(255.0f, ex) < extent) ++ex;
        ex = max(ex, -126);
        e[k] = uint8_t(ex + 127);
        scale[k] = ldexpf(1.0f, -ex);
    }
    node.ex = e[0];
    node.ey = e[1];
    node.ez = e[2];
    uint8_t imask = 0;
    for (int s = 0; s < 8; ++s) {
        node.meta[s] = 0;
        node.qlox[s] = node.qloy[s] = node.qloz[s] = 0;
        node.qhix[s] = node.qhiy[s] = node.qhiz[s] = 0;
    }
    // Internal children are numbered from childBase in slot order; leaf triangles from triBase in slot order.
    int internalRank = 0, triOffset = 0;
    for (int s = 0; s < 8; ++s) {
        int i = -1;
        for (int j = 0; j < nc; ++j)
            if (slotOf[j] == s) i = j;
        if (i < 0) continue;
        const Aabb& b = a.box[c[i]];
        const float p[3] = {nb.lo[0], nb.lo[1], nb.lo[2]};
        uint8_t ql[3], qh[3];
        for (int k = 0; k < 3; ++k) {
            const float lo = floorf(__fsub_rd(b.lo[k], p[k]) * scale[k]);
            const float hi = ceilf(__fsub_ru(b.hi[k], p[k]) * scale[k]);
            ql[k] = uint8_t(fminf(fmaxf(lo, 0.0f), 255.0f));
            qh[k] = uint8_t(fminf(fmaxf(hi, 0.0f), 255.0f));
        }
        node.qlox[s] = ql[0];
        node.qloy[s] = ql[1];
        node.qloz[s] = ql[2];
        node.qhix[s] = qh[0];
        node.qhiy[s] = qh[1];
        node.qhiz[s] = qh[2];
        if (internal[i]) {
            imask |= uint8_t(1u << s);
            node.meta[s] = uint8_t(0x20u | (24u + uint32_t(s)));
            a.queueOut[outBase + internalRank] = make_uint2(c[i], childBase + uint32_t(internalRank));
            ++internalRank;
        } else {
            const int cnt = triCount[i];
            node.meta[s] = uint8_t((((1u << cnt) - 1u) << 5) | uint32_t(triOffset));
            // The subtree's leaves (at most three): walk it.
            uint32_t stack[4];
            int sp = 0;
            stack[sp++] = c[i];
            while (sp) {
                const uint32_t b2 = stack[--sp];
                if (isLeafNode(b2, n)) {
                    const uint32_t tri = a.order[b2 - (n - 1)];
                    const uint32_t ia = a.triangles[3 * tri], ib = a.triangles[3 * tri + 1], ic = a.triangles[3 * tri + 2];
                    TriRec r;
                    r.v0 = make_float4(a.vertices[3 * ia], a.vertices[3 * ia + 1], a.vertices[3 * ia + 2], __uint_as_float(tri));
                    r.v1 = make_float4(a.vertices[3 * ib], a.vertices[3 * ib + 1], a.vertices[3 * ib + 2], 0.0f);
                    r.v2 = make_float4(a.vertices[3 * ic], a.vertices[3 * ic + 1], a.vertices[3 * ic + 2], 0.0f);
                    a.tris[triBase + uint32_t(triOffset)] = r;
                    ++triOffset;
                } else if (sp + 2 <= 4) {
                    stack[sp++] = a.right[b2];
                    stack[sp++] = a.left[b2];
                } else {
                    atomicAdd(a.overflow, 1u);
                }
            }
        }
    }
    node.imask = imask;
    node.childBase = childBase;
    node.triBase = triBase;
    a.nodes[item.y] = node;
}

#define CK(x)                                                                                \
    do {                                                                                     \
        cudaError_t e_ = (x);                                                                \
        if (e_ != cudaSuccess) {                                                             \
            setError("%s:%d %s: %s", __FILE__, __LINE__, #x, cudaGetErrorString(e_));        \
            goto fail;                                                                       \
        }                                                                                    \
    } while (0)

}  // namespace

int buildBvh(const float* dVertices, const uint32_t* dTriangles, uint32_t n, cudaStream_t stream, DeviceBvh* out) {
    if (n == 0) {
        setError("an empty scene has no BVH");
        return 1;
    }
    const uint32_t bn = n > 1 ? 2 * n - 1 : 1;
    Aabb *triBox = nullptr, *box = nullptr;
    uint64_t *keys = nullptr, *keysSorted = nullptr;
    uint32_t *values = nullptr, *order = nullptr, *left = nullptr, *right = nullptr, *parent = nullptr, *count = nullptr;
    float* cost = nullptr;
    unsigned *flags = nullptr, *sceneBox = nullptr, *counters = nullptr;
    uint2 *qa = nullptr, *qb = nullptr;
    void* temp = nullptr;
    size_t tempBytes = 0;
    Node8* nodes = nullptr;
    TriRec* tris = nullptr;
    uint32_t maxNodes = n > 1 ? n - 1 : 1;
    uint32_t host[4] = {0, 0, 0, 0};
    const unsigned boxInit[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
    uint32_t queueCount = 1;
    const uint2 rootItem = make_uint2(0u, 0u);
    int level = 0;
    const int grid = int((n + kBlock - 1) / kBlock);
    CK(cudaMallocAsync(&triBox, sizeof(Aabb) * n, stream));
    CK(cudaMallocAsync(&box, sizeof(Aabb) * bn, stream));
    CK(cudaMallocAsync(&keys, sizeof(uint64_t) * n, stream));
    CK(cudaMallocAsync(&keysSorted, sizeof(uint64_t) * n, stream));
    CK(cudaMallocAsync(&values, sizeof(uint32_t) * n, stream));
    CK(cudaMallocAsync(&order, sizeof(uint32_t) * n, stream));
    CK(cudaMallocAsync(&left, sizeof(uint32_t) * n, stream));
    CK(cudaMallocAsync(&right, sizeof(uint32_t) * n, stream));
    CK(cudaMallocAsync(&parent, sizeof(uint32_t) * bn, stream));
    CK(cudaMallocAsync(&count, sizeof(uint32_t) * bn, stream));
    CK(cudaMallocAsync(&cost, sizeof(float) * bn, stream));
    CK(cudaMallocAsync(&flags, sizeof(unsigned) * n, stream));
    CK(cudaMallocAsync(&sceneBox, sizeof(unsigned) * 6, stream));
    CK(cudaMallocAsync(&counters, sizeof(uint32_t) * 4, stream));
    CK(cudaMallocAsync(&qa, sizeof(uint2) * maxNodes, stream));
    CK(cudaMallocAsync(&qb, sizeof(uint2) * maxNodes, stream));
    CK(cudaMallocAsync(&nodes, sizeof(Node8) * maxNodes, stream));
    CK(cudaMallocAsync(&tris, sizeof(TriRec) * n, stream));
    CK(cudaMemcpyAsync(sceneBox, boxInit, sizeof(boxInit), cudaMemcpyHostToDevice, stream));
    CK(cudaMemsetAsync(flags, 0, sizeof(unsigned) * n, stream));
    CK(cudaMemsetAsync(counters, 0, sizeof(uint32_t) * 4, stream));
    triBounds<<<grid, kBlock, 0, stream>>>(dVertices, dTriangles, n, triBox, sceneBox);
    mortonCodes<<<grid, kBlock, 0, stream>>>(triBox, n, sceneBox, keys, values);
    CK(cudaGetLastError());
    CK(cub::DeviceRadixSort::SortPairs(nullptr, tempBytes, keys, keysSorted, values, order, int(n), 0, 64, stream));
    CK(cudaMallocAsync(&temp, tempBytes, stream));
    CK(cub::DeviceRadixSort::SortPairs(temp, tempBytes, keys, keysSorted, values, order, int(n), 0, 64, stream));
    if (n > 1) karras<<<int((n - 1 + kBlock - 1) / kBlock), kBlock, 0, stream>>>(keysSorted, n, left, right, parent);
    refit<<<grid, kBlock, 0, stream>>>(n, order, triBox, left, right, parent, box, count, flags);
    CK(cudaGetLastError());
    for (int pass = 0; pass < kRestructurePasses && n >= uint32_t(kTreelet); ++pass) {
        CK(cudaMemsetAsync(flags, 0, sizeof(unsigned) * n, stream));
        restructure<<<grid, kBlock, 0, stream>>>(n, left, right, parent, box, count, cost, flags);
        CK(cudaGetLastError());
    }
    // Wide node 0 is the root; counters: [0] wide nodes, [1] triangles placed, [2] next queue size, [3] overflow.
    host[0] = 1;
    CK(cudaMemcpyAsync(counters, host, sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
    CK(cudaMemcpyAsync(qa, &rootItem, sizeof(uint2), cudaMemcpyHostToDevice, stream));
    while (queueCount) {
        CollapseArgs a;
        a.n = n;
        a.left = left;
        a.right = right;
        a.box = box;
        a.count = count;
        a.order = order;
        a.vertices = dVertices;
        a.triangles = dTriangles;
        a.nodes = nodes;
        a.tris = tris;
        a.nodeCounter = counters;
        a.triCounter = counters + 1;
        a.queueIn = qa;
        a.queueOut = qb;
        a.queueOutCount = counters + 2;
        a.queueInCount = queueCount;
        a.overflow = counters + 3;
        CK(cudaMemsetAsync(counters + 2, 0, sizeof(uint32_t), stream));
        collapse<<<int((queueCount + 127) / 128), 128, 0, stream>>>(a);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(host, counters, sizeof(host), cudaMemcpyDeviceToHost, stream));
        CK(cudaStreamSynchronize(stream));
        queueCount = host[2];
        uint2* t = qa;
        qa = qb;
        qb = t;
        if (++level > 4096) {
            setError("BVH collapse did not finish");
            goto fail;
        }
    }
    if (host[1] != n || host[3] != 0) {
        setError("BVH collapse placed %u of %u triangles (%u overflows)", host[1], n, host[3]);
        goto fail;
    }
    // Every scene triangle in exactly one leaf (the restructured hierarchy is a tree over all of them).
    CK(cudaMemsetAsync(flags, 0, sizeof(unsigned) * n, stream));
    CK(cudaMemsetAsync(counters + 3, 0, sizeof(uint32_t), stream));
    countLeafTriangles<<<grid, kBlock, 0, stream>>>(tris, n, flags);
    checkLeafTriangles<<<grid, kBlock, 0, stream>>>(flags, n, counters + 3);
    CK(cudaMemcpyAsync(host + 3, counters + 3, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
    if (host[3] != 0) {
        setError("BVH build: %u triangles not in exactly one leaf", host[3]);
        goto fail;
    }
    CK(cudaMallocAsync(&out->rot[0], sizeof(TriRec) * n, stream));
    CK(cudaMallocAsync(&out->rot[1], sizeof(TriRec) * n, stream));
    rotateTriangles<<<grid, kBlock, 0, stream>>>(tris, n, out->rot[0], out->rot[1]);
    CK(cudaGetLastError());
    out->nodes = nodes;
    out->tris = tris;
    out->nodeCount = host[0];
    out->triCount = n;
    out->levels = uint32_t(level);
    nodes = nullptr;
    tris = nullptr;
fail:
    cudaFreeAsync(triBox, stream);
    cudaFreeAsync(box, stream);
    cudaFreeAsync(keys, stream);
    cudaFreeAsync(keysSorted, stream);
    cudaFreeAsync(values, stream);
    cudaFreeAsync(order, stream);
    cudaFreeAsync(left, stream);
    cudaFreeAsync(right, stream);
    cudaFreeAsync(parent, stream);
    cudaFreeAsync(count, stream);
    cudaFreeAsync(cost, stream);
    cudaFreeAsync(flags, stream);
    cudaFreeAsync(sceneBox, stream);
    cudaFreeAsync(counters, stream);
    cudaFreeAsync(qa, stream);
    cudaFreeAsync(qb, stream);
    cudaFreeAsync(temp, stream);
    if (nodes) cudaFreeAsync(nodes, stream);
    if (tris) cudaFreeAsync(tris, stream);
    if (!out->nodes)
        for (TriRec*& r : out->rot) {
            if (r) cudaFreeAsync(r, stream);
            r = nullptr;
        }
    cudaStreamSynchronize(stream);
    return out->nodes ? 0 : 1;
}

}  // namespace x2
