// Closest-hit and any-hit traversal of the compressed 8-wide BVH (bvh.cuh) for one ray a thread.
//
// A node is five 16-byte read-only loads. Its eight children are tested with one FMA a slab (Ylitie et al. 2017:
// the ray is expressed in the node's quantised frame once, t = q * (2^e / d) + (p - o) / d), widened by a bound on
// its rounding so the quantised boxes stay conservative (visitNode). Hit children enter a 32-bit mask: internal
// children on bits 24..31 in near-to-far order for the ray's octant (the build places each child in the slot of
// the octant it lies toward), leaf triangles on bits 0..23. The stack holds (child base, mask | imask) pairs and
// lives in registers/local memory; an overflow is counted, never silent.
//
// The triangle test is Woop, Benthin and Wald's watertight test in fp32 without contraction (the library is built
// with -fmad=false): the same operations, in the same order, as the oracle's, so both pick the same triangle. Ties
// go to the nearest t, then the lowest scene triangle index (the reference's triangle::nearer rule, triangle_hit.h:26).
#pragma once
#include "bvh.cuh"

#include <cfloat>

namespace x2 {

constexpr int kStack = 32;

struct RayQ {
    float ox, oy, oz, dx, dy, dz;
    float ix, iy, iz;  // inverse direction for the box test (components below 1e-18 clamped)
    uint32_t oct7;     // XOR pattern that orders a node's slots near to far
    int kz;            // the shear's axes: kz the dominant one, kx = kz + 1 and ky = kz + 2 (mod 3)
    float Sx, Sy, Sz;
    float okx, oky, okz;  // the origin's components along kx, ky, kz
    const TriRec* tris;   // the leaf-order triangles rotated to (kx, ky, kz)
    // The triangle test's t carries an absolute error of a few ulps of the distance to the vertices (its sheared
    // products cancel), which a near hit can make large relative to t: boxes are tested against [tmin - eps,
    // tmax + eps], eps = 2^-18 times the ray origin's distance to the farthest corner of the scene's bounds.
    float eps;
};

__device__ __forceinline__ float pick3(float x, float y, float z, int k) { return k == 0 ? x : (k == 1 ? y : z); }

__device__ __forceinline__ float rayTolerance(const Bvh8& b, float ox, float oy, float oz) {
    const float x = fmaxf(fabsf(b.lo[0] - ox), fabsf(b.hi[0] - ox)), y = fmaxf(fabsf(b.lo[1] - oy), fabsf(b.hi[1] - oy)),
                z = fmaxf(fabsf(b.lo[2] - oz), fabsf(b.hi[2] - oz));
    return (x + y + z) * 0x1p-18f;
}

__device__ __forceinline__ RayQ makeRay(const Bvh8& bvh, float ox, float oy, float oz, float dx, float dy, float dz) {
    RayQ r;
    r.eps = rayTolerance(bvh, ox, oy, oz);
    r.ox = ox;
    r.oy = oy;
    r.oz = oz;
    r.dx = dx;
    r.dy = dy;
    r.dz = dz;
    const float tiny = 1e-18f;
    r.ix = 1.0f / (fabsf(dx) > tiny ? dx : copysignf(tiny, dx));
    r.iy = 1.0f / (fabsf(dy) > tiny ? dy : copysignf(tiny, dy));
    r.iz = 1.0f / (fabsf(dz) > tiny ? dz : copysignf(tiny, dz));
    const uint32_t oct = (signbit(dx) ? 1u : 0u) | (signbit(dy) ? 2u : 0u) | (signbit(dz) ? 4u : 0u);
    r.oct7 = ~oct & 7u;
    const float ax = fabsf(dx), ay = fabsf(dy), az = fabsf(dz);
    const int kz = ax > ay ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
    const int kx = kz == 2 ? 0 : kz + 1;
    const int ky = kx == 2 ? 0 : kx + 1;
    const float dzz = pick3(dx, dy, dz, kz);
    r.kz = kz;
    r.Sx = pick3(dx, dy, dz, kx) / dzz;
    r.Sy = pick3(dx, dy, dz, ky) / dzz;
    r.Sz = 1.0f / dzz;
    r.okx = pick3(ox, oy, oz, kx);
    r.oky = pick3(ox, oy, oz, ky);
    r.okz = pick3(ox, oy, oz, kz);
    r.tris = kz == 0 ? bvh.rot[0] : kz == 1 ? bvh.rot[1] : bvh.rot[2];  // constant indices: bvh stays in registers
    return r;
}

// Watertight ray/triangle test on vertices whose coordinates come in the ray's (kx, ky, kz) order. The oracle's triHit
// swaps kx and ky when the dominant direction component is negative, to keep the edge functions' signs; here the axes
// stay in rotation order, which negates U, V, W, their sum and T exactly (a product's operands commute, and a
// difference's operands exchanged give its exact negation, in float and in the double fallback alike), so the test's
// outcome (the same-sign test, the zero determinant) and t = T / det are bit for bit the oracle's.
__device__ __forceinline__ bool triTestRotated(const RayQ& r, const float4& a, const float4& b, const float4& c, float tmin, float tmax,
                                               float& tOut) {
    const float Akx = a.x - r.okx, Aky = a.y - r.oky, Akz = a.z - r.okz;
    const float Bkx = b.x - r.okx, Bky = b.y - r.oky, Bkz = b.z - r.okz;
    const float Ckx = c.x - r.okx, Cky = c.y - r.oky, Ckz = c.z - r.okz;
    const float Ax = Akx - r.Sx * Akz, Ay = Aky - r.Sy * Akz;
    const float Bx = Bkx - r.Sx * Bkz, By = Bky - r.Sy * Bkz;
    const float Cx = Ckx - r.Sx * Ckz, Cy = Cky - r.Sy * Ckz;
    float U = Cx * By - Cy * Bx, V = Ax * Cy - Ay * Cx, W = Bx * Ay - By * Ax;
    if (U == 0.0f || V == 0.0f || W == 0.0f) {
        U = float(double(Cx) * double(By) - double(Cy) * double(Bx));
        V = float(double(Ax) * double(Cy) - double(Ay) * double(Cx));
        W = float(double(Bx) * double(Ay) - double(By) * double(Ax));
    }
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
    const float det = U + V + W;
    if (det == 0.0f) return false;
    const float Az = r.Sz * Akz, Bz = r.Sz * Bkz, Cz = r.Sz * Ckz;
    const float T = U * Az + V * Bz + W * Cz;
    const float t = T / det;
    if (!(t >= tmin && t <= tmax)) return false;
    tOut = t;
    return true;
}
// The same test on vertices in scene order (x, y, z): picks each vertex's coordinates in the ray's axis order.
__device__ __forceinline__ bool triTest(const RayQ& r, const float4& a, const float4& b, const float4& c, float tmin, float tmax, float& tOut) {
    const int kx = r.kz == 2 ? 0 : r.kz + 1, ky = kx == 2 ? 0 : kx + 1;
    auto rotate = [&](const float4& v) { return make_float4(pick3(v.x, v.y, v.z, kx), pick3(v.x, v.y, v.z, ky), pick3(v.x, v.y, v.z, r.kz), v.w); };
    return triTestRotated(r, rotate(a), rotate(b), rotate(c), tmin, tmax, tOut);
}

// Three-input max / min (one instruction on sm_100; same NaN rule as fmaxf / fminf).
__device__ __forceinline__ float max3f(float a, float b, float c) {
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}
__device__ __forceinline__ float min3f(float a, float b, float c) {
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

// Byte j of w with 2^23 added, as an exact float: 0x4B0000bb is 2^23 + bb (one byte permute, no conversion).
__device__ __forceinline__ float qbyte23(uint32_t w, int j) { return __uint_as_float(__byte_perm(w, 0x4B000000u, 0x7440u | uint32_t(j))); }

// One node: the hit mask (bits 24..31 internal children in traversal order, 0..23 leaf triangles), its child and
// triangle bases and its internal-child mask.
//
// Conservative by construction: the quantised child boxes contain the exact ones (the build rounds outward). The slab
// distance q * s + a (s = 2^e * (1/d), a = (p - o) * (1/d)) is computed as one FMA of the byte with 2^23 added,
// (2^23 + q) * s + c with c = (a -+ w) - 2^23 s, which saves the byte's conversion: against q * s + a exactly, it errs
// by the four roundings of a and s (under 2^-22 (|a| + 255 |s|)), by c's rounding at the magnitude of 2^23 s (at most
// |s| / 2 + 2^-24 (|a| + w)) and by the FMA's (under 2^-24 (|a| + 257 |s| + w)). Every slab is widened by
// w = |s| / 2 + 2^-19 (|a| + 256 |s|) each way, which covers them; 2^23 s stays finite for the scene extents the
// loader admits.
__device__ __forceinline__ uint32_t visitNode(const Node8* __restrict__ nodes, uint32_t index, const RayQ& r, float tmin, float tmax,
                                              uint32_t& childBase, uint32_t& triBase, uint32_t& imask) {
    const uint4* p = reinterpret_cast<const uint4*>(nodes + index);
    const uint4 n0 = __ldg(p), n1 = __ldg(p + 1), n2 = __ldg(p + 2), n3 = __ldg(p + 3), n4 = __ldg(p + 4);
    const float px = __uint_as_float(n0.x), py = __uint_as_float(n0.y), pz = __uint_as_float(n0.z);
    const uint32_t ex = n0.w & 0xffu, ey = (n0.w >> 8) & 0xffu, ez = (n0.w >> 16) & 0xffu;
    imask = n0.w >> 24;
    childBase = n1.x;
    triBase = n1.y;
    const float sx = __uint_as_float(ex << 23) * r.ix, sy = __uint_as_float(ey << 23) * r.iy, sz = __uint_as_float(ez << 23) * r.iz;
    const float ax = (px - r.ox) * r.ix, ay = (py - r.oy) * r.iy, az = (pz - r.oz) * r.iz;
    const float wx = 0.5f * fabsf(sx) + (fabsf(ax) + 256.0f * fabsf(sx)) * 0x1p-19f,
                wy = 0.5f * fabsf(sy) + (fabsf(ay) + 256.0f * fabsf(sy)) * 0x1p-19f,
                wz = 0.5f * fabsf(sz) + (fabsf(az) + 256.0f * fabsf(sz)) * 0x1p-19f;
    const float axn = __fmaf_rn(-8388608.0f, sx, ax - wx), axf = __fmaf_rn(-8388608.0f, sx, ax + wx);
    const float ayn = __fmaf_rn(-8388608.0f, sy, ay - wy), ayf = __fmaf_rn(-8388608.0f, sy, ay + wy);
    const float azn = __fmaf_rn(-8388608.0f, sz, az - wz), azf = __fmaf_rn(-8388608.0f, sz, az + wz);
    // The near and far planes' quantised words for the ray's direction signs, chosen once a node.
    const bool fx = r.ix >= 0.0f, fy = r.iy >= 0.0f, fz = r.iz >= 0.0f;
    const uint32_t nx0 = fx ? n2.x : n3.z, nx1 = fx ? n2.y : n3.w, fx0 = fx ? n3.z : n2.x, fx1 = fx ? n3.w : n2.y;
    const uint32_t ny0 = fy ? n2.z : n4.x, ny1 = fy ? n2.w : n4.y, fy0 = fy ? n4.x : n2.z, fy1 = fy ? n4.y : n2.w;
    const uint32_t nz0 = fz ? n3.x : n4.z, nz1 = fz ? n3.y : n4.w, fz0 = fz ? n4.z : n3.x, fz1 = fz ? n4.w : n3.y;
    // Child metadata with internal slots' bit positions (24 + slot: bits 3 and 4 both set, which no triangle offset
    // has) permuted to the ray's near-to-far order; an empty slot's byte is 0 and sets nothing.
    const uint32_t m0 = n1.z ^ ((((n1.z & (n1.z << 1)) & 0x10101010u) >> 4) * r.oct7);
    const uint32_t m1 = n1.w ^ ((((n1.w & (n1.w << 1)) & 0x10101010u) >> 4) * r.oct7);
    uint32_t hits = 0;
#pragma unroll
    for (int s = 0; s < 8; ++s) {
        const int j = s & 3;
        const float nx = __fmaf_rn(qbyte23(s < 4 ? nx0 : nx1, j), sx, axn), fxx = __fmaf_rn(qbyte23(s < 4 ? fx0 : fx1, j), sx, axf);
        const float ny = __fmaf_rn(qbyte23(s < 4 ? ny0 : ny1, j), sy, ayn), fyy = __fmaf_rn(qbyte23(s < 4 ? fy0 : fy1, j), sy, ayf);
        const float nz = __fmaf_rn(qbyte23(s < 4 ? nz0 : nz1, j), sz, azn), fzz = __fmaf_rn(qbyte23(s < 4 ? fz0 : fz1, j), sz, azf);
        const float entry = max3f(nx, ny, fmaxf(nz, tmin)), exit = min3f(fxx, fyy, fminf(fzz, tmax));
        const uint32_t meta = ((s < 4 ? m0 : m1) >> (8 * j)) & 0xffu;
        if (entry <= exit) hits |= (meta >> 5) << (meta & 31u);
    }
    return hits;
}

// Traversal work of a counting run (node visits and triangle tests), for the roofline's algorithmic bytes. The
// timed kernels are instantiated without it.
// The persistent kernels also count their warps' lane use: warp steps and the live lanes in them, steps that ran the
// node visit and the lanes that visited, triangle-test iterations and the lanes that tested.
struct TraversalStats {
    unsigned long long rays, nodes, tris;
    unsigned long long steps, liveLanes, nodeSteps, nodeLanes, triSteps, triLanes;
};

// Closest hit on [tmin, tmax]: the scene triangle index (~0u: none), its t and its position in leaf order.
template <bool kStats>
static __device__ __noinline__ uint32_t traceClosest(const Bvh8 bvh, const RayQ& r, float tmin, float tmax, float& tHit, uint32_t* leafOut,
                                                     uint32_t* overflow, TraversalStats* stats) {
    uint2 stack[kStack];
    int sp = 0;
    uint32_t best = ~0u, bestLeaf = 0, nodes = 0, tris = 0;
    float tBest = tmax;
    uint32_t gBase = 0, gBits = 0x80000000u, gImask = 1u << (7u ^ r.oct7);
    for (;;) {
        while (gBits & 0xff000000u) {
            const uint32_t b = __ffs(gBits >> 24) - 1;
            gBits &= ~(1u << (24 + b));
            const uint32_t slot = b ^ r.oct7;
            const uint32_t child = gBase + __popc(gImask & ((1u << slot) - 1u));
            if (gBits & 0xff000000u) {
                if (sp < kStack) stack[sp++] = make_uint2(gBase, gBits | (gImask << 16));
                else atomicAdd(overflow, 1u);
            }
            uint32_t childBase, triBase, imask;
            const uint32_t hits = visitNode(bvh.nodes, child, r, tmin - r.eps, tBest + r.eps, childBase, triBase, imask);
            if (kStats) ++nodes;
            uint32_t tBits = hits & 0x00ffffffu;
            while (tBits) {
                const uint32_t k = __ffs(tBits) - 1;
                tBits &= tBits - 1;
                const float4* tp = reinterpret_cast<const float4*>(r.tris + triBase + k);
                const float4 v0 = __ldg(tp), v1 = __ldg(tp + 1), v2 = __ldg(tp + 2);
                if (kStats) ++tris;
                float t;
                if (triTestRotated(r, v0, v1, v2, tmin, tBest, t)) {
                    const uint32_t id = __float_as_uint(v0.w);
                    if (t < tBest || (t == tBest && id < best)) {
                        tBest = t;
                        best = id;
                        bestLeaf = triBase + k;
                    }
                }
            }
            gBase = childBase;
            gBits = hits & 0xff000000u;
            gImask = imask;
        }
        if (sp == 0) break;
        const uint2 e = stack[--sp];
        gBase = e.x;
        gBits = e.y & 0xff000000u;
        gImask = (e.y >> 16) & 0xffu;
    }
    if (kStats) {
        atomicAdd(&stats->rays, 1ull);
        atomicAdd(&stats->nodes, (unsigned long long)nodes);
        atomicAdd(&stats->tris, (unsigned long long)tris);
    }
    tHit = tBest;
    *leafOut = bestLeaf;
    return best;
}

// A ray traced one node a step, for kernels that keep every lane of a warp busy by handing a lane whose ray is done
// the next ray of the queue (persistent threads with dynamic ray fetch; Aila and Laine 2009). The steps visit the
// same nodes and test the same triangles, in the same order, as traceClosest / traceAny, so the results are the same.
//
// The stack's first kShort entries may live in shared memory, entry-major (entry e of thread t at
// shortStack[e * blockDim.x + t], so a warp's accesses fall in distinct banks), the deeper ones in the thread's local
// array `deep` (kStack - kShort entries); with kShort 0 all of them are local (the shared memory then stays L1's).
// The local array is the caller's, not a member of Walk: an array indexed at run time keeps its whole aggregate in
// local memory, and Walk's scalars, updated every step, must stay in registers.
constexpr int kShortStack = 8;
template <int kShort>
struct Walk {
    uint2* shortStack;  // this thread's column: entry e at shortStack[e * blockDim.x]
    int sp;
    uint32_t base, bits, imask;  // the node group being visited: its child base, hit mask, internal-child mask
    uint32_t tbase, tbits;       // triangles of the last node still to test: first leaf-order index, mask
    float tmin, tmax;            // closest hit: tmax is the nearest hit so far
    uint32_t best, bestLeaf;     // closest hit: scene triangle (~0u none) and leaf-order index; any hit: 1 if occluded
    uint32_t nodes, tris;        // counting mode
};

template <int kShort>
__device__ __forceinline__ void walkPush(Walk<kShort>& w, uint2* deep, uint2 e, uint32_t* overflow) {
    if (w.sp < kShort) w.shortStack[size_t(w.sp) * blockDim.x] = e;
    else if (w.sp < kStack) deep[w.sp - kShort] = e;
    else {
        atomicAdd(overflow, 1u);
        return;
    }
    ++w.sp;
}
template <int kShort>
__device__ __forceinline__ uint2 walkPop(Walk<kShort>& w, const uint2* deep) {
    --w.sp;
    return w.sp < kShort ? w.shortStack[size_t(w.sp) * blockDim.x] : deep[w.sp - kShort];
}

template <bool kAny, int kShort>
__device__ __forceinline__ void walkStart(Walk<kShort>& w, const RayQ& r, float tmin, float tmax) {
    w.sp = 0;
    w.base = 0;
    w.bits = 0x80000000u;
    w.imask = 1u << (7u ^ r.oct7);
    w.tbase = 0;
    w.tbits = 0;
    w.tmin = tmin;
    w.tmax = tmax;
    w.best = kAny ? 0u : ~0u;
    w.bestLeaf = 0;
}

// One step: a node visit (when no triangles are pending) and then at most `triLimit` triangle tests, the rest left
// for the next steps, so that a lane with a full leaf does not hold its warp for all of them at once. The tests run
// in the same order whatever the limit. True once the ray is done.
//
// `lanes` is the set of the warp's lanes that make this step (all of them call it): they meet at a __syncwarp after
// the stack pop, so that the lanes that popped and those that went on with their node group visit their nodes
// together, and again before the triangle tests. The compiler may otherwise give each way its own copy of the code
// that follows, and the warp then runs it once for each group of lanes.
template <bool kAny, int kShort>
__device__ __forceinline__ bool walkStep(const Bvh8& bvh, const RayQ& r, Walk<kShort>& w, uint2* deep, uint32_t* overflow,
                                         uint32_t triLimit, unsigned lanes) {
    bool visit = !w.tbits, done = false;
    if (visit && !(w.bits & 0xff000000u)) {
        if (w.sp == 0) {
            visit = false;
            done = true;
        } else {
            const uint2 e = walkPop(w, deep);
            w.base = e.x;
            w.bits = e.y & 0xff000000u;
            w.imask = (e.y >> 16) & 0xffu;
        }
    }
    __syncwarp(lanes);
    if (visit) {
        const uint32_t b = __ffs(w.bits >> 24) - 1;
        w.bits &= ~(1u << (24 + b));
        const uint32_t slot = b ^ r.oct7;
        const uint32_t child = w.base + __popc(w.imask & ((1u << slot) - 1u));
        if (w.bits & 0xff000000u) walkPush(w, deep, make_uint2(w.base, w.bits | (w.imask << 16)), overflow);
        uint32_t childBase, imask;
        const uint32_t hits = visitNode(bvh.nodes, child, r, w.tmin - r.eps, w.tmax + r.eps, childBase, w.tbase, imask);
        ++w.nodes;
        w.tbits = hits & 0x00ffffffu;
        w.base = childBase;
        w.bits = hits & 0xff000000u;
        w.imask = imask;
    }
    __syncwarp(lanes);  // and the triangle tests together, the lanes that visited and those that held triangles
    for (uint32_t n = 0; w.tbits && n < triLimit; ++n) {
        const uint32_t k = __ffs(w.tbits) - 1;
        w.tbits &= w.tbits - 1;
        const float4* tp = reinterpret_cast<const float4*>(r.tris + w.tbase + k);
        const float4 v0 = __ldg(tp), v1 = __ldg(tp + 1), v2 = __ldg(tp + 2);
        ++w.tris;
        float t;
        if (triTestRotated(r, v0, v1, v2, w.tmin, w.tmax, t)) {
            if (kAny) {
                w.best = 1;
                return true;
            }
            const uint32_t id = __float_as_uint(v0.w);
            if (t < w.tmax || (t == w.tmax && id < w.best)) {
                w.tmax = t;
                w.best = id;
                w.bestLeaf = w.tbase + k;
            }
        }
    }
    return done || (!w.tbits && !(w.bits & 0xff000000u) && w.sp == 0);
}

// The entry on top of the stack, left there.
template <int kShort>
__device__ __forceinline__ uint2 walkTop(const Walk<kShort>& w, const uint2* deep) {
    const int t = w.sp - 1;
    return t < kShort ? w.shortStack[size_t(t) * blockDim.x] : deep[t - kShort];
}

// walkStep with a lane's node visits and triangle tests overlapped: a lane that holds a leaf's triangles tests one of
// them and also visits its next node in the same step, instead of visiting no node until the leaf is done. A leaf met
// while one is held goes onto the stack as a triangle group (an entry whose top byte is zero, where a node group
// always has an internal child); once the held leaf is done, a triangle group on top of the stack becomes the held
// one. Every node and triangle walkStep would reach is still reached, in another order (a closest hit's culling sees
// a larger tmax for a while, so it may visit a few more nodes); a closest hit does not depend on the order (nearest t,
// then lowest triangle), and an any hit only asks whether one exists.
//
// `any` is the ray's kind (any hit, or closest hit); a kernel whose lanes walk rays of both kinds in the same steps
// passes it at run time, so that one copy of the step's code serves them all (start a closest-hit ray with
// walkStart<false> and an any-hit ray with walkStart<true>).
template <int kShort>
__device__ __forceinline__ bool walkStepOverlapKind(const Bvh8& bvh, const RayQ& r, Walk<kShort>& w, uint2* deep, uint32_t* overflow,
                                                    unsigned lanes, bool any) {
    bool visit = (w.bits & 0xff000000u) != 0;
    if (!visit && w.sp > 0) {
        const uint2 e = walkTop(w, deep);
        if (e.y >> 24) {  // a node group
            --w.sp;
            w.base = e.x;
            w.bits = e.y & 0xff000000u;
            w.imask = (e.y >> 16) & 0xffu;
            visit = true;
        } else if (!w.tbits) {  // a triangle group, taken once the held one is done
            --w.sp;
            w.tbase = e.x;
            w.tbits = e.y;
        }
    }
    __syncwarp(lanes);
    if (visit) {
        const uint32_t b = __ffs(w.bits >> 24) - 1;
        w.bits &= ~(1u << (24 + b));
        const uint32_t slot = b ^ r.oct7;
        const uint32_t child = w.base + __popc(w.imask & ((1u << slot) - 1u));
        if (w.bits & 0xff000000u) walkPush(w, deep, make_uint2(w.base, w.bits | (w.imask << 16)), overflow);
        uint32_t childBase, imask, triBase;
        const uint32_t hits = visitNode(bvh.nodes, child, r, w.tmin - r.eps, w.tmax + r.eps, childBase, triBase, imask);
        ++w.nodes;
        const uint32_t nt = hits & 0x00ffffffu;
        if (nt) {
            if (w.tbits) {
                walkPush(w, deep, make_uint2(triBase, nt), overflow);
            } else {
                w.tbase = triBase;
                w.tbits = nt;
            }
        }
        w.base = childBase;
        w.bits = hits & 0xff000000u;
        w.imask = imask;
    }
    __syncwarp(lanes);
    if (w.tbits) {
        const uint32_t k = __ffs(w.tbits) - 1;
        w.tbits &= w.tbits - 1;
        const float4* tp = reinterpret_cast<const float4*>(r.tris + w.tbase + k);
        const float4 v0 = __ldg(tp), v1 = __ldg(tp + 1), v2 = __ldg(tp + 2);
        ++w.tris;
        float t;
        if (triTestRotated(r, v0, v1, v2, w.tmin, w.tmax, t)) {
            if (any) {
                w.best = 1;
                return true;
            }
            const uint32_t id = __float_as_uint(v0.w);
            if (t < w.tmax || (t == w.tmax && id < w.best)) {
                w.tmax = t;
                w.best = id;
                w.bestLeaf = w.tbase + k;
            }
        }
    }
    return !w.tbits && !(w.bits & 0xff000000u) && w.sp == 0;
}
template <bool kAny, int kShort>
__device__ __forceinline__ bool walkStepOverlap(const Bvh8& bvh, const RayQ& r, Walk<kShort>& w, uint2* deep, uint32_t* overflow,
                                                unsigned lanes) {
    return walkStepOverlapKind<kShort>(bvh, r, w, deep, overflow, lanes, kAny);
}

// Any hit on [tmin, tmax].
template <bool kStats>
static __device__ __noinline__ bool traceAny(const Bvh8 bvh, const RayQ& r, float tmin, float tmax, uint32_t* overflow, TraversalStats* stats) {
    uint2 stack[kStack];
    int sp = 0;
    uint32_t nodes = 0, tris = 0;
    bool hit = false;
    uint32_t gBase = 0, gBits = 0x80000000u, gImask = 1u << (7u ^ r.oct7);
    for (;;) {
        while (gBits & 0xff000000u) {
            const uint32_t b = __ffs(gBits >> 24) - 1;
            gBits &= ~(1u << (24 + b));
            const uint32_t slot = b ^ r.oct7;
            const uint32_t child = gBase + __popc(gImask & ((1u << slot) - 1u));
            if (gBits & 0xff000000u) {
                if (sp < kStack) stack[sp++] = make_uint2(gBase, gBits | (gImask << 16));
                else atomicAdd(overflow, 1u);
            }
            uint32_t childBase, triBase, imask;
            const uint32_t hits = visitNode(bvh.nodes, child, r, tmin - r.eps, tmax + r.eps, childBase, triBase, imask);
            if (kStats) ++nodes;
            uint32_t tBits = hits & 0x00ffffffu;
            while (tBits) {
                const uint32_t k = __ffs(tBits) - 1;
                tBits &= tBits - 1;
                const float4* tp = reinterpret_cast<const float4*>(r.tris + triBase + k);
                const float4 v0 = __ldg(tp), v1 = __ldg(tp + 1), v2 = __ldg(tp + 2);
                if (kStats) ++tris;
                float t;
                if (triTestRotated(r, v0, v1, v2, tmin, tmax, t)) {
                    hit = true;
                    goto done;
                }
            }
            gBase = childBase;
            gBits = hits & 0xff000000u;
            gImask = imask;
        }
        if (sp == 0) break;
        const uint2 e = stack[--sp];
        gBase = e.x;
        gBits = e.y & 0xff000000u;
        gImask = (e.y >> 16) & 0xffu;
    }
done:
    if (kStats) {
        atomicAdd(&stats->rays, 1ull);
        atomicAdd(&stats->nodes, (unsigned long long)nodes);
        atomicAdd(&stats->tris, (unsigned long long)tris);
    }
    return hit;
}

}  // namespace x2
