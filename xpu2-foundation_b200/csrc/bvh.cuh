// Compressed 8-wide BVH (Ylitie, Karras, Laine 2017, "Efficient Incoherent Ray Traversal on GPUs Through
// Compressed Wide BVHs") and the watertight triangle test (Woop, Benthin, Wald 2013) shared by the closest-hit
// and any-hit traversals.
//
// Layout in HBM:
//   Node8[nodes]    80 B each, five 16-byte words: the node's origin p and per-axis exponents (child boxes are
//                   p + 2^e * q with 8-bit q), the internal-child mask, the first child node and first triangle,
//                   8 meta bytes and 48 quantised bounds. Children of a node are contiguous (internal ones in slot
//                   order from childBase, leaf triangles from triBase), so a node costs five 16-byte loads.
//   TriRec[tris]    48 B each, three float4: the vertices (fp32, as the scene gives them) with the triangle's
//                   scene index in v0.w (bit cast), stored in leaf order so a leaf's 1-3 triangles are adjacent.
//   two more TriRec[tris] copies with each vertex's coordinates rotated to (y, z, x) and (z, x, y): the watertight
//                   test wants a vertex's coordinates in the order (kx, ky, kz) of its ray's dominant axis kz, and
//                   a ray reads the copy of its axis (the original serves kz = 2) instead of picking components.
// The reference delegates traversal to Embree / OptiX RT cores (async_cpu.h:669-720, async_gpu_device.h:
// 330-355, 521-533); B200 has no RT cores, so this is the engine's own.
#pragma once
#include <cstdint>

namespace x2 {

struct alignas(16) Node8 {
    float px, py, pz;
    uint8_t ex, ey, ez, imask;  // exponents biased by 127; bit i: slot i holds an internal node
    uint32_t childBase, triBase;
    uint8_t meta[8];            // 0: empty; internal: 0x20 | (24 + slot); leaf: (unary count << 5) | triangle offset
    uint8_t qlox[8], qloy[8], qloz[8], qhix[8], qhiy[8], qhiz[8];
};
static_assert(sizeof(Node8) == 80, "80-byte wide nodes");

struct alignas(16) TriRec {
    float4 v0, v1, v2;  // v0.w: the triangle's index in the scene (bits)
};
static_assert(sizeof(TriRec) == 48, "48-byte triangles");

struct Bvh8 {
    const Node8* nodes;
    const TriRec* tris;
    uint32_t nodeCount, triCount;
    float lo[3], hi[3];     // the scene's bounds, for each ray's distance tolerance (traverse.cuh, makeRay)
    const TriRec* rot[3];   // by dominant axis kz: the triangles rotated to (kx, ky, kz) (rot[2] is tris)
};

}  // namespace x2
