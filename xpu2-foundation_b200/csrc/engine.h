// Internal interfaces of libx2 shared by its translation units (not part of the C ABI).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "bvh.cuh"

namespace x2 {

// The last failure's text, per host thread (x2_last_error).
void setError(const char* fmt, ...);

}  // namespace x2
struct x2_ctx;
namespace x2 {
// A context's stream and SM count, with its device made current (api.cu).
int contextStream(x2_ctx* ctx, cudaStream_t* stream, int* smCount);

struct DeviceBvh {
    Node8* nodes = nullptr;
    TriRec* tris = nullptr;
    TriRec* rot[2] = {nullptr, nullptr};  // the triangles rotated to (y, z, x) and (z, x, y)
    uint32_t nodeCount = 0, triCount = 0, levels = 0;
};

// Builds the compressed 8-wide BVH of n triangles (3 vertex indices each) over fp32 vertices, all on the device.
// Returns 0 on success; the nodes and triangles are the caller's to free (cudaFree).
int buildBvh(const float* dVertices, const uint32_t* dTriangles, uint32_t n, cudaStream_t stream, DeviceBvh* out);

}  // namespace x2
