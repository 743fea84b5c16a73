// Cache bandwidth probes: the L2 and L1 read rates of this GPU, the ceilings the traversal kernels' node and triangle
// fetches run against (their working sets mostly hit L1 and L2, not HBM). Measurement only; no part of the path.
//
// x2_probe_bandwidth reads a device buffer of `bytes` `passes` times in one launch with 16-byte read-only loads:
//  - level 2: the whole buffer by every block in turn (a grid-stride sweep over all of it each pass), so with a buffer
//    well under the L2's 126 MB every read after the first pass is an L2 hit;
//  - level 1: each block re-reads its own slice of at most 96 KB, which stays in its SM's L1.
// Returns the bytes read over the launch's device time (CUDA events), in GB/s.
#include <cuda_runtime.h>

#include "../../include/x2.h"
#include "engine.h"

namespace x2 {
namespace {

__global__ void sweepL2(const uint4* __restrict__ buf, unsigned long long n, uint32_t passes, unsigned* sink) {
    uint32_t acc = 0;
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (uint32_t p = 0; p < passes; ++p)
        for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
            const uint4 v = __ldg(buf + i);
            acc ^= v.x ^ v.y ^ v.z ^ v.w;
        }
    if (acc == 0x9e3779b9u) atomicAdd(sink, 1u);  // keeps the loads; practically never true
}

__global__ void sweepL1(const uint4* __restrict__ buf, uint32_t slice, uint32_t passes, unsigned* sink) {
    uint32_t acc = 0;
    const uint4* mine = buf + (unsigned long long)blockIdx.x * slice;
    for (uint32_t p = 0; p < passes; ++p)
        for (uint32_t i = threadIdx.x; i < slice; i += blockDim.x) {
            const uint4 v = __ldg(mine + i);
            acc ^= v.x ^ v.y ^ v.z ^ v.w;
        }
    if (acc == 0x9e3779b9u) atomicAdd(sink, 1u);
}

}  // namespace
}  // namespace x2

using namespace x2;

extern "C" int x2_probe_bandwidth(x2_ctx* ctx, uint32_t level, uint64_t bytes, uint32_t passes, float* gbs) {
    cudaStream_t st;
    int smCount = 0;
    if (int rc = contextStream(ctx, &st, &smCount)) return rc;
    if (!gbs || !passes || bytes < 4096 || (level != 1 && level != 2)) {
        setError("x2_probe_bandwidth: level 1 or 2, at least 4096 bytes and one pass");
        return X2_EINVAL;
    }
    const uint32_t threads = 512, blocks = uint32_t(smCount) * 2;
    uint32_t slice = 0;
    unsigned long long total = bytes;
    if (level == 1) {
        slice = uint32_t(std::min<uint64_t>(bytes, 96u << 10) / 16);
        total = (unsigned long long)slice * 16 * blocks;
    }
    void* buf = nullptr;
    unsigned* sink = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = X2_OK;
    if (cudaMalloc(&buf, total) != cudaSuccess || cudaMalloc(&sink, sizeof(unsigned)) != cudaSuccess ||
        cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        setError("x2_probe_bandwidth: allocation failed");
        rc = X2_ENOMEM;
    }
    if (rc == X2_OK) {
        cudaMemsetAsync(buf, 1, total, st);
        const uint4* b = static_cast<const uint4*>(buf);
        // One warm pass, then the timed launch.
        if (level == 2) sweepL2<<<blocks, threads, 0, st>>>(b, total / 16, 1, sink);
        else sweepL1<<<blocks, threads, 0, st>>>(b, slice, 1, sink);
        cudaEventRecord(e0, st);
        if (level == 2) sweepL2<<<blocks, threads, 0, st>>>(b, total / 16, passes, sink);
        else sweepL1<<<blocks, threads, 0, st>>>(b, slice, passes, sink);
        cudaEventRecord(e1, st);
        float ms = 0.0f;
        if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess || ms <= 0.0f) {
            setError("x2_probe_bandwidth: %s", cudaGetErrorString(cudaGetLastError()));
            rc = X2_ECUDA;
        } else {
            *gbs = float(double(total) * passes / (ms * 1e-3) / 1e9);
        }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(buf);
    cudaFree(sink);
    return rc;
}
