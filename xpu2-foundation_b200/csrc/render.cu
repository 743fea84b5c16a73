// The plain megakernel and the small kernels around it.
//
// renderChunks: persistent warps claim 32 work items at a time (one atomic a warp); an item is a (chunk, tile
// position, sample) triple laid out sample-minor, so a warp renders consecutive samples of one or two pixels:
// its camera rays are coherent and its film update is one segmented warp reduction and one set of FP64 atomics
// a pixel (warp-aggregated atomics) instead of one a sample. The film is the reference's: FP64 sums (rgb + alpha),
// FP64 odd-index sums (adaptive frames), U32 counts (async_gpu.cu:320-364).
#include "integrator.cuh"
#include "render.h"

namespace x2 {

cudaError_t uploadSobol(const uint32_t directions[17][32]) {
    return cudaMemcpyToSymbol(c_sobol, directions, sizeof(uint32_t) * 17 * 32);
}

namespace {

__device__ __forceinline__ uint32_t tilePixel(uint32_t tile, uint32_t position, uint32_t width, uint32_t height) {
    const uint32_t tilesX = (width + 7) / 8;
    const uint32_t x = (tile % tilesX) * 8 + position % 8;
    const uint32_t y = (tile / tilesX) * 8 + position / 8;
    return x < width && y < height ? y * width + x : ~0u;
}

__device__ __forceinline__ void addCounters(Counters* dst, unsigned long long trace, unsigned long long nee, unsigned long long bsdf,
                                            unsigned long long held, unsigned long long samples, unsigned long long errors) {
    const unsigned full = 0xffffffffu;
#pragma unroll
    for (int off = 16; off; off >>= 1) {
        trace += __shfl_down_sync(full, trace, off);
        nee += __shfl_down_sync(full, nee, off);
        bsdf += __shfl_down_sync(full, bsdf, off);
        held += __shfl_down_sync(full, held, off);
        samples += __shfl_down_sync(full, samples, off);
        errors += __shfl_down_sync(full, errors, off);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&dst->trace, trace);
        atomicAdd(&dst->nee, nee);
        atomicAdd(&dst->bsdf, bsdf);
        atomicAdd(&dst->held, held);
        atomicAdd(&dst->samples, samples);
        atomicAdd(&dst->errors, errors);
    }
}

}  // namespace

template <bool kVolumes, bool kTextures>
__device__ __forceinline__ void renderChunksBody(const RenderArgs& a) {
    const unsigned full = 0xffffffffu;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t width = a.scene.config.width, height = a.scene.config.height;
    const unsigned long long perChunk = 64ull * a.samplesPerChunk;
    unsigned long long trace = 0, nee = 0, bsdf = 0, held = 0, samples = 0, errors = 0;
    for (;;) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(a.claimed, 32ull);
        base = __shfl_sync(full, base, 0);
        if (base >= a.itemCount) break;
        const unsigned long long item = base + lane;
        uint32_t pixel = ~0u, index = 0;
        if (item < a.itemCount) {
            const unsigned long long chunkIndex = item / perChunk;
            const uint32_t offset = uint32_t(item - chunkIndex * perChunk);
            const uint32_t position = offset / a.samplesPerChunk, s = offset % a.samplesPerChunk;
            const x2_chunk chunk = a.chunks[chunkIndex];
            if (s < chunk.count) {
                pixel = tilePixel(chunk.tile, position, width, height);
                index = chunk.first + s;
            }
        }
        SampleOut o;
        o.status = X2_SKIP;
        o.rgb[0] = o.rgb[1] = o.rgb[2] = o.alpha = 0.0f;
        if (pixel != ~0u) {
            integrate<kVolumes, kTextures>(a.scene, pixel, index, o);
            trace += o.trace;
            nee += o.nee;
            bsdf += o.bsdf;
            held += o.held;
            if (o.status == X2_DONE) ++samples;
            else if (o.status != X2_SKIP) ++errors;
        }
        // Film: one segmented reduction over the warp's lanes that finished a sample of the same pixel.
        const bool done = pixel != ~0u && o.status == X2_DONE;
        const uint32_t key = done ? pixel : ~0u;
        const uint32_t peers = __match_any_sync(full, key);
        double v0 = done ? double(o.rgb[0]) : 0.0, v1 = done ? double(o.rgb[1]) : 0.0, v2 = done ? double(o.rgb[2]) : 0.0,
               v3 = done ? double(o.alpha) : 0.0;
        uint32_t cnt = done ? 1u : 0u;
        const bool isOdd = done && (index & 1u) && a.odd;
        double w0 = isOdd ? v0 : 0.0, w1 = isOdd ? v1 : 0.0, w2 = isOdd ? v2 : 0.0, w3 = isOdd ? v3 : 0.0;
        const bool anyOdd = __any_sync(full, isOdd);
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const double t0 = __shfl_down_sync(full, v0, off), t1 = __shfl_down_sync(full, v1, off);
            const double t2 = __shfl_down_sync(full, v2, off), t3 = __shfl_down_sync(full, v3, off);
            const uint32_t tc = __shfl_down_sync(full, cnt, off);
            const bool same = lane + off < 32 && ((peers >> (lane + off)) & 1u);
            if (same) {
                v0 += t0;
                v1 += t1;
                v2 += t2;
                v3 += t3;
                cnt += tc;
            }
            if (anyOdd) {
                const double u0 = __shfl_down_sync(full, w0, off), u1 = __shfl_down_sync(full, w1, off);
                const double u2 = __shfl_down_sync(full, w2, off), u3 = __shfl_down_sync(full, w3, off);
                if (same) {
                    w0 += u0;
                    w1 += u1;
                    w2 += u2;
                    w3 += u3;
                }
            }
        }
        if (done && lane == uint32_t(__ffs(peers) - 1)) {
            double* s = a.sums + 4ull * key;
            atomicAdd(s, v0);
            atomicAdd(s + 1, v1);
            atomicAdd(s + 2, v2);
            atomicAdd(s + 3, v3);
            atomicAdd(a.counts + key, cnt);
            if (a.odd && (w0 != 0.0 || w1 != 0.0 || w2 != 0.0 || w3 != 0.0)) {
                double* d = a.odd + 4ull * key;
                atomicAdd(d, w0);
                atomicAdd(d + 1, w1);
                atomicAdd(d + 2, w2);
                atomicAdd(d + 3, w3);
            }
        }
    }
    addCounters(a.counters, trace, nee, bsdf, held, samples, errors);
}
__global__ void __launch_bounds__(kRenderBlock) renderChunks(RenderArgs a) { renderChunksBody<false, false>(a); }
__global__ void __launch_bounds__(kRenderBlock) renderChunksTextured(RenderArgs a) { renderChunksBody<false, true>(a); }
__global__ void __launch_bounds__(kRenderBlock) renderChunksVolumes(RenderArgs a) { renderChunksBody<true, true>(a); }

// The per-sample API: integrate() for n (pixel, index) pairs.
template <bool kVolumes, bool kTextures>
__device__ __forceinline__ void integratePairsBody(const SceneView& s, const uint32_t* __restrict__ pairs, unsigned long long n,
                                                   double* __restrict__ rgba, uint32_t* __restrict__ status, Counters* counters) {
    unsigned long long trace = 0, nee = 0, bsdf = 0, held = 0, samples = 0, errors = 0;
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    const unsigned long long first = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
    // Every lane of a warp runs the same number of rounds, so the counters' shuffles below see a full warp.
    const unsigned long long rounds = (n + stride - 1) / stride;
    for (unsigned long long r = 0; r < rounds; ++r) {
        const unsigned long long i = first + r * stride;
        if (i >= n) continue;
        SampleOut o;
        integrate<kVolumes, kTextures>(s, pairs[2 * i], pairs[2 * i + 1], o);
        rgba[4 * i] = double(o.rgb[0]);
        rgba[4 * i + 1] = double(o.rgb[1]);
        rgba[4 * i + 2] = double(o.rgb[2]);
        rgba[4 * i + 3] = double(o.alpha);
        status[i] = o.status;
        trace += o.trace;
        nee += o.nee;
        bsdf += o.bsdf;
        held += o.held;
        if (o.status == X2_DONE) ++samples;
        else errors += o.status == X2_SKIP ? 0 : 1;
    }
    addCounters(counters, trace, nee, bsdf, held, samples, errors);
}
__global__ void __launch_bounds__(kRenderBlock) integratePairs(SceneView s, const uint32_t* __restrict__ pairs, unsigned long long n,
                                                               double* __restrict__ rgba, uint32_t* __restrict__ status, Counters* counters) {
    integratePairsBody<false, false>(s, pairs, n, rgba, status, counters);
}
__global__ void __launch_bounds__(kRenderBlock) integratePairsTextured(SceneView s, const uint32_t* __restrict__ pairs, unsigned long long n,
                                                                       double* __restrict__ rgba, uint32_t* __restrict__ status,
                                                                       Counters* counters) {
    integratePairsBody<false, true>(s, pairs, n, rgba, status, counters);
}
__global__ void __launch_bounds__(kRenderBlock) integratePairsVolumes(SceneView s, const uint32_t* __restrict__ pairs, unsigned long long n,
                                                                      double* __restrict__ rgba, uint32_t* __restrict__ status,
                                                                      Counters* counters) {
    integratePairsBody<true, true>(s, pairs, n, rgba, status, counters);
}

// Closest hit and occlusion for n rays (8 floats each: origin, direction, near, far).
__global__ void traceRays(SceneView s, const float* __restrict__ rays, unsigned long long n, uint32_t* __restrict__ tri, float* __restrict__ t,
                          uint32_t* __restrict__ occluded) {
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const float* r = rays + 8 * i;
        const RayQ q = makeRay(s.bvh, r[0], r[1], r[2], r[3], r[4], r[5]);
        float th;
        uint32_t leaf;
        const uint32_t id = traceClosest<false>(s.bvh, q, r[6], r[7], th, &leaf, s.overflow, nullptr);
        if (tri) tri[i] = id;
        if (t) t[i] = id == ~0u ? 0.0f : th;
        if (occluded) occluded[i] = traceAny<false>(s.bvh, q, r[6], r[7], s.overflow, nullptr) ? 1u : 0u;
    }
}

// sample::samplingWord for n identities.
__global__ void sampleWords(const x2_identity* __restrict__ ids, const uint32_t* __restrict__ dims, unsigned long long n, uint32_t policy,
                            uint32_t* __restrict__ out) {
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const x2_identity x = ids[i];
        const Identity id{x.pixel, x.index, x.stream, x.branch};
        const uint32_t d = dims[i];
        if (d >= 16 && d <= 19) {  // the BSDF and light pairs, as the integrator draws them
            uint32_t a, b;
            samplingWordPair(id, d & ~1u, policy, a, b);
            out[i] = d & 1u ? b : a;
        } else {
            out[i] = samplingWord(id, d, policy);
        }
    }
}

// The audit (async_render.h:1010-1040): the first pixel whose count differs from its expected count.
__global__ void auditCounts(const uint32_t* __restrict__ counts, const uint32_t* __restrict__ expected, uint32_t spp, uint32_t pixels,
                            unsigned long long* firstBad) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= pixels) return;
    const uint32_t want = expected ? expected[i] : spp;
    if (counts[i] != want) atomicMin(firstBad, (unsigned long long)i);
}

}  // namespace x2

#ifdef X2_DIAG
// The diagnostic build's switches for this file's kernels (the per-sample API, x2_integrate): mathfn.cuh's mode bits
// and the call record buffer, set on the current device.
extern "C" int x2_diag_set(int mode, void* d_calls, uint32_t capacity) {
    const uint32_t zero = 0;
    x2::mf::DiagCall* calls = static_cast<x2::mf::DiagCall*>(d_calls);
    if (cudaMemcpyToSymbol(x2::mf::g_mode, &mode, sizeof(int)) != cudaSuccess ||
        cudaMemcpyToSymbol(x2::mf::g_calls, &calls, sizeof(calls)) != cudaSuccess ||
        cudaMemcpyToSymbol(x2::mf::g_cap, &capacity, sizeof(uint32_t)) != cudaSuccess ||
        cudaMemcpyToSymbol(x2::mf::g_count, &zero, sizeof(uint32_t)) != cudaSuccess)
        return X2_ECUDA;
    return X2_OK;
}
extern "C" int x2_diag_count(uint32_t* count) {
    return cudaMemcpyFromSymbol(count, x2::mf::g_count, sizeof(uint32_t)) == cudaSuccess ? X2_OK : X2_ECUDA;
}
#endif
