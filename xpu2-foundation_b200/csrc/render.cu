// The plain megakernel and the small kernels around it.
//
// An item of a launch is a (chunk, tile position, sample) triple laid out sample-minor, so consecutive items are
// consecutive samples of one pixel: a warp's camera rays are coherent and its film update is one set of FP64 atomics a
// pixel (warp-aggregated atomics) instead of one a sample. The film is the reference's: FP64 sums (rgb + alpha), FP64
// odd-index sums (adaptive frames), U32 counts (async_gpu.cu:320-364).
//
// renderSteps (surface scenes): a bounce at a time, a lane taking the next item as soon as its sample is done, rays
// walked a node a step across the warp (below). renderChunks (volumes, counting launches): persistent warps claim 32
// items at a time (one atomic a warp) and each lane runs its sample's whole path (integrate).
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

// Work item `item` of a launch (item < itemCount): its pixel and sample index, or pixel ~0u when it is no sample (past
// its chunk's count, or outside the frame).
__device__ __forceinline__ void itemSample(const RenderArgs& a, unsigned long long item, uint32_t& pixel, uint32_t& index) {
    const unsigned long long perChunk = 64ull * a.samplesPerChunk;
    const unsigned long long chunkIndex = item / perChunk;
    const uint32_t offset = uint32_t(item - chunkIndex * perChunk);
    const uint32_t position = offset / a.samplesPerChunk, s = offset % a.samplesPerChunk;
    const x2_chunk chunk = a.chunks[chunkIndex];
    pixel = ~0u;
    index = 0;
    if (s < chunk.count) {
        pixel = tilePixel(chunk.tile, position, a.scene.config.width, a.scene.config.height);
        index = chunk.first + s;
    }
}

// The film update of a warp step: the lanes that finished a sample of the same pixel are summed by the lowest of them
// (its peers' values added in lane order, whichever lanes they are), which then makes one set of FP64 atomics for the
// pixel. Every lane of the warp calls it; done: the lane finished a sample this step.
__device__ __forceinline__ void warpFilm(const RenderArgs& a, bool done, uint32_t pixel, uint32_t index, float r, float g, float b,
                                         float al) {
    const unsigned full = 0xffffffffu;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t key = done ? pixel : ~0u;
    const uint32_t peers = __match_any_sync(full, key);
    const bool leader = done && lane == uint32_t(__ffs(peers) - 1);
    const bool isOdd = done && (index & 1u) && a.odd;
    const double v0 = done ? double(r) : 0.0, v1 = done ? double(g) : 0.0, v2 = done ? double(b) : 0.0, v3 = done ? double(al) : 0.0;
    double s0 = v0, s1 = v1, s2 = v2, s3 = v3;
    double w0 = isOdd ? v0 : 0.0, w1 = isOdd ? v1 : 0.0, w2 = isOdd ? v2 : 0.0, w3 = isOdd ? v3 : 0.0;
    const double o0 = w0, o1 = w1, o2 = w2, o3 = w3;
    const bool anyOdd = __any_sync(full, isOdd);
    uint32_t rest = leader ? peers & ~(1u << lane) : 0u;
    const uint32_t cnt = leader ? uint32_t(__popc(peers)) : 0u;
    while (__any_sync(full, rest != 0)) {
        const int src = rest ? __ffs(rest) - 1 : int(lane);
        const double t0 = __shfl_sync(full, v0, src), t1 = __shfl_sync(full, v1, src);
        const double t2 = __shfl_sync(full, v2, src), t3 = __shfl_sync(full, v3, src);
        double u0 = 0.0, u1 = 0.0, u2 = 0.0, u3 = 0.0;
        if (anyOdd) {
            u0 = __shfl_sync(full, o0, src);
            u1 = __shfl_sync(full, o1, src);
            u2 = __shfl_sync(full, o2, src);
            u3 = __shfl_sync(full, o3, src);
        }
        if (rest) {
            s0 += t0;
            s1 += t1;
            s2 += t2;
            s3 += t3;
            w0 += u0;
            w1 += u1;
            w2 += u2;
            w3 += u3;
            rest &= rest - 1;
        }
    }
    if (leader) {
        double* s = a.sums + 4ull * key;
        atomicAdd(s, s0);
        atomicAdd(s + 1, s1);
        atomicAdd(s + 2, s2);
        atomicAdd(s + 3, s3);
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

}  // namespace

template <bool kVolumes, bool kTextures>
__device__ __forceinline__ void renderChunksBody(const RenderArgs& a) {
    const unsigned full = 0xffffffffu;
    const uint32_t lane = threadIdx.x & 31u;
    unsigned long long trace = 0, nee = 0, bsdf = 0, held = 0, samples = 0, errors = 0;
    for (;;) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(a.claimed, 32ull);
        base = __shfl_sync(full, base, 0);
        if (base >= a.itemCount) break;
        const unsigned long long item = base + lane;
        uint32_t pixel = ~0u, index = 0;
        if (item < a.itemCount) itemSample(a, item, pixel, index);
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
        warpFilm(a, pixel != ~0u && o.status == X2_DONE, pixel, index, o.rgb[0], o.rgb[1], o.rgb[2], o.alpha);
    }
    addCounters(a.counters, trace, nee, bsdf, held, samples, errors);
}
__global__ void __launch_bounds__(kRenderBlock) renderChunks(RenderArgs a) { renderChunksBody<false, false>(a); }
__global__ void __launch_bounds__(kRenderBlock) renderChunksTextured(RenderArgs a) { renderChunksBody<false, true>(a); }
__global__ void __launch_bounds__(kRenderBlock) renderChunksVolumes(RenderArgs a) { renderChunksBody<true, true>(a); }

// renderSteps: the plain megakernel for surface scenes, a bounce at a time. A lane holds one sample's path (its pending
// rays on a local stack, its radiance) and takes the launch's next item as soon as the sample is done, so a warp never
// waits for its longest path (path regeneration). A warp step is one vertex of every live lane's path: the closest hit
// of its next pending ray, walked a node a step together with the warp's other rays (walkStep); the vertex shaded
// (afterTrace, shadeVertex) with its shadow rays written to a list of the lane's own; then the lists walked together,
// a lane whose ray is done starting its next one at once; then the unoccluded rays' contributions added in the list's
// order. That is the order in which integrate (one thread a sample, shadow rays traced as they come) adds them, and
// the steps visit the nodes and test the triangles traceClosest / traceAny do, so a sample's radiance is the same bit
// for bit. Scenes with volumes, vertices with more than kStepRecords shadow rays and counting launches use renderChunks.
struct StepSink {
    ShadowReq* reqs;
    uint32_t& n;
    Pending* stack;
    uint32_t& size;
    unsigned long long &nee, &bsdf, &heldRays;
    bool full;  // a shadow ray beyond kStepRecords (the launch checks the scene's bound, so never set)
    __device__ void shadow(const ShadowReq& q, bool fromBsdf) {
        if (fromBsdf) ++bsdf;
        else ++nee;
        if (n < kStepRecords) reqs[n++] = q;
        else full = true;
    }
    __device__ void held() { ++heldRays; }
    __device__ void vertex(uint32_t, const Bsdf&, V3, const TexHit*) {}
    __device__ uint32_t top(uint32_t) const { return size; }
    __device__ void push(const Pending& p) { stack[size++] = p; }
};

template <bool kTextures>
__device__ __forceinline__ void renderStepsBody(const RenderArgs& a) {
    __shared__ uint2 shortStacks[kShortStack * kRenderBlock];
    const unsigned full = 0xffffffffu;
    const uint32_t lane = threadIdx.x & 31u;
    const SceneView& s = a.scene;
    const Bvh8 bvh = s.bvh;
    uint32_t* overflow = s.overflow;
    Walk<kShortStack> walk;
    uint2 deep[kStack - kShortStack];
    walk.shortStack = shortStacks + threadIdx.x;
    walk.nodes = walk.tris = 0;
    Pending stack[kMaxPending];
    ShadowReq reqs[kStepRecords];
    uint32_t size = 0, n = 0, pixel = 0, index = 0;
    uint32_t hitTri = ~0u, hitLeaf = 0;  // the closest hit of the pending stack's top ray, once walked
    float hitT = 0.0f;
    V3 cameraPosition{0, 0, 0}, radiance{0, 0, 0};
    float alpha = 0.0f;
    RayQ r;
    unsigned long long trace = 0, nee = 0, bsdf = 0, held = 0, samples = 0, errors = 0;
    bool live = false, drained = false;
    for (;;) {
        // Idle lanes take the next items (one atomic a warp); an item that is no sample leaves its lane idle.
        const uint32_t idle = __ballot_sync(full, !live);
        if (idle && !drained) {
            const uint32_t leader = __ffs(idle) - 1, want = __popc(idle);
            unsigned long long base = 0;
            if (lane == leader) base = atomicAdd(a.claimed, (unsigned long long)want);
            base = __shfl_sync(full, base, leader);
            drained = base + want >= a.itemCount;
            if (!live) {
                const unsigned long long item = base + __popc(idle & ((1u << lane) - 1u));
                if (item < a.itemCount) {
                    itemSample(a, item, pixel, index);
                    if (pixel != ~0u) {
                        CameraRay camera;
                        if (cameraRay(s, pixel, index, camera)) {
                            cameraPending(camera, stack[0]);
                            size = 1;
                            n = 0;
                            cameraPosition = camera.origin;
                            radiance = V3{0, 0, 0};
                            alpha = 0.0f;
                            live = true;
                        } else {
                            ++errors;
                        }
                    }
                }
            }
        }
        if (!__any_sync(full, live)) {
            if (drained) break;
            continue;
        }
        // Each live lane's rays, walked a step at a time with the warp's others: the last vertex's shadow rays in
        // order, then the closest hit of the next pending ray; a lane whose ray is done starts its next at once.
        uint32_t j = 0, vis = 0;
        bool tracing = live && (n > 0 || size > 0), any = n > 0;
        if (tracing) {
            const V3 o = any ? reqs[0].origin : stack[size - 1].origin, d = any ? reqs[0].dir : stack[size - 1].dir;
            r = makeRay(bvh, o.x, o.y, o.z, d.x, d.y, d.z);
            if (any) walkStart<true, kShortStack>(walk, r, reqs[0].near, reqs[0].far);
            else walkStart<false, kShortStack>(walk, r, stack[size - 1].nearT, stack[size - 1].farT);
        }
        for (;;) {
            const uint32_t lanes = __ballot_sync(full, tracing);
            if (!lanes) break;
            if (tracing && walkStepOverlapKind<kShortStack>(bvh, r, walk, deep, overflow, lanes, any)) {
                if (any) {
                    if (!walk.best) vis |= 1u << j;
                    ++j;
                } else {
                    hitTri = walk.best;
                    hitLeaf = walk.bestLeaf;
                    hitT = walk.tmax;
                }
                tracing = false;
                if (any && j < n) {
                    const ShadowReq& q = reqs[j];
                    r = makeRay(bvh, q.origin.x, q.origin.y, q.origin.z, q.dir.x, q.dir.y, q.dir.z);
                    walkStart<true, kShortStack>(walk, r, q.near, q.far);
                    tracing = true;
                } else if (any && size > 0) {
                    const Pending& next = stack[size - 1];
                    r = makeRay(bvh, next.origin.x, next.origin.y, next.origin.z, next.dir.x, next.dir.y, next.dir.z);
                    walkStart<false, kShortStack>(walk, r, next.nearT, next.farT);
                    any = false;
                    tracing = true;
                }
            }
        }
        // The shadow rays' contributions in the list's order, then the next vertex: the hit rebuilt as trace() does,
        // afterTrace and shadeVertex, its shadow rays to the list.
        for (uint32_t k = 0; k < n; ++k)
            if ((vis >> k) & 1u) radiance = add(radiance, reqs[k].contribution);
        n = 0;
        if (live && size > 0) {
            Pending pv = stack[--size];
            const uint32_t top = size;
            ++trace;
            Hit hit;
            hit.geom = ~0u;
            hit.prim = 0;
            hit.t = hit.u = hit.v = 0;
            hit.normal = hit.origin = hit.below = hit.point = V3{0, 0, 0};
            V3 va{0, 0, 0}, vb{0, 0, 0}, vc{0, 0, 0};
            if (hitTri != ~0u) {
                const float4* tp = reinterpret_cast<const float4*>(bvh.tris + hitLeaf);
                const float4 A = __ldg(tp), B = __ldg(tp + 1), Cc = __ldg(tp + 2);
                va = V3{A.x, A.y, A.z};
                vb = V3{B.x, B.y, B.z};
                vc = V3{Cc.x, Cc.y, Cc.z};
                hit.geom = __ldg(s.triMesh + hitTri);
                hit.prim = hitTri - __ldg(s.meshFirst + hit.geom);
                hit.t = hitT;
                if (!geometryHit(hit, pv.origin, pv.dir, va, vb, vc)) hit.normal = V3{0, 0, 0};
            }
            const Identity root{pixel, U64(index), U64(s.config.seed), 0};
            afterTrace<false>(s, root, pv, hit, cameraPosition, radiance, alpha);
            if (hit.geom != ~0u) {
                StepSink sink{reqs, n, stack, size, nee, bsdf, held, false};
                if (!shadeVertex<false, kTextures>(s, root, pixel, index, pv, hit, va, vb, vc, top, radiance, alpha, sink) || sink.full) {
                    ++errors;
                    live = false;
                    n = 0;
                }
            }
        }
        const bool done = live && size == 0 && n == 0;
        if (__any_sync(full, done)) warpFilm(a, done, pixel, index, radiance.x, radiance.y, radiance.z, alpha);
        if (done) {
            ++samples;
            live = false;
        }
    }
    addCounters(a.counters, trace, nee, bsdf, held, samples, errors);
}
template <int kMinBlocks>
__global__ void __launch_bounds__(kRenderBlock, kMinBlocks) renderSteps(RenderArgs a) { renderStepsBody<false>(a); }
template <int kMinBlocks>
__global__ void __launch_bounds__(kRenderBlock, kMinBlocks) renderStepsTextured(RenderArgs a) { renderStepsBody<true>(a); }
template __global__ void renderSteps<4>(RenderArgs);
template __global__ void renderStepsTextured<4>(RenderArgs);

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
