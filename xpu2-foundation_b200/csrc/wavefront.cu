// The wavefront form of the path tracer: the same samples as the plain megakernel, split into small kernels that each
// run one kind of work over compacted queues, with path regeneration.
//
// Path state lives in HBM, structure of arrays, one slot a path in flight (P slots). One iteration:
//   logic   each slot: add the previous vertex's unoccluded shadow-ray contributions in the reference's order
//           (light samples in light order, then the BSDF sample's), write a finished sample to the per-item output,
//           claim a new sample for an empty slot (regeneration: a camera ray), and append every slot with a ray to
//           trace to the extend queue (warp-aggregated atomics);
//   extend  closest hit of every queued ray (traverse.cuh);
//   sort    the extended paths into per-lobe queues by their hit's material (GGX, Lambert, none or missed);
//   shade   each queued path's vertex, the queues in that order (integrator.cuh shadeVertex): its shadow rays go to fixed per-path record slots
//           and, by one warp-aggregated reservation a warp, to the shadow queue; its child becomes the slot's ray;
//   shadow  any hit of every queued shadow ray, a visibility flag each.
// Iterations are captured once as a CUDA graph and replayed until every item is done. The per-item output (rgb,
// alpha, status) is then summed into the film in sample order by filmReduce, so the film does not depend on the
// order paths finish in.
#include "credits.cuh"
#include "wavefront.h"

namespace x2 {

enum : uint32_t { kEmpty = 0, kTrace = 1, kDone = 2, kError = 3 };

// This translation unit's copy of the Sobol direction table (sampler.cuh): filled at x2_open like render.cu's.
cudaError_t uploadSobolWavefront(const uint32_t directions[17][32]) {
    return cudaMemcpyToSymbol(c_sobol, directions, sizeof(uint32_t) * 17 * 32);
}

namespace {

__device__ __forceinline__ uint32_t tilePixelW(uint32_t tile, uint32_t position, uint32_t width, uint32_t height) {
    const uint32_t tilesX = (width + 7) / 8;
    const uint32_t x = (tile % tilesX) * 8 + position % 8;
    const uint32_t y = (tile / tilesX) * 8 + position / 8;
    return x < width && y < height ? y * width + x : ~0u;
}

// Warp-aggregated append: each lane with `want` items gets a contiguous range; one atomic a warp. Every lane of the
// warp must call it (the callers' loops keep their warps whole).
__device__ __forceinline__ uint32_t warpReserve(uint32_t* counter, uint32_t want) {
    const unsigned full = 0xffffffffu;
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t incl = want;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const uint32_t v = __shfl_up_sync(full, incl, off);
        if (lane >= uint32_t(off)) incl += v;
    }
    const uint32_t total = __shfl_sync(full, incl, 31);
    uint32_t base = 0;
    if (lane == 31 && total) base = atomicAdd(counter, total);
    base = __shfl_sync(full, base, 31);
    return base + incl - want;
}

__device__ __forceinline__ void warpAddCounters(Counters* dst, unsigned long long trace, unsigned long long nee, unsigned long long bsdf,
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
        if (trace) atomicAdd(&dst->trace, trace);
        if (nee) atomicAdd(&dst->nee, nee);
        if (bsdf) atomicAdd(&dst->bsdf, bsdf);
        if (held) atomicAdd(&dst->held, held);
        if (samples) atomicAdd(&dst->samples, samples);
        if (errors) atomicAdd(&dst->errors, errors);
    }
}

// The adjoint's credits into a block's shared partials (x2_adjoint's wavefront form).
constexpr uint32_t kVertLambert = 0u, kVertGgx = 1u, kVertNone = 3u;  // a vertex record's kind (material bits 30-31)

__device__ __forceinline__ void creditLightTo(float* partial, const Layout& at, const SceneView& s, float4 d, V3 c, uint32_t j) {
    if (j == ~0u) return;
    const x2_light& L = s.lights[j];
    const float w[3] = {d.x * c.x, d.y * c.y, d.z * c.z};
    for (int k = 0; k < 3; ++k)
        if (L.radiance[k] != 0.0f && w[k] != 0.0f) atomicAdd(partial + at.radiance(j) + k, w[k] / L.radiance[k]);
}
__device__ __forceinline__ void creditRoughnessTo(float* partial, const Layout& at, uint32_t m, float4 d, V3 c, float g) {
    const float v = (d.x * c.x + d.y * c.y + d.z * c.z) * g;
    if (v != 0.0f && finitef(v)) atomicAdd(partial + at.roughness(m), v);
}
// A block's partials: zeroed at the kernel's start, added to the block's gradient row at its end.
__device__ __forceinline__ void partialsBegin(float* partial, const Layout& at) {
    for (uint32_t i = threadIdx.x; i < at.count(); i += blockDim.x) partial[i] = 0.0f;
    __syncthreads();
}
__device__ __forceinline__ void partialsEnd(float* partial, const Layout& at, const AdjointWave& adj) {
    __syncthreads();
    float* row = adj.rows + size_t(blockIdx.x % adj.rowCount) * at.count();
    for (uint32_t i = threadIdx.x; i < at.count(); i += blockDim.x)
        if (partial[i] != 0.0f) atomicAdd(row + i, partial[i]);
}

__device__ __forceinline__ uint32_t packDepths(const Pending& p) {
    return (p.depth & 0xffu) | ((p.nonMirror & 0xffu) << 8) | ((p.diffuse & 0xffu) << 16) | ((p.glossy & 0xffu) << 24);
}

__device__ __forceinline__ void loadPending(const WaveState& w, uint32_t p, Pending& pv) {
    const float4 r0 = w.ray0[p], r1 = w.ray1[p], T = w.T[p], h = w.held[p];
    const uint4 m = w.meta[p];
    pv.origin = V3{r0.x, r0.y, r0.z};
    pv.nearT = r0.w;
    pv.dir = V3{r1.x, r1.y, r1.z};
    pv.farT = r1.w;
    pv.T = V3{T.x, T.y, T.z};
    pv.heldFar = T.w;
    pv.held = V3{h.x, h.y, h.z};
    pv.heldLight = __float_as_uint(h.w);
    pv.depth = m.z & 0xffu;
    pv.nonMirror = (m.z >> 8) & 0xffu;
    pv.diffuse = (m.z >> 16) & 0xffu;
    pv.glossy = m.z >> 24;
    pv.mirror = m.w & 0xffu;
    pv.lobeType = (m.w >> 8) & 0xffu;
    pv.volumeDepth = (m.w >> 16) & 0xffu;
    const uint2 b = w.branch[p];
    pv.branch = (U64(b.y) << 32) | b.x;
}

// meta.w: mirror depth (bits 0..7), lobe type (8..15), volume depth (16..23), the path's request in a batch (24..31).
__device__ __forceinline__ void storePending(const WaveState& w, uint32_t p, const Pending& c, uint32_t pixel, uint32_t index,
                                             uint32_t request = 0) {
    w.ray0[p] = make_float4(c.origin.x, c.origin.y, c.origin.z, c.nearT);
    w.ray1[p] = make_float4(c.dir.x, c.dir.y, c.dir.z, c.farT);
    w.T[p] = make_float4(c.T.x, c.T.y, c.T.z, c.heldFar);
    w.held[p] = make_float4(c.held.x, c.held.y, c.held.z, __uint_as_float(c.heldLight));
    w.meta[p] = make_uint4(pixel, index, packDepths(c),
                           (c.mirror & 0xffu) | ((c.lobeType & 0xffu) << 8) | ((c.volumeDepth & 0xffu) << 16) | (request << 24));
    w.branch[p] = make_uint2(uint32_t(c.branch), uint32_t(c.branch >> 32));
}

}  // namespace

// The request a path slot's sample belongs to (batches; 0 otherwise) and that request's scene.
__device__ __forceinline__ uint32_t requestOf(const WaveState& w, uint32_t p) { return w.meta[p].w >> 24; }
template <bool kBatch>
__device__ __forceinline__ const SceneView& sceneOf(const WaveArgs& a, uint32_t request) {
    return kBatch ? a.scenes[request] : a.scene;
}

// A work item's chunk. One launch: chunks of 64 x samplesPerChunk items. A batch: chunks of 64 x count items each
// (each request its own samples a pixel), found by binary search of the chunks' first items.
template <bool kBatch>
__device__ __forceinline__ uint32_t chunkOfItem(const WaveArgs& a, unsigned long long item, unsigned long long& first, uint32_t& perPixel) {
    if (!kBatch) {
        const unsigned long long perChunk = 64ull * a.samplesPerChunk;
        const uint32_t c = uint32_t(item / perChunk);
        first = c * perChunk;
        perPixel = a.samplesPerChunk;
        return c;
    }
    uint32_t lo = 0, hi = a.chunkCount;  // chunkItems[lo] <= item < chunkItems[hi]
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (a.chunkItems[mid] <= item) lo = mid;
        else hi = mid;
    }
    first = a.chunkItems[lo];
    perPixel = uint32_t((a.chunkItems[lo + 1] - first) / 64ull);
    return lo;
}

// ---- logic ----
template <bool kBatch, bool kAdjoint = false>
__device__ __forceinline__ void logicBody(const WaveArgs& a) {
    const WaveState& w = a.w;
    unsigned long long samples = 0, errors = 0;
    extern __shared__ float partial[];  // the adjoint's block partials
    const Layout at{a.adj.materials, a.adj.lights};
    if (kAdjoint) partialsBegin(partial, at);
    const unsigned long long itemCount = a.liveChunks ? (unsigned long long)(*a.liveChunks) * 64ull * a.samplesPerChunk : a.itemCount;
    for (uint32_t base = blockIdx.x * blockDim.x; base < a.paths; base += gridDim.x * blockDim.x) {
        const uint32_t p = base + threadIdx.x;
        uint32_t st = p < a.paths ? w.state[p] : kTrace + 100;  // out of range: no work, no claim
        if (p < a.paths) {
            // The previous vertex's shadow rays, in the order they were made.
            const uint32_t n = w.ncount[p];
            if (n && !kAdjoint) {
                float4 rad = w.rad[p];
                const size_t first = size_t(p) * a.recordsPerPath;
                for (uint32_t k = 0; k < n; ++k)
                    if (w.svis[first + k]) {
                        const float4 c = w.scontrib[first + k];
                        rad.x = rad.x + c.x;
                        rad.y = rad.y + c.y;
                        rad.z = rad.z + c.z;
                    }
                w.rad[p] = rad;
                w.ncount[p] = 0;
            } else if (n && kAdjoint) {
                // The same, crediting each unoccluded record to its light and, made by a GGX vertex's light sample, to
                // that vertex's roughness with its own factor; a GGX vertex's suffix then starts after its light
                // samples (its records come first, its BSDF sample's last).
                float4 rad = w.rad[p];
                const size_t first = size_t(p) * a.recordsPerPath;
                const size_t vj = size_t(p) * a.adj.vertsPerPath + (a.adj.vcount[p] - 1);
                const uint4 v = a.adj.vert[vj];
                const bool ggx = (v.x >> 30) == kVertGgx;
                const float4 d = a.adj.delta[p];
                float4 afterLights = make_float4(__uint_as_float(v.y), __uint_as_float(v.z), __uint_as_float(v.w), 0.0f);
                for (uint32_t k = 0; k < n; ++k) {
                    const uint2 aux = a.adj.aux[first + k];
                    if (w.svis[first + k]) {
                        const float4 c = w.scontrib[first + k];
                        rad.x = rad.x + c.x;
                        rad.y = rad.y + c.y;
                        rad.z = rad.z + c.z;
                        creditLightTo(partial, at, a.scene, d, V3{c.x, c.y, c.z}, aux.x & 0x7fffffffu);
                        if (ggx && !(aux.x >> 31)) creditRoughnessTo(partial, at, v.x & 0x3fffffffu, d, V3{c.x, c.y, c.z}, __uint_as_float(aux.y));
                    }
                    if (!(aux.x >> 31)) afterLights = rad;
                }
                if (ggx) a.adj.vert[vj] = make_uint4(v.x, __float_as_uint(afterLights.x), __float_as_uint(afterLights.y), __float_as_uint(afterLights.z));
                w.rad[p] = rad;
                w.ncount[p] = 0;
            }
            if (kAdjoint && st == kDone) {
                // The path's end: each vertex credited once with what the path gathered after it acted.
                const float4 total = w.rad[p], d = a.adj.delta[p];
                const uint32_t nv = a.adj.vcount[p];
                for (uint32_t k = 0; k < nv; ++k) {
                    const size_t vk = size_t(p) * a.adj.vertsPerPath + k;
                    const uint4 v = a.adj.vert[vk];
                    const uint32_t kind = v.x >> 30, m = v.x & 0x3fffffffu;
                    if (kind == kVertNone) continue;
                    const V3 after{total.x - __uint_as_float(v.y), total.y - __uint_as_float(v.z), total.z - __uint_as_float(v.w)};
                    const float4 sc = a.adj.scale[vk];
                    if (kind == kVertGgx) {
                        creditRoughnessTo(partial, at, m, d, after, sc.x);
                        continue;
                    }
                    creditLambert(partial, at, a.scene, m, d, after, V3{sc.x, sc.y, sc.z}, a.adj.tex ? &a.adj.tex[vk] : nullptr, a.adj.texGrad);
                }
            }
            if (st == kDone || st == kError) {
                const unsigned long long item = w.item[p];
                a.out[item] = st == kDone ? w.rad[p] : make_float4(0, 0, 0, 0);
                a.outStatus[item] = st == kDone ? uint8_t(X2_DONE) : uint8_t(X2_ERROR);
                if (st == kDone) ++samples;
                else ++errors;
                st = kEmpty;
                w.state[p] = kEmpty;
            }
        }
        // Regeneration: every empty slot of the warp claims one item, one atomic a warp, in item order.
        const bool wants = st == kEmpty;
        const unsigned full = 0xffffffffu;
        const unsigned want = __ballot_sync(full, wants);
        unsigned long long first = 0;
        if (want) {
            if ((threadIdx.x & 31u) == 0) first = atomicAdd(a.claimed, (unsigned long long)__popc(want));
            first = __shfl_sync(full, first, 0);
        }
        if (wants) {
            const unsigned long long item = first + __popc(want & ((1u << (threadIdx.x & 31u)) - 1u));
            if (item < itemCount) {
                unsigned long long chunkFirst;
                uint32_t perPixel;
                const uint32_t chunkIndex = chunkOfItem<kBatch>(a, item, chunkFirst, perPixel);
                const uint32_t offset = uint32_t(item - chunkFirst);
                const uint32_t position = offset / perPixel, s = offset % perPixel;
                const x2_chunk chunk = a.chunks[chunkIndex];
                const uint32_t request = kBatch ? a.chunkRequest[chunkIndex] : 0u;
                const SceneView& sv = sceneOf<kBatch>(a, request);
                const bool masked = a.chunkMask && !((a.chunkMask[chunkIndex] >> position) & 1ull);
                const uint32_t pixel = s < chunk.count && !masked ? tilePixelW(chunk.tile, position, sv.config.width, sv.config.height) : ~0u;
                if (pixel == ~0u) {
                    a.outStatus[item] = uint8_t(X2_SKIP);  // not a sample of this launch
                } else {
                    const uint32_t index = (a.pixelBase ? a.pixelBase[pixel] : chunk.first) + s;
                    CameraRay camera;
                    if (!cameraRay(sv, pixel, index, camera)) {
                        a.out[item] = make_float4(0, 0, 0, 0);
                        a.outStatus[item] = uint8_t(X2_ERROR);
                        ++errors;
                    } else {
                        Pending p0;
                        cameraPending(camera, p0);
                        storePending(w, p, p0, pixel, index, request);
                        w.rad[p] = make_float4(0, 0, 0, 0);
                        if (kAdjoint) {
                            const float inv = 1.0f / float(chunk.count);
                            a.adj.delta[p] = make_float4(a.adj.dLdI[3ull * pixel] * inv, a.adj.dLdI[3ull * pixel + 1] * inv,
                                                         a.adj.dLdI[3ull * pixel + 2] * inv, 0.0f);
                            a.adj.vcount[p] = 0;
                        }
                        w.item[p] = uint32_t(item);
                        w.state[p] = kTrace;
                        st = kTrace;
                    }
                }
            }
        }
        // The extend queue: every slot with a ray to trace (binned: in the bin of its direction's octant).
        const bool trace = st == kTrace;
        const uint32_t slot = warpReserve(a.extendCount, trace ? 1u : 0u);
        if (!a.extendSlots) {
            if (trace) a.extendQ[slot] = p;
        } else {
            uint32_t octant = kOctants;
            if (trace) {
                const float4 d = w.ray1[p];
                octant = (signbit(d.x) ? 1u : 0u) | (signbit(d.y) ? 2u : 0u) | (signbit(d.z) ? 4u : 0u);
            }
            const unsigned peers = __match_any_sync(full, octant);
            const uint32_t lane = threadIdx.x & 31u, leader = __ffs(peers) - 1;
            uint32_t at = 0;
            if (octant < kOctants && lane == leader) at = atomicAdd(a.extendSlots + octant, uint32_t(__popc(peers)));
            at = __shfl_sync(peers, at, leader);
            if (trace) a.extendQ[size_t(octant) * a.paths + at + __popc(peers & ((1u << lane) - 1u))] = p;
        }
    }
    warpAddCounters(a.counters, 0, 0, 0, 0, samples, errors);
    if (kAdjoint) partialsEnd(partial, at, a.adj);
}

__global__ void __launch_bounds__(kWaveBlock) wfLogic(WaveArgs a) { logicBody<false>(a); }
__global__ void __launch_bounds__(kWaveBlock) wfLogicBatch(WaveArgs a) { logicBody<true>(a); }
__global__ void __launch_bounds__(kWaveBlock) wfLogicAdjoint(WaveArgs a) { logicBody<false, true>(a); }

// ---- extend: closest hits ----
// Persistent traversal over a queue: each lane walks its ray a node a step; a warp fetches the next rays of the queue
// (one atomic a warp) for its idle lanes once `refill` of them are idle, so lanes whose rays end early are not left
// waiting for the warp's longest ray. kAny: shadow records (visibility out), else extend rays (closest hit out).
// A queue in segments (the shadow queue by record): entry i lies in the segment s with start[s] <= i < start[s + 1],
// at queue[s * stride + i - start[s]]. segments 0: a plain queue.
struct QueueSegments {
    const uint32_t* start;  // segments + 1 running totals (shared memory)
    uint32_t segments, stride;
    __device__ __forceinline__ uint32_t at(const uint32_t* __restrict__ queue, uint32_t i) const {
        if (!segments) return queue[i];
        uint32_t s = 0;
        while (s + 1 < segments && start[s + 1] <= i) ++s;
        return queue[size_t(s) * stride + (i - start[s])];
    }
};

// shortStacks: the block's kShortStack x kWaveBlock short traversal stacks (shared memory).
template <bool kAny, bool kStats, bool kBatch, int kShort, bool kOverlap = false>
__device__ __forceinline__ void persistentTrace(const WaveArgs& a, uint32_t n, const uint32_t* __restrict__ queue, uint32_t* next,
                                                uint2* shortStacks, const QueueSegments seg = QueueSegments{nullptr, 0, 0}) {
    const WaveState& w = a.w;
    Bvh8 bvh = a.scene.bvh;  // a batch: the lane's ray's scene, set at each fetch
    uint32_t* overflow = a.scene.overflow;
    const unsigned full = 0xffffffffu;
    const uint32_t lane = threadIdx.x & 31u;
    Walk<kShort> walk;
    uint2 deep[kStack - kShort];
    walk.shortStack = shortStacks + threadIdx.x;
    walk.nodes = walk.tris = 0;
    RayQ r;
    uint32_t k = 0, rays = 0;
    uint32_t steps = 0, liveLanes = 0, nodeSteps = 0, nodeLanes = 0, triSteps = 0, triLanes = 0;  // kStats, lane 0
    bool live = false, drained = false;
    for (;;) {
        const uint32_t idle = __ballot_sync(full, !live);
        if (!drained && __popc(idle) >= a.refill) {
            const uint32_t leader = __ffs(idle) - 1, want = __popc(idle);
            uint32_t base = 0;
            if (lane == leader) base = atomicAdd(next, want);
            base = __shfl_sync(full, base, leader);
            drained = base + want >= n;
            if (!live) {
                const uint32_t i = base + __popc(idle & ((1u << lane) - 1u));
                if (i < n) {
                    k = seg.at(queue, i);
                    if (kBatch) {
                        const SceneView& sv = a.scenes[requestOf(w, kAny ? k / a.recordsPerPath : k)];
                        bvh = sv.bvh;
                        overflow = sv.overflow;
                    }
                    const float4 r0 = kAny ? w.sray0[k] : w.ray0[k], r1 = kAny ? w.sray1[k] : w.ray1[k];
                    r = makeRay(bvh, r0.x, r0.y, r0.z, r1.x, r1.y, r1.z);
                    walkStart<kAny, kShort>(walk, r, r0.w, r1.w);
                    live = true;
                    ++rays;
                }
            }
        }
        if (!__any_sync(full, live)) break;
        const uint32_t liveMask = __ballot_sync(full, live), tris0 = walk.tris, nodes0 = walk.nodes;
        uint32_t nodeMask = 0;
        if (kStats && !kOverlap) nodeMask = __ballot_sync(full, live && !walk.tbits && ((walk.bits & 0xff000000u) || walk.sp));
        if (live && (kOverlap ? walkStepOverlap<kAny, kShort>(bvh, r, walk, deep, overflow, liveMask)
                              : walkStep<kAny, kShort>(bvh, r, walk, deep, overflow, a.triLimit, liveMask))) {
            if (kAny) w.svis[k] = walk.best ? 0 : 1;
            else w.hit[k] = make_uint2(walk.best == ~0u ? ~0u : walk.bestLeaf, __float_as_uint(walk.tmax));
            live = false;
        }
        if (kStats && kOverlap) nodeMask = __ballot_sync(full, walk.nodes != nodes0);
        if (kStats) {
            const uint32_t tested = walk.tris - tris0;
            const uint32_t most = __reduce_max_sync(full, tested), all = __reduce_add_sync(full, tested);
            if (lane == 0) {
                ++steps;
                liveLanes += __popc(liveMask);
                nodeSteps += nodeMask != 0;
                nodeLanes += __popc(nodeMask);
                triSteps += most;
                triLanes += all;
            }
        }
    }
    if (kStats) {
        TraversalStats* st = a.scene.stats + (kAny ? 1 : 0);
        atomicAdd(&st->rays, (unsigned long long)rays);
        atomicAdd(&st->nodes, (unsigned long long)walk.nodes);
        atomicAdd(&st->tris, (unsigned long long)walk.tris);
        if (lane == 0) {
            atomicAdd(&st->steps, (unsigned long long)steps);
            atomicAdd(&st->liveLanes, (unsigned long long)liveLanes);
            atomicAdd(&st->nodeSteps, (unsigned long long)nodeSteps);
            atomicAdd(&st->nodeLanes, (unsigned long long)nodeLanes);
            atomicAdd(&st->triSteps, (unsigned long long)triSteps);
            atomicAdd(&st->triLanes, (unsigned long long)triLanes);
        }
    }
}

template <bool kBatch, int kShort = kShortStack, bool kStats = false, bool kOverlap = false>
__device__ __forceinline__ void extendBody(const WaveArgs& a) {
    __shared__ uint2 shortStacks[kShort > 0 ? kShort * kWaveBlock : 1];
    __shared__ uint32_t start[kOctants + 1];
    QueueSegments seg{start, 0, a.paths};
    const uint32_t n = *a.extendCount;
    if (a.extendSlots) {
        seg.segments = kOctants;
        if (threadIdx.x == 0) {
            uint32_t run = 0;
            for (uint32_t o = 0; o < kOctants; ++o) {
                start[o] = run;
                run += a.extendSlots[o];
            }
            start[kOctants] = run;
        }
        __syncthreads();
    }
    persistentTrace<false, kStats && !kBatch, kBatch, kShort, kOverlap>(a, n, a.extendQ, a.extendNext, shortStacks, seg);
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&a.counters->trace, (unsigned long long)n);
}

// ---- shade ----
// The wavefront's sink: shadow rays to the path's record slots, the child to the slot. kAdjoint: also the vertex
// records the adjoint credits at the path's end and each record's light and own roughness factor.
// A vertex's LightJob in the wave state (kLightJobWords uint4 a slot) and back.
__device__ __forceinline__ void storeLightJob(const WaveState& w, uint32_t p, const LightJob& j) {
    uint4* q = w.lightJob + size_t(p) * kLightJobWords;
    auto f = [](float x) { return __float_as_uint(x); };
    const Lobe& l = j.lobe;
    const uint32_t flags = (j.hasCull ? 1u : 0u) | (j.split ? 2u : 0u) | (j.clampHere ? 4u : 0u) | (j.rr ? 8u : 0u) | (l.kind << 4);
    q[0] = make_uint4(f(j.P.x), f(j.P.y), f(j.P.z), f(j.Ng.x));
    q[1] = make_uint4(f(j.Ng.y), f(j.Ng.z), f(j.wo.x), f(j.wo.y));
    q[2] = make_uint4(f(j.wo.z), f(j.T.x), f(j.T.y), f(j.T.z));
    q[3] = make_uint4(f(j.above.x), f(j.above.y), f(j.above.z), f(j.below.x));
    q[4] = make_uint4(f(j.below.y), f(j.below.z), f(j.cull.x), f(j.cull.y));
    q[5] = make_uint4(f(j.cull.z), f(l.frame.x.x), f(l.frame.x.y), f(l.frame.x.z));
    q[6] = make_uint4(f(l.frame.y.x), f(l.frame.y.y), f(l.frame.y.z), f(l.frame.z.x));
    q[7] = make_uint4(f(l.frame.z.y), f(l.frame.z.z), f(l.albedo.x), f(l.albedo.y));
    q[8] = make_uint4(f(l.albedo.z), f(l.spec.x), f(l.spec.y), f(l.spec.z));
    q[9] = make_uint4(f(l.roughness), uint32_t(j.branch), uint32_t(j.branch >> 32), l.type);
    q[10] = make_uint4(j.pixel, j.index, j.depth | (flags << 16), j.nl | (j.nk << 16));
}
__device__ __forceinline__ LightJob loadLightJob(const WaveState& w, uint32_t p) {
    const uint4* q = w.lightJob + size_t(p) * kLightJobWords;
    uint4 v[kLightJobWords];
#pragma unroll
    for (uint32_t k = 0; k < kLightJobWords; ++k) v[k] = q[k];
    auto f = [](uint32_t x) { return __uint_as_float(x); };
    LightJob j;
    j.P = V3{f(v[0].x), f(v[0].y), f(v[0].z)};
    j.Ng = V3{f(v[0].w), f(v[1].x), f(v[1].y)};
    j.wo = V3{f(v[1].z), f(v[1].w), f(v[2].x)};
    j.T = V3{f(v[2].y), f(v[2].z), f(v[2].w)};
    j.above = V3{f(v[3].x), f(v[3].y), f(v[3].z)};
    j.below = V3{f(v[3].w), f(v[4].x), f(v[4].y)};
    j.cull = V3{f(v[4].z), f(v[4].w), f(v[5].x)};
    j.lobe.frame.x = V3{f(v[5].y), f(v[5].z), f(v[5].w)};
    j.lobe.frame.y = V3{f(v[6].x), f(v[6].y), f(v[6].z)};
    j.lobe.frame.z = V3{f(v[6].w), f(v[7].x), f(v[7].y)};
    j.lobe.albedo = V3{f(v[7].z), f(v[7].w), f(v[8].x)};
    j.lobe.spec = V3{f(v[8].y), f(v[8].z), f(v[8].w)};
    j.lobe.roughness = f(v[9].x);
    j.branch = U64(v[9].y) | (U64(v[9].z) << 32);
    j.lobe.type = v[9].w;
    j.pixel = v[10].x;
    j.index = v[10].y;
    j.depth = v[10].z & 0xffffu;
    const uint32_t flags = v[10].z >> 16;
    j.hasCull = flags & 1u;
    j.split = flags & 2u;
    j.clampHere = flags & 4u;
    j.rr = flags & 8u;
    j.lobe.kind = (flags >> 4) & 1u;
    j.nl = v[10].w & 0xffffu;
    j.nk = v[10].w >> 16;
    return j;
}

// kDefer: the light samples are deferred to the light kernel (sink.lights stores the vertex's job), and the BSDF
// sample's shadow record waits in the slot's last record, which the light kernel moves after the light records.
template <bool kAdjoint = false, bool kDefer = false>
struct WaveSink {
    const WaveState& w;
    uint32_t p, n, recordsPerPath;
    bool pushed;
    Pending child;
    unsigned long long nNee, nBsdf, nHeld;
    // Adjoint only.
    const AdjointWave* adj;
    const SceneView* s;
    const V3* radiance;
    uint32_t depth;
    Lobe lobe;
    V3 wo;
    float materialRoughness;
    bool ggx, sampled;

    bool deferred = false, stashed = false;  // kDefer: a job stored; the BSDF record stashed

    __device__ void lights(const LightJob& j) {
        if constexpr (kDefer) {
            storeLightJob(w, p, j);
            deferred = true;
        }
    }
    __device__ void shadow(const ShadowReq& q, bool isBsdf) {
        size_t k;
        if (kDefer && isBsdf) {
            k = size_t(p) * recordsPerPath + recordsPerPath - 1;
            stashed = true;
        } else {
            k = size_t(p) * recordsPerPath + n++;
        }
        w.sray0[k] = make_float4(q.origin.x, q.origin.y, q.origin.z, q.near);
        w.sray1[k] = make_float4(q.dir.x, q.dir.y, q.dir.z, q.far);
        w.scontrib[k] = make_float4(q.contribution.x, q.contribution.y, q.contribution.z, 0.0f);
        if (isBsdf) ++nBsdf;
        else ++nNee;
        if (kAdjoint) {
            if (isBsdf) bsdfDirection(q.dir);
            const float g = !isBsdf && ggx ? ggxLogDerivative(lobe, materialRoughness, wo, q.dir) : 0.0f;
            adj->aux[k] = make_uint2(q.light | (isBsdf ? 0x80000000u : 0u), __float_as_uint(g));
        }
    }
    __device__ void held() { ++nHeld; }
    __device__ void vertex(uint32_t m, const Bsdf& b, V3 out, const TexHit* tex) {
        if (!kAdjoint) return;
        const bool lambert = b.count && b.lobe.kind == 0;
        ggx = b.count && b.lobe.kind == 1;
        sampled = false;
        const uint32_t kind = lambert ? kVertLambert : ggx ? kVertGgx : kVertNone;
        const size_t v = size_t(p) * adj->vertsPerPath + depth;
        adj->vert[v] = make_uint4(m | (kind << 30), __float_as_uint(radiance->x), __float_as_uint(radiance->y), __float_as_uint(radiance->z));
        const V3 a = b.lobe.albedo;
        adj->scale[v] = lambert ? make_float4(a.x != 0.0f ? 1.0f / a.x : 0.0f, a.y != 0.0f ? 1.0f / a.y : 0.0f, a.z != 0.0f ? 1.0f / a.z : 0.0f, 0.0f)
                                : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        adj->vcount[p] = depth + 1;
        if (lambert && tex && adj->tex) adj->tex[v] = make_float4(tex->s, tex->t, tex->primary ? 1.0f : 0.0f, 0.0f);
        if (ggx) {
            lobe = b.lobe;
            wo = out;
            materialRoughness = s->materials[m].roughness;
        }
    }
    // The BSDF sample's direction, the first time the vertex hands on something that came through it.
    __device__ void bsdfDirection(V3 wi) {
        if (!ggx || sampled) return;
        sampled = true;
        adj->scale[size_t(p) * adj->vertsPerPath + depth].x = ggxLogDerivative(lobe, materialRoughness, wo, wi);
    }
    __device__ uint32_t top(uint32_t t) const { return t; }
    __device__ void push(const Pending& c) {
        if (kAdjoint) bsdfDirection(c.dir);
        child = c;
        pushed = true;
    }
};

// Entry i of the extend queue, its bins read in octant order when it is binned.
__device__ __forceinline__ uint32_t extendAt(const WaveArgs& a, uint32_t i) {
    if (!a.extendSlots) return a.extendQ[i];
    uint32_t o = 0, start = 0;
    for (; o + 1 < kOctants; ++o) {
        const uint32_t c = a.extendSlots[o];
        if (i < start + c) break;
        start += c;
    }
    return a.extendQ[size_t(o) * a.paths + (i - start)];
}

// ---- sort: per-lobe shade queues ----
// Each extended path goes to the queue of the lobe its hit's material makes (shading.cuh lobeClass: 0 Lambert, 1 GGX,
// 2 none) or, when its ray hit nothing, to queue 2; queue order: GGX (0), Lambert (1), none or missed (2). One
// warp-aggregated atomic a queue a warp round.
template <bool kBatch>
__device__ __forceinline__ void sortBody(const WaveArgs& a) {
    const WaveState& w = a.w;
    const uint32_t n = *a.extendCount;
    const unsigned full = 0xffffffffu;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += stride) {
        const uint32_t i = base + threadIdx.x;
        uint32_t queue = 3, p = 0;
        if (i < n) {
            p = extendAt(a, i);
            queue = 2;
            const uint2 hr = w.hit[p];
            if (hr.x != ~0u) {
                const SceneView& s = sceneOf<kBatch>(a, requestOf(w, p));
                const uint32_t tri = __float_as_uint(__ldg(reinterpret_cast<const float*>(s.bvh.tris + hr.x) + 3));
                const uint32_t c = lobeClass(s.materials[__ldg(s.meshMaterial + __ldg(s.triMesh + tri))]);
                queue = c == 1 ? 0u : c == 0 ? 1u : 2u;
            }
        }
#pragma unroll
        for (uint32_t q = 0; q < 3; ++q) {
            const unsigned mask = __ballot_sync(full, queue == q);
            if (!mask) continue;
            const uint32_t leader = __ffs(mask) - 1;
            uint32_t at = 0;
            if (lane == leader) at = atomicAdd(a.shadeCount + q, uint32_t(__popc(mask)));
            at = __shfl_sync(full, at, leader);
            if (queue == q) a.shadeQ[size_t(q) * a.paths + at + __popc(mask & ((1u << lane) - 1u))] = p;
        }
    }
}
__global__ void __launch_bounds__(kWaveBlock) wfSortShade(WaveArgs a) { sortBody<false>(a); }
__global__ void __launch_bounds__(kWaveBlock) wfSortShadeBatch(WaveArgs a) { sortBody<true>(a); }

// The i-th path shade takes: from the per-lobe queues in their order when they are on, else the extend queue's.
__device__ __forceinline__ uint32_t shadeEntry(const WaveArgs& a, uint32_t i, uint32_t c0, uint32_t c1) {
    if (!a.shadeQ) return extendAt(a, i);
    if (i < c0) return a.shadeQ[i];
    if (i < c0 + c1) return a.shadeQ[a.paths + (i - c0)];
    return a.shadeQ[2ull * a.paths + (i - c0 - c1)];
}

// A path's `records` shadow records into the shadow queue (every lane of the warp calls it, each with its own count):
// by record (record k of each lane's path into segment k) or by path.
__device__ __forceinline__ void reserveShadows(const WaveArgs& a, uint32_t p, uint32_t records) {
    if (a.shadowSlots) {
        warpReserve(a.shadowCount, records);  // the total, for the host's statistics
        const uint32_t most = __reduce_max_sync(0xffffffffu, records);
        for (uint32_t k = 0; k < most; ++k) {
            const uint32_t slot = warpReserve(a.shadowSlots + k, records > k ? 1u : 0u);
            if (records > k) a.shadowQ[size_t(k) * a.paths + slot] = p * a.recordsPerPath + k;
        }
    } else {
        const uint32_t slot = warpReserve(a.shadowCount, records);
        for (uint32_t k = 0; k < records; ++k) a.shadowQ[slot + k] = p * a.recordsPerPath + k;
    }
}

// The light samples of one per-lobe queue's vertices (kQueue 0 GGX, 1 Lambert), after its deferring shade kernel: each
// slot's job through lightSamples — the arithmetic the fused shade runs — its records written from the slot's first,
// then the BSDF sample's stashed record moved after them, the count and the shadow queue as the fused shade leaves
// them.
template <int kQueue>
__device__ __forceinline__ void lightsBody(const WaveArgs& a) {
    const WaveState& w = a.w;
    const SceneView& s = a.scene;
    const uint32_t n = a.shadeCount[kQueue];
    const uint32_t R = a.recordsPerPath;
    unsigned long long nee = 0;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += stride) {
        const uint32_t i = base + threadIdx.x;
        uint32_t records = 0, p = 0;
        if (i < n) {
            p = a.shadeQ[size_t(kQueue) * a.paths + i];
            const uint32_t flags = w.lightFlags[p];
            WaveSink<false> sink{w, p, 0, R, false, Pending{}, 0, 0, 0};
            if (flags & 1u) {
                const LightJob j = loadLightJob(w, p);
                const Identity root{j.pixel, U64(j.index), U64(s.config.seed), 0};
                lightSamples<false, kQueue == 0 ? 2 : 1>(s, root, j, sink);
            }
            records = sink.n;
            nee += sink.nNee;
            const size_t first = size_t(p) * R;
            if (flags & 2u) {
                if (records != R - 1) {
                    w.sray0[first + records] = w.sray0[first + R - 1];
                    w.sray1[first + records] = w.sray1[first + R - 1];
                    w.scontrib[first + records] = w.scontrib[first + R - 1];
                }
                ++records;
            }
            w.ncount[p] = records;
            for (uint32_t k = 0; k < records; ++k) w.svis[first + k] = 0;
        }
        reserveShadows(a, p, records);
    }
    warpAddCounters(a.counters, 0, nee, 0, 0, 0, 0);
}

// kQueue: -1 every extended path (the per-lobe queues in order when they are on, else the extend queue); 0, 1, 2 one
// per-lobe queue (GGX, Lambert, the rest), its kernel holding that lobe's code only.
template <bool kBatch, bool kVolumes, bool kAdjoint = false, bool kTextures = true, int kQueue = -1, bool kDefer = false>
__device__ __forceinline__ void shadeBody(const WaveArgs& a) {
    const WaveState& w = a.w;
    const uint32_t n = kQueue < 0 ? *a.extendCount : a.shadeCount[kQueue];
    extern __shared__ float partial[];  // the adjoint's block partials
    const Layout at{a.adj.materials, a.adj.lights};
    if (kAdjoint) partialsBegin(partial, at);
    const uint32_t c0 = a.shadeQ ? a.shadeCount[0] : 0u, c1 = a.shadeQ ? a.shadeCount[1] : 0u;
    unsigned long long nee = 0, bsdf = 0, held = 0;
    // Every lane of a warp runs the same rounds: the shadow queue's reservation is a warp-wide scan.
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += stride) {
        const uint32_t i = base + threadIdx.x;
        uint32_t records = 0, p = 0, lightFlags = 0;
        if (i < n) {
            p = kQueue < 0 ? shadeEntry(a, i, c0, c1) : a.shadeQ[size_t(kQueue) * a.paths + i];
            Pending pv;
            loadPending(w, p, pv);
            const uint4 m = w.meta[p];
            const uint32_t pixel = m.x, index = m.y, request = m.w >> 24;
            const SceneView& s = sceneOf<kBatch>(a, request);
            const Identity root{pixel, U64(index), U64(s.config.seed), 0};
            const uint2 hr = w.hit[p];
            Hit hit;
            hit.geom = ~0u;
            hit.prim = 0;
            hit.t = hit.u = hit.v = 0;
            hit.normal = hit.origin = hit.below = hit.point = V3{0, 0, 0};
            V3 va{0, 0, 0}, vb{0, 0, 0}, vc{0, 0, 0};
            if (hr.x != ~0u) {
                const float4* tp = reinterpret_cast<const float4*>(s.bvh.tris + hr.x);
                const float4 A = __ldg(tp), B = __ldg(tp + 1), Cc = __ldg(tp + 2);
                va = V3{A.x, A.y, A.z};
                vb = V3{B.x, B.y, B.z};
                vc = V3{Cc.x, Cc.y, Cc.z};
                const uint32_t tri = __float_as_uint(A.w);
                hit.geom = __ldg(s.triMesh + tri);
                hit.prim = tri - __ldg(s.meshFirst + hit.geom);
                hit.t = __uint_as_float(hr.y);
                if (!geometryHit(hit, pv.origin, pv.dir, va, vb, vc)) hit.normal = V3{0, 0, 0};
            }
            float4 rad4 = w.rad[p];
            V3 radiance{rad4.x, rad4.y, rad4.z};
            float alpha = rad4.w;
            // The camera's position (a pinhole: every camera ray's origin).
            const V3 cameraPosition = add(mvector(s.camera.camera_to_render, V3{0, 0, 0}),
                                          V3{s.camera.camera_to_render[3][0], s.camera.camera_to_render[3][1], s.camera.camera_to_render[3][2]});
            float4 d{0, 0, 0, 0};
            if (kAdjoint) {
                // The held light (bounce-ray reuse), reached unless the ray met something short of it.
                d = a.adj.delta[p];
                if (pv.heldLight != ~0u && !(hit.geom != ~0u && hit.t < pv.heldFar)) creditLightTo(partial, at, s, d, pv.held, pv.heldLight);
            }
            const V3 prior = radiance;
            afterTrace<kVolumes>(s, root, pv, hit, cameraPosition, radiance, alpha);
            if (kAdjoint && pv.depth == 0 && s.config.visible_lights) {
                // The light a camera ray sees (afterTrace added it).
                const bool missed = hit.geom == ~0u;
                creditLightTo(partial, at, s, d, sub(radiance, prior),
                              visibleLightIndex(s, root, missed ? pv.origin : cameraPosition, pv.dir, missed ? 3.4028234663852886e+38f : hit.t));
            }
            uint32_t next = kDone;
            if (hit.geom != ~0u) {
                WaveSink<kAdjoint, kDefer> sink{w, p, 0, a.recordsPerPath, false, Pending{}, 0, 0, 0};
                if (kAdjoint) {
                    sink.adj = &a.adj;
                    sink.s = &s;
                    sink.radiance = &radiance;
                    sink.depth = pv.depth;
                    sink.ggx = sink.sampled = false;
                }
                const bool ok = shadeVertex<kVolumes, kTextures, kQueue == 0 ? 2 : kQueue == 1 ? 1 : 0, kDefer>(
                    s, root, pixel, index, pv, hit, va, vb, vc, 0u, radiance, alpha, sink);
                if (kDefer) lightFlags = (sink.deferred ? 1u : 0u) | (sink.stashed ? 2u : 0u);
                if (!ok) {
                    next = kError;
                } else {
                    records = sink.n;
                    if (sink.pushed) {
                        storePending(w, p, sink.child, pixel, index, request);
                        next = kTrace;
                    }
                }
                nee += sink.nNee;
                bsdf += sink.nBsdf;
                held += sink.nHeld;
            }
            w.rad[p] = make_float4(radiance.x, radiance.y, radiance.z, alpha);
            w.state[p] = next;
            if (kDefer) {
                w.lightFlags[p] = lightFlags;  // the light kernel makes the slot's records
            } else {
                w.ncount[p] = records;
                const size_t first = size_t(p) * a.recordsPerPath;
                for (uint32_t k = 0; k < records; ++k) w.svis[first + k] = 0;
            }
        }
        if (!kDefer) reserveShadows(a, p, records);
    }
    warpAddCounters(a.counters, 0, nee, bsdf, held, 0, 0);
    if (kAdjoint) partialsEnd(partial, at, a.adj);
}

// ---- shadow: any hits ----
template <bool kBatch, int kShort = kShortStack, bool kStats = false, bool kOverlap = false>
__device__ __forceinline__ void shadowBody(const WaveArgs& a) {
    __shared__ uint32_t start[kRecordSegments + 1];
    QueueSegments seg{start, 0, a.paths};
    uint32_t n = *a.shadowCount;
    if (a.shadowSlots) {
        seg.segments = a.recordsPerPath;
        if (threadIdx.x == 0) {
            uint32_t run = 0;
            for (uint32_t k = 0; k < seg.segments; ++k) {
                start[k] = run;
                run += a.shadowSlots[k];
            }
            start[seg.segments] = run;
        }
        __syncthreads();
        n = start[seg.segments];
    }
    __shared__ uint2 shortStacks[kShort > 0 ? kShort * kWaveBlock : 1];
    persistentTrace<true, kStats && !kBatch, kBatch, kShort, kOverlap>(a, n, a.shadowQ, a.shadowNext, shortStacks, seg);
}

// The kernels, each in a few occupancy variants (blocks of kWaveBlock threads a SM that the register allocation must
// allow), chosen at launch (x2_wavefront_tune); batches in the compiler's allocation. Shade comes in a form for
// scenes without volumes (the volume code compiled out) and one for scenes with them.
__global__ void __launch_bounds__(kWaveBlock) wfExtend(WaveArgs a) { extendBody<false>(a); }
__global__ void __launch_bounds__(kWaveBlock) wfShade(WaveArgs a) { shadeBody<false, false, false, false>(a); }
// Volume scenes' shade (the march inside it), with the texture lookup compiled in (kTextures) or out.
template <bool kTextures>
__global__ void __launch_bounds__(kWaveBlock, 4) wfShadeVolumes(WaveArgs a) { shadeBody<false, true, false, kTextures>(a); }
__global__ void __launch_bounds__(kWaveBlock, 4) wfShadeBatchVolumes(WaveArgs a) { shadeBody<true, true>(a); }
__global__ void __launch_bounds__(kWaveBlock, 4) wfShadeAdjoint(WaveArgs a) { shadeBody<false, false, true>(a); }

// The adjoint's gradient rows summed in FP64 into grads (one thread a gradient).
__global__ void wfGradRows(const float* rows, uint32_t rowCount, uint32_t params, double* grads) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= params) return;
    double sum = 0.0;
    for (uint32_t r = 0; r < rowCount; ++r) sum += double(rows[size_t(r) * params + i]);
    grads[i] += sum;
}
__global__ void __launch_bounds__(kWaveBlock) wfShadow(WaveArgs a) { shadowBody<false>(a); }
// Counting mode's traversal kernels (node visits, triangle tests, lane use; x2_count_traversal): kernels of their own,
// so that the timed ones carry none of the counting's registers.
__global__ void __launch_bounds__(kWaveBlock) wfExtendCount(WaveArgs a) { extendBody<false, kShortStack, true>(a); }
__global__ void __launch_bounds__(kWaveBlock) wfShadowCount(WaveArgs a) { shadowBody<false, kShortStack, true>(a); }
// Node visits and triangle tests overlapped in a lane's steps (wavefront shape tri_overlap), timed and counting.
__global__ void __launch_bounds__(kWaveBlock) wfExtendOverlap(WaveArgs a) { extendBody<false, kShortStack, false, true>(a); }
__global__ void __launch_bounds__(kWaveBlock) wfShadowOverlap(WaveArgs a) { shadowBody<false, kShortStack, false, true>(a); }
__global__ void __launch_bounds__(kWaveBlock) wfExtendOverlapCount(WaveArgs a) { extendBody<false, kShortStack, true, true>(a); }
__global__ void __launch_bounds__(kWaveBlock) wfShadowOverlapCount(WaveArgs a) { shadowBody<false, kShortStack, true, true>(a); }
// The traversal kernels with their whole stacks in local memory (wavefront shape short_stack 0).
__global__ void __launch_bounds__(kWaveBlock) wfExtendLocal(WaveArgs a) { extendBody<false, 0>(a); }
__global__ void __launch_bounds__(kWaveBlock) wfShadowLocal(WaveArgs a) { shadowBody<false, 0>(a); }
__global__ void __launch_bounds__(kWaveBlock) wfExtendBatch(WaveArgs a) { extendBody<true>(a); }
__global__ void __launch_bounds__(kWaveBlock) wfShadowBatch(WaveArgs a) { shadowBody<true>(a); }
template <int kMinBlocks>
__global__ void __launch_bounds__(kWaveBlock, kMinBlocks) wfExtendOcc(WaveArgs a) {
    extendBody<false>(a);
}
template <int kMinBlocks, bool kBatch, bool kTextures = false>
__global__ void __launch_bounds__(kWaveBlock, kMinBlocks) wfShadeOcc(WaveArgs a) {
    shadeBody<kBatch, false, false, kTextures>(a);
}
template <int kMinBlocks>
__global__ void __launch_bounds__(kWaveBlock, kMinBlocks) wfShadowOcc(WaveArgs a) {
    shadowBody<false>(a);
}
// Shade split by lobe (wavefront shape shade_split): one kernel a per-lobe queue, each with one lobe's code.
template <int kQueue, bool kTextures, int kMinBlocks>
__global__ void __launch_bounds__(kWaveBlock, kMinBlocks) wfShadeQueue(WaveArgs a) {
    shadeBody<false, false, false, kTextures, kQueue>(a);
}
// The batch form's shade split by lobe (each path's scene from the request table).
template <int kQueue, bool kTextures>
__global__ void __launch_bounds__(kWaveBlock, 4) wfShadeQueueBatch(WaveArgs a) {
    shadeBody<true, false, false, kTextures, kQueue>(a);
}
// With the light samples split off (light_split): the GGX and Lambert queues' shade without them, and their light
// kernels.
template <int kQueue, bool kTextures>
__global__ void __launch_bounds__(kWaveBlock, 4) wfShadeDefer(WaveArgs a) {
    shadeBody<false, false, false, kTextures, kQueue, true>(a);
}
template <int kQueue, int kMinBlocks>
__global__ void __launch_bounds__(kWaveBlock, kMinBlocks) wfLightsQueue(WaveArgs a) {
    lightsBody<kQueue>(a);
}

void launchShade(const WaveKernels& k, const WaveArgs& a, int grid, cudaStream_t st, bool batch) {
    if (a.shadeQ) (batch ? wfSortShadeBatch : wfSortShade)<<<grid, kWaveBlock, 0, st>>>(a);
    if (a.shadeQ && k.shadeBy[0]) {
        for (int q = 0; q < 3; ++q) k.shadeBy[q]<<<grid, kWaveBlock, 0, st>>>(a);
        if (k.lightsBy[0])
            for (int q = 0; q < 2; ++q) k.lightsBy[q]<<<grid, kWaveBlock, 0, st>>>(a);
    } else {
        k.shade<<<grid, kWaveBlock, 0, st>>>(a);
    }
}

WaveKernels waveKernels(uint32_t traceBlocks, uint32_t shadeBlocks, bool volumes, bool textures, bool shortStack, bool counting,
                        bool shadeSplit, uint32_t lightSplit, bool overlap) {
    const bool lightSplit8 = lightSplit == 2;
    WaveKernels k;
    k.shadeBy[0] = k.shadeBy[1] = k.shadeBy[2] = nullptr;
    k.lightsBy[0] = k.lightsBy[1] = nullptr;
    if (shadeSplit && !volumes) {
        // The GGX and Lambert kernels at 4 blocks a SM (128 registers) or, with shade_blocks 5, at 5 (96, more spilled).
        const bool five = shadeBlocks >= 5;
        k.shadeBy[0] = textures ? (five ? wfShadeQueue<0, true, 5> : wfShadeQueue<0, true, 4>) : (five ? wfShadeQueue<0, false, 5> : wfShadeQueue<0, false, 4>);
        k.shadeBy[1] = textures ? (five ? wfShadeQueue<1, true, 5> : wfShadeQueue<1, true, 4>) : (five ? wfShadeQueue<1, false, 5> : wfShadeQueue<1, false, 4>);
        k.shadeBy[2] = textures ? wfShadeQueue<2, true, 4> : wfShadeQueue<2, false, 4>;
        if (lightSplit) {
            k.shadeBy[0] = textures ? wfShadeDefer<0, true> : wfShadeDefer<0, false>;
            k.shadeBy[1] = textures ? wfShadeDefer<1, true> : wfShadeDefer<1, false>;
            // The light kernels at 6 blocks a SM (80 registers; 64 B of the GGX kernel's spilled) or, light_split 2, at 8
            // (64 registers, more spilled).
            k.lightsBy[0] = lightSplit8 ? wfLightsQueue<0, 8> : wfLightsQueue<0, 6>;
            k.lightsBy[1] = lightSplit8 ? wfLightsQueue<1, 8> : wfLightsQueue<1, 6>;
        }
    }
    k.logic = wfLogic;
    k.extend = traceBlocks >= 10 ? wfExtendOcc<10> : traceBlocks >= 9 ? wfExtendOcc<9> : shortStack ? wfExtend : wfExtendLocal;
    k.shadow = traceBlocks >= 10 ? wfShadowOcc<10> : traceBlocks >= 9 ? wfShadowOcc<9> : shortStack ? wfShadow : wfShadowLocal;
    if (overlap) {
        k.extend = counting ? wfExtendOverlapCount : wfExtendOverlap;
        k.shadow = counting ? wfShadowOverlapCount : wfShadowOverlap;
    } else if (counting) {
        k.extend = wfExtendCount;
        k.shadow = wfShadowCount;
    }
    if (volumes) k.shade = textures ? wfShadeVolumes<true> : wfShadeVolumes<false>;
    else if (textures) k.shade = wfShadeOcc<4, false, true>;
    else k.shade = shadeBlocks >= 4 ? wfShadeOcc<4, false> : shadeBlocks >= 3 ? wfShadeOcc<3, false> : wfShade;
    return k;
}

WaveKernels waveKernelsBatch(bool volumes, bool textures, bool shadeSplit) {
    WaveKernels k;
    k.shadeBy[0] = k.shadeBy[1] = k.shadeBy[2] = nullptr;
    k.lightsBy[0] = k.lightsBy[1] = nullptr;
    if (shadeSplit && !volumes) {
        k.shadeBy[0] = textures ? wfShadeQueueBatch<0, true> : wfShadeQueueBatch<0, false>;
        k.shadeBy[1] = textures ? wfShadeQueueBatch<1, true> : wfShadeQueueBatch<1, false>;
        k.shadeBy[2] = textures ? wfShadeQueueBatch<2, true> : wfShadeQueueBatch<2, false>;
    }
    k.logic = wfLogicBatch;
    k.extend = wfExtendBatch;
    k.shadow = wfShadowBatch;
    k.shade = volumes ? wfShadeBatchVolumes : textures ? wfShadeOcc<4, true, true> : wfShadeOcc<4, true>;
    return k;
}

// Queue counters for the next iteration: the extend and shadow counts start at zero; the previous counts are kept
// for the host (the graph's last extend count tells whether paths remain).
__global__ void wfResetQueues(WaveArgs a) {
    if (threadIdx.x == 0) {
        *a.lastExtend = *a.extendCount;
        *a.extendCount = 0;
        *a.shadowCount = 0;
        *a.extendNext = 0;
        if (a.shadowSlots)
            for (uint32_t k = 0; k < a.recordsPerPath; ++k) a.shadowSlots[k] = 0;
        if (a.extendSlots)
            for (uint32_t o = 0; o < kOctants; ++o) a.extendSlots[o] = 0;
        *a.shadowNext = 0;
        if (a.shadeQ) a.shadeCount[0] = a.shadeCount[1] = a.shadeCount[2] = 0;
    }
}

__global__ void wfDrainCheck(WaveArgs a, cudaGraphConditionalHandle loop, uint32_t* iterations, uint32_t maxIterations,
                             uint32_t* overrun) {
    if (threadIdx.x != 0) return;
    const uint32_t n = ++iterations[0];
    ++iterations[1];
    const bool more = *a.extendCount != 0;
    if (more && n >= maxIterations) *overrun = 1;
    cudaGraphSetConditional(loop, more && n < maxIterations ? 1u : 0u);
}

// The film: each (chunk, position)'s samples summed in sample order, then added to the pixel (async_gpu.cu:320-364's
// sums and counts, without the per-sample atomics).
__global__ void wfFilmReduce(WaveArgs a, uint32_t chunkCount, double* sums, double* odd, uint32_t* counts) {
    const uint32_t width = a.scene.config.width, height = a.scene.config.height;
    const unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (a.liveChunks && *a.liveChunks < chunkCount) chunkCount = *a.liveChunks;
    if (i >= 64ull * chunkCount) return;
    const uint32_t chunkIndex = uint32_t(i / 64), position = uint32_t(i % 64);
    const x2_chunk chunk = a.chunks[chunkIndex];
    const uint32_t pixel = tilePixelW(chunk.tile, position, width, height);
    if (pixel == ~0u) return;
    double v[4] = {0, 0, 0, 0}, o[4] = {0, 0, 0, 0};
    uint32_t n = 0;
    const unsigned long long first = (unsigned long long)chunkIndex * 64ull * a.samplesPerChunk + (unsigned long long)position * a.samplesPerChunk;
    const uint32_t indexBase = a.pixelBase ? a.pixelBase[pixel] : chunk.first;
    // A chunk holds at most samplesPerChunk items a pixel; a larger count (caller input the device-memory entry points
    // do not check on the host) is clamped as the logic kernel clamps it, so no read leaves the chunk's items.
    const uint32_t count = min(chunk.count, a.samplesPerChunk);
    for (uint32_t s = 0; s < count; ++s) {
        if (a.outStatus[first + s] != X2_DONE) continue;
        const float4 r = a.out[first + s];
        v[0] += double(r.x);
        v[1] += double(r.y);
        v[2] += double(r.z);
        v[3] += double(r.w);
        if (odd && ((indexBase + s) & 1u)) {
            o[0] += double(r.x);
            o[1] += double(r.y);
            o[2] += double(r.z);
            o[3] += double(r.w);
        }
        ++n;
    }
    if (!n) return;
    for (int k = 0; k < 4; ++k) atomicAdd(sums + 4ull * pixel + k, v[k]);
    if (odd)
        for (int k = 0; k < 4; ++k)
            if (o[k] != 0.0) atomicAdd(odd + 4ull * pixel + k, o[k]);
    atomicAdd(counts + pixel, n);
}

// A batch's films: each chunk's samples (64 x its count items from chunkItems[c]) into its request's film.
__global__ void wfFilmReduceBatch(WaveArgs a, const BatchFilm* __restrict__ films) {
    const unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 64ull * a.chunkCount) return;
    const uint32_t chunkIndex = uint32_t(i / 64), position = uint32_t(i % 64);
    const x2_chunk chunk = a.chunks[chunkIndex];
    const uint32_t request = a.chunkRequest[chunkIndex];
    const SceneView& sv = a.scenes[request];
    const uint32_t pixel = tilePixelW(chunk.tile, position, sv.config.width, sv.config.height);
    if (pixel == ~0u) return;
    const BatchFilm f = films[request];
    const unsigned long long begin = a.chunkItems[chunkIndex], perPixel = (a.chunkItems[chunkIndex + 1] - begin) / 64ull;
    const unsigned long long first = begin + position * perPixel;
    double v[4] = {0, 0, 0, 0}, o[4] = {0, 0, 0, 0};
    uint32_t n = 0;
    const uint32_t count = uint32_t(min((unsigned long long)chunk.count, perPixel));
    for (uint32_t s = 0; s < count; ++s) {
        if (a.outStatus[first + s] != X2_DONE) continue;
        const float4 r = a.out[first + s];
        v[0] += double(r.x);
        v[1] += double(r.y);
        v[2] += double(r.z);
        v[3] += double(r.w);
        if (f.odd && ((chunk.first + s) & 1u)) {
            o[0] += double(r.x);
            o[1] += double(r.y);
            o[2] += double(r.z);
            o[3] += double(r.w);
        }
        ++n;
    }
    if (!n) return;
    for (int k = 0; k < 4; ++k) atomicAdd(f.sums + 4ull * pixel + k, v[k]);
    if (f.odd)
        for (int k = 0; k < 4; ++k)
            if (o[k] != 0.0) atomicAdd(f.odd + 4ull * pixel + k, o[k]);
    atomicAdd(f.counts + pixel, n);
}

}  // namespace x2
