// x2_launch_wavefront_static: the wavefront launch for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc: a process whose device memory is already reserved by another allocator (a
// framework's caching allocator holding the GPU), or code on a latency-bound path where cudaMalloc's implicit device
// synchronisation is not allowed. This entry point runs the same wavefront kernels as x2_launch_wavefront with all
// of their scratch — path slots, shadow-ray records, queues, per-item outputs, counters — in one file-scope array
// of kScratchBytes that every GPU which loads the library holds until the process exits. It allocates nothing: no
// cudaMalloc/cudaFree, no events, no graph; the caller passes the chunks and the film (device pointers).
//
// Limits (calls beyond them return X2_EINVAL): at most kMaxItems work items a call (chunks x 64 x samples a chunk),
// at most kMaxRecords - 1 light samples a vertex (light_count x light_samples), one BSDF sample (bsdf_samples = 1),
// kPaths paths in flight.
//
// Set-up: every call looks up the array's device address (cudaGetSymbolAddress, with the scene's device current: a
// lookup, not an allocation), so a context that was destroyed and created again is never handed a stale address.
// The first call on a device also loads the library's module there: make that first call before any stream capture.
// Every call shares the array and keeps the last call's contents; each call clears what must start at zero. Calls
// that overlap on the GPU (two host threads, two streams, two contexts on one device) race on the array and must not
// be made. A call returns only once its kernels have finished, error returns included, except X2_ETIMEOUT (the
// stream still busy after the wait's limit): after that, wait for the scene's stream (x2_synchronize) before the
// next call.
#include <cuda_runtime.h>

#include <chrono>
#include <mutex>
#include <thread>

#include "../../include/x2.h"
#include "engine.h"
#include "wavefront.h"

namespace x2 {

namespace {

constexpr uint32_t kPaths = 8192, kMaxRecords = 33, kMaxItems = 1u << 20;

constexpr size_t align256(size_t n) { return (n + 255) & ~size_t(255); }
// The array's parts, in order.
constexpr size_t kRay0 = 0, kRay1 = kRay0 + align256(16ull * kPaths), kT = kRay1 + align256(16ull * kPaths),
                 kHeld = kT + align256(16ull * kPaths), kMeta = kHeld + align256(16ull * kPaths), kBranch = kMeta + align256(16ull * kPaths),
                 kRad = kBranch + align256(8ull * kPaths), kHit = kRad + align256(16ull * kPaths), kState = kHit + align256(8ull * kPaths),
                 kItem = kState + align256(4ull * kPaths), kNcount = kItem + align256(4ull * kPaths),
                 kSray0 = kNcount + align256(4ull * kPaths), kSray1 = kSray0 + align256(16ull * kPaths * kMaxRecords),
                 kScontrib = kSray1 + align256(16ull * kPaths * kMaxRecords), kSvis = kScontrib + align256(16ull * kPaths * kMaxRecords),
                 kExtendQ = kSvis + align256(1ull * kPaths * kMaxRecords), kShadowQ = kExtendQ + align256(4ull * kPaths),
                 kOut = kShadowQ + align256(4ull * kPaths * kMaxRecords), kOutStatus = kOut + align256(16ull * kMaxItems),
                 kQueueCounters = kOutStatus + align256(1ull * kMaxItems), kClaimed = kQueueCounters + align256(32),
                 kCounters = kClaimed + align256(8), kScratchBytes = kCounters + align256(sizeof(Counters));
static_assert(kScratchBytes <= 36ull << 20, "the static scratch stays modest (36 MiB)");

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

std::mutex g_mutex;

int waitStream(cudaStream_t st, int timeoutMs) {
    const auto until = std::chrono::steady_clock::now() + std::chrono::milliseconds(timeoutMs);
    for (;;) {
        const cudaError_t q = cudaStreamQuery(st);
        if (q == cudaSuccess) return X2_OK;
        if (q != cudaErrorNotReady) {
            setError("device error: %s", cudaGetErrorString(q));
            return X2_ECUDA;
        }
        if (std::chrono::steady_clock::now() >= until) {
            setError("wait timed out after %d ms", timeoutMs);
            return X2_ETIMEOUT;
        }
        std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
}

}  // namespace

// Internal: the scene's device view and stream (api.cu).
int sceneView(x2_scene* scene, SceneView* view, cudaStream_t* stream, int* device, int* smCount);

}  // namespace x2

using namespace x2;

extern "C" int x2_launch_wavefront_static(x2_scene* scene, const x2_chunk* d_chunks, uint32_t count, uint32_t samples_per_chunk,
                                          double* d_sums, uint32_t* d_counts, uint64_t* samples_done) {
    SceneView view;
    cudaStream_t st;
    int device = 0, smCount = 0;
    if (int rc = sceneView(scene, &view, &st, &device, &smCount)) return rc;
    const x2_config& c = view.config;
    if (!d_chunks || !d_sums || !d_counts || samples_per_chunk == 0) {
        setError("null chunks or film, or zero samples a chunk");
        return X2_EINVAL;
    }
    const unsigned long long items = (unsigned long long)count * 64ull * samples_per_chunk;
    if (items > kMaxItems) {
        setError("%llu work items in one call; the static scratch holds at most %u", items, kMaxItems);
        return X2_EINVAL;
    }
    const uint32_t records = c.light_count * c.light_samples + 1;
    if (records > kMaxRecords || c.bsdf_samples != 1) {
        setError("at most %u light samples a vertex and one BSDF sample (%u lights x %u samples, %u BSDF samples)", kMaxRecords - 1,
                 c.light_count, c.light_samples, c.bsdf_samples);
        return X2_EINVAL;
    }
    if (!count) return X2_OK;
    unsigned char* base = nullptr;
    {
        // The array's address in the current context of the scene's device (sceneView made it current).
        std::lock_guard<std::mutex> lock(g_mutex);
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess || !p) {
            setError("cudaGetSymbolAddress of the static scratch failed on device %d: %s", device, cudaGetErrorString(e));
            return X2_ECUDA;
        }
        base = static_cast<unsigned char*>(p);
    }
    WaveArgs a;
    a.scene = view;
    a.w.ray0 = reinterpret_cast<float4*>(base + kRay0);
    a.w.ray1 = reinterpret_cast<float4*>(base + kRay1);
    a.w.T = reinterpret_cast<float4*>(base + kT);
    a.w.held = reinterpret_cast<float4*>(base + kHeld);
    a.w.meta = reinterpret_cast<uint4*>(base + kMeta);
    a.w.branch = reinterpret_cast<uint2*>(base + kBranch);
    a.w.rad = reinterpret_cast<float4*>(base + kRad);
    a.w.hit = reinterpret_cast<uint2*>(base + kHit);
    a.w.state = reinterpret_cast<uint32_t*>(base + kState);
    a.w.item = reinterpret_cast<uint32_t*>(base + kItem);
    a.w.ncount = reinterpret_cast<uint32_t*>(base + kNcount);
    a.w.sray0 = reinterpret_cast<float4*>(base + kSray0);
    a.w.sray1 = reinterpret_cast<float4*>(base + kSray1);
    a.w.scontrib = reinterpret_cast<float4*>(base + kScontrib);
    a.w.svis = base + kSvis;
    a.paths = kPaths;
    a.recordsPerPath = records;
    a.chunks = d_chunks;
    a.itemCount = items;
    a.samplesPerChunk = samples_per_chunk;
    a.claimed = reinterpret_cast<unsigned long long*>(base + kClaimed);
    a.extendQ = reinterpret_cast<uint32_t*>(base + kExtendQ);
    uint32_t* queues = reinterpret_cast<uint32_t*>(base + kQueueCounters);
    a.extendCount = queues;
    a.lastExtend = queues + 1;
    a.shadowQ = reinterpret_cast<uint32_t*>(base + kShadowQ);
    a.shadowCount = queues + 2;
    a.shadowSlots = nullptr;  // the shadow queue by path
    a.extendSlots = nullptr;  // the extend queue in slot order
    a.extendNext = queues + 3;
    a.shadowNext = queues + 4;
    a.shadeQ = nullptr;  // shade in the extend queue's order
    a.shadeCount = nullptr;
    a.adj = AdjointWave{};
    a.chunkMask = nullptr;
    a.pixelBase = nullptr;
    a.liveChunks = nullptr;
    a.refill = kDefaultRefill;
    a.triLimit = kDefaultTriLimit;
    a.out = reinterpret_cast<float4*>(base + kOut);
    a.outStatus = base + kOutStatus;
    a.counters = reinterpret_cast<Counters*>(base + kCounters);
    a.scenes = nullptr;
    a.chunkRequest = nullptr;
    a.chunkItems = nullptr;
    a.chunkCount = count;
    // What must start at zero; the rest is written before it is read.
    const struct {
        void* p;
        int v;
        size_t n;
    } clears[] = {{a.w.state, 0, 4ull * kPaths}, {a.w.ncount, 0, 4ull * kPaths}, {queues, 0, 32}, {a.claimed, 0, 8},
                  {a.counters, 0, sizeof(Counters)}, {a.outStatus, X2_SKIP, size_t(items)}};
    for (const auto& z : clears) {
        const cudaError_t e = cudaMemsetAsync(z.p, z.v, z.n, st);
        if (e != cudaSuccess) {
            setError("clearing the static scratch failed: %s", cudaGetErrorString(e));
            waitStream(st, 600000);
            return X2_ECUDA;
        }
    }
    const int gridLogic = int((kPaths + kWaveBlock - 1) / kWaveBlock);
    const int gridWork = smCount * int(kDefaultBlocksPerSm);
    const WaveKernels wk = waveKernels(kDefaultTraceBlocks, kDefaultShadeBlocks, view.config.volume_count != 0, view.triUV != nullptr);
    const uint64_t maxIter = items * (uint64_t(c.max_depth) + 2) / kPaths + uint64_t(c.max_depth) + 64;
    // Iterations go in rounds of kRound between reads of the last one's traced-ray count: once an iteration traces
    // nothing, no path is live and no item is left, and the iterations after it change nothing.
    constexpr uint64_t kRound = 4;
    uint32_t last = 1;
    for (uint64_t it = 0; last; it += kRound) {
        if (it > maxIter) {
            setError("wavefront did not drain after %llu iterations", (unsigned long long)it);
            return X2_EDEVICE;  // the stream is idle here: the last round was waited for
        }
        for (uint64_t k = 0; k < kRound; ++k) {
            wfResetQueues<<<1, 32, 0, st>>>(a);
            wk.logic<<<gridLogic, kWaveBlock, 0, st>>>(a);
            wk.extend<<<gridWork, kWaveBlock, 0, st>>>(a);
            wk.shade<<<gridWork, kWaveBlock, 0, st>>>(a);
            wk.shadow<<<gridWork, kWaveBlock, 0, st>>>(a);
            wfResetQueues<<<1, 32, 0, st>>>(a);
        }
        const cudaError_t e = cudaMemcpyAsync(&last, queues + 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
        if (e != cudaSuccess) {
            setError("launch failed: %s", cudaGetErrorString(e));
            waitStream(st, 600000);
            return X2_ECUDA;
        }
        if (int rc = waitStream(st, 600000)) return rc;
    }
    wfFilmReduce<<<int((64ull * count + 255) / 256), 256, 0, st>>>(a, count, d_sums, nullptr, d_counts);
    Counters h{};
    cudaMemcpyAsync(&h, a.counters, sizeof(Counters), cudaMemcpyDeviceToHost, st);
    if (int rc = waitStream(st, 600000)) return rc;
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        setError("launch failed: %s", cudaGetErrorString(e));
        return X2_ECUDA;
    }
    if (samples_done) *samples_done = h.samples;
    return h.errors ? X2_EDEVICE : X2_OK;
}
