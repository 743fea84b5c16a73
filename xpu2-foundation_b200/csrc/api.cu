// The C ABI (include/x2.h): context, scene upload and BVH build, the per-sample API and the lane API
// (GpuLane's begin/launch/poll/downloadFilm, async_gpu.h:1372-1707). One CUDA stream a context; every device
// wait is bounded (x2_wait, x2_synchronize poll events with a timeout instead of blocking).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/x2.h"
#include "engine.h"
#include "adaptive.h"
#include "generations.h"
#include "adjoint.h"
#include "render.h"
#include "wavefront.h"

namespace x2 {

namespace {
thread_local std::string g_error;
}

void setError(const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_error = buf;
}

namespace {

// Sobol direction numbers: dimension 0 van der Corput, 1..16 by the Bratley-Fox recurrence from Joe and Kuo's
// primitive polynomials (degree s, coefficients a, initial m) for their dimensions 2..17.
void sobolDirections(uint32_t out[17][32]) {
    static const uint32_t s[16] = {1, 2, 3, 3, 4, 4, 5, 5, 5, 5, 5, 5, 6, 6, 6, 6};
    static const uint32_t a[16] = {0, 1, 1, 2, 1, 4, 2, 4, 7, 11, 13, 14, 1, 13, 16, 19};
    static const uint32_t m0[16][6] = {{1}, {1, 3}, {1, 3, 1}, {1, 1, 1}, {1, 1, 3, 3}, {1, 3, 5, 13}, {1, 1, 5, 5, 17},
                                       {1, 1, 5, 5, 5}, {1, 1, 7, 11, 19}, {1, 1, 5, 1, 1}, {1, 1, 1, 3, 11}, {1, 3, 5, 5, 31},
                                       {1, 3, 3, 9, 7, 49}, {1, 1, 1, 15, 21, 21}, {1, 3, 1, 13, 27, 49}, {1, 1, 1, 15, 7, 5}};
    for (int i = 0; i < 32; ++i) out[0][i] = 1u << (31 - i);
    for (int d = 0; d < 16; ++d) {
        uint64_t m[32];
        for (uint32_t i = 0; i < s[d]; ++i) m[i] = m0[d][i];
        for (uint32_t i = s[d]; i < 32; ++i) {
            uint64_t v = m[i - s[d]] ^ (m[i - s[d]] << s[d]);
            for (uint32_t k = 1; k < s[d]; ++k)
                if ((a[d] >> (s[d] - 1 - k)) & 1u) v ^= m[i - k] << k;
            m[i] = v;
        }
        for (int i = 0; i < 32; ++i) out[d + 1][i] = uint32_t(m[i] << (31 - i));
    }
}

#define CUDA_OR(expr, code)                                                                         \
    do {                                                                                            \
        cudaError_t e_ = (expr);                                                                    \
        if (e_ != cudaSuccess) {                                                                    \
            setError("%s:%d %s: %s", __FILE__, __LINE__, #expr, cudaGetErrorString(e_));            \
            return code;                                                                            \
        }                                                                                           \
    } while (0)

// Waits for an event with a deadline (no unbounded cudaEventSynchronize).
int waitEvent(cudaEvent_t e, int timeoutMs) {
    const auto until = std::chrono::steady_clock::now() + std::chrono::milliseconds(timeoutMs < 0 ? 0 : timeoutMs);
    for (;;) {
        const cudaError_t q = cudaEventQuery(e);
        if (q == cudaSuccess) return X2_OK;
        if (q != cudaErrorNotReady) {
            setError("device error while waiting: %s", cudaGetErrorString(q));
            return X2_ECUDA;
        }
        if (std::chrono::steady_clock::now() >= until) {
            setError("wait timed out after %d ms", timeoutMs);
            return X2_ETIMEOUT;
        }
        std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
}

constexpr int kSlots = 2;  // launches in flight, as GpuLane keeps (async_gpu.h:1425)
constexpr uint32_t kQueueLog = 4096;
// extend count, last extend count, shadow count, extend fetch, shadow fetch, 3 shade queue counts, then the shadow
// queue's record segments (x2::kRecordSegments), then the extend queue's octant bins (x2::kOctants)
constexpr int kWaveCounters = 8 + int(x2::kRecordSegments) + int(x2::kOctants);

struct Slot {
    bool busy = false;
    uint64_t seq = 0;
    x2_chunk* chunks = nullptr;  // device
    uint32_t chunkCap = 0;
    unsigned long long* claimed = nullptr;
    Counters* counters = nullptr;      // device
    Counters* hostCounters = nullptr;  // pinned
    cudaEvent_t begin = nullptr, end = nullptr, done = nullptr;  // done: the counters have reached the host
};

}  // namespace
}  // namespace x2

using namespace x2;

struct x2_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    int smCount = 0;
    int renderBlocksPerSm = 0;
};

// An adaptive frame's device state (adaptive.h AdaptiveArgs) and its host-side layout.
struct AdaptiveState {
    uint32_t width = 0, height = 0, tiles = 0, tilesX = 0, regionCount = 0;
    float target = 0;
    x2::rg::RegionGrid grid;
    // Per region (device): boxes (4 ints), table offsets, node bounds, node counts, ready / open flags, and the
    // first row and column index of each region among all regions' rows and columns.
    int32_t* boxes = nullptr;
    unsigned long long* satOffset = nullptr;
    uint32_t *bound = nullptr, *nodes = nullptr, *ready = nullptr, *open = nullptr, *rowStart = nullptr, *colStart = nullptr;
    uint32_t rows = 0, cols = 0;
    double* sat = nullptr;
    // The node pool (structure of arrays) and its words: [0] nodes allocated, [1] [2] the level under decision.
    uint32_t poolCapacity = 0;
    float *px0 = nullptr, *py0 = nullptr, *px1 = nullptr, *py1 = nullptr;
    int32_t* pchild = nullptr;
    uint8_t* pfate = nullptr;
    uint32_t *pregion = nullptr, *poolWords = nullptr;
    float* errors = nullptr;
    uint64_t* inImage = nullptr;
    uint64_t* reach = nullptr;
    uint64_t* tileMask = nullptr;
    uint32_t* planned = nullptr;
    uint32_t* base = nullptr;
    uint32_t* stop = nullptr;
    uint64_t* chunkMasks = nullptr;  // a pass's active tiles' masks, in its chunks' order
    uint32_t* blockTiles = nullptr;  // the compaction's counts, a block of tiles each
    // A queued frame's words: [0] the pass's active chunks, [1] passes launched, [2] the pass's drain iterations,
    // [3] all passes' drain iterations, [4] a drain that hit its bound, [5] a cellular generation's live tiles; its
    // planned samples; their host copies (pinned).
    uint32_t* words = nullptr;
    unsigned long long* samples = nullptr;
    uint32_t* hostWords = nullptr;
    unsigned long long* hostSamples = nullptr;
    // Cellular generations: two generations of live tiles (a byte a tile each), the first every tile in the image, and
    // each tile's error ratio.
    uint8_t* alive = nullptr;
    float* ratio = nullptr;
    std::vector<uint8_t> firstAlive;
    ~AdaptiveState() {
        void* p[] = {boxes, satOffset, bound, nodes, ready, open, rowStart, colStart, sat, px0, py0, px1, py1, pchild, pfate, pregion,
                     poolWords, errors, inImage, reach, tileMask, planned, base, stop, chunkMasks, blockTiles, words, samples, alive, ratio};
        for (void* q : p) cudaFree(q);
        if (hostWords) cudaFreeHost(hostWords);
        if (hostSamples) cudaFreeHost(hostSamples);
    }
};

struct x2_scene {
    x2_ctx* ctx = nullptr;
    DeviceBvh bvh;
    uint32_t* triMesh = nullptr;
    uint32_t* meshFirst = nullptr;
    uint32_t* meshMaterial = nullptr;
    MaterialRec* materials = nullptr;
    TexRec* textures = nullptr;       // the textures (device) and their texels
    float* texels = nullptr;
    float* triUV = nullptr;           // scene triangle -> st of its vertices (6 floats), when a material has a texture
    std::vector<TexRec> hostTextures;
    x2_light* lights = nullptr;
    uint32_t* overflow = nullptr;
    uint32_t lightCount = 0, triangleCount = 0, materialCount = 0;
    // volumes (device): records, bounds' triangles, grids and their values
    VolumeRec* volumes = nullptr;
    float* volumeTris = nullptr;
    GridRec* grids = nullptr;
    std::vector<float*> gridValues;
    std::vector<float*> majorants;  // each volume's majorant grid (device)
    bool greyVolumes = true;        // every volume's gain has three equal channels (the tracking estimator's condition)
    uint32_t volumeCount = 0, gridCount = 0;
    x2_camera camera{};
    x2_config config{};
    bool configured = false;
    float buildMs = 0.0f;
    // film
    double* sums = nullptr;
    double* odd = nullptr;
    uint32_t* counts = nullptr;
    uint32_t filmPixels = 0, samplesPerChunk = 0;
    bool adaptive = false;
    // launches
    Slot slots[kSlots];
    uint64_t nextSeq = 1;
    x2_chunk* staging = nullptr;  // pinned
    uint32_t stagingCap = 0;
    Counters total{};
    // the per-sample API's scratch (device pairs/outputs for host callers)
    Slot integrateSlot;
    unsigned long long* auditWord = nullptr;
    TraversalStats* stats = nullptr;  // device
    bool counting = false;
    float lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};  // the vertices' bounds
    // wavefront
    WaveState wave{};
    uint32_t wavePaths = 0, waveRecords = 0, reservePaths = 0;  // the last launch's paths; records a path
    uint32_t waveCap = 0;                                          // paths the wave's buffers hold
    uint32_t* extendQ = nullptr;
    uint32_t* shadowQ = nullptr;
    uint32_t* waveCounters = nullptr;  // kWaveCounters words
    uint32_t refill = kDefaultRefill;  // idle lanes that make a traversal warp fetch rays (0: one ray a thread)
    uint32_t blocksPerSm = kDefaultBlocksPerSm;  // traversal and shade grids: blocks a SM
    uint32_t traceBlocks = kDefaultTraceBlocks, shadeBlocks = kDefaultShadeBlocks;  // occupancy variants
    uint32_t triLimit = kDefaultTriLimit;  // triangle tests a traversal step
    uint32_t lobeQueues = 1;               // shade from per-lobe queues (wfSortShade)
    uint32_t shadowOrder = kDefaultShadowOrder;  // the shadow queue by record (1) or by path (0)
    uint32_t extendBins = kDefaultExtendBins;    // the extend queue binned by octant (1) or in slot order (0)
    uint32_t shortStack = kDefaultShortStack;    // traversal stacks' top entries in shared memory (1) or local (0)
    uint32_t shadeSplit = kDefaultShadeSplit;    // shade as one kernel a per-lobe queue (1) or one kernel (0)
    uint32_t lightSplit = kDefaultLightSplit;    // the lobe queues' light samples in kernels of their own (1)
    uint32_t triOverlap = kDefaultTriOverlap;    // a lane's node visits and triangle tests overlapped (1)
    uint32_t* shadeQ = nullptr;            // the per-lobe queues: 3 x wavePaths entries
    uint32_t batchWindow = 0;              // x2_render_batch: items a window (0: the default)
    uint32_t* hostLast = nullptr;      // pinned
    unsigned long long* claimed = nullptr;
    float4* out = nullptr;
    uint8_t* outStatus = nullptr;
    uint64_t outCap = 0, lastItems = 0;
    uint32_t waveIterations = 0;       // of the last wavefront launch
    // The asynchronous wavefront launch's drain: [0] its iterations, [1] a running total, [2] its overrun word
    // (device; 4 words), their host copy (pinned), the launch they belong to (0: none pending) and its bound.
    uint32_t* drainWords = nullptr;
    uint32_t* hostDrain = nullptr;
    uint64_t drainSeq = 0;
    uint32_t drainBound = 0;
    bool waveTiming = false;           // time each kernel kind (no graph)
    float waveMs[5] = {0, 0, 0, 0, 0}; // logic, extend, shade, shadow, film reduce
    uint32_t queueLog[2 * 4096] = {};  // timed launches: each iteration's extend and shadow queue sizes
    // an adaptive pass's launch: each chunk's pixel mask and each pixel's first sample index (device; null otherwise)
    const uint64_t* launchMask = nullptr;
    const uint32_t* launchBase = nullptr;
    // the adaptive frame's state (x2_render_adaptive, x2_adaptive_step)
    AdaptiveState* adaptiveState = nullptr;
    // the adjoint's wavefront state (x2_adjoint): vertex records, scales, counts, dL/dI shares, record auxiliaries
    uint4* avert = nullptr;
    float4* ascale = nullptr;
    uint32_t* avcount = nullptr;
    float4* adelta = nullptr;
    uint2* aaux = nullptr;
    float4* atex = nullptr;
    uint32_t adjPaths = 0, adjVerts = 0, adjRecords = 0;  // paths the adjoint's buffers hold; their vertices, records
};

namespace {

SceneView viewOf(const x2_scene* s) {
    SceneView v;
    v.bvh = Bvh8{s->bvh.nodes, s->bvh.tris, s->bvh.nodeCount, s->bvh.triCount, {s->lo[0], s->lo[1], s->lo[2]}, {s->hi[0], s->hi[1], s->hi[2]},
                 {s->bvh.rot[0], s->bvh.rot[1], s->bvh.tris}};
    v.triMesh = s->triMesh;
    v.meshFirst = s->meshFirst;
    v.meshMaterial = s->meshMaterial;
    v.materials = s->materials;
    v.lights = s->lights;
    v.camera = s->camera;
    v.config = s->config;
    v.overflow = s->overflow;
    v.stats = s->counting ? s->stats : nullptr;
    v.volumes = s->volumes;
    v.grids = s->grids;
    v.volumeTris = s->volumeTris;
    v.gridCount = s->gridCount;
    v.textures = s->textures;
    v.texels = s->texels;
    v.triUV = s->triUV;
    return v;
}

int ensureSlot(Slot& sl, uint32_t chunks) {
    if (!sl.begin) {
        CUDA_OR(cudaEventCreate(&sl.begin), X2_ECUDA);
        CUDA_OR(cudaEventCreate(&sl.end), X2_ECUDA);
        CUDA_OR(cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming), X2_ECUDA);
        CUDA_OR(cudaMalloc(&sl.claimed, sizeof(unsigned long long)), X2_ENOMEM);
        CUDA_OR(cudaMalloc(&sl.counters, sizeof(Counters)), X2_ENOMEM);
        CUDA_OR(cudaMallocHost(&sl.hostCounters, sizeof(Counters)), X2_ENOMEM);
        std::memset(sl.hostCounters, 0, sizeof(Counters));
    }
    if (chunks > sl.chunkCap) {
        if (sl.chunks) cudaFree(sl.chunks);
        sl.chunks = nullptr;
        const uint32_t cap = chunks < 1024 ? 1024 : chunks;
        CUDA_OR(cudaMalloc(&sl.chunks, sizeof(x2_chunk) * cap), X2_ENOMEM);
        sl.chunkCap = cap;
    }
    return X2_OK;
}
void freeSlot(Slot& sl) {
    if (sl.begin) cudaEventDestroy(sl.begin);
    if (sl.end) cudaEventDestroy(sl.end);
    if (sl.done) cudaEventDestroy(sl.done);
    if (sl.claimed) cudaFree(sl.claimed);
    if (sl.counters) cudaFree(sl.counters);
    if (sl.hostCounters) cudaFreeHost(sl.hostCounters);
    if (sl.chunks) cudaFree(sl.chunks);
    sl = Slot{};
}
void accumulate(Counters& t, const Counters& c) {
    t.trace += c.trace;
    t.nee += c.nee;
    t.bsdf += c.bsdf;
    t.held += c.held;
    t.samples += c.samples;
    t.errors += c.errors;
}

int checkDevice(x2_ctx* ctx) {
    if (!ctx) {
        setError("null context");
        return X2_EINVAL;
    }
    CUDA_OR(cudaSetDevice(ctx->device), X2_ECUDA);
    return X2_OK;
}

// Collects a finished slot (its end event has fired).
void retire(x2_scene* s, Slot& sl, x2_completion* out) {
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, sl.begin, sl.end);
    accumulate(s->total, *sl.hostCounters);
    if (out) {
        out->launch = sl.seq;
        out->samples = sl.hostCounters->samples;
        out->errors = sl.hostCounters->errors;
        out->milliseconds = ms;
        out->pad = 0;
    }
    sl.busy = false;
}

void freeWave(x2_scene* s) {
    WaveState& w = s->wave;
    void* ptrs[] = {w.ray0, w.ray1, w.T, w.held, w.meta, w.branch, w.rad, w.hit, w.state, w.item, w.ncount, w.sray0, w.sray1, w.scontrib, w.svis,
                    w.lightJob, w.lightFlags};
    for (void* p : ptrs) cudaFree(p);
    w = WaveState{};
    cudaFree(s->extendQ);
    cudaFree(s->shadowQ);
    cudaFree(s->shadeQ);
    s->extendQ = s->shadowQ = s->shadeQ = nullptr;
    s->wavePaths = s->waveRecords = s->waveCap = 0;
}

// The paths in flight when the caller reserved none: kDefaultPaths, or fewer (a power of two, at least 2^18) when the
// path state (slot, light job, queues and `records` shadow records a path) would pass kWaveBudgetBytes, as a scene with
// many lights would.
constexpr double kWaveBudgetBytes = 12e9;
static uint32_t defaultPaths(uint32_t records) {
    const double perPath = 128.0 + 16.0 * kLightJobWords + 4.0 * (kOctants + 3 + 1) + 53.0 * records;
    uint32_t paths = kDefaultPaths;
    while (paths > (1u << 18) && double(paths) * perPath > kWaveBudgetBytes) paths >>= 1;
    return paths;
}

// Path slots for `paths` paths with `records` shadow records each.
// Buffers that already hold at least `paths` paths are kept (a launch indexes them by its own path count), so launches
// of varying sizes (an adaptive frame's passes) allocate once.
int ensureWave(x2_scene* s, uint32_t paths, uint32_t records) {
    if (paths <= s->waveCap && s->waveRecords == records) {
        s->wavePaths = paths;
        return X2_OK;
    }
    freeWave(s);
    WaveState& w = s->wave;
    const size_t P = paths, R = size_t(paths) * records;
    bool ok = cudaMalloc(&w.ray0, sizeof(float4) * P) == cudaSuccess && cudaMalloc(&w.ray1, sizeof(float4) * P) == cudaSuccess &&
              cudaMalloc(&w.T, sizeof(float4) * P) == cudaSuccess && cudaMalloc(&w.held, sizeof(float4) * P) == cudaSuccess &&
              cudaMalloc(&w.meta, sizeof(uint4) * P) == cudaSuccess && cudaMalloc(&w.branch, sizeof(uint2) * P) == cudaSuccess &&
              cudaMalloc(&w.rad, sizeof(float4) * P) == cudaSuccess && cudaMalloc(&w.hit, sizeof(uint2) * P) == cudaSuccess &&
              cudaMalloc(&w.state, sizeof(uint32_t) * P) == cudaSuccess && cudaMalloc(&w.item, sizeof(uint32_t) * P) == cudaSuccess &&
              cudaMalloc(&w.ncount, sizeof(uint32_t) * P) == cudaSuccess && cudaMalloc(&w.sray0, sizeof(float4) * R) == cudaSuccess &&
              cudaMalloc(&w.sray1, sizeof(float4) * R) == cudaSuccess && cudaMalloc(&w.scontrib, sizeof(float4) * R) == cudaSuccess &&
              cudaMalloc(&w.svis, R) == cudaSuccess && cudaMalloc(&s->extendQ, sizeof(uint32_t) * kOctants * P) == cudaSuccess &&
              cudaMalloc(&s->shadowQ, sizeof(uint32_t) * R) == cudaSuccess && cudaMalloc(&s->shadeQ, sizeof(uint32_t) * 3 * P) == cudaSuccess &&
              cudaMalloc(&w.lightJob, sizeof(uint4) * kLightJobWords * P) == cudaSuccess &&
              cudaMalloc(&w.lightFlags, sizeof(uint32_t) * P) == cudaSuccess;
    if (ok && !s->waveCounters) ok = cudaMalloc(&s->waveCounters, sizeof(uint32_t) * kWaveCounters) == cudaSuccess;
    if (ok && !s->claimed) ok = cudaMalloc(&s->claimed, sizeof(unsigned long long)) == cudaSuccess;
    if (ok && !s->hostLast) ok = cudaMallocHost(&s->hostLast, sizeof(uint32_t) * 4) == cudaSuccess;
    if (ok && !s->drainWords) ok = cudaMalloc(&s->drainWords, sizeof(uint32_t) * 4) == cudaSuccess;
    if (ok && !s->hostDrain) ok = cudaMallocHost(&s->hostDrain, sizeof(uint32_t) * 4) == cudaSuccess;
    if (!ok) {
        freeWave(s);
        setError("device allocation failed for %u wavefront paths", paths);
        return X2_ENOMEM;
    }
    s->wavePaths = s->waveCap = paths;
    s->waveRecords = records;
    return X2_OK;
}

int ensureItems(x2_scene* s, uint64_t items) {
    if (items <= s->outCap) return X2_OK;
    cudaFree(s->out);
    cudaFree(s->outStatus);
    s->out = nullptr;
    s->outStatus = nullptr;
    s->outCap = 0;
    if (cudaMalloc(&s->out, sizeof(float4) * items) != cudaSuccess || cudaMalloc(&s->outStatus, items) != cudaSuccess) {
        setError("device allocation failed for %llu item outputs", (unsigned long long)items);
        return X2_ENOMEM;
    }
    s->outCap = items;
    return X2_OK;
}

}  // namespace

namespace x2 {
__global__ void addInto(double* dst, const double* src, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] += src[i];
}
__global__ void addFloatInto(double* dst, const float* src, uint64_t n) {
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) dst[i] += double(src[i]);
}

// The scene's device view, stream and device for entry points in other translation units (noalloc.cu).
int sceneView(x2_scene* s, SceneView* view, cudaStream_t* stream, int* device, int* smCount) {
    if (!s || !s->configured) {
        setError("scene not configured");
        return X2_EINVAL;
    }
    if (int rc = checkDevice(s->ctx)) return rc;
    *view = viewOf(s);
    *stream = s->ctx->stream;
    *device = s->ctx->device;
    *smCount = s->ctx->smCount;
    return X2_OK;
}
// A context's stream and SM count, its device current (probe.cu).
int contextStream(x2_ctx* ctx, cudaStream_t* stream, int* smCount) {
    if (!ctx) {
        setError("null context");
        return X2_EINVAL;
    }
    if (int rc = checkDevice(ctx)) return rc;
    *stream = ctx->stream;
    *smCount = ctx->smCount;
    return X2_OK;
}
}  // namespace x2

namespace {
// A volume's majorant grid: kMajorantCells^3 cells over its bounds, each a bound on the density any of the lookups
// can read at a point of the cell — the largest of the voxels whose index box the cell's corners span, one more each
// way, which bounds the nearest voxel and the trilinear lookup, times the quadratic lookup's overshoot when the volume
// uses it — times its largest gain channel; *largest the grid's maximum. Corners go to grid space by the volume's affine
// map and to index space by the grid's, so any affine placement stays conservative.
std::vector<float> majorantGrid(const x2_volume& v, const x2_grid* grids, uint32_t gridCount, float* largest) {
    const int n = x2::kMajorantCells;
    std::vector<float> out(size_t(n) * n * n, 0.0f);
    *largest = 0.0f;
    if (v.density_grid >= gridCount || grids[v.density_grid].channels != 1) return out;
    const x2_grid& g = grids[v.density_grid];
    // The quadratic lookup (interpolation 2) is a Lagrange quadratic through three voxels an axis, which at its
    // parameter w in [0, 1) reaches up to (1 + w - w^2) <= 1.25 times the largest of them: 1.25^3 over three axes.
    const float overshoot = v.interpolation == 2 ? 1.953125f : 1.0f;
    const float gain = overshoot * std::max(0.0f, std::max(v.gain[0], std::max(v.gain[1], v.gain[2])));
    auto toIndex = [&](double x, double y, double z, double out3[3]) {
        const float* a = v.world_to_grid;
        const double gx = a[0] * x + a[1] * y + a[2] * z + a[3], gy = a[4] * x + a[5] * y + a[6] * z + a[7], gz = a[8] * x + a[9] * y + a[10] * z + a[11];
        const double* m = g.world_to_index;
        for (int c = 0; c < 3; ++c) out3[c] = gx * m[c] + gy * m[4 + c] + gz * m[8 + c] + m[12 + c];
    };
    for (int k = 0; k < n; ++k)
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
                for (int corner = 0; corner < 8; ++corner) {
                    const int q[3] = {i + (corner & 1), j + (corner >> 1 & 1), k + (corner >> 2 & 1)};
                    double w[3], ix[3];
                    for (int a = 0; a < 3; ++a) w[a] = v.bound_lo[a] + (double(v.bound_hi[a]) - v.bound_lo[a]) * q[a] / n;
                    toIndex(w[0], w[1], w[2], ix);
                    for (int a = 0; a < 3; ++a) lo[a] = std::min(lo[a], ix[a]), hi[a] = std::max(hi[a], ix[a]);
                }
                int from[3], to[3];
                for (int a = 0; a < 3; ++a) {
                    from[a] = std::max(int(std::floor(lo[a])) - 1 - g.lo[a], 0);
                    to[a] = std::min(int(std::ceil(hi[a])) + 1 - g.lo[a], g.dims[a] - 1);
                }
                float most = 0.0f;
                for (int z = from[2]; z <= to[2]; ++z)
                    for (int y = from[1]; y <= to[1]; ++y)
                        for (int x = from[0]; x <= to[0]; ++x)
                            most = std::max(most, g.values[(size_t(z) * g.dims[1] + size_t(y)) * g.dims[0] + size_t(x)]);
                out[(size_t(k) * n + j) * n + i] = most * gain;
                *largest = std::max(*largest, most * gain);
            }
    return out;
}
}  // namespace

extern "C" {

const char* x2_version(void) { return "x2-b200 0.1 (sm_100a)"; }
const char* x2_last_error(void) { return g_error.c_str(); }

int x2_open(int device, x2_ctx** out) {
    if (!out) return X2_EINVAL;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        setError("no CUDA device");
        return X2_ENODEV;
    }
    if (device < 0 || device >= count) {
        setError("device %d out of range (%d devices)", device, count);
        return X2_EINVAL;
    }
    CUDA_OR(cudaSetDevice(device), X2_ECUDA);
    auto* ctx = new x2_ctx();
    ctx->device = device;
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
        setError("stream creation failed");
        delete ctx;
        return X2_ECUDA;
    }
    uint32_t dirs[17][32];
    sobolDirections(dirs);
    if (uploadSobol(dirs) != cudaSuccess || uploadSobolWavefront(dirs) != cudaSuccess || uploadSobolAdjoint(dirs) != cudaSuccess) {
        setError("sobol table upload failed");
        cudaStreamDestroy(ctx->stream);
        delete ctx;
        return X2_ECUDA;
    }
    cudaDeviceGetAttribute(&ctx->smCount, cudaDevAttrMultiProcessorCount, device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ctx->renderBlocksPerSm, renderChunks, kRenderBlock, 0);
    if (ctx->renderBlocksPerSm < 1) ctx->renderBlocksPerSm = 1;
    *out = ctx;
    return X2_OK;
}

int x2_close(x2_ctx* ctx) {
    if (!ctx) return X2_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    cudaStreamDestroy(ctx->stream);
    delete ctx;
    return X2_OK;
}

int x2_synchronize(x2_ctx* ctx, int timeoutMs) {
    if (int rc = checkDevice(ctx)) return rc;
    cudaEvent_t e;
    CUDA_OR(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), X2_ECUDA);
    cudaEventRecord(e, ctx->stream);
    const int rc = waitEvent(e, timeoutMs);
    cudaEventDestroy(e);
    return rc;
}

int x2_sample_words_device(x2_ctx* ctx, const x2_identity* ids, const uint32_t* dims, uint64_t n, uint32_t policy, uint32_t* out) {
    if (int rc = checkDevice(ctx)) return rc;
    if (!n) return X2_OK;
    if (!ids || !dims || !out) {
        setError("null array");
        return X2_EINVAL;
    }
    const int blocks = ctx->smCount * 8;
    sampleWords<<<blocks, 256, 0, ctx->stream>>>(ids, dims, n, policy, out);
    CUDA_OR(cudaGetLastError(), X2_ECUDA);
    return X2_OK;
}

int x2_sample_words(x2_ctx* ctx, const x2_identity* ids, const uint32_t* dims, uint64_t n, uint32_t policy, uint32_t* out) {
    if (int rc = checkDevice(ctx)) return rc;
    if (!n) return X2_OK;
    if (!ids || !dims || !out) {
        setError("null array");
        return X2_EINVAL;
    }
    x2_identity* dIds = nullptr;
    uint32_t *dDims = nullptr, *dOut = nullptr;
    CUDA_OR(cudaMallocAsync(&dIds, sizeof(x2_identity) * n, ctx->stream), X2_ENOMEM);
    CUDA_OR(cudaMallocAsync(&dDims, sizeof(uint32_t) * n, ctx->stream), X2_ENOMEM);
    CUDA_OR(cudaMallocAsync(&dOut, sizeof(uint32_t) * n, ctx->stream), X2_ENOMEM);
    cudaMemcpyAsync(dIds, ids, sizeof(x2_identity) * n, cudaMemcpyHostToDevice, ctx->stream);
    cudaMemcpyAsync(dDims, dims, sizeof(uint32_t) * n, cudaMemcpyHostToDevice, ctx->stream);
    int rc = x2_sample_words_device(ctx, dIds, dDims, n, policy, dOut);
    if (rc == X2_OK) cudaMemcpyAsync(out, dOut, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, ctx->stream);
    cudaFreeAsync(dIds, ctx->stream);
    cudaFreeAsync(dDims, ctx->stream);
    cudaFreeAsync(dOut, ctx->stream);
    const int w = x2_synchronize(ctx, 600000);
    return rc ? rc : w;
}

int x2_scene_load(x2_ctx* ctx, const x2_scene_desc* d, x2_scene** out) {
    if (int rc = checkDevice(ctx)) return rc;
    if (!d || !out || !d->vertices || !d->triangles || !d->mesh_first || !d->mesh_material || !d->materials ||
        (d->light_count && !d->lights) || d->triangle_count == 0 || d->mesh_count == 0) {
        setError("incomplete scene description");
        return X2_EINVAL;
    }
    // Admission (as the reference's plan admission rejects what its port does not carry).
    for (uint32_t i = 0; i < d->material_count; ++i) {
        const x2_material& m = d->materials[i];
        if (m.kind != X2_MAT_LAMBERT && m.kind != X2_MAT_GGX) {
            setError("material %u: unknown kind %u", i, m.kind);
            return X2_EINVAL;
        }
        if (m.diffuse_texture > d->texture_count) {
            setError("material %u: texture %u of %u", i, m.diffuse_texture - 1, d->texture_count);
            return X2_EINVAL;
        }
        if (m.kind == X2_MAT_GGX) {
            const bool specBlack = m.specular[0] <= 1e-6f && m.specular[1] <= 1e-6f && m.specular[2] <= 1e-6f;
            const bool diffBlack = m.diffuse[0] <= 1e-6f && m.diffuse[1] <= 1e-6f && m.diffuse[2] <= 1e-6f;
            if (!specBlack && !diffBlack) {
                setError("material %u: a GGX lobe over a diffuse base is not admitted", i);
                return X2_EINVAL;
            }
            if (!specBlack && !(m.roughness > 1e-6f)) {
                setError("material %u: a mirror (roughness 0) is not admitted", i);
                return X2_EINVAL;
            }
        }
    }
    for (uint32_t i = 0; i < d->texture_count; ++i) {
        const x2_texture& t = d->textures[i];
        if (!d->textures || !t.rgb || t.width == 0 || t.height == 0 || t.wrap > 1 || uint64_t(t.width) * t.height > (1ull << 28)) {
            setError("texture %u: %ux%u texels (at most 2^28), wrap %u (0 or 1)", i, t.width, t.height, t.wrap);
            return X2_EINVAL;
        }
    }
    for (uint32_t i = 0; i < d->light_count; ++i) {
        const x2_light& l = d->lights[i];
        if ((l.type != X2_LIGHT_ENV && l.type != X2_LIGHT_RECT && l.type != X2_LIGHT_DISTANT) || l.sidedness > X2_SIDE_TWO) {
            setError("light %u: type %u / sidedness %u not admitted", i, l.type, l.sidedness);
            return X2_EINVAL;
        }
    }
    if (d->volume_count > kDeviceVolumes || (d->volume_count && !d->volumes) || (d->grid_count && !d->grids)) {
        setError("at most %u volumes, with their records and grids", kDeviceVolumes);
        return X2_EINVAL;
    }
    for (uint32_t g = 0; g < d->grid_count; ++g) {
        const x2_grid& x = d->grids[g];
        if ((x.channels != 1 && x.channels != 3) || x.dims[0] <= 0 || x.dims[1] <= 0 || x.dims[2] <= 0 || !x.values) {
            setError("grid %u: 1 or 3 channels, positive dims, values", g);
            return X2_EINVAL;
        }
    }
    for (uint32_t v = 0; v < d->volume_count; ++v) {
        const x2_volume& x = d->volumes[v];
        if (x.density_grid >= d->grid_count || d->grids[x.density_grid].channels != 1 ||
            (x.emission_grid != kNoGrid && (x.emission_grid >= d->grid_count || d->grids[x.emission_grid].channels != 3)) ||
            x.interpolation > kInterpQuadratic || !(x.feature_size > 0.0f) || x.light_set != ~0u) {
            setError("volume %u: density grid (1 channel), emission grid (3 channels or none), interpolation 0..2, feature size > 0, "
                     "all lights (light sets not admitted)", v);
            return X2_EINVAL;
        }
        for (int k = 0; k < 3; ++k)
            if (!(x.bound_lo[k] < x.bound_hi[k])) {
                setError("volume %u: empty bounds", v);
                return X2_EINVAL;
            }
    }
    if (d->mesh_first[0] != 0 || d->mesh_first[d->mesh_count] != d->triangle_count) {
        setError("mesh ranges do not cover the triangles");
        return X2_EINVAL;
    }
    std::vector<uint32_t> triMesh(d->triangle_count);
    for (uint32_t m = 0; m < d->mesh_count; ++m) {
        if (d->mesh_first[m + 1] < d->mesh_first[m] || d->mesh_material[m] >= d->material_count) {
            setError("mesh %u: bad range or material", m);
            return X2_EINVAL;
        }
        for (uint32_t t = d->mesh_first[m]; t < d->mesh_first[m + 1]; ++t) triMesh[t] = m;
    }
    for (uint64_t i = 0; i < uint64_t(d->triangle_count) * 3; ++i)
        if (d->triangles[i] >= d->vertex_count) {
            setError("triangle %llu: vertex index out of range", (unsigned long long)(i / 3));
            return X2_EINVAL;
        }
    // The vertices' bounds. Coordinates are finite and within 1e14 of the origin: the traversal's slab arithmetic
    // (traverse.cuh visitNode) scales a node's quantum by 2^23 and must stay finite.
    float lo[3] = {3.402823466e38f, 3.402823466e38f, 3.402823466e38f}, hi[3] = {-3.402823466e38f, -3.402823466e38f, -3.402823466e38f};
    for (uint64_t i = 0; i < uint64_t(d->triangle_count) * 3; ++i)
        for (int k = 0; k < 3; ++k) {
            const float v = d->vertices[3 * size_t(d->triangles[i]) + k];
            if (!(fabsf(v) <= 1e14f)) {
                setError("triangle %llu: a vertex coordinate %g is not finite or beyond 1e14", (unsigned long long)(i / 3), double(v));
                return X2_EINVAL;
            }
            lo[k] = v < lo[k] ? v : lo[k];
            hi[k] = v > hi[k] ? v : hi[k];
        }
    auto* s = new x2_scene();
    s->ctx = ctx;
    s->camera = d->camera;
    for (int k = 0; k < 3; ++k) {
        s->lo[k] = lo[k];
        s->hi[k] = hi[k];
    }
    s->lightCount = d->light_count;
    s->triangleCount = d->triangle_count;
    s->materialCount = d->material_count;
    cudaStream_t st = ctx->stream;
    float* dVerts = nullptr;
    uint32_t* dTris = nullptr;
    std::vector<MaterialRec> mats(d->material_count);
    for (uint32_t i = 0; i < d->material_count; ++i) {
        const x2_material& m = d->materials[i];
        mats[i].kind = m.kind;
        for (int k = 0; k < 3; ++k) {
            mats[i].diffuse[k] = m.diffuse[k];
            mats[i].specular[k] = m.specular[k];
            mats[i].emission[k] = m.emission[k];
        }
        mats[i].roughness = m.roughness;
        mats[i].texture = m.diffuse_texture;
    }
    bool textured = false;
    for (uint32_t i = 0; i < d->material_count; ++i) textured = textured || d->materials[i].diffuse_texture != 0;
    // A scene with texture coordinates keeps them on the device even without a texture: they set the hits' partial
    // derivatives, as the reference binds them for every mesh.
    textured = textured || d->uvs != nullptr;
    cudaEvent_t b0, b1;
    cudaEventCreate(&b0);
    cudaEventCreate(&b1);
    auto fail = [&](int code) {
        cudaFree(dVerts);
        cudaFree(dTris);
        x2_scene_free(s);
        cudaEventDestroy(b0);
        cudaEventDestroy(b1);
        return code;
    };
    if (cudaMalloc(&dVerts, sizeof(float) * 3 * size_t(d->vertex_count)) != cudaSuccess ||
        cudaMalloc(&dTris, sizeof(uint32_t) * 3 * size_t(d->triangle_count)) != cudaSuccess ||
        cudaMalloc(&s->triMesh, sizeof(uint32_t) * d->triangle_count) != cudaSuccess ||
        cudaMalloc(&s->meshFirst, sizeof(uint32_t) * (d->mesh_count + 1)) != cudaSuccess ||
        cudaMalloc(&s->meshMaterial, sizeof(uint32_t) * d->mesh_count) != cudaSuccess ||
        cudaMalloc(&s->materials, sizeof(MaterialRec) * (d->material_count ? d->material_count : 1)) != cudaSuccess ||
        cudaMalloc(&s->lights, sizeof(x2_light) * (d->light_count ? d->light_count : 1)) != cudaSuccess ||
        cudaMalloc(&s->overflow, sizeof(uint32_t)) != cudaSuccess || cudaMalloc(&s->auditWord, sizeof(unsigned long long)) != cudaSuccess ||
        cudaMalloc(&s->stats, 2 * sizeof(TraversalStats)) != cudaSuccess) {
        setError("device allocation failed for the scene");
        return fail(X2_ENOMEM);
    }
    cudaMemcpyAsync(dVerts, d->vertices, sizeof(float) * 3 * size_t(d->vertex_count), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(dTris, d->triangles, sizeof(uint32_t) * 3 * size_t(d->triangle_count), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(s->triMesh, triMesh.data(), sizeof(uint32_t) * d->triangle_count, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(s->meshFirst, d->mesh_first, sizeof(uint32_t) * (d->mesh_count + 1), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(s->meshMaterial, d->mesh_material, sizeof(uint32_t) * d->mesh_count, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(s->materials, mats.data(), sizeof(MaterialRec) * d->material_count, cudaMemcpyHostToDevice, st);
    if (d->light_count) cudaMemcpyAsync(s->lights, d->lights, sizeof(x2_light) * d->light_count, cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(s->overflow, 0, sizeof(uint32_t), st);
    cudaMemsetAsync(s->stats, 0, 2 * sizeof(TraversalStats), st);
    // Textures: every texture's texels in one array; each triangle's vertices' st (hitState's st1..st3: the vertices'
    // uvs, or the default (0,0), (1,0), (1,1) of a mesh without them), when a material reads a texture.
    if (d->texture_count) {
        uint64_t total = 0;
        s->hostTextures.resize(d->texture_count);
        for (uint32_t i = 0; i < d->texture_count; ++i) {
            s->hostTextures[i] = TexRec{total, d->textures[i].width, d->textures[i].height, d->textures[i].wrap, 0};
            total += uint64_t(d->textures[i].width) * d->textures[i].height;
        }
        if (cudaMalloc(&s->textures, sizeof(TexRec) * d->texture_count) != cudaSuccess ||
            cudaMalloc(&s->texels, sizeof(float) * 3 * total) != cudaSuccess) {
            setError("device allocation failed for %llu texels", (unsigned long long)total);
            return fail(X2_ENOMEM);
        }
        cudaMemcpyAsync(s->textures, s->hostTextures.data(), sizeof(TexRec) * d->texture_count, cudaMemcpyHostToDevice, st);
        for (uint32_t i = 0; i < d->texture_count; ++i)
            cudaMemcpyAsync(s->texels + 3 * s->hostTextures[i].first, d->textures[i].rgb,
                            sizeof(float) * 3 * size_t(d->textures[i].width) * d->textures[i].height, cudaMemcpyHostToDevice, st);
    }
    if (textured) {
        std::vector<float> uv(size_t(d->triangle_count) * 6);
        for (uint32_t t = 0; t < d->triangle_count; ++t)
            for (int k = 0; k < 3; ++k) {
                const uint32_t v = d->triangles[3 * t + k];
                uv[6 * size_t(t) + 2 * k] = d->uvs ? d->uvs[2 * size_t(v)] : (k == 0 ? 0.0f : 1.0f);
                uv[6 * size_t(t) + 2 * k + 1] = d->uvs ? d->uvs[2 * size_t(v) + 1] : (k == 2 ? 1.0f : 0.0f);
            }
        if (cudaMalloc(&s->triUV, sizeof(float) * uv.size()) != cudaSuccess) {
            setError("device allocation failed for the triangles' st");
            return fail(X2_ENOMEM);
        }
        cudaMemcpyAsync(s->triUV, uv.data(), sizeof(float) * uv.size(), cudaMemcpyHostToDevice, st);
        CUDA_OR(cudaStreamSynchronize(st), fail(X2_ECUDA));
    }
    // Volumes: their records, their bounds' twelve triangles each (the oracle's table), their grids' values.
    s->volumeCount = d->volume_count;
    s->gridCount = d->grid_count;
    if (d->volume_count) {
        static const int kBox[12][3] = {{0, 4, 6}, {0, 6, 2}, {1, 3, 7}, {1, 7, 5}, {0, 1, 5}, {0, 5, 4},
                                        {2, 6, 7}, {2, 7, 3}, {0, 2, 3}, {0, 3, 1}, {4, 5, 7}, {4, 7, 6}};
        std::vector<VolumeRec> recs(d->volume_count);
        std::vector<float> tris;
        for (uint32_t v = 0; v < d->volume_count; ++v) {
            const x2_volume& x = d->volumes[v];
            VolumeRec& r = recs[v];
            for (int i = 0; i < 12; ++i) r.worldToGrid[i] = x.world_to_grid[i];
            r.gain = V3{x.gain[0], x.gain[1], x.gain[2]};
            r.colorMult = V3{x.color_mult[0], x.color_mult[1], x.color_mult[2]};
            r.incandescence = V3{x.incandescence[0], x.incandescence[1], x.incandescence[2]};
            r.g = x.g;
            r.featureSize = x.feature_size;
            r.surfaceThreshold = x.surface_opacity_threshold;
            r.densityGrid = x.density_grid;
            r.emissionGrid = x.emission_grid;
            r.interpolation = x.interpolation;
            r.lo = V3{x.bound_lo[0], x.bound_lo[1], x.bound_lo[2]};
            r.hi = V3{x.bound_hi[0], x.bound_hi[1], x.bound_hi[2]};
            r.majorant = nullptr;
            r.majorantMax = 0.0f;
            if (!(x.gain[0] == x.gain[1] && x.gain[1] == x.gain[2])) s->greyVolumes = false;
            for (const auto& t : kBox)
                for (int k = 0; k < 3; ++k)
                    for (int a = 0; a < 3; ++a) tris.push_back((t[k] >> a) & 1 ? x.bound_hi[a] : x.bound_lo[a]);
        }
        std::vector<GridRec> grids(d->grid_count);
        s->gridValues.assign(d->grid_count, nullptr);
        bool ok = cudaMalloc(&s->volumes, sizeof(VolumeRec) * d->volume_count) == cudaSuccess &&
                  cudaMalloc(&s->volumeTris, sizeof(float) * tris.size()) == cudaSuccess &&
                  cudaMalloc(&s->grids, sizeof(GridRec) * (d->grid_count ? d->grid_count : 1)) == cudaSuccess;
        for (uint32_t g = 0; ok && g < d->grid_count; ++g) {
            const x2_grid& x = d->grids[g];
            const size_t n = size_t(x.dims[0]) * x.dims[1] * x.dims[2] * x.channels;
            ok = cudaMalloc(&s->gridValues[g], sizeof(float) * n) == cudaSuccess;
            if (!ok) break;
            cudaMemcpyAsync(s->gridValues[g], x.values, sizeof(float) * n, cudaMemcpyHostToDevice, st);
            GridRec& r = grids[g];
            for (int i = 0; i < 16; ++i) r.worldToIndex[i] = x.world_to_index[i];
            r.values = s->gridValues[g];
            for (int a = 0; a < 3; ++a) r.lo[a] = x.lo[a], r.dims[a] = x.dims[a];
            r.channels = x.channels;
        }
        // Each volume's majorant grid for the tracking estimator.
        std::vector<std::vector<float>> majorant(d->volume_count);
        s->majorants.assign(d->volume_count, nullptr);
        for (uint32_t v = 0; ok && v < d->volume_count; ++v) {
            majorant[v] = majorantGrid(d->volumes[v], d->grids, d->grid_count, &recs[v].majorantMax);
            ok = cudaMalloc(&s->majorants[v], sizeof(float) * majorant[v].size()) == cudaSuccess;
            if (!ok) break;
            cudaMemcpyAsync(s->majorants[v], majorant[v].data(), sizeof(float) * majorant[v].size(), cudaMemcpyHostToDevice, st);
            recs[v].majorant = s->majorants[v];
        }
        if (!ok) {
            setError("device allocation failed for the volumes");
            return fail(X2_ENOMEM);
        }
        cudaMemcpyAsync(s->volumes, recs.data(), sizeof(VolumeRec) * recs.size(), cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(s->volumeTris, tris.data(), sizeof(float) * tris.size(), cudaMemcpyHostToDevice, st);
        if (d->grid_count) cudaMemcpyAsync(s->grids, grids.data(), sizeof(GridRec) * grids.size(), cudaMemcpyHostToDevice, st);
        // The copies read host vectors that go out of scope here.
        if (cudaStreamSynchronize(st) != cudaSuccess) {
            setError("volume upload failed");
            return fail(X2_ECUDA);
        }
    }
    cudaEventRecord(b0, st);
    if (buildBvh(dVerts, dTris, d->triangle_count, st, &s->bvh) != 0) return fail(X2_ECUDA);
    cudaEventRecord(b1, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) {
        setError("scene upload failed: %s", cudaGetErrorString(cudaGetLastError()));
        return fail(X2_ECUDA);
    }
    cudaEventElapsedTime(&s->buildMs, b0, b1);
    cudaEventDestroy(b0);
    cudaEventDestroy(b1);
    cudaFree(dVerts);
    cudaFree(dTris);
    *out = s;
    return X2_OK;
}

void freeAdjointWave(x2_scene* s) {
    cudaFree(s->avert);
    cudaFree(s->ascale);
    cudaFree(s->avcount);
    cudaFree(s->adelta);
    cudaFree(s->aaux);
    cudaFree(s->atex);
    s->atex = nullptr;
    s->avert = nullptr;
    s->ascale = nullptr;
    s->avcount = nullptr;
    s->adelta = nullptr;
    s->aaux = nullptr;
    s->adjPaths = s->adjVerts = s->adjRecords = 0;
}

int x2_scene_free(x2_scene* s) {
    if (!s) return X2_OK;
    if (s->ctx) cudaSetDevice(s->ctx->device);
    if (s->ctx) cudaStreamSynchronize(s->ctx->stream);
    freeAdjointWave(s);
    delete s->adaptiveState;
    s->adaptiveState = nullptr;
    cudaFree(s->bvh.nodes);
    cudaFree(s->bvh.tris);
    cudaFree(s->bvh.rot[0]);
    cudaFree(s->bvh.rot[1]);
    cudaFree(s->triMesh);
    cudaFree(s->meshFirst);
    cudaFree(s->meshMaterial);
    cudaFree(s->materials);
    cudaFree(s->textures);
    cudaFree(s->texels);
    cudaFree(s->triUV);
    cudaFree(s->lights);
    cudaFree(s->overflow);
    cudaFree(s->auditWord);
    cudaFree(s->stats);
    cudaFree(s->volumes);
    cudaFree(s->volumeTris);
    cudaFree(s->grids);
    for (float* g : s->gridValues) cudaFree(g);
    for (float* m : s->majorants) cudaFree(m);
    freeWave(s);
    cudaFree(s->out);
    cudaFree(s->outStatus);
    cudaFree(s->extendQ);
    cudaFree(s->shadowQ);
    cudaFree(s->waveCounters);
    cudaFree(s->claimed);
    if (s->hostLast) cudaFreeHost(s->hostLast);
    cudaFree(s->drainWords);
    if (s->hostDrain) cudaFreeHost(s->hostDrain);
    cudaFree(s->sums);
    cudaFree(s->odd);
    cudaFree(s->counts);
    for (auto& sl : s->slots) freeSlot(sl);
    freeSlot(s->integrateSlot);
    if (s->staging) cudaFreeHost(s->staging);
    delete s;
    return X2_OK;
}

int x2_config_set(x2_scene* s, const x2_config* c) {
    if (!s || !c) return X2_EINVAL;
    if (c->width == 0 || c->height == 0 || uint64_t(c->width) * c->height > 0xffffffffull) {
        setError("bad image size %ux%u", c->width, c->height);
        return X2_EINVAL;
    }
    if (c->filter != X2_FILTER_BOX) {
        setError("filter %u not admitted (box only)", c->filter);
        return X2_EINVAL;
    }
    if (c->light_count != s->lightCount) {
        setError("config light_count %u differs from the scene's %u lights", c->light_count, s->lightCount);
        return X2_EINVAL;
    }
    if (c->bsdf_samples == 0 || c->bsdf_samples > 64 || c->light_samples == 0 || c->light_samples > 64) {
        setError("bsdf/light samples out of [1, 64]");
        return X2_EINVAL;
    }
    if (c->volume_count != s->volumeCount) {
        setError("config volume_count %u differs from the scene's %u volumes", c->volume_count, s->volumeCount);
        return X2_EINVAL;
    }
    if (c->volume_count && (c->max_volume_depth > 64 || c->volume_overlap_mode > kOverlapRnd || c->max_depth > 120)) {
        setError("volumes: max_volume_depth <= 64, overlap mode 0..2, max_depth <= 120");
        return X2_EINVAL;
    }
    if (c->volume_estimator > 1 ||
        (c->volume_estimator == 1 && c->volume_count &&
         (!s->greyVolumes || c->max_volume_depth > 1 || c->volume_overlap_mode == kOverlapRnd))) {
        setError("volume_estimator: 0 (march) or 1 (tracking: grey extinction, max_volume_depth <= 1, overlap sum or max)");
        return X2_EINVAL;
    }
    s->config = *c;
    s->configured = true;
    return X2_OK;
}

int x2_scene_info(x2_scene* s, uint64_t* nodes, uint64_t* bvhBytes, uint64_t* triBytes, float* buildMs) {
    if (!s) return X2_EINVAL;
    if (nodes) *nodes = s->bvh.nodeCount;
    if (bvhBytes) *bvhBytes = uint64_t(s->bvh.nodeCount) * sizeof(Node8);
    if (triBytes) *triBytes = uint64_t(s->bvh.triCount) * sizeof(TriRec) * 3;  // the leaf-order triangles and their two rotations
    if (buildMs) *buildMs = s->buildMs;
    return X2_OK;
}

int x2_integrate_device(x2_scene* s, const uint32_t* pairs, uint64_t n, double* rgba, uint32_t* status) {
    if (!s || !s->configured) {
        setError("scene not configured");
        return X2_EINVAL;
    }
    if (int rc = checkDevice(s->ctx)) return rc;
    if (!n) return X2_OK;
    if (int rc = ensureSlot(s->integrateSlot, 1)) return rc;
    Slot& sl = s->integrateSlot;
    cudaStream_t st = s->ctx->stream;
    cudaMemsetAsync(sl.counters, 0, sizeof(Counters), st);
    const int blocks = s->ctx->smCount * s->ctx->renderBlocksPerSm;
    (s->volumeCount ? integratePairsVolumes : s->triUV ? integratePairsTextured : integratePairs)<<<blocks, kRenderBlock, 0, st>>>(
        viewOf(s), pairs, n, rgba, status, sl.counters);
    CUDA_OR(cudaGetLastError(), X2_ECUDA);
    cudaMemcpyAsync(sl.hostCounters, sl.counters, sizeof(Counters), cudaMemcpyDeviceToHost, st);
    cudaEventRecord(sl.done, st);
    sl.busy = true;
    return X2_OK;
}

int x2_integrate(x2_scene* s, const uint32_t* pairs, uint64_t n, double* rgba, uint32_t* status) {
    if (!s || !s->configured) {
        setError("scene not configured");
        return X2_EINVAL;
    }
    if (int rc = checkDevice(s->ctx)) return rc;
    if (!n) return X2_OK;
    if (!pairs || !rgba || !status) {
        setError("null array");
        return X2_EINVAL;
    }
    cudaStream_t st = s->ctx->stream;
    uint32_t *dPairs = nullptr, *dStatus = nullptr;
    double* dRgba = nullptr;
    CUDA_OR(cudaMallocAsync(&dPairs, sizeof(uint32_t) * 2 * n, st), X2_ENOMEM);
    CUDA_OR(cudaMallocAsync(&dRgba, sizeof(double) * 4 * n, st), X2_ENOMEM);
    CUDA_OR(cudaMallocAsync(&dStatus, sizeof(uint32_t) * n, st), X2_ENOMEM);
    cudaMemcpyAsync(dPairs, pairs, sizeof(uint32_t) * 2 * n, cudaMemcpyHostToDevice, st);
    int rc = x2_integrate_device(s, dPairs, n, dRgba, dStatus);
    if (rc == X2_OK) {
        cudaMemcpyAsync(rgba, dRgba, sizeof(double) * 4 * n, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(status, dStatus, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, st);
    }
    cudaFreeAsync(dPairs, st);
    cudaFreeAsync(dRgba, st);
    cudaFreeAsync(dStatus, st);
    const int w = x2_synchronize(s->ctx, 600000);
    if (rc == X2_OK && w == X2_OK && s->integrateSlot.busy) {
        accumulate(s->total, *s->integrateSlot.hostCounters);
        s->integrateSlot.busy = false;
    }
    return rc ? rc : w;
}

int x2_trace_rays_device(x2_scene* s, const float* rays, uint64_t n, uint32_t* tri, float* t, uint32_t* occluded) {
    if (!s) return X2_EINVAL;
    if (int rc = checkDevice(s->ctx)) return rc;
    if (!n) return X2_OK;
    if (!rays) {
        setError("null rays");
        return X2_EINVAL;
    }
    traceRays<<<s->ctx->smCount * 8, 128, 0, s->ctx->stream>>>(viewOf(s), rays, n, tri, t, occluded);
    CUDA_OR(cudaGetLastError(), X2_ECUDA);
    return X2_OK;
}

int x2_trace_rays(x2_scene* s, const float* rays, uint64_t n, uint32_t* tri, float* t, uint32_t* occluded) {
    if (!s) return X2_EINVAL;
    if (int rc = checkDevice(s->ctx)) return rc;
    if (!n) return X2_OK;
    if (!rays || !tri || !t || !occluded) {
        setError("null array");
        return X2_EINVAL;
    }
    cudaStream_t st = s->ctx->stream;
    float *dRays = nullptr, *dT = nullptr;
    uint32_t *dTri = nullptr, *dOcc = nullptr;
    CUDA_OR(cudaMallocAsync(&dRays, sizeof(float) * 8 * n, st), X2_ENOMEM);
    CUDA_OR(cudaMallocAsync(&dT, sizeof(float) * n, st), X2_ENOMEM);
    CUDA_OR(cudaMallocAsync(&dTri, sizeof(uint32_t) * n, st), X2_ENOMEM);
    CUDA_OR(cudaMallocAsync(&dOcc, sizeof(uint32_t) * n, st), X2_ENOMEM);
    cudaMemcpyAsync(dRays, rays, sizeof(float) * 8 * n, cudaMemcpyHostToDevice, st);
    const int rc = x2_trace_rays_device(s, dRays, n, dTri, dT, dOcc);
    if (rc == X2_OK) {
        cudaMemcpyAsync(tri, dTri, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(t, dT, sizeof(float) * n, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(occluded, dOcc, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, st);
    }
    cudaFreeAsync(dRays, st);
    cudaFreeAsync(dT, st);
    cudaFreeAsync(dTri, st);
    cudaFreeAsync(dOcc, st);
    const int w = x2_synchronize(s->ctx, 600000);
    return rc ? rc : w;
}

int x2_frame_begin(x2_scene* s, uint32_t samplesPerChunk) {
    if (!s || !s->configured || samplesPerChunk == 0) {
        setError("scene not configured or zero samples a chunk");
        return X2_EINVAL;
    }
    if (int rc = checkDevice(s->ctx)) return rc;
    // No launch of the previous frame may still write the film.
    if (int rc = x2_wait(s, 600000, nullptr)) return rc;
    const uint32_t pixels = s->config.width * s->config.height;
    cudaStream_t st = s->ctx->stream;
    if (pixels != s->filmPixels) {
        cudaFree(s->sums);
        cudaFree(s->odd);
        cudaFree(s->counts);
        s->sums = s->odd = nullptr;
        s->counts = nullptr;
        CUDA_OR(cudaMalloc(&s->sums, sizeof(double) * 4 * size_t(pixels)), X2_ENOMEM);
        CUDA_OR(cudaMalloc(&s->odd, sizeof(double) * 4 * size_t(pixels)), X2_ENOMEM);
        CUDA_OR(cudaMalloc(&s->counts, sizeof(uint32_t) * size_t(pixels)), X2_ENOMEM);
        s->filmPixels = pixels;
    }
    cudaMemsetAsync(s->sums, 0, sizeof(double) * 4 * size_t(pixels), st);
    cudaMemsetAsync(s->odd, 0, sizeof(double) * 4 * size_t(pixels), st);
    cudaMemsetAsync(s->counts, 0, sizeof(uint32_t) * size_t(pixels), st);
    cudaMemsetAsync(s->overflow, 0, sizeof(uint32_t), st);
    s->samplesPerChunk = samplesPerChunk;
    s->adaptive = false;
    CUDA_OR(cudaGetLastError(), X2_ECUDA);
    return X2_OK;
}

int x2_frame_begin_adaptive(x2_scene* s, uint32_t samplesPerChunk) {
    if (int rc = x2_frame_begin(s, samplesPerChunk)) return rc;
    s->adaptive = true;
    if (s->adaptiveState) {
        AdaptiveState& a = *s->adaptiveState;
        cudaMemsetAsync(a.planned, 0, sizeof(uint32_t) * size_t(a.width) * a.height, s->ctx->stream);
        cudaMemsetAsync(a.base, 0, sizeof(uint32_t) * size_t(a.width) * a.height, s->ctx->stream);
        cudaMemsetAsync(a.stop, 0, sizeof(uint32_t), s->ctx->stream);
    }
    CUDA_OR(cudaGetLastError(), X2_ECUDA);
    return X2_OK;
}

int x2_launch(x2_scene* s, const x2_chunk* chunks, uint32_t count) {
    if (!s || !s->configured || !s->filmPixels || !s->samplesPerChunk) {
        setError("x2_frame_begin first");
        return X2_EINVAL;
    }
    if (int rc = checkDevice(s->ctx)) return rc;
    if (!count) return X2_OK;
    if (!chunks) return X2_EINVAL;
    const uint32_t tiles = ((s->config.width + 7) / 8) * ((s->config.height + 7) / 8);
    for (uint32_t i = 0; i < count; ++i)
        if (chunks[i].tile >= tiles || chunks[i].count > s->samplesPerChunk) {
            setError("chunk %u: tile %u of %u or count %u over %u samples a chunk", i, chunks[i].tile, tiles, chunks[i].count,
                     s->samplesPerChunk);
            return X2_EINVAL;
        }
    // A free slot: at most two launches in flight; wait (bounded) for the older one otherwise.
    Slot* sl = nullptr;
    for (auto& c : s->slots)
        if (!c.busy) sl = &c;
    if (!sl) {
        Slot* oldest = &s->slots[0];
        for (auto& c : s->slots)
            if (c.seq < oldest->seq) oldest = &c;
        if (int rc = waitEvent(oldest->done, 600000)) return rc;
        retire(s, *oldest, nullptr);
        sl = oldest;
    }
    if (int rc = ensureSlot(*sl, count)) return rc;
    cudaStream_t st = s->ctx->stream;
    CUDA_OR(cudaMemcpyAsync(sl->chunks, chunks, sizeof(x2_chunk) * count, cudaMemcpyHostToDevice, st), X2_ECUDA);
    cudaMemsetAsync(sl->claimed, 0, sizeof(unsigned long long), st);
    cudaMemsetAsync(sl->counters, 0, sizeof(Counters), st);
    RenderArgs a;
    a.scene = viewOf(s);
    a.chunks = sl->chunks;
    a.samplesPerChunk = s->samplesPerChunk;
    a.itemCount = (unsigned long long)count * 64ull * s->samplesPerChunk;
    a.claimed = sl->claimed;
    a.sums = s->sums;
    a.odd = s->adaptive ? s->odd : nullptr;
    a.counts = s->counts;
    a.counters = sl->counters;
    // The bounce-at-a-time form for surface scenes (renderSteps); renderChunks for volumes, counting launches and
    // vertices with more shadow rays than its list holds.
    void (*kernel)(RenderArgs) = s->volumeCount ? renderChunksVolumes : s->triUV ? renderChunksTextured : renderChunks;
    if (!s->volumeCount && !a.scene.stats &&
        uint64_t(s->config.light_count) * s->config.light_samples + s->config.bsdf_samples <= kStepRecords)
        kernel = s->triUV ? renderStepsTextured<4> : renderSteps<4>;
    int perSm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kernel, kRenderBlock, 0);
    const int blocks = s->ctx->smCount * std::max(perSm, 1);
    cudaEventRecord(sl->begin, st);
    kernel<<<blocks, kRenderBlock, 0, st>>>(a);
    CUDA_OR(cudaGetLastError(), X2_ECUDA);
    cudaEventRecord(sl->end, st);
    cudaMemcpyAsync(sl->hostCounters, sl->counters, sizeof(Counters), cudaMemcpyDeviceToHost, st);
    cudaEventRecord(sl->done, st);
    sl->busy = true;
    sl->seq = s->nextSeq++;
    return X2_OK;
}

int x2_poll(x2_scene* s, x2_completion* out) {
    if (!s) return X2_EINVAL;
    Slot* oldest = nullptr;
    for (auto& c : s->slots)
        if (c.busy && (!oldest || c.seq < oldest->seq)) oldest = &c;
    if (!oldest) return 0;
    const cudaError_t q = cudaEventQuery(oldest->done);
    if (q == cudaErrorNotReady) return 0;
    if (q != cudaSuccess) {
        setError("launch failed: %s", cudaGetErrorString(q));
        return -X2_ECUDA;
    }
    const uint64_t seq = oldest->seq;
    retire(s, *oldest, out);
    if (s->drainSeq && seq == s->drainSeq) {  // an asynchronous wavefront launch: its drain's outcome
        s->drainSeq = 0;
        s->waveIterations = s->hostDrain[0];
        if (s->hostDrain[2]) {
            setError("wavefront did not drain after %u iterations", s->drainBound);
            return -X2_EDEVICE;
        }
    }
    return 1;
}

int x2_wait(x2_scene* s, int timeoutMs, x2_completion* out) {
    if (!s) return X2_EINVAL;
    if (out) std::memset(out, 0, sizeof(*out));
    if (int rc = x2_synchronize(s->ctx, timeoutMs)) return rc;
    for (;;) {
        x2_completion c;
        const int r = x2_poll(s, &c);
        if (r < 0) return -r;
        if (r == 0) break;
        if (out) {
            out->launch = c.launch;
            out->samples += c.samples;
            out->errors += c.errors;
            out->milliseconds += c.milliseconds;
        }
    }
    return X2_OK;
}

int x2_render_frame(x2_scene* s, uint32_t first, uint32_t count) {
    if (!s || !s->configured) return X2_EINVAL;
    if (!s->filmPixels || s->samplesPerChunk < count) {
        setError("x2_frame_begin with at least %u samples a chunk first", count);
        return X2_EINVAL;
    }
    const uint32_t tiles = ((s->config.width + 7) / 8) * ((s->config.height + 7) / 8);
    // Staging must not be rewritten while an earlier launch's copy may still read it: wait for the stream.
    if (int rc = x2_synchronize(s->ctx, 600000)) return rc;
    if (tiles > s->stagingCap) {
        if (s->staging) cudaFreeHost(s->staging);
        s->staging = nullptr;
        CUDA_OR(cudaMallocHost(&s->staging, sizeof(x2_chunk) * tiles), X2_ENOMEM);
        s->stagingCap = tiles;
    }
    for (uint32_t t = 0; t < tiles; ++t) s->staging[t] = x2_chunk{t, first, count, 0};
    return x2_launch(s, s->staging, tiles);
}

int x2_wavefront_reserve(x2_scene* s, uint32_t paths) {
    if (!s) return X2_EINVAL;
    s->reservePaths = paths;
    return X2_OK;
}

void x2_wavefront_shape_defaults(x2_wavefront_shape* shape) {
    if (!shape) return;
    *shape = x2_wavefront_shape{};
    shape->refill = kDefaultRefill;
    shape->blocks_per_sm = kDefaultBlocksPerSm;
    shape->trace_blocks = kDefaultTraceBlocks;
    shape->shade_blocks = kDefaultShadeBlocks;
    shape->tri_limit = kDefaultTriLimit;
    shape->lobe_queues = 1;
    shape->shadow_order = kDefaultShadowOrder;
    shape->extend_bins = kDefaultExtendBins;
    shape->short_stack = kDefaultShortStack;
    shape->shade_split = kDefaultShadeSplit;
    shape->light_split = kDefaultLightSplit;
    shape->tri_overlap = kDefaultTriOverlap;
}

int x2_wavefront_tune(x2_scene* s, const x2_wavefront_shape* shape) {
    if (!s || !shape || shape->refill < 1 || shape->refill > 32 || shape->blocks_per_sm < 1 || shape->blocks_per_sm > 32 ||
        shape->trace_blocks > 32 || shape->shade_blocks > 32 || shape->tri_limit < 1 || shape->tri_limit > 32 || shape->lobe_queues > 1 ||
        shape->shadow_order > 1 || shape->extend_bins > 1 || shape->short_stack > 1 || shape->shade_split > 1 ||
        shape->light_split > 2 || shape->tri_overlap > 1) {
        setError("refill is 1..32 lanes, blocks_per_sm 1..32, trace_blocks and shade_blocks 0..32, tri_limit 1..32, lobe_queues, "
                 "shadow_order, extend_bins, short_stack and shade_split 0 or 1, light_split 0..2, tri_overlap 0 or 1");
        return X2_EINVAL;
    }
    s->reservePaths = shape->paths;
    s->refill = shape->refill;
    s->blocksPerSm = shape->blocks_per_sm;
    s->traceBlocks = shape->trace_blocks;
    s->shadeBlocks = shape->shade_blocks;
    s->triLimit = shape->tri_limit;
    s->batchWindow = shape->batch_window;
    s->lobeQueues = shape->lobe_queues;
    s->shadowOrder = shape->shadow_order;
    s->extendBins = shape->extend_bins;
    s->shortStack = shape->short_stack;
    s->shadeSplit = shape->shade_split;
    s->lightSplit = shape->light_split;
    s->triOverlap = shape->tri_overlap;
    return X2_OK;
}

namespace {
// A single scene's wavefront launch of `count` chunks (sl.chunks) and `items` items over `paths` path slots.
WaveArgs launchArgs(x2_scene* s, Slot& sl, uint32_t paths, uint32_t records, unsigned long long items, uint32_t count) {
    WaveArgs a;
    a.scene = viewOf(s);
    a.w = s->wave;
    a.paths = paths;
    a.recordsPerPath = records;
    a.chunks = sl.chunks;
    a.itemCount = items;
    a.samplesPerChunk = s->samplesPerChunk;
    a.claimed = s->claimed;
    a.extendQ = s->extendQ;
    a.extendCount = s->waveCounters;
    a.lastExtend = s->waveCounters + 1;
    a.shadowQ = s->shadowQ;
    a.shadowCount = s->waveCounters + 2;
    a.shadowSlots = s->shadowOrder && a.recordsPerPath <= x2::kRecordSegments ? s->waveCounters + 8 : nullptr;
    a.extendSlots = s->extendBins ? s->waveCounters + 8 + x2::kRecordSegments : nullptr;
    a.extendNext = s->waveCounters + 3;
    a.shadowNext = s->waveCounters + 4;
    // Volume scenes are shaded in the extend queue's order: its neighbouring slots hold samples of one pixel, whose
    // marches are alike; a per-lobe sort (or one by march length) scatters them and the march's lanes diverge more.
    a.shadeQ = s->lobeQueues && !s->volumeCount ? s->shadeQ : nullptr;
    a.shadeCount = s->waveCounters + 5;
    a.adj = AdjointWave{};
    a.chunkMask = s->launchMask;
    a.pixelBase = s->launchBase;
    a.liveChunks = nullptr;
    a.refill = s->refill;
    a.triLimit = s->triLimit;
    a.out = s->out;
    a.outStatus = s->outStatus;
    a.counters = sl.counters;
    a.scenes = nullptr;
    a.chunkRequest = nullptr;
    a.chunkItems = nullptr;
    a.chunkCount = count;
    return a;
}
}  // namespace

int x2_launch_wavefront(x2_scene* s, const x2_chunk* chunks, uint32_t count) {
    if (!s || !s->configured || !s->filmPixels || !s->samplesPerChunk) {
        setError("x2_frame_begin first");
        return X2_EINVAL;
    }
    if (s->config.bsdf_samples != 1) {
        setError("the wavefront form takes one BSDF sample a lobe (bsdf_samples = 1)");
        return X2_EINVAL;
    }
    if (int rc = checkDevice(s->ctx)) return rc;
    if (!count) return X2_OK;
    if (!chunks) return X2_EINVAL;
    const uint32_t tiles = ((s->config.width + 7) / 8) * ((s->config.height + 7) / 8);
    for (uint32_t i = 0; i < count; ++i)
        if (chunks[i].tile >= tiles || chunks[i].count > s->samplesPerChunk) {
            setError("chunk %u: tile %u of %u or count %u over %u samples a chunk", i, chunks[i].tile, tiles, chunks[i].count,
                     s->samplesPerChunk);
            return X2_EINVAL;
        }
    // Every earlier launch has finished: the wavefront's host loop waits on the stream anyway.
    if (int rc = x2_wait(s, 600000, nullptr)) return rc;
    Slot& sl = s->slots[0];
    if (int rc = ensureSlot(sl, count)) return rc;
    const unsigned long long items = (unsigned long long)count * 64ull * s->samplesPerChunk;
    if (items > 0xffffffffull) {
        setError("%llu work items in one wavefront launch (at most 2^32 - 1)", items);
        return X2_EINVAL;
    }
    const uint32_t records = s->config.light_count * s->config.light_samples + 1;
    uint32_t paths = s->reservePaths ? s->reservePaths : defaultPaths(records);
    if (paths > items) paths = uint32_t(items < 1024 ? 1024 : items);
    if (int rc = ensureWave(s, paths, records)) return rc;
    if (int rc = ensureItems(s, items)) return rc;
    cudaStream_t st = s->ctx->stream;
    CUDA_OR(cudaMemcpyAsync(sl.chunks, chunks, sizeof(x2_chunk) * count, cudaMemcpyHostToDevice, st), X2_ECUDA);
    cudaMemsetAsync(s->wave.state, 0, sizeof(uint32_t) * paths, st);
    cudaMemsetAsync(s->wave.ncount, 0, sizeof(uint32_t) * paths, st);
    cudaMemsetAsync(s->claimed, 0, sizeof(unsigned long long), st);
    cudaMemsetAsync(s->waveCounters, 0, sizeof(uint32_t) * kWaveCounters, st);
    cudaMemsetAsync(sl.counters, 0, sizeof(Counters), st);
    cudaMemsetAsync(s->outStatus, X2_SKIP, items, st);
    const WaveArgs a = launchArgs(s, sl, paths, records, items, count);
    const int gridLogic = int((paths + kWaveBlock - 1) / kWaveBlock);
    const int gridWork = s->ctx->smCount * int(s->blocksPerSm);
    const WaveKernels wk = waveKernels(s->traceBlocks, s->shadeBlocks, s->volumeCount != 0, s->triUV != nullptr, s->shortStack != 0,
                                       a.scene.stats != nullptr, s->shadeSplit != 0,
                                       s->wave.lightJob != nullptr ? s->lightSplit : 0u, s->triOverlap != 0 && s->shortStack != 0 && s->traceBlocks < 9);
    const uint64_t maxIter = items * (uint64_t(s->config.max_depth) + 2) / paths + uint64_t(s->config.max_depth) + 64;
    if (s->waveTiming) {
        // Diagnostic form: no graph; events around every kernel, the iteration's times added once it is done.
        cudaEvent_t ev[6];
        for (auto& e : ev) cudaEventCreate(&e);
        for (float& m : s->waveMs) m = 0.0f;
        cudaEventRecord(sl.begin, st);
        uint32_t iterations = 0;
        int rc = X2_OK;
        for (;;) {
            wfResetQueues<<<1, 32, 0, st>>>(a);
            cudaEventRecord(ev[0], st);
            wk.logic<<<gridLogic, kWaveBlock, 0, st>>>(a);
            cudaEventRecord(ev[1], st);
            wk.extend<<<gridWork, kWaveBlock, 0, st>>>(a);
            cudaEventRecord(ev[2], st);
            launchShade(wk, a, gridWork, st);
            cudaEventRecord(ev[3], st);
            wk.shadow<<<gridWork, kWaveBlock, 0, st>>>(a);
            cudaEventRecord(ev[4], st);
            cudaMemcpyAsync(s->hostLast, s->waveCounters, 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
            wfResetQueues<<<1, 32, 0, st>>>(a);
            if ((rc = x2_synchronize(s->ctx, 600000)) != X2_OK) break;
            for (int k = 0; k < 4; ++k) {
                float ms = 0.0f;
                cudaEventElapsedTime(&ms, ev[k], ev[k + 1]);
                s->waveMs[k] += ms;
            }
            if (iterations < kQueueLog) {
                s->queueLog[2 * iterations] = s->hostLast[0];      // rays extended
                s->queueLog[2 * iterations + 1] = s->hostLast[2];  // shadow rays
            }
            ++iterations;
            if (s->hostLast[0] == 0) break;
            if (iterations > maxIter) {
                setError("wavefront did not drain after %u iterations", iterations);
                rc = X2_EDEVICE;
                break;
            }
        }
        if (rc == X2_OK) {
            cudaEventRecord(ev[0], st);
            wfFilmReduce<<<int((64ull * count + 255) / 256), 256, 0, st>>>(a, count, s->sums, s->adaptive ? s->odd : nullptr, s->counts);
            cudaEventRecord(ev[5], st);
            cudaEventRecord(sl.end, st);
            cudaMemcpyAsync(sl.hostCounters, sl.counters, sizeof(Counters), cudaMemcpyDeviceToHost, st);
            cudaEventRecord(sl.done, st);
            rc = x2_synchronize(s->ctx, 600000);
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, ev[0], ev[5]);
            s->waveMs[4] = ms;
        }
        for (auto& e : ev) cudaEventDestroy(e);
        if (rc) return rc;
        sl.busy = true;
        sl.seq = s->nextSeq++;
        s->lastItems = items;
        s->waveIterations = iterations;
        return X2_OK;
    }
    // One graph: the launch's iterations in a conditional while node, each iteration's last kernel deciding whether
    // another follows (at most maxIter; past that it raises the overrun word), then the film reduce. The launch runs
    // without the host; x2_poll / x2_wait collect it like any launch.
    cudaGraph_t graph = nullptr;
    CUDA_OR(cudaGraphCreate(&graph, 0), X2_ECUDA);
    cudaError_t err = cudaSuccess;
    auto check = [&](cudaError_t e) {
        if (err == cudaSuccess && e != cudaSuccess) err = e;
        return err == cudaSuccess;
    };
    cudaGraphConditionalHandle loop;
    cudaGraphNode_t node = nullptr;
    cudaGraphNodeParams cp = {};
    if (check(cudaGraphConditionalHandleCreate(&loop, graph, 1, cudaGraphCondAssignDefault))) {
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = loop;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        check(cudaGraphAddNode(&node, graph, nullptr, 0, &cp));
    }
    const uint32_t bound = uint32_t(std::min<uint64_t>(maxIter, 0xffffffffu));
    if (err == cudaSuccess && check(cudaStreamBeginCaptureToGraph(st, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                                                  cudaStreamCaptureModeThreadLocal))) {
        wfResetQueues<<<1, 32, 0, st>>>(a);
        wk.logic<<<gridLogic, kWaveBlock, 0, st>>>(a);
        wk.extend<<<gridWork, kWaveBlock, 0, st>>>(a);
        launchShade(wk, a, gridWork, st);
        wk.shadow<<<gridWork, kWaveBlock, 0, st>>>(a);
        wfDrainCheck<<<1, 32, 0, st>>>(a, loop, s->drainWords, bound, s->drainWords + 2);
        check(cudaGetLastError());
        cudaGraph_t body = nullptr;
        check(cudaStreamEndCapture(st, &body));
    }
    if (err == cudaSuccess && check(cudaStreamBeginCaptureToGraph(st, graph, &node, nullptr, 1, cudaStreamCaptureModeThreadLocal))) {
        wfFilmReduce<<<int((64ull * count + 255) / 256), 256, 0, st>>>(a, count, s->sums, s->adaptive ? s->odd : nullptr, s->counts);
        check(cudaGetLastError());
        cudaGraph_t out = nullptr;
        check(cudaStreamEndCapture(st, &out));
    }
    cudaGraphExec_t exec = nullptr;
    if (err == cudaSuccess) check(cudaGraphInstantiate(&exec, graph, 0));
    cudaGraphDestroy(graph);
    if (err != cudaSuccess) {
        setError("x2_launch_wavefront: building the launch's graph: %s", cudaGetErrorString(err));
        return X2_ECUDA;
    }
    cudaMemsetAsync(s->drainWords, 0, sizeof(uint32_t) * 4, st);
    cudaEventRecord(sl.begin, st);
    const cudaError_t launched = cudaGraphLaunch(exec, st);
    cudaGraphExecDestroy(exec);  // released once the launch completes
    if (launched != cudaSuccess) {
        setError("graph launch failed: %s", cudaGetErrorString(launched));
        return X2_ECUDA;
    }
    cudaEventRecord(sl.end, st);
    // The extend kernels counted the traced rays; the launch's counters go to the host as x2_launch's do, with the
    // drain's iteration count and overrun word.
    cudaMemcpyAsync(sl.hostCounters, sl.counters, sizeof(Counters), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(s->hostDrain, s->drainWords, sizeof(uint32_t) * 4, cudaMemcpyDeviceToHost, st);
    cudaEventRecord(sl.done, st);
    sl.busy = true;
    sl.seq = s->nextSeq++;
    s->lastItems = items;
    s->drainSeq = sl.seq;
    s->drainBound = bound;
    return X2_OK;
}

int x2_render_frame_wavefront(x2_scene* s, uint32_t first, uint32_t count) {
    if (!s || !s->configured) return X2_EINVAL;
    if (!s->filmPixels || s->samplesPerChunk < count) {
        setError("x2_frame_begin with at least %u samples a chunk first", count);
        return X2_EINVAL;
    }
    const uint32_t tiles = ((s->config.width + 7) / 8) * ((s->config.height + 7) / 8);
    if (int rc = x2_synchronize(s->ctx, 600000)) return rc;
    if (tiles > s->stagingCap) {
        if (s->staging) cudaFreeHost(s->staging);
        s->staging = nullptr;
        CUDA_OR(cudaMallocHost(&s->staging, sizeof(x2_chunk) * tiles), X2_ENOMEM);
        s->stagingCap = tiles;
    }
    for (uint32_t t = 0; t < tiles; ++t) s->staging[t] = x2_chunk{t, first, count, 0};
    return x2_launch_wavefront(s, s->staging, tiles);
}

int x2_items_download(x2_scene* s, float* rgba, uint8_t* status, uint64_t n) {
    if (!s || !s->out) {
        setError("no wavefront launch yet");
        return X2_EINVAL;
    }
    if (n > s->lastItems) {
        setError("%llu items asked, the last launch had %llu", (unsigned long long)n, (unsigned long long)s->lastItems);
        return X2_EINVAL;
    }
    cudaStream_t st = s->ctx->stream;
    if (rgba) cudaMemcpyAsync(rgba, s->out, sizeof(float4) * n, cudaMemcpyDeviceToHost, st);
    if (status) cudaMemcpyAsync(status, s->outStatus, n, cudaMemcpyDeviceToHost, st);
    return x2_wait(s, 600000, nullptr);
}

// The differentiable parameters: each material's diffuse colour (its Lambert albedo) and each light's radiance, set in
// place on the device (the BVH and everything else stay). Host arrays, 3 floats each; null leaves a set as it is.
int x2_scene_set_params(x2_scene* s, const float* albedo, const float* roughness, const float* radiance) {
    if (!s) return X2_EINVAL;
    if (int rc = x2_wait(s, 600000, nullptr)) return rc;
    cudaStream_t st = s->ctx->stream;
    if (albedo || roughness) {
        std::vector<MaterialRec> mats(s->materialCount);
        CUDA_OR(cudaMemcpyAsync(mats.data(), s->materials, sizeof(MaterialRec) * mats.size(), cudaMemcpyDeviceToHost, st), X2_ECUDA);
        CUDA_OR(cudaStreamSynchronize(st), X2_ECUDA);
        for (uint32_t m = 0; m < s->materialCount; ++m) {
            if (albedo)
                for (int k = 0; k < 3; ++k) mats[m].diffuse[k] = albedo[3 * m + k];
            if (roughness) mats[m].roughness = roughness[m];
        }
        CUDA_OR(cudaMemcpyAsync(s->materials, mats.data(), sizeof(MaterialRec) * mats.size(), cudaMemcpyHostToDevice, st), X2_ECUDA);
        CUDA_OR(cudaStreamSynchronize(st), X2_ECUDA);
    }
    if (radiance && s->lightCount) {
        std::vector<x2_light> lights(s->lightCount);
        CUDA_OR(cudaMemcpyAsync(lights.data(), s->lights, sizeof(x2_light) * lights.size(), cudaMemcpyDeviceToHost, st), X2_ECUDA);
        CUDA_OR(cudaStreamSynchronize(st), X2_ECUDA);
        for (uint32_t l = 0; l < s->lightCount; ++l)
            for (int k = 0; k < 3; ++k) lights[l].radiance[k] = radiance[3 * l + k];
        CUDA_OR(cudaMemcpyAsync(s->lights, lights.data(), sizeof(x2_light) * lights.size(), cudaMemcpyHostToDevice, st), X2_ECUDA);
        CUDA_OR(cudaStreamSynchronize(st), X2_ECUDA);
    }
    return X2_OK;
}

int x2_scene_set_texture(x2_scene* s, uint32_t texture, const float* rgb) {
    if (!s || !rgb || texture >= s->hostTextures.size()) {
        setError("x2_scene_set_texture: texture %u of %zu", texture, s ? s->hostTextures.size() : size_t(0));
        return X2_EINVAL;
    }
    if (int rc = x2_wait(s, 600000, nullptr)) return rc;
    const TexRec& t = s->hostTextures[texture];
    cudaStream_t st = s->ctx->stream;
    CUDA_OR(cudaMemcpyAsync(s->texels + 3 * t.first, rgb, sizeof(float) * 3 * size_t(t.width) * t.height, cudaMemcpyHostToDevice, st), X2_ECUDA);
    CUDA_OR(cudaStreamSynchronize(st), X2_ECUDA);
    return X2_OK;
}

// The adjoint of a frame's samples [first, first + count) of every pixel: gradients of a loss with respect to each
// material's albedo and roughness and each light's radiance, given the loss's derivative with respect to the image
// (device, 3 floats a pixel, the image being the film's mean). Device outputs (FP64), added to; a null roughness
// output skips that set.
// The replay in the plain megakernel's form (one thread a sample): x2_adjoint's arguments and results.
// The texel count of the scene's textures (3 gradients each).
uint64_t texelCount(const x2_scene* s) {
    uint64_t n = 0;
    for (const TexRec& t : s->hostTextures) n += uint64_t(t.width) * t.height;
    return n;
}

int x2_adjoint_plain(x2_scene* s, uint32_t first, uint32_t count, const float* d_dloss_dimage, double* d_albedo_grad,
                     double* d_roughness_grad, double* d_radiance_grad, double* d_texture_grad) {
    if (!s || !s->configured || !d_dloss_dimage || !d_albedo_grad || !d_radiance_grad || count == 0) {
        setError("x2_adjoint: configured scene, device arrays and a sample count");
        return X2_EINVAL;
    }
    if (s->config.volume_count || s->config.max_depth >= 128 || s->config.bsdf_samples != 1) {
        setError("x2_adjoint: no volumes, max_depth < 128, bsdf_samples = 1");
        return X2_EINVAL;
    }
    const uint32_t params = 4 * s->materialCount + 3 * s->lightCount;
    if (size_t(params) * sizeof(float) > 96 * 1024) {
        setError("x2_adjoint: 4 x materials + 3 x lights must be at most %u", 96 * 1024 / 4);
        return X2_EINVAL;
    }
    if (int rc = checkDevice(s->ctx)) return rc;
    if (int rc = x2_wait(s, 600000, nullptr)) return rc;
    cudaStream_t st = s->ctx->stream;
    const uint32_t tiles = ((s->config.width + 7) / 8) * ((s->config.height + 7) / 8);
    std::vector<x2_chunk> chunks(tiles);
    for (uint32_t t = 0; t < tiles; ++t) chunks[t] = x2_chunk{t, first, count, 0};
    x2_chunk* d = nullptr;
    double* grads = nullptr;
    float* texGrad = nullptr;
    const uint64_t texGrads = d_texture_grad ? 3 * texelCount(s) : 0;
    CUDA_OR(cudaMalloc(&d, sizeof(x2_chunk) * tiles), X2_ENOMEM);
    if (cudaMalloc(&grads, sizeof(double) * params) != cudaSuccess || (texGrads && cudaMalloc(&texGrad, sizeof(float) * texGrads) != cudaSuccess)) {
        cudaFree(d);
        cudaFree(grads);
        setError("x2_adjoint: allocation failed");
        return X2_ENOMEM;
    }
    if (texGrads) cudaMemsetAsync(texGrad, 0, sizeof(float) * texGrads, s->ctx->stream);
    cudaMemcpyAsync(d, chunks.data(), sizeof(x2_chunk) * tiles, cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(grads, 0, sizeof(double) * params, st);
    const size_t shared = sizeof(float) * params;
    if (shared > 48 * 1024) cudaFuncSetAttribute(adjointKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(shared));
    SceneView v = viewOf(s);
    v.stats = nullptr;
    adjointKernel<<<s->ctx->smCount * 8, 128, shared, st>>>(v, d, tiles, count, d_dloss_dimage, grads, s->materialCount, s->lightCount, texGrad);
    int rc = cudaGetLastError() == cudaSuccess ? X2_OK : X2_ECUDA;
    if (!rc) {
        // Added to the caller's arrays: albedo, roughness, radiance.
        addInto<<<(params + 255) / 256, 256, 0, st>>>(d_albedo_grad, grads, 3 * s->materialCount);
        if (d_roughness_grad) addInto<<<(params + 255) / 256, 256, 0, st>>>(d_roughness_grad, grads + 3 * s->materialCount, s->materialCount);
        addInto<<<(params + 255) / 256, 256, 0, st>>>(d_radiance_grad, grads + 4 * s->materialCount, 3 * s->lightCount);
        if (texGrads) addFloatInto<<<unsigned((texGrads + 255) / 256), 256, 0, st>>>(d_texture_grad, texGrad, texGrads);
        rc = x2_synchronize(s->ctx, 600000);
    } else {
        setError("x2_adjoint: launch failed");
    }
    cudaFree(d);
    cudaFree(grads);
    cudaFree(texGrad);
    return rc;
}

// The adjoint in the wavefront form: the samples' paths replayed by the wavefront's kernels (logic, extend, per-lobe
// sort, shade, shadow; the adjoint forms of logic and shade credit as they go), as one graph of iterations replayed
// until no path is left; the gradient rows then summed into FP64 and added to the caller's arrays.
int x2_adjoint(x2_scene* s, uint32_t first, uint32_t count, const float* d_dloss_dimage, double* d_albedo_grad, double* d_roughness_grad,
               double* d_radiance_grad, double* d_texture_grad) {
    if (!s || !s->configured || !d_dloss_dimage || !d_albedo_grad || !d_radiance_grad || count == 0) {
        setError("x2_adjoint: configured scene, device arrays and a sample count");
        return X2_EINVAL;
    }
    if (s->config.volume_count || s->config.max_depth >= 128 || s->config.bsdf_samples != 1) {
        setError("x2_adjoint: no volumes, max_depth < 128, bsdf_samples = 1");
        return X2_EINVAL;
    }
    const uint32_t params = 4 * s->materialCount + 3 * s->lightCount;
    if (size_t(params) * sizeof(float) > 96 * 1024 || s->materialCount >= (1u << 30)) {
        setError("x2_adjoint: 4 x materials + 3 x lights must be at most %u", 96 * 1024 / 4);
        return X2_EINVAL;
    }
    if (int rc = checkDevice(s->ctx)) return rc;
    if (int rc = x2_wait(s, 600000, nullptr)) return rc;
    const uint32_t tiles = ((s->config.width + 7) / 8) * ((s->config.height + 7) / 8);
    const unsigned long long items = (unsigned long long)tiles * 64ull * count;
    if (items > 0xffffffffull) {
        setError("x2_adjoint: %llu work items (at most 2^32 - 1)", items);
        return X2_EINVAL;
    }
    const uint32_t records = s->config.light_count * s->config.light_samples + 1;
    uint32_t paths = s->reservePaths ? s->reservePaths : defaultPaths(records);
    if (paths > items) paths = uint32_t(items < 1024 ? 1024 : items);
    const uint32_t verts = s->config.max_depth + 1;
    if (int rc = ensureWave(s, paths, records)) return rc;
    if (int rc = ensureItems(s, items)) return rc;
    if (s->adjPaths < paths || s->adjVerts != verts || s->adjRecords != records) {
        freeAdjointWave(s);
        const size_t V = size_t(paths) * verts;
        const bool ok = cudaMalloc(&s->avert, sizeof(uint4) * V) == cudaSuccess && cudaMalloc(&s->ascale, sizeof(float4) * V) == cudaSuccess &&
                        cudaMalloc(&s->avcount, sizeof(uint32_t) * paths) == cudaSuccess &&
                        cudaMalloc(&s->adelta, sizeof(float4) * paths) == cudaSuccess &&
                        cudaMalloc(&s->aaux, sizeof(uint2) * size_t(paths) * records) == cudaSuccess &&
                        (!s->triUV || cudaMalloc(&s->atex, sizeof(float4) * V) == cudaSuccess);
        if (!ok) {
            freeAdjointWave(s);
            setError("x2_adjoint: device allocation failed for %u paths", paths);
            return X2_ENOMEM;
        }
        s->adjPaths = paths;
        s->adjVerts = verts;
        s->adjRecords = records;
    }
    Slot& sl = s->slots[0];
    if (int rc = ensureSlot(sl, tiles)) return rc;
    constexpr uint32_t kRows = 1024;
    float* rows = nullptr;
    double* grads = nullptr;
    float* texGrad = nullptr;
    const uint64_t texGrads = d_texture_grad ? 3 * texelCount(s) : 0;
    if (cudaMalloc(&rows, sizeof(float) * size_t(kRows) * params) != cudaSuccess || cudaMalloc(&grads, sizeof(double) * params) != cudaSuccess ||
        (texGrads && cudaMalloc(&texGrad, sizeof(float) * texGrads) != cudaSuccess)) {
        cudaFree(rows);
        cudaFree(grads);
        setError("x2_adjoint: allocation failed");
        return X2_ENOMEM;
    }
    cudaStream_t st = s->ctx->stream;
    std::vector<x2_chunk> chunks(tiles);
    for (uint32_t t = 0; t < tiles; ++t) chunks[t] = x2_chunk{t, first, count, 0};
    cudaMemcpyAsync(sl.chunks, chunks.data(), sizeof(x2_chunk) * tiles, cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(rows, 0, sizeof(float) * size_t(kRows) * params, st);
    cudaMemsetAsync(grads, 0, sizeof(double) * params, st);
    if (texGrads) cudaMemsetAsync(texGrad, 0, sizeof(float) * texGrads, st);
    cudaMemsetAsync(s->wave.state, 0, sizeof(uint32_t) * paths, st);
    cudaMemsetAsync(s->wave.ncount, 0, sizeof(uint32_t) * paths, st);
    cudaMemsetAsync(s->claimed, 0, sizeof(unsigned long long), st);
    cudaMemsetAsync(s->waveCounters, 0, sizeof(uint32_t) * kWaveCounters, st);
    cudaMemsetAsync(sl.counters, 0, sizeof(Counters), st);
    WaveArgs a;
    a.scene = viewOf(s);
    a.scene.stats = nullptr;
    a.w = s->wave;
    a.paths = paths;
    a.recordsPerPath = records;
    a.chunks = sl.chunks;
    a.itemCount = items;
    a.samplesPerChunk = count;
    a.claimed = s->claimed;
    a.extendQ = s->extendQ;
    a.extendCount = s->waveCounters;
    a.lastExtend = s->waveCounters + 1;
    a.shadowQ = s->shadowQ;
    a.shadowCount = s->waveCounters + 2;
    a.shadowSlots = s->shadowOrder && a.recordsPerPath <= x2::kRecordSegments ? s->waveCounters + 8 : nullptr;
    a.extendSlots = s->extendBins ? s->waveCounters + 8 + x2::kRecordSegments : nullptr;
    a.extendNext = s->waveCounters + 3;
    a.shadowNext = s->waveCounters + 4;
    a.shadeQ = s->lobeQueues ? s->shadeQ : nullptr;
    a.shadeCount = s->waveCounters + 5;
    a.refill = s->refill;
    a.triLimit = s->triLimit;
    a.out = s->out;
    a.outStatus = s->outStatus;
    a.counters = sl.counters;
    a.scenes = nullptr;
    a.chunkRequest = nullptr;
    a.chunkItems = nullptr;
    a.chunkCount = tiles;
    a.adj = AdjointWave{d_dloss_dimage, rows, kRows, s->materialCount, s->lightCount, verts, s->avert, s->ascale, s->avcount, s->adelta, s->aaux,
                        s->atex, texGrad};
    a.chunkMask = nullptr;
    a.pixelBase = nullptr;
    a.liveChunks = nullptr;
    const size_t shared = sizeof(float) * params;
    if (shared > 48 * 1024) {
        cudaFuncSetAttribute(wfLogicAdjoint, cudaFuncAttributeMaxDynamicSharedMemorySize, int(shared));
        cudaFuncSetAttribute(wfShadeAdjoint, cudaFuncAttributeMaxDynamicSharedMemorySize, int(shared));
    }
    // Logic in a grid of a few blocks a SM (each block's partials go to a gradient row once a launch).
    const int gridLogic = std::min(int((paths + kWaveBlock - 1) / kWaveBlock), s->ctx->smCount * 8);
    const int gridWork = s->ctx->smCount * int(s->blocksPerSm);
    const WaveKernels wk = waveKernels(s->traceBlocks, s->shadeBlocks, false, s->triUV != nullptr);
    const uint64_t maxIter = items * (uint64_t(s->config.max_depth) + 2) / paths + uint64_t(s->config.max_depth) + 64;
    constexpr int kIter = 8;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int rc = X2_OK;
    if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        setError("x2_adjoint: stream capture failed");
        rc = X2_ECUDA;
    } else {
        for (int it = 0; it < kIter; ++it) {
            wfResetQueues<<<1, 32, 0, st>>>(a);
            wfLogicAdjoint<<<gridLogic, kWaveBlock, shared, st>>>(a);
            wk.extend<<<gridWork, kWaveBlock, 0, st>>>(a);
            if (a.shadeQ) wfSortShade<<<gridWork, kWaveBlock, 0, st>>>(a);
            wfShadeAdjoint<<<gridWork, kWaveBlock, shared, st>>>(a);
            wk.shadow<<<gridWork, kWaveBlock, 0, st>>>(a);
        }
        wfResetQueues<<<1, 32, 0, st>>>(a);
        if (cudaStreamEndCapture(st, &graph) != cudaSuccess || cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess) {
            setError("x2_adjoint: graph capture failed");
            rc = X2_ECUDA;
        }
    }
    uint32_t iterations = 0;
    while (rc == X2_OK) {
        if (cudaGraphLaunch(exec, st) != cudaSuccess) {
            setError("x2_adjoint: graph launch failed");
            rc = X2_ECUDA;
            break;
        }
        iterations += kIter;
        cudaMemcpyAsync(s->hostLast, s->waveCounters + 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
        if ((rc = x2_synchronize(s->ctx, 600000)) != X2_OK) break;
        if (s->hostLast[0] == 0) break;
        if (iterations > maxIter) {
            setError("x2_adjoint: the wavefront did not drain after %u iterations", iterations);
            rc = X2_EDEVICE;
        }
    }
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (rc == X2_OK) {
        wfGradRows<<<(params + 255) / 256, 256, 0, st>>>(rows, kRows, params, grads);
        addInto<<<(params + 255) / 256, 256, 0, st>>>(d_albedo_grad, grads, 3 * s->materialCount);
        if (d_roughness_grad) addInto<<<(params + 255) / 256, 256, 0, st>>>(d_roughness_grad, grads + 3 * s->materialCount, s->materialCount);
        addInto<<<(params + 255) / 256, 256, 0, st>>>(d_radiance_grad, grads + 4 * s->materialCount, 3 * s->lightCount);
        if (texGrads) addFloatInto<<<unsigned((texGrads + 255) / 256), 256, 0, st>>>(d_texture_grad, texGrad, texGrads);
        rc = cudaGetLastError() == cudaSuccess ? x2_synchronize(s->ctx, 600000) : X2_ECUDA;
    }
    cudaFree(rows);
    cudaFree(grads);
    cudaFree(texGrad);
    return rc;
}

// ---- adaptive sampling (row f2): the reference's adaptive frame (async_render.h, async_adaptive.h) on the device ----
namespace {

// The overlapping regions of a width x height image (the reference's Regions: up to 4 x 4 regions of whole 8-pixel
// tiles, each widened by an 8-pixel overlap, clamped to the image), their tables, node bounds and the node pool.
int ensureAdaptive(x2_scene* s, float target) {
    const uint32_t width = s->config.width, height = s->config.height;
    AdaptiveState* a = s->adaptiveState;
    if (a && a->width == width && a->height == height) {
        a->target = target;
        return X2_OK;
    }
    delete a;
    a = s->adaptiveState = new AdaptiveState();
    a->width = width;
    a->height = height;
    a->target = target;
    a->tilesX = (width + 7) / 8;
    a->tiles = a->tilesX * ((height + 7) / 8);
    a->grid = x2::rg::regionGrid(int(width), int(height));
    a->regionCount = uint32_t(a->grid.across * a->grid.across);
    std::vector<int32_t> boxes(4 * a->regionCount);
    std::vector<uint32_t> bound(a->regionCount), rowStart(a->regionCount), colStart(a->regionCount);
    std::vector<unsigned long long> satOffset(a->regionCount);
    unsigned long long sat = 0, pool = 0;
    for (uint32_t r = 0; r < a->regionCount; ++r) {
        int* b = boxes.data() + 4 * r;
        x2::rg::regionBox(a->grid, int(r), int(width), int(height), b);
        const int w = b[2] - b[0], h = b[3] - b[1];
        bound[r] = uint32_t(std::max(1, x2::rg::regionNodeBound(w, h)));
        satOffset[r] = sat;
        rowStart[r] = a->rows;
        colStart[r] = a->cols;
        a->rows += uint32_t(h);
        a->cols += uint32_t(w);
        sat += (unsigned long long)(w + 1) * (unsigned long long)(h + 1);
        pool += bound[r];
    }
    a->poolCapacity = uint32_t(std::min<unsigned long long>(pool, 0x7fffffffull));
    std::vector<uint64_t> inImage(a->tiles);
    a->firstAlive.assign(a->tiles, 0);
    for (uint32_t t = 0; t < a->tiles; ++t) {
        uint64_t m = 0;
        const uint32_t tx = (t % a->tilesX) * 8, ty = (t / a->tilesX) * 8;
        for (uint32_t p = 0; p < 64; ++p)
            if (tx + p % 8 < width && ty + p / 8 < height) m |= uint64_t(1) << p;
        inImage[t] = m;
        a->firstAlive[t] = m ? 1 : 0;
    }
    const size_t pixels = size_t(width) * height, regions = a->regionCount, cap = a->poolCapacity;
    const size_t blocks = (a->tiles + x2::kCompactBlock - 1) / x2::kCompactBlock;
    bool ok = true;
    auto get = [&](auto** p, size_t bytes) { ok = ok && cudaMalloc(reinterpret_cast<void**>(p), bytes) == cudaSuccess; };
    get(&a->boxes, sizeof(int32_t) * 4 * regions);
    get(&a->satOffset, sizeof(unsigned long long) * regions);
    for (uint32_t** p : {&a->bound, &a->nodes, &a->ready, &a->open, &a->rowStart, &a->colStart}) get(p, sizeof(uint32_t) * regions);
    get(&a->sat, sizeof(double) * sat);
    for (float** p : {&a->px0, &a->py0, &a->px1, &a->py1}) get(p, sizeof(float) * cap);
    get(&a->pchild, sizeof(int32_t) * cap);
    get(&a->pfate, cap);
    get(&a->pregion, sizeof(uint32_t) * cap);
    get(&a->poolWords, sizeof(uint32_t) * 4);
    get(&a->errors, sizeof(float) * pixels);
    for (uint64_t** p : {&a->inImage, &a->reach, &a->tileMask, &a->chunkMasks}) get(p, sizeof(uint64_t) * a->tiles);
    get(&a->blockTiles, sizeof(uint32_t) * blocks);
    get(&a->planned, sizeof(uint32_t) * pixels);
    get(&a->base, sizeof(uint32_t) * pixels);
    get(&a->stop, sizeof(uint32_t));
    get(&a->words, sizeof(uint32_t) * 8);
    get(&a->samples, sizeof(unsigned long long));
    get(&a->alive, 2 * size_t(a->tiles));
    get(&a->ratio, sizeof(float) * a->tiles);
    ok = ok && cudaMallocHost(&a->hostWords, sizeof(uint32_t) * 8) == cudaSuccess &&
         cudaMallocHost(&a->hostSamples, sizeof(unsigned long long)) == cudaSuccess;
    if (!ok) {
        delete a;
        s->adaptiveState = nullptr;
        setError("device allocation failed for the adaptive frame");
        return X2_ENOMEM;
    }
    cudaStream_t st = s->ctx->stream;
    cudaMemcpyAsync(a->boxes, boxes.data(), sizeof(int32_t) * boxes.size(), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(a->satOffset, satOffset.data(), sizeof(unsigned long long) * regions, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(a->bound, bound.data(), sizeof(uint32_t) * regions, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(a->rowStart, rowStart.data(), sizeof(uint32_t) * regions, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(a->colStart, colStart.data(), sizeof(uint32_t) * regions, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(a->inImage, inImage.data(), sizeof(uint64_t) * a->tiles, cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(a->open, 0, sizeof(uint32_t) * regions, st);
    cudaMemsetAsync(a->planned, 0, sizeof(uint32_t) * pixels, st);
    cudaMemsetAsync(a->base, 0, sizeof(uint32_t) * pixels, st);
    cudaMemsetAsync(a->stop, 0, sizeof(uint32_t), st);
    CUDA_OR(cudaStreamSynchronize(st), X2_ECUDA);
    return X2_OK;
}

// The chain's arguments; a queued frame's (chunks: its compacted chunks) or a host-run step's (chunks null).
x2::AdaptiveArgs adaptiveArgs(const AdaptiveState& a, x2_chunk* chunks = nullptr) {
    x2::AdaptiveArgs g{};
    g.width = a.width;
    g.height = a.height;
    g.tilesX = a.tilesX;
    g.tiles = a.tiles;
    g.target = a.target;
    g.regions = x2::RegionState{a.boxes, a.satOffset, a.bound, a.nodes, a.ready, a.open, a.regionCount, a.rowStart, a.colStart, a.rows, a.cols,
                                a.grid};
    g.pool = x2::TreePool{a.px0, a.py0, a.px1, a.py1, a.pchild, a.pfate, a.pregion, a.poolCapacity, a.poolWords, a.poolWords + 1};
    g.sat = a.sat;
    g.errors = a.errors;
    g.inImage = a.inImage;
    g.reach = a.reach;
    g.tileMask = a.tileMask;
    g.planned = a.planned;
    g.base = a.base;
    g.stop = a.stop;
    g.queued = chunks ? 1u : 0u;
    g.chunks = chunks;
    g.chunkMasks = a.chunkMasks;
    g.live = a.words;
    g.passes = a.words + 1;
    g.samples = a.samples;
    g.blockTiles = a.blockTiles;
    g.alive = nullptr;
    g.liveTiles = a.words + 5;
    g.ratio = a.ratio;
    return g;
}

// A graph built in segments of captured work on one stream, each after the last segment's end nodes, with
// conditional while nodes between them.
struct GraphSegments {
    cudaStream_t st;
    cudaGraph_t graph = nullptr;
    std::vector<cudaGraphNode_t> tail;
    cudaError_t err = cudaSuccess;
    bool check(cudaError_t e) {
        if (err == cudaSuccess && e != cudaSuccess) err = e;
        return err == cudaSuccess;
    }
    bool begin(cudaGraph_t g, bool chained) {
        return check(cudaStreamBeginCaptureToGraph(st, g, chained && !tail.empty() ? tail.data() : nullptr, nullptr, chained ? tail.size() : 0,
                                                   cudaStreamCaptureModeThreadLocal));
    }
    bool end(bool chained) {
        cudaStreamCaptureStatus status;
        const cudaGraphNode_t* deps = nullptr;
        size_t n = 0;
        const cudaError_t info = cudaStreamGetCaptureInfo(st, &status, nullptr, nullptr, &deps, &n);
        if (info == cudaSuccess && chained) tail.assign(deps, deps + n);
        cudaGraph_t out = nullptr;
        check(info);
        return check(cudaStreamEndCapture(st, &out));
    }
    // A while node after the tail; returns its body graph (null on failure) and its handle.
    cudaGraph_t whileNode(cudaGraphConditionalHandle* handle) {
        if (!check(cudaGraphConditionalHandleCreate(handle, graph, 1, cudaGraphCondAssignDefault))) return nullptr;
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = *handle;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        if (!check(cudaGraphAddNode(&node, graph, tail.data(), tail.size(), &cp))) return nullptr;
        tail.assign(1, node);
        return cp.conditional.phGraph_out[0];
    }
};

// The region trees of a pass, appended to a graph: the roots and the summed-area tables, then a while node growing
// every region's trees a level an iteration, then the open leaves' reach over the tiles.
bool appendTrees(GraphSegments& g, const x2::AdaptiveArgs& args, const AdaptiveState& a, int smCount) {
    cudaStream_t st = g.st;
    if (!g.begin(g.graph, true)) return false;
    x2::treeRoots<<<(a.regionCount + 31) / 32, 32, 0, st>>>(args);
    x2::tableRows<<<(a.rows + 127) / 128, 128, 0, st>>>(args);
    x2::tableColumns<<<(a.cols + 127) / 128, 128, 0, st>>>(args);
    g.check(cudaGetLastError());
    if (!g.end(true)) return false;
    cudaGraphConditionalHandle loop;
    cudaGraph_t body = g.whileNode(&loop);
    if (!body || !g.begin(body, false)) return false;
    x2::treeLevel<<<smCount * 4, 256, 0, st>>>(args);
    x2::treeNextLevel<<<1, 32, 0, st>>>(args, loop);
    g.check(cudaGetLastError());
    if (!g.end(false)) return false;
    if (!g.begin(g.graph, true)) return false;
    cudaMemsetAsync(a.reach, 0, sizeof(uint64_t) * a.tiles, st);
    x2::leafReach<<<smCount * 8, 256, 0, st>>>(args);
    g.check(cudaGetLastError());
    return g.end(true);
}

// One chain step on the frame's film, run from the host: errors and trees (not in a uniform pass), then the pass's
// tile masks; as one small graph, since the trees grow in a while node.
int adaptiveChain(x2_scene* s, const x2::AdaptiveArgs& args, uint32_t uniform, uint32_t size) {
    AdaptiveState& a = *s->adaptiveState;
    GraphSegments g;
    g.st = s->ctx->stream;
    CUDA_OR(cudaGraphCreate(&g.graph, 0), X2_ECUDA);
    const uint32_t pixels = a.width * a.height;
    if (!uniform && g.begin(g.graph, true)) {
        x2::chainPixelErrors<<<(pixels + 255) / 256, 256, 0, g.st>>>(args, s->sums, s->odd, s->counts);
        g.check(cudaGetLastError());
        if (g.end(true)) appendTrees(g, args, a, s->ctx->smCount);
    }
    if (g.begin(g.graph, true)) {
        x2::tileMasks<<<(a.tiles + 255) / 256, 256, 0, g.st>>>(args, uniform, size);
        g.check(cudaGetLastError());
        g.end(true);
    }
    cudaGraphExec_t exec = nullptr;
    if (g.err == cudaSuccess) g.check(cudaGraphInstantiate(&exec, g.graph, 0));
    cudaGraphDestroy(g.graph);
    if (g.err == cudaSuccess) g.check(cudaGraphLaunch(exec, g.st));
    if (g.err == cudaSuccess) g.check(cudaStreamSynchronize(g.st));
    if (exec) cudaGraphExecDestroy(exec);
    if (g.err != cudaSuccess) {
        setError("adaptive chain step: %s", cudaGetErrorString(g.err));
        return X2_ECUDA;
    }
    return X2_OK;
}

// MoonRay's pass schedule for maxSamples: one sample, then 4, 6, 8, ... more, the rest last.
std::vector<std::pair<uint32_t, uint32_t>> adaptiveSchedule(uint32_t maxSamples) {
    std::vector<std::pair<uint32_t, uint32_t>> passes{{0, 1}};
    uint32_t current = 1, remaining = maxSamples - 1, size = 4;
    while (remaining > size && passes.size() < 999) {
        passes.push_back({current, current + size});
        remaining -= size;
        current += size;
        size += 2;
    }
    if (remaining) passes.push_back({current, current + remaining});
    return passes;
}

}  // namespace

int x2_adaptive_step(x2_scene* s, float target, uint32_t uniform, uint32_t size, float* errors, uint64_t* masks, uint32_t* stop) {
    if (!s || !s->configured || !s->filmPixels || !s->adaptive) {
        setError("x2_adaptive_step: an adaptive frame first (x2_frame_begin_adaptive)");
        return X2_EINVAL;
    }
    if (int rc = x2_wait(s, 600000, nullptr)) return rc;
    if (int rc = ensureAdaptive(s, target)) return rc;
    if (int rc = adaptiveChain(s, adaptiveArgs(*s->adaptiveState), uniform, size)) return rc;
    AdaptiveState& a = *s->adaptiveState;
    cudaStream_t st = s->ctx->stream;
    if (errors) cudaMemcpyAsync(errors, a.errors, sizeof(float) * a.width * a.height, cudaMemcpyDeviceToHost, st);
    if (masks) cudaMemcpyAsync(masks, a.tileMask, sizeof(uint64_t) * a.tiles, cudaMemcpyDeviceToHost, st);
    if (stop) cudaMemcpyAsync(stop, a.stop, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
    CUDA_OR(cudaStreamSynchronize(st), X2_ECUDA);
    return X2_OK;
}

// The whole frame as one graph, queued at once: for each pass of the schedule the chain, the compaction of its active
// tiles and the pass's wavefront launch, whose iterations run in a conditional while node until no path is left, then
// its film reduce. The host waits once, at the frame's end; a pass that finds nothing to do costs a few empty launches.
namespace {
int renderAdaptive(x2_scene* s, uint32_t minSamples, uint32_t maxSamples, float target, bool cellular, x2_adaptive_result* result) {
    if (!s || !s->configured || maxSamples == 0 || !(target > 0)) {
        setError("x2_render_adaptive: a configured scene, at least one sample and a positive target");
        return X2_EINVAL;
    }
    if (s->config.bsdf_samples != 1) {
        setError("the wavefront form takes one BSDF sample a lobe (bsdf_samples = 1)");
        return X2_EINVAL;
    }
    const auto t0 = std::chrono::steady_clock::now();
    const auto passes = adaptiveSchedule(maxSamples);
    uint32_t most = 0;
    for (const auto& p : passes) most = std::max(most, p.second - p.first);
    if (int rc = x2_frame_begin_adaptive(s, most)) return rc;
    if (int rc = ensureAdaptive(s, target)) return rc;
    if (int rc = checkDevice(s->ctx)) return rc;
    if (int rc = x2_wait(s, 600000, nullptr)) return rc;
    AdaptiveState& ad = *s->adaptiveState;
    const unsigned long long maxItems = (unsigned long long)ad.tiles * 64ull * most;
    if (maxItems > 0xffffffffull) {
        setError("x2_render_adaptive: %llu work items in a pass (at most 2^32 - 1)", maxItems);
        return X2_EINVAL;
    }
    Slot& sl = s->slots[0];
    if (int rc = ensureSlot(sl, ad.tiles)) return rc;
    const uint32_t records = s->config.light_count * s->config.light_samples + 1;
    uint32_t paths = s->reservePaths ? s->reservePaths : defaultPaths(records);
    if (paths > maxItems) paths = uint32_t(maxItems < 1024 ? 1024 : maxItems);
    if (int rc = ensureWave(s, paths, records)) return rc;
    if (int rc = ensureItems(s, maxItems)) return rc;
    cudaStream_t st = s->ctx->stream;
    cudaMemsetAsync(ad.planned, 0, sizeof(uint32_t) * ad.width * ad.height, st);
    cudaMemsetAsync(ad.stop, 0, sizeof(uint32_t), st);
    cudaMemsetAsync(ad.words, 0, sizeof(uint32_t) * 8, st);
    cudaMemsetAsync(ad.samples, 0, sizeof(unsigned long long), st);
    cudaMemsetAsync(sl.counters, 0, sizeof(Counters), st);
    if (cellular) cudaMemcpyAsync(ad.alive, ad.firstAlive.data(), ad.tiles, cudaMemcpyHostToDevice, st);
    CUDA_OR(cudaGetLastError(), X2_ECUDA);
    const x2::AdaptiveArgs chain = adaptiveArgs(ad, sl.chunks);
    uint32_t generation = 0;
    WaveArgs a = launchArgs(s, sl, paths, records, maxItems, ad.tiles);
    a.chunkMask = ad.chunkMasks;
    a.pixelBase = ad.base;
    a.liveChunks = ad.words;
    const int gridLogic = int((paths + kWaveBlock - 1) / kWaveBlock);
    const int gridWork = s->ctx->smCount * int(s->blocksPerSm);
    const WaveKernels wk = waveKernels(s->traceBlocks, s->shadeBlocks, s->volumeCount != 0, s->triUV != nullptr, s->shortStack != 0,
                                       a.scene.stats != nullptr, s->shadeSplit != 0,
                                       s->wave.lightJob != nullptr ? s->lightSplit : 0u, s->triOverlap != 0 && s->shortStack != 0 && s->traceBlocks < 9);
    const uint64_t bound = maxItems * (uint64_t(s->config.max_depth) + 2) / paths + uint64_t(s->config.max_depth) + 64;
    const uint32_t maxIter = uint32_t(std::min<uint64_t>(bound, 0xffffffffu));

    // The graph, built in segments: each captured onto the graph after the last segment's end nodes.
    GraphSegments g;
    g.st = st;
    CUDA_OR(cudaGraphCreate(&g.graph, 0), X2_ECUDA);
    const uint32_t pixels = ad.width * ad.height;
    const int compactBlocks = int((ad.tiles + x2::kCompactBlock - 1) / x2::kCompactBlock);
    for (size_t k = 0; k < passes.size() && g.err == cudaSuccess; ++k) {
        const uint32_t size = passes[k].second - passes[k].first;
        const uint32_t uniform = passes[k].first < minSamples ? 1u : 0u;
        a.samplesPerChunk = size;
        a.itemCount = (unsigned long long)ad.tiles * 64ull * size;
        x2::AdaptiveArgs pass = chain;
        if (!uniform) {
            if (!g.begin(g.graph, true)) break;
            x2::chainPixelErrors<<<(pixels + 255) / 256, 256, 0, st>>>(chain, s->sums, s->odd, s->counts);
            if (cellular) {
                // The next generation from the film so far; the pass's masks come from it.
                const uint8_t* aliveIn = ad.alive + size_t(generation % 2) * ad.tiles;
                uint8_t* aliveOut = ad.alive + size_t((generation + 1) % 2) * ad.tiles;
                ++generation;
                cudaMemsetAsync(chain.liveTiles, 0, sizeof(uint32_t), st);
                x2::tileRatios<<<(ad.tiles + 255) / 256, 256, 0, st>>>(chain);
                x2::nextGeneration<<<(ad.tiles + 255) / 256, 256, 0, st>>>(chain, aliveIn, aliveOut);
                pass.alive = aliveOut;
            }
            g.check(cudaGetLastError());
            if (!g.end(true)) break;
            if (!cellular && !appendTrees(g, chain, ad, s->ctx->smCount)) break;
        }
        if (!g.begin(g.graph, true)) break;
        x2::tileMasks<<<(ad.tiles + 255) / 256, 256, 0, st>>>(pass, uniform, size);
        x2::compactCount<<<compactBlocks, x2::kCompactBlock, 0, st>>>(chain);
        x2::compactWrite<<<compactBlocks, x2::kCompactBlock, 0, st>>>(chain, size);
        cudaMemsetAsync(s->wave.state, 0, sizeof(uint32_t) * paths, st);
        cudaMemsetAsync(s->wave.ncount, 0, sizeof(uint32_t) * paths, st);
        cudaMemsetAsync(s->claimed, 0, sizeof(unsigned long long), st);
        cudaMemsetAsync(s->waveCounters, 0, sizeof(uint32_t) * kWaveCounters, st);
        cudaMemsetAsync(s->outStatus, X2_SKIP, a.itemCount, st);
        cudaMemsetAsync(ad.words + 2, 0, sizeof(uint32_t), st);
        g.check(cudaGetLastError());
        if (!g.end(true)) break;
        // The pass's drain: a while node whose body is one iteration and the test that decides the next.
        cudaGraphConditionalHandle loop;
        cudaGraph_t body = g.whileNode(&loop);
        if (!body || !g.begin(body, false)) break;
        wfResetQueues<<<1, 32, 0, st>>>(a);
        wk.logic<<<gridLogic, kWaveBlock, 0, st>>>(a);
        wk.extend<<<gridWork, kWaveBlock, 0, st>>>(a);
        launchShade(wk, a, gridWork, st);
        wk.shadow<<<gridWork, kWaveBlock, 0, st>>>(a);
        wfDrainCheck<<<1, 32, 0, st>>>(a, loop, ad.words + 2, maxIter, ad.words + 4);
        g.check(cudaGetLastError());
        if (!g.end(false)) break;
        if (!g.begin(g.graph, true)) break;
        wfFilmReduce<<<int((64ull * ad.tiles + 255) / 256), 256, 0, st>>>(a, ad.tiles, s->sums, s->odd, s->counts);
        g.check(cudaGetLastError());
        g.end(true);
    }
    cudaError_t err = g.err;
    auto check = [&](cudaError_t e) {
        if (err == cudaSuccess && e != cudaSuccess) err = e;
        return err == cudaSuccess;
    };
    cudaGraph_t graph = g.graph;
    cudaGraphExec_t exec = nullptr;
    if (err == cudaSuccess) check(cudaGraphInstantiate(&exec, graph, 0));
    cudaGraphDestroy(graph);
    if (err != cudaSuccess) {
        setError("x2_render_adaptive: building the frame's graph: %s", cudaGetErrorString(err));
        return X2_ECUDA;
    }
    cudaEventRecord(sl.begin, st);
    check(cudaGraphLaunch(exec, st));
    cudaEventRecord(sl.end, st);
    cudaMemcpyAsync(sl.hostCounters, sl.counters, sizeof(Counters), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(ad.hostWords, ad.words, sizeof(uint32_t) * 8, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(ad.hostSamples, ad.samples, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(ad.hostWords + 5, ad.stop, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
    cudaEventRecord(sl.done, st);
    sl.busy = true;
    sl.seq = s->nextSeq++;
    s->lastItems = 0;  // the passes' per-item outputs are not kept
    int rc = x2_synchronize(s->ctx, 600000);
    cudaGraphExecDestroy(exec);
    if (err != cudaSuccess) {
        setError("x2_render_adaptive: graph launch failed: %s", cudaGetErrorString(err));
        return X2_ECUDA;
    }
    if (rc) return rc;
    s->waveIterations = ad.hostWords[3];
    if (ad.hostWords[4]) {
        setError("x2_render_adaptive: a pass did not drain after %u iterations", maxIter);
        return X2_EDEVICE;
    }
    x2_adaptive_result r{};
    r.passes = ad.hostWords[1];
    r.samples = *ad.hostSamples;
    r.converged = ad.hostWords[5] ? 1u : 0u;
    r.milliseconds = float(std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
    if (result) *result = r;
    return X2_OK;
}

}  // namespace

int x2_render_adaptive(x2_scene* s, uint32_t minSamples, uint32_t maxSamples, float target, x2_adaptive_result* result) {
    return renderAdaptive(s, minSamples, maxSamples, target, false, result);
}

int x2_render_adaptive_cellular(x2_scene* s, uint32_t minSamples, uint32_t maxSamples, float target, x2_adaptive_result* result) {
    return renderAdaptive(s, minSamples, maxSamples, target, true, result);
}

// A frame by sampling generations under a sample budget: the generations made on the host between passes, as the
// reference makes them (async_render.h Adaptive: rebuild, generate, samplesLeft with budgetBySamples), each pass's
// errors read back from the device and its masks sent to it.
int x2_render_adaptive_budget(x2_scene* s, uint32_t minSamples, uint32_t maxSamples, float floor, uint64_t budget,
                              x2_adaptive_result* result) {
    if (!s || !s->configured || maxSamples == 0 || !(floor >= 0) || budget == 0) {
        setError("x2_render_adaptive_budget: a configured scene, at least one sample, a floor of 0 or more and a budget");
        return X2_EINVAL;
    }
    const auto t0 = std::chrono::steady_clock::now();
    const auto passes = adaptiveSchedule(maxSamples);
    uint32_t most = 0;
    for (const auto& p : passes) most = std::max(most, p.second - p.first);
    if (int rc = x2_frame_begin_adaptive(s, most)) return rc;
    if (int rc = ensureAdaptive(s, floor > 0 ? floor : 1.0f)) return rc;
    AdaptiveState& ad = *s->adaptiveState;
    cudaStream_t st = s->ctx->stream;
    const uint32_t pixels = ad.width * ad.height;
    std::vector<uint64_t> inImage(ad.tiles);
    for (uint32_t t = 0; t < ad.tiles; ++t) {
        uint64_t m = 0;
        const uint32_t tx = (t % ad.tilesX) * 8, ty = (t / ad.tilesX) * 8;
        for (uint32_t p = 0; p < 64; ++p)
            if (tx + p % 8 < ad.width && ty + p / 8 < ad.height) m |= uint64_t(1) << p;
        inImage[t] = m;
    }
    x2::TileGenerations cells(ad.width, ad.height, floor, inImage);
    std::vector<uint32_t> planned(pixels, 0), base(pixels, 0);
    std::vector<float> errors(pixels);
    std::vector<x2_chunk> chunks;
    std::vector<uint64_t> chunkMasks;
    const x2::AdaptiveArgs args = adaptiveArgs(ad);
    double spent = 0;
    x2_adaptive_result r{};
    int rc = X2_OK;
    for (size_t k = 0; k < passes.size() && rc == X2_OK; ++k) {
        const uint32_t size = passes[k].second - passes[k].first;
        const bool uniform = passes[k].first < minSamples;
        std::vector<uint8_t> take;
        if (!uniform) {
            if (spent >= double(budget)) break;  // the budget is spent
            x2::chainPixelErrors<<<(pixels + 255) / 256, 256, 0, st>>>(args, s->sums, s->odd, s->counts);
            cudaMemcpyAsync(errors.data(), ad.errors, sizeof(float) * pixels, cudaMemcpyDeviceToHost, st);
            if (cudaStreamSynchronize(st) != cudaSuccess) {
                rc = X2_ECUDA;
                break;
            }
            const double left = std::max(0.0, double(budget) - spent);
            if (cells.advance(errors.data(), planned, left, maxSamples) == 0) {
                r.converged = 1;
                break;
            }
            take = cells.chosen(size, left);
        }
        chunks.clear();
        chunkMasks.clear();
        uint64_t samples = 0;
        for (uint32_t t = 0; t < ad.tiles; ++t) {
            uint64_t m = inImage[t];
            if (!uniform && !take[t]) m = 0;
            if (!m) continue;
            for (uint32_t p = 0; p < 64; ++p)
                if (m >> p & 1) {
                    const uint32_t pixel = ((t / ad.tilesX) * 8 + p / 8) * ad.width + (t % ad.tilesX) * 8 + p % 8;
                    base[pixel] = planned[pixel];
                    planned[pixel] += size;
                    samples += size;
                }
            chunks.push_back(x2_chunk{t, 0, size, 0});
            chunkMasks.push_back(m);
        }
        if (chunks.empty()) {
            r.converged = 1;
            break;
        }
        spent += double(samples);
        cudaMemcpyAsync(ad.chunkMasks, chunkMasks.data(), sizeof(uint64_t) * chunkMasks.size(), cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(ad.base, base.data(), sizeof(uint32_t) * pixels, cudaMemcpyHostToDevice, st);
        s->launchMask = ad.chunkMasks;
        s->launchBase = ad.base;
        s->samplesPerChunk = size;
        rc = x2_launch_wavefront(s, chunks.data(), uint32_t(chunks.size()));
        s->launchMask = nullptr;
        s->launchBase = nullptr;
        s->samplesPerChunk = most;
        if (rc == X2_OK) rc = x2_wait(s, 600000, nullptr);
        r.passes++;
        r.samples += samples;
    }
    if (rc == X2_OK && cudaMemcpy(ad.planned, planned.data(), sizeof(uint32_t) * pixels, cudaMemcpyHostToDevice) != cudaSuccess) rc = X2_ECUDA;
    r.milliseconds = float(std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
    if (result) *result = r;
    return rc;
}

// ---- the work grid's GPU broker (row f1): launches fed from a grid (grid.cpp), as the reference's feeder feeds
// its GPU lane (async_render.h:780-797) ----
int x2_render_workgrid(x2_scene* s, x2_workgrid* g, uint32_t want, x2_workgrid_result* result) {
    uint32_t width = 0, height = 0, spp = 0;
    x2_workgrid_options o;
    if (!s || !s->configured || !g || !want || x2_workgrid_info(g, &width, &height, &spp, &o) != X2_OK) {
        setError("x2_render_workgrid: a configured scene, a grid and at least one chunk a launch");
        return X2_EINVAL;
    }
    if (width != s->config.width || height != s->config.height) {
        setError("x2_render_workgrid: a %ux%u grid for a %ux%u frame", width, height, s->config.width, s->config.height);
        return X2_EINVAL;
    }
    const auto t0 = std::chrono::steady_clock::now();
    if (int rc = x2_frame_begin(s, o.samples_per_chunk)) return rc;
    std::vector<x2_chunk> chunks(want);
    const uint32_t tilesX = (width + 7) / 8;
    x2_workgrid_result r{};
    int rc = X2_OK;
    for (;;) {
        // A launch holds up to `want` chunks: the broker's takes until it is full or nothing more is handed out (each
        // take moves the frontier on as it claims, so one launch may span several ranges).
        uint32_t got = 0;
        while (got < want) {
            const uint32_t n = x2_workgrid_take(g, want - got, chunks.data() + got);
            if (!n) break;
            got += n;
        }
        if (!got) break;
        // The launch's items are its chunks x 64 x its largest count (the progressive order's first ranges are short).
        uint32_t most = 1;
        uint64_t samples = 0;
        for (uint32_t i = 0; i < got; ++i) {
            const x2_chunk& c = chunks[i];
            most = std::max(most, c.count);
            const uint32_t x = (c.tile % tilesX) * 8, y = (c.tile / tilesX) * 8;
            const uint64_t pixels = uint64_t(std::min(8u, width - x)) * std::min(8u, height - y);
            samples += pixels * c.count;
        }
        s->samplesPerChunk = most;
        rc = x2_launch_wavefront(s, chunks.data(), got);
        s->samplesPerChunk = o.samples_per_chunk;
        x2_completion c{};
        if (rc == X2_OK) rc = x2_wait(s, 600000, &c);
        if (rc) break;
        r.launches++;
        r.chunks += got;
        r.samples += samples;
        r.gpu_milliseconds += c.milliseconds;
    }
    r.milliseconds = float(std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
    if (result) *result = r;
    return rc;
}

int x2_adaptive_planned(x2_scene* s, uint32_t* planned) {
    if (!s || !planned || !s->adaptiveState) {
        setError("x2_adaptive_planned: no adaptive frame");
        return X2_EINVAL;
    }
    if (int rc = x2_wait(s, 600000, nullptr)) return rc;
    const AdaptiveState& a = *s->adaptiveState;
    CUDA_OR(cudaMemcpy(planned, a.planned, sizeof(uint32_t) * a.width * a.height, cudaMemcpyDeviceToHost), X2_ECUDA);
    return X2_OK;
}

// The launch-shape autotuner: coordinate descent over the shape's knobs (paths in flight, refill, triangle tests a step,
// traversal and shade occupancy variants), each candidate timed as a wavefront launch of `tiles` evenly spaced tiles
// at `spp` samples (best of two launches), keeping a knob's best value before the next knob. The results of a launch
// do not depend on its shape, so any choice renders the same film. Leaves the best shape set and the film reset.
int x2_wavefront_autotune(x2_scene* s, uint32_t tiles, uint32_t spp, x2_wavefront_shape* best, float* bestMs) {
    if (!s || !s->configured || spp == 0) {
        setError("autotune: scene not configured or zero spp");
        return X2_EINVAL;
    }
    const uint32_t all = ((s->config.width + 7) / 8) * ((s->config.height + 7) / 8);
    if (tiles == 0 || tiles > all) tiles = all;
    std::vector<x2_chunk> chunks(tiles);
    for (uint32_t i = 0; i < tiles; ++i) chunks[i] = x2_chunk{uint32_t(uint64_t(i) * all / tiles), 0, spp, 0};
    x2_wavefront_shape cur;
    x2_wavefront_shape_defaults(&cur);
    cur.paths = s->reservePaths;
    cur.batch_window = s->batchWindow;
    auto timeShape = [&](const x2_wavefront_shape& sh, float& ms) -> int {
        if (int rc = x2_wavefront_tune(s, &sh)) return rc;
        ms = 3.4e38f;
        for (int k = 0; k < 2; ++k) {
            if (int rc = x2_frame_begin(s, spp)) return rc;
            if (int rc = x2_launch_wavefront(s, chunks.data(), tiles)) return rc;
            x2_completion c{};
            if (int rc = x2_wait(s, 600000, &c)) return rc;
            ms = std::min(ms, c.milliseconds);
        }
        return X2_OK;
    };
    float curMs = 0.0f;
    if (int rc = timeShape(cur, curMs)) return rc;
    const uint64_t items = uint64_t(tiles) * 64ull * spp;
    std::vector<uint32_t> pathOptions;
    for (uint32_t p = 1u << 18; p <= (1u << 23); p <<= 1)
        if (p <= items) pathOptions.push_back(p);
    struct Knob {
        uint32_t x2_wavefront_shape::*field;
        std::vector<uint32_t> values;
    };
    const Knob knobs[] = {{&x2_wavefront_shape::paths, pathOptions},
                          {&x2_wavefront_shape::refill, {4, 8, 16}},
                          {&x2_wavefront_shape::tri_limit, {1, 2, 4}},
                          {&x2_wavefront_shape::shade_blocks, {0, 3, 4, 5}},
                          {&x2_wavefront_shape::trace_blocks, {0, 9}},
                          {&x2_wavefront_shape::blocks_per_sm, {8, 16, 32}},
                          {&x2_wavefront_shape::lobe_queues, {0, 1}},
                          {&x2_wavefront_shape::shadow_order, {0, 1}},
                          {&x2_wavefront_shape::extend_bins, {0, 1}},
                          {&x2_wavefront_shape::short_stack, {0, 1}},
                          {&x2_wavefront_shape::shade_split, {0, 1}},
                          {&x2_wavefront_shape::light_split, {0, 1, 2}},
                          {&x2_wavefront_shape::tri_overlap, {0, 1}}};
    for (const Knob& k : knobs) {
        x2_wavefront_shape keep = cur;
        for (uint32_t v : k.values) {
            if (cur.*k.field == v) continue;
            x2_wavefront_shape trial = cur;
            trial.*k.field = v;
            float ms = 0.0f;
            if (int rc = timeShape(trial, ms)) return rc;
            if (ms < curMs) {
                curMs = ms;
                keep = trial;
            }
        }
        cur = keep;
    }
    if (int rc = x2_wavefront_tune(s, &cur)) return rc;
    if (int rc = x2_frame_begin(s, spp)) return rc;
    if (best) *best = cur;
    if (bestMs) *bestMs = curMs;
    return X2_OK;
}

// Many renders in one wavefront launch: the requests' chunks (every tile of each frame, its sample range) are one work
// list; path slots regenerate across requests, each path shading and tracing in its own request's scene. The work list
// runs in windows of at most kBatchWindow items (the per-item outputs' size); each window's samples are summed into
// their films in sample order, as a single launch's are, so each film equals the one x2_launch_wavefront gives.
int x2_render_batch(x2_ctx* ctx, const x2_request* req, uint32_t n, x2_completion* out) {
    if (!ctx || !req || n == 0 || n > 256 || !req[0].scene) {
        setError("a batch takes 1..256 requests");
        return X2_EINVAL;
    }
    const uint64_t kBatchWindow = req[0].scene->batchWindow ? req[0].scene->batchWindow : (1ull << 27);
    if (int rc = checkDevice(ctx)) return rc;
    uint32_t records = 1, maxDepth = 0;
    for (uint32_t r = 0; r < n; ++r) {
        x2_scene* s = req[r].scene;
        if (!s || s->ctx != ctx || !s->configured || req[r].count == 0 || req[r].count > (1u << 21)) {
            setError("batch request %u: no configured scene of this context, or a sample count outside 1..2^21", r);
            return X2_EINVAL;
        }
        if (s->config.bsdf_samples != 1) {
            setError("batch request %u: the wavefront form takes one BSDF sample a lobe (bsdf_samples = 1)", r);
            return X2_EINVAL;
        }
        for (uint32_t q = 0; q < r; ++q)
            if (req[q].scene == s) {
                setError("batch requests %u and %u render the same scene (one film a scene)", q, r);
                return X2_EINVAL;
            }
        records = std::max(records, s->config.light_count * s->config.light_samples + 1);
        maxDepth = std::max(maxDepth, s->config.max_depth);
    }
    for (uint32_t r = 0; r < n; ++r)
        if (int rc = x2_frame_begin(req[r].scene, req[r].count)) return rc;
    // Host tables: each request's scene and film, each chunk's request.
    std::vector<SceneView> views(n);
    std::vector<BatchFilm> films(n);
    std::vector<x2_chunk> chunks;
    std::vector<uint32_t> chunkReq;
    for (uint32_t r = 0; r < n; ++r) {
        x2_scene* s = req[r].scene;
        views[r] = viewOf(s);
        views[r].stats = nullptr;
        films[r] = BatchFilm{s->sums, s->adaptive ? s->odd : nullptr, s->counts};
        const uint32_t tiles = ((s->config.width + 7) / 8) * ((s->config.height + 7) / 8);
        for (uint32_t t = 0; t < tiles; ++t) {
            chunks.push_back(x2_chunk{t, req[r].first, req[r].count, 0});
            chunkReq.push_back(r);
        }
    }
    const uint32_t chunkTotal = uint32_t(chunks.size());
    // Windows of whole chunks.
    std::vector<uint32_t> windowStart{0};
    uint64_t windowMax = 0;
    {
        uint64_t acc = 0;
        for (uint32_t c = 0; c < chunkTotal; ++c) {
            const uint64_t items = 64ull * chunks[c].count;
            if (acc && acc + items > kBatchWindow) {
                windowStart.push_back(c);
                windowMax = std::max(windowMax, acc);
                acc = 0;
            }
            acc += items;
        }
        windowMax = std::max(windowMax, acc);
        windowStart.push_back(chunkTotal);
    }
    x2_scene* s0 = req[0].scene;
    cudaStream_t st = ctx->stream;
    uint32_t paths = s0->reservePaths ? s0->reservePaths : defaultPaths(records);
    if (uint64_t(paths) > windowMax) paths = uint32_t(windowMax);
    if (int rc = ensureWave(s0, paths, records)) return rc;
    if (int rc = ensureItems(s0, windowMax)) return rc;
    SceneView* dViews = nullptr;
    BatchFilm* dFilms = nullptr;
    x2_chunk* dChunks = nullptr;
    uint32_t* dChunkReq = nullptr;
    unsigned long long* dChunkItems = nullptr;
    Counters* dCounters = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    Counters hc{};
    int rc = X2_OK;
    const int gridLogic = int((paths + kWaveBlock - 1) / kWaveBlock);
    const int gridWork = ctx->smCount * int(s0->blocksPerSm);
    bool anyVolumes = false, anyTextures = false;
    for (const SceneView& v : views) {
        anyVolumes = anyVolumes || v.config.volume_count != 0;
        anyTextures = anyTextures || v.triUV != nullptr;
    }
    const WaveKernels wk = waveKernelsBatch(anyVolumes, anyTextures, s0->shadeSplit != 0);
    std::vector<unsigned long long> items;
    uint32_t iterations = 0;
    if (cudaMalloc(&dViews, sizeof(SceneView) * n) != cudaSuccess || cudaMalloc(&dFilms, sizeof(BatchFilm) * n) != cudaSuccess ||
        cudaMalloc(&dChunks, sizeof(x2_chunk) * chunkTotal) != cudaSuccess || cudaMalloc(&dChunkReq, sizeof(uint32_t) * chunkTotal) != cudaSuccess ||
        cudaMalloc(&dChunkItems, sizeof(unsigned long long) * (chunkTotal + 1)) != cudaSuccess ||
        cudaMalloc(&dCounters, sizeof(Counters)) != cudaSuccess || cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        setError("device allocation failed for a batch of %u requests", n);
        rc = X2_ENOMEM;
    }
    if (!rc) {
        cudaMemcpyAsync(dViews, views.data(), sizeof(SceneView) * n, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(dFilms, films.data(), sizeof(BatchFilm) * n, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(dChunks, chunks.data(), sizeof(x2_chunk) * chunkTotal, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(dChunkReq, chunkReq.data(), sizeof(uint32_t) * chunkTotal, cudaMemcpyHostToDevice, st);
        cudaMemsetAsync(dCounters, 0, sizeof(Counters), st);
        cudaEventRecord(e0, st);
    }
    for (size_t wi = 0; !rc && wi + 1 < windowStart.size(); ++wi) {
        const uint32_t c0 = windowStart[wi], c1 = windowStart[wi + 1];
        items.assign(c1 - c0 + 1, 0ull);
        for (uint32_t c = c0; c < c1; ++c) items[c - c0 + 1] = items[c - c0] + 64ull * chunks[c].count;
        const uint64_t windowItems = items.back();
        // The host table is read by the copy before the next window rewrites it.
        cudaMemcpyAsync(dChunkItems, items.data(), sizeof(unsigned long long) * items.size(), cudaMemcpyHostToDevice, st);
        cudaMemsetAsync(s0->wave.state, 0, sizeof(uint32_t) * paths, st);
        cudaMemsetAsync(s0->wave.ncount, 0, sizeof(uint32_t) * paths, st);
        cudaMemsetAsync(s0->claimed, 0, sizeof(unsigned long long), st);
        cudaMemsetAsync(s0->waveCounters, 0, sizeof(uint32_t) * kWaveCounters, st);
        cudaMemsetAsync(s0->outStatus, X2_SKIP, windowItems, st);
        WaveArgs a{};
        a.scene = views[0];
        a.w = s0->wave;
        a.paths = paths;
        a.recordsPerPath = records;
        a.chunks = dChunks + c0;
        a.itemCount = windowItems;
        a.samplesPerChunk = 0;
        a.claimed = s0->claimed;
        a.extendQ = s0->extendQ;
        a.extendCount = s0->waveCounters;
        a.lastExtend = s0->waveCounters + 1;
        a.shadowQ = s0->shadowQ;
        a.shadowCount = s0->waveCounters + 2;
        a.shadowSlots = s0->shadowOrder && a.recordsPerPath <= x2::kRecordSegments ? s0->waveCounters + 8 : nullptr;
        a.extendSlots = s0->extendBins ? s0->waveCounters + 8 + x2::kRecordSegments : nullptr;
        a.extendNext = s0->waveCounters + 3;
        a.shadowNext = s0->waveCounters + 4;
        a.shadeQ = s0->lobeQueues ? s0->shadeQ : nullptr;
        a.shadeCount = s0->waveCounters + 5;
        a.adj = AdjointWave{};
        a.chunkMask = nullptr;
        a.pixelBase = nullptr;
        a.liveChunks = nullptr;
        a.refill = s0->refill;
        a.triLimit = s0->triLimit;
        a.out = s0->out;
        a.outStatus = s0->outStatus;
        a.counters = dCounters;
        a.scenes = dViews;
        a.chunkRequest = dChunkReq + c0;
        a.chunkItems = dChunkItems;
        a.chunkCount = c1 - c0;
        const uint64_t maxIter = windowItems * (uint64_t(maxDepth) + 2) / paths + uint64_t(maxDepth) + 64;
        constexpr int kIter = 8;
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            setError("stream capture failed");
            rc = X2_ECUDA;
            break;
        }
        for (int it = 0; it < kIter; ++it) {
            wfResetQueues<<<1, 32, 0, st>>>(a);
            wk.logic<<<gridLogic, kWaveBlock, 0, st>>>(a);
            wk.extend<<<gridWork, kWaveBlock, 0, st>>>(a);
            launchShade(wk, a, gridWork, st, true);
            wk.shadow<<<gridWork, kWaveBlock, 0, st>>>(a);
        }
        wfResetQueues<<<1, 32, 0, st>>>(a);
        if (cudaStreamEndCapture(st, &graph) != cudaSuccess || cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess) {
            if (graph) cudaGraphDestroy(graph);
            setError("batch graph capture failed");
            rc = X2_ECUDA;
            break;
        }
        for (uint64_t it = 0;;) {
            if (cudaGraphLaunch(exec, st) != cudaSuccess) {
                setError("graph launch failed");
                rc = X2_ECUDA;
                break;
            }
            it += kIter;
            iterations += kIter;
            cudaMemcpyAsync(s0->hostLast, s0->waveCounters + 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
            if ((rc = x2_synchronize(ctx, 600000)) != X2_OK) break;
            if (s0->hostLast[0] == 0) break;
            if (it > maxIter) {
                setError("batch window did not drain after %llu iterations", (unsigned long long)it);
                rc = X2_EDEVICE;
                break;
            }
        }
        cudaGraphExecDestroy(exec);
        cudaGraphDestroy(graph);
        if (rc) break;
        wfFilmReduceBatch<<<int((64ull * (c1 - c0) + 255) / 256), 256, 0, st>>>(a, dFilms);
        if (cudaGetLastError() != cudaSuccess) {
            setError("batch film reduction failed to launch");
            rc = X2_ECUDA;
        }
    }
    if (!rc) {
        cudaEventRecord(e1, st);
        cudaMemcpyAsync(&hc, dCounters, sizeof(Counters), cudaMemcpyDeviceToHost, st);
        rc = x2_synchronize(ctx, 600000);
    }
    float ms = 0.0f;
    if (!rc) cudaEventElapsedTime(&ms, e0, e1);
    if (out) {
        out->launch = 0;
        out->samples = hc.samples;
        out->errors = hc.errors;
        out->milliseconds = ms;
        out->pad = 0;
    }
    if (!rc) {
        for (uint32_t r = 0; r < n; ++r) req[r].scene->waveIterations = iterations;
        accumulate(s0->total, hc);
    }
    cudaFree(dViews);
    cudaFree(dFilms);
    cudaFree(dChunks);
    cudaFree(dChunkReq);
    cudaFree(dChunkItems);
    cudaFree(dCounters);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (!rc && hc.errors) {
        setError("%llu samples of the batch ended in error", (unsigned long long)hc.errors);
        return X2_EDEVICE;
    }
    return rc;
}

int x2_wavefront_timing(x2_scene* s, int on, float* ms) {
    if (!s) return X2_EINVAL;
    if (ms)
        for (int k = 0; k < 5; ++k) ms[k] = s->waveMs[k];
    if (on >= 0) s->waveTiming = on != 0;
    return X2_OK;
}

int x2_wavefront_queues(x2_scene* s, uint32_t* sizes, uint32_t max) {
    if (!s || !sizes) return X2_EINVAL;
    const uint32_t n = s->waveIterations < kQueueLog ? s->waveIterations : kQueueLog;
    for (uint32_t i = 0; i < 2 * n && i < max; ++i) sizes[i] = s->queueLog[i];
    return X2_OK;
}

int x2_wavefront_info(x2_scene* s, uint32_t* paths, uint32_t* records, uint32_t* iterations) {
    if (!s) return X2_EINVAL;
    if (paths) *paths = s->wavePaths;
    if (records) *records = s->waveRecords;
    if (iterations) *iterations = s->waveIterations;
    return X2_OK;
}

int x2_film_device(x2_scene* s, double** sums, double** odd, uint32_t** counts) {
    if (!s || !s->filmPixels) return X2_EINVAL;
    if (sums) *sums = s->sums;
    if (odd) *odd = s->odd;
    if (counts) *counts = s->counts;
    return X2_OK;
}

int x2_film_download(x2_scene* s, double* sums, double* odd, uint32_t* counts) {
    if (!s || !s->filmPixels) {
        setError("no film");
        return X2_EINVAL;
    }
    if (int rc = checkDevice(s->ctx)) return rc;
    cudaStream_t st = s->ctx->stream;
    const size_t p = s->filmPixels;
    if (sums) cudaMemcpyAsync(sums, s->sums, sizeof(double) * 4 * p, cudaMemcpyDeviceToHost, st);
    if (odd) cudaMemcpyAsync(odd, s->odd, sizeof(double) * 4 * p, cudaMemcpyDeviceToHost, st);
    if (counts) cudaMemcpyAsync(counts, s->counts, sizeof(uint32_t) * p, cudaMemcpyDeviceToHost, st);
    return x2_wait(s, 600000, nullptr);
}

int x2_audit(x2_scene* s, const uint32_t* expected, int64_t* badPixel) {
    if (!s || !s->filmPixels) return X2_EINVAL;
    if (int rc = checkDevice(s->ctx)) return rc;
    cudaStream_t st = s->ctx->stream;
    const unsigned long long none = ~0ull;
    uint32_t* dExpected = nullptr;
    if (expected) {
        CUDA_OR(cudaMallocAsync(&dExpected, sizeof(uint32_t) * s->filmPixels, st), X2_ENOMEM);
        cudaMemcpyAsync(dExpected, expected, sizeof(uint32_t) * s->filmPixels, cudaMemcpyHostToDevice, st);
    }
    cudaMemcpyAsync(s->auditWord, &none, sizeof(none), cudaMemcpyHostToDevice, st);
    auditCounts<<<(s->filmPixels + 255) / 256, 256, 0, st>>>(s->counts, dExpected, s->config.spp, s->filmPixels, s->auditWord);
    unsigned long long first = ~0ull;
    cudaMemcpyAsync(&first, s->auditWord, sizeof(first), cudaMemcpyDeviceToHost, st);
    if (dExpected) cudaFreeAsync(dExpected, st);
    if (int rc = x2_wait(s, 600000, nullptr)) return rc;
    if (badPixel) *badPixel = first == ~0ull ? -1 : int64_t(first);
    if (first != ~0ull) {
        setError("Sample audit failure at pixel %llu", first);
        return X2_EAUDIT;
    }
    return X2_OK;
}

int x2_counters_read(x2_scene* s, x2_counters* out) {
    if (!s || !out) return X2_EINVAL;
    if (int rc = x2_wait(s, 600000, nullptr)) return rc;
    uint32_t overflow = 0;
    cudaMemcpy(&overflow, s->overflow, sizeof(uint32_t), cudaMemcpyDeviceToHost);
    out->trace = s->total.trace;
    out->shadow_nee = s->total.nee;
    out->shadow_bsdf = s->total.bsdf;
    out->held = s->total.held;
    out->samples = s->total.samples;
    out->errors = s->total.errors;
    out->stack_overflows = overflow;
    out->pad = 0;
    return X2_OK;
}

int x2_count_traversal(x2_scene* s, int on) {
    if (!s) return X2_EINVAL;
    if (int rc = x2_wait(s, 600000, nullptr)) return rc;
    s->counting = on != 0;
    return X2_OK;
}

int x2_traversal_counts(x2_scene* s, uint64_t* rays, uint64_t* nodes, uint64_t* triangles) {
    if (!s) return X2_EINVAL;
    if (int rc = x2_wait(s, 600000, nullptr)) return rc;
    TraversalStats h[2]{};
    CUDA_OR(cudaMemcpy(h, s->stats, sizeof(h), cudaMemcpyDeviceToHost), X2_ECUDA);
    CUDA_OR(cudaMemset(s->stats, 0, sizeof(h)), X2_ECUDA);
    for (int k = 0; k < 2; ++k) {
        if (rays) rays[k] = h[k].rays;
        if (nodes) nodes[k] = h[k].nodes;
        if (triangles) triangles[k] = h[k].tris;
    }
    return X2_OK;
}

int x2_traversal_lanes(x2_scene* s, uint64_t* lanes) {
    if (!s || !lanes) return X2_EINVAL;
    if (int rc = x2_wait(s, 600000, nullptr)) return rc;
    TraversalStats h[2]{};
    CUDA_OR(cudaMemcpy(h, s->stats, sizeof(h), cudaMemcpyDeviceToHost), X2_ECUDA);
    for (int k = 0; k < 2; ++k) {
        const unsigned long long v[6] = {h[k].steps, h[k].liveLanes, h[k].nodeSteps, h[k].nodeLanes, h[k].triSteps, h[k].triLanes};
        for (int j = 0; j < 6; ++j) lanes[6 * k + j] = v[j];
    }
    return X2_OK;
}

int x2_counters_reset(x2_scene* s) {
    if (!s) return X2_EINVAL;
    if (int rc = x2_wait(s, 600000, nullptr)) return rc;
    s->total = Counters{};
    return X2_OK;
}

}  // extern "C"
