// The wavefront form's state and kernels (internal to libx2).
#pragma once
#include "integrator.cuh"

namespace x2 {

constexpr int kWaveBlock = 128;
constexpr uint32_t kRecordSegments = 64;
// Launch-shape defaults (x2_wavefront_tune changes them a scene). Paths in flight: 2^22 (each launch of the traversal
// kernels then has four times the rays of 2^20 for the same ramp-down at its end: 145.3 -> 143.0 -> 155.4 ms for
// 2^21, 2^22, 2^20 on config 1's 4096 tiles).
constexpr uint32_t kDefaultPaths = 1u << 23;
constexpr uint32_t kDefaultRefill = 8, kDefaultBlocksPerSm = 32, kDefaultTraceBlocks = 0, kDefaultShadeBlocks = 4,
                   kDefaultTriLimit = 1, kDefaultShadowOrder = 0, kDefaultExtendBins = 0, kDefaultShortStack = 1,
                   kDefaultShadeSplit = 1, kDefaultLightSplit = 1, kDefaultTriOverlap = 1;
constexpr uint32_t kOctants = 8;

// Path slots (structure of arrays, `paths` slots) and shadow-ray records (recordsPerPath a slot).
struct WaveState {
    float4* ray0;      // origin, near
    float4* ray1;      // direction, far
    float4* T;         // throughput, held light's shadow end
    float4* held;      // held light's contribution, held light index (bits)
    uint4* meta;       // pixel, sample index, packed depths, mirror depth | lobe type << 8
    uint2* branch;     // the vertex's branch address (lo, hi)
    float4* rad;       // radiance so far, alpha
    uint2* hit;        // the extend kernel's closest hit: leaf-order triangle (~0u: none), t bits
    uint32_t* state;   // empty / trace / done / error
    uint32_t* item;    // the slot's work item
    uint32_t* ncount;  // shadow records the last vertex made
    float4* sray0;     // records: origin, near
    float4* sray1;     // direction, far
    float4* scontrib;  // contribution when unoccluded
    uint8_t* svis;     // 1: nothing occludes [near, far]
    // Light samples in a kernel of their own (wavefront shape light_split): each shaded vertex's LightJob (11 uint4),
    // and a word a slot: bit 0 a job waits, bit 1 the BSDF sample's shadow record waits in the slot's last record.
    uint4* lightJob;
    uint32_t* lightFlags;
};
constexpr uint32_t kLightJobWords = 11;

// The adjoint's wavefront form (x2_adjoint): per path slot the vertices it passed (material, the radiance before the
// vertex acted, its credit scale), the sample's dL/dI share, and per shadow record its light and own factor; the
// credits go to per-block shared partials and from there into FP32 gradient rows, summed in FP64 at the end.
struct AdjointWave {
    const float* dLdI;   // 3 floats a pixel; null: not an adjoint launch
    float* rows;         // rowCount x params FP32 partial rows
    uint32_t rowCount, materials, lights;
    uint32_t vertsPerPath;  // max_depth + 1
    uint4* vert;         // slot * vertsPerPath + depth: material | kind bits, radiance before it acted (float bits)
    float4* scale;       // the same: credit scale (Lambert: 1 / albedo; GGX: dlog f/dr at its BSDF direction in x)
    uint32_t* vcount;    // a slot's vertices
    float4* delta;       // a slot's dL/dI share (dL/dI of its pixel over the pixel's samples)
    uint2* aux;          // per shadow record: light | (BSDF record << 31), own roughness factor (float bits)
    float4* tex;         // per vertex record of a textured Lambert vertex: its st and whether primary (bilinear)
    float* texGrad;      // FP32 dL/dtexel, 3 a texel over the scene's textures; null: not wanted
};

struct WaveArgs {
    SceneView scene;
    WaveState w;
    uint32_t paths, recordsPerPath;
    const x2_chunk* chunks;
    unsigned long long itemCount;
    uint32_t samplesPerChunk;
    unsigned long long* claimed;
    uint32_t* extendQ;
    uint32_t* extendCount;
    // The extend queue binned by direction octant (null: one queue in slot order): the rays of octant o at
    // extendQ + o * paths, extendSlots[o] of them (extendCount their total).
    uint32_t* extendSlots;
    uint32_t* lastExtend;
    uint32_t* shadowQ;
    uint32_t* shadowCount;
    // The shadow queue by record (null: by path, each path's records together): record k of every path that made
    // one goes to segment k of the queue (shadowQ + k * paths), shadowSlots[k] entries, so a warp traces the k-th
    // shadow rays of neighbouring paths (mostly toward the same light) instead of one path's rays toward every light.
    // At most kRecordSegments records a path.
    uint32_t* shadowSlots;
    uint32_t* extendNext;  // the extend and shadow kernels' fetch counters over their queues
    uint32_t* shadowNext;
    // Per-lobe shade queues (null: shade walks the extend queue as it is): after extend, wfSortShade sorts the
    // extended paths by the lobe their hit's material makes (GGX, Lambert, none or missed) into three queues of
    // `paths` entries each (shadeQ + k * paths) with counts shadeCount[0..2]; shade walks them in that order, so a
    // warp's lanes run one lobe's code.
    uint32_t* shadeQ;
    uint32_t* shadeCount;
    AdjointWave adj;      // adjoint launches only (adj.dLdI null otherwise)
    // Adaptive passes (null otherwise): each chunk's 8x8 mask of the pixels it samples (bit y * 8 + x) and each
    // pixel's first sample index of the pass (in place of the chunk's first).
    const uint64_t* chunkMask;
    const uint32_t* pixelBase;
    // A launch queued before its chunks are known (an adaptive frame's pass): its chunk count in device memory, read
    // when the launch runs; its items are that count x 64 x samplesPerChunk (null: itemCount and the count given).
    const uint32_t* liveChunks;
    uint32_t refill;       // a warp fetches new rays once this many of its lanes are idle (1..32)
    uint32_t triLimit;     // triangle tests a lane makes a traversal step
    float4* out;          // per item: rgb, alpha
    uint8_t* outStatus;   // per item: SampleStatus (Skip for items that are not samples)
    Counters* counters;
    // Batches (many renders in one launch): each request's scene, each chunk's request and first item (chunkCount + 1
    // entries, the last the item count), the chunk count. Unused by single launches.
    const SceneView* scenes;
    const uint32_t* chunkRequest;
    const unsigned long long* chunkItems;
    uint32_t chunkCount;
};

// A batch request's film (device).
struct BatchFilm {
    double* sums;
    double* odd;  // null: not kept
    uint32_t* counts;
};

// Fills wavefront.cu's copy of the Sobol direction table (every translation unit with sampling kernels has one).
cudaError_t uploadSobolWavefront(const uint32_t directions[17][32]);

// The logic, extend, shade and shadow kernels for an occupancy: at least `traceBlocks` / `shadeBlocks` blocks a SM
// (10, 9 or 0 for the traversals; 4, 3 or 0 for shade; 0 leaves the register allocation to the compiler); and the
// batch forms, which take each path's scene from WaveArgs::scenes. `volumes`: a scene (or any request) has volumes,
// which takes the shade kernel with the volume code (4 blocks a SM); `textures`: a material reads a texture, which
// takes a shade kernel with the lookup.
struct WaveKernels {
    void (*logic)(WaveArgs);
    void (*extend)(WaveArgs);
    void (*shade)(WaveArgs);
    void (*shadow)(WaveArgs);
    void (*shadeBy[3])(WaveArgs);  // shade split by lobe queue (GGX, Lambert, the rest), or null: shade in one kernel
    void (*lightsBy[2])(WaveArgs);  // light samples of the GGX and Lambert queues in kernels of their own, or null
};
// counting: the traversal kernels that count node visits, triangle tests and lane use (the scene view's stats must
// be set).
// shadeSplit: shade as one kernel a per-lobe queue (surface scenes); lightSplit (with shadeSplit; 1 or 2, 0 off): the
// GGX and Lambert queues' light samples in kernels of their own after shade, at 6 (1) or 8 (2) blocks a SM (the wave
// state's lightJob must be allocated).
// overlap: the traversal kernels that overlap a lane's node visits and triangle tests (walkStepOverlap; short stack).
WaveKernels waveKernels(uint32_t traceBlocks, uint32_t shadeBlocks, bool volumes, bool textures, bool shortStack = kDefaultShortStack != 0,
                        bool counting = false, bool shadeSplit = false, uint32_t lightSplit = 0, bool overlap = false);
// The iteration's shade step: the per-lobe sort (when the queues are on) and the shade kernel or kernels (batch: the
// batch form's sort).
void launchShade(const WaveKernels& k, const WaveArgs& a, int grid, cudaStream_t st, bool batch = false);
WaveKernels waveKernelsBatch(bool volumes, bool textures, bool shadeSplit = kDefaultShadeSplit != 0);
__global__ void wfSortShade(WaveArgs a);
__global__ void wfSortShadeBatch(WaveArgs a);
// The adjoint's logic and shade kernels (dynamic shared memory: the gradient count in floats) and the final sum of the
// gradient rows into FP64 (added to grads).
__global__ void wfLogicAdjoint(WaveArgs a);
__global__ void wfShadeAdjoint(WaveArgs a);
__global__ void wfGradRows(const float* rows, uint32_t rowCount, uint32_t params, double* grads);
__global__ void wfResetQueues(WaveArgs a);
// The drain loop's test, last in the body of a conditional while node: go on while the iteration extended a ray, at
// most maxIterations times (then *overrun is set and the loop ends). iterations[0] counts this loop's iterations,
// iterations[1] a running total.
__global__ void wfDrainCheck(WaveArgs a, cudaGraphConditionalHandle loop, uint32_t* iterations, uint32_t maxIterations,
                             uint32_t* overrun);
__global__ void wfFilmReduce(WaveArgs a, uint32_t chunkCount, double* sums, double* odd, uint32_t* counts);
__global__ void wfFilmReduceBatch(WaveArgs a, const BatchFilm* films);

}  // namespace x2
