// Kernels of the render path and their arguments (internal to libx2).
#pragma once
#include "integrator.cuh"

namespace x2 {

constexpr int kRenderBlock = 128;
// Shadow rays a vertex may make in the bounce-at-a-time megakernel (light_count x light_samples + bsdf_samples).
constexpr uint32_t kStepRecords = 24;

struct RenderArgs {
    SceneView scene;
    const x2_chunk* chunks;
    unsigned long long itemCount;   // chunks * 64 * samplesPerChunk
    uint32_t samplesPerChunk;
    unsigned long long* claimed;    // the launch's item counter
    double* sums;
    double* odd;                    // null unless the frame is adaptive
    uint32_t* counts;
    Counters* counters;             // the launch's counters
};

// Fills the Sobol direction table the render kernels read (this device, current context).
cudaError_t uploadSobol(const uint32_t directions[17][32]);

// The plain megakernel and the per-sample kernel, each in three forms: for scenes without volumes or textures (their
// code compiled out), with textures, and with volumes (and textures).
__global__ void renderChunks(RenderArgs a);
__global__ void renderChunksTextured(RenderArgs a);
__global__ void renderChunksVolumes(RenderArgs a);
// The plain megakernel a bounce at a time (surface scenes whose vertices make at most kStepRecords shadow rays), in
// occupancy variants: kMinBlocks blocks a SM that the register allocation must allow.
template <int kMinBlocks>
__global__ void renderSteps(RenderArgs a);
template <int kMinBlocks>
__global__ void renderStepsTextured(RenderArgs a);
__global__ void integratePairs(SceneView s, const uint32_t* pairs, unsigned long long n, double* rgba, uint32_t* status, Counters* counters);
__global__ void integratePairsTextured(SceneView s, const uint32_t* pairs, unsigned long long n, double* rgba, uint32_t* status,
                                       Counters* counters);
__global__ void integratePairsVolumes(SceneView s, const uint32_t* pairs, unsigned long long n, double* rgba, uint32_t* status,
                                      Counters* counters);
__global__ void traceRays(SceneView s, const float* rays, unsigned long long n, uint32_t* tri, float* t, uint32_t* occluded);
__global__ void sampleWords(const x2_identity* ids, const uint32_t* dims, unsigned long long n, uint32_t policy, uint32_t* out);
__global__ void auditCounts(const uint32_t* counts, const uint32_t* expected, uint32_t spp, uint32_t pixels, unsigned long long* firstBad);

}  // namespace x2
