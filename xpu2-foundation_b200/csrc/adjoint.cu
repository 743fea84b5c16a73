// The adjoint of the path tracer: gradients of an image loss with respect to each Lambert material's albedo and each
// light's radiance, by replaying each sample's path from its identity (path replay: nothing of the primal pass is
// stored; Vicini, Speierer and Jakob 2021).
//
// Both parameters enter a sample's radiance multiplicatively: a contribution that reaches light i carries its radiance
// channel by channel, and one that passed Lambert vertices carries each vertex's albedo once per vertex (the BSDF
// weight of a cosine-sampled Lambert lobe is its albedo; its light-sample value is albedo / pi times the cosine), while
// the sampling decisions (directions, light choices, Russian roulette) are held fixed. So d(contribution)/d(param) =
// contribution / param for every channel where the parameter is not zero, and the replay credits each contribution,
// weighted by the loss's derivative for its pixel (dL/dI / samples a pixel), to the light it reached and to every Lambert
// vertex on its way (each vertex credited once at the path's end with what the path gathered after it). Credits are FP32
// sums in the thread and atomics into per-block partials in shared memory, reduced once a block into the
// FP64 gradients.
#include "integrator.cuh"
#include "adjoint.h"

namespace x2 {

// This translation unit's copy of the Sobol direction table (sampler.cuh).
cudaError_t uploadSobolAdjoint(const uint32_t directions[17][32]) {
    return cudaMemcpyToSymbol(c_sobol, directions, sizeof(uint32_t) * 17 * 32);
}

namespace {

constexpr uint32_t kMaxPathVertices = 128;  // x2_adjoint admits max_depth < 128

__device__ __forceinline__ uint32_t tilePixelA(uint32_t tile, uint32_t position, uint32_t width, uint32_t height) {
    const uint32_t tilesX = (width + 7) / 8;
    const uint32_t x = (tile % tilesX) * 8 + position % 8;
    const uint32_t y = (tile / tilesX) * 8 + position / 8;
    return x < width && y < height ? y * width + x : ~0u;
}

constexpr uint32_t kLightSlots = 32;  // lights whose credits a thread keeps to itself (more: straight to shared memory)

// A thread's credits. Lights: each contribution, weighted by the loss's derivative for its pixel, over its light's
// radiance, summed in the thread's own array over all its samples, then into the block's partials once. Albedos: a
// Lambert vertex's lobe scales everything its path gathers after the vertex (its own light samples and BSDF sample,
// and all that later vertices add through its throughput), so at the path's end each Lambert vertex k is credited
// once with (radiance at the end - radiance before k's lobe acted) / its albedo (path replay's suffix sums).
struct Credits {
    float* partial;  // the block's: 3 a material's albedo, then 3 a light's radiance
    uint32_t materials, lights;
    const SceneView& s;
    V3 delta;  // dL/dI of the sample's pixel over its samples
    float* lightSum;  // the thread's light credits (kLightSlots x 3)
    // The path's vertices by depth: Lambert material (~0u: none) and albedo, and the radiance before its lobe acted.
    uint32_t* material;
    V3* albedo;
    V3* before;
    uint32_t vertices;

    __device__ void light(V3 c, uint32_t j) {
        if (j == ~0u) return;
        const x2_light& L = s.lights[j];
        const float w[3] = {delta.x * c.x, delta.y * c.y, delta.z * c.z};
        for (int k = 0; k < 3; ++k) {
            if (L.radiance[k] == 0.0f || w[k] == 0.0f) continue;
            const float v = w[k] / L.radiance[k];
            if (j < kLightSlots) lightSum[3 * j + k] += v;
            else atomicAdd(partial + 3 * (materials + j) + k, v);
        }
    }
    __device__ void albedos(V3 total) {
        for (uint32_t k = 0; k < vertices; ++k) {
            if (material[k] == ~0u) continue;
            const V3 after = sub(total, before[k]);
            const V3 a = albedo[k];
            float* g = partial + 3 * material[k];
            if (a.x != 0.0f && after.x != 0.0f) atomicAdd(g, delta.x * after.x / a.x);
            if (a.y != 0.0f && after.y != 0.0f) atomicAdd(g + 1, delta.y * after.y / a.y);
            if (a.z != 0.0f && after.z != 0.0f) atomicAdd(g + 2, delta.z * after.z / a.z);
        }
    }
};

// The replay's sink: shadow rays traced at once as the plain megakernel's; each unoccluded one credited to its light.
struct AdjointSink {
    const SceneView& s;
    Credits& cr;
    V3& radiance;
    Pending* stack;
    uint32_t& size;
    uint32_t depth;  // the current vertex's depth
    __device__ void vertex(uint32_t material, const Bsdf& b) {
        const bool lambert = b.count && b.lobe.kind == 0;
        cr.material[depth] = lambert ? material : ~0u;
        cr.albedo[depth] = lambert ? b.lobe.albedo : V3{0, 0, 0};
        cr.before[depth] = radiance;
        cr.vertices = depth + 1;
    }
    __device__ void shadow(const ShadowReq& q, bool) {
        if (!visible(s, q.origin, q.dir, q.near, q.far)) return;
        radiance = add(radiance, q.contribution);
        cr.light(q.contribution, q.light);
    }
    __device__ void held() {}
    __device__ uint32_t top(uint32_t) const { return size; }
    __device__ void push(const Pending& p) { stack[size++] = p; }
};

// One sample's replay (the plain megakernel's loop, integrator.cuh's integrate, with the credits).
__device__ __noinline__ void adjointSample(const SceneView& s, uint32_t pixel, uint32_t index, V3 delta, float* partial, uint32_t materials,
                                           uint32_t lights, float* lightSum) {
    CameraRay camera;
    if (!cameraRay(s, pixel, index, camera)) return;
    const Identity root{pixel, U64(index), U64(s.config.seed), 0};
    Pending stack[kMaxPending];
    uint32_t top = 0;
    cameraPending(camera, stack[top++]);
    const V3 cameraPosition = camera.origin;
    V3 radiance{0, 0, 0};
    float alpha = 0.0f;
    uint32_t material[kMaxPathVertices];
    V3 albedo[kMaxPathVertices], before[kMaxPathVertices];
    Credits cr{partial, materials, lights, s, delta, lightSum, material, albedo, before, 0};
    while (top) {
        Pending pv = stack[--top];
        if (pv.depth >= kMaxPathVertices) continue;
        V3 va, vb, vc;
        const Hit hit = trace(s, pv.origin, pv.dir, pv.nearT, pv.farT, va, vb, vc);
        // The held light (bounce-ray reuse): reached unless the ray met something short of it.
        if (pv.heldLight != ~0u && !(hit.geom != ~0u && hit.t < pv.heldFar)) cr.light(pv.held, pv.heldLight);
        const V3 prior = radiance;
        afterTrace(s, root, pv, hit, cameraPosition, radiance, alpha);
        // The light a camera ray sees (afterTrace added it).
        if (pv.depth == 0 && s.config.visible_lights) {
            const bool missed = hit.geom == ~0u;
            cr.light(sub(radiance, prior),
                     visibleLightIndex(s, root, missed ? pv.origin : cameraPosition, pv.dir, missed ? 3.4028234663852886e+38f : hit.t));
        }
        if (hit.geom == ~0u) continue;
        AdjointSink sink{s, cr, radiance, stack, top, pv.depth};
        if (!shadeVertex(s, root, pixel, index, pv, hit, va, vb, vc, top, radiance, alpha, sink)) return;
    }
    cr.albedos(radiance);
}

}  // namespace

// One thread a sample: chunks of 64 x count items (item = chunk * 64 * count + position * count + sample).
__global__ void __launch_bounds__(128) adjointKernel(SceneView s, const x2_chunk* chunks, uint32_t chunkCount, uint32_t count,
                                                     const float* dLossdImage, double* gradients, uint32_t materials, uint32_t lights) {
    extern __shared__ float partial[];
    const uint32_t params = 3 * (materials + lights);
    for (uint32_t i = threadIdx.x; i < params; i += blockDim.x) partial[i] = 0.0f;
    float lightSum[3 * kLightSlots];
    for (uint32_t i = 0; i < 3 * kLightSlots; ++i) lightSum[i] = 0.0f;
    __syncthreads();
    const unsigned long long items = 64ull * chunkCount * count;
    // Rounds a warp takes together (one item a lane, the warp reconverged between rounds), so its lanes replay
    // neighbouring samples of one pixel side by side instead of drifting apart through their own item sequences.
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long base = (unsigned long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < items; base += stride) {
        const unsigned long long item = base + (threadIdx.x & 31u);
        __syncwarp();
        if (item >= items) continue;
        const uint32_t chunk = uint32_t(item / (64ull * count));
        const uint32_t offset = uint32_t(item - (unsigned long long)chunk * 64ull * count);
        const uint32_t position = offset / count, sample = offset % count;
        const x2_chunk ch = chunks[chunk];
        if (sample >= ch.count) continue;
        const uint32_t pixel = tilePixelA(ch.tile, position, s.config.width, s.config.height);
        if (pixel == ~0u) continue;
        const float inv = 1.0f / float(ch.count);
        const V3 delta{dLossdImage[3ull * pixel] * inv, dLossdImage[3ull * pixel + 1] * inv, dLossdImage[3ull * pixel + 2] * inv};
        if (delta.x == 0.0f && delta.y == 0.0f && delta.z == 0.0f) continue;
        adjointSample(s, pixel, ch.first + sample, delta, partial, materials, lights, lightSum);
    }
    for (uint32_t j = 0; j < lights && j < kLightSlots; ++j)
        for (int k = 0; k < 3; ++k)
            if (lightSum[3 * j + k] != 0.0f) atomicAdd(partial + 3 * (materials + j) + k, lightSum[3 * j + k]);
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < params; i += blockDim.x)
        if (partial[i] != 0.0f) atomicAdd(gradients + i, double(partial[i]));
}

}  // namespace x2
