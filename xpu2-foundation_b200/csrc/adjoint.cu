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
// vertex on its way. Credits are FP32 atomics into per-block partials in shared memory, reduced once a block into the
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

// The block's partial gradients: albedo (3 a material) then radiance (3 a light), in shared memory.
struct Credits {
    float* partial;
    uint32_t materials;
    const SceneView& s;
    V3 delta;  // dL/dI of the sample's pixel over its samples
    // The Lambert vertices on the current path, by depth: material (~0u: not a Lambert vertex) and albedo.
    uint32_t* material;
    V3* albedo;

    __device__ void credit(V3 c, uint32_t upTo, uint32_t light) {
        const V3 w{delta.x * c.x, delta.y * c.y, delta.z * c.z};
        if (w.x == 0.0f && w.y == 0.0f && w.z == 0.0f) return;
        if (light != ~0u) {
            const x2_light& L = s.lights[light];
            float* g = partial + 3 * (materials + light);
            if (L.radiance[0] != 0.0f) atomicAdd(g, w.x / L.radiance[0]);
            if (L.radiance[1] != 0.0f) atomicAdd(g + 1, w.y / L.radiance[1]);
            if (L.radiance[2] != 0.0f) atomicAdd(g + 2, w.z / L.radiance[2]);
        }
        for (uint32_t k = 0; k < upTo; ++k) {
            if (material[k] == ~0u) continue;
            float* g = partial + 3 * material[k];
            const V3 a = albedo[k];
            if (a.x != 0.0f) atomicAdd(g, w.x / a.x);
            if (a.y != 0.0f) atomicAdd(g + 1, w.y / a.y);
            if (a.z != 0.0f) atomicAdd(g + 2, w.z / a.z);
        }
    }
};

// The replay's sink: shadow rays traced at once as the plain megakernel's; each unoccluded one credited to its light
// and to the path's Lambert vertices up to and with the current one.
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
    }
    __device__ void shadow(const ShadowReq& q, bool) {
        if (!visible(s, q.origin, q.dir, q.near, q.far)) return;
        radiance = add(radiance, q.contribution);
        cr.credit(q.contribution, depth + 1, q.light);
    }
    __device__ void held() {}
    __device__ uint32_t top(uint32_t) const { return size; }
    __device__ void push(const Pending& p) { stack[size++] = p; }
};

// One sample's replay (the plain megakernel's loop, integrator.cuh's integrate, with the credits).
__device__ __noinline__ void adjointSample(const SceneView& s, uint32_t pixel, uint32_t index, V3 delta, float* partial, uint32_t materials) {
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
    V3 albedo[kMaxPathVertices];
    Credits cr{partial, materials, s, delta, material, albedo};
    while (top) {
        Pending pv = stack[--top];
        if (pv.depth >= kMaxPathVertices) continue;
        V3 va, vb, vc;
        const Hit hit = trace(s, pv.origin, pv.dir, pv.nearT, pv.farT, va, vb, vc);
        // The held light (bounce-ray reuse): the parent's BSDF sample reached it, so it passed the parent too.
        if (pv.heldLight != ~0u && !(hit.geom != ~0u && hit.t < pv.heldFar)) cr.credit(pv.held, pv.depth, pv.heldLight);
        const V3 before = radiance;
        afterTrace(s, root, pv, hit, cameraPosition, radiance, alpha);
        // What afterTrace added besides the held light: the light a camera ray sees (no vertex before it).
        if (pv.depth == 0 && s.config.visible_lights) {
            const V3 added = sub(radiance, before);
            const bool missed = hit.geom == ~0u;
            const uint32_t j = visibleLightIndex(s, root, missed ? pv.origin : cameraPosition, pv.dir, missed ? 3.4028234663852886e+38f : hit.t);
            if (j != ~0u) cr.credit(added, 0, j);
        }
        if (hit.geom == ~0u) continue;
        // The hit's emission (shadeVertex adds it first): through the vertices before it.
        AdjointSink sink{s, cr, radiance, stack, top, pv.depth};
        const uint32_t m = __ldg(s.meshMaterial + hit.geom);
        const MaterialRec& mr = s.materials[m];
        const V3 emission{mr.emission[0], mr.emission[1], mr.emission[2]};
        if (!shadeVertex(s, root, pixel, index, pv, hit, va, vb, vc, top, radiance, alpha, sink)) return;
        if (!isBlack(emission)) cr.credit(mulv(pv.T, emission), pv.depth, ~0u);
    }
}

}  // namespace

// One thread a sample: chunks of 64 x count items (item = chunk * 64 * count + position * count + sample).
__global__ void __launch_bounds__(128) adjointKernel(SceneView s, const x2_chunk* chunks, uint32_t chunkCount, uint32_t count,
                                                     const float* dLossdImage, double* gradients, uint32_t materials, uint32_t lights) {
    extern __shared__ float partial[];
    const uint32_t params = 3 * (materials + lights);
    for (uint32_t i = threadIdx.x; i < params; i += blockDim.x) partial[i] = 0.0f;
    __syncthreads();
    const unsigned long long items = 64ull * chunkCount * count;
    for (unsigned long long item = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; item < items;
         item += (unsigned long long)gridDim.x * blockDim.x) {
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
        adjointSample(s, pixel, ch.first + sample, delta, partial, materials);
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < params; i += blockDim.x)
        if (partial[i] != 0.0f) atomicAdd(gradients + i, double(partial[i]));
}

}  // namespace x2
