// The adjoint of the path tracer: gradients of an image loss with respect to each Lambert material's albedo, each GGX
// material's roughness and each light's radiance, by replaying each sample's path from its identity (path replay:
// nothing of the primal pass is stored; Vicini, Speierer and Jakob 2021).
//
// The sampling decisions (directions, light choices, Russian roulette and its scale, MIS weights, pdfs) are held fixed
// at their values for the current parameters: the estimator differentiates only the values a contribution carries.
// Its expectation is the derivative of the image's expectation (each sampling density, held fixed, still integrates
// the differentiated integrand; each decision's weight keeps its expectation), so it is unbiased, and finite
// differences with common random numbers converge to it.
//
// - Light radiance and Lambert albedo enter a contribution multiplicatively: a contribution that reaches light i
//   carries its radiance channel by channel, and one that passed Lambert vertices carries each vertex's albedo once a
//   vertex (the BSDF weight of a cosine-sampled Lambert lobe is its albedo; its light-sample value is albedo / pi
//   times the cosine). So d(contribution)/d(param) = contribution / param channel by channel.
// - GGX roughness enters through the lobe's value f(wo, wi) = F G1(wo) G1(wi) D(m) / cos(wo) at the directions the
//   vertex used: d(contribution)/dr = contribution * dlog f/dr at the light sample's direction for that light
//   sample, and at the BSDF sample's direction for everything the path gathered after the BSDF sample (its light hit
//   and all later vertices).
//
// Each vertex's credit is taken once at the path's end from suffix sums (the radiance gathered after the vertex acted),
// weighted by the loss's derivative for its pixel (dL/dI / samples a pixel). Credits are FP32 sums in the thread and
// atomics into per-block partials in shared memory, reduced once a block into the FP64 gradients.
#include "adjoint.h"
#include "credits.cuh"

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
constexpr uint32_t kGgxVertex = 0x80000000u;  // a vertex record's material index with this bit: a GGX vertex

// A thread's credits. Lights: each contribution, weighted by the loss's derivative for its pixel, over its light's
// radiance, summed in the thread's own array over all its samples, then into the block's partials once. Materials: a
// vertex's lobe scales everything its path gathers after the vertex acted, so at the path's end each vertex k is
// credited once with (radiance at the end - radiance before k acted) * scale[k]: scale = 1 / albedo channel by channel
// for a Lambert vertex (which acts from its light samples on), dlog f/dr at the BSDF sample's direction for a GGX
// vertex (which acts from its BSDF sample on; its light samples are credited one by one as they land).
struct Credits {
    float* partial;
    Layout at;
    const SceneView& s;
    V3 delta;  // dL/dI of the sample's pixel over its samples
    float* lightSum;  // the thread's light credits (kLightSlots x 3)
    // The path's vertices by depth: material (~0u: none; kGgxVertex set: GGX), the radiance before it acted, the scale,
    // a textured Lambert vertex's st and filter.
    uint32_t* material;
    V3* before;
    V3* scale;
    float4* texc;
    float* texGrad;
    uint32_t vertices;

    __device__ void light(V3 c, uint32_t j) {
        if (j == ~0u) return;
        const x2_light& L = s.lights[j];
        const float w[3] = {delta.x * c.x, delta.y * c.y, delta.z * c.z};
        for (int k = 0; k < 3; ++k) {
            if (L.radiance[k] == 0.0f || w[k] == 0.0f) continue;
            const float v = w[k] / L.radiance[k];
            if (j < kLightSlots) lightSum[3 * j + k] += v;
            else atomicAdd(partial + at.radiance(j) + k, v);
        }
    }
    __device__ void roughness(uint32_t m, V3 c, float g) {
        const float v = (delta.x * c.x + delta.y * c.y + delta.z * c.z) * g;
        if (v != 0.0f && finitef(v)) atomicAdd(partial + at.roughness(m), v);
    }
    __device__ void vertexCredits(V3 total) {
        for (uint32_t k = 0; k < vertices; ++k) {
            if (material[k] == ~0u) continue;
            const V3 after = sub(total, before[k]);
            const V3 f = scale[k];
            if (material[k] & kGgxVertex) {
                roughness(material[k] & ~kGgxVertex, after, f.x);
                continue;
            }
            creditLambert(partial, at, s, material[k], make_float4(delta.x, delta.y, delta.z, 0.0f), after, f, texc + k, texGrad);
        }
    }
};

// The replay's sink: shadow rays traced at once as the plain megakernel's; each unoccluded one credited to its light
// (and, at a GGX vertex, a light sample to its roughness).
struct AdjointSink {
    const SceneView& s;
    Credits& cr;
    V3& radiance;
    Pending* stack;
    uint32_t& size;
    uint32_t depth;  // the current vertex's depth
    Lobe lobe;       // the current vertex's lobe, when it is GGX
    V3 wo;
    uint32_t material;
    float materialRoughness;
    bool ggx, sampled;

    __device__ void vertex(uint32_t m, const Bsdf& b, V3 out, const TexHit* tex) {
        const bool lambert = b.count && b.lobe.kind == 0;
        ggx = b.count && b.lobe.kind == 1;
        sampled = false;
        cr.before[depth] = radiance;
        cr.vertices = depth + 1;
        if (lambert) {
            const V3 a = b.lobe.albedo;
            cr.material[depth] = m;
            if (tex) cr.texc[depth] = make_float4(tex->s, tex->t, tex->primary ? 1.0f : 0.0f, 0.0f);
            cr.scale[depth] = V3{a.x != 0.0f ? 1.0f / a.x : 0.0f, a.y != 0.0f ? 1.0f / a.y : 0.0f, a.z != 0.0f ? 1.0f / a.z : 0.0f};
        } else if (ggx) {
            cr.material[depth] = m | kGgxVertex;
            cr.scale[depth] = V3{0, 0, 0};  // until the BSDF sample is taken
            lobe = b.lobe;
            wo = out;
            material = m;
            materialRoughness = s.materials[m].roughness;
        } else {
            cr.material[depth] = ~0u;
        }
    }
    // The BSDF sample's direction, the first time the vertex hands on something that came through it.
    __device__ void bsdfDirection(V3 wi) {
        if (!ggx || sampled) return;
        sampled = true;
        cr.scale[depth] = V3{ggxLogDerivative(lobe, materialRoughness, wo, wi), 0, 0};
    }
    __device__ void shadow(const ShadowReq& q, bool bsdf) {
        if (bsdf) bsdfDirection(q.dir);
        if (!visible(s, q.origin, q.dir, q.near, q.far)) return;
        radiance = add(radiance, q.contribution);
        cr.light(q.contribution, q.light);
        if (ggx && !bsdf) {
            cr.roughness(material, q.contribution, ggxLogDerivative(lobe, materialRoughness, wo, q.dir));
            cr.before[depth] = radiance;  // a GGX vertex's suffix starts after its light samples
        }
    }
    __device__ void held() {}
    __device__ uint32_t top(uint32_t) const { return size; }
    __device__ void push(const Pending& p) {
        bsdfDirection(p.dir);
        stack[size++] = p;
    }
};

// One sample's replay (the plain megakernel's loop, integrator.cuh's integrate, with the credits).
__device__ __noinline__ void adjointSample(const SceneView& s, uint32_t pixel, uint32_t index, V3 delta, float* partial, Layout at,
                                           float* lightSum, float* texGrad) {
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
    V3 before[kMaxPathVertices], scale[kMaxPathVertices];
    float4 texc[kMaxPathVertices];
    Credits cr{partial, at, s, delta, lightSum, material, before, scale, texc, texGrad, 0};
    while (top) {
        Pending pv = stack[--top];
        if (pv.depth >= kMaxPathVertices) continue;
        V3 va, vb, vc;
        const Hit hit = trace(s, pv.origin, pv.dir, pv.nearT, pv.farT, va, vb, vc);
        // The held light (bounce-ray reuse): reached unless the ray met something short of it.
        if (pv.heldLight != ~0u && !(hit.geom != ~0u && hit.t < pv.heldFar)) cr.light(pv.held, pv.heldLight);
        const V3 prior = radiance;
        afterTrace<false>(s, root, pv, hit, cameraPosition, radiance, alpha);
        // The light a camera ray sees (afterTrace added it).
        if (pv.depth == 0 && s.config.visible_lights) {
            const bool missed = hit.geom == ~0u;
            cr.light(sub(radiance, prior),
                     visibleLightIndex(s, root, missed ? pv.origin : cameraPosition, pv.dir, missed ? 3.4028234663852886e+38f : hit.t));
        }
        if (hit.geom == ~0u) continue;
        AdjointSink sink{s, cr, radiance, stack, top, pv.depth};
        if (!shadeVertex<false>(s, root, pixel, index, pv, hit, va, vb, vc, top, radiance, alpha, sink)) return;
    }
    cr.vertexCredits(radiance);
}

}  // namespace

// One thread a sample: chunks of 64 x count items (item = chunk * 64 * count + position * count + sample).
__global__ void __launch_bounds__(128) adjointKernel(SceneView s, const x2_chunk* chunks, uint32_t chunkCount, uint32_t count,
                                                     const float* dLossdImage, double* gradients, uint32_t materials, uint32_t lights,
                                                     float* texGrad) {
    extern __shared__ float partial[];
    const Layout at{materials, lights};
    const uint32_t params = 4 * materials + 3 * lights;
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
        adjointSample(s, pixel, ch.first + sample, delta, partial, at, lightSum, texGrad);
    }
    for (uint32_t j = 0; j < lights && j < kLightSlots; ++j)
        for (int k = 0; k < 3; ++k)
            if (lightSum[3 * j + k] != 0.0f) atomicAdd(partial + at.radiance(j) + k, lightSum[3 * j + k]);
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < params; i += blockDim.x)
        if (partial[i] != 0.0f) atomicAdd(gradients + i, double(partial[i]));
}

}  // namespace x2
