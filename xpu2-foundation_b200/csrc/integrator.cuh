// The path tracer's per-sample loop on the device: the admitted subset of the reference's integratePaths
// (xpu2/interactive/async_integrator.h:1986-3042).
//
// A vertex is shaded by shadeVertex (held light, camera-visible lights, emission, light samples, BSDF sample and the
// child ray). It hands its shadow rays and its child to a Sink: the plain megakernel's sink traces shadow rays at
// once and pushes children on a per-thread pending stack (integrate, below); the wavefront's sink (wavefront.cu)
// writes shadow-ray records for the any-hit kernel and the child ray for the next extend kernel. Contributions are
// added to the sample's radiance in the reference's order in both forms, so both give the same sums.
#pragma once
#include "shading.cuh"

namespace x2 {

constexpr uint32_t kMaxPending = 32, kPendingReserve = 16;

// paths::Pending (async_integrator.h:201-235), the fields the admitted paths use.
struct Pending {
    V3 origin, dir, T;
    U64 branch;
    uint32_t depth, nonMirror, diffuse, glossy, mirror, lobeType;
    uint32_t volumeDepth;  // the volume scattering it has been through, every bounce counting one
    float nearT, farT;
    uint32_t heldLight;
    float heldFar;
    V3 held;
};
struct SampleOut {
    float rgb[3];
    float alpha;
    uint32_t status;
    uint32_t trace, nee, bsdf, held;
};

}  // namespace x2

#include "volume.cuh"
#include "tracking.cuh"

namespace x2 {

// paths::roulette (async_integrator.h:141-149).
__device__ __forceinline__ bool roulette(float lum, float threshold, float u, float& scale) {
    scale = 1;
    if (lum >= threshold) return true;
    if (lum < u * threshold) return false;
    scale = threshold / lum;
    return true;
}

// visibleLightRadiance (async_integrator.h:383-412): the lights a camera ray meets, one chosen uniformly.
__device__ __forceinline__ V3 visibleLights(const SceneView& s, const Identity& root, V3 origin, V3 dir, float maxDistance) {
    const x2_config& c = s.config;
    uint32_t hits = 0;
    for (uint32_t pass = 0; pass < 3; ++pass)
        for (uint32_t j = 0; j < c.light_count; ++j) {
            const x2_light& L = s.lights[j];
            LightHit lh;
            const uint32_t vp = L.type == X2_LIGHT_ENV ? 2u : L.type == X2_LIGHT_DISTANT ? 1u : 0u;
            if (L.visible_in_camera && vp == pass && lightIntersect(L, origin, dir, maxDistance, lh)) ++hits;
        }
    if (!hits) return V3{0, 0, 0};
    Identity id = root;
    id.branch = childBranch(0x5649534c49474854ull, 0, 0);
    Stream st(id, 0, 0);
    const float choice = st.next();
    const uint32_t chosen = uint32_t(choice * float(hits)) < hits ? uint32_t(choice * float(hits)) : hits - 1;
    uint32_t seen = 0;
    for (uint32_t pass = 0; pass < 3; ++pass)
        for (uint32_t j = 0; j < c.light_count; ++j) {
            const x2_light& L = s.lights[j];
            LightHit lh;
            const uint32_t vp = L.type == X2_LIGHT_ENV ? 2u : 0u;
            if (!L.visible_in_camera || vp != pass || !lightIntersect(L, origin, dir, maxDistance, lh)) continue;
            if (seen++ != chosen) continue;
            float pdf;
            const V3 Li = lightEval(L, dir, lh, pdf);
            return finite3(Li) ? mul(Li, float(hits)) : V3{0, 0, 0};
        }
    return V3{0, 0, 0};
}

// The light visibleLights picks for the same ray (~0u: none): the adjoint credits that light.
__device__ __forceinline__ uint32_t visibleLightIndex(const SceneView& s, const Identity& root, V3 origin, V3 dir, float maxDistance) {
    const x2_config& c = s.config;
    uint32_t hits = 0;
    for (uint32_t pass = 0; pass < 3; ++pass)
        for (uint32_t j = 0; j < c.light_count; ++j) {
            const x2_light& L = s.lights[j];
            LightHit lh;
            const uint32_t vp = L.type == X2_LIGHT_ENV ? 2u : L.type == X2_LIGHT_DISTANT ? 1u : 0u;
            if (L.visible_in_camera && vp == pass && lightIntersect(L, origin, dir, maxDistance, lh)) ++hits;
        }
    if (!hits) return ~0u;
    Identity id = root;
    id.branch = childBranch(0x5649534c49474854ull, 0, 0);
    Stream st(id, 0, 0);
    const float choice = st.next();
    const uint32_t chosen = uint32_t(choice * float(hits)) < hits ? uint32_t(choice * float(hits)) : hits - 1;
    uint32_t seen = 0;
    for (uint32_t pass = 0; pass < 3; ++pass)
        for (uint32_t j = 0; j < c.light_count; ++j) {
            const x2_light& L = s.lights[j];
            LightHit lh;
            const uint32_t vp = L.type == X2_LIGHT_ENV ? 2u : L.type == X2_LIGHT_DISTANT ? 1u : 0u;
            if (!L.visible_in_camera || vp != pass || !lightIntersect(L, origin, dir, maxDistance, lh)) continue;
            if (seen++ == chosen) return j;
        }
    return ~0u;
}

// The camera ray of sample (pixel, index) as integratePaths makes it (async_integrator.h:1994-2026).
__device__ __forceinline__ bool cameraRay(const SceneView& s, uint32_t pixel, uint32_t index, CameraRay& camera) {
    const x2_config& c = s.config;
    if (pixel >= c.width * c.height || c.bsdf_samples == 0 || c.bsdf_samples > 64 || c.light_samples == 0 || c.light_samples > 64)
        return false;
    const Identity root{pixel, U64(index), U64(c.seed), 0};
    float x, y;
    if (!boxFilter(c.filter_width, draw(root, 0, c.sampling), x) || !boxFilter(c.filter_width, draw(root, 1, c.sampling), y)) return false;
    return perspectiveRay(s.camera, float(pixel % c.width) + x, float(pixel / c.width) + y, camera);
}

__device__ __forceinline__ void cameraPending(const CameraRay& camera, Pending& p0) {
    p0.origin = camera.origin;
    p0.dir = camera.direction;
    p0.T = V3{1, 1, 1};
    p0.branch = 0;
    p0.depth = p0.nonMirror = p0.diffuse = p0.glossy = p0.mirror = p0.lobeType = 0;
    p0.volumeDepth = 0;
    p0.nearT = camera.nearT;  // a camera ray is traced on the camera's clip range
    p0.farT = camera.farT;
    p0.heldLight = ~0u;
    p0.heldFar = 0.0f;
    p0.held = V3{0, 0, 0};
}

// After a ray is traced, before its hit is shaded: the light its BSDF sample held is settled (bounce-ray reuse:
// reached unless the ray met something short of the shadow ray's end; lightShadowKept is 0 without a clear radius),
// then, on a camera ray, the lights the camera sees (async_integrator.h:2095-2106, :2172-2185).
// With volumes, the volumes the ray passes on its way (async_integrator.h:2107-2118): their light, the throughput
// through them (pv's T and volume depth change) and, for a camera ray that hits nothing, their opacity as its alpha.
// kVolumes false compiles the volume code out (the kernels for scenes without volumes: the march's state would
// otherwise take registers and stack from every surface vertex); a scene with volumes takes the kVolumes form.
template <bool kVolumes = true>
__device__ __forceinline__ void afterTrace(const SceneView& s, const Identity& root, Pending& pv, const Hit& hit, V3 cameraPosition,
                                           V3& radiance, float& alpha) {
    if (pv.heldLight != ~0u) {
        const float kept = hit.geom != ~0u && hit.t < pv.heldFar ? 0.0f : 1.0f;
        if (kept > 0.0f) radiance = add(radiance, kept < 1.0f ? mul(pv.held, kept) : pv.held);
    }
    V3 volumeAlphaT{1, 1, 1};
    if (kVolumes && s.config.volume_count) {
        const float tEnd = hit.geom == ~0u ? pv.farT : hit.t;
        const V3 volumeLight = s.config.volume_estimator == 1 ? volumeRadianceTracked(s, root, pv, pv.origin, pv.dir, pv.nearT, tEnd, volumeAlphaT)
                                                              : volumeRadiance(s, root, pv, pv.origin, pv.dir, pv.nearT, tEnd, volumeAlphaT);
        radiance = add(radiance, volumeLight);
    }
    // A camera ray that hits nothing: the volumes' opacity (none without volumes: 1 - (1+1+1)/3); a hit adds one (its
    // holdouts' minimum transmittance is zero with no holdouts; shadeVertex).
    if (hit.geom == ~0u && pv.depth == 0) alpha += 1.0f * (1.0f - (volumeAlphaT.x + volumeAlphaT.y + volumeAlphaT.z) / 3.0f);
    if (pv.depth == 0 && s.config.visible_lights) {
        const bool missed = hit.geom == ~0u;
        const V3 Lv = mulv(pv.T, visibleLights(s, root, missed ? pv.origin : cameraPosition, pv.dir, missed ? 3.4028234663852886e+38f : hit.t));
        radiance = add(radiance, Lv);
    }
}

// A shadow ray and what it carries when nothing occludes [near, far].
struct ShadowReq {
    V3 origin, dir;
    float near, far;
    V3 contribution;
    uint32_t light;  // the light it reaches
};

// What a vertex's light samples read: the shading point and its frame, the path's throughput and identity, the lobe,
// and the vertex's sampling switches (shadeVertex fills it).
struct LightJob {
    V3 P, Ng, wo, T, above, below, cull;
    Lobe lobe;
    U64 branch;
    uint32_t pixel, index, depth, nl, nk;
    bool hasCull, split, clampHere, rr;
};

// A vertex's light samples (async_integrator.h:2633-2772): every light of the set that can light the hit, each sample's
// contribution, MIS-weighted against the lobe, clamped and rouletted, to the sink as a shadow request, in light order.
// root: the sample's identity (pixel, index, the frame seed, branch 0).
template <bool kVolumes, int kLobe, class Sink>
__device__ __forceinline__ void lightSamples(const SceneView& s, const Identity& root, const LightJob& j, Sink& sink) {
    const x2_config& c = s.config;
    const uint32_t policy = c.sampling;
    const bool volumes = kVolumes && c.volume_count;
    const V3* cullN = j.hasCull ? &j.cull : nullptr;
    const Slice slice{j.Ng, j.wo};
    const uint32_t nl = j.nl, nk = j.nk;
    const uint32_t pixel = j.pixel, index = j.index;
    const Lobe& lobe = j.lobe;
    const V3 above = j.above, below = j.below;
    const U64 lightBranch = childBranch(j.branch, 0xfffe, 0);
    for (uint32_t i = 0; i < c.light_count; ++i) {
        const x2_light& L = s.lights[i];
        if (!canIlluminate(L, j.P, cullN)) continue;
        const U64 lightAddress = childBranch(lightBranch, i, 0);
        Identity lid = root;
        lid.branch = lightAddress;
        Stream ls(lid, j.depth, 0);
        for (uint32_t si = 0; si < nl; ++si) {
            float r[3];
            r[0] = ls.next();
            r[1] = ls.next();
            r[2] = ls.next();
            const float u = ls.next();
            if (j.split) {
                const Identity strat{pixel, U64(index) * nl + si, U64(c.seed), lightAddress};
                drawPair(strat, CameraDimensions + 2, policy, r[0], r[1]);
            }
            V3 wi;
            LightHit lh;
            if (!lightSample(L, j.P, cullN, r, wi, lh)) continue;
            float pdfL;
            const V3 Li = lightEval(L, wi, lh, pdfL);
            if (pdfL == 0.0f || isExactlyZero(Li) || !(fabsf(pdfL) < 3.4e38f) || !finite3(Li)) continue;
            const V3 factor = mul(mulv(j.T, Li), 1.0f / (float(nl) * pdfL * 1.0f));
            const uint32_t flags = surfaceFlags(slice, wi);
            V3 t{0, 0, 0};
            bool any = false;
            if (matchesFlags(lobe.type, flags) && (lobeRayMask(lobe.type) & L.visibility_mask)) {
                float pdf;
                const V3 f = lobeEvalAs<kLobe>(lobe, slice, wi, pdf);
                if (!(pdf == 0.0f || isExactlyZero(f))) {
                    V3 tk = mul(mulv(factor, f), powerHeuristic(float(nl) * pdfL, float(nk) * pdf));
                    if (j.clampHere && c.clamp_value > 0) {
                        const float mx = fmaxf(tk.x, fmaxf(tk.y, tk.z));
                        if (mx > c.clamp_value) tk = mul(tk, c.clamp_value / mx);
                    }
                    t = add(t, tk);
                    any = true;
                }
            }
            if (!any) continue;
            if (j.rr) {
                float scale;
                if (!roulette(luminance(t), c.rr_threshold, u, scale)) continue;
                t = mul(t, scale);
            }
            if (!finite3(t) || isExactlyZero(t)) continue;
            ShadowReq q;
            q.origin = dot(wi, j.Ng) >= 0.0f ? above : below;
            q.dir = wi;
            q.near = fmaxf(0.0f, 0.0f);
            q.far = fmaxf((lh.distance - 0.0f) * kHitEpsilonEnd, 2.0f * q.near);
            if (volumes) {
                // The volumes on the shadow ray's way (transmittance(), async_integrator.h:2722-2731); it matters only
                // when nothing occludes the ray, and its stream is its own, so it is taken here.
                Identity tid = lid;
                tid.branch = childBranch(lightAddress, si, 0xfffb);
                Stream vs(tid, j.depth, 0);
                t = s.config.volume_estimator == 1 ? mul(t, trackedTransmittance(s, vs, q.origin, wi, q.near, q.far))
                                                   : mulv(t, volumeTransmittance(s, vs, q.origin, wi, q.near, q.far, 1.0f, int(j.depth) + 1));
            }
            q.contribution = t;
            q.light = i;
            sink.shadow(q, false);
        }
    }
}

// One hit (async_integrator.h:2222-3031 for the admitted materials): shading state, emission, a light sample of
// every light that can light the hit, the lobe's BSDF sample, and its child. `top` is the pending stack's size after
// this vertex was popped. The sink takes shadow rays (shadow(req, bsdf)) and the child (push(child) -> bool).
// Returns false when the hit's shading state cannot be made (SampleStatus::Error). kVolumes as afterTrace's; kTextures
// false compiles the texture lookup out (the kernels for scenes whose materials read no texture).
// kLobe: the lobe kind every vertex of the launch makes (1 Lambert, 2 GGX; 0 any), as the per-lobe shade queues sort
// them; the kernel then holds one lobe's evaluation and sampling code.
// kDeferLights: the light samples are not taken here; the sink gets the vertex's LightJob (sink.lights) instead.
template <bool kVolumes = true, bool kTextures = true, int kLobe = 0, bool kDeferLights = false, class Sink>
__device__ __forceinline__ bool shadeVertex(const SceneView& s, const Identity& root, uint32_t pixel, uint32_t index, const Pending& pv,
                                            const Hit& hit, V3 va, V3 vb, V3 vc, uint32_t top, V3& radiance, float& alpha, Sink& sink) {
    const x2_config& c = s.config;
    const uint32_t policy = c.sampling;
    const bool volumes = kVolumes && c.volume_count;
    State st;
    // A mesh's texture coordinates set its partial derivatives (the reference binds them for every mesh of a scene that
    // has them); the device keeps them for scenes with textures.
    const float* stCoords = kTextures && s.triUV ? s.triUV + 6ull * (__ldg(s.meshFirst + hit.geom) + hit.prim) : nullptr;
    if (!hitState(va, vb, vc, hit.u, hit.v, hit.point, pv.dir, st, stCoords)) return false;
    Bsdf bsdf;
    const uint32_t material = __ldg(s.meshMaterial + hit.geom);
    const MaterialRec& mr = s.materials[material];
    TexHit th;
    th.primary = 0;
    if (kTextures && mr.texture) {
        // The hit's st (hitState, shade_material.h:142-153: w st1 + u st2 + v st3) and the texture's lookup there; the
        // path type picks the filter (PathPrimary: no diffuse, glossy or mirror bounce yet, async_integrator.h:2222).
        const float* uv = s.triUV + 6ull * (__ldg(s.meshFirst + hit.geom) + hit.prim);
        const float w = 1.0f - hit.u - hit.v;
        th.s = w * uv[0] + hit.u * uv[2] + hit.v * uv[4];
        th.t = w * uv[1] + hit.u * uv[3] + hit.v * uv[5];
        th.primary = pv.diffuse == 0 && pv.glossy == 0 && pv.mirror == 0;
        if (!texLookup(s, mr.texture - 1, th)) return false;
    }
    shadeMaterial(mr, st, bsdf, kTextures && mr.texture ? th.texel : V3{1, 1, 1});
    if (pv.depth == 0) alpha += 1.0f * (1.0f - (0.0f + 0.0f + 0.0f) / 3.0f);
    radiance = add(radiance, mulv(pv.T, bsdf.emission));
    sink.vertex(material, bsdf, st.wo, kTextures && mr.texture ? &th : nullptr);  // the vertex, its emission added: what comes after passes its lobe
    if (bsdf.count == 0) return true;

    uint32_t indirectFlags = 0;
    if (c.bsdf_samples > 0 && c.max_depth > 0 && pv.depth < c.max_depth) {
        if (pv.diffuse < c.max_diffuse_depth) indirectFlags |= kAllDiffuse;
        if (pv.glossy < c.max_glossy_depth) indirectFlags |= kAllGlossy;
        if (pv.mirror < c.max_mirror_depth) indirectFlags |= kAllMirror;
        if (0u < c.max_hair_depth) indirectFlags |= kAllSurfaceSides;
    }
    const bool doIndirect = indirectFlags != 0;
    V3 cull{0, 0, 0};
    const V3* cullN = nullptr;
    if ((bsdf.type & kAllSurfaceSides) != kAllSurfaceSides) {
        cull = (bsdf.type & kReflection) ? st.Ng : neg(st.Ng);
        cullN = &cull;
    }
    const Slice slice{st.Ng, st.wo};
    const bool split = pv.nonMirror == 0;
    const uint32_t nl = split ? c.light_samples : 1;
    const bool clampHere = pv.nonMirror >= c.clamp_depth;
    const bool rr = pv.nonMirror > 0 && c.rr_threshold > 0;
    const Lobe& lobe = bsdf.lobe;
    const bool mirror = (lobe.type & kMirror) != 0;
    const uint32_t nk = (!split || mirror) ? 1u : c.bsdf_samples;
    const float thinning = [&] {
        const uint32_t room = top < kPendingReserve ? kPendingReserve - top : 1u;
        return nk > room ? float(room) / float(nk) : 1.0f;
    }();
    const V3 above = hit.origin, below = hit.below;

    // Light samples: here, or (kDeferLights) handed to the sink for a kernel of their own, which runs lightSamples on the
    // same job.
    {
        LightJob job;
        job.P = st.P;
        job.Ng = st.Ng;
        job.wo = st.wo;
        job.T = pv.T;
        job.above = above;
        job.below = below;
        job.cull = cull;
        job.hasCull = cullN != nullptr;
        job.lobe = lobe;
        job.branch = pv.branch;
        job.pixel = pixel;
        job.index = index;
        job.depth = pv.depth;
        job.nl = nl;
        job.nk = nk;
        job.split = split;
        job.clampHere = clampHere;
        job.rr = rr;
        if constexpr (kDeferLights) sink.lights(job);
        else lightSamples<kVolumes, kLobe>(s, root, job, sink);
    }

    // The lobe's BSDF samples (async_integrator.h:2792-3031).
    const uint32_t lobeMask = lobeRayMask(lobe.type);
    const bool lobeIndirect = matchesFlags(lobe.type, indirectFlags);
    const U64 lobeBranch = childBranch(pv.branch, 0, 0xffff);
    for (uint32_t i = 0; i < nk; ++i) {
        const U64 sampleBranch = childBranch(lobeBranch, i, 0);
        Identity bid = root;
        bid.branch = sampleBranch;
        Stream bs(bid, pv.depth, 0);
        float r1 = bs.next(), r2 = bs.next();
        const float choice = bs.next(), u = bs.next();
        if (split && !mirror) {
            const Identity strat{pixel, U64(index) * nk + i, U64(c.seed), lobeBranch};
            drawPair(strat, CameraDimensions, policy, r1, r2);
        }
        V3 wi;
        float pdf;
        const V3 f = lobeSampleAs<kLobe>(lobe, slice, r1, r2, wi, pdf);
        if (pdf == 0.0f || isExactlyZero(f) || !finite3(f) || !finite3(wi)) continue;
        if (!matchesFlags(lobe.type, surfaceFlags(slice, wi))) continue;
        const V3 pt = mul(mulv(pv.T, f), 1.0f / (float(nk) * pdf));
        uint32_t hits = 0;
        for (uint32_t j = 0; j < c.light_count; ++j) {
            LightHit lh;
            if ((lobeMask & s.lights[j].visibility_mask) && lightIntersect(s.lights[j], st.P, wi, 3.4028234663852886e+38f, lh)) ++hits;
        }
        V3 direct{0, 0, 0};
        float lightDistance = 0;
        bool lightHit = false;
        uint32_t lightIndex = 0;
        if (hits) {
            const uint32_t chosen = uint32_t(choice * float(hits)) < hits ? uint32_t(choice * float(hits)) : hits - 1;
            for (uint32_t j = 0, seen = 0; j < c.light_count; ++j) {
                LightHit lh;
                if (!(lobeMask & s.lights[j].visibility_mask) || !lightIntersect(s.lights[j], st.P, wi, 3.4028234663852886e+38f, lh)) continue;
                if (seen++ != chosen) continue;
                float pdfL;
                const V3 Li = mul(lightEval(s.lights[j], wi, lh, pdfL), float(hits));
                if (!(pdfL == 0.0f || isExactlyZero(Li)) && fabsf(pdfL) < 3.4e38f && finite3(Li)) {
                    direct = mirror ? mulv(Li, pt) : mul(mulv(Li, pt), powerHeuristic(float(nk) * pdf, float(nl) * pdfL));
                    lightDistance = lh.distance;
                    lightHit = true;
                    lightIndex = j;
                }
                break;
            }
        }
        if (!lightHit && !doIndirect) continue;
        if (clampHere && c.clamp_value > 0) {
            const float mx = fmaxf(direct.x, fmaxf(direct.y, direct.z));
            if (mx > c.clamp_value) direct = mul(direct, c.clamp_value / mx);
        }
        V3 indirect = doIndirect ? pt : V3{0, 0, 0};
        if (rr) {
            float scale;
            if (!roulette(fmaxf(luminance(direct), luminance(indirect)), c.rr_threshold, u, scale)) continue;
            direct = mul(direct, scale);
            indirect = mul(indirect, scale);
        }
        const V3 origin = dot(wi, st.Ng) >= 0.0f ? above : below;
        const float start = 0.0f;
        float shadowNear = start, shadowFar = 0.0f;
        const bool bounces = lobeIndirect && !isExactlyZero(indirect) && finite3(indirect);
        bool held = false;
        const uint32_t topNow = sink.top(top);
        if (lightHit && !isBlack(direct) && finite3(direct)) {
            shadowNear = fmaxf(shadowNear, 0.0f);
            shadowFar = fmaxf((lightDistance - 0.0f) * kHitEpsilonEnd, 2.0f * shadowNear);
            held = bounces && thinning >= 1.0f && topNow + kPendingReserve < kMaxPending && lobeMask && (c.shadow_reuse & lobeMask) == lobeMask &&
                   !volumes && shadowNear == start;
            if (held) {
                sink.held();
            } else {
                ShadowReq q;
                q.origin = origin;
                q.dir = wi;
                q.near = shadowNear;
                q.far = shadowFar;
                q.contribution = direct;
                q.light = lightIndex;
                if (volumes) {
                    Identity tid = bid;
                    tid.branch = childBranch(sampleBranch, 0xfffb, 0);
                    Stream vs(tid, pv.depth, 0);
                    q.contribution = s.config.volume_estimator == 1
                                         ? mul(direct, trackedTransmittance(s, vs, origin, wi, shadowNear, shadowFar))
                                         : mulv(direct, volumeTransmittance(s, vs, origin, wi, shadowNear, shadowFar, 1.0f, int(pv.depth) + 1));
                }
                sink.shadow(q, true);
            }
        }
        const V3 directBefore = direct;
        if (!bounces) continue;
        float keptShare = 1.0f;
        if (thinning < 1.0f || topNow + kPendingReserve >= kMaxPending) {
            Identity kid = bid;
            kid.branch = childBranch(sampleBranch, 0xfff7, 0);
            Stream chance(kid, pv.depth, 0);
            if (thinning < 1.0f) {
                if (chance.next() >= thinning) continue;
                keptShare = 1.0f / thinning;
            }
            if (topNow + kPendingReserve >= kMaxPending) {
                if (topNow >= kMaxPending) continue;
                const float ch = float(kMaxPending - topNow) / float(kPendingReserve + 1);
                if (chance.next() >= ch) continue;
                keptShare *= 1.0f / ch;
            }
        }
        Pending child;
        child.origin = origin;
        child.dir = wi;
        child.T = mul(indirect, keptShare);
        child.branch = sampleBranch;
        child.depth = pv.depth + 1;
        child.diffuse = pv.diffuse + ((lobe.type & kDiffuse) ? 1 : 0);
        child.glossy = pv.glossy + ((lobe.type & kGlossy) ? 1 : 0);
        child.mirror = pv.mirror + (mirror ? 1 : 0);
        child.nonMirror = pv.nonMirror + (mirror ? 0 : 1);
        child.farT = kFltMax;
        child.nearT = start;
        child.lobeType = lobe.type;
        child.volumeDepth = pv.volumeDepth + 1;
        child.heldLight = held ? lightIndex : ~0u;
        child.heldFar = held ? shadowFar : 0.0f;
        child.held = held ? directBefore : V3{0, 0, 0};
        sink.push(child);
    }
    return true;
}

// The plain megakernel's sink: shadow rays traced at once, children on the thread's pending stack.
// The pending stack's top entry lives in registers (topSlot, hasTop) and the rest in `stack`, so a path that never
// branches (one BSDF sample of one lobe: every admitted wavefront scene) touches no local memory for its pending rays;
// the order is the stack's, last pushed first popped.
struct PlainSink {
    const SceneView& s;
    V3& radiance;
    Pending* stack;
    uint32_t& size;
    Pending& topSlot;
    bool& hasTop;
    SampleOut& out;
    __device__ void shadow(const ShadowReq& q, bool bsdf) {
        if (bsdf) ++out.bsdf;
        else ++out.nee;
        if (visible(s, q.origin, q.dir, q.near, q.far)) {
            radiance = add(radiance, q.contribution);
            X2_DIAG_RECORD(mf::kAdded, bsdf ? 1.0f : 0.0f, q.contribution.x, q.contribution.y, q.contribution.z);
        }
    }
    __device__ void held() { ++out.held; }
    __device__ void vertex(uint32_t, const Bsdf&, V3, const TexHit*) {}
    __device__ uint32_t top(uint32_t) const { return size + (hasTop ? 1u : 0u); }
    __device__ void push(const Pending& p) {
        if (hasTop) stack[size++] = topSlot;
        topSlot = p;
        hasTop = true;
    }
};

// integratePaths for one sample (pixel, index): the plain megakernel's whole path loop on one thread.
template <bool kVolumes, bool kTextures>
static __device__ __noinline__ void integrate(const SceneView& s, uint32_t pixel, uint32_t index, SampleOut& out) {
    const x2_config& c = s.config;
    out.rgb[0] = out.rgb[1] = out.rgb[2] = 0.0f;
    out.alpha = 0.0f;
    out.trace = out.nee = out.bsdf = out.held = 0;
    CameraRay camera;
    if (!cameraRay(s, pixel, index, camera)) {
        out.status = X2_ERROR;
        return;
    }
    const Identity root{pixel, U64(index), U64(c.seed), 0};
    Pending stack[kMaxPending];
    uint32_t size = 0;
    Pending topSlot;
    bool hasTop = true;
    cameraPending(camera, topSlot);
    const V3 cameraPosition = camera.origin;
    V3 radiance{0, 0, 0};
    float alpha = 0.0f;
    PlainSink sink{s, radiance, stack, size, topSlot, hasTop, out};
    while (hasTop || size) {
        Pending pv;
        if (hasTop) {
            pv = topSlot;
            hasTop = false;
        } else {
            pv = stack[--size];
        }
        const uint32_t top = size;  // the pending stack's size after the pop
        V3 va, vb, vc;
        const Hit hit = trace(s, pv.origin, pv.dir, pv.nearT, pv.farT, va, vb, vc);
        ++out.trace;
        afterTrace<kVolumes>(s, root, pv, hit, cameraPosition, radiance, alpha);
        if (hit.geom == ~0u) continue;
        if (!shadeVertex<kVolumes, kTextures>(s, root, pixel, index, pv, hit, va, vb, vc, top, radiance, alpha, sink)) {
            out.status = X2_ERROR;
            return;
        }
    }
    out.rgb[0] = radiance.x;
    out.rgb[1] = radiance.y;
    out.rgb[2] = radiance.z;
    out.alpha = alpha;
    out.status = X2_DONE;
}

}  // namespace x2
