// Delta and ratio tracking over coarse majorant grids: a second estimator of the volume integrals the reference's
// decoupled march estimates (x2_config.volume_estimator = 1; the march, volume.cuh, is the reference's and the
// default).
//
// The integrals are the reference's, term for term (async_integrator.h:1152-1291 volumeRadiance with its march
// :616-798, transmittance() :425-476 and the source term :573-591), so that both estimators converge to the same
// image up to the march's quadrature; only how each integral is sampled differs:
//   camera-ray emission   E = int T(t) e(t) dt (each volume's nearest-voxel emission, no extinction factor): ratio
//                         tracking's tentative collisions, a Poisson process of rate mu (the majorant) along the ray,
//                         each adding w e(t) / mu with w the running ratio-tracking weight (E[w(t)] = T(t));
//   transmittance         T to the surface behind: the same walk's final weight, w = prod (1 - sigma_t / mu);
//   single scattering     int T(t) sigma_s(t) Ls(t) dt: delta tracking's real collision (pdf sigma_t T), weighted by
//                         sigma_s / sigma_t, and at it each light's source term with its surface shadow ray and the
//                         volumes' transmittance on the way by ratio tracking (at the nearest voxel, as the reference's
//                         shadow march reads the grid);
//   shadow rays           surfaces' light samples through the volumes: ratio tracking at the nearest voxel.
// The extinction inside a ray's stretch is the march's (the volume's own interpolation); the majorant of a cell is
// the largest density any interpolation can read there (the voxels the cell's box reaches, one more each way), times
// the largest gain channel (api.cu makes the grids at scene load). Free-flight distances are drawn a majorant cell at
// a time along a 3D DDA walk of the 32^3 grid over the volume's bounds, so an empty cell costs a step and no lookup.
// Weights below 0.1 go through Russian roulette, which keeps every estimate unbiased.
//
// Admitted (x2_config_set refuses the rest): grey extinction (the gain's three channels equal), max_volume_depth 1
// (single scattering: the reference's multiple-scattering approximation rides on the march's steps), the sum or max
// overlap modes.
#pragma once
#include "volume.cuh"

namespace x2 {

// The majorant along a ray inside one volume's bounds: the DDA state over its cells.
struct MajorantWalk {
    const float* cells;  // kMajorantCells^3, x fastest
    int ix, iy, iz, sx, sy, sz;
    float tNextX, tNextY, tNextZ, dtX, dtY, dtZ;
    float t, tEnd;  // the walk's position and its end
};

__device__ __forceinline__ bool majorantStart(const VolumeRec& v, V3 org, V3 dir, float t0, float t1, MajorantWalk& w) {
    if (!v.majorant || !(t1 > t0)) return false;
    const float n = float(kMajorantCells);
    const V3 ext{v.hi.x - v.lo.x, v.hi.y - v.lo.y, v.hi.z - v.lo.z};
    const V3 p{org.x + dir.x * t0, org.y + dir.y * t0, org.z + dir.z * t0};
    auto cellOf = [&](float x, float lo, float e) { return min(max(int(floorf((x - lo) / e * n)), 0), kMajorantCells - 1); };
    w.cells = v.majorant;
    w.ix = cellOf(p.x, v.lo.x, ext.x);
    w.iy = cellOf(p.y, v.lo.y, ext.y);
    w.iz = cellOf(p.z, v.lo.z, ext.z);
    auto axis = [&](float d, float o, float lo, float e, int i, int& s, float& tNext, float& dt) {
        const float size = e / n;
        if (d > 0.0f) {
            s = 1;
            tNext = (lo + float(i + 1) * size - o) / d;
            dt = size / d;
        } else if (d < 0.0f) {
            s = -1;
            tNext = (lo + float(i) * size - o) / d;
            dt = -size / d;
        } else {
            s = 0;
            tNext = 3.4e38f;
            dt = 3.4e38f;
        }
    };
    axis(dir.x, org.x, v.lo.x, ext.x, w.ix, w.sx, w.tNextX, w.dtX);
    axis(dir.y, org.y, v.lo.y, ext.y, w.iy, w.sy, w.tNextY, w.dtY);
    axis(dir.z, org.z, v.lo.z, ext.z, w.iz, w.sz, w.tNextZ, w.dtZ);
    w.t = t0;
    w.tEnd = t1;
    return true;
}
// The current cell's majorant and where the ray leaves it (at most the walk's end).
__device__ __forceinline__ float majorantHere(const MajorantWalk& w, float& exitT) {
    exitT = fminf(fminf(w.tNextX, w.tNextY), fminf(w.tNextZ, w.tEnd));
    return __ldg(w.cells + (size_t(w.iz) * kMajorantCells + size_t(w.iy)) * kMajorantCells + size_t(w.ix));
}
// Steps to the next cell; false past the walk's end or the grid.
__device__ __forceinline__ bool majorantNext(MajorantWalk& w) {
    if (w.tNextX <= w.tNextY && w.tNextX <= w.tNextZ) {
        w.t = w.tNextX;
        w.ix += w.sx;
        w.tNextX += w.dtX;
        if (w.ix < 0 || w.ix >= kMajorantCells) return false;
    } else if (w.tNextY <= w.tNextZ) {
        w.t = w.tNextY;
        w.iy += w.sy;
        w.tNextY += w.dtY;
        if (w.iy < 0 || w.iy >= kMajorantCells) return false;
    } else {
        w.t = w.tNextZ;
        w.iz += w.sz;
        w.tNextZ += w.dtZ;
        if (w.iz < 0 || w.iz >= kMajorantCells) return false;
    }
    return w.t < w.tEnd;
}

// One stretch [t0, t1) of a ray inside the volumes of `regions`: the tentative collisions of a Poisson process whose
// rate bounds the combined extinction — one volume: its majorant cells; several: their largest majorants, summed —
// each handed to visit(t, mu), which returns false to stop. Returns false if stopped.
template <class Visit>
__device__ __forceinline__ bool trackStretch(const SceneView& s, uint32_t regions, V3 org, V3 dir, float t0, float t1, Stream& st, Visit& visit) {
    uint32_t only = kMaxVolumes, count = 0;
    float bound = 0.0f;
    for (uint32_t v = 0; v < s.config.volume_count; ++v)
        if (regions >> v & 1) {
            only = v;
            ++count;
            bound += s.volumes[v].majorantMax;
        }
    if (!count) return true;
    if (count == 1) {
        MajorantWalk w;
        if (!majorantStart(s.volumes[only], org, dir, t0, t1, w)) return true;
        for (int cells = 0; cells < 4 * kMajorantCells; ++cells) {
            float exitT;
            const float mu = majorantHere(w, exitT);
            if (mu > 0.0f) {
                for (float t = w.t;;) {
                    t -= mf::log(1.0f - st.next()) / mu;
                    if (!(t < exitT)) break;
                    if (!visit(t, mu, regions)) return false;
                }
            }
            if (exitT >= w.tEnd || !majorantNext(w)) return true;
        }
        return true;
    }
    if (!(bound > 0.0f)) return true;
    for (float t = t0;;) {
        t -= mf::log(1.0f - st.next()) / bound;
        if (!(t < t1)) return true;
        if (!visit(t, bound, regions)) return false;
    }
}

// Walks a ray's volume intervals on [tnear, tfar] (its crossings, in order), each stretch by trackStretch.
template <class Visit>
__device__ __forceinline__ void trackIntervals(const SceneView& s, const Crossing* x, uint32_t n, uint32_t regions, V3 org, V3 dir, float tnear,
                                               float tfar, Stream& st, Visit& visit) {
    float tStart = tnear;
    for (uint32_t i = 0; i < n; ++i) {
        if (x[i].t > tfar) break;
        if (x[i].t - tStart > kVolumeEpsilon) {
            if (regions && !trackStretch(s, regions, org, dir, tStart, x[i].t, st, visit)) return;
            tStart = x[i].t;
        }
        applyCrossing(regions, x[i]);
    }
    if (tfar - tStart > kVolumeEpsilon && regions && tfar < kFarLimit) trackStretch(s, regions, org, dir, tStart, tfar, st, visit);
}

// The ratio-tracking weight's step at a tentative collision, with Russian roulette below 0.1; false once it is zero.
__device__ __forceinline__ bool ratioStep(float& w, float sigmaT, float mu, Stream& st) {
    w *= 1.0f - fminf(sigmaT / mu, 1.0f);
    if (w < 0.1f) {
        if (st.next() >= w) {
            w = 0.0f;
            return false;
        }
        w = 1.0f;
    }
    return true;
}

// Ratio tracking: an unbiased estimate of the (grey) transmittance of [tnear, tfar] at the nearest voxel.
static __device__ __noinline__ float trackedTransmittance(const SceneView& s, Stream& st, V3 org, V3 dir, float tnear, float tfar) {
    Crossing x[kMaxCrossings];
    uint32_t regions;
    const uint32_t n = volumeIntervals(s, org, dir, tnear, x, regions);
    if (n == 0 && regions == 0) return 1.0f;
    float w = 1.0f;
    auto visit = [&](float t, float mu, uint32_t here) {
        const V3 p = add(org, mul(dir, t));
        return ratioStep(w, evalShadersAt(s, here, s.config.volume_overlap_mode, 0.0f, p, kInterpPoint, nullptr, nullptr).sigmaT.x, mu, st);
    };
    trackIntervals(s, x, n, regions, org, dir, tnear, tfar, st, visit);
    return w;
}

// A light's source term at a scattering point (estimateInScatteringSourceTermDirect with the tracked transmittance).
static __device__ __noinline__ V3 trackedSourceTerm(const SceneView& s, Stream& st, const x2_light& L, V3 P, V3 rayDir, float g, const float ul[3]) {
    V3 wi;
    LightHit lh;
    float r[3] = {ul[0], ul[1], ul[2]};
    if (!lightSample(L, P, nullptr, r, wi, lh)) return V3{0, 0, 0};
    float pdfL;
    const V3 Li = lightEval(L, wi, lh, pdfL);
    if (pdfL == 0.0f || isExactlyZero(Li) || !vfinite(pdfL)) return V3{0, 0, 0};
    const float near = fmaxf(kHitEpsilonStart, 0.0f), far = fmaxf(kHitEpsilonEnd * lh.distance, near);
    if (!visible(s, P, wi, near, far)) return V3{0, 0, 0};
    const float tr = trackedTransmittance(s, st, P, wi, 0.0f, far);
    if (tr <= 0.0f) return V3{0, 0, 0};
    return vscaled(Li, tr * phaseEval(g, V3{-rayDir.x, -rayDir.y, -rayDir.z}, wi) / pdfL);
}

// volumeRadiance by tracking: the camera ray's emission, the single scattering of every light (a volume depth on) and
// the path's throughput through the volumes, as volume.cuh's volumeRadiance returns them. pv's T and volume depth are
// updated.
static __device__ __noinline__ V3 volumeRadianceTracked(const SceneView& s, const Identity& root, Pending& pv, V3 org, V3 dir, float tnear, float tfar,
                                                        V3& alphaTransmittance) {
    const x2_config& c = s.config;
    V3 radiance{0, 0, 0};
    alphaTransmittance = V3{1, 1, 1};
    Crossing x[kMaxCrossings];
    uint32_t regions;
    const uint32_t n = volumeIntervals(s, org, dir, tnear, x, regions);
    if (n == 0 && regions == 0) return radiance;
    const U64 volumeBranch = childBranch(pv.branch, 0xfffa, pv.volumeDepth);
    Identity vid = root;
    vid.branch = childBranch(volumeBranch, 0, 0);
    Stream st(vid, pv.depth, 0);
    const V3 T = pv.T;
    // Ratio tracking along the ray: its transmittance and (a camera ray) its emission.
    const bool sampleEmission = pv.depth == 0;
    float w = 1.0f;
    V3 emitted{0, 0, 0};
    auto along = [&](float t, float mu, uint32_t here) {
        V3 e[kMaxVolumes];
        uint32_t chosen = kMaxVolumes;
        const V3 p = add(org, mul(dir, t));
        const VolumeCoefficients k = evalShadersAt(s, here, c.volume_overlap_mode, 0.0f, p, kNoGrid, sampleEmission ? e : nullptr, &chosen);
        if (sampleEmission) {
            V3 sum{0, 0, 0};
            if (c.volume_overlap_mode == kOverlapSum) {
                for (uint32_t v = 0; v < c.volume_count; ++v)
                    if (here >> v & 1) sum = vplus(sum, e[v]);
            } else if (chosen < kMaxVolumes) {
                sum = e[0];
            }
            emitted = vplus(emitted, vscaled(sum, w / mu));
        }
        return ratioStep(w, k.sigmaT.x, mu, st);
    };
    trackIntervals(s, x, n, regions, org, dir, tnear, tfar, st, along);
    if (sampleEmission) radiance = vplus(radiance, vtimes(T, emitted));
    alphaTransmittance = V3{w, w, w};
    if (pv.volumeDepth < c.max_volume_depth) {
        // Single scattering: delta tracking's collision (none: the ray passed), then every light's source term there.
        const bool highQuality = pv.nonMirror == 0;
        const uint32_t samplesPerLight = highQuality ? c.light_samples : 1, scatterCount = highQuality ? c.volume_illumination_samples : 1;
        const float invN = 1.0f / float(samplesPerLight * (scatterCount ? scatterCount : 1));
        for (uint32_t ts = 0; ts < scatterCount; ++ts) {
            Identity did = root;
            did.branch = childBranch(volumeBranch, 0xfff0, ts);
            Stream ds(did, pv.depth, 0);
            float hitT = -1.0f, sigmaT = 0.0f, g = 0.0f;
            V3 sigmaS{0, 0, 0};
            auto collide = [&](float t, float mu, uint32_t here) {
                const VolumeCoefficients k = evalShadersAt(s, here, c.volume_overlap_mode, 0.0f, add(org, mul(dir, t)), kNoGrid, nullptr, nullptr);
                if (ds.next() * mu < k.sigmaT.x) {
                    hitT = t;
                    sigmaS = k.sigmaS;
                    sigmaT = k.sigmaT.x;
                    g = k.g;
                    return false;
                }
                return true;
            };
            trackIntervals(s, x, n, regions, org, dir, tnear, tfar, ds, collide);
            if (hitT < 0.0f || !(sigmaT > 0.0f)) continue;
            const V3 P = add(org, mul(dir, hitT));
            const V3 albedo = vscaled(sigmaS, 1.0f / sigmaT);
            for (uint32_t li = 0; li < c.light_count; ++li)
                for (uint32_t ls = 0; ls < samplesPerLight; ++ls) {
                    Identity sid = root;
                    sid.branch = childBranch(volumeBranch, 1 + li, ls * scatterCount + ts);
                    Stream ss(sid, pv.depth, 0);
                    const float ul[3] = {ss.next(), ss.next(), ss.next()};
                    const V3 Ls = trackedSourceTerm(s, ss, s.lights[li], P, dir, g, ul);
                    radiance = vplus(radiance, vscaled(vtimes(vtimes(T, albedo), Ls), invN));
                }
        }
        ++pv.volumeDepth;
    }
    pv.T = vscaled(pv.T, w);
    return radiance;
}

}  // namespace x2
