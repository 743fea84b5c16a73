// Participating media along a path's rays: the reference's volume integration (async_integrator.h:414-591 and
// :616-1291, volume_core.h, volume_grid.h) for VdbVolumes over dense grids, restated for the device with the same
// arithmetic in the same order, so a sample's radiance agrees with the reference's CPU lane.
//
//   crossings     a ray's entries and exits of the volumes' bounds (closed box meshes), found one at a time from
//                 tnear as the reference's backends do (async_cpu.h:1089-1149), then interiority's outermost pairs;
//   march         decoupled ray marching (VolumeMarch::run): each heterogeneous stretch in steps of its least feature
//                 size over the volume quality, the first at a random place in the first step; a step's coefficients
//                 at its end; the transmittance and (camera rays) each volume's emission accumulated; the march stops
//                 below the transmittance threshold;
//   lookups       the light sampling's step lookups re-run the march (ReplaySteps) from the first march's checkpoints
//                 (MarchRecord: every stride steps, the stride doubling as the eight slots fill), the same steps bit
//                 for bit: distance sampling over the steps' weights (pick) and the step at a distance (at);
//   scattering    integrateVolumeScatteringDirect: per light, equi-angular (bounded lights) and distance samples with
//                 MIS, each through the light's source term (a light sample, its surface shadow ray, the volumes'
//                 transmittance on the way by ray marching at the nearest voxel, the Henyey-Greenstein phase);
//   shadows       transmittance(): the volumes' optical thickness along a surface's shadow ray;
//   multiple      (max_volume_depth > 1) the multiple-scattering approximation: scatter events picked from the
//                 march's steps, then free paths from each, each order's extinction, contribution and anisotropy
//                 shrunk by its factor, every light's source term at each event.
//
// Not built: homogeneous BaseVolumes and mapped ones (their ramps and map programs), holdouts (cutouts), motion and
// velocity, emissive regions as light sources, light sets and LPEs; x2_scene_load and x2_config_set refuse scenes and
// configs that would need them.
#pragma once
#include "shading.cuh"

namespace x2 {

constexpr uint32_t kMaxVolumes = 32, kMaxCrossings = 32, kMarchLimit = 1u << 14, kNoGrid = 0xffffffffu;
constexpr uint32_t kDeviceVolumes = 8;  // volumes a scene may hold here (a march keeps an emission sum for each)
constexpr float kVolumeEpsilon = 1.1920928955078125e-07f, kHitEpsilonStart = 1e-5f, kFarLimit = 0.999f * kDistantDistance;
constexpr float kOneOverFourPi = 0.07957747154594766788f;
enum : uint32_t { kOverlapSum = 0, kOverlapMax = 1, kOverlapRnd = 2 };
enum : uint32_t { kEntry = 1, kExit = 2 };
enum : uint32_t { kInterpPoint = 0, kInterpBox = 1, kInterpQuadratic = 2 };

struct Crossing {
    float t;
    uint32_t volume, flags;
};

// ---- component helpers (volume_core.h:197-206) ----
__device__ __forceinline__ V3 vtimes(V3 a, V3 b) { return V3{a.x * b.x, a.y * b.y, a.z * b.z}; }
__device__ __forceinline__ V3 vscaled(V3 a, float s) { return V3{a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ V3 vplus(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3 cmax0(V3 a) { return V3{fmaxf(a.x, 0.0f), fmaxf(a.y, 0.0f), fmaxf(a.z, 0.0f)}; }
__device__ __forceinline__ V3 expNeg(V3 a, float s) { return V3{mf::exp(-a.x * s), mf::exp(-a.y * s), mf::exp(-a.z * s)}; }
__device__ __forceinline__ float vlum(V3 a) { return 0.299f * a.x + 0.587f * a.y + 0.114f * a.z; }
__device__ __forceinline__ bool vblack(V3 a) { return a.x == 0.0f && a.y == 0.0f && a.z == 0.0f; }
__device__ __forceinline__ bool vIsZero(float x) { return fabsf(x) < kVolumeEpsilon; }
__device__ __forceinline__ bool vfinite(float x) { return x - x == 0.0f; }

// ---- dense grids (volume_grid.h:42-134): OpenVDB's world-to-index in doubles, point / box / quadratic sampling ----
__device__ __forceinline__ void gridIndex(const GridRec& g, V3 p, double out[3]) {
    const double* m = g.worldToIndex;
    for (int c = 0; c < 3; ++c) out[c] = double(p.x) * m[0 * 4 + c] + double(p.y) * m[1 * 4 + c] + double(p.z) * m[2 * 4 + c] + m[3 * 4 + c];
}
__device__ __forceinline__ float voxel(const GridRec& g, int i, int j, int k, int c) {
    const int x = i - g.lo[0], y = j - g.lo[1], z = k - g.lo[2];
    if (x < 0 || y < 0 || z < 0 || x >= g.dims[0] || y >= g.dims[1] || z >= g.dims[2]) return 0.0f;
    return __ldg(g.values + g.channels * ((size_t(z) * size_t(g.dims[1]) + size_t(y)) * size_t(g.dims[0]) + size_t(x)) + c);
}
__device__ __forceinline__ float boxLerp(float a, float b, double w) { return a + float(double(b - a) * w); }
__device__ __forceinline__ float quadratic(const float* v, double w) {
    const float a = float(0.5 * double(v[0] + v[2]) - double(v[1])), b = float(0.5 * double(v[2] - v[0])), c = v[1];
    return float(w * (w * double(a) + double(b)) + double(c));
}
// One channel of the grid at p (its world space) by the interpolation mode.
static __device__ __noinline__ float sampleGrid(const GridRec& g, V3 p, uint32_t mode, int c) {
    double ip[3];
    gridIndex(g, p, ip);
    if (mode == kInterpPoint) return voxel(g, int(round(ip[0])), int(round(ip[1])), int(round(ip[2])), c);
    const int i0 = int(floor(ip[0])), j0 = int(floor(ip[1])), k0 = int(floor(ip[2]));
    const double u = ip[0] - i0, v = ip[1] - j0, w = ip[2] - k0;
    if (mode == kInterpBox) {
        float d[2][2][2];
        for (int i = 0; i < 2; ++i)
            for (int j = 0; j < 2; ++j)
                for (int k = 0; k < 2; ++k) d[i][j][k] = voxel(g, i0 + i, j0 + j, k0 + k, c);
        return boxLerp(boxLerp(boxLerp(d[0][0][0], d[0][0][1], w), boxLerp(d[0][1][0], d[0][1][1], w), v),
                       boxLerp(boxLerp(d[1][0][0], d[1][0][1], w), boxLerp(d[1][1][0], d[1][1][1], w), v), u);
    }
    float vx[3];
    for (int i = 0; i < 3; ++i) {
        float vy[3];
        for (int j = 0; j < 3; ++j) {
            const float vz[3] = {voxel(g, i0 - 1 + i, j0 - 1 + j, k0 - 1, c), voxel(g, i0 - 1 + i, j0 - 1 + j, k0, c),
                                 voxel(g, i0 - 1 + i, j0 - 1 + j, k0 + 1, c)};
            vy[j] = quadratic(vz, w);
        }
        vx[i] = quadratic(vy, v);
    }
    return quadratic(vx, u);
}

// ---- a volume's coefficients at a point (localAt, volume_core.h:241-273, for a VdbVolume with no maps) ----
struct VolumeLocal {
    V3 sigmaT, albedo, emission;
    float g;
};
__device__ __forceinline__ V3 affine34(const float* m, V3 p) {
    return V3{m[0] * p.x + m[1] * p.y + m[2] * p.z + m[3], m[4] * p.x + m[5] * p.y + m[6] * p.z + m[7], m[8] * p.x + m[9] * p.y + m[10] * p.z + m[11]};
}
__device__ __forceinline__ VolumeLocal localAt(const SceneView& s, const VolumeRec& v, V3 p, uint32_t interpolation) {
    const V3 gp = affine34(v.worldToGrid, p);
    const float density = v.densityGrid < s.gridCount && s.grids[v.densityGrid].channels == 1 ? sampleGrid(s.grids[v.densityGrid], gp, interpolation, 0) : 0.0f;
    V3 temperature{0, 0, 0};
    if (v.emissionGrid != kNoGrid && v.emissionGrid < s.gridCount && s.grids[v.emissionGrid].channels == 3) {
        const GridRec& e = s.grids[v.emissionGrid];
        temperature = V3{sampleGrid(e, gp, kInterpPoint, 0), sampleGrid(e, gp, kInterpPoint, 1), sampleGrid(e, gp, kInterpPoint, 2)};
    }
    return VolumeLocal{cmax0(vscaled(v.gain, density)), cmax0(v.colorMult), cmax0(vtimes(temperature, v.incandescence)),
                       fminf(fmaxf(v.g, -1.0f), 1.0f)};
}

// evalShadersAt (volume_core.h:284-378) without holdouts: the regions' volumes combined by the overlap mode.
struct VolumeCoefficients {
    V3 sigmaT, sigmaS;
    float g;
    float surfaceThreshold;
};
static __device__ __noinline__ VolumeCoefficients evalShadersAt(const SceneView& s, uint32_t regions, uint32_t mode, float rnd, V3 p,
                                                         uint32_t interpolationOverride, V3* emissions, uint32_t* chosenVolume) {
    VolumeCoefficients c{{0, 0, 0}, {0, 0, 0}, 0.0f, 1.0f};
    V3 anisotropy{0, 0, 0}, sigmaTSum{0, 0, 0};
    float maxSigmaTLum = -3.402823466e+38f;
    uint32_t first = kMaxVolumes, chosen = kMaxVolumes;
    auto local = [&](uint32_t v) {
        const VolumeRec& vr = s.volumes[v];
        return localAt(s, vr, p, interpolationOverride != kNoGrid ? interpolationOverride : vr.interpolation);
    };
    for (uint32_t v = 0; v < s.config.volume_count; ++v) {
        if (!(regions >> v & 1)) continue;
        const VolumeLocal L = local(v);
        const V3 scatter = vtimes(L.albedo, L.sigmaT);
        if (first == kMaxVolumes) first = v;
        const float l = vlum(L.sigmaT);
        if (mode == kOverlapSum) {
            c.sigmaT = vplus(c.sigmaT, L.sigmaT);
            c.sigmaS = vplus(c.sigmaS, scatter);
            anisotropy = vplus(anisotropy, vscaled(scatter, L.g));
            if (emissions) emissions[v] = L.emission;
            if (l > maxSigmaTLum) {
                maxSigmaTLum = l;
                chosen = v;
            }
        } else if (mode == kOverlapMax) {
            if (l > maxSigmaTLum) {
                maxSigmaTLum = l;
                c.sigmaT = L.sigmaT;
                c.sigmaS = scatter;
                anisotropy = vscaled(scatter, L.g);
                chosen = v;
                if (emissions) emissions[0] = L.emission;
            }
        } else {
            sigmaTSum = vplus(sigmaTSum, L.sigmaT);
        }
    }
    if (mode == kOverlapRnd && first != kMaxVolumes) {
        // The volume rnd picks by its share of the luminance of the summed extinction (each volume's coefficients are
        // evaluated again here: the same values as in the first pass).
        const float total = vlum(sigmaTSum);
        uint32_t pick = first;
        float weight = 1.0f;
        if (total != 0.0f) {
            V3 running{0, 0, 0};
            pick = kMaxVolumes;
            uint32_t last = first;
            for (uint32_t v = 0; v < s.config.volume_count; ++v) {
                if (!(regions >> v & 1)) continue;
                running = vplus(running, local(v).sigmaT);
                last = v;
                if (rnd < vlum(running) / total) {
                    pick = v;
                    break;
                }
            }
            if (pick == kMaxVolumes) pick = last;
            weight = total / vlum(local(pick).sigmaT);
        }
        const VolumeLocal L = local(pick);
        const V3 scatter = vtimes(L.albedo, L.sigmaT);
        c.sigmaT = vscaled(L.sigmaT, weight);
        c.sigmaS = vscaled(scatter, weight);
        anisotropy = vscaled(vscaled(scatter, L.g), weight);
        chosen = pick;
        if (emissions) emissions[0] = vscaled(L.emission, weight);
    }
    if (chosenVolume) *chosenVolume = chosen;
    if (chosen < kMaxVolumes) c.surfaceThreshold = s.volumes[chosen].surfaceThreshold;
    c.g = vlum(anisotropy);
    const float normalization = vlum(c.sigmaS);
    if (normalization > 0.0f) c.g /= normalization;
    return c;
}

__device__ __forceinline__ float minFeatureSize(const SceneView& s, uint32_t regions) {
    float m = 3.402823466e+38f;
    for (uint32_t v = 0; v < s.config.volume_count; ++v)
        if (regions >> v & 1) m = fminf(m, s.volumes[v].featureSize);
    return m;
}

// ---- crossings (async_cpu.h:1089-1149, with the box meshes' triangles tested one by one) and interiority ----
static __device__ __noinline__ uint32_t volumeCrossings(const SceneView& s, V3 o, V3 d, float tnear, Crossing* x) {
    const RayQ r = makeRay(s.bvh, o.x, o.y, o.z, d.x, d.y, d.z);
    const uint32_t tris = 12u * s.config.volume_count;
    uint32_t n = 0;
    float t = tnear;
    for (uint32_t k = 0; k < 4 * kMaxCrossings && n < kMaxCrossings; ++k) {
        float best = __int_as_float(0x7f800000);
        uint32_t hitTri = ~0u;
        for (uint32_t i = 0; i < tris; ++i) {
            const float* v = s.volumeTris + 9 * i;
            const float4 a = make_float4(v[0], v[1], v[2], 0.0f), b = make_float4(v[3], v[4], v[5], 0.0f), c = make_float4(v[6], v[7], v[8], 0.0f);
            float th;
            if (triTest(r, a, b, c, t, __int_as_float(0x7f800000), th) && th < best) {
                best = th;
                hitTri = i;
            }
        }
        if (hitTri == ~0u) break;
        const float* v = s.volumeTris + 9 * hitTri;
        const V3 e1{v[3] - v[0], v[4] - v[1], v[5] - v[2]}, e2{v[6] - v[0], v[7] - v[1], v[8] - v[2]};
        const V3 ng{e1.y * e2.z - e1.z * e2.y, e1.z * e2.x - e1.x * e2.z, e1.x * e2.y - e1.y * e2.x};
        const uint32_t vol = hitTri / 12u;
        const uint32_t flags = d.x * ng.x + d.y * ng.y + d.z * ng.z < 0.0f ? kEntry : kExit;
        if (!(n > 0 && x[n - 1].t == best && x[n - 1].volume == vol && x[n - 1].flags == flags)) x[n++] = Crossing{best, vol, flags};
        t = best + fmaxf(1e-6f, best * 1e-6f);
    }
    return n;
}
// collectVolumeIntervals' interiority (volume_core.h:471-502): only each volume's outermost entry and exit stay; the
// regions the ray starts in are returned.
__device__ __forceinline__ uint32_t interiority(Crossing* x, uint32_t& n) {
    int count[kDeviceVolumes];
    for (uint32_t v = 0; v < kDeviceVolumes; ++v) count[v] = 0;
    uint32_t regions = 0;
    bool redundant = false;
    for (int i = int(n) - 1; i >= 0; --i) {
        const uint32_t v = x[i].volume;
        if (x[i].flags & kEntry) {
            --count[v];
            if (count[v] == 0) regions &= ~(1u << v);
            else if (count[v] > 0) {
                x[i].flags &= ~kEntry;
                redundant = true;
            }
        }
        if (x[i].flags & kExit) {
            if (count[v] == 0) regions |= 1u << v;
            else if (count[v] > 0) {
                x[i].flags &= ~kExit;
                redundant = true;
            }
            ++count[v];
        }
    }
    if (redundant) {
        uint32_t m = 0;
        for (uint32_t i = 0; i < n; ++i)
            if (x[i].flags) x[m++] = x[i];
        n = m;
    }
    return regions;
}
__device__ __forceinline__ void applyCrossing(uint32_t& regions, const Crossing& x) {
    if (x.flags & kEntry) regions |= 1u << x.volume;
    if (x.flags & kExit) regions &= ~(1u << x.volume);
}
__device__ __forceinline__ uint32_t volumeIntervals(const SceneView& s, V3 o, V3 d, float tnear, Crossing* x, uint32_t& regions) {
    uint32_t n = volumeCrossings(s, o, d, tnear, x);
    regions = interiority(x, n);
    return n;
}

// ---- phase function and distance sampling (volume_core.h:505-530) ----
__device__ __forceinline__ float phaseEval(float g, V3 wo, V3 wi) {
    if (fabsf(g) <= 1e-3f) return kOneOverFourPi;
    const float cosTheta = dot(wo, wi), denom = 1 + g * g + 2 * g * cosTheta;
    return vIsZero(denom) ? 0.0f : kOneOverFourPi * (1 - g * g) / (denom * sqrtf(denom));
}
__device__ __forceinline__ float sampleDistanceExponential(float u, float sigma, float a, float b) {
    return a - mf::log(1.0f - u * (1.0f - mf::exp(sigma * (a - b)))) / sigma;
}
__device__ __forceinline__ float pdfDistanceExponential(float t, float sigma, float a, float b) {
    return sigma / (mf::exp((t - a) * sigma) - mf::exp((t - b) * sigma));
}
__device__ __forceinline__ float sampleEquiAngular(float u, float D, float thetaA, float thetaB) { return D * mf::tan((1 - u) * thetaA + u * thetaB); }
__device__ __forceinline__ float pdfEquiAngular(float t, float D, float thetaA, float thetaB) { return D / ((thetaB - thetaA) * (D * D + t * t)); }

// A light's equi-angular pivot (volume_core.h:630-662) for the admitted lights: a point on a rect.
__device__ __forceinline__ bool boundedLight(const x2_light& l) { return l.type != X2_LIGHT_ENV && l.type != X2_LIGHT_DISTANT; }
__device__ __forceinline__ V3 lightPivot(const x2_light& l, const float r[3]) {
    const V3 local{(0.5f - r[0]) * 2.0f * l.half_width, (0.5f - r[1]) * 2.0f * l.half_height, 0.0f};
    return add(V3{l.position[0], l.position[1], l.position[2]}, rowsMul(l.local2render, local));
}

// ---- the march (async_integrator.h:616-798) ----
struct VolumeStep {  // volume::Step without holdouts
    V3 sigmaT, sigmaS, tr;
    float g, tStart, delta;
};
__device__ __forceinline__ float stepWeight(const VolumeStep& s) { return vlum(vtimes(vscaled(s.sigmaS, s.delta), s.tr)) + 0.0f; }

struct MarchCheckpoint {
    Stream marching;
    V3 vt;
    float t, stepStart, stepSize, partial;
    uint32_t interval, regions, count, visited;
};
struct MarchRecord {
    static constexpr uint32_t kSlots = 8;
    MarchCheckpoint at[kSlots];
    uint32_t used = 0, stride = 8, last = 0;
    __device__ bool wants(uint32_t count) const {
        if (count == 0 || count == last || count % stride) return false;
        return used < kSlots || count % (2 * stride) == 0;
    }
    __device__ MarchCheckpoint& slot(uint32_t count) {
        if (used == kSlots) {
            for (uint32_t i = 0; i < kSlots / 2; ++i) at[i] = at[2 * i + 1];
            used = kSlots / 2;
            stride *= 2;
        }
        last = count;
        return at[used++];
    }
};

struct VolumeMarch {
    const SceneView& s;
    const Crossing* x;
    uint32_t n, regionsAtStart;
    V3 org, dir;
    float tnear, tfar;
    uint32_t depth;
    bool sampleEmission;
    Stream start;
    uint32_t limit;
    // What a march leaves.
    V3 vt;
    V3 emitted[kDeviceVolumes];
    uint32_t visited, count;
    bool reachedThreshold, stopped;
    MarchRecord* record;
    const float* weightsSoFar;

    template <class Emit>
    __device__ void stepping(Emit& emit, Stream& marching, uint32_t regions, float t1, float t, float stepStart, float stepSize, uint32_t interval) {
        const x2_config& c = s.config;
        auto step = [&](float at) {
            const float rnd = c.volume_overlap_mode == kOverlapRnd ? marching.next() : 0.0f;
            V3 emissions[kDeviceVolumes];
            uint32_t chosen = kMaxVolumes;
            const VolumeCoefficients k =
                evalShadersAt(s, regions, c.volume_overlap_mode, rnd, add(org, mul(dir, at)), kNoGrid, sampleEmission ? emissions : nullptr, &chosen);
            const float delta = at - stepStart;
            if (!emit(VolumeStep{k.sigmaT, k.sigmaS, vt, k.g, stepStart, delta}, count)) stopped = true;
            ++count;
            const V3 te = vt;
            if (sampleEmission) {
                if (c.volume_overlap_mode == kOverlapSum) {
                    for (uint32_t v = 0; v < c.volume_count; ++v)
                        if (regions >> v & 1) emitted[v] = vplus(emitted[v], vscaled(vtimes(te, emissions[v]), delta));
                } else if (chosen < kMaxVolumes) {
                    emitted[chosen] = vplus(emitted[chosen], vscaled(vtimes(te, emissions[0]), delta));
                }
            }
            vt = vtimes(vt, expNeg(k.sigmaT, delta));
        };
        while (t < t1) {
            if (record && weightsSoFar && record->wants(count))
                record->slot(count) = MarchCheckpoint{marching, vt, t, stepStart, stepSize, *weightsSoFar, interval, regions, count, visited};
            if (vlum(vt) < c.volume_transmittance_threshold) {
                reachedThreshold = true;
                return;
            }
            step(t);
            if (stopped) return;
            stepStart = t;
            t += stepSize;
            if (count + 1 >= limit) return;
        }
        if (vlum(vt) < c.volume_transmittance_threshold) {
            reachedThreshold = true;
            return;
        }
        if (t - t1 > kVolumeEpsilon) step(t1);
    }

    template <class Emit>
    __device__ void marchStretch(Emit& emit, Stream& marching, uint32_t regions, float t0, float t1, uint32_t interval) {
        if (!regions || t1 >= kFarLimit || count + 1 >= limit || reachedThreshold || stopped) return;
        visited |= regions;
        // Every admitted volume is heterogeneous: steps of the least feature size over the volume quality (wider
        // deeper in the path), the first at a random place in the first step.
        const float u = marching.next();
        const float stepSize = minFeatureSize(s, regions) * s.config.inv_volume_quality * fmaxf(float(int(depth) - 1), 1.0f);
        stepping(emit, marching, regions, t1, t0 + stepSize * u, t0, stepSize, interval);
    }

    // The march from its start, or from a checkpoint (the same steps from there, bit for bit).
    template <class Emit>
    __device__ void run(Emit& emit, const MarchCheckpoint* from = nullptr) {
        Stream marching = from ? from->marching : start;
        uint32_t regions = from ? from->regions : regionsAtStart;
        if (from) {
            vt = from->vt;
            visited = from->visited;
            count = from->count;
        } else {
            vt = V3{1, 1, 1};
            visited = count = 0;
        }
        for (uint32_t v = 0; v < kDeviceVolumes; ++v) emitted[v] = V3{0, 0, 0};
        reachedThreshold = stopped = false;
        float tStart = tnear;
        uint32_t first = 0;
        if (from) {
            const uint32_t k = from->interval;
            stepping(emit, marching, regions, k < n ? x[k].t : tfar, from->t, from->stepStart, from->stepSize, k);
            if (k >= n) return;
            tStart = x[k].t;
            applyCrossing(regions, x[k]);
            first = k + 1;
        }
        for (uint32_t i = first; i < n; ++i) {
            if (x[i].t > tfar || reachedThreshold || stopped) break;
            if (x[i].t - tStart > kVolumeEpsilon) {
                marchStretch(emit, marching, regions, tStart, x[i].t, i);
                tStart = x[i].t;
            }
            applyCrossing(regions, x[i]);
        }
        if (tfar - tStart > kVolumeEpsilon && !reachedThreshold && !stopped) marchStretch(emit, marching, regions, tStart, tfar, n);
    }
};

// The steps as the light sampling asks for them, by marching again (ReplaySteps, async_integrator.h:830-898).
struct ReplaySteps {
    VolumeMarch& m;
    uint32_t count;
    float total;
    bool weightless;
    const MarchRecord* record;
    __device__ float cdfBefore(const MarchCheckpoint& c) const { return weightless ? float(c.count) / float(count) : c.partial; }
    __device__ float cdf(float& partial, const VolumeStep& s, uint32_t index) const {
        if (index + 1 >= count) return total;
        if (weightless) return float(index + 1) / float(count);
        partial += stepWeight(s);
        if (partial > total) partial = total;
        return partial;
    }
    __device__ __noinline__ VolumeStep pick(float r, float& pdf, float& remapped) const {
        const float rw = r * total;
        const MarchCheckpoint* from = nullptr;
        if (record)
            for (uint32_t j = record->used; j-- > 0;)
                if (record->at[j].count < count && cdfBefore(record->at[j]) < rw) {
                    from = &record->at[j];
                    break;
                }
        float partial = from ? from->partial : 0.0f, prev = from ? cdfBefore(*from) : 0.0f, found = total, before = 0.0f;
        VolumeStep chosen{};
        auto emit = [&](const VolumeStep& s, uint32_t i) {
            const float here = cdf(partial, s, i);
            chosen = s;
            if (here >= rw || i + 1 >= count) {
                found = here, before = prev;
                return false;
            }
            prev = here;
            return true;
        };
        m.run(emit, from);
        const float value = found - before;
        pdf = value / total;
        remapped = (rw - before) / value;
        return chosen;
    }
    __device__ __noinline__ VolumeStep at(float t, float& pdf) const {
        const MarchCheckpoint* from = nullptr;
        if (record)
            for (uint32_t j = record->used; j-- > 0;)
                if (record->at[j].count < count && record->at[j].stepStart <= t) {
                    from = &record->at[j];
                    break;
                }
        float partial = from ? from->partial : 0.0f, here = from ? cdfBefore(*from) : 0.0f, kept = 0.0f, keptPrev = 0.0f;
        VolumeStep chosen{};
        auto emit = [&](const VolumeStep& s, uint32_t i) {
            if (i > 0 && s.tStart > t) return false;
            const float before = here;
            here = cdf(partial, s, i);
            chosen = s, kept = here, keptPrev = i > 0 ? before : 0.0f;
            return i + 1 < count;
        };
        m.run(emit, from);
        pdf = (kept - keptPrev) / total;
        return chosen;
    }
};

// ---- shadow rays through the volumes (transmittance(), async_integrator.h:425-476) ----
static __device__ __noinline__ V3 volumeTransmittance(const SceneView& s, Stream& st, V3 org, V3 dir, float tnear, float tfar, float scale, int depth) {
    const x2_config& c = s.config;
    Crossing x[kMaxCrossings];
    uint32_t regions;
    const uint32_t n = volumeIntervals(s, org, dir, tnear, x, regions);
    V3 tr{1, 1, 1};
    if (n == 0 && regions == 0) return tr;
    float tStart = tnear;
    auto segment = [&](float t0, float t1) -> bool {
        if (!regions) return true;
        if (t1 >= kFarLimit) return false;
        const float fs = minFeatureSize(s, regions);
        const float tauThreshold = c.volume_transmittance_threshold == 0.0f ? 3.402823466e+38f : -mf::log(c.volume_transmittance_threshold / vlum(tr));
        const float u = st.next();
        const float stepSize = fs * c.inv_volume_shadow_quality * fmaxf(float(depth - 1), 1.0f);
        float t = t0 + stepSize * u;
        V3 tau{0, 0, 0};
        while (t < t1) {
            const float rnd = c.volume_overlap_mode == kOverlapRnd ? st.next() : 0.0f;
            tau = vplus(tau, evalShadersAt(s, regions, c.volume_overlap_mode, rnd, add(org, mul(dir, t)), kInterpPoint, nullptr, nullptr).sigmaT);
            if (vlum(vscaled(tau, stepSize * scale)) > tauThreshold) return false;
            t += stepSize;
        }
        tr = vtimes(tr, expNeg(tau, stepSize * scale));
        return vlum(tr) > c.volume_transmittance_threshold;
    };
    for (uint32_t i = 0; i < n; ++i) {
        if (x[i].t > tfar) break;
        if (x[i].t - tStart > kVolumeEpsilon) {
            if (!segment(tStart, x[i].t)) return V3{0, 0, 0};
            tStart = x[i].t;
        }
        applyCrossing(regions, x[i]);
    }
    if (tfar - tStart > kVolumeEpsilon && !segment(tStart, tfar)) return V3{0, 0, 0};
    return tr;
}

// estimateInScatteringSourceTermDirect (async_integrator.h:573-591): a light sample from a point in a volume, its
// surface shadow ray, the volumes' transmittance on its way, the phase function.
static __device__ __noinline__ V3 volumeSourceTerm(const SceneView& s, Stream& st, const x2_light& L, V3 P, V3 rayDir, float g, const float ul[3], float scale) {
    V3 wi;
    LightHit lh;
    float r[3] = {ul[0], ul[1], ul[2]};
    if (!lightSample(L, P, nullptr, r, wi, lh)) return V3{0, 0, 0};
    float pdfL;
    const V3 Li = lightEval(L, wi, lh, pdfL);
    if (pdfL == 0.0f || isExactlyZero(Li) || !vfinite(pdfL)) return V3{0, 0, 0};
    float near = kHitEpsilonStart, far = kHitEpsilonEnd * lh.distance;
    near = fmaxf(near, 0.0f);
    far = fmaxf(far - 0.0f, near);
    const float keep = visible(s, P, wi, near, far) ? 1.0f : 0.0f;
    if (keep <= 0.0f) return V3{0, 0, 0};
    const V3 tr = volumeTransmittance(s, st, P, wi, 0.0f, far, scale, 1);
    const float ph = phaseEval(g, V3{-rayDir.x, -rayDir.y, -rayDir.z}, wi);
    return vscaled(vtimes(tr, Li), ph / pdfL * keep);
}

// Henyey-Greenstein sampling about the reversed outgoing direction (volume_core.h phaseSample): uniform over the
// sphere when |g| is at most 1e-3.
__device__ __forceinline__ V3 phaseSample(float g, V3 wo, float u1, float u2) {
    if (fabsf(g) <= 1e-3f) {
        const float cosTheta = 1.0f - 2.0f * u1, sinTheta = sqrtf(fmaxf(0.0f, 1.0f - cosTheta * cosTheta));
        return localSpherical(cosTheta, sinTheta, u2 * kTwoPi);
    }
    u1 = fmaxf(u1, kVolumeEpsilon);
    const float sqrTerm = (1.0f - g * g) / (1.0f - g + 2.0f * g * u1);
    const float cosTheta = (1.0f + g * g - sqrTerm * sqrTerm) / (2.0f * g);
    const float sinTheta = sqrtf(fmaxf(0.0f, 1.0f - cosTheta * cosTheta));
    return localToGlobal(frameN(V3{-wo.x, -wo.y, -wo.z}), localSpherical(cosTheta, sinTheta, kTwoPi * u2));
}

// approximateVolumeMultipleScattering (async_integrator.h:1058-1150, after Wrenninge 2015), pv's volume depth already
// one on: for each of the volume illumination samples, a scatter event picked from the march's steps and a distance
// in it, then free paths from it through the volumes, order after order up to max_volume_depth while the throughput
// stays above the transmittance threshold; at each event every light's source term with the order's attenuation,
// added with the order's contribution factor, and the next direction from the phase function with the order's
// anisotropy. The draws come from one stream a sample, in the reference's order.
static __device__ __noinline__ void volumeMultipleScatter(const SceneView& s, const Identity& root, const Pending& pv, U64 volumeBranch,
                                                          const ReplaySteps& lookup, V3 org, V3 dir, V3 T, V3& radiance) {
    const x2_config& c = s.config;
    if (!(pv.volumeDepth < c.max_volume_depth && c.volume_illumination_samples > 0)) return;
    const uint32_t scatterSamples = c.volume_illumination_samples;
    const float invN = 1.0f / float(scatterSamples);
    for (uint32_t i = 0; i < scatterSamples; ++i) {
        Identity mid = root;
        mid.branch = childBranch(volumeBranch, 0xffff, i);
        Stream ms(mid, pv.depth, 0);
        float pdfDensity, utRemapped;
        const VolumeStep vp = lookup.pick(ms.next(), pdfDensity, utRemapped);
        float sigmaT = vlum(vp.sigmaT);
        const float t0 = vp.tStart, t1 = vp.tStart + vp.delta;
        const float td = sampleDistanceExponential(utRemapped, sigmaT, t0, t1);
        const float pdfT = pdfDensity * pdfDistanceExponential(td, sigmaT, t0, t1);
        if (pdfT == 0.0f || !vfinite(pdfT)) continue;
        const V3 trScatter = vtimes(vp.tr, expNeg(vp.sigmaT, td - t0));
        V3 scatterPoint = add(org, mul(dir, td));
        V3 throughput = vscaled(vtimes(vtimes(T, vp.sigmaS), trScatter), 1.0f / pdfT);
        const float up0 = ms.next(), up1 = ms.next();
        V3 scatterDir = phaseSample(vp.g, V3{-dir.x, -dir.y, -dir.z}, up0, up1);
        for (uint32_t depth = pv.volumeDepth; depth < c.max_volume_depth; ++depth) {
            if (vlum(throughput) < c.volume_transmittance_threshold) break;
            const float ai = mf::pow(c.volume_attenuation_factor, float(depth)), bi = mf::pow(c.volume_contribution_factor, float(depth)),
                        ci = mf::pow(c.volume_phase_attenuation_factor, float(depth));
            const float tFreePath = -mf::log(1.0f - ms.next()) / sigmaT;
            Crossing y[kMaxCrossings];
            uint32_t here;
            const uint32_t m = volumeIntervals(s, scatterPoint, scatterDir, kVolumeEpsilon, y, here);
            for (uint32_t j = 0; j < m && y[j].t <= tFreePath; ++j) applyCrossing(here, y[j]);
            const V3 rayDir = scatterDir;
            scatterPoint = add(scatterPoint, mul(scatterDir, tFreePath));
            if (!here) break;
            const float rnd = c.volume_overlap_mode == kOverlapRnd ? ms.next() : 0.0f;
            const VolumeCoefficients kk = evalShadersAt(s, here, c.volume_overlap_mode, rnd, scatterPoint, kNoGrid, nullptr, nullptr);
            const float g = kk.g * ci;
            sigmaT = vlum(kk.sigmaT);
            if (vIsZero(sigmaT)) break;
            throughput = vscaled(vtimes(throughput, kk.sigmaS), 1.0f / sigmaT);
            for (uint32_t li = 0; li < c.light_count; ++li) {
                const float usl[3] = {ms.next(), ms.next(), ms.next()};
                const V3 Ls = volumeSourceTerm(s, ms, s.lights[li], scatterPoint, rayDir, g, usl, ai);
                radiance = vplus(radiance, vscaled(vtimes(throughput, Ls), invN * bi));
            }
            const float uq0 = ms.next(), uq1 = ms.next();
            scatterDir = phaseSample(g, V3{-rayDir.x, -rayDir.y, -rayDir.z}, uq0, uq1);
        }
    }
}

// What volumeRadiance leaves besides its light: the transmittance the path's throughput takes and the alpha's.
struct VolumePass {
    V3 transmittance, alphaTransmittance;
};

// computeRadianceVolume over [tnear, tfar] of a ray (volumeRadiance, async_integrator.h:1152-1291): the camera ray's
// volume emission, the single scattering of every light at the march's steps (a volume depth on), and the path's
// throughput through the volumes. pv's T and volume depth are updated.
static __device__ __noinline__ V3 volumeRadiance(const SceneView& s, const Identity& root, Pending& pv, V3 org, V3 dir, float tnear, float tfar,
                                          V3& alphaTransmittance) {
    const x2_config& c = s.config;
    V3 radiance{0, 0, 0};
    alphaTransmittance = V3{1, 1, 1};
    Crossing x[kMaxCrossings];
    uint32_t regions;
    const uint32_t n = volumeIntervals(s, org, dir, tnear, x, regions);
    if (n == 0 && regions == 0) return radiance;
    const U64 volumeBranch = childBranch(pv.branch, 0xfffc, pv.volumeDepth);
    Identity vid = root;
    vid.branch = childBranch(volumeBranch, 0, 0);
    const bool sampleEmission = pv.depth == 0;
    VolumeMarch march{s, x, n, regions, org, dir, tnear, tfar, pv.depth, sampleEmission, Stream(vid, pv.depth, 0), kMarchLimit};
    float weights = 0.0f, firstStart = 0.0f, lastEnd = 0.0f;
    auto first = [&](const VolumeStep& st, uint32_t i) {
        if (i == 0) firstStart = st.tStart;
        lastEnd = st.tStart + st.delta;
        weights += stepWeight(st);
        return true;
    };
    MarchRecord record;
    march.record = &record;
    march.weightsSoFar = &weights;
    march.run(first);
    march.record = nullptr;
    const uint32_t count = march.count;
    if (count == 0) return radiance;
    V3 vt = march.vt, vta = march.vt;
    if (march.reachedThreshold) vt = vta = V3{0, 0, 0};
    alphaTransmittance = vta;
    const V3 T = pv.T;
    if (sampleEmission)
        for (uint32_t v = 0; v < c.volume_count; ++v) {
            if (!(march.visited >> v & 1)) continue;
            const V3 emission = vtimes(T, march.emitted[v]);
            if (vblack(emission)) continue;
            radiance = vplus(radiance, emission);
        }
    if (pv.volumeDepth < c.max_volume_depth) {
        const ReplaySteps lookup{march, count, weights != 0.0f ? weights : 1.0f, weights == 0.0f, &record};
        const float rayEnd = lastEnd;
        // integrateVolumeScatteringDirect (async_integrator.h:921-997).
        const bool highQuality = pv.nonMirror == 0;
        const uint32_t samplesPerLight = highQuality ? c.light_samples : 1, scatterCount = highQuality ? c.volume_illumination_samples : 1;
        if (scatterCount > 0) {
            const float invN = 1.0f / float(samplesPerLight * scatterCount);
            for (uint32_t li = 0; li < c.light_count; ++li) {
                const x2_light& L = s.lights[li];
                const bool equiAngular = boundedLight(L);
                V3 direct{0, 0, 0};
                for (uint32_t ls = 0; ls < samplesPerLight; ++ls) {
                    for (uint32_t ts = 0; ts < scatterCount; ++ts) {
                        Identity sid = root;
                        sid.branch = childBranch(volumeBranch, 1 + li, ls * scatterCount + ts);
                        Stream ss(sid, pv.depth, 0);
                        float D = 0.0f, thetaA = 0.0f, thetaB = 0.0f, offset = 0.0f;
                        float uel[3] = {0.0f, 0.0f, 0.0f};
                        if (equiAngular) {
                            const float ue = ss.next();
                            uel[0] = ss.next();
                            uel[1] = ss.next();
                            uel[2] = ss.next();
                            const V3 pivot = lightPivot(L, uel);
                            offset = dot(add(pivot, mul(org, -1.0f)), dir);
                            const V3 foot = add(org, mul(dir, offset));
                            D = length(add(pivot, mul(foot, -1.0f)));
                            thetaA = mf::atan2(firstStart - offset, D);
                            thetaB = mf::atan2(rayEnd - offset, D);
                            const float te = sampleEquiAngular(ue, D, thetaA, thetaB);
                            const float pdfTe = pdfEquiAngular(te, D, thetaA, thetaB);
                            if (pdfTe != 0.0f && vfinite(pdfTe)) {
                                const float tePrime = te + offset;
                                float pdfK;
                                const VolumeStep vp = lookup.at(tePrime, pdfK);
                                if (!vblack(vp.sigmaS)) {
                                    const V3 trScatter = vtimes(vp.tr, expNeg(vp.sigmaT, tePrime - vp.tStart));
                                    float mis = 1.0f;
                                    const float pdfTd = pdfK * pdfDistanceExponential(tePrime, vlum(vp.sigmaT), vp.tStart, vp.tStart + vp.delta);
                                    if (vfinite(pdfTd)) mis = powerHeuristic(pdfTe, pdfTd);
                                    const V3 Ls = volumeSourceTerm(s, ss, L, add(org, mul(dir, tePrime)), dir, vp.g, uel, 1.0f);
                                    direct = vplus(direct, vscaled(vtimes(vtimes(T, vp.sigmaS), vtimes(trScatter, Ls)), invN * mis / pdfTe));
                                }
                            }
                        }
                        const float ud = ss.next();
                        const float udl[3] = {ss.next(), ss.next(), ss.next()};
                        float pdfDensity, udRemapped;
                        const VolumeStep vp = lookup.pick(ud, pdfDensity, udRemapped);
                        if (pdfDensity == 0.0f) continue;
                        if (vblack(vp.sigmaS)) continue;
                        const float sigmaT = vlum(vp.sigmaT), t0 = vp.tStart, t1 = vp.tStart + vp.delta;
                        const float td = sampleDistanceExponential(udRemapped, sigmaT, t0, t1);
                        const float pdfTd = pdfDensity * pdfDistanceExponential(td, sigmaT, t0, t1);
                        if (pdfTd == 0.0f || !vfinite(pdfTd)) continue;
                        const V3 trScatter = vtimes(vp.tr, expNeg(vp.sigmaT, td - t0));
                        float mis = 1.0f;
                        if (equiAngular) {
                            const float pdfTe = pdfEquiAngular(td - offset, D, thetaA, thetaB);
                            if (vfinite(pdfTe)) mis = powerHeuristic(pdfTd, pdfTe);
                        }
                        // (The diagnostic build's shared-pivot switch gives this sample the equi-angular sample's light
                        // point, the pivot its MIS weight was computed with; the reference draws a point of its own.)
                        const V3 Ls = volumeSourceTerm(s, ss, L, add(org, mul(dir, td)), dir, vp.g,
                                                       equiAngular && mf::sharedPivot() ? uel : udl, 1.0f);
                        direct = vplus(direct, vscaled(vtimes(vtimes(T, vp.sigmaS), vtimes(trScatter, Ls)), invN * mis / pdfTd));
                    }
                }
                radiance = vplus(radiance, direct);
            }
        }
        ++pv.volumeDepth;
        volumeMultipleScatter(s, root, pv, volumeBranch, lookup, org, dir, T, radiance);
    }
    pv.T = vtimes(pv.T, vt);
    return radiance;
}

}  // namespace x2
