// The pieces one path vertex is made of, on the device, for the admitted subset of the reference's integratePaths
// (xpu2/interactive/async_integrator.h:1986-3042): a box-filtered pinhole camera, hit reconstruction, the shading
// state, Lambert and Schlick-GGX UsdPreviewSurface lobes, Rect and constant Env lights. No presence, volumes,
// subsurface or AOVs.
//
// The arithmetic follows the reference operation for operation (same association, same float/double types,
// the same signed-zero behaviour) so that, built without contraction (-fmad=false) like the reference's CPU lane
// (-ffp-contract=off), a sample's random numbers are bit-exact and its radiance agrees to rounding of the
// transcendental functions (CUDA's on the device, libm on the host; mathfn.cuh). Each function cites what it follows.
#pragma once
#include <cfloat>
#include <cstdint>

#include "../../include/x2.h"
#include "bvh.cuh"
#include "mathfn.cuh"
#include "sampler.cuh"
#include "traverse.cuh"

namespace x2 {

// ---------------------------------------------------------------------------------------------------------------
// Vector arithmetic with the reference's association (surface_core.h:12-18, shade_math.h:14-27).
struct V3 {
    float x, y, z;
};
__device__ __forceinline__ V3 v3(float x, float y, float z) { return V3{x, y, z}; }
__device__ __forceinline__ V3 add(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3 sub(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3 mul(V3 a, float b) { return V3{a.x * b, a.y * b, a.z * b}; }
__device__ __forceinline__ V3 mulv(V3 a, V3 b) { return V3{a.x * b.x, a.y * b.y, a.z * b.z}; }
__device__ __forceinline__ V3 divs(V3 a, float b) { return V3{a.x / b, a.y / b, a.z / b}; }
__device__ __forceinline__ V3 neg(V3 a) { return V3{-a.x, -a.y, -a.z}; }
__device__ __forceinline__ float dot(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
__device__ __forceinline__ V3 cross(V3 a, V3 b) { return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
__device__ __forceinline__ bool finitef(float a) { return a == a && a <= 3.402823466e38f && a >= -3.402823466e38f; }
__device__ __forceinline__ bool finite3(V3 a) { return finitef(a.x) && finitef(a.y) && finitef(a.z); }
// surface::normalize (surface_core.h:19): checked.
__device__ __forceinline__ bool normalizeChecked(V3 a, V3& b) {
    const float l = dot(a, a);
    if (!finitef(l) || l <= 0) return false;
    b = mul(a, 1.0f / sqrtf(l));
    return true;
}
// shade::normalize, length (shade_math.h:68-69): unchecked.
__device__ __forceinline__ float length(V3 a) { return sqrtf(dot(a, a)); }
__device__ __forceinline__ V3 normalizeU(V3 a) { return mul(a, 1.0f / sqrtf(dot(a, a))); }
__device__ __forceinline__ bool isExactlyZero(V3 c) { return c.x == 0 && c.y == 0 && c.z == 0; }
__device__ __forceinline__ bool isEqual0(float x) { return fabsf(x - 0.0f) <= fmaxf(fabsf(x), 1.0f) * 1e-6f; }
__device__ __forceinline__ bool isBlack(V3 c) { return isEqual0(c.x) && isEqual0(c.y) && isEqual0(c.z); }
__device__ __forceinline__ float luminance(V3 c) { return 0.299f * c.x + 0.587f * c.y + 0.114f * c.z; }

constexpr float kEpsilon = 1e-6f, kPi = 3.14159265358979323846f, kTwoPi = 6.28318530717958647692f;
constexpr float kOneOverPi = 0.318309886183790671538f;
constexpr float kInfiniteDistance = 3.4028234663852886e+38f - 1e32f;
constexpr float kEnvDistance = kInfiniteDistance * 0.9f;
constexpr float kDistantDistance = kInfiniteDistance * 0.8f;
constexpr float kHitEpsilonEnd = 1.0f - 1e-3f;
constexpr float kFltMax = 3.402823466e+38f;

// Lobe types and flags (shade_lobes.h:21-38).
enum : uint32_t {
    kReflection = 1u, kTransmission = 2u, kDiffuse = 4u, kGlossy = 16u, kMirror = 64u,
    kAllSurfaceSides = 3u, kAllLobes = 84u, kAllDiffuse = 7u, kAllGlossy = 19u, kAllMirror = 67u, kAllLobeTypes = 87u
};
__device__ __forceinline__ bool matchesFlags(uint32_t type, uint32_t flags) {
    return (type & kAllSurfaceSides & flags) && (type & kAllLobes & flags);
}
// lights::lobeRayMask (light_core.h:191).
__device__ __forceinline__ uint32_t lobeRayMask(uint32_t t) {
    uint32_t m = 0;
    if (t & 1u) m |= t & 0x54u;
    if (t & 2u) m |= (t & 0x54u) << 1;
    return m;
}

// ---------------------------------------------------------------------------------------------------------------
// The scene as the kernels read it.
struct MaterialRec {
    uint32_t kind;
    float diffuse[3], specular[3], emission[3], roughness;
    uint32_t texture;  // 0: none; k + 1: texture k bound to the diffuse colour
};
// A texture on the device: fp32 RGB texels (3 floats each, row-major, row 0 the top) from `first` texel on.
struct TexRec {
    uint64_t first;
    uint32_t width, height, wrap, pad;
};
struct Counters {
    unsigned long long trace, nee, bsdf, held, samples, errors, overflow, pad;
};
// A volume on the device (x2_volume; volume::Shader's VdbVolume fields, volume_core.h:64-111) and a dense grid.
constexpr int kMajorantCells = 32;  // a volume's majorant grid: kMajorantCells^3 over its bounds
struct VolumeRec {
    float worldToGrid[12];
    V3 gain, colorMult, incandescence;
    float g, featureSize, surfaceThreshold;
    uint32_t densityGrid, emissionGrid, interpolation;
    V3 lo, hi;              // its bounds (world)
    const float* majorant;  // the largest extinction any lookup can read in each cell (the tracking estimator's)
    float majorantMax;
};
struct GridRec {
    double worldToIndex[16];
    const float* values;
    int lo[3], dims[3];
    uint32_t channels;
};

struct SceneView {
    const VolumeRec* volumes;       // volume_count of them (config.volume_count), their bounds' triangles (12 a volume,
    const GridRec* grids;           // 9 floats each) and the grids they read
    const float* volumeTris;
    uint32_t gridCount;
    Bvh8 bvh;
    const uint32_t* triMesh;        // scene triangle -> mesh
    const uint32_t* meshFirst;      // mesh -> first triangle
    const uint32_t* meshMaterial;   // mesh -> material
    const MaterialRec* materials;
    const x2_light* lights;
    x2_camera camera;
    x2_config config;
    uint32_t* overflow;             // traversal stack overflows
    TraversalStats* stats;          // a counting run's traversal work ([0] closest hits, [1] any hits); null when timed
    const TexRec* textures;         // the scene's textures and their texels (null without textures)
    const float* texels;
    const float* triUV;             // scene triangle -> its vertices' st (6 floats); null: no texture is read
};

// ---------------------------------------------------------------------------------------------------------------
// Camera: the box filter (surface_core.h:48-51) and perspectiveRay without depth of field (camera_core.h:217-263).
__device__ __forceinline__ bool boxFilter(float width, float r, float& out) {
    if (!finitef(width) || width <= 0 || !finitef(r) || r < 0 || r > 1) return false;
    out = (r - .5f) * width + .5f;
    return finitef(out);
}
__device__ __forceinline__ V3 mvector(const float m[4][4], V3 a) {
    return V3{(a.x * m[0][0] + a.y * m[1][0]) + a.z * m[2][0], (a.x * m[0][1] + a.y * m[1][1]) + a.z * m[2][1],
              (a.x * m[0][2] + a.y * m[1][2]) + a.z * m[2][2]};
}
__device__ __forceinline__ V3 transformH(const float m[4][4], V3 p) {
    const V3 v = add(mvector(m, p), V3{m[3][0], m[3][1], m[3][2]});
    const float w = ((p.x * m[0][3] + p.y * m[1][3]) + p.z * m[2][3]) + m[3][3];
    if (w == 0.0f) return V3{0, 0, 0};
    return V3{v.x / w, v.y / w, v.z / w};
}
struct CameraRay {
    V3 origin, direction;
    float nearT, farT;
};
__device__ __forceinline__ bool perspectiveRay(const x2_camera& c, float x, float y, CameraRay& out) {
    const V3 fp{0, 0, 0};
    const V3 dir = sub(transformH(c.raster_to_camera, V3{x, y, -1.0f}), fp);
    const V3 origin = add(mvector(c.camera_to_render, fp), V3{c.camera_to_render[3][0], c.camera_to_render[3][1], c.camera_to_render[3][2]});
    V3 n;
    if (!normalizeChecked(dir, n) || n.z >= 0) return false;
    out.nearT = (-c.near_clip - fp.z) / n.z;
    out.farT = (-c.far_clip - fp.z) / n.z;
    if (!normalizeChecked(mvector(c.camera_to_render, dir), out.direction) || !finite3(origin) || !finitef(out.nearT) || !finitef(out.farT))
        return false;
    out.origin = origin;
    return true;
}

// ---------------------------------------------------------------------------------------------------------------
// Hits: resume::geometryHit (resume_core.h:17-45) with triangle::coordinates (triangle_hit.h:6-21), in double.
struct Hit {
    uint32_t geom, prim;
    float t, u, v;
    V3 normal, origin, below, point;
};
__device__ __forceinline__ bool geometryHit(Hit& h, V3 ro, V3 rd, V3 a, V3 b, V3 c) {
    const V3 e1 = add(b, mul(a, -1)), e2 = add(c, mul(a, -1));
    if (!normalizeChecked(cross(e1, e2), h.normal)) return false;
    if (dot(h.normal, rd) > 0) h.normal = mul(h.normal, -1);
    const double ax = a.x, ay = a.y, az = a.z;
    const double ex = double(b.x) - ax, ey = double(b.y) - ay, ez = double(b.z) - az;
    const double fx = double(c.x) - ax, fy = double(c.y) - ay, fz = double(c.z) - az;
    const double dx = rd.x, dy = rd.y, dz = rd.z;
    const double px = dy * fz - dz * fy, py = dz * fx - dx * fz, pz = dx * fy - dy * fx;
    const double determinant = (ex * px + ey * py) + ez * pz;
    if (determinant == 0) return false;
    const double tx = double(ro.x) - ax, ty = double(ro.y) - ay, tz = double(ro.z) - az;
    const double qx = ty * ez - tz * ey, qy = tz * ex - tx * ez, qz = tx * ey - ty * ex;
    const double u = ((tx * px + ty * py) + tz * pz) / determinant;
    const double v = ((dx * qx + dy * qy) + dz * qz) / determinant;
    const double t = ((fx * qx + fy * qy) + fz * qz) / determinant;
    if (!finitef(float(t)) || !finitef(float(u)) || !finitef(float(v))) return false;
    h.t = float(t);
    h.u = float(u);
    h.v = float(v);
    const V3 p{float(double(a.x) + ((double(b.x) - a.x) * u + (double(c.x) - a.x) * v)),
               float(double(a.y) + ((double(b.y) - a.y) * u + (double(c.y) - a.y) * v)),
               float(double(a.z) + ((double(b.z) - a.z) * u + (double(c.z) - a.z) * v))};
    h.point = p;
    const V3 error{fabsf(a.x) + fabsf(e1.x) + fabsf(e2.x), fabsf(a.y) + fabsf(e1.y) + fabsf(e2.y), fabsf(a.z) + fabsf(e1.z) + fabsf(e2.z)};
    const float extent = fmaxf(fmaxf(fabsf(e1.x), fabsf(e1.y)), fmaxf(fabsf(e1.z), fmaxf(fabsf(e2.x), fmaxf(fabsf(e2.y), fabsf(e2.z)))));
    const float d = 16 * 0x1p-23f * (fabsf(h.normal.x) * error.x + fabsf(h.normal.y) * error.y + fabsf(h.normal.z) * error.z + extent);
    h.origin = add(p, mul(h.normal, d));
    if (h.normal.x != 0) h.origin.x = nextafterf(h.origin.x, h.normal.x > 0 ? kFltMax : -kFltMax);
    if (h.normal.y != 0) h.origin.y = nextafterf(h.origin.y, h.normal.y > 0 ? kFltMax : -kFltMax);
    if (h.normal.z != 0) h.origin.z = nextafterf(h.origin.z, h.normal.z > 0 ? kFltMax : -kFltMax);
    h.below = add(p, mul(h.normal, -d));
    if (h.normal.x != 0) h.below.x = nextafterf(h.below.x, h.normal.x > 0 ? -kFltMax : kFltMax);
    if (h.normal.y != 0) h.below.y = nextafterf(h.below.y, h.normal.y > 0 ? -kFltMax : kFltMax);
    if (h.normal.z != 0) h.below.z = nextafterf(h.below.z, h.normal.z > 0 ? -kFltMax : kFltMax);
    return finite3(h.origin) && finite3(h.below);
}

// Closest hit through the BVH, then the reference's reconstruction (CpuBackend::trace, async_cpu.h:669-720).
__device__ __forceinline__ Hit trace(const SceneView& s, V3 o, V3 d, float tmin, float tmax, V3& va, V3& vb, V3& vc) {
    Hit h;
    h.geom = ~0u;
    h.prim = 0;
    h.t = h.u = h.v = 0;
    h.normal = h.origin = h.below = h.point = V3{0, 0, 0};
    const RayQ r = makeRay(s.bvh, o.x, o.y, o.z, d.x, d.y, d.z);
    float t;
    uint32_t leaf;
    const uint32_t tri = s.stats ? traceClosest<true>(s.bvh, r, tmin, tmax, t, &leaf, s.overflow, s.stats + 0)
                                 : traceClosest<false>(s.bvh, r, tmin, tmax, t, &leaf, s.overflow, nullptr);
    X2_DIAG_RECORD(mf::kHit, __uint_as_float(tri), tri == ~0u ? 0.0f : t, d.x, d.y);
    if (tri == ~0u) return h;
    const float4* tp = reinterpret_cast<const float4*>(s.bvh.tris + leaf);
    const float4 a = __ldg(tp), b = __ldg(tp + 1), c = __ldg(tp + 2);
    va = V3{a.x, a.y, a.z};
    vb = V3{b.x, b.y, b.z};
    vc = V3{c.x, c.y, c.z};
    h.geom = __ldg(s.triMesh + tri);
    h.prim = tri - __ldg(s.meshFirst + h.geom);
    h.t = t;
    if (!geometryHit(h, o, d, va, vb, vc)) h.normal = V3{0, 0, 0};
    return h;
}
__device__ __forceinline__ bool visible(const SceneView& s, V3 o, V3 d, float near, float far) {
    const RayQ r = makeRay(s.bvh, o.x, o.y, o.z, d.x, d.y, d.z);
    const bool v = !(s.stats ? traceAny<true>(s.bvh, r, near, far, s.overflow, s.stats + 1) : traceAny<false>(s.bvh, r, near, far, s.overflow, nullptr));
    X2_DIAG_RECORD(mf::kVisible, v ? 1.0f : 0.0f, far, d.x, d.y);
    return v;
}

// ---------------------------------------------------------------------------------------------------------------
// Shading state and the material's lobe (shade_material.h:121-283, :338-383; shade_builder.h:541-556, :689-697).
struct Frame {
    V3 x, y, z;
};
// shade::frame(N) (shade_math.h:138-141), Duff et al. 2017.
__device__ __forceinline__ Frame frameN(V3 N) {
    const float sign = copysignf(1.0f, N.z), a = -1.0f / (sign + N.z), b = N.x * N.y * a;
    return Frame{V3{1.0f + sign * N.x * N.x * a, sign * b, -sign * N.x}, V3{b, sign + N.y * N.y * a, -N.y}, N};
}
// shade::frame(N, T) (shade_math.h:142-148).
__device__ __forceinline__ Frame frameNT(V3 N, V3 T) {
    Frame f;
    f.z = N;
    f.y = normalizeU(cross(N, T));
    f.x = cross(f.y, f.z);
    return f;
}
__device__ __forceinline__ V3 localToGlobal(const Frame& f, V3 v) { return add(add(mul(f.x, v.x), mul(f.y, v.y)), mul(f.z, v.z)); }

// scene_rdl2 differenceOfProducts with its error term (shade_material.h:95-101).
__device__ __forceinline__ float differenceOfProducts(float a, float b, float c, float d) {
    const float cd = c * d;
    const float err = fmaf(-c, d, cd);
    const float dop = fmaf(a, b, -cd);
    return dop + err;
}
// computeTrianglePartials at the default st (0,0), (1,0), (1,1) (shade_material.h:102-116).
// st: the triangle's three texture coordinates (s, t each), or null for the reference's default (0, 0), (1, 0), (1, 1)
// of a mesh without them.
__device__ __forceinline__ bool trianglePartials(V3 x0, V3 x1, V3 x2, const float* st, V3& dPds) {
    const float A0 = st ? st[2] - st[0] : 1.0f - 0.0f, A1 = st ? st[3] - st[1] : 0.0f - 0.0f;
    const float A2 = st ? st[4] - st[0] : 1.0f - 0.0f, A3 = st ? st[5] - st[1] : 1.0f - 0.0f;
    const V3 b0 = sub(x1, x0), b1 = sub(x2, x0);
    const float det = differenceOfProducts(A0, A3, A1, A2);
    if (!(fabsf(det) >= 1.17549435e-38f) || !(fabsf(det) <= 3.402823466e38f)) return false;
    const float inv = 1.0f / det;
    dPds = mul(V3{differenceOfProducts(b0.x, A3, b1.x, A1), differenceOfProducts(b0.y, A3, b1.y, A1),
                  differenceOfProducts(b0.z, A3, b1.z, A1)}, inv);
    const V3 dPdt = mul(V3{differenceOfProducts(b1.x, A0, b0.x, A2), differenceOfProducts(b1.y, A0, b0.y, A2),
                           differenceOfProducts(b1.z, A0, b0.z, A2)}, inv);
    return finite3(dPds) && finite3(dPdt);
}

struct State {
    V3 P, Ng, N, wo, dPds;
    bool entering;
};
// hitState for a mesh without normals (shade_material.h:121-283); st: its texture coordinates (null: none), which set
// dPds (and through it the shading frame's rounding, down to the sign of a zero normal component).
__device__ __forceinline__ bool hitState(V3 a, V3 b, V3 c, float u, float v, V3 P, V3 rayDir, State& st, const float* stCoords = nullptr) {
    (void)u;
    (void)v;
    V3 ng = cross(sub(b, a), sub(c, a));
    float l = length(ng);
    if (!(l > 0)) {
        const double ux = double(b.x) - a.x, uy = double(b.y) - a.y, uz = double(b.z) - a.z;
        const double vx = double(c.x) - a.x, vy = double(c.y) - a.y, vz = double(c.z) - a.z;
        const double nx = uy * vz - uz * vy, ny = uz * vx - ux * vz, nz = ux * vy - uy * vx;
        const double dl = sqrt(nx * nx + ny * ny + nz * nz);
        ng = dl > 0 ? V3{float(nx / dl), float(ny / dl), float(nz / dl)} : neg(rayDir);
        l = length(ng);
        if (!(l > 0)) return false;
    }
    st.Ng = divs(ng, l);
    V3 N = st.Ng;
    if (!trianglePartials(a, b, c, stCoords, st.dPds)) st.dPds = frameN(N).x;
    st.P = P;
    st.wo = neg(rayDir);
    st.entering = dot(st.Ng, rayDir) < 0.0f;
    if (!st.entering) {
        N = neg(N);
        st.Ng = neg(st.Ng);
    }
    st.N = N;
    return finite3(st.N) && finite3(st.Ng);
}
// Intersection_adaptNormal (shade_state.h:256-264).
__device__ __forceinline__ V3 adaptNormal(const State& st, V3 Ns) {
    const V3 wo = st.wo, Ng = st.Ng;
    const V3 r = sub(mul(Ns, 2.f * dot(Ns, wo)), wo);
    const float rDotNg = dot(r, Ng), eps = 0.001f;
    if (rDotNg < eps) {
        const V3 rBent = normalizeU(add(r, mul(Ng, eps - rDotNg)));
        return normalizeU(add(wo, rBent));
    }
    return Ns;
}

// The hit's single lobe (kind 0: Lambert, 1: GGX with Schlick Fresnel), or none.
struct Lobe {
    uint32_t kind, type;  // kind: 0 Lambert, 1 GGX; type: lobe type bits
    Frame frame;
    V3 albedo;            // Lambert
    V3 spec;              // GGX: the Schlick F0
    float roughness;      // GGX: max(0.001, r^2)
};
struct Bsdf {
    uint32_t count;  // 0 or 1 lobes
    uint32_t type;
    V3 emission;
    Lobe lobe;
};
__device__ __forceinline__ float saturate(float x) { return fminf(fmaxf(x, 0.0f), 1.0f); }
// ---------------------------------------------------------------------------------------------------------------
// Textures: UsdUVTexture's lookup (shade_mapnodes.h:972-997) with no filter footprint — texture_core.h lookup at
// (s, 1 - t): level 0 only; on primary paths the anisotropic filter reduces to one bilinear lookup, on indirect paths
// (trilinear and one-level modes) to the closest texel (textureMode, shade_mapnodes.h:344-347).
struct TexHit {
    float s, t;       // the hit's st (hitState's interpolation of the vertices' uvs)
    uint32_t primary; // 1: a primary path (bilinear), 0: indirect (closest texel)
    V3 texel;         // the lookup's value
};
__device__ __forceinline__ int texAddress(int x, int n, uint32_t wrap) {
    if (wrap) {
        const int v = x % n;
        return v < 0 ? v + n : v;
    }
    return x < 0 ? 0 : x >= n ? n - 1 : x;
}
__device__ __forceinline__ V3 texFetch(const SceneView& s, const TexRec& t, int x, int y) {
    const float* p = s.texels + 3 * (t.first + uint64_t(texAddress(y, int(t.height), t.wrap)) * t.width + uint64_t(texAddress(x, int(t.width), t.wrap)));
    return V3{__ldg(p), __ldg(p + 1), __ldg(p + 2)};
}
// The lookup's texels and weights (up to 4: bilinear x, x+1 over y, y+1; closest: 1), its value in `out`. False where
// the reference's lookup is Invalid (a non-finite or far coordinate or value).
__device__ __forceinline__ bool texLookup(const SceneView& s, uint32_t texture, TexHit& h, uint64_t* texels = nullptr, float* weights = nullptr) {
    const TexRec tr = s.textures[texture];
    float u = 1.0f * h.s + 0.0f, v = 1.0f - (1.0f * h.t + 0.0f);
    if (!finitef(u) || !finitef(v)) return false;
    if (fabsf(u) > 1024) u = tr.wrap ? u - floorf(u) : fminf(fmaxf(u, -1.0f), 2.0f);
    if (fabsf(v) > 1024) v = tr.wrap ? v - floorf(v) : fminf(fmaxf(v, -1.0f), 2.0f);
    float fx = u * float(tr.width) - .5f, fy = v * float(tr.height) - .5f;
    if (!finitef(fx) || !finitef(fy) || fabsf(fx) > 1.e8f || fabsf(fy) > 1.e8f) return false;
    int x = int(floorf(fx)), y = int(floorf(fy));
    auto index = [&](int xx, int yy) {
        return tr.first + uint64_t(texAddress(yy, int(tr.height), tr.wrap)) * tr.width + uint64_t(texAddress(xx, int(tr.width), tr.wrap));
    };
    if (h.primary) {
        fx -= float(x);
        fy -= float(y);
        const V3 a = texFetch(s, tr, x, y), b = texFetch(s, tr, x + 1, y), c = texFetch(s, tr, x, y + 1), d = texFetch(s, tr, x + 1, y + 1);
        h.texel = add(mul(add(mul(a, 1 - fx), mul(b, fx)), 1 - fy), mul(add(mul(c, 1 - fx), mul(d, fx)), fy));
        if (texels) {
            texels[0] = index(x, y);
            texels[1] = index(x + 1, y);
            texels[2] = index(x, y + 1);
            texels[3] = index(x + 1, y + 1);
            weights[0] = (1 - fx) * (1 - fy);
            weights[1] = fx * (1 - fy);
            weights[2] = (1 - fx) * fy;
            weights[3] = fx * fy;
        }
    } else {
        if (fx - float(x) > .5f) ++x;
        if (fy - float(y) > .5f) ++y;
        h.texel = texFetch(s, tr, x, y);
        if (texels) {
            texels[0] = index(x, y);
            weights[0] = 1.0f;
            for (int k = 1; k < 4; ++k) {
                texels[k] = texels[0];
                weights[k] = 0.0f;
            }
        }
    }
    X2_DIAG_RECORD(mf::kTexLookup, h.s, h.t, h.texel.x, h.texel.y);
    X2_DIAG_RECORD(mf::kTexLookupRest, float(h.primary), 0.0f, h.texel.z, 0.0f);
    return finite3(h.texel);
}

// The lobe shadeMaterial makes for a material: 1 a GGX lobe, 0 a Lambert lobe, 2 none (the wavefront's per-lobe
// queues sort paths by it before shading).
__device__ __forceinline__ uint32_t lobeClass(const MaterialRec& m) {
    if (m.kind == X2_MAT_GGX && !isBlack(V3{saturate(m.specular[0]), saturate(m.specular[1]), saturate(m.specular[2])})) return 1;
    return isBlack(V3{m.diffuse[0], m.diffuse[1], m.diffuse[2]}) ? 2 : 0;
}
// shadeUsdPreviewSurface with useSpecularWorkflow = 1 (shade_material.h:338-383); a textured material's diffuse colour
// times its texel when not black (the map binding's BindColor rule, shade_maps.h applyRule).
__device__ __forceinline__ void shadeMaterial(const MaterialRec& m, const State& st, Bsdf& b, V3 texel = V3{1, 1, 1}) {
    b.count = 0;
    b.type = 0;
    b.emission = V3{0, 0, 0};
    V3 N;
    if (fabsf(length(st.dPds)) <= kEpsilon) N = st.N;
    else N = normalizeU(localToGlobal(frameNT(st.N, normalizeU(st.dPds)), V3{0, 0, 1}));
    V3 albedo{m.diffuse[0], m.diffuse[1], m.diffuse[2]};
    if (m.texture && !isBlack(albedo)) albedo = mulv(albedo, texel);
    const float roughness = saturate(m.roughness);
    const V3 emissive{m.emission[0], m.emission[1], m.emission[2]};
    if (!isBlack(emissive)) b.emission = add(b.emission, emissive);
    if (m.kind == X2_MAT_GGX) {
        const V3 spec{saturate(m.specular[0]), saturate(m.specular[1]), saturate(m.specular[2])};
        if (!isBlack(spec)) {
            // addSchlickReflection: a GGX lobe about the adapted normal, Schlick Fresnel (factor 1, neta 1).
            const V3 Na = adaptNormal(st, N);
            b.lobe.kind = 1;
            b.lobe.type = kReflection | kGlossy;
            b.lobe.frame = frameN(Na);
            b.lobe.spec = spec;
            b.lobe.roughness = fmaxf(0.001f, roughness * roughness);
            b.lobe.albedo = V3{0, 0, 0};
            b.count = 1;
            b.type = b.lobe.type;
            return;  // a black diffuse colour: no Lambert lobe under it (admitted GGX materials have none)
        }
    }
    if (!isBlack(albedo)) {
        b.lobe.kind = 0;
        b.lobe.type = kReflection | kDiffuse;
        b.lobe.frame = frameN(N);
        b.lobe.albedo = albedo;
        b.lobe.spec = V3{0, 0, 0};
        b.lobe.roughness = 1.0f;
        b.count = 1;
        b.type = b.lobe.type;
    }
}

// ---------------------------------------------------------------------------------------------------------------
// Lobe evaluation and sampling (shade_lobes_eval.h: Lambert :611-620, :659-664; GGX :93-146).
struct Slice {
    V3 Ng, wo;
};
__device__ __forceinline__ uint32_t surfaceFlags(const Slice& s, V3 wi) {
    return dot(s.Ng, s.wo) * dot(s.Ng, wi) > 0.0f ? (kAllLobeTypes & ~kTransmission) : (kAllLobeTypes & ~kReflection);
}
__device__ __forceinline__ V3 localSpherical(float cosTheta, float sinTheta, float phi) {
    float s, c;
    mf::sincos(phi, &s, &c);
    return V3{sinTheta * c, sinTheta * s, cosTheta};
}
__device__ __forceinline__ V3 schlick(V3 a, float hDotWi) {
    const float tmp = 1.0f - hDotWi;
    float power = tmp * tmp;
    power = tmp * power * power;
    return add(a, mul(mul(sub(V3{1, 1, 1}, a), 1.0f), power));
}
__device__ __forceinline__ V3 evalGGX(const Lobe& l, const Slice& s, V3 wi, float& pdf) {
    const Frame& f = l.frame;
    const float roughness = l.roughness, cosNO = dot(f.z, s.wo), cosNI = dot(f.z, wi);
    pdf = 0.0f;
    if (cosNO <= 0.0f || cosNI <= 0.0f) return V3{0, 0, 0};
    V3 m = add(s.wo, wi);
    const float lm = length(m);
    if (!(lm > 0.001f)) return V3{0, 0, 0};
    m = mul(m, 1.0f / lm);
    const float cosMI = dot(m, wi);
    if (cosMI <= 0.0f) return V3{0, 0, 0};
    const float cosThetaM = dot(m, f.z);
    if (cosThetaM <= 0.0f) return V3{0, 0, 0};
    float alpha2 = roughness * roughness;
    const float cosThetaM2 = cosThetaM * cosThetaM, piCosThetaM4 = kPi * cosThetaM2 * cosThetaM2;
    const float tanThetaM2 = (1.0f - cosThetaM2) / cosThetaM2;
    float tmp = alpha2 + tanThetaM2, D4 = 0.25f * alpha2 / (piCosThetaM4 * tmp * tmp);
    const float invCosNO = 1.0f / cosNO, invCosNI = 1.0f / cosNI;
    const float G1o = 2.0f / (1.0f + sqrtf(1.0f + alpha2 * (1.0f - cosNO * cosNO) * (invCosNO * invCosNO)));
    const float G1i = 2.0f / (1.0f + sqrtf(1.0f + alpha2 * (1.0f - cosNI * cosNI) * (invCosNI * invCosNI)));
    const V3 F = mulv(V3{1, 1, 1}, schlick(l.spec, cosMI));
    const V3 fr = mul(mul(mul(mul(mul(F, G1o), G1i), D4), invCosNO), 1.0f);
    const float alpha = (1.2f - 0.2f * sqrtf(cosNO)) * roughness;
    alpha2 = alpha * alpha;
    tmp = alpha2 + tanThetaM2;
    D4 = 0.25f * alpha2 / (piCosThetaM4 * tmp * tmp);
    const float p1 = D4 * cosThetaM / cosMI;
    pdf = (1.0f - 0.0f) * p1 + 0.0f * 0.0f;
    return mul(fr, 1.0f);
}
__device__ __forceinline__ V3 evalLambert(const Lobe& l, V3 wi, float& pdf) {
    const V3 N = l.frame.z;
    const float cosWi = fmaxf(dot(N, wi), 0.0f);
    pdf = cosWi * kOneOverPi;
    return mul(mul(mulv(mul(l.albedo, 1.0f), V3{1, 1, 1}), kOneOverPi), cosWi);
}
__device__ __forceinline__ V3 lobeEval(const Lobe& l, const Slice& s, V3 wi, float& pdf) {
    return l.kind == 0 ? evalLambert(l, wi, pdf) : evalGGX(l, s, wi, pdf);
}
__device__ __forceinline__ V3 lobeSample(const Lobe& l, const Slice& s, float r1, float r2, V3& wi, float& pdf) {
    if (l.kind == 0) {
        const float cosTheta = r1 > 1.0f ? 1.0f : sqrtf(r1), sinTheta = sqrtf(1.0f - r1);
        wi = localToGlobal(l.frame, localSpherical(cosTheta, sinTheta, r2 * kTwoPi));
        return evalLambert(l, wi, pdf);
    }
    const float cosNO = dot(l.frame.z, s.wo);
    if (cosNO <= 0.0f) {
        wi = V3{0, 0, 0};
        pdf = 0.0f;
        return V3{0, 0, 0};
    }
    const float rr = (r1 - 0.0f) / (1.0f - 0.0f);
    const float alpha = (1.2f - 0.2f * sqrtf(cosNO)) * l.roughness, alpha2 = alpha * alpha;
    const float tanThetaM2 = alpha2 * rr / (1.0f - rr), cosThetaM = 1.0f / sqrtf(1.0f + tanThetaM2);
    const float sinThetaM = cosThetaM * sqrtf(tanThetaM2);
    const V3 m = localToGlobal(l.frame, localSpherical(cosThetaM, sinThetaM, 2.0f * kPi * r2));
    const float NdotWo = dot(m, s.wo);
    wi = add(mul(s.wo, -1.0f), mul(m, 2.0f * NdotWo));
    return evalGGX(l, s, wi, pdf);
}

// The same evaluation and sampling in a kernel that knows the lobe's kind (kLobe 1: Lambert, 2: GGX; 0: read from
// the lobe), so that it holds one lobe's code.
template <int kLobe>
__device__ __forceinline__ V3 lobeEvalAs(const Lobe& l, const Slice& s, V3 wi, float& pdf) {
    if (kLobe == 1) return evalLambert(l, wi, pdf);
    if (kLobe == 2) return evalGGX(l, s, wi, pdf);
    return lobeEval(l, s, wi, pdf);
}
template <int kLobe>
__device__ __forceinline__ V3 lobeSampleAs(const Lobe& l, const Slice& s, float r1, float r2, V3& wi, float& pdf) {
    if (kLobe == 0) return lobeSample(l, s, r1, r2, wi, pdf);
    Lobe k = l;
    k.kind = kLobe == 1 ? 0 : 1;
    return lobeSample(k, s, r1, r2, wi, pdf);
}

// ---------------------------------------------------------------------------------------------------------------
// Lights (light_core.h): Rect and constant Env.
struct LightHit {
    V3 N;
    float distance;
};
__device__ __forceinline__ V3 lrow(const float m[3][3], int i) { return V3{m[i][0], m[i][1], m[i][2]}; }
__device__ __forceinline__ V3 rowsMul(const float m[3][3], V3 v) {
    return add(add(mul(lrow(m, 0), v.x), mul(lrow(m, 1), v.y)), mul(lrow(m, 2), v.z));
}
__device__ __forceinline__ V3 lpos(const x2_light& l) { return V3{l.position[0], l.position[1], l.position[2]}; }
__device__ __forceinline__ V3 ldir(const x2_light& l) { return V3{l.direction[0], l.direction[1], l.direction[2]}; }
__device__ __forceinline__ float planeDistance(const x2_light& l, V3 p) {
    float d = dot(ldir(l), p) + l.plane_offset;
    if (l.sidedness == X2_SIDE_REVERSE) d = -d;
    else if (l.sidedness == X2_SIDE_TWO) d = fabsf(d);
    return d;
}
// surface::sincosSample (surface_core.h:127-137): the shared sine/cosine polynomial the lights use.
__device__ __forceinline__ void sincosPoly(float angle, float& sn, float& cs) {
    const float kf = floorf(angle * .6366197466850281f), x = angle - kf * 1.5707963705062866f, x2 = x * x;
    const int k = int(kf) & 3;
    float s = -2.5029327943570934e-8f;
    s = s * x2 + .000002760012648650445f;
    s = s * x2 - .00019842604524455965f;
    s = s * x2 + .008333347737789154f;
    s = s * x2 - .1666666716337204f;
    s = (s * x2 + 1) * x;
    float c = -.0000002596301840185333f;
    c = c * x2 + .000024756234779488295f;
    c = c * x2 - .001388833043165505f;
    c = c * x2 + .04166664183139801f;
    c = c * x2 - .5f;
    c = c * x2 + 1;
    sn = k == 0 ? s : k == 1 ? c : k == 2 ? -s : -c;
    cs = k == 0 ? c : k == 1 ? -s : k == 2 ? -c : s;
}
// lights::sample for Env and Rect (light_core.h:476-501, :523-585).
__device__ __forceinline__ bool lightSample(const x2_light& l, V3 p, const V3* n, const float r[3], V3& wi, LightHit& h) {
    if (l.type == X2_LIGHT_ENV) {
        if (l.hemispherical) {
            const float cosTheta = r[0] > 1.0f ? 1.0f : r[0];
            float s, c;
            sincosPoly(r[1] * kTwoPi, s, c);
            const float sinTheta = sqrtf(1.0f - cosTheta * cosTheta);
            wi = rowsMul(l.local2render, V3{sinTheta * c, sinTheta * s, cosTheta});
        } else {
            const float cosTheta = 1.0f - 2.0f * r[0];
            float s, c;
            sincosPoly(r[1] * kTwoPi, s, c);
            const float sinTheta = sqrtf(fmaxf(0.0f, 1.0f - cosTheta * cosTheta));
            wi = V3{sinTheta * c, sinTheta * s, cosTheta};
        }
        if (n && dot(*n, wi) < kEpsilon) return false;
        h.N = mul(wi, -1);
        h.distance = kEnvDistance;
        return true;
    }
    if (l.type == X2_LIGHT_DISTANT) {
        // A cone about the light's direction, uniform in solid angle (light_core.h:502-522 without an image).
        const float versine = fmaxf(r[0] * l.versine_theta_max, 0.0f);
        const float cosTheta = 1.0f - versine;
        float s, c;
        sincosPoly(r[1] * kTwoPi, s, c);
        const float sinTheta = sqrtf(fmaxf(0.0f, versine * (2.0f - versine)));
        wi = rowsMul(l.local2render, mul(V3{sinTheta * c, sinTheta * s, cosTheta}, -1));
        if (n && dot(*n, wi) < kEpsilon) return false;
        h.N = mul(wi, -1);
        h.distance = kDistantDistance;
        return true;
    }
    const float distance = planeDistance(l, p);
    if (l.sidedness != X2_SIDE_TWO && distance < kEpsilon) return false;
    const V3 local{(0.5f - r[0]) * (2 * l.half_width), (0.5f - r[1]) * (2 * l.half_height), 0.0f};
    wi = sub(add(rowsMul(l.local2render, local), lpos(l)), p);
    h.distance = sqrtf(dot(wi, wi));
    if (h.distance < kEpsilon) return false;
    wi = mul(wi, 1.0f / h.distance);
    if (n && dot(*n, wi) < kEpsilon) return false;
    h.N = dot(ldir(l), wi) < 0.0f ? ldir(l) : mul(ldir(l), -1);
    return true;
}
__device__ __forceinline__ float areaToSolidAngleScale(V3 wi, V3 lightNormal, float dist) {
    const float denom = -dot(wi, lightNormal);
    return denom < 0.00001f ? 0.0f : (dist * dist) / denom;
}
// lights::eval (light_core.h:740-786).
__device__ __forceinline__ V3 lightEval(const x2_light& l, V3 wi, const LightHit& h, float& pdf) {
    const V3 radiance{l.radiance[0] * 1.0f, l.radiance[1] * 1.0f, l.radiance[2] * 1.0f};
    if (l.type == X2_LIGHT_ENV || l.type == X2_LIGHT_DISTANT) {
        pdf = l.inv_area;
        return radiance;
    }
    pdf = l.inv_area;
    pdf *= areaToSolidAngleScale(wi, h.N, h.distance);
    return radiance;
}
// lights::intersect (light_core.h:813-848).
__device__ __forceinline__ bool lightIntersect(const x2_light& l, V3 p, V3 wi, float maxDistance, LightHit& h) {
    if (l.type == X2_LIGHT_ENV) {
        if (l.hemispherical && dot(wi, ldir(l)) < 0.0f) return false;
        if (kEnvDistance > maxDistance) return false;
        h.N = mul(wi, -1);
        h.distance = kEnvDistance;
        return true;
    }
    if (l.type == X2_LIGHT_DISTANT) {
        if (dot(wi, ldir(l)) > -l.cos_theta_max || kDistantDistance > maxDistance) return false;
        h.N = mul(wi, -1);
        h.distance = kDistantDistance;
        return true;
    }
    const V3 localWi = rowsMul(l.render2local_rot, wi), localP = rowsMul(l.render2local, sub(p, lpos(l)));
    if ((localP.z < 0.0f) == (localWi.z < 0.0f)) return false;
    if (localP.z < 0.0f ? l.sidedness == X2_SIDE_REGULAR : l.sidedness == X2_SIDE_REVERSE) return false;
    const float localDistance = -localP.z / localWi.z, renderDistance = l.scale * localDistance;
    if (renderDistance > maxDistance) return false;
    const V3 hit = add(localP, mul(localWi, localDistance));
    if (fabsf(hit.x) >= l.half_width || fabsf(hit.y) >= l.half_height) return false;
    h.N = localWi.z < 0.0f ? ldir(l) : mul(ldir(l), -1);
    h.distance = renderDistance;
    return true;
}
// lights::canIlluminate (light_core.h:1025-1069) with no subsurface radius.
__device__ __forceinline__ bool canIlluminate(const x2_light& l, V3 p, const V3* n) {
    if (l.type == X2_LIGHT_ENV) return true;
    if (l.type == X2_LIGHT_DISTANT) {
        const float cullThreshold = -mf::cos(fminf(mf::acos(fminf(fmaxf(l.cos_theta_max, -1.0f), 1.0f)) + 0.5f * kPi, kPi));
        return !(n && dot(*n, ldir(l)) > cullThreshold);
    }
    const float threshold = kEpsilon - 0.0f;
    if (l.sidedness != X2_SIDE_TWO && planeDistance(l, p) < threshold) return false;
    if (!n) return true;
    const float hx = l.half_width, hy = l.half_height;
    const float c[4][2] = {{hx, hy}, {hx, -hy}, {-hx, hy}, {-hx, -hy}};
    for (int i = 0; i < 4; ++i)
        if (dot(*n, sub(add(rowsMul(l.local2render, V3{c[i][0], c[i][1], 0.0f}), lpos(l)), p)) > threshold) return true;
    return false;
}
__device__ __forceinline__ float powerHeuristic(float f, float g) { return (f * f) / (f * f + g * g); }


}  // namespace x2
