// ORACLE — test infrastructure only. Never linked into, called by or shipped with the product path.
//
// The FP64 CPU adjoint: the path tracer's estimator for the admitted surface scenes (no volumes, bsdf_samples = 1)
// restated in double precision, sample by sample, with the gradients of an image loss with respect to each Lambert
// material's albedo, each GGX material's roughness and each light's radiance accumulated in FP64 — the check of the
// device adjoint (x2_adjoint), which computes the same estimator in FP32 with FP32 atomics into per-block partials.
//
// What is shared with the reference and what is restated:
// - random numbers: the reference's own sampler (sample::draw, paths::Stream, paths::childBranch; sample_stream.h,
//   async_integrator.h:151-176, 281-287), so every random number is the device's, bit for bit;
// - traversal: this oracle's float BVH (the Embree stand-in of ref_backend.cpp) on the double ray rounded to float,
//   and the reference's resume::geometryHit (resume_core.h:17-45) for the hit point and the offset ray origins;
// - the estimator (async_integrator.h:1986-3042 for the admitted materials and lights): camera ray, shading state,
//   UsdPreviewSurface -> one Lambert or Schlick-GGX lobe, light samples of every light with MIS, the BSDF sample with
//   its light hit, bounce-ray reuse, Russian roulette, clamping, camera-visible lights — restated here in double
//   (shade_lobes_eval.h:93-146, 611-664; light_core.h:476-1069; shade_material.h:121-383), decisions included;
// - the credits: the same estimator as the device's (sampling decisions held fixed; d(contribution)/d(param) =
//   contribution / param for radiance and albedo; contribution x dlog f/d(roughness) at the direction a GGX vertex
//   used), summed in double.
// A discrete decision (a roulette draw, a validity test) may go the other way in double than in float on a rare
// sample; the gradients are sums over many samples, which such a sample moves by far less than 1%.
//
// Included by ref_backend.cpp inside its file-local namespace, after its traversal (closest, occluded) and Scene.
#pragma once

namespace adj64 {

struct D3 {
    double x, y, z;
};
inline D3 d3(V3 v) { return D3{v.x, v.y, v.z}; }
inline D3 d3(const float* v) { return D3{v[0], v[1], v[2]}; }
inline V3 f3(D3 v) { return V3{float(v.x), float(v.y), float(v.z)}; }
inline D3 operator+(D3 a, D3 b) { return D3{a.x + b.x, a.y + b.y, a.z + b.z}; }
inline D3 operator-(D3 a, D3 b) { return D3{a.x - b.x, a.y - b.y, a.z - b.z}; }
inline D3 operator*(D3 a, double s) { return D3{a.x * s, a.y * s, a.z * s}; }
inline D3 mulv(D3 a, D3 b) { return D3{a.x * b.x, a.y * b.y, a.z * b.z}; }
inline D3 neg(D3 a) { return D3{-a.x, -a.y, -a.z}; }
inline double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline D3 cross(D3 a, D3 b) { return D3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double len(D3 a) { return std::sqrt(dot(a, a)); }
inline D3 unit(D3 a) { return a * (1.0 / len(a)); }
inline bool finite(D3 a) { return std::isfinite(a.x) && std::isfinite(a.y) && std::isfinite(a.z); }
inline bool zero(D3 a) { return a.x == 0 && a.y == 0 && a.z == 0; }
inline bool black(D3 c) {
    auto z = [](double x) { return std::fabs(x) <= std::fmax(std::fabs(x), 1.0) * 1e-6; };
    return z(c.x) && z(c.y) && z(c.z);
}
inline double luminance(D3 c) { return 0.299 * c.x + 0.587 * c.y + 0.114 * c.z; }

constexpr double kPi = 3.14159265358979323846;
constexpr double kEps = 1e-6;
constexpr float kInfinite = 3.4028234663852886e+38f - 1e32f;
constexpr double kEnvDistance = double(kInfinite * 0.9f), kDistantDistance = double(kInfinite * 0.8f);
constexpr double kHitEpsilonEnd = 1.0 - 1e-3;
constexpr double kFar = double(FLT_MAX);

enum : U32 {
    kReflection = 1u, kTransmission = 2u, kDiffuse = 4u, kGlossy = 16u, kMirror = 64u,
    kAllSurfaceSides = 3u, kAllLobes = 84u, kAllDiffuse = 7u, kAllGlossy = 19u, kAllMirror = 67u, kAllLobeTypes = 87u
};
inline bool matchesFlags(U32 type, U32 flags) { return (type & kAllSurfaceSides & flags) && (type & kAllLobes & flags); }
inline U32 lobeRayMask(U32 t) {
    U32 m = 0;
    if (t & 1u) m |= t & 0x54u;
    if (t & 2u) m |= (t & 0x54u) << 1;
    return m;
}

struct Frame {
    D3 x, y, z;
};
inline Frame frameN(D3 N) {  // Duff et al. 2017 (shade_math.h:138-141)
    const double sign = std::copysign(1.0, N.z), a = -1.0 / (sign + N.z), b = N.x * N.y * a;
    return Frame{D3{1.0 + sign * N.x * N.x * a, sign * b, -sign * N.x}, D3{b, sign + N.y * N.y * a, -N.y}, N};
}
inline D3 toWorld(const Frame& f, D3 v) { return f.x * v.x + f.y * v.y + f.z * v.z; }

// The scene as this restatement reads it (the engine's own descriptor records, copied at open).
struct Texture64 {
    U32 width, height, wrap;
    U64 first;  // its first texel among all textures' (for the texel gradients)
    std::vector<float> rgb;
};
struct Scene64 {
    std::vector<x2_material> materials;
    std::vector<U32> meshMaterial;
    std::vector<x2_light> lights;
    x2_camera camera{};
    x2_config config{};
    std::vector<float> uvs;  // 2 a vertex, or empty
    std::vector<Texture64> textures;
    U64 texels = 0;
};

// UsdUVTexture's zero-footprint lookup (texture_core.h lookup at (s, 1 - t), level 0): bilinear on a primary path,
// else the closest texel; in double. Its texels (global indices) and weights go to idx / wt (4 each).
inline int texAddress(long long x, long long n, U32 wrap) {
    if (wrap) {
        const long long v = x % n;
        return int(v < 0 ? v + n : v);
    }
    return int(x < 0 ? 0 : x >= n ? n - 1 : x);
}
inline bool texLookup(const Texture64& t, double s, double tt, bool primary, D3& out, U64 idx[4], double wt[4]) {
    double u = s, v = 1.0 - tt;
    if (!std::isfinite(u) || !std::isfinite(v)) return false;
    if (std::fabs(u) > 1024) u = t.wrap ? u - std::floor(u) : std::fmin(std::fmax(u, -1.0), 2.0);
    if (std::fabs(v) > 1024) v = t.wrap ? v - std::floor(v) : std::fmin(std::fmax(v, -1.0), 2.0);
    double fx = u * t.width - 0.5, fy = v * t.height - 0.5;
    long long x = (long long)std::floor(fx), y = (long long)std::floor(fy);
    auto at = [&](long long xx, long long yy) {
        return U64(texAddress(yy, t.height, t.wrap)) * t.width + U64(texAddress(xx, t.width, t.wrap));
    };
    auto texel = [&](U64 i) { return D3{t.rgb[3 * i], t.rgb[3 * i + 1], t.rgb[3 * i + 2]}; };
    if (primary) {
        fx -= double(x);
        fy -= double(y);
        idx[0] = at(x, y);
        idx[1] = at(x + 1, y);
        idx[2] = at(x, y + 1);
        idx[3] = at(x + 1, y + 1);
        wt[0] = (1 - fx) * (1 - fy);
        wt[1] = fx * (1 - fy);
        wt[2] = (1 - fx) * fy;
        wt[3] = fx * fy;
    } else {
        if (fx - double(x) > 0.5) ++x;
        if (fy - double(y) > 0.5) ++y;
        idx[0] = idx[1] = idx[2] = idx[3] = at(x, y);
        wt[0] = 1;
        wt[1] = wt[2] = wt[3] = 0;
    }
    out = D3{0, 0, 0};
    for (int k = 0; k < 4; ++k) out = out + texel(idx[k]) * wt[k];
    for (int k = 0; k < 4; ++k) idx[k] += t.first;
    return finite(out);
}

struct Lobe {
    int kind = -1;  // -1 none, 0 Lambert, 1 GGX
    U32 type = 0;
    Frame frame{};
    D3 albedo{}, spec{};
    double alpha = 1.0;      // GGX: max(0.001, r^2)
    double roughness = 0.0;  // the material's roughness parameter r
};

struct State {
    D3 P, Ng, N, wo, dPds;
};

// ---- lobes (shade_lobes_eval.h) ----
inline D3 schlick(D3 a, double hDotWi) {
    const double t = 1.0 - hDotWi, p = t * t * t * t * t;
    return a + (D3{1, 1, 1} - a) * p;
}
inline D3 evalGGX(const Lobe& l, D3 wo, D3 wi, double& pdf) {
    const D3 n = l.frame.z;
    const double cosNO = dot(n, wo), cosNI = dot(n, wi);
    pdf = 0;
    if (cosNO <= 0 || cosNI <= 0) return D3{0, 0, 0};
    D3 m = wo + wi;
    const double lm = len(m);
    if (!(lm > 0.001)) return D3{0, 0, 0};
    m = m * (1.0 / lm);
    const double cosMI = dot(m, wi);
    if (cosMI <= 0) return D3{0, 0, 0};
    const double cosThetaM = dot(m, n);
    if (cosThetaM <= 0) return D3{0, 0, 0};
    const double a2 = l.alpha * l.alpha, c2 = cosThetaM * cosThetaM, tan2 = (1 - c2) / c2;
    double t = a2 + tan2;
    const double D4 = 0.25 * a2 / (kPi * c2 * c2 * t * t);
    const double G1o = 2 / (1 + std::sqrt(1 + a2 * (1 - cosNO * cosNO) / (cosNO * cosNO)));
    const double G1i = 2 / (1 + std::sqrt(1 + a2 * (1 - cosNI * cosNI) / (cosNI * cosNI)));
    const D3 f = schlick(l.spec, cosMI) * (G1o * G1i * D4 / cosNO);
    const double aw = (1.2 - 0.2 * std::sqrt(cosNO)) * l.alpha, aw2 = aw * aw;
    t = aw2 + tan2;
    pdf = 0.25 * aw2 / (kPi * c2 * c2 * t * t) * cosThetaM / cosMI;
    return f;
}
// d log f / d r of the GGX lobe at (wo, wi) (0 where f is 0 or the roughness is clamped).
inline double ggxLogDerivative(const Lobe& l, D3 wo, D3 wi) {
    const double r = l.roughness;
    if (!(r > 0 && r < 1) || r * r <= 0.001) return 0;
    const D3 n = l.frame.z;
    const double cosNO = dot(n, wo), cosNI = dot(n, wi);
    if (cosNO <= 0 || cosNI <= 0) return 0;
    D3 m = wo + wi;
    const double lm = len(m);
    if (!(lm > 0.001)) return 0;
    m = m * (1.0 / lm);
    const double cosThetaM = dot(m, n);
    if (cosThetaM <= 0 || dot(m, wi) <= 0) return 0;
    // tan^2 as |x cross n|^2 / (x . n)^2: exact near the normal, where 1 - cos^2 cancels.
    auto tan2 = [&](D3 x, double c) {
        const D3 k = cross(x, n);
        return dot(k, k) / (c * c);
    };
    const double a = l.alpha, a2 = a * a, T = tan2(m, cosThetaM);
    const double to = tan2(wo, cosNO), ti = tan2(wi, cosNI);
    const double so = std::sqrt(1 + a2 * to), si = std::sqrt(1 + a2 * ti);
    return (2 / a - 4 * a / (a2 + T) - a * to / (so * (1 + so)) - a * ti / (si * (1 + si))) * 2 * r;
}
inline D3 evalLambert(const Lobe& l, D3 wi, double& pdf) {
    const double c = std::fmax(dot(l.frame.z, wi), 0.0);
    pdf = c / kPi;
    return l.albedo * (c / kPi);
}
inline D3 lobeEval(const Lobe& l, D3 wo, D3 wi, double& pdf) { return l.kind == 0 ? evalLambert(l, wi, pdf) : evalGGX(l, wo, wi, pdf); }
inline D3 lobeSample(const Lobe& l, D3 wo, double r1, double r2, D3& wi, double& pdf) {
    if (l.kind == 0) {
        const double ct = r1 > 1 ? 1 : std::sqrt(r1), st = std::sqrt(1 - r1), phi = r2 * 2 * kPi;
        wi = toWorld(l.frame, D3{st * std::cos(phi), st * std::sin(phi), ct});
        return evalLambert(l, wi, pdf);
    }
    const double cosNO = dot(l.frame.z, wo);
    if (cosNO <= 0) {
        wi = D3{0, 0, 0};
        pdf = 0;
        return D3{0, 0, 0};
    }
    const double aw = (1.2 - 0.2 * std::sqrt(cosNO)) * l.alpha, aw2 = aw * aw;
    const double tan2 = aw2 * r1 / (1 - r1), cm = 1 / std::sqrt(1 + tan2), sm = cm * std::sqrt(tan2), phi = 2 * kPi * r2;
    const D3 m = toWorld(l.frame, D3{sm * std::cos(phi), sm * std::sin(phi), cm});
    wi = neg(wo) + m * (2 * dot(m, wo));
    return evalGGX(l, wo, wi, pdf);
}

// ---- lights (light_core.h) ----
struct LightHit {
    D3 N;
    double distance;
};
inline D3 rows(const float m[3][3], D3 v) { return d3(m[0]) * v.x + d3(m[1]) * v.y + d3(m[2]) * v.z; }
inline double planeDistance(const x2_light& l, D3 p) {
    double d = dot(d3(l.direction), p) + l.plane_offset;
    if (l.sidedness == X2_SIDE_REVERSE) d = -d;
    else if (l.sidedness == X2_SIDE_TWO) d = std::fabs(d);
    return d;
}
inline bool lightSample(const x2_light& l, D3 p, const D3* n, const double r[3], D3& wi, LightHit& h) {
    if (l.type == X2_LIGHT_ENV) {
        if (l.hemispherical) {
            const double ct = r[0] > 1 ? 1 : r[0], st = std::sqrt(1 - ct * ct), phi = r[1] * 2 * kPi;
            wi = rows(l.local2render, D3{st * std::cos(phi), st * std::sin(phi), ct});
        } else {
            const double ct = 1 - 2 * r[0], st = std::sqrt(std::fmax(0.0, 1 - ct * ct)), phi = r[1] * 2 * kPi;
            wi = D3{st * std::cos(phi), st * std::sin(phi), ct};
        }
        if (n && dot(*n, wi) < kEps) return false;
        h.N = neg(wi);
        h.distance = kEnvDistance;
        return true;
    }
    if (l.type == X2_LIGHT_DISTANT) {
        const double v = std::fmax(r[0] * l.versine_theta_max, 0.0), ct = 1 - v, st = std::sqrt(std::fmax(0.0, v * (2 - v)));
        const double phi = r[1] * 2 * kPi;
        wi = rows(l.local2render, neg(D3{st * std::cos(phi), st * std::sin(phi), ct}));
        if (n && dot(*n, wi) < kEps) return false;
        h.N = neg(wi);
        h.distance = kDistantDistance;
        return true;
    }
    const double distance = planeDistance(l, p);
    if (l.sidedness != X2_SIDE_TWO && distance < kEps) return false;
    const D3 local{(0.5 - r[0]) * (2.0 * l.half_width), (0.5 - r[1]) * (2.0 * l.half_height), 0};
    wi = rows(l.local2render, local) + d3(l.position) - p;
    h.distance = len(wi);
    if (h.distance < kEps) return false;
    wi = wi * (1.0 / h.distance);
    if (n && dot(*n, wi) < kEps) return false;
    h.N = dot(d3(l.direction), wi) < 0 ? d3(l.direction) : neg(d3(l.direction));
    return true;
}
inline D3 lightEval(const x2_light& l, D3 wi, const LightHit& h, double& pdf) {
    pdf = l.inv_area;
    if (l.type == X2_LIGHT_RECT) {
        const double denom = -dot(wi, h.N);
        pdf *= denom < 0.00001 ? 0.0 : h.distance * h.distance / denom;
    }
    return d3(l.radiance);
}
inline bool lightIntersect(const x2_light& l, D3 p, D3 wi, double maxDistance, LightHit& h) {
    if (l.type == X2_LIGHT_ENV) {
        if (l.hemispherical && dot(wi, d3(l.direction)) < 0) return false;
        if (kEnvDistance > maxDistance) return false;
        h.N = neg(wi);
        h.distance = kEnvDistance;
        return true;
    }
    if (l.type == X2_LIGHT_DISTANT) {
        if (dot(wi, d3(l.direction)) > -double(l.cos_theta_max) || kDistantDistance > maxDistance) return false;
        h.N = neg(wi);
        h.distance = kDistantDistance;
        return true;
    }
    const D3 lw = rows(l.render2local_rot, wi), lp = rows(l.render2local, p - d3(l.position));
    if ((lp.z < 0) == (lw.z < 0)) return false;
    if (lp.z < 0 ? l.sidedness == X2_SIDE_REGULAR : l.sidedness == X2_SIDE_REVERSE) return false;
    const double ld = -lp.z / lw.z, rd = l.scale * ld;
    if (rd > maxDistance) return false;
    const D3 hit = lp + lw * ld;
    if (std::fabs(hit.x) >= l.half_width || std::fabs(hit.y) >= l.half_height) return false;
    h.N = lw.z < 0 ? d3(l.direction) : neg(d3(l.direction));
    h.distance = rd;
    return true;
}
inline bool canIlluminate(const x2_light& l, D3 p, const D3* n) {
    if (l.type == X2_LIGHT_ENV) return true;
    if (l.type == X2_LIGHT_DISTANT) {
        const double ct = std::fmin(std::fmax(double(l.cos_theta_max), -1.0), 1.0);
        const double cull = -std::cos(std::fmin(std::acos(ct) + 0.5 * kPi, kPi));
        return !(n && dot(*n, d3(l.direction)) > cull);
    }
    if (l.sidedness != X2_SIDE_TWO && planeDistance(l, p) < kEps) return false;
    if (!n) return true;
    const double hx = l.half_width, hy = l.half_height, c[4][2] = {{hx, hy}, {hx, -hy}, {-hx, hy}, {-hx, -hy}};
    for (int i = 0; i < 4; ++i)
        if (dot(*n, rows(l.local2render, D3{c[i][0], c[i][1], 0}) + d3(l.position) - p) > kEps) return true;
    return false;
}
inline double powerHeuristic(double f, double g) { return f * f / (f * f + g * g); }
inline bool roulette(double lum, double threshold, double u, double& scale) {
    scale = 1;
    if (lum >= threshold) return true;
    if (lum < u * threshold) return false;
    scale = threshold / lum;
    return true;
}

// ---- one sample ----
struct Pending {
    D3 origin, dir, T;
    U64 branch;
    U32 depth, nonMirror, diffuse, glossy, mirror;
    double nearT, farT;
    U32 heldLight;
    double heldFar;
    D3 held;
};

// Gradients of one thread (FP64): 3 a material's albedo, 1 a material's roughness, 3 a light's radiance; and each
// gradient's mass, the sum of its credits' magnitudes (a gradient much smaller than its mass is a near-cancelling sum,
// whose value the last bits of every credit move: its conditioning).
struct Grads {
    std::vector<double> albedo, roughness, radiance;
    std::vector<double> albedoMass, roughnessMass, radianceMass;
    std::vector<double> texture;  // 3 a texel (empty: not wanted)
};

struct Tracer {
    const Scene& s;
    const Scene64& x;
    Grads& g;
    D3 delta;  // dL/dI of the pixel over its samples

    xi::resume::Hit trace(D3 o, D3 d, double nearT, double farT, U32& tri) const {
        xi::resume::Hit out;
        xi::surface::Ray ray{};
        ray.origin = f3(o);
        ray.direction = f3(d);
        ray.nearT = float(nearT);
        ray.farT = float(farT);
        float t;
        tri = closest(s, ray.origin, ray.direction, ray.nearT, ray.farT, t);
        if (tri == ~0u) return out;
        out.geom = s.triGeom[tri];
        out.prim = tri - s.meshFirst[out.geom];
        out.t = t;
        if (!xi::resume::geometryHit(out, ray, s.vertex(s.tris[3 * tri]), s.vertex(s.tris[3 * tri + 1]), s.vertex(s.tris[3 * tri + 2])))
            out.normal = {};
        return out;
    }
    bool visible(D3 o, D3 d, double near, double far) const { return !occluded(s, f3(o), f3(d), float(near), float(far)); }

    void creditLight(D3 c, U32 j) {
        if (j == ~0u) return;
        const x2_light& L = x.lights[j];
        const double w[3] = {delta.x * c.x, delta.y * c.y, delta.z * c.z};
        for (int k = 0; k < 3; ++k)
            if (L.radiance[k] != 0.0f && w[k] != 0.0) {
                g.radiance[3 * j + k] += w[k] / L.radiance[k];
                g.radianceMass[3 * j + k] += std::fabs(w[k] / L.radiance[k]);
            }
    }
    void creditRoughness(U32 m, D3 c, double gl) {
        const double v = (delta.x * c.x + delta.y * c.y + delta.z * c.z) * gl;
        g.roughness[m] += v;
        g.roughnessMass[m] += std::fabs(v);
    }
    void creditAlbedo(U32 m, int k, double v) {
        g.albedo[3 * m + k] += v;
        g.albedoMass[3 * m + k] += std::fabs(v);
    }

    // visibleLightRadiance (async_integrator.h:383-412): the light a camera ray sees, one chosen uniformly.
    D3 visibleLights(const xi::sample::Identity& root, D3 origin, D3 dir, double maxDistance, U32& which) const {
        const x2_config& c = x.config;
        which = ~0u;
        U32 hits = 0;
        for (U32 pass = 0; pass < 3; ++pass)
            for (U32 j = 0; j < c.light_count; ++j) {
                const x2_light& L = x.lights[j];
                LightHit lh;
                const U32 vp = L.type == X2_LIGHT_ENV ? 2u : L.type == X2_LIGHT_DISTANT ? 1u : 0u;
                if (L.visible_in_camera && vp == pass && lightIntersect(L, origin, dir, maxDistance, lh)) ++hits;
            }
        if (!hits) return D3{0, 0, 0};
        xi::sample::Identity id = root;
        id.branch = xi::async::paths::childBranch(0x5649534c49474854ull, 0, 0);
        xi::async::paths::Stream st(id, 0, 0);
        const double choice = st.next();
        const U32 chosen = U32(choice * hits) < hits ? U32(choice * hits) : hits - 1;
        U32 seen = 0;
        for (U32 pass = 0; pass < 3; ++pass)
            for (U32 j = 0; j < c.light_count; ++j) {
                const x2_light& L = x.lights[j];
                LightHit lh;
                const U32 vp = L.type == X2_LIGHT_ENV ? 2u : L.type == X2_LIGHT_DISTANT ? 1u : 0u;
                if (!L.visible_in_camera || vp != pass || !lightIntersect(L, origin, dir, maxDistance, lh)) continue;
                if (seen++ != chosen) continue;
                double pdf;
                const D3 Li = lightEval(L, dir, lh, pdf);
                which = j;
                return finite(Li) ? Li * double(hits) : D3{0, 0, 0};
            }
        return D3{0, 0, 0};
    }

    // integratePaths for one sample in double, crediting as it goes; returns its radiance (rgb).
    D3 sample(U32 pixel, U32 index) {
        const x2_config& c = x.config;
        const x2_camera& cam = x.camera;
        const xi::sample::Identity root{pixel, U64(index), U64(c.seed), 0};
        const double fx = (double(xi::sample::draw(root, 0, c.sampling)) - 0.5) * c.filter_width + 0.5;
        const double fy = (double(xi::sample::draw(root, 1, c.sampling)) - 0.5) * c.filter_width + 0.5;
        // perspectiveRay without depth of field (camera_core.h:217-263), in double.
        const double rx = double(pixel % c.width) + fx, ry = double(pixel / c.width) + fy, rz = -1.0;
        const auto& m = cam.raster_to_camera;
        const D3 v{rx * m[0][0] + ry * m[1][0] + rz * m[2][0] + m[3][0], rx * m[0][1] + ry * m[1][1] + rz * m[2][1] + m[3][1],
                   rx * m[0][2] + ry * m[1][2] + rz * m[2][2] + m[3][2]};
        const double w = rx * m[0][3] + ry * m[1][3] + rz * m[2][3] + m[3][3];
        const D3 dirCam = v * (1.0 / w);
        const D3 n = unit(dirCam);
        const auto& q = cam.camera_to_render;
        const D3 origin{q[3][0], q[3][1], q[3][2]};
        const D3 dir = unit(D3{dirCam.x * q[0][0] + dirCam.y * q[1][0] + dirCam.z * q[2][0], dirCam.x * q[0][1] + dirCam.y * q[1][1] + dirCam.z * q[2][1],
                               dirCam.x * q[0][2] + dirCam.y * q[1][2] + dirCam.z * q[2][2]});
        Pending stack[32];
        U32 top = 0;
        Pending p0{};
        p0.origin = origin;
        p0.dir = dir;
        p0.T = D3{1, 1, 1};
        p0.nearT = -double(cam.near_clip) / n.z;
        p0.farT = -double(cam.far_clip) / n.z;
        p0.heldLight = ~0u;
        stack[top++] = p0;
        D3 radiance{0, 0, 0};
        // The path's vertices by depth: material (~0u none), kind, radiance before it acted, scale; a textured
        // Lambert vertex's texel value, texels and weights.
        U32 vm[128];
        int vk[128];
        D3 before[128], scale[128], texelAt[128];
        bool textured[128];
        U64 texIdx[128][4];
        double texWt[128][4];
        U32 vertices = 0;
        while (top) {
            Pending pv = stack[--top];
            if (pv.depth >= 128) continue;
            U32 tri;
            const xi::resume::Hit hit = trace(pv.origin, pv.dir, pv.nearT, pv.farT, tri);
            const bool missed = hit.geom == ~0u;
            if (pv.heldLight != ~0u && !(!missed && double(hit.t) < pv.heldFar)) {
                radiance = radiance + pv.held;
                creditLight(pv.held, pv.heldLight);
            }
            if (pv.depth == 0 && c.visible_lights) {
                U32 which;
                const D3 Lv = mulv(pv.T, visibleLights(root, missed ? pv.origin : origin, pv.dir, missed ? double(FLT_MAX) : double(hit.t), which));
                radiance = radiance + Lv;
                creditLight(Lv, which);
            }
            if (missed) continue;
            // Shading state (hitState for a mesh without normals or texture coordinates), in double.
            const D3 a = d3(s.vertex(s.tris[3 * tri])), b = d3(s.vertex(s.tris[3 * tri + 1])), cc = d3(s.vertex(s.tris[3 * tri + 2]));
            State st;
            const D3 ng = cross(b - a, cc - a);
            if (!(len(ng) > 0)) return radiance;
            st.Ng = unit(ng);
            st.dPds = b - a;
            st.P = d3(hit.point);
            st.wo = neg(pv.dir);
            if (!(dot(st.Ng, pv.dir) < 0)) st.Ng = neg(st.Ng);
            st.N = st.Ng;
            // UsdPreviewSurface, specular workflow: one lobe.
            const U32 mat = x.meshMaterial[hit.geom];
            const x2_material& M = x.materials[mat];
            Lobe lobe;
            const D3 emission = d3(M.emission);
            // A textured diffuse colour: the lookup at the hit's st (w st1 + u st2 + v st3 of the vertices' uvs).
            D3 diffuse = d3(M.diffuse), texel{1, 1, 1};
            U64 tidx[4] = {0, 0, 0, 0};
            double twt[4] = {0, 0, 0, 0};
            bool isTextured = false;
            if (M.diffuse_texture) {
                const double hu = hit.u, hv = hit.v, w = 1.0 - hu - hv;
                double uv[6] = {0, 0, 1, 0, 1, 1};
                if (!x.uvs.empty())
                    for (int k = 0; k < 3; ++k) {
                        uv[2 * k] = x.uvs[2 * size_t(s.tris[3 * tri + k])];
                        uv[2 * k + 1] = x.uvs[2 * size_t(s.tris[3 * tri + k]) + 1];
                    }
                const double ss = w * uv[0] + hu * uv[2] + hv * uv[4], tt = w * uv[1] + hu * uv[3] + hv * uv[5];
                const bool primary = pv.diffuse == 0 && pv.glossy == 0 && pv.mirror == 0;
                if (!texLookup(x.textures[M.diffuse_texture - 1], ss, tt, primary, texel, tidx, twt)) return radiance;
                if (!black(diffuse)) {
                    diffuse = mulv(diffuse, texel);
                    isTextured = true;
                }
            }
            if (!black(emission)) radiance = radiance + mulv(pv.T, emission);
            const double r = std::fmin(std::fmax(double(M.roughness), 0.0), 1.0);
            const D3 spec{std::fmin(std::fmax(double(M.specular[0]), 0.0), 1.0), std::fmin(std::fmax(double(M.specular[1]), 0.0), 1.0),
                          std::fmin(std::fmax(double(M.specular[2]), 0.0), 1.0)};
            if (M.kind == X2_MAT_GGX && !black(spec)) {
                // Intersection_adaptNormal (shade_state.h:256-264) of the shading normal.
                D3 Na = st.N;
                const D3 rr = st.N * (2 * dot(st.N, st.wo)) - st.wo;
                const double rDotNg = dot(rr, st.Ng);
                if (rDotNg < 0.001) Na = unit(st.wo + unit(rr + st.Ng * (0.001 - rDotNg)));
                lobe.kind = 1;
                lobe.type = kReflection | kGlossy;
                lobe.frame = frameN(Na);
                lobe.spec = spec;
                lobe.alpha = std::fmax(0.001, r * r);
                lobe.roughness = M.roughness;
            } else if (!black(diffuse)) {
                lobe.kind = 0;
                lobe.type = kReflection | kDiffuse;
                lobe.frame = frameN(st.N);
                lobe.albedo = diffuse;
            }
            const U32 k = pv.depth;
            vertices = k + 1;
            before[k] = radiance;
            vm[k] = lobe.kind >= 0 ? mat : ~0u;
            vk[k] = lobe.kind;
            scale[k] = D3{0, 0, 0};
            textured[k] = lobe.kind == 0 && isTextured;
            texelAt[k] = texel;
            for (int i = 0; i < 4; ++i) {
                texIdx[k][i] = tidx[i];
                texWt[k][i] = twt[i];
            }
            if (lobe.kind == 0)
                scale[k] = D3{lobe.albedo.x != 0 ? 1 / lobe.albedo.x : 0, lobe.albedo.y != 0 ? 1 / lobe.albedo.y : 0,
                              lobe.albedo.z != 0 ? 1 / lobe.albedo.z : 0};
            if (lobe.kind < 0) continue;

            U32 indirectFlags = 0;
            if (c.bsdf_samples > 0 && c.max_depth > 0 && pv.depth < c.max_depth) {
                if (pv.diffuse < c.max_diffuse_depth) indirectFlags |= kAllDiffuse;
                if (pv.glossy < c.max_glossy_depth) indirectFlags |= kAllGlossy;
                if (pv.mirror < c.max_mirror_depth) indirectFlags |= kAllMirror;
                if (0u < c.max_hair_depth) indirectFlags |= kAllSurfaceSides;
            }
            const bool doIndirect = indirectFlags != 0;
            const D3 cull = st.Ng;  // a reflection lobe culls lights behind the geometric normal
            const D3* cullN = &cull;
            const bool split = pv.nonMirror == 0;
            const U32 nl = split ? c.light_samples : 1;
            const bool clampHere = pv.nonMirror >= c.clamp_depth;
            const bool rr = pv.nonMirror > 0 && c.rr_threshold > 0;
            const U32 nk = 1;
            const D3 above = d3(hit.origin), below = d3(hit.below);
            auto surfaceFlags = [&](D3 wi) {
                return dot(st.Ng, st.wo) * dot(st.Ng, wi) > 0 ? (kAllLobeTypes & ~kTransmission) : (kAllLobeTypes & ~kReflection);
            };

            // Light samples of every light that can light the hit.
            const U64 lightBranch = xi::async::paths::childBranch(pv.branch, 0xfffe, 0);
            for (U32 i = 0; i < c.light_count; ++i) {
                const x2_light& L = x.lights[i];
                if (!canIlluminate(L, st.P, cullN)) continue;
                const U64 lightAddress = xi::async::paths::childBranch(lightBranch, i, 0);
                xi::sample::Identity lid = root;
                lid.branch = lightAddress;
                xi::async::paths::Stream ls(lid, pv.depth, 0);
                for (U32 si = 0; si < nl; ++si) {
                    double rv[3];
                    rv[0] = ls.next();
                    rv[1] = ls.next();
                    rv[2] = ls.next();
                    const double u = ls.next();
                    if (split) {
                        const xi::sample::Identity strat{pixel, U64(index) * nl + si, U64(c.seed), lightAddress};
                        rv[0] = xi::sample::draw(strat, xi::sample::CameraDimensions + 2, c.sampling);
                        rv[1] = xi::sample::draw(strat, xi::sample::CameraDimensions + 3, c.sampling);
                    }
                    D3 wi;
                    LightHit lh;
                    if (!lightSample(L, st.P, cullN, rv, wi, lh)) continue;
                    double pdfL;
                    const D3 Li = lightEval(L, wi, lh, pdfL);
                    if (pdfL == 0 || zero(Li) || !(std::fabs(pdfL) < 3.4e38) || !finite(Li)) continue;
                    const D3 factor = mulv(pv.T, Li) * (1.0 / (double(nl) * pdfL));
                    if (!(matchesFlags(lobe.type, surfaceFlags(wi)) && (lobeRayMask(lobe.type) & L.visibility_mask))) continue;
                    double pdf;
                    const D3 f = lobeEval(lobe, st.wo, wi, pdf);
                    if (pdf == 0 || zero(f)) continue;
                    D3 t = mulv(factor, f) * powerHeuristic(double(nl) * pdfL, double(nk) * pdf);
                    if (clampHere && c.clamp_value > 0) {
                        const double mx = std::fmax(t.x, std::fmax(t.y, t.z));
                        if (mx > c.clamp_value) t = t * (c.clamp_value / mx);
                    }
                    if (rr) {
                        double sc;
                        if (!roulette(luminance(t), c.rr_threshold, u, sc)) continue;
                        t = t * sc;
                    }
                    if (!finite(t) || zero(t)) continue;
                    const D3 o = dot(wi, st.Ng) >= 0 ? above : below;
                    const double far = std::fmax(lh.distance * kHitEpsilonEnd, 0.0);
                    if (!visible(o, wi, 0.0, far)) continue;
                    radiance = radiance + t;
                    creditLight(t, i);
                    if (lobe.kind == 1) {
                        creditRoughness(mat, t, ggxLogDerivative(lobe, st.wo, wi));
                        before[k] = radiance;
                    }
                }
            }

            // The lobe's BSDF sample.
            const U32 lobeMask = lobeRayMask(lobe.type);
            const bool lobeIndirect = matchesFlags(lobe.type, indirectFlags);
            const U64 lobeBranch = xi::async::paths::childBranch(pv.branch, 0, 0xffff);
            const U64 sampleBranch = xi::async::paths::childBranch(lobeBranch, 0, 0);
            xi::sample::Identity bid = root;
            bid.branch = sampleBranch;
            xi::async::paths::Stream bs(bid, pv.depth, 0);
            double r1 = bs.next(), r2 = bs.next();
            const double choice = bs.next(), u = bs.next();
            if (split) {
                const xi::sample::Identity strat{pixel, U64(index) * nk, U64(c.seed), lobeBranch};
                r1 = xi::sample::draw(strat, xi::sample::CameraDimensions, c.sampling);
                r2 = xi::sample::draw(strat, xi::sample::CameraDimensions + 1, c.sampling);
            }
            D3 wi;
            double pdf;
            const D3 f = lobeSample(lobe, st.wo, r1, r2, wi, pdf);
            if (pdf == 0 || zero(f) || !finite(f) || !finite(wi)) continue;
            if (!matchesFlags(lobe.type, surfaceFlags(wi))) continue;
            if (lobe.kind == 1) scale[k] = D3{ggxLogDerivative(lobe, st.wo, wi), 0, 0};
            const D3 pt = mulv(pv.T, f) * (1.0 / (double(nk) * pdf));
            U32 hits = 0;
            for (U32 j = 0; j < c.light_count; ++j) {
                LightHit lh;
                if ((lobeMask & x.lights[j].visibility_mask) && lightIntersect(x.lights[j], st.P, wi, double(FLT_MAX), lh)) ++hits;
            }
            D3 direct{0, 0, 0};
            double lightDistance = 0;
            bool lightHit = false;
            U32 lightIndex = 0;
            if (hits) {
                const U32 chosen = U32(choice * hits) < hits ? U32(choice * hits) : hits - 1;
                for (U32 j = 0, seen = 0; j < c.light_count; ++j) {
                    LightHit lh;
                    if (!(lobeMask & x.lights[j].visibility_mask) || !lightIntersect(x.lights[j], st.P, wi, double(FLT_MAX), lh)) continue;
                    if (seen++ != chosen) continue;
                    double pdfL;
                    const D3 Li = lightEval(x.lights[j], wi, lh, pdfL) * double(hits);
                    if (!(pdfL == 0 || zero(Li)) && std::fabs(pdfL) < 3.4e38 && finite(Li)) {
                        direct = mulv(Li, pt) * powerHeuristic(double(nk) * pdf, double(nl) * pdfL);
                        lightDistance = lh.distance;
                        lightHit = true;
                        lightIndex = j;
                    }
                    break;
                }
            }
            if (!lightHit && !doIndirect) continue;
            if (clampHere && c.clamp_value > 0) {
                const double mx = std::fmax(direct.x, std::fmax(direct.y, direct.z));
                if (mx > c.clamp_value) direct = direct * (c.clamp_value / mx);
            }
            D3 indirect = doIndirect ? pt : D3{0, 0, 0};
            if (rr) {
                double sc;
                if (!roulette(std::fmax(luminance(direct), luminance(indirect)), c.rr_threshold, u, sc)) continue;
                direct = direct * sc;
                indirect = indirect * sc;
            }
            const D3 o = dot(wi, st.Ng) >= 0 ? above : below;
            const bool bounces = lobeIndirect && !zero(indirect) && finite(indirect);
            bool held = false;
            double shadowFar = 0;
            if (lightHit && !black(direct) && finite(direct)) {
                shadowFar = std::fmax(lightDistance * kHitEpsilonEnd, 0.0);
                held = bounces && top + 16 < 32 && lobeMask && (c.shadow_reuse & lobeMask) == lobeMask;
                if (!held && visible(o, wi, 0.0, shadowFar)) {
                    radiance = radiance + direct;
                    creditLight(direct, lightIndex);
                }
            }
            if (!bounces) continue;
            Pending child{};
            child.origin = o;
            child.dir = wi;
            child.T = indirect;
            child.branch = sampleBranch;
            child.depth = pv.depth + 1;
            child.diffuse = pv.diffuse + ((lobe.type & kDiffuse) ? 1 : 0);
            child.glossy = pv.glossy + ((lobe.type & kGlossy) ? 1 : 0);
            child.mirror = pv.mirror;
            child.nonMirror = pv.nonMirror + 1;
            child.nearT = 0;
            child.farT = kFar;
            child.heldLight = held ? lightIndex : ~0u;
            child.heldFar = held ? shadowFar : 0;
            child.held = held ? direct : D3{0, 0, 0};
            stack[top++] = child;
        }
        // Suffix credits: each vertex once, with what the path gathered after it acted.
        for (U32 k = 0; k < vertices; ++k) {
            if (vm[k] == ~0u) continue;
            const D3 after = radiance - before[k];
            if (vk[k] == 1) {
                creditRoughness(vm[k], after, scale[k].x);
            } else {
                // d albedo / d diffuse: the texel (1 untextured); d albedo / d texel: diffuse x the texel's weight.
                const double w[3] = {delta.x * after.x * scale[k].x, delta.y * after.y * scale[k].y, delta.z * after.z * scale[k].z};
                const double tv[3] = {texelAt[k].x, texelAt[k].y, texelAt[k].z};
                const x2_material& M = x.materials[vm[k]];
                for (int c = 0; c < 3; ++c) {
                    creditAlbedo(vm[k], c, w[c] * (textured[k] ? tv[c] : 1.0));
                    if (textured[k] && !g.texture.empty())
                        for (int i = 0; i < 4; ++i)
                            if (texWt[k][i] != 0) g.texture[3 * texIdx[k][i] + c] += w[c] * M.diffuse[c] * texWt[k][i];
                }
            }
        }
        return radiance;
    }
};

}  // namespace adj64
