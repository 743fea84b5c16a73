// The adjoint's shared pieces (adjoint.cu's replay and wavefront.cu's adjoint form): where a block's partial
// gradients sit, and the GGX lobe's log-derivative with respect to its material's roughness.
#pragma once
#include "integrator.cuh"

namespace x2 {

// Where a block's partial gradients sit in its shared memory (and a gradient row): albedo (3 a material), roughness
// (1 a material), radiance (3 a light).
struct Layout {
    uint32_t materials, lights;
    __device__ uint32_t albedo(uint32_t m) const { return 3 * m; }
    __device__ uint32_t roughness(uint32_t m) const { return 3 * materials + m; }
    __device__ uint32_t radiance(uint32_t j) const { return 4 * materials + 3 * j; }
    __device__ uint32_t count() const { return 4 * materials + 3 * lights; }
};

// d log f / d(material roughness) of the GGX lobe l (shading.cuh evalGGX) at directions wo, wi; 0 where f is 0 or
// the roughness is clamped. With a = the lobe roughness max(0.001, r^2) (r the material's roughness, saturated),
// T = tan^2 of the half vector's angle and t = tan^2 of a direction's angle:
//   log D  = log(a^2) - 2 log(a^2 + T) + const         -> 2/a - 4a/(a^2 + T)
//   log G1 = log 2 - log(1 + S), S = sqrt(1 + a^2 t)   -> -a t / (S (1 + S))
// and da/dr = 2r where r^2 > 0.001 (0 < r < 1). The Schlick Fresnel does not depend on the roughness.
// Near a mirror (a of 1e-3..1e-2) the two terms of dlog D are hundreds each and a path's credits cancel over samples to
// a gradient thousands of times smaller, so T must be exact to far better than float's 1 - cos^2 gives: the tangents
// are taken from |x cross n|^2 / (x . n)^2, in double (a few dozen FP64 operations a vertex).
__device__ __forceinline__ float ggxLogDerivative(const Lobe& l, float materialRoughness, V3 wo, V3 wi) {
    const double r = materialRoughness;
    if (!(r > 0.0 && r < 1.0) || materialRoughness * materialRoughness <= 0.001f) return 0.0f;
    const double nx = l.frame.z.x, ny = l.frame.z.y, nz = l.frame.z.z;
    const double ox = wo.x, oy = wo.y, oz = wo.z, ix = wi.x, iy = wi.y, iz = wi.z;
    const double cosNO = ox * nx + oy * ny + oz * nz, cosNI = ix * nx + iy * ny + iz * nz;
    if (cosNO <= 0.0 || cosNI <= 0.0) return 0.0f;
    double mx = ox + ix, my = oy + iy, mz = oz + iz;
    const double lm = sqrt(mx * mx + my * my + mz * mz);
    if (!(lm > 0.001)) return 0.0f;
    mx /= lm;
    my /= lm;
    mz /= lm;
    const double cosThetaM = mx * nx + my * ny + mz * nz;
    if (cosThetaM <= 0.0 || mx * ix + my * iy + mz * iz <= 0.0) return 0.0f;
    auto sin2 = [&](double x, double y, double z) {
        const double cx = y * nz - z * ny, cy = z * nx - x * nz, cz = x * ny - y * nx;
        return cx * cx + cy * cy + cz * cz;
    };
    const double a = l.roughness, a2 = a * a;
    const double T = sin2(mx, my, mz) / (cosThetaM * cosThetaM);
    const double to = sin2(ox, oy, oz) / (cosNO * cosNO), ti = sin2(ix, iy, iz) / (cosNI * cosNI);
    const double so = sqrt(1.0 + a2 * to), si = sqrt(1.0 + a2 * ti);
    const double dlogf = 2.0 / a - 4.0 * a / (a2 + T) - a * to / (so * (1.0 + so)) - a * ti / (si * (1.0 + si));
    return float(dlogf * 2.0 * r);
}

// A Lambert vertex's credit from what its path gathered after it (`after`), its scale 1 / albedo: to its material's
// diffuse colour (d albedo / d diffuse = the texel of a textured one, else 1) and, textured, to the texels its lookup
// read (d albedo / d texel = diffuse x the texel's weight), those as FP32 atomics into texGrad.
__device__ __forceinline__ void creditLambert(float* partial, const Layout& at, const SceneView& s, uint32_t m, float4 d, V3 after, V3 sc,
                                              const float4* texc, float* texGrad) {
    const MaterialRec& mr = s.materials[m];
    const float w[3] = {d.x * after.x * sc.x, d.y * after.y * sc.y, d.z * after.z * sc.z};
    V3 texel{1, 1, 1};
    uint64_t ti[4];
    float tw[4];
    bool textured = false;
    if (mr.texture && texc) {
        const float4 tc = *texc;
        TexHit th;
        th.s = tc.x;
        th.t = tc.y;
        th.primary = tc.z != 0.0f ? 1u : 0u;
        textured = texLookup(s, mr.texture - 1, th, ti, tw);
        if (textured) texel = th.texel;
    }
    const float tv[3] = {texel.x, texel.y, texel.z};
    for (int c = 0; c < 3; ++c) {
        if (w[c] == 0.0f) continue;
        atomicAdd(partial + at.albedo(m) + c, w[c] * tv[c]);
        if (textured && texGrad)
            for (int i = 0; i < 4; ++i)
                if (tw[i] != 0.0f) atomicAdd(texGrad + 3 * ti[i] + c, w[c] * mr.diffuse[c] * tw[i]);
    }
}

}  // namespace x2
