// The transcendental functions the path calls, in one place.
//
// The product calls CUDA's single-precision functions (sincosf, expf, logf, tanf, atan2f, powf, acosf, cosf), as the
// reference's own GPU lane does (shade_math.h:123-129 picks sincosf under nvcc, libm's sinf/cosf on the host). They
// and the host's libm may differ in the last unit of their results; everything else on the path (add, multiply,
// divide, square root, without contraction) rounds alike on both sides.
//
// A diagnostic build (-DX2_DIAG, libx2diag.so; never the product, and only the per-sample kernels of render.cu) adds
// switches, set by x2_diag_set: mode bit 0 evaluates each function in double and rounds the result to float (the
// correctly rounded value but for rare double roundings — what a libm within half an ulp returns), and bit 1 records
// every call of the launch (function, arguments, results) into a caller's device buffer, in call order for a
// one-sample launch. The records let the host replay a sample through the reference with the device's values. Bit 2
// (sharedPivot) changes the volume march's single scattering, for the estimator study only: a distance sample's light
// point is its pair's equi-angular light point, the pivot both MIS weights were computed with.
#pragma once
#include <cstdint>

namespace x2 {
namespace mf {

enum : uint32_t { kSincos = 1, kExp = 2, kLog = 3, kTan = 4, kAtan2 = 5, kPow = 6, kAcos = 7, kCos = 8 };
// Other values the diagnostic build records beside the functions' calls: a texture lookup's (s, t) and texel.
enum : uint32_t { kTexLookup = 20, kTexLookupRest = 21, kHit = 40, kVisible = 41, kAdded = 42 };

struct DiagCall {
    uint32_t fn;
    float a, b;    // arguments (b: atan2's x, pow's exponent)
    float r0, r1;  // results (r1: sincos's cosine)
};

#ifdef X2_DIAG
#define X2_DIAG_RECORD(fn, a, b, r0, r1) x2::mf::record(fn, a, b, r0, r1)
static __device__ int g_mode;
static __device__ DiagCall* g_calls;
static __device__ uint32_t g_cap;
static __device__ uint32_t g_count;

__device__ __forceinline__ void record(uint32_t fn, float a, float b, float r0, float r1) {
    if (!(g_mode & 2) || !g_calls) return;
    const uint32_t k = atomicAdd(&g_count, 1u);
    if (k < g_cap) g_calls[k] = DiagCall{fn, a, b, r0, r1};
}
__device__ __forceinline__ bool wide() { return g_mode & 1; }
__device__ __forceinline__ bool sharedPivot() { return g_mode & 4; }
#define X2_MF(fn, a, b, r0, r1) record(fn, a, b, r0, r1)
#else
#define X2_DIAG_RECORD(fn, a, b, r0, r1) ((void)0)
__device__ __forceinline__ constexpr bool wide() { return false; }
__device__ __forceinline__ constexpr bool sharedPivot() { return false; }
#define X2_MF(fn, a, b, r0, r1) ((void)0)
#endif

__device__ __forceinline__ void sincos(float x, float* s, float* c) {
    if (wide()) {
        *s = float(::sin(double(x)));
        *c = float(::cos(double(x)));
    } else {
        sincosf(x, s, c);
    }
    X2_MF(kSincos, x, 0.0f, *s, *c);
}
__device__ __forceinline__ float exp(float x) {
    const float r = wide() ? float(::exp(double(x))) : expf(x);
    X2_MF(kExp, x, 0.0f, r, 0.0f);
    return r;
}
__device__ __forceinline__ float log(float x) {
    const float r = wide() ? float(::log(double(x))) : logf(x);
    X2_MF(kLog, x, 0.0f, r, 0.0f);
    return r;
}
__device__ __forceinline__ float tan(float x) {
    const float r = wide() ? float(::tan(double(x))) : tanf(x);
    X2_MF(kTan, x, 0.0f, r, 0.0f);
    return r;
}
__device__ __forceinline__ float atan2(float y, float x) {
    const float r = wide() ? float(::atan2(double(y), double(x))) : atan2f(y, x);
    X2_MF(kAtan2, y, x, r, 0.0f);
    return r;
}
__device__ __forceinline__ float pow(float x, float y) {
    const float r = wide() ? float(::pow(double(x), double(y))) : powf(x, y);
    X2_MF(kPow, x, y, r, 0.0f);
    return r;
}
__device__ __forceinline__ float acos(float x) {
    const float r = wide() ? float(::acos(double(x))) : acosf(x);
    X2_MF(kAcos, x, 0.0f, r, 0.0f);
    return r;
}
__device__ __forceinline__ float cos(float x) {
    const float r = wide() ? float(::cos(double(x))) : cosf(x);
    X2_MF(kCos, x, 0.0f, r, 0.0f);
    return r;
}

#undef X2_MF

}  // namespace mf
}  // namespace x2
