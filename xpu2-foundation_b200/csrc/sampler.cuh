// Identity-hashed sampler on the device: bit-exact with the reference's sample_stream.h.
//
// Philox4x32-10 on the counter {pixel, index lo, index hi, dimension group} keyed by stream ^ branch * phi
// (sample_stream.h:31-54), Owen-scrambled Sobol for the policy-gated dimensions (sample_stream.h:102-147), the
// per-vertex stream (async_integrator.h:151-176) and the child-branch hash (async_integrator.h:281-287).
// The Sobol direction numbers (17 dimensions x 32 bits) are generated on the host from Joe and Kuo's published
// primitive-polynomial parameters by the Bratley-Fox recurrence (x2_sobol_directions in api.cu) and placed in
// constant memory; every thread reads the same entry at the same step, so the reads broadcast.
#pragma once
#include <cstdint>

namespace x2 {

typedef uint32_t U32;
typedef uint64_t U64;

// One copy a translation unit (whole-program compilation): every unit with sampling kernels (render.cu,
// wavefront.cu) exports an upload function that x2_open calls for its copy.
static __constant__ U32 c_sobol[17][32];

struct Identity {
    U32 pixel;
    U64 index, stream, branch;
};

// Philox4x32-10: ten rounds of two 32x32->64 products (mul.wide as __umulhi + mul.lo).
__device__ __forceinline__ void philox(U32& c0, U32& c1, U32& c2, U32& c3, U32 ka, U32 kb) {
#pragma unroll
    for (int round = 0; round < 10; ++round) {
        const U32 hiA = __umulhi(c0, 0xd2511f53u), loA = c0 * 0xd2511f53u;
        const U32 hiB = __umulhi(c2, 0xcd9e8d57u), loB = c2 * 0xcd9e8d57u;
        const U32 n0 = hiB ^ c1 ^ ka, n2 = hiA ^ c3 ^ kb;
        c0 = n0;
        c1 = loB;
        c2 = n2;
        c3 = loA;
        ka += 0x9e3779b9u;
        kb += 0xbb67ae85u;
    }
}

struct Words {
    U32 v0, v1, v2, v3;
};

__device__ __forceinline__ Words block(U32 pixel, U64 index, U64 stream, U64 branch, U32 group) {
    const U64 k = stream ^ (branch * 0x9e3779b97f4a7c15ull);
    U32 c0 = pixel, c1 = U32(index), c2 = U32(index >> 32), c3 = group;
    philox(c0, c1, c2, c3, U32(k), U32(k >> 32));
    return Words{c0, c1, c2, c3};
}
__device__ __forceinline__ U32 pick(const Words& w, U32 i) {
    return i == 0 ? w.v0 : i == 1 ? w.v1 : i == 2 ? w.v2 : w.v3;
}
__device__ __forceinline__ U32 word(const Identity& id, U32 dimension) {
    return pick(block(id.pixel, id.index, id.stream, id.branch, dimension >> 2), dimension & 3);
}
// Exact: a 24-bit integer times 2^-24, in [0, 1).
__device__ __forceinline__ float unit(U32 bits) { return float(bits >> 8) * 0x1p-24f; }

__device__ __forceinline__ U32 sobol(U32 index, U32 dimension) {
    U32 gray = index ^ (index >> 1), result = 0;
    for (U32 bit = 0; gray; ++bit, gray >>= 1)
        if (gray & 1u) result ^= c_sobol[dimension][bit];
    return result;
}
// Burley's hash-based Owen scramble (JCGT 2020): each bit flipped by a hash of the bits above it.
__device__ __forceinline__ U32 owenScramble(U32 x, U32 seed) {
    x = __brev(x);
    x += seed;
    x ^= x * 0x6c50b47cu;
    x ^= x * 0xb82f1e52u;
    x ^= x * 0xc7afe638u;
    x ^= x * 0x8d22f6e6u;
    return __brev(x);
}
// The policy: bit 1 the camera's dimensions 0..4, bit 2 the first BSDF sample's 16/17, bit 4 the first light
// sample's 18/19, bit 8 the subsurface dimensions 20..27 take scrambled Sobol; all else is Philox.
__device__ __forceinline__ U32 samplingWord(const Identity& id, U32 dimension, U32 policy) {
    const bool camera = dimension < 5, diffuse = dimension == 16 || dimension == 17, light = dimension == 18 || dimension == 19,
               subsurface = dimension >= 20 && dimension <= 27;
    if ((!camera || !(policy & 1)) && (!diffuse || !(policy & 2)) && (!light || !(policy & 4)) && (!subsurface || !(policy & 8)))
        return word(id, dimension);
    const U32 d = camera ? (dimension < 2 ? dimension : dimension < 4 ? dimension + 12 : 16) : dimension - 14;
    const U64 high = id.index >> 32;
    if (camera && dimension >= 2) {  // the lens and the shutter: Sobol in a sample order of their own
        const Words seeds = block(id.pixel, high, id.stream, id.branch, dimension < 4 ? 0x50414444u : 0x50414445u);
        return owenScramble(sobol(owenScramble(U32(id.index), seeds.v0), dimension < 4 ? dimension - 2 : 0u),
                            dimension < 4 ? (dimension == 2 ? seeds.v1 : seeds.v2) : seeds.v1);
    }
    const Words seeds = block(id.pixel, high, id.stream, id.branch, 0x534f424fu + (d >> 2));
    return owenScramble(sobol(U32(id.index), d), pick(seeds, d & 3));
}
__device__ __forceinline__ float draw(const Identity& id, U32 dimension, U32 policy) {
    return unit(samplingWord(id, dimension, policy));
}

// samplingWord(id, d) and samplingWord(id, d + 1) for the BSDF pair (d = 16) or the light pair (d = 18): the two
// dimensions share their Philox group (and, where the policy takes Sobol, their seed block and the index's Gray-code
// bits), so one block and one pass over the bits give both words.
__device__ __forceinline__ void samplingWordPair(const Identity& id, U32 dimension, U32 policy, U32& a, U32& b) {
    const bool sobolPair = dimension == 16 ? (policy & 2) != 0 : (policy & 4) != 0;
    if (!sobolPair) {
        const Words w = block(id.pixel, id.index, id.stream, id.branch, dimension >> 2);
        a = pick(w, dimension & 3);
        b = pick(w, (dimension + 1) & 3);
        return;
    }
    const U32 d = dimension - 14;
    const Words seeds = block(id.pixel, id.index >> 32, id.stream, id.branch, 0x534f424fu + (d >> 2));
    U32 gray = U32(id.index) ^ (U32(id.index) >> 1), r0 = 0, r1 = 0;
    for (U32 bit = 0; gray; ++bit, gray >>= 1)
        if (gray & 1u) {
            r0 ^= c_sobol[d][bit];
            r1 ^= c_sobol[d + 1][bit];
        }
    a = owenScramble(r0, pick(seeds, d & 3));
    b = owenScramble(r1, pick(seeds, (d + 1) & 3));
}
__device__ __forceinline__ void drawPair(const Identity& id, U32 dimension, U32 policy, float& a, float& b) {
    U32 wa, wb;
    samplingWordPair(id, dimension, policy, wa, wb);
    a = unit(wa);
    b = unit(wb);
}

constexpr U32 CameraDimensions = 16, DimensionsPerBounce = 256;

// A vertex's uniform numbers: dimension 16 + bounce * 256 + offset of its branch's Philox stream, one block per
// four draws.
struct Stream {
    Identity id;
    U32 dimension, group;
    Words w;
    Stream() = default;
    __device__ Stream(const Identity& i, U32 bounce, U32 offset)
        : id(i), dimension(CameraDimensions + bounce * DimensionsPerBounce + offset), group(~0u) {}
    __device__ float next() {
        if ((dimension >> 2) != group) {
            group = dimension >> 2;
            w = block(id.pixel, id.index, id.stream, id.branch, group);
        }
        return unit(pick(w, dimension++ & 3));
    }
};

// A child's address in the sample's tree: a splitmix64 finaliser of (parent, a, b).
__device__ __forceinline__ U64 childBranch(U64 parent, U32 a, U32 b) {
    U64 z = parent + 0x9e3779b97f4a7c15ull * (U64(a) * 0x10001u + U64(b) + 1);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

}  // namespace x2
