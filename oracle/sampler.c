/*
 * ORACLE — test infrastructure only (tests/, __graft_entry__.smoke and bench.py's CPU baseline may load it; the
 * product never does). A plain-C restatement of the reference's identity-hashed sampler,
 * xpu2/interactive/sample_stream.h, and of the path tracer's stream and branch addressing,
 * xpu2/interactive/async_integrator.h:151-176 and :281-287. Pinned against the reference's known-answer vectors
 * (sample_fixture.h:17-20, qmc_fixture.h:14-28) and against the reference compiled from source (oracle/_ref).
 */
#include <stdint.h>

typedef uint32_t U32;
typedef uint64_t U64;

/* sample::philox, sample_stream.h:31-38: Philox4x32-10 (Salmon et al., Random123, SC'11). */
static void philox(U32 c[4], U32 ka, U32 kb) {
    for (int round = 0; round < 10; ++round) {
        const U64 a = (U64)c[0] * 0xd2511f53u, b = (U64)c[2] * 0xcd9e8d57u;
        const U32 n0 = (U32)(b >> 32) ^ c[1] ^ ka, n1 = (U32)b, n2 = (U32)(a >> 32) ^ c[3] ^ kb, n3 = (U32)a;
        c[0] = n0; c[1] = n1; c[2] = n2; c[3] = n3;
        ka += 0x9e3779b9u;
        kb += 0xbb67ae85u;
    }
}

/* sample::key / block / word, sample_stream.h:43-54: counter {pixel, index lo, index hi, dimension group},
 * key = stream ^ branch * golden ratio. */
void oracle_block(U32 pixel, U64 index, U64 stream, U64 branch, U32 group, U32 out[4]) {
    const U64 k = stream ^ (branch * 0x9e3779b97f4a7c15ull);
    out[0] = pixel;
    out[1] = (U32)index;
    out[2] = (U32)(index >> 32);
    out[3] = group;
    philox(out, (U32)k, (U32)(k >> 32));
}
U32 oracle_word(U32 pixel, U64 index, U64 stream, U64 branch, U32 dimension) {
    U32 b[4];
    oracle_block(pixel, index, stream, branch, dimension >> 2, b);
    return b[dimension & 3];
}
/* sample::unit, sample_stream.h:56: the top 24 bits times 2^-24. */
float oracle_unit(U32 bits) { return (float)(bits >> 8) * 0x1p-24f; }

/* Sobol direction numbers, 17 dimensions x 32 bits: dimension 0 is van der Corput, dimensions 1..16 follow the
 * primitive-polynomial recurrence (Bratley & Fox 1988) with Joe and Kuo's published parameters (degree s,
 * coefficients a, initial m) for their dimensions 2..17 — the table sample_stream.h:82-100 holds. */
static U32 directions[17][32];
static int directionsReady = 0;
static void makeDirections(void) {
    static const U32 s[16] = {1, 2, 3, 3, 4, 4, 5, 5, 5, 5, 5, 5, 6, 6, 6, 6};
    static const U32 a[16] = {0, 1, 1, 2, 1, 4, 2, 4, 7, 11, 13, 14, 1, 13, 16, 19};
    static const U32 m0[16][6] = {{1}, {1, 3}, {1, 3, 1}, {1, 1, 1}, {1, 1, 3, 3}, {1, 3, 5, 13}, {1, 1, 5, 5, 17},
                                  {1, 1, 5, 5, 5}, {1, 1, 7, 11, 19}, {1, 1, 5, 1, 1}, {1, 1, 1, 3, 11}, {1, 3, 5, 5, 31},
                                  {1, 3, 3, 9, 7, 49}, {1, 1, 1, 15, 21, 21}, {1, 3, 1, 13, 27, 49}, {1, 1, 1, 15, 7, 5}};
    for (int i = 0; i < 32; ++i) directions[0][i] = 1u << (31 - i);
    for (int d = 0; d < 16; ++d) {
        U64 m[32];
        for (U32 i = 0; i < s[d]; ++i) m[i] = m0[d][i];
        for (U32 i = s[d]; i < 32; ++i) {
            U64 v = m[i - s[d]] ^ (m[i - s[d]] << s[d]);
            for (U32 k = 1; k < s[d]; ++k)
                if ((a[d] >> (s[d] - 1 - k)) & 1u) v ^= m[i - k] << k;
            m[i] = v;
        }
        for (int i = 0; i < 32; ++i) directions[d + 1][i] = (U32)(m[i] << (31 - i));
    }
    directionsReady = 1;
}
U32 oracle_direction(U32 dimension, U32 bit) {
    if (!directionsReady) makeDirections();
    return directions[dimension][bit];
}

/* sample::sobol, sample_stream.h:102-107: the Gray-code index's bits select direction numbers. */
U32 oracle_sobol(U32 index, U32 dimension) {
    if (!directionsReady) makeDirections();
    U32 gray = index ^ (index >> 1), result = 0, bit = 0;
    while (gray) {
        if (gray & 1u) result ^= directions[dimension][bit];
        gray >>= 1;
        ++bit;
    }
    return result;
}
static U32 reverseBits(U32 x) {
    U32 r = 0;
    for (int i = 0; i < 32; ++i) r |= ((x >> i) & 1u) << (31 - i);
    return r;
}
/* sample::owenScramble, sample_stream.h:122-126: Burley's hash-based nested uniform scramble (JCGT 2020). */
U32 oracle_owen(U32 x, U32 seed) {
    x = reverseBits(x);
    x += seed;
    x ^= x * 0x6c50b47cu;
    x ^= x * 0xb82f1e52u;
    x ^= x * 0xc7afe638u;
    x ^= x * 0x8d22f6e6u;
    return reverseBits(x);
}
/* sample::samplingWord, sample_stream.h:127-144: policy bits 1 (camera dims 0..4), 2 (BSDF 16/17), 4 (light 18/19)
 * and 8 (subsurface 20..27) route a dimension to scrambled Sobol; every other draw is the Philox word. */
U32 oracle_sampling_word(U32 pixel, U64 index, U64 stream, U64 branch, U32 dimension, U32 policy) {
    const int camera = dimension < 5, diffuse = dimension == 16 || dimension == 17, light = dimension == 18 || dimension == 19,
              subsurface = dimension >= 20 && dimension <= 27;
    if ((!camera || !(policy & 1)) && (!diffuse || !(policy & 2)) && (!light || !(policy & 4)) && (!subsurface || !(policy & 8)))
        return oracle_word(pixel, index, stream, branch, dimension);
    const U32 d = camera ? (dimension < 2 ? dimension : dimension < 4 ? dimension + 12 : 16) : dimension - 14;
    const U64 high = index >> 32;
    U32 seeds[4];
    if (camera && dimension >= 2) {
        oracle_block(pixel, high, stream, branch, dimension < 4 ? 0x50414444u : 0x50414445u, seeds);
        const U32 order = oracle_owen((U32)index, seeds[0]);
        return oracle_owen(oracle_sobol(order, dimension < 4 ? dimension - 2 : 0u), seeds[dimension < 4 ? dimension - 1 : 1]);
    }
    oracle_block(pixel, high, stream, branch, 0x534f424fu + (d >> 2), seeds);
    return oracle_owen(oracle_sobol((U32)index, d), seeds[d & 3]);
}
/* paths::childBranch, async_integrator.h:281-287: a splitmix64 finaliser of (parent, a, b). */
U64 oracle_child_branch(U64 parent, U32 a, U32 b) {
    U64 z = parent + 0x9e3779b97f4a7c15ull * ((U64)a * 0x10001u + (U64)b + 1);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
/* paths::Stream::next, async_integrator.h:151-176: the n-th draw of a vertex's stream at bounce `bounce`:
 * dimension 16 + bounce * 256 + n, one Philox block per four draws. */
float oracle_stream_draw(U32 pixel, U64 index, U64 stream, U64 branch, U32 bounce, U32 n) {
    return oracle_unit(oracle_word(pixel, index, stream, branch, 16u + bounce * 256u + n));
}
/* Batch forms for ctypes callers: ids as (pixel, pad, index, stream, branch) records of 32 bytes. */
typedef struct { U32 pixel, pad; U64 index, stream, branch; } Identity;
void oracle_sampling_words(const Identity* ids, const U32* dims, U64 n, U32 policy, U32* out) {
    for (U64 i = 0; i < n; ++i) out[i] = oracle_sampling_word(ids[i].pixel, ids[i].index, ids[i].stream, ids[i].branch, dims[i], policy);
}
void oracle_philox(const U32* counters, const U32* keys, U64 n, U32* out) {
    for (U64 i = 0; i < n; ++i) {
        U32 c[4] = {counters[4 * i], counters[4 * i + 1], counters[4 * i + 2], counters[4 * i + 3]};
        philox(c, keys[2 * i], keys[2 * i + 1]);
        for (int k = 0; k < 4; ++k) out[4 * i + k] = c[k];
    }
}
