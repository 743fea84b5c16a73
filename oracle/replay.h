// ORACLE (test infrastructure only) — the replay build of the reference integrator (oracle/_ref/libx2ref_replay.so,
// ref_backend.cpp compiled with -DX2REF_REPLAY and linked with -Wl,--wrap for the float functions below).
//
// It answers one question about a sample whose device radiance differs from the reference's: do the device's values
// of the transcendental functions alone account for it? The device's diagnostic build records every call of a sample
// (include/x2_diag.h: function, arguments, results). Replaying the sample here, each wrapped libm call whose function
// and arguments match a recorded call returns the device's result instead of libm's; every other call goes to libm
// and counts as a miss. The reference's own code runs unchanged; only the link redirects its calls. The replay also
// logs every call it made (with the value it used) and the backend's events (closest hits and shadow-ray
// visibilities), so two replays of a sample — with libm's values and with the device's — show the first call whose
// value differs and the first discrete decision that follows from it.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>
#include <unordered_map>
#include <vector>

#include "../include/x2_diag.h"

extern "C" {
float __real_sinf(float);
float __real_cosf(float);
void __real_sincosf(float, float*, float*);
float __real_expf(float);
float __real_logf(float);
float __real_tanf(float);
float __real_atan2f(float, float);
float __real_powf(float, float);
float __real_acosf(float);
}

namespace replay {

enum : uint32_t { kSincos = 1, kExp = 2, kLog = 3, kTan = 4, kAtan2 = 5, kPow = 6, kAcos = 7, kCos = 8 };

inline uint32_t bits(float x) {
    uint32_t u;
    std::memcpy(&u, &x, 4);
    return u;
}
inline uint64_t key(uint32_t fn, float a, float b) { return (uint64_t(fn) << 56) ^ (uint64_t(bits(b)) << 24) ^ uint64_t(bits(a)); }

// A backend event: kind 1 a closest hit (value: triangle or ~0u, t), kind 2 a shadow ray's visibility (value 0/1,
// t: its far distance); x, y, z the ray's direction. Kind 3 a texture lookup (value: its mode, t and x: its s and t,
// y and z: the texel's red and green) and kind 4 its rest (value: its status, t: the texel's blue).
struct Event {
    uint32_t kind, value;
    float t, x, y, z;
};

struct State {
    std::unordered_map<uint64_t, std::pair<float, float>> table;  // the device's values by (function, arguments)
    bool useTable = false;
    std::vector<x2_diag_call> calls;                                // every call made, with the value used
    std::vector<Event> events;
    uint64_t misses = 0;                                            // calls the table had no value for
};
inline thread_local State* t_state = nullptr;

inline bool find(uint32_t fn, float a, float b, float& r0, float& r1) {
    State* s = t_state;
    if (!s || !s->useTable) return false;
    auto it = s->table.find(key(fn, a, b));
    if (it == s->table.end()) {
        ++s->misses;
        return false;
    }
    r0 = it->second.first;
    r1 = it->second.second;
    return true;
}
inline void log(uint32_t fn, float a, float b, float r0, float r1) {
    if (t_state) t_state->calls.push_back(x2_diag_call{fn, a, b, r0, r1});
}
inline void event(uint32_t kind, uint32_t value, float t, float x, float y, float z) {
    if (t_state) t_state->events.push_back(Event{kind, value, t, x, y, z});
}

}  // namespace replay

// The wrapped functions. sinf and cosf of one argument are one recorded sincos on the device.
extern "C" float __wrap_sinf(float x) {
    float s, c;
    if (!replay::find(replay::kSincos, x, 0.0f, s, c)) s = __real_sinf(x), c = __real_cosf(x);
    replay::log(replay::kSincos, x, 0.0f, s, c);
    return s;
}
extern "C" float __wrap_cosf(float x) {
    float s, c;
    if (!replay::find(replay::kSincos, x, 0.0f, s, c)) {
        float v, d;
        if (replay::find(replay::kCos, x, 0.0f, v, d)) return replay::log(replay::kCos, x, 0.0f, v, 0.0f), v;
        s = __real_sinf(x), c = __real_cosf(x);
    }
    replay::log(replay::kSincos, x, 0.0f, s, c);
    return c;
}
extern "C" void __wrap_sincosf(float x, float* s, float* c) {
    if (!replay::find(replay::kSincos, x, 0.0f, *s, *c)) __real_sincosf(x, s, c);
    replay::log(replay::kSincos, x, 0.0f, *s, *c);
}
#define X2REF_WRAP1(name, fn)                                                  \
    extern "C" float __wrap_##name(float x) {                                  \
        float r, u;                                                            \
        if (!replay::find(replay::fn, x, 0.0f, r, u)) r = __real_##name(x);    \
        replay::log(replay::fn, x, 0.0f, r, 0.0f);                             \
        return r;                                                              \
    }
X2REF_WRAP1(expf, kExp)
X2REF_WRAP1(logf, kLog)
X2REF_WRAP1(tanf, kTan)
X2REF_WRAP1(acosf, kAcos)
#undef X2REF_WRAP1
extern "C" float __wrap_atan2f(float y, float x) {
    float r, u;
    if (!replay::find(replay::kAtan2, y, x, r, u)) r = __real_atan2f(y, x);
    replay::log(replay::kAtan2, y, x, r, 0.0f);
    return r;
}
extern "C" float __wrap_powf(float x, float y) {
    float r, u;
    if (!replay::find(replay::kPow, x, y, r, u)) r = __real_powf(x, y);
    replay::log(replay::kPow, x, y, r, 0.0f);
    return r;
}
