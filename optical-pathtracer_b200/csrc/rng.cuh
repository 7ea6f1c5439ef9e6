// Deterministic random numbers: the reference's PCG32 streams and its 53-bit uniforms
// (src/owe/core/sampling.hpp:11-33; pcg32Next, mixBits, hashCombine in
// src/owe/core/shared/warps.hpp:12-30), drawn in the same order so that a device path follows the
// CPU path with the same seed until rounding makes one of its decisions differ.
#pragma once

#include "common.cuh"

namespace owec {

OWEC_HD uint64_t mixBits(uint64_t v) {
    v ^= v >> 31;
    v *= 0x7fb5d329728ea185ULL;
    v ^= v >> 27;
    v *= 0x81dadef4bc2dd44dULL;
    v ^= v >> 33;
    return v;
}
OWEC_HD uint64_t hashCombine(uint64_t a, uint64_t b) { return mixBits(a ^ (mixBits(b) + 0x9e3779b97f4a7c15ULL)); }

// One PCG32 stream (O'Neill): 64-bit LCG state, output by xorshift and a random rotation.
struct Pcg32 {
    uint64_t state, inc;
    OWEC_HD uint32_t next() {
        const uint64_t old = state;
        state = old * 6364136223846793005ULL + inc;
        const uint32_t xs = uint32_t(((old >> 18u) ^ old) >> 27u);
        const uint32_t rot = uint32_t(old >> 59u);
        return (xs >> rot) | (xs << ((~rot + 1u) & 31u));
    }
    // Stream `stream` of seed `seed`: state 0, one step, add the seed, one step.
    OWEC_HD static Pcg32 seeded(uint64_t seed, uint64_t stream) {
        Pcg32 r{0, (stream << 1u) | 1u};
        r.next();
        r.state += seed;
        r.next();
        return r;
    }
    // Uniform in [0, 1) with 53 bits, from two outputs (27 + 26 bits).
    OWEC_HD double uniform() {
        const uint64_t a = next() >> 5, b = next() >> 6;
        return (double(a) * 67108864.0 + double(b)) * (1.0 / 9007199254740992.0);
    }
};

// The uniform in the precision of the arithmetic. Rounding toward zero keeps a float below 1.
template <class T> OWEC_HD T uniformAs(Pcg32& r);
template <> OWEC_HD double uniformAs<double>(Pcg32& r) { return r.uniform(); }
template <> OWEC_HD float uniformAs<float>(Pcg32& r) {
#if defined(__CUDA_ARCH__)
    return __double2float_rz(r.uniform());
#else
    float f = float(r.uniform());
    return f < 1.0f ? f : 0.99999994f;
#endif
}

// Two and three uniforms in the reference's fixed order (src/owe/core/sampling.hpp:37-51): the
// last one is drawn first.
template <class T>
struct Draw2 {
    T u1, u2;
    OWEC_HD explicit Draw2(Pcg32& r) { u2 = uniformAs<T>(r); u1 = uniformAs<T>(r); }
};
template <class T>
struct Draw3 {
    T u1, u2, u3;
    OWEC_HD explicit Draw3(Pcg32& r) { u3 = uniformAs<T>(r); u2 = uniformAs<T>(r); u1 = uniformAs<T>(r); }
};

}  // namespace owec
