// Exact, order-independent film splats for the light integrator.
//
// Each pixel channel (X, Y, Z) is a 192-bit unsigned fixed-point sum held in three 64-bit words,
// least significant first, whose lowest bit weighs 2^kSplatExp0 = 2^-80. A splat's FP64
// significand is shifted to its binary exponent and added with 64-bit atomics, carries propagated
// word by word. Integer addition does not depend on order, so a film that many threads add to in
// no fixed order is still the same bit for bit from run to run (the reference's GPU particle film
// does the same with 32-bit words, src/owe/backends/gpu/shaders/particle.slang:6-46).
#pragma once

#include "spectral.cuh"

namespace owec {

constexpr int kSplatWordsPerChannel = 3;
constexpr int kSplatWordsPerPixel = 3 * kSplatWordsPerChannel;
constexpr int kSplatExp0 = -80;

// Where connections land: the film's splat words, and the pixel of each pending connection
// (indexed like the shadow queue).
struct SplatTarget {
    unsigned long long* words;
    uint32_t* pixel;
};

// Adds v to word w of a channel, carrying into the words above it.
__device__ __forceinline__ void splatAddWord(unsigned long long* acc, int w, unsigned long long v) {
    const unsigned long long old = atomicAdd(acc + w, v);
    if (old + v >= old) return;  // no wrap-around
    for (int k = w + 1; k < kSplatWordsPerChannel; ++k)
        if (atomicAdd(acc + k, 1ull) != ~0ull) return;
}

// Adds v exactly to a channel's sum. Zero, negative and NaN add nothing; bits below 2^-80 are
// dropped. False when v does not fit (infinite, or 2^112 and above).
__device__ __forceinline__ bool splatAdd(unsigned long long* acc, double v) {
    if (!(v > 0)) return true;
    const unsigned long long bits = static_cast<unsigned long long>(__double_as_longlong(v));
    const int e = int((bits >> 52) & 0x7FF);
    if (e == 0x7FF) return false;
    if (e == 0) return true;  // subnormal: far below the lowest bit
    unsigned long long mant = (bits & 0xFFFFFFFFFFFFFull) | (1ull << 52);  // v = mant * 2^(e - 1075)
    int p = e - 1075 - kSplatExp0;  // position of mant's lowest bit in the sum
    if (p < 0) {
        if (p <= -53) return true;
        mant >>= -p;
        p = 0;
    }
    const int w = p >> 6, r = p & 63;
    if (w >= kSplatWordsPerChannel) return false;
    const unsigned long long hi = r ? mant >> (64 - r) : 0ull;
    if (hi && w + 1 >= kSplatWordsPerChannel) return false;
    splatAddWord(acc, w, mant << r);
    if (hi) splatAddWord(acc, w + 1, hi);
    return true;
}

// Adds a spectral contribution to a pixel as XYZ: c[k] is already the value over its wavelength's
// pdf and NW * the integral of y-bar (Wavelengths::toXYZ, src/owe/core/wavelengths.hpp:71-84), T[k]
// a transmittance. False when a channel did not fit.
template <class R>
__device__ __forceinline__ bool splatXyz(unsigned long long* words, uint32_t pixel, const float lambda[NW],
                                         const float c[NW], const R T[NW]) {
    double x = 0, y = 0, z = 0;
    for (int k = 0; k < NW; ++k) {
        const double w = double(c[k]) * double(T[k]);
        if (w == 0) continue;
        const double l = double(lambda[k]);
        x += w * cieX(l);
        y += w * cieY(l);
        z += w * cieZ(l);
    }
    if (!isfinite(x + y + z)) return true;
    unsigned long long* px = words + size_t(pixel) * kSplatWordsPerPixel;
    bool ok = splatAdd(px, x);
    ok = splatAdd(px + kSplatWordsPerChannel, y) && ok;
    ok = splatAdd(px + 2 * kSplatWordsPerChannel, z) && ok;
    return ok;
}

}  // namespace owec
