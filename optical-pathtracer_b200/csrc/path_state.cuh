// Path state of the wavefront loop: structure-of-arrays in HBM, one slot per path in flight, and
// the queues that join the kernels.
#pragma once

#include "device_scene.cuh"
#include "rng.cuh"
#include "traverse.cuh"

namespace owec {

// Precision modes (owec.h OWEC_PRECISION_*): R is the arithmetic of directions, throughput and
// optics; Ro the analytic roots; Rr their refinement; origins are FP64 unless PlainOrigin.
template <int M> struct Mode;
template <> struct Mode<OWEC_PRECISION_MIXED> {
    using R = float; using Ro = float; using Rr = double; static constexpr bool plainOrigin = false;
};
template <> struct Mode<OWEC_PRECISION_FP32> {
    using R = float; using Ro = float; using Rr = float; static constexpr bool plainOrigin = true;
};
template <> struct Mode<OWEC_PRECISION_FP64> {
    using R = double; using Ro = double; using Rr = double; static constexpr bool plainOrigin = false;
};

// The ray a path travels next, and what the intersect kernel needs of it.
template <class R>
struct alignas(16) PathRay {
    double o[3];      // camera-relative origin (rounded to FP32 after every update in the plain mode)
    R d[3];
    uint32_t region;  // region the ray travels in
    uint32_t depB;    // boundary and primitive it left (kNone)
    uint32_t depP;
    float errN;       // its anchor's error normal to a surface
};

// Throughput and spectral state.
template <class R>
struct alignas(16) PathSpec {
    R beta[4];
    float lambda[4];
    float pdf[4];     // 0: terminated secondary
    float L[4];       // radiance gathered so far
};

// Bookkeeping of a path.
struct alignas(16) PathAux {
    uint64_t rngState;
    uint32_t stream;    // PCG32 stream (the pass index of this sample)
    uint32_t pixel;
    uint32_t depth;     // bounce count (the reference's loop variable)
    uint32_t flags;     // kFlagSpecular | kFlagAlive
    float prevPdf;
    float weight;       // detector importance / pdf
    double prevP[3];    // last scattering vertex (camera-relative FP64: emission MIS decides inside or
                        // outside an emitting sphere from it, which FP32 rounding can flip)
    uint32_t lastBoundary;
};
constexpr uint32_t kFlagSpecular = 1u, kFlagAlive = 2u;

// Path state passes through the L2 once per kernel, far more of it than the L2 holds. Its loads and
// stores are marked evict-first (ld.global.cs / st.global.cs), so that it does not displace the
// BVH nodes and primitives, which every traversal kernel reads again.
#ifndef OWEC_STREAM_STATE
#define OWEC_STREAM_STATE 1
#endif
template <class T>
__device__ __forceinline__ T loadStream(const T* p) {
#if OWEC_STREAM_STATE
    if constexpr (alignof(T) >= 16 && sizeof(T) % 16 == 0) {
        constexpr int n = int(sizeof(T) / 16);
        uint4 w[n];
#pragma unroll
        for (int k = 0; k < n; ++k) w[k] = __ldcs(reinterpret_cast<const uint4*>(p) + k);
        T v;
        memcpy(&v, w, sizeof(T));
        return v;
    } else {
        static_assert(sizeof(T) % 8 == 0 && alignof(T) >= 8, "path state records are whole 8-byte words");
        constexpr int n = int(sizeof(T) / 8);
        unsigned long long w[n];
#pragma unroll
        for (int k = 0; k < n; ++k) w[k] = __ldcs(reinterpret_cast<const unsigned long long*>(p) + k);
        T v;
        memcpy(&v, w, sizeof(T));
        return v;
    }
#else
    return *p;
#endif
}
template <class T>
__device__ __forceinline__ void storeStream(T* p, const T& v) {
#if OWEC_STREAM_STATE
    if constexpr (alignof(T) >= 16 && sizeof(T) % 16 == 0) {
        constexpr int n = int(sizeof(T) / 16);
        uint4 w[n];
        memcpy(w, &v, sizeof(T));
#pragma unroll
        for (int k = 0; k < n; ++k) __stcs(reinterpret_cast<uint4*>(p) + k, w[k]);
    } else {
        static_assert(sizeof(T) % 8 == 0 && alignof(T) >= 8, "path state records are whole 8-byte words");
        constexpr int n = int(sizeof(T) / 8);
        unsigned long long w[n];
        memcpy(w, &v, sizeof(T));
#pragma unroll
        for (int k = 0; k < n; ++k) __stcs(reinterpret_cast<unsigned long long*>(p) + k, w[k]);
    }
#else
    *p = v;
#endif
}

// A pending next-event visibility query and its contribution if the segment is clear.
template <class R>
struct alignas(16) ShadowRay {
    double o[3];
    R d[3];
    double tmax;          // Inf for the sun
    uint32_t region;      // region the segment starts in
    uint32_t endRegion;   // region it must arrive in (kNone: the ambient region for the sun)
    uint32_t depB, depP;
    uint32_t endB;        // the light's boundary (kNone: the sun, or an eye the ray connects to)
    uint32_t path;
    float errN;
    float contrib[4];     // beta * f * Le * cos * w / pdf, before transmittance
};
static_assert(sizeof(ShadowRay<float>) == 96, "a mixed-precision shadow record stays six 16-byte words");

struct Queues {
    uint32_t* active[2];
    uint32_t* surface;        // surface events with any optics
    uint32_t* shadow;
    uint32_t* counts;         // [0], [1] active ping-pong, [2] surface, [3] shadow, [4], [5] fetch
                              // counters of the persistent kernels, [6] simple surface
    uint32_t* surfaceSimple;  // surface events on Lambertian, absorbing and detecting boundaries
};

struct StatCounters {
    unsigned long long paths, segments, inconsistencies, leaks, shadowRays, faults;
};

template <class R>
struct PathBuffers {
    PathRay<R>* ray;
    PathSpec<R>* spec;
    PathAux* aux;
    HitRec* hit;
    ShadowRay<R>* shadow;  // indexed by shadow-queue position
    float* sampleXyz;      // 3 per path slot: the path's XYZ estimate once the batch is done
};

struct PassParams {
    uint64_t seed;
    int32_t maxDepth, rrDepth;
    int32_t wavelengthMode;
    float lambdaMin, lambdaMax;
    float fresnelFloor;
    uint32_t nPixels;        // detector pixels
    uint32_t nPaths;         // paths in this batch: nPixels * samples
    uint32_t streamBase;     // PCG32 stream of the batch's first sample
    int32_t anyHitShadows;   // 1: no null boundaries, shadow rays stop at the first crossing
    // The adjoint's first phase: a path about to meet boundary ckptBoundary (kNone: never) stops there
    // and leaves its state as a PathCheckpoint (slot from ckptCount) for the derivative replay.
    uint32_t ckptBoundary = kNone;
    uint32_t* ckptCount = nullptr;
    void* ckpt = nullptr;
};

// A path's state at the surface event where it first meets the heightfield: what kSurface would
// load for it (after the free flight of the segment), and the hit.
template <class R>
struct alignas(16) PathCheckpoint {
    PathRay<R> ray;
    PathSpec<R> spec;
    PathAux aux;
    HitRec hit;
};

}  // namespace owec
