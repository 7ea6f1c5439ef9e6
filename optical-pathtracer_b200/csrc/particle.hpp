// Launcher of the particle-tracing kernel (particle.cu): the "light" integrator.
#pragma once

#include <cuda_runtime.h>

#include "device_scene.cuh"
#include "path_state.cuh"

namespace owec {

// Words of a film pixel's particle splats: three channels (X, Y, Z), each a 192-bit fixed-point sum
// in three 64-bit words, least significant first.
constexpr int kSplatWordsPerChannel = 3;
constexpr int kSplatWordsPerPixel = 3 * kSplatWordsPerChannel;
// The weight of a channel's lowest bit: 2^kSplatExp0. The sum spans 2^-80 .. 2^112.
constexpr int kSplatExp0 = -80;

struct ParticleParams {
    uint64_t seed;
    uint64_t stream;        // PCG32 stream of the pass's particles: the index of its first sample
    uint64_t first, n;      // the particles [first, first + n) of the pass
    int32_t maxDepth, rrDepth;
    int32_t wavelengthMode;
    float lambdaMin, lambdaMax;
    float fresnelFloor;
    int32_t anyHitShadows;  // 1: no null boundaries, connections stop at the first crossing
    double pSky;            // probability that a particle leaves the sky rather than a light
    double discRadius;      // radius of the disc that light from beyond the world leaves from
    double discCentre[3];   // its centre, the scene's (camera-relative)
    double pixelArea;       // observer: a pixel's area on the image plane at unit distance;
                            // sensor: a pixel's area on the sensor
};

// n particles of a pass, splatted into `splat` (kSplatWordsPerPixel words per pixel).
void launchParticles(int mode, const DeviceScene& sc, const ParticleParams& P, unsigned long long* splat,
                     StatCounters* st, int grid, cudaStream_t s);

// XYZ per pixel from the splat sums: sum * 2^kSplatExp0 * scale.
void launchResolveSplats(const unsigned long long* splat, uint32_t nPixels, double scale, double* xyz, cudaStream_t s);

}  // namespace owec
