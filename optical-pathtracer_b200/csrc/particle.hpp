// Launchers of the particle-tracing kernels (particle.cu): the "light" integrator.
#pragma once

#include <cuda_runtime.h>

#include "device_scene.cuh"
#include "path_state.cuh"
#include "splat.cuh"
#include "wavefront.hpp"

namespace owec {

struct ParticleParams {
    uint64_t seed;
    uint64_t stream;        // PCG32 stream of the pass's particles: the index of its first sample
    uint64_t first;         // index within the pass of the batch's first particle
    int32_t maxDepth, rrDepth;
    int32_t wavelengthMode;
    float lambdaMin, lambdaMax;
    float fresnelFloor;
    double pSky;            // probability that a particle leaves the sky rather than a light
    double discRadius;      // radius of the disc that light from beyond the world leaves from
    double discCentre[3];   // its centre, the scene's (camera-relative)
    double pixelArea;       // observer: a pixel's area on the image plane at unit distance;
                            // sensor: a pixel's area on the sensor
};

// Starts n particles (P.first onward) in path slots 0..n-1: active queue 0, and the emitters' own
// connections in the shadow queue.
template <int M>
void launchEmit(const DeviceScene&, const ParticleParams&, const PathBuffers<ModeR<M>>&, const Queues&, StatCounters*,
                const SplatTarget&, uint32_t n, cudaStream_t);
// One event of every particle in active queue `cur` (after its closest-hit query): survivors go to
// the other active queue, connections to the shadow queue, sensor records to the film.
template <int M>
void launchParticleEvent(const DeviceScene&, const ParticleParams&, const PathBuffers<ModeR<M>>&, const Queues&,
                         int cur, StatCounters*, const SplatTarget&, int grid, cudaStream_t);

// XYZ per pixel from the splat sums: sum * 2^kSplatExp0 * scale.
void launchResolveSplats(const unsigned long long* splat, uint32_t nPixels, double scale, double* xyz, cudaStream_t s);

}  // namespace owec
