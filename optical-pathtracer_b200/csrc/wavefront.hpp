// Launchers of the wavefront kernels (wavefront.cu), one instantiation per precision mode.
#pragma once

#include <cuda_runtime.h>

#include "path_state.cuh"
#include "splat.cuh"

namespace owec {

template <int M>
using ModeR = typename Mode<M>::R;

size_t traversalSharedBytes(int block);
void configureKernels();

template <int M>
void launchGenerate(const DeviceScene&, const PassParams&, const PathBuffers<ModeR<M>>&, const Queues&, StatCounters*,
                    cudaStream_t);
template <int M>
void launchIntersect(const DeviceScene&, const PathBuffers<ModeR<M>>&, const Queues&, int cur, StatCounters*,
                     uint32_t* fetch, int grid, cudaStream_t);
template <int M>
void launchMedium(const DeviceScene&, const PassParams&, const PathBuffers<ModeR<M>>&, const Queues&, int cur,
                  StatCounters*, int grid, cudaStream_t);
template <int M>
void launchSurface(const DeviceScene&, const PassParams&, const PathBuffers<ModeR<M>>&, const Queues&, int cur,
                   StatCounters*, int grid, cudaStream_t);
template <int M>
void launchShadow(const DeviceScene&, const PassParams&, const PathBuffers<ModeR<M>>&, const Queues&, StatCounters*,
                  uint32_t* fetch, uint8_t* vis, int grid, cudaStream_t);
// The light integrator's connections to the eye: their visibility, transmittance and splats.
template <int M>
void launchConnect(const DeviceScene&, const PassParams&, const PathBuffers<ModeR<M>>&, const Queues&, StatCounters*,
                   uint32_t* fetch, uint8_t* vis, const SplatTarget& film, int grid, cudaStream_t);
void launchResolve(const double* film, const double* comp, const double* samples, uint32_t nPixels, double* xyz,
                   cudaStream_t);
// out[i] = film[i] - comp[i] (the compensated sums as plain sums), n values, on stream s.
void launchFoldFilm(const double* film, const double* comp, double* out, size_t n, cudaStream_t s);
template <int M>
void launchFilm(const DeviceScene&, const PassParams&, const PathBuffers<ModeR<M>>&, double* film, double* comp,
                double* samples, uint32_t spp, cudaStream_t);
template <int M>
void launchCastRays(const DeviceScene&, uint64_t n, const double* o, const double* d, uint32_t* b, uint32_t* p,
                    double* t, int grid, cudaStream_t);
void launchCastRaysF(const DeviceScene&, uint64_t n, const float* o, const float* d, uint32_t* b, uint32_t* p, float* t,
                     int grid, cudaStream_t);
void launchMaterialize(const uint32_t* leafOrder, uint32_t n, const float4* tri, const double* tri64, PrimRec* prims,
                       PrimRec64* prims64, cudaStream_t);

}  // namespace owec
