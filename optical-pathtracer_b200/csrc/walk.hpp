// Launcher of the forward light-walk kernel (walk.cu).
#pragma once

#include <cuda_runtime.h>

#include "device_scene.cuh"
#include "wavefront.hpp"

namespace owec {

// The heightfield a walk adjoint differentiates: its boundary, its mesh's triangles (vertex
// indices), and the world direction in which its heights raise the vertices.
struct HeightfieldParams {
    uint32_t boundary;
    const uint32_t* tris;
    double zdir[3];
};

// n walks starting at walk index `first`, binned into `bins` (width * height 64-bit fixed-point
// sums, 2^-32 per unit throughput); stats: [walks, binned, escaped, events, faults].
void launchWalk(int mode, const DeviceScene& sc, const owec_walk_desc& w, const Xform& targetToLocal, uint64_t first,
                uint64_t n, unsigned long long* bins, unsigned long long* stats, int grid, cudaStream_t s);

// Path-replay adjoint of n walks: accumulates scale * d(sum_b g_b bins_b)/d heights into dH; walks
// whose derivative could not be followed are counted in stats[4].
void launchWalkAdjoint(int mode, const DeviceScene& sc, const owec_walk_desc& w, const Xform& targetToLocal,
                       const HeightfieldParams& hf, uint64_t first, uint64_t n, double scale, const double* g,
                       double* dH, unsigned long long* stats, int grid, cudaStream_t s);

}  // namespace owec
