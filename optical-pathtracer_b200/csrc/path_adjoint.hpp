// Launcher of the camera-path adjoint kernel (path_adjoint.cu).
#pragma once

#include <cuda_runtime.h>

#include "device_scene.cuh"
#include "walk.hpp"
#include "wavefront.hpp"

namespace owec {

// What the adjoint replay reads and writes on the device.
struct PathAdjointTargets {
    const double* g;          // dLoss / dFilm: 3 per pixel (XYZ), row-major
    double invSamples;        // 1 / samples per pixel of the replayed film
    double* dH;               // height gradient, one per heightfield vertex (added to)
    double* replay;           // 3 per pixel: the replayed paths' mean XYZ (added to), or null
    unsigned long long* counters;  // [paths, paths that met the heightfield, dropped, faults]
};

// Replays the camera paths of pass settings pp (pp.nPaths of them from stream pp.streamBase) and adds
// d(sum_p g_p . film_p)/d heights into t.dH.
void launchPathAdjoint(int mode, const DeviceScene& sc, const PassParams& pp, const HeightfieldParams& hf,
                       const PathAdjointTargets& t, int grid, cudaStream_t s);

}  // namespace owec
