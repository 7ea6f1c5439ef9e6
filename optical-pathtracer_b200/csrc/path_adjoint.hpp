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
// d(sum_p g_p . film_p)/d heights into t.dH. fixedDecisions: the derivative of the estimator at
// fixed random numbers (branch and roulette probabilities attached) instead of the unbiased gradient
// of the expected film. With ckpt, the paths are resumed from the *ckptCount checkpoints
// (PathCheckpoint records of the precision `mode`) the wavefront left at their first heightfield
// surface events, instead of replayed from the camera.
void launchPathAdjoint(int mode, const DeviceScene& sc, const PassParams& pp, const HeightfieldParams& hf,
                       const PathAdjointTargets& t, bool fixedDecisions, const void* ckpt, const uint32_t* ckptCount,
                       int grid, cudaStream_t s);
// Bytes of one path checkpoint in precision mode `mode`.
size_t pathCheckpointBytes(int mode);

}  // namespace owec
