// Device throughput probes (peaks.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

namespace owec {

// FP32 and FP64 fused multiply-add rates (flop/s) and the L2 read bandwidth (bytes/s) of the current
// device, measured on stream s: out[0], out[1], out[2]. sms: its multiprocessors; l2Bytes: its L2 size.
void measurePeaks(int sms, size_t l2Bytes, cudaStream_t s, double out[3]);

}  // namespace owec
