// Throughput probes of the device the bench's roofline divides by, where no driver-measured figure
// exists: the FP32 and FP64 fused multiply-add rates (the shading and traversal arithmetic's issue
// ceiling) and the L2 read bandwidth (the ceiling of a BVH that stays resident in the L2).
//
// Each probe is one kernel over the whole device, timed with CUDA events after a warm-up launch:
//   kFma     eight independent FMA chains per thread, 2 flops per FMA;
//   kL2Read  128-bit loads that bypass L1 (ld.global.cg) over a buffer a quarter of the L2's size,
//            read again and again, so that every load after the first pass hits the L2.
// The results are stored only when a value no input can produce appears, so nothing is removed as
// dead code.
#include <cuda_runtime.h>

#include <stdexcept>
#include <string>

#include "peaks.hpp"

namespace owec {

namespace {

template <class T>
__global__ void __launch_bounds__(256) kFma(T a0, T b, int iters, T* sink) {
    T a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = a0 + T(threadIdx.x + k);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) a[k] = fma(a[k], b, T(1e-7));
    }
    T s = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += a[k];
    if (s == T(-1.2345e30)) sink[threadIdx.x] = s;
}

__global__ void __launch_bounds__(256) kL2Read(const uint4* buf, size_t n, int reps, unsigned* sink) {
    unsigned acc = 0;
    const size_t stride = size_t(gridDim.x) * blockDim.x;
    for (int r = 0; r < reps; ++r)
        for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += stride) {
            const uint4 v = __ldcg(buf + i);
            acc ^= v.x + v.y + v.z + v.w;
        }
    if (acc == 0x9e3779b9u) sink[threadIdx.x] = acc;
}

struct Timer {
    cudaEvent_t a, b;
    cudaStream_t s;
    explicit Timer(cudaStream_t st) : s(st) {
        cudaEventCreate(&a);
        cudaEventCreate(&b);
    }
    ~Timer() {
        cudaEventDestroy(a);
        cudaEventDestroy(b);
    }
    void start() { cudaEventRecord(a, s); }
    double stop() {
        cudaEventRecord(b, s);
        cudaEventSynchronize(b);
        float ms = 0;
        cudaEventElapsedTime(&ms, a, b);
        return ms * 1e-3;
    }
};

template <class T>
double fmaRate(int sms, cudaStream_t s, T* sink) {
    const int blocks = sms * 8, threads = 256, iters = 1 << 14;
    kFma<T><<<blocks, threads, 0, s>>>(T(1), T(0.999999), 256, sink);  // warm-up
    Timer t(s);
    t.start();
    kFma<T><<<blocks, threads, 0, s>>>(T(1), T(0.999999), iters, sink);
    const double sec = t.stop();
    return 2.0 * 8 * double(iters) * blocks * threads / sec;
}

}  // namespace

void measurePeaks(int sms, size_t l2Bytes, cudaStream_t s, double out[3]) {
    void* sink = nullptr;
    void* buf = nullptr;
    const size_t bytes = (l2Bytes / 4) & ~size_t(255);
    if (cudaMalloc(&sink, 256 * sizeof(double)) != cudaSuccess || cudaMalloc(&buf, bytes) != cudaSuccess) {
        cudaFree(sink);
        throw std::runtime_error("device peaks: allocation failed");
    }
    cudaMemsetAsync(buf, 1, bytes, s);
    out[0] = fmaRate<float>(sms, s, static_cast<float*>(sink));
    out[1] = fmaRate<double>(sms, s, static_cast<double*>(sink));
    const size_t n = bytes / sizeof(uint4);
    const int reps = 64;
    kL2Read<<<sms * 8, 256, 0, s>>>(static_cast<const uint4*>(buf), n, 2, static_cast<unsigned*>(sink));  // resident
    Timer t(s);
    t.start();
    kL2Read<<<sms * 8, 256, 0, s>>>(static_cast<const uint4*>(buf), n, reps, static_cast<unsigned*>(sink));
    const double sec = t.stop();
    out[2] = double(bytes) * reps / sec;
    const cudaError_t e = cudaGetLastError();
    cudaFree(buf);
    cudaFree(sink);
    if (e != cudaSuccess) throw std::runtime_error(std::string("device peaks: ") + cudaGetErrorString(e));
}

}  // namespace owec
