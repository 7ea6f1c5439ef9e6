// Device buffers owned by a context (RAII) and the CUDA error check used by the host runtime.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <stdexcept>
#include <string>

namespace owec {

struct CudaError : std::runtime_error {
    cudaError_t code;
    CudaError(cudaError_t c, const std::string& what) : std::runtime_error(what), code(c) {}
};

#define OWEC_CUDA(call)                                                                                    \
    do {                                                                                                   \
        cudaError_t err_ = (call);                                                                         \
        if (err_ != cudaSuccess)                                                                           \
            throw ::owec::CudaError(err_, std::string(#call) + ": " + cudaGetErrorString(err_));         \
    } while (0)

template <class T>
class DBuf {
public:
    DBuf() = default;
    explicit DBuf(size_t n) { resize(n); }
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    DBuf(DBuf&& o) noexcept : p_(o.p_), n_(o.n_) { o.p_ = nullptr; o.n_ = 0; }
    DBuf& operator=(DBuf&& o) noexcept {
        if (this != &o) { release(); p_ = o.p_; n_ = o.n_; o.p_ = nullptr; o.n_ = 0; }
        return *this;
    }
    ~DBuf() { release(); }
    // Grows to hold at least n elements (contents are not kept).
    void reserve(size_t n) {
        if (n <= n_) return;
        resize(n);
    }
    void resize(size_t n) {
        release();
        if (n == 0) return;
        void* p = nullptr;
        cudaError_t e = cudaMalloc(&p, n * sizeof(T));
        if (e != cudaSuccess) throw CudaError(e, "cudaMalloc of " + std::to_string(n * sizeof(T)) + " bytes failed");
        p_ = static_cast<T*>(p);
        n_ = n;
    }
    void release() {
        if (p_) cudaFree(p_);
        p_ = nullptr;
        n_ = 0;
    }
    T* get() const { return p_; }
    size_t size() const { return n_; }
    size_t bytes() const { return n_ * sizeof(T); }
    void upload(const T* src, size_t n, cudaStream_t s) {
        reserve(n);
        if (n) OWEC_CUDA(cudaMemcpyAsync(p_, src, n * sizeof(T), cudaMemcpyHostToDevice, s));
    }

private:
    T* p_ = nullptr;
    size_t n_ = 0;
};

}  // namespace owec
