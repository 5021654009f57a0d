// Device memory and stream helpers (single B200, one context per process).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <string>
#include <utility>
#include <vector>

#include "capi_util.hpp"

#define QCM_CUDA(call)                                                                                  \
    do {                                                                                                \
        cudaError_t e_ = (call);                                                                        \
        if (e_ != cudaSuccess)                                                                          \
            throw qcm::cuda_error(std::string(#call) + ": " + cudaGetErrorString(e_) + " (" + __FILE__ + \
                                  ":" + std::to_string(__LINE__) + ")");                               \
    } while (0)

namespace qcm {

// Owning device buffer (cudaMalloc / cudaFree).
template <class T>
class DBuf {
  public:
    DBuf() = default;
    explicit DBuf(std::size_t n) { alloc(n); }
    ~DBuf() { reset(); }
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    DBuf(DBuf&& o) noexcept : p_(o.p_), n_(o.n_) { o.p_ = nullptr; o.n_ = 0; }
    DBuf& operator=(DBuf&& o) noexcept {
        if (this != &o) { reset(); p_ = o.p_; n_ = o.n_; o.p_ = nullptr; o.n_ = 0; }
        return *this;
    }
    void alloc(std::size_t n) {
        reset();
        if (n) QCM_CUDA(cudaMalloc(&p_, n * sizeof(T)));
        n_ = n;
    }
    void reset() {
        if (p_) cudaFree(p_);
        p_ = nullptr;
        n_ = 0;
    }
    void upload(const T* h, std::size_t n, cudaStream_t s = 0) {
        if (n > n_) alloc(n);
        if (n) QCM_CUDA(cudaMemcpyAsync(p_, h, n * sizeof(T), cudaMemcpyHostToDevice, s));
    }
    void upload(const std::vector<T>& v, cudaStream_t s = 0) { upload(v.data(), v.size(), s); }
    T* get() const { return p_; }
    std::size_t size() const { return n_; }

  private:
    T* p_ = nullptr;
    std::size_t n_ = 0;
};

inline void ensure_device() {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) throw qcm::cuda_error("no CUDA device available (there is no CPU fallback)");
}

}  // namespace qcm
