// Device memory and stream helpers (single B200, one context per process).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <memory>
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

// Stream-ordered device memory.  While an AllocStream scope is active on this
// thread, DBuf allocations come from the library's own memory pool on that stream
// (cudaMallocFromPoolAsync) and are released on it (cudaFreeAsync), so freeing and
// re-allocating between the steps of a sweep neither synchronises the device nor
// returns memory to the driver.  Outside a scope, or once the stream has been
// retired, plain cudaMalloc / cudaFree are used.
cudaStream_t& alloc_stream();
struct AllocStream {
    cudaStream_t prev;
    explicit AllocStream(cudaStream_t s) : prev(alloc_stream()) { alloc_stream() = s; }
    ~AllocStream() { alloc_stream() = prev; }
    AllocStream(const AllocStream&) = delete;
    AllocStream& operator=(const AllocStream&) = delete;
};
void* device_alloc(std::size_t bytes, cudaStream_t* used);
void device_free(void* p, cudaStream_t used);
// streams that may carry pool frees; retire (after synchronising) before destroying one
void register_stream(cudaStream_t s);
void retire_stream(cudaStream_t s);

// Host vector whose resize() leaves trivially constructible elements uninitialised
// (for large work lists that are filled in parallel right after sizing).
template <class T>
struct NoInitAlloc : std::allocator<T> {
    template <class U> struct rebind { using other = NoInitAlloc<U>; };
    NoInitAlloc() = default;
    template <class U> NoInitAlloc(const NoInitAlloc<U>&) noexcept {}
    template <class U> void construct(U* p) noexcept { ::new (static_cast<void*>(p)) U; }
    template <class U, class... Args> void construct(U* p, Args&&... a) { ::new (static_cast<void*>(p)) U(std::forward<Args>(a)...); }
};
template <class T>
using hvec = std::vector<T, NoInitAlloc<T>>;

// Owning device buffer.
template <class T>
class DBuf {
  public:
    DBuf() = default;
    explicit DBuf(std::size_t n) { alloc(n); }
    ~DBuf() { reset(); }
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    DBuf(DBuf&& o) noexcept : p_(o.p_), n_(o.n_), s_(o.s_) { o.p_ = nullptr; o.n_ = 0; o.s_ = nullptr; }
    DBuf& operator=(DBuf&& o) noexcept {
        if (this != &o) { reset(); p_ = o.p_; n_ = o.n_; s_ = o.s_; o.p_ = nullptr; o.n_ = 0; o.s_ = nullptr; }
        return *this;
    }
    void alloc(std::size_t n) {
        reset();
        if (n) p_ = static_cast<T*>(device_alloc(n * sizeof(T), &s_));
        n_ = n;
    }
    void reset() {
        if (p_) device_free(p_, s_);
        p_ = nullptr;
        n_ = 0;
        s_ = nullptr;
    }
    void upload(const T* h, std::size_t n, cudaStream_t s = 0) {
        if (n > n_) alloc(n);
        if (n) QCM_CUDA(cudaMemcpyAsync(p_, h, n * sizeof(T), cudaMemcpyHostToDevice, s));
    }
    template <class A>
    void upload(const std::vector<T, A>& v, cudaStream_t s = 0) { upload(v.data(), v.size(), s); }
    T* get() const { return p_; }
    std::size_t size() const { return n_; }

  private:
    T* p_ = nullptr;
    std::size_t n_ = 0;
    cudaStream_t s_ = nullptr;  // stream the pool allocation is ordered on (null: cudaMalloc)
};

inline void ensure_device() {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) throw qcm::cuda_error("no CUDA device available (there is no CPU fallback)");
}

}  // namespace qcm
