// Stream-ordered device memory pool (see device.hpp).
#include <map>
#include <mutex>
#include <set>

#include "device.hpp"

namespace qcm {

namespace {
std::mutex g_mu;
std::set<cudaStream_t> g_live;
std::map<int, cudaMemPool_t> g_pools;

cudaMemPool_t pool_for_current_device() {
    int dev = 0;
    QCM_CUDA(cudaGetDevice(&dev));
    auto it = g_pools.find(dev);
    if (it != g_pools.end()) return it->second;
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool;
    QCM_CUDA(cudaMemPoolCreate(&pool, &props));
    uint64_t keep = ~uint64_t(0);  // keep freed memory in the pool between steps
    QCM_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    g_pools[dev] = pool;
    return pool;
}
}  // namespace

cudaStream_t& alloc_stream() {
    thread_local cudaStream_t s = nullptr;
    return s;
}

void register_stream(cudaStream_t s) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_live.insert(s);
}

void retire_stream(cudaStream_t s) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_live.erase(s);
}

void* device_alloc(std::size_t bytes, cudaStream_t* used) {
    void* p = nullptr;
    cudaStream_t s = alloc_stream();
    if (s) {
        std::lock_guard<std::mutex> lk(g_mu);
        if (g_live.count(s)) {
            QCM_CUDA(cudaMallocFromPoolAsync(&p, bytes, pool_for_current_device(), s));
            *used = s;
            return p;
        }
    }
    QCM_CUDA(cudaMalloc(&p, bytes));
    *used = nullptr;
    return p;
}

void device_free(void* p, cudaStream_t used) {
    if (!p) return;
    if (used) {
        {
            std::lock_guard<std::mutex> lk(g_mu);
            if (g_live.count(used)) {
                cudaFreeAsync(p, used);
                return;
            }
        }
        // pool memory whose stream was retired: cudaFree does not wait for it, so drain the device first
        cudaDeviceSynchronize();
    }
    cudaFree(p);
}

}  // namespace qcm
