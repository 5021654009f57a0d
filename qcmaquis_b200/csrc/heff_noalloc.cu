// H_eff apply for callers that cannot allocate device memory.
//
// Some host codes cannot call cudaMalloc at the point where they need H.psi:
// a code whose device memory is owned by its own caching allocator (which may
// hold nearly all of HBM, so a cudaMalloc here fails or fragments it), or an
// inner solver loop that must not stall, since cudaFree synchronises the whole
// device.  qcm_heff_apply_device_noalloc serves them.  It runs the same
// T-GEMM -> S build -> split-K L.S kernels as qcm_heff_apply_device.  Its
// scratch (T, S and the split-K partial tiles) is not the plan's buffers but
// the fixed array below, which every GPU that loads this library holds until
// the process exits.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/qcm_b200.h"
#include "capi_types.hpp"
#include "capi_util.hpp"
#include "device.hpp"
#include "heff.hpp"

namespace {

// QCM_NOALLOC_SCRATCH_DOUBLES doubles (64 MiB), shared by every call on a device.
static __device__ __align__(256) double g_noalloc_scratch[QCM_NOALLOC_SCRATCH_DOUBLES];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device, looked up once per
// device (the array's host-side name is only a stand-in, never a device address).
double* scratch_for_current_device() {
    int dev = 0;
    QCM_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) throw std::runtime_error("qcm_heff_apply_device_noalloc: device index out of range");
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_ptr[dev]) {
        void* ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess)
            throw qcm::cuda_error(std::string("cudaGetSymbolAddress(noalloc scratch): ") + cudaGetErrorString(e));
        g_scratch_ptr[dev] = static_cast<double*>(ptr);
    }
    return g_scratch_ptr[dev];
}

uint64_t round32(uint64_t n) { return (n + 31) / 32 * 32; }

}  // namespace

extern "C" int qcm_heff_apply_device_noalloc(qcm_heff* h, const double* x_dev, double* y_dev) {
    QCM_TRY
    if (!h || !x_dev || !y_dev) return qcm::fail(QCM_ERR_ARG, "qcm_heff_apply_device_noalloc: NULL argument");
    if (!h->ctx) return qcm::fail(QCM_ERR_ARG, "qcm_heff_apply_device_noalloc: host-only plan");
    qcm::HeffPlan& p = *h->p;
    const uint64_t need = round32(p.t_len) + round32(p.s_len) + round32(p.p_len);
    if (need > QCM_NOALLOC_SCRATCH_DOUBLES)
        return qcm::fail(QCM_ERR_ARG, "qcm_heff_apply_device_noalloc: plan needs " + std::to_string(need) +
                                          " scratch doubles, the fixed array holds " +
                                          std::to_string(uint64_t(QCM_NOALLOC_SCRATCH_DOUBLES)) +
                                          "; use qcm_heff_apply_device for this plan");
    QCM_CUDA(cudaSetDevice(h->ctx->device));
    double* base = scratch_for_current_device();
    double* Tb = base;
    double* Sb = Tb + round32(p.t_len);
    double* Pb = Sb + round32(p.s_len);
    // T and the partial tiles are fully written by their kernels; the S buffer is cleared
    // inside the apply (rows without coefficients must read as zero).
    qcm::heff_apply_device_scratch(p, x_dev, y_dev, Tb, Sb, Pb);
    return QCM_OK;
    QCM_CATCH
}
