// H_eff apply for callers that cannot allocate device memory.
//
// Some host codes cannot call cudaMalloc at the point where they need H.psi:
// a code whose device memory is owned by its own caching allocator (which may
// hold nearly all of HBM, so a cudaMalloc here fails or fragments it), or an
// inner solver loop that must not stall, since cudaFree synchronises the whole
// device.  qcm_heff_apply_device_noalloc serves them.  It runs the same
// T-GEMM -> S build -> split-K L.S kernels as qcm_heff_apply_device (FP64).
// Its scratch (T, S and the split-K partial tiles) is not the plan's buffers
// but the fixed array below, which every GPU that loads this library holds
// until the process exits.  Each context looks the array's device address up
// when it is created (qcm_ctx_create), so the apply itself does no set-up.
#include <cuda_runtime.h>

#include <string>

#include "../../include/qcm_b200.h"
#include "capi_types.hpp"
#include "capi_util.hpp"
#include "device.hpp"
#include "heff.hpp"

namespace {

// QCM_NOALLOC_SCRATCH_DOUBLES doubles (64 MiB), shared by every call on a device.
static __device__ __align__(256) double g_noalloc_scratch[QCM_NOALLOC_SCRATCH_DOUBLES];

}  // namespace

namespace qcm {

// The array's host-side name is only a stand-in: its device address on the current device comes
// from cudaGetSymbolAddress, which loads this file's module there if it is not loaded yet.
double* noalloc_scratch_address() {
    void* ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess) throw cuda_error(std::string("cudaGetSymbolAddress(noalloc scratch): ") + cudaGetErrorString(e));
    return static_cast<double*>(ptr);
}

}  // namespace qcm

namespace {

// makes a device current for one call and gives the caller's back
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        QCM_CUDA(cudaGetDevice(&prev));
        if (prev != dev) QCM_CUDA(cudaSetDevice(dev));
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

uint64_t round32(uint64_t n) { return (n + 31) / 32 * 32; }

}  // namespace

extern "C" int qcm_heff_apply_device_noalloc(qcm_heff* h, const double* x_dev, double* y_dev) {
    QCM_TRY
    if (!h || !x_dev || !y_dev) return qcm::fail(QCM_ERR_ARG, "qcm_heff_apply_device_noalloc: NULL argument");
    if (!h->ctx) return qcm::fail(QCM_ERR_ARG, "qcm_heff_apply_device_noalloc: host-only plan");
    qcm::HeffPlan& p = *h->p;
    if (p.sector_chunked())
        return qcm::fail(QCM_ERR_ARG, "qcm_heff_apply_device_noalloc: a chunked plan applies through qcm_heff_apply_device");
    const uint64_t need = round32(p.t_len) + round32(p.s_len) + round32(p.p_len);
    if (need > QCM_NOALLOC_SCRATCH_DOUBLES)
        return qcm::fail(QCM_ERR_ARG, "qcm_heff_apply_device_noalloc: plan needs " + std::to_string(need) +
                                          " scratch doubles, the fixed array holds " +
                                          std::to_string(uint64_t(QCM_NOALLOC_SCRATCH_DOUBLES)) +
                                          "; use qcm_heff_apply_device for this plan");
    if (!h->ctx->noalloc_scratch) return qcm::fail(QCM_ERR_INTERNAL, "qcm_heff_apply_device_noalloc: context without scratch address");
    DeviceGuard dg(h->ctx->device);
    double* base = h->ctx->noalloc_scratch;
    double* Tb = base;
    double* Sb = Tb + round32(p.t_len);
    double* Pb = Sb + round32(p.s_len);
    // T and the partial tiles are fully written by their kernels; the S buffer is cleared
    // inside the apply (rows without coefficients must read as zero).
    qcm::heff_apply_device_scratch(p, x_dev, y_dev, Tb, Sb, Pb);
    return QCM_OK;
    QCM_CATCH
}
