// Definitions of the opaque C-ABI handles shared by the translation units that use them.
#pragma once

#include <cuda_runtime.h>

#include <memory>

#include "heff.hpp"

struct qcm_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    // device address of the allocation-free apply's fixed scratch array on this device, looked
    // up when the context is created (qcm_heff_apply_device_noalloc)
    double* noalloc_scratch = nullptr;
};

namespace qcm {
// Device address of the allocation-free apply's scratch array on the current device
// (cudaGetSymbolAddress, which also loads the array's module there).
double* noalloc_scratch_address();
}  // namespace qcm

struct qcm_boundary {
    qcm_ctx* ctx = nullptr;
    qcm::DevBoundary b;
};

struct qcm_heff {
    qcm_ctx* ctx = nullptr;
    std::unique_ptr<qcm::HeffPlan> p;
};
