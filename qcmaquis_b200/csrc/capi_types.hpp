// Definitions of the opaque C-ABI handles shared by the translation units that use them.
#pragma once

#include <cuda_runtime.h>

#include <memory>

#include "heff.hpp"

struct qcm_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
};

struct qcm_boundary {
    qcm_ctx* ctx = nullptr;
    qcm::DevBoundary b;
};

struct qcm_heff {
    qcm_ctx* ctx = nullptr;
    std::unique_ptr<qcm::HeffPlan> p;
};
