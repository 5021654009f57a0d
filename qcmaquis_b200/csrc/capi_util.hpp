// Error handling shared by the C-ABI translation units: every entry point returns
// an int status and never exits the process (the reference exit()s on CUDA and
// cuBLAS errors, utils/cuda_helpers.hpp:41-50; a library must not).
#pragma once

#include <exception>
#include <new>
#include <stdexcept>
#include <string>

#include "../../include/qcm_b200.h"

namespace qcm {
void set_error(const std::string& msg);
inline int fail(int code, const std::string& msg) {
    set_error(msg);
    return code;
}
struct cuda_error : std::runtime_error {
    using std::runtime_error::runtime_error;
};
}  // namespace qcm

#define QCM_TRY try {
#define QCM_CATCH                                                              \
    }                                                                          \
    catch (const qcm::cuda_error& e) { return qcm::fail(QCM_ERR_CUDA, e.what()); } \
    catch (const std::bad_alloc&) { return qcm::fail(QCM_ERR_NOMEM, "out of memory"); } \
    catch (const std::exception& e) { return qcm::fail(QCM_ERR_INTERNAL, e.what()); } \
    catch (...) { return qcm::fail(QCM_ERR_INTERNAL, "unknown error"); }
