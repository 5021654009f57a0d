// C-ABI: error reporting and version.
#include <string>

#include "../../include/qcm_b200.h"
#include "capi_util.hpp"

namespace {
thread_local std::string g_last_error;
}

namespace qcm {
void set_error(const std::string& msg) { g_last_error = msg; }
}  // namespace qcm

extern "C" {
const char* qcm_last_error(void) { return g_last_error.c_str(); }
const char* qcm_version(void) { return "qcm_b200 0.1 (sm_100a)"; }
}
