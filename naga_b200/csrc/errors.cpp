// Status codes and the per-thread error message of the C ABI.
#include "naga_internal.hpp"

namespace naga {

static thread_local std::string g_last_error;

int set_error(int rc, const std::string& msg) {
    if (rc != NAGA_OK) g_last_error = msg;
    return rc;
}

void clear_error() { g_last_error.clear(); }

}  // namespace naga

extern "C" const char* naga_last_error(void) { return naga::g_last_error.c_str(); }

extern "C" int naga_version(void) { return 100; }
