// Library-level C ABI helpers: error strings and version.
#include <stdio.h>
#include <string.h>

#include "gm_common.cuh"

namespace gm {

static thread_local char g_last_error[512] = "";

void set_error(const char *where, cudaError_t err)
{
    snprintf(g_last_error, sizeof(g_last_error), "%s: %s (%d)", where, cudaGetErrorString(err),
             (int)err);
}

void set_error_msg(const char *msg) { snprintf(g_last_error, sizeof(g_last_error), "%s", msg); }

}  // namespace gm

extern "C" const char *gm_last_error(void) { return gm::g_last_error; }

extern "C" const char *gm_version(void) { return "gm_b200 0.1 sm_100a"; }
