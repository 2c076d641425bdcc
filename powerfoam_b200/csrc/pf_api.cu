// pf_api.cu -- error reporting and version of the C ABI.
#include <cstdio>
#include <cstring>

#include "pf_api.h"

static thread_local char g_err[512] = "";

int pf_fail(int code, const char* msg) {
    std::snprintf(g_err, sizeof(g_err), "%s", msg);
    return code;
}

int pf_check_launch(const char* where) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        std::snprintf(g_err, sizeof(g_err), "%s: %s", where, cudaGetErrorString(e));
        return PF_ERR_CUDA;
    }
    return PF_OK;
}

extern "C" int pf_abi_version(void) { return PF_ABI_VERSION; }

extern "C" const char* pf_last_error(void) { return g_err; }
