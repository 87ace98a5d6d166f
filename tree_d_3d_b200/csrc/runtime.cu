// Library-wide entry points: version and the per-thread last CUDA error.
#include <string.h>

#include "common.cuh"

namespace {
thread_local char g_last_error[256] = "";
}

int td3_cuda_error(cudaError_t err) {
    const char* msg = cudaGetErrorString(err);
    strncpy(g_last_error, msg ? msg : "unknown CUDA error", sizeof(g_last_error) - 1);
    g_last_error[sizeof(g_last_error) - 1] = '\0';
    return TD3_ECUDA;
}

void td3_set_error(const char* message) {
    strncpy(g_last_error, message ? message : "", sizeof(g_last_error) - 1);
    g_last_error[sizeof(g_last_error) - 1] = '\0';
}

extern "C" int td3_version(void) { return 100; }

extern "C" const char* td3_last_error(void) { return g_last_error; }
