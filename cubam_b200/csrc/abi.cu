// Library-wide entry points of the C ABI: version, error text, device properties.

#include <cstdio>
#include <cstring>

#include "common.cuh"

static thread_local char g_err[256] = "";

int cb_set_error(cudaError_t e) {
    if (e == cudaSuccess) return CB_OK;
    std::snprintf(g_err, sizeof(g_err), "%s: %s", cudaGetErrorName(e), cudaGetErrorString(e));
    return CB_ERR_CUDA;
}

int cb_set_error_text(int code, const char* text) {
    std::snprintf(g_err, sizeof(g_err), "%s", text);
    return code;
}

extern "C" const char* cb_version(void) { return "cubam_b200 0.1.0 (sm_100a)"; }

extern "C" const char* cb_last_error(void) { return g_err; }

extern "C" int cb_device_sm_count(void) {
    static int cache[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    if (!cache[dev]) {
        int v = 0;
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) v = 148;
        cache[dev] = v;
    }
    return cache[dev];
}
