// Library-wide entry points of the C ABI: version, error text, device properties.

#include <atomic>
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

// ---- launch parameters: one value per key for the process, read at every launch
namespace {
struct Param {
    int key;
    int64_t lo, hi, def;
};
constexpr Param kParams[] = {
    {CB_PARAM_CHAIN_TILE, 0, 65536, 0},
    {CB_PARAM_INFLATE_FORM, 1, 3, 3},
    {CB_PARAM_DECODE_ROOT, 6, 8, 7},
    {CB_PARAM_COPY_WARPS, 2, 24, 12},
    {CB_PARAM_DECODE_STEPS, 1, 64, 16},
    {CB_PARAM_DECODE_PREFETCH, 0, 16, 4},
    {CB_PARAM_SPLIT_MIN_JOBS, 0, 1LL << 40, 8192},
    {CB_PARAM_COPY_UNITS, 1, 4, 2},
    {CB_PARAM_DECODE_PIPELINE, 0, 2, 1},
};
constexpr int kNParams = sizeof(kParams) / sizeof(kParams[0]);
std::atomic<int64_t> g_param[kNParams] = {};
std::atomic<bool> g_param_set[kNParams] = {};

int param_index(int key) {
    for (int i = 0; i < kNParams; i++)
        if (kParams[i].key == key) return i;
    return -1;
}
}  // namespace

int64_t cb_param(int key) {
    const int i = param_index(key);
    if (i < 0) return 0;
    return g_param_set[i].load(std::memory_order_acquire) ? g_param[i].load(std::memory_order_relaxed) : kParams[i].def;
}

extern "C" int64_t cb_get_param(int key) { return param_index(key) < 0 ? -1 : cb_param(key); }

extern "C" int cb_set_param(int key, int64_t value) {
    const int i = param_index(key);
    if (i < 0) return cb_set_error_text(CB_ERR_ARG, "cb_set_param: unknown key");
    if (value == -1) {  // back to the default
        g_param_set[i].store(false, std::memory_order_release);
        return CB_OK;
    }
    if (value < kParams[i].lo || value > kParams[i].hi)
        return cb_set_error_text(CB_ERR_ARG, "cb_set_param: value out of range");
    if (key == CB_PARAM_CHAIN_TILE && value && (value < 2048 || (value & (value - 1))))
        return cb_set_error_text(CB_ERR_ARG, "cb_set_param: the chain tile is 0 (by size) or a power of two from 2048 to 65536");
    if (key == CB_PARAM_COPY_UNITS && value == 3)
        return cb_set_error_text(CB_ERR_ARG, "cb_set_param: copy units per lane are 1, 2 or 4");
    if (key == CB_PARAM_COPY_WARPS && value != 2 && value != 3 && value != 6 && value != 12 && value != 24)
        return cb_set_error_text(CB_ERR_ARG, "cb_set_param: copy warps per CTA are 2, 3, 6, 12 or 24");
    g_param[i].store(value, std::memory_order_relaxed);
    g_param_set[i].store(true, std::memory_order_release);
    return CB_OK;
}

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
