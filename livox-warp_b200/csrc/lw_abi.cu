// Status plumbing of the C ABI: per-thread error messages, the library version and the SM count the persistent
// kernels size their grids with.
#include <stdarg.h>
#include <stdio.h>
#include "lw_common.cuh"

namespace lw {

static thread_local char g_err[512] = "";

int set_error(int code, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

int check_cuda(cudaError_t e, const char* what) {
    return set_error(LW_ECUDA, "%s: %s (%s)", what, cudaGetErrorString(e), cudaGetErrorName(e));
}

int device_sms() {
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 1;
    static thread_local int cached_dev = -1, cached_sms = 0;
    if (dev == cached_dev) return cached_sms;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 1;
    cached_dev = dev;
    cached_sms = sms;
    return sms;
}

}  // namespace lw

extern "C" {

const char* lw_version(void) { return "livox-b200 0.1.0 (sm_100a)"; }

const char* lw_last_error(void) { return lw::g_err; }

int lw_device_sms(int* out_sms) {
    if (!out_sms) return lw::set_error(LW_EINVAL, "lw_device_sms: null argument");
    int dev = 0;
    LW_CUDA(cudaGetDevice(&dev));
    *out_sms = lw::device_sms();
    return LW_OK;
}

}  // extern "C"
