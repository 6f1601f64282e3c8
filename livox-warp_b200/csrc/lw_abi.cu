// Status plumbing of the C ABI: per-thread error messages, the library version and the SM count the persistent
// kernels size their grids with.
#include <stdarg.h>
#include <stdio.h>
#include <string.h>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>
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

static long long g_launches = 0;
static std::mutex g_launch_mu;

void count_launches(int n) {
    std::lock_guard<std::mutex> g(g_launch_mu);
    g_launches += n;
}

// ---- opt-in launch timing --------------------------------------------------------------------------------
// When enabled, the entry points bracket their main launches with CUDA events on the launching stream; the
// elapsed times are summed per name when read. Off by default: no events are recorded.
namespace {
struct Pending {
    cudaEvent_t a, b;
};
struct Slot {
    std::vector<Pending> pending;
    double ms = 0.0;
    long long count = 0;
};
std::mutex g_prof_mu;
bool g_prof_on = false;
std::unordered_map<std::string, Slot> g_prof;
std::vector<cudaEvent_t> g_free_events;

cudaEvent_t take_event() {
    if (!g_free_events.empty()) {
        cudaEvent_t e = g_free_events.back();
        g_free_events.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}
}  // namespace

ProfScope::ProfScope(const char* name, cudaStream_t s) : name_(name), s_(s), a_(nullptr) {
    std::lock_guard<std::mutex> g(g_prof_mu);
    if (!g_prof_on) return;
    a_ = take_event();
    cudaEventRecord((cudaEvent_t)a_, s_);
}

ProfScope::~ProfScope() {
    if (!a_) return;
    std::lock_guard<std::mutex> g(g_prof_mu);
    cudaEvent_t b = take_event();
    cudaEventRecord(b, s_);
    g_prof[name_].pending.push_back({(cudaEvent_t)a_, b});
}

}  // namespace lw

extern "C" {

int lw_prof_enable(int on) {
    std::lock_guard<std::mutex> g(lw::g_prof_mu);
    lw::g_prof_on = on != 0;
    return LW_OK;
}

int lw_prof_read(const char* name, double* ms, int64_t* count) {
    if (!name || !ms || !count) return lw::set_error(LW_EINVAL, "lw_prof_read: null argument");
    std::lock_guard<std::mutex> g(lw::g_prof_mu);
    auto it = lw::g_prof.find(name);
    if (it == lw::g_prof.end()) {
        *ms = 0.0;
        *count = 0;
        return LW_OK;
    }
    lw::Slot& sl = it->second;
    for (auto& p : sl.pending) {
        float t = 0.0f;
        LW_CUDA(cudaEventSynchronize(p.b));
        LW_CUDA(cudaEventElapsedTime(&t, p.a, p.b));
        sl.ms += t;
        sl.count += 1;
        lw::g_free_events.push_back(p.a);
        lw::g_free_events.push_back(p.b);
    }
    sl.pending.clear();
    *ms = sl.ms;
    *count = sl.count;
    return LW_OK;
}

int64_t lw_launches(int reset) {
    std::lock_guard<std::mutex> g(lw::g_launch_mu);
    int64_t v = lw::g_launches;
    if (reset) lw::g_launches = 0;
    return v;
}

int lw_prof_reset(void) {
    std::lock_guard<std::mutex> g(lw::g_prof_mu);
    for (auto& kv : lw::g_prof) {
        for (auto& p : kv.second.pending) {
            lw::g_free_events.push_back(p.a);
            lw::g_free_events.push_back(p.b);
        }
    }
    lw::g_prof.clear();
    return LW_OK;
}

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
