// Library-wide C ABI: status strings, last-error text, launch counting and the
// optional CUDA-event timing of kernel families.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdio>
#include <mutex>
#include <vector>

#include "fugal_host.h"

namespace {

thread_local char g_last_error[512] = "";

std::atomic<int64_t> g_launches{0};
std::atomic<int> g_timing_on{0};

struct Pending {
    int family;
    cudaEvent_t start, stop;
};

std::mutex g_mu;
std::vector<Pending> g_pending;
std::vector<cudaEvent_t> g_pool;
int64_t g_count[FUGAL_KERNEL_FAMILIES] = {0};
double g_ms[FUGAL_KERNEL_FAMILIES] = {0.0};

cudaEvent_t take_event() {
    if (!g_pool.empty()) {
        cudaEvent_t e = g_pool.back();
        g_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    return e;
}

// Fold completed pairs; with `block`, wait for every pair first. Caller holds g_mu.
void fold_locked(bool block) {
    size_t keep = 0;
    for (size_t i = 0; i < g_pending.size(); ++i) {
        Pending& p = g_pending[i];
        cudaError_t q = block ? cudaEventSynchronize(p.stop) : cudaEventQuery(p.stop);
        if (q == cudaSuccess) {
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, p.start, p.stop) == cudaSuccess) {
                g_count[p.family] += 1;
                g_ms[p.family] += ms;
            }
            g_pool.push_back(p.start);
            g_pool.push_back(p.stop);
        } else {
            if (q != cudaErrorNotReady) (void)cudaGetLastError();
            g_pending[keep++] = p;
        }
    }
    g_pending.resize(keep);
}

}  // namespace

namespace fugal {

fugal_status fail(fugal_status s, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
    return s;
}

fugal_status cuda_check(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return FUGAL_OK;
    return fail(FUGAL_CUDA_ERROR, "%s: %s (%s)", what, cudaGetErrorName(e), cudaGetErrorString(e));
}

LaunchScope::LaunchScope(int family, cudaStream_t stream) : family_(family), stream_(stream) {
    g_launches.fetch_add(1, std::memory_order_relaxed);
    if (g_timing_on.load(std::memory_order_relaxed)) {
        std::lock_guard<std::mutex> lock(g_mu);
        start_ = take_event();
        if (start_ != nullptr) cudaEventRecord(start_, stream_);
    }
}

LaunchScope::~LaunchScope() {
    if (start_ == nullptr) return;
    std::lock_guard<std::mutex> lock(g_mu);
    cudaEvent_t stop = take_event();
    if (stop == nullptr) return;
    cudaEventRecord(stop, stream_);
    g_pending.push_back({family_, start_, stop});
    if (g_pending.size() > 4096) fold_locked(false);
}

void timing_poll() {
    if (!g_timing_on.load(std::memory_order_relaxed)) return;
    std::lock_guard<std::mutex> lock(g_mu);
    fold_locked(false);
}

int sm_count() {
    static int cached[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    if (cached[dev] == 0) {
        int v = 0;
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
        cached[dev] = v > 0 ? v : 148;
    }
    return cached[dev];
}

}  // namespace fugal

extern "C" {

const char* fugal_status_string(int status) {
    switch (status) {
        case FUGAL_OK: return "ok";
        case FUGAL_BAD_SHAPE: return "bad shape";
        case FUGAL_BAD_ARGUMENT: return "bad argument";
        case FUGAL_CUDA_ERROR: return "CUDA error";
        case FUGAL_ITER_LIMIT: return "iteration limit";
        case FUGAL_NONFINITE: return "non-finite value";
        case FUGAL_DEVICE_TIMEOUT: return "device wait timed out";
        case FUGAL_WORKSPACE_TOO_SMALL: return "workspace too small";
        case FUGAL_UNSUPPORTED: return "unsupported";
        default: return "unknown status";
    }
}

const char* fugal_last_error(void) { return g_last_error; }

int fugal_version(void) { return 1; }

void fugal_timing_enable(int on) { g_timing_on.store(on ? 1 : 0); }

void fugal_timing_reset(void) {
    std::lock_guard<std::mutex> lock(g_mu);
    fold_locked(true);
    for (int i = 0; i < FUGAL_KERNEL_FAMILIES; ++i) {
        g_count[i] = 0;
        g_ms[i] = 0.0;
    }
}

fugal_status fugal_timing_query(int family, int64_t* launches, double* milliseconds) {
    if (family < 0 || family >= FUGAL_KERNEL_FAMILIES || launches == nullptr || milliseconds == nullptr)
        return fugal::fail(FUGAL_BAD_ARGUMENT, "fugal_timing_query: bad family or null output");
    std::lock_guard<std::mutex> lock(g_mu);
    fold_locked(true);
    *launches = g_count[family];
    *milliseconds = g_ms[family];
    return FUGAL_OK;
}

int64_t fugal_launch_count(void) { return g_launches.load(); }

}  // extern "C"
