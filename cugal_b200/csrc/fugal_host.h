// Host-side helpers shared by the .cu files: error reporting, argument checks,
// launch counting and the optional per-kernel event timing.
#pragma once

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdint>

#include "../../include/fugal_b200.h"

namespace fugal {

// Record a message for fugal_last_error() and return `s`.
fugal_status fail(fugal_status s, const char* fmt, ...);

// Map a CUDA error to FUGAL_CUDA_ERROR (with message) or FUGAL_OK.
fugal_status cuda_check(cudaError_t e, const char* what);

// Check the launch that was just issued (cudaGetLastError).
inline fugal_status launch_check(const char* what) { return cuda_check(cudaGetLastError(), what); }

// Count one launch of `family`; if timing is enabled, bracket it with events.
class LaunchScope {
   public:
    LaunchScope(int family, cudaStream_t stream);
    ~LaunchScope();
    LaunchScope(const LaunchScope&) = delete;
    LaunchScope& operator=(const LaunchScope&) = delete;

   private:
    int family_;
    cudaStream_t stream_;
    cudaEvent_t start_ = nullptr;
};

// Fold completed timing events into the totals (non-blocking).
void timing_poll();

inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// Number of SMs of the current device (cached per device).
int sm_count();

}  // namespace fugal

#define FUGAL_TRY(expr)                              \
    do {                                             \
        fugal_status _s = (expr);                    \
        if (_s != FUGAL_OK) return _s;               \
    } while (0)
