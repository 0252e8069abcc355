// Frank-Wolfe gradient for callers that cannot allocate device memory.
//
// fugal_fw_gradient needs an n x roundup(n, 4) FP32 workspace for the
// intermediate (A P)^T, which the caller allocates and passes in.  Some callers
// have no way to do that: a host whose device memory is owned by a pool
// allocator that every allocation has to go through (a cudaMalloc of its own
// competes with the pool, and fails once the pool has reserved the device), or
// a foreign-language binding that passes plain input/output pointers and never
// manages device memory itself.  fugal_fw_gradient_fixed_scratch serves them:
// it takes the workspace from one array compiled into this library, so it
// allocates nothing, and only works up to a fixed size.
//
// The array is FUGAL_FIXED_SCRATCH_BYTES (16 MiB) of device memory.  Every GPU
// on which this library's device code is loaded holds it until the process
// exits.  It is shared by every call on that device and keeps whatever the last
// call left in it; nothing in it has to start at zero, because the first kernel
// of the gradient writes every element that the second one reads.  Two calls
// whose kernels overlap on the GPU (unordered streams, or several host threads)
// race on the array and corrupt each other's results.
#include <cuda_runtime.h>

#include <mutex>

#include "fugal_host.h"

namespace fugal {
namespace {

constexpr int kMaxDevices = 64;

static_assert(FUGAL_FIXED_SCRATCH_BYTES % 256 == 0, "scratch size must keep 256-byte alignment");
static_assert(static_cast<long long>(FUGAL_FIXED_SCRATCH_MAX_N) * ((FUGAL_FIXED_SCRATCH_MAX_N + 3) / 4 * 4) *
                      sizeof(float) <=
                  FUGAL_FIXED_SCRATCH_BYTES,
              "largest n must fit the scratch array");

// In host code this name is only a handle for the runtime; the device address
// comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char fixed_scratch[FUGAL_FIXED_SCRATCH_BYTES];

std::mutex setup_lock;
void* scratch_address[kMaxDevices] = {};

// Device address of the scratch array on the current device, looked up once per
// device (the lookup loads this library's device code on that device).  The
// address belongs to the runtime's primary context of that device; a device
// reset or a different driver context would make it stale (documented as
// unsupported for this entry point).
fugal_status scratch_for_current_device(void** out) {
    int dev = -1;
    FUGAL_TRY(cuda_check(cudaGetDevice(&dev), "fugal_fw_gradient_fixed_scratch: cudaGetDevice"));
    if (dev < 0 || dev >= kMaxDevices)
        return fail(FUGAL_UNSUPPORTED, "fugal_fw_gradient_fixed_scratch: device ordinal %d >= %d", dev, kMaxDevices);
    std::lock_guard<std::mutex> guard(setup_lock);
    if (scratch_address[dev] == nullptr) {
        void* p = nullptr;
        FUGAL_TRY(cuda_check(cudaGetSymbolAddress(&p, fixed_scratch),
                             "fugal_fw_gradient_fixed_scratch: cudaGetSymbolAddress"));
        if (p == nullptr)
            return fail(FUGAL_CUDA_ERROR, "fugal_fw_gradient_fixed_scratch: null scratch address on device %d", dev);
        scratch_address[dev] = p;
    }
    *out = scratch_address[dev];
    return FUGAL_OK;
}

}  // namespace
}  // namespace fugal

using namespace fugal;

extern "C" fugal_status fugal_fw_gradient_fixed_scratch(
    int64_t n, const int32_t* a_row_pointers, const int32_t* a_col_indices, const int32_t* b_row_pointers,
    const int32_t* b_col_indices, const float* P, int64_t ldp, const float* source_features,
    const float* target_features, const float* D, int64_t ldd, double lambda, double lambda_scale, double out_scale,
    const double* U, const double* V, float* out, int64_t ldo, fugal_stream_t stream) {
    if (n <= 0) return fail(FUGAL_BAD_SHAPE, "fugal_fw_gradient_fixed_scratch: n must be positive");
    if (n > FUGAL_FIXED_SCRATCH_MAX_N)
        return fail(FUGAL_BAD_SHAPE,
                    "fugal_fw_gradient_fixed_scratch: n = %lld is above the fixed scratch limit n <= %d (%d bytes); "
                    "use fugal_fw_gradient with a caller-allocated workspace",
                    static_cast<long long>(n), FUGAL_FIXED_SCRATCH_MAX_N, FUGAL_FIXED_SCRATCH_BYTES);
    void* scratch = nullptr;
    FUGAL_TRY(scratch_for_current_device(&scratch));
    return fugal_fw_gradient(n, a_row_pointers, a_col_indices, b_row_pointers, b_col_indices, P, ldp,
                             source_features, target_features, D, ldd, lambda, lambda_scale, out_scale, U, V, out,
                             ldo, scratch, FUGAL_FIXED_SCRATCH_BYTES, stream);
}
