// Exact Frank-Wolfe line search (opt-in; the reference steps with alpha = 2/(2+it),
// cugal/pred.py:133-141).  On the FUGAL objective
//   f(P) = -<P, A P B> + <D, P> + lam' <P, 1 - P>      (gradient -2 A P B + D + lam' (1 - 2P))
// the step along d = q - P is exactly quadratic:
//   f(P + a d) - f(P) = a g + a^2 Q,   g = <G, d>,   Q = -<d, A d B> - lam' <d, d>,
// so the best a in [0, 1] is -g / 2Q clipped (Q > 0), else 1 when g + Q < 0, else 0.
//   fugal_fw_direction          d = q - P, g and <d, d> (one read of P and the cost)
//   fugal_fw_gradient           W = -2 A d B (the gradient kernels with P := d, lam = 0)
//   fugal_fw_line_search_update <d, W>, then a and P += a d
// Every reduction is FP64; a never leaves the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "fugal_common.cuh"
#include "fugal_host.h"

namespace fugal {

constexpr int kLsThreads = 256;
constexpr int kLsChunk = kLsThreads * 4;  // columns of one (row, chunk) unit

// Grid-stride over (row, 1024-column chunk) units; thread t of a unit handles
// columns chunk*1024 + 4t .. +3.
struct Units {
    int n, chunks;
    long long count;
    __device__ Units(int n_) : n(n_), chunks((n_ + kLsChunk - 1) / kLsChunk) {
        count = static_cast<long long>(n) * chunks;
    }
};

// Log form: q = exp(L + u_i + v_j), G = -reg (L - U_i - V_j).  Scaling form
// (K != nullptr): q = (K v_j) u_i, G = L.  dir = q - P; sums[0] += <G, dir>,
// sums[1] += <dir, dir>.
__global__ void __launch_bounds__(kLsThreads) direction_kernel(const float* __restrict__ P, long long ldp,
                                                               const float* __restrict__ L, long long ldl,
                                                               const float* __restrict__ K, long long ldk,
                                                               const float* __restrict__ u,
                                                               const float* __restrict__ v,
                                                               const double* __restrict__ U,
                                                               const double* __restrict__ V, double reg,
                                                               float* __restrict__ dir, long long ldd, int n,
                                                               double* sums) {
    __shared__ double red[32];
    const Units un(n);
    double g = 0.0, dd = 0.0;
    for (long long w = blockIdx.x; w < un.count; w += gridDim.x) {
        const int i = static_cast<int>(w / un.chunks);
        const int j0 = static_cast<int>(w % un.chunks) * kLsChunk + threadIdx.x * 4;
        const float ui = u[i];
        const double Ui = U ? U[i] : 0.0;
        const int jend = min(n, j0 + 4);
        for (int j = j0; j < jend; ++j) {
            const float l = L[static_cast<size_t>(i) * ldl + j];
            const float p = P[static_cast<size_t>(i) * ldp + j];
            float q;
            double G;
            if (K != nullptr) {
                q = (K[static_cast<size_t>(i) * ldk + j] * v[j]) * ui;
                G = static_cast<double>(l);
            } else {
                q = expf(l + ui + v[j]);
                G = -reg * (static_cast<double>(l) - Ui - (V ? V[j] : 0.0));
            }
            const float d = q - p;
            dir[static_cast<size_t>(i) * ldd + j] = d;
            g += static_cast<double>(d) * G;
            dd += static_cast<double>(d) * static_cast<double>(d);
        }
    }
    g = block_sum(g, red);
    dd = block_sum(dd, red);
    if (threadIdx.x == 0) {
        atomicAdd(&sums[0], g);
        atomicAdd(&sums[1], dd);
    }
}

__global__ void commit_kernel(const float* u, const float* v, double* U, double* V, int n) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        U[j] += static_cast<double>(u[j]);
        V[j] += static_cast<double>(v[j]);
    }
}

// sums[2] += <dir, W>
__global__ void __launch_bounds__(kLsThreads) curvature_kernel(const float* __restrict__ dir, long long ldd,
                                                               const float* __restrict__ W, long long ldw, int n,
                                                               double* sums) {
    __shared__ double red[32];
    const Units un(n);
    double s = 0.0;
    for (long long w = blockIdx.x; w < un.count; w += gridDim.x) {
        const int i = static_cast<int>(w / un.chunks);
        const int j0 = static_cast<int>(w % un.chunks) * kLsChunk + threadIdx.x * 4;
        const int jend = min(n, j0 + 4);
        for (int j = j0; j < jend; ++j)
            s += static_cast<double>(dir[static_cast<size_t>(i) * ldd + j]) *
                 static_cast<double>(W[static_cast<size_t>(i) * ldw + j]);
    }
    s = block_sum(s, red);
    if (threadIdx.x == 0) atomicAdd(&sums[2], s);
}

// The minimiser over [0, 1] of a g + a^2 Q with Q = <d, W>/2 - lam' <d, d>.
__device__ __forceinline__ double step_length(const double* sums, double lambda_eff) {
    const double g = sums[0];
    const double Q = 0.5 * sums[2] - lambda_eff * sums[1];
    if (Q > 0.0) return fmin(1.0, fmax(0.0, -g / (2.0 * Q)));
    return (g + Q < 0.0) ? 1.0 : 0.0;
}

// P += a dir; block 0 also stores a and the signed gap <G, dir>.
__global__ void __launch_bounds__(kLsThreads) step_kernel(float* __restrict__ P, long long ldp,
                                                          const float* __restrict__ dir, long long ldd, int n,
                                                          const double* sums, double lambda_eff, double* alpha_out,
                                                          double* gap) {
    const double a = step_length(sums, lambda_eff);
    const float af = static_cast<float>(a);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        if (alpha_out) *alpha_out = a;
        if (gap) *gap = sums[0];
    }
    const Units un(n);
    for (long long w = blockIdx.x; w < un.count; w += gridDim.x) {
        const int i = static_cast<int>(w / un.chunks);
        const int j0 = static_cast<int>(w % un.chunks) * kLsChunk + threadIdx.x * 4;
        const int jend = min(n, j0 + 4);
        for (int j = j0; j < jend; ++j) {
            float* pp = P + static_cast<size_t>(i) * ldp + j;
            *pp = fmaf(af, dir[static_cast<size_t>(i) * ldd + j], *pp);
        }
    }
}

namespace {

fugal_status check_matrix(const void* p, int64_t ld, int64_t n, const char* who, const char* what) {
    if (p == nullptr) return fail(FUGAL_BAD_ARGUMENT, "%s: %s is null", who, what);
    if (n <= 0 || n > (1ll << 30)) return fail(FUGAL_BAD_SHAPE, "%s: bad n", who);
    if (ld < n) return fail(FUGAL_BAD_SHAPE, "%s: leading dimension of %s < n", who, what);
    return FUGAL_OK;
}

int ls_blocks(int64_t n) {
    const int64_t units = n * ((n + kLsChunk - 1) / kLsChunk);
    return static_cast<int>(std::min<int64_t>(units, static_cast<int64_t>(sm_count()) * 8));
}

}  // namespace

}  // namespace fugal

using namespace fugal;

extern "C" fugal_status fugal_fw_direction(int64_t n, const float* P, int64_t ldp, const float* cost32, int64_t ld32,
                                           const float* K, int64_t ldk, const float* u, const float* v, double* U,
                                           double* V, double regularization, float* dir, int64_t ldd, double* sums,
                                           int commit, fugal_stream_t stream_) {
    cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
    const char* who = "fugal_fw_direction";
    FUGAL_TRY(check_matrix(P, ldp, n, who, "P"));
    FUGAL_TRY(check_matrix(cost32, ld32, n, who, "cost32"));
    FUGAL_TRY(check_matrix(dir, ldd, n, who, "dir"));
    if (K != nullptr) FUGAL_TRY(check_matrix(K, ldk, n, who, "K"));
    if (u == nullptr || v == nullptr || sums == nullptr) return fail(FUGAL_BAD_ARGUMENT, "%s: null u, v or sums", who);
    if ((U == nullptr) != (V == nullptr)) return fail(FUGAL_BAD_ARGUMENT, "%s: give both U and V", who);
    if (commit && (U == nullptr || K != nullptr))
        return fail(FUGAL_BAD_ARGUMENT, "%s: commit needs U and V (log form)", who);
    FUGAL_TRY(cuda_check(cudaMemsetAsync(sums, 0, 3 * sizeof(double), stream), "fugal_fw_direction: clear sums"));
    {
        LaunchScope scope(FUGAL_KERNEL_UPDATE, stream);
        direction_kernel<<<ls_blocks(n), kLsThreads, 0, stream>>>(P, ldp, cost32, ld32, K, ldk, u, v, U, V,
                                                                  regularization, dir, ldd, static_cast<int>(n),
                                                                  sums);
        FUGAL_TRY(launch_check(who));
    }
    if (commit) {
        LaunchScope scope(FUGAL_KERNEL_OTHER, stream);
        const int blocks = static_cast<int>(std::min<int64_t>((n + 255) / 256, 1024));
        commit_kernel<<<blocks, 256, 0, stream>>>(u, v, U, V, static_cast<int>(n));
        FUGAL_TRY(launch_check("fugal_fw_direction: commit"));
    }
    return FUGAL_OK;
}

extern "C" fugal_status fugal_fw_line_search_update(int64_t n, float* P, int64_t ldp, const float* dir, int64_t ldd,
                                                    const float* W, int64_t ldw, double lambda_eff, double* sums,
                                                    double* alpha, double* gap, fugal_stream_t stream_) {
    cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
    const char* who = "fugal_fw_line_search_update";
    FUGAL_TRY(check_matrix(P, ldp, n, who, "P"));
    FUGAL_TRY(check_matrix(dir, ldd, n, who, "dir"));
    FUGAL_TRY(check_matrix(W, ldw, n, who, "W"));
    if (sums == nullptr) return fail(FUGAL_BAD_ARGUMENT, "%s: null sums", who);
    if (!std::isfinite(lambda_eff)) return fail(FUGAL_BAD_ARGUMENT, "%s: lambda is not finite", who);
    FUGAL_TRY(cuda_check(cudaMemsetAsync(sums + 2, 0, sizeof(double), stream), "fugal_fw_line_search_update"));
    LaunchScope scope(FUGAL_KERNEL_UPDATE, stream);
    curvature_kernel<<<ls_blocks(n), kLsThreads, 0, stream>>>(dir, ldd, W, ldw, static_cast<int>(n), sums);
    FUGAL_TRY(launch_check("fugal_fw_line_search_update: <d, W>"));
    step_kernel<<<ls_blocks(n), kLsThreads, 0, stream>>>(P, ldp, dir, ldd, static_cast<int>(n), sums, lambda_eff,
                                                         alpha, gap);
    return launch_check("fugal_fw_line_search_update: step");
}
