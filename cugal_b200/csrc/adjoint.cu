// Differentiation of the log-domain Sinkhorn solve (the plan P of
// cugal/sinkhorn.py:90-120 as a function of the cost C).
//
// At the converged potentials the plan P = exp(-C/reg + u 1^T + 1 v^T) has unit
// row and column sums.  Implicit differentiation of those constraints gives,
// for a loss L(P) with G = dL/dP,
//     a = (G o P) 1,  b = (G o P)^T 1,
//     [ I  P ; P^T  I ] [alpha; beta] = [a; b]      (consistent, one null vector [1; -1]),
//     dL/dK = P o (G - alpha 1^T - 1 beta^T),   dL/dC = -dL/dK / reg.
// The block system is symmetric positive semi-definite (eigenvalues 1 +- the
// singular values of P), so conjugate gradients solve it with one pass over P
// per iteration: the kernel below forms P y and P^T x from the same read.
//
// Kernels:
//   plan_kernel        P = exp(L + u_i + v_j) from the absorbed cost and duals;
//   matvec_part_kernel tiles of 64 rows x 1024 columns: row partials of P y and
//                      column partials of P^T x (P optionally weighted by G);
//   matvec_merge_*     FP64 sums of the partials;
//   adjoint_kernel     out = scale * P o (G - alpha_i - beta_j).
#include <cuda_runtime.h>

#include <algorithm>

#include "fugal_common.cuh"
#include "fugal_host.h"

namespace fugal {

constexpr int kMvRows = 64;
constexpr int kMvThreads = 256;
constexpr int kMvCols = kMvThreads * 4;

__global__ void plan_kernel(const float* __restrict__ L, long long ldl, int n, const float* __restrict__ u,
                            const float* __restrict__ v, float* __restrict__ P, long long ldp) {
    for (int i = blockIdx.y; i < n; i += gridDim.y) {
        const float ui = u[i];
        for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
            P[static_cast<size_t>(i) * ldp + j] = expf(L[static_cast<size_t>(i) * ldl + j] + ui + v[j]);
    }
}

// Block (cx, ry) covers rows [ry*64, +64) and columns [cx*1024, +1024); each
// thread owns 4 consecutive columns.  row_part[cx][i] = sum_j M_ij y_j over the
// block's columns, col_part[ry][j] = sum_i M_ij x_i over its rows, with
// M = P or P o W.
__global__ void __launch_bounds__(kMvThreads) matvec_part_kernel(const float* __restrict__ P, long long ldp,
                                                                 const float* __restrict__ W, long long ldw, int n,
                                                                 const double* __restrict__ x,
                                                                 const double* __restrict__ y, double* row_part,
                                                                 double* col_part) {
    __shared__ double red[kMvThreads / 32][kMvRows];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int r0 = blockIdx.y * kMvRows;
    const int j0 = blockIdx.x * kMvCols + threadIdx.x * 4;
    double yj[4], cs[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        yj[q] = (j0 + q < n) ? y[j0 + q] : 0.0;
        cs[q] = 0.0;
    }
    for (int r = 0; r < kMvRows; ++r) {
        const int i = r0 + r;
        double rs = 0.0;
        if (i < n) {
            const double xi = x[i];
            const float* prow = P + static_cast<size_t>(i) * ldp;
            const float* wrow = W ? W + static_cast<size_t>(i) * ldw : nullptr;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int j = j0 + q;
                if (j < n) {
                    double m = static_cast<double>(prow[j]);
                    if (wrow) m *= static_cast<double>(wrow[j]);
                    rs += m * yj[q];
                    cs[q] += m * xi;
                }
            }
        }
        rs = warp_sum(rs);
        if (lane == 0) red[warp][r] = rs;
    }
    __syncthreads();
    if (threadIdx.x < kMvRows) {
        const int i = r0 + threadIdx.x;
        double s = 0.0;
#pragma unroll
        for (int w = 0; w < kMvThreads / 32; ++w) s += red[w][threadIdx.x];
        if (i < n) row_part[static_cast<size_t>(blockIdx.x) * n + i] = s;
    }
#pragma unroll
    for (int q = 0; q < 4; ++q)
        if (j0 + q < n) col_part[static_cast<size_t>(blockIdx.y) * n + j0 + q] = cs[q];
}

__global__ void matvec_merge_kernel(const double* part, int parts, int n, double* out) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int p = 0; p < parts; ++p) s += part[static_cast<size_t>(p) * n + k];
        out[k] = s;
    }
}

__global__ void adjoint_kernel(const float* __restrict__ P, long long ldp, const float* __restrict__ G,
                               long long ldg, int n, const double* __restrict__ alpha,
                               const double* __restrict__ beta, double scale, float* __restrict__ out,
                               long long ldo) {
    for (int i = blockIdx.y; i < n; i += gridDim.y) {
        const double ai = alpha[i];
        for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
            const double p = static_cast<double>(P[static_cast<size_t>(i) * ldp + j]);
            const double g = static_cast<double>(G[static_cast<size_t>(i) * ldg + j]);
            out[static_cast<size_t>(i) * ldo + j] = static_cast<float>(scale * p * (g - ai - beta[j]));
        }
    }
}

// Backward of one half step of the unrolled log-domain iteration (no momentum).
// axis 1 (row half, out_i = -LSE_j(K_ij + other_j)):  E_ij = exp(K_ij + other_j + out_i),
//     gK_ij -= g_i E_ij,   g_other_j -= sum_i g_i E_ij        (column partials)
// axis 0 (column half, out_j = -LSE_i(K_ij + other_i)): E_ij = exp(K_ij + other_i + out_j),
//     gK_ij -= g_j E_ij,   g_other_i -= sum_j g_j E_ij        (row partials)
__global__ void __launch_bounds__(kMvThreads) unrolled_step_kernel(const float* __restrict__ K, long long ldk, int n,
                                                                   const float* __restrict__ out_dual,
                                                                   const float* __restrict__ other_dual,
                                                                   const double* __restrict__ g, int axis,
                                                                   float* __restrict__ gK, long long ldg,
                                                                   double* row_part, double* col_part) {
    __shared__ double red[kMvThreads / 32][kMvRows];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int r0 = blockIdx.y * kMvRows;
    const int j0 = blockIdx.x * kMvCols + threadIdx.x * 4;
    double cs[4] = {0.0, 0.0, 0.0, 0.0};
    for (int r = 0; r < kMvRows; ++r) {
        const int i = r0 + r;
        double rs = 0.0;
        if (i < n) {
            const float* krow = K + static_cast<size_t>(i) * ldk;
            float* grow = gK + static_cast<size_t>(i) * ldg;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int j = j0 + q;
                if (j < n) {
                    double e, w;
                    if (axis == 1) {
                        e = exp(static_cast<double>(krow[j]) + other_dual[j] + out_dual[i]);
                        w = g[i] * e;
                        cs[q] -= w;
                    } else {
                        e = exp(static_cast<double>(krow[j]) + other_dual[i] + out_dual[j]);
                        w = g[j] * e;
                        rs -= w;
                    }
                    grow[j] = static_cast<float>(static_cast<double>(grow[j]) - w);
                }
            }
        }
        if (axis == 0) {
            rs = warp_sum(rs);
            if (lane == 0) red[warp][r] = rs;
        }
    }
    if (axis == 0) {
        __syncthreads();
        if (threadIdx.x < kMvRows) {
            const int i = r0 + threadIdx.x;
            double s = 0.0;
#pragma unroll
            for (int w = 0; w < kMvThreads / 32; ++w) s += red[w][threadIdx.x];
            if (i < n) row_part[static_cast<size_t>(blockIdx.x) * n + i] = s;
        }
    } else {
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (j0 + q < n) col_part[static_cast<size_t>(blockIdx.y) * n + j0 + q] = cs[q];
    }
}

__global__ void merge_add_kernel(const double* part, int parts, int n, double* out) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int p = 0; p < parts; ++p) s += part[static_cast<size_t>(p) * n + k];
        out[k] += s;
    }
}

inline dim3 ew2d(int64_t n) {
    return dim3(static_cast<unsigned>(std::min<int64_t>((n + 255) / 256, 32)),
                static_cast<unsigned>(std::min<int64_t>(n, 8 * sm_count())));
}

}  // namespace fugal

using namespace fugal;

extern "C" fugal_status fugal_sinkhorn_plan(const float* cost32, int64_t ld32, int64_t n, const float* u,
                                            const float* v, float* P, int64_t ldp, fugal_stream_t stream_) {
    cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
    if (cost32 == nullptr || u == nullptr || v == nullptr || P == nullptr)
        return fail(FUGAL_BAD_ARGUMENT, "fugal_sinkhorn_plan: null argument");
    if (n <= 0 || ld32 < n || ldp < n) return fail(FUGAL_BAD_SHAPE, "fugal_sinkhorn_plan: bad shape");
    LaunchScope scope(FUGAL_KERNEL_OTHER, stream);
    plan_kernel<<<ew2d(n), 256, 0, stream>>>(cost32, ld32, static_cast<int>(n), u, v, P, ldp);
    return launch_check("fugal_sinkhorn_plan");
}

extern "C" fugal_status fugal_plan_matvec_workspace_size(int64_t n, size_t* bytes) {
    if (bytes == nullptr) return fail(FUGAL_BAD_ARGUMENT, "fugal_plan_matvec_workspace_size: null output");
    if (n <= 0 || n > (1ll << 30)) return fail(FUGAL_BAD_SHAPE, "fugal_plan_matvec_workspace_size: bad n");
    const int64_t cb = (n + kMvCols - 1) / kMvCols, rb = (n + kMvRows - 1) / kMvRows;
    *bytes = static_cast<size_t>((cb + rb) * n) * 8 + 256;
    return FUGAL_OK;
}

extern "C" fugal_status fugal_plan_matvec(const float* P, int64_t ldp, const float* W, int64_t ldw, int64_t n,
                                          const double* x, const double* y, double* Ptx, double* Py,
                                          void* workspace, size_t workspace_bytes, fugal_stream_t stream_) {
    cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
    size_t need = 0;
    FUGAL_TRY(fugal_plan_matvec_workspace_size(n, &need));
    if (P == nullptr || x == nullptr || y == nullptr || Ptx == nullptr || Py == nullptr || workspace == nullptr)
        return fail(FUGAL_BAD_ARGUMENT, "fugal_plan_matvec: null argument");
    if (ldp < n || (W != nullptr && ldw < n)) return fail(FUGAL_BAD_SHAPE, "fugal_plan_matvec: bad leading dimension");
    if (workspace_bytes < need)
        return fail(FUGAL_WORKSPACE_TOO_SMALL, "fugal_plan_matvec: workspace %zu < %zu", workspace_bytes, need);
    const int nn = static_cast<int>(n);
    const int cb = static_cast<int>((n + kMvCols - 1) / kMvCols), rb = static_cast<int>((n + kMvRows - 1) / kMvRows);
    double* row_part = static_cast<double*>(workspace);
    double* col_part = row_part + static_cast<size_t>(cb) * n;
    {
        LaunchScope scope(FUGAL_KERNEL_OTHER, stream);
        matvec_part_kernel<<<dim3(cb, rb), kMvThreads, 0, stream>>>(P, ldp, W, ldw, nn, x, y, row_part, col_part);
        FUGAL_TRY(launch_check("fugal_plan_matvec: partials"));
    }
    {
        LaunchScope scope(FUGAL_KERNEL_OTHER, stream);
        const int blocks = static_cast<int>(std::min<int64_t>((n + 255) / 256, 4 * sm_count()));
        matvec_merge_kernel<<<blocks, 256, 0, stream>>>(row_part, cb, nn, Py);
        matvec_merge_kernel<<<blocks, 256, 0, stream>>>(col_part, rb, nn, Ptx);
        FUGAL_TRY(launch_check("fugal_plan_matvec: merge"));
    }
    return FUGAL_OK;
}

extern "C" fugal_status fugal_sinkhorn_adjoint(const float* P, int64_t ldp, const float* G, int64_t ldg, int64_t n,
                                               const double* alpha, const double* beta, double scale, float* out,
                                               int64_t ldo, fugal_stream_t stream_) {
    cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
    if (P == nullptr || G == nullptr || alpha == nullptr || beta == nullptr || out == nullptr)
        return fail(FUGAL_BAD_ARGUMENT, "fugal_sinkhorn_adjoint: null argument");
    if (n <= 0 || ldp < n || ldg < n || ldo < n) return fail(FUGAL_BAD_SHAPE, "fugal_sinkhorn_adjoint: bad shape");
    LaunchScope scope(FUGAL_KERNEL_OTHER, stream);
    adjoint_kernel<<<ew2d(n), 256, 0, stream>>>(P, ldp, G, ldg, static_cast<int>(n), alpha, beta, scale, out, ldo);
    return launch_check("fugal_sinkhorn_adjoint");
}

extern "C" fugal_status fugal_sinkhorn_unrolled_step_backward(const float* K, int64_t ldk, int64_t n,
                                                              const float* out_dual, const float* other_dual,
                                                              const double* g, int axis, float* gK, int64_t ldg,
                                                              double* g_other, void* workspace,
                                                              size_t workspace_bytes, fugal_stream_t stream_) {
    cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
    size_t need = 0;
    FUGAL_TRY(fugal_plan_matvec_workspace_size(n, &need));
    if (K == nullptr || out_dual == nullptr || other_dual == nullptr || g == nullptr || gK == nullptr ||
        g_other == nullptr || workspace == nullptr)
        return fail(FUGAL_BAD_ARGUMENT, "fugal_sinkhorn_unrolled_step_backward: null argument");
    if (axis != 0 && axis != 1) return fail(FUGAL_BAD_ARGUMENT, "fugal_sinkhorn_unrolled_step_backward: axis 0 or 1");
    if (ldk < n || ldg < n) return fail(FUGAL_BAD_SHAPE, "fugal_sinkhorn_unrolled_step_backward: bad shape");
    if (workspace_bytes < need)
        return fail(FUGAL_WORKSPACE_TOO_SMALL, "fugal_sinkhorn_unrolled_step_backward: workspace too small");
    const int nn = static_cast<int>(n);
    const int cb = static_cast<int>((n + kMvCols - 1) / kMvCols), rb = static_cast<int>((n + kMvRows - 1) / kMvRows);
    double* row_part = static_cast<double*>(workspace);
    double* col_part = row_part + static_cast<size_t>(cb) * n;
    {
        LaunchScope scope(FUGAL_KERNEL_OTHER, stream);
        unrolled_step_kernel<<<dim3(cb, rb), kMvThreads, 0, stream>>>(K, ldk, nn, out_dual, other_dual, g, axis, gK,
                                                                      ldg, row_part, col_part);
        FUGAL_TRY(launch_check("fugal_sinkhorn_unrolled_step_backward"));
    }
    {
        LaunchScope scope(FUGAL_KERNEL_OTHER, stream);
        const int blocks = static_cast<int>(std::min<int64_t>((n + 255) / 256, 4 * sm_count()));
        if (axis == 0)
            merge_add_kernel<<<blocks, 256, 0, stream>>>(row_part, cb, nn, g_other);
        else
            merge_add_kernel<<<blocks, 256, 0, stream>>>(col_part, rb, nn, g_other);
        FUGAL_TRY(launch_check("fugal_sinkhorn_unrolled_step_backward: merge"));
    }
    return FUGAL_OK;
}
