// Frank-Wolfe update and the reference-compatible elementwise / row kernels:
//   fugal_fw_update                    cugal/pred.py:133-141 on the absorbed cost
//   fugal_update_quasi_permutation_log cuda_kernels/update_quasi_permutation.cu:7-56
//   fugal_regularize                   cuda_kernels/regularize.cu:10-39
//   fugal_add_distance                 cuda_kernels/distance.cu:11-53
//   fugal_sinkhorn_log_step            cuda_kernels/sinkhorn_log.cu:8-66,100-114
//   fugal_sinkhorn_log_marginal        cuda_kernels/sinkhorn_log.cu:68-98
//   fugal_count_le                     cugal/pred.py:152-153
// All reductions accumulate in FP64 and land in a caller-owned device double.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "fugal_common.cuh"
#include "fugal_host.h"

namespace fugal {

constexpr int kEwThreads = 256;

// Grid over (row, 1024-column chunk): blockIdx.x = row, blockIdx.y = chunk;
// each thread handles 4 consecutive columns.
inline dim3 ew_grid(int64_t n) {
    return dim3(static_cast<unsigned>(n), static_cast<unsigned>((n + kEwThreads * 4 - 1) / (kEwThreads * 4)));
}

// Where the update records the plan's nonzero entries (fugal_fw_update_collect):
// per row k, counts[k] entries (column, q) at entries[k * slots ...] in no
// particular order (counts zeroed before the kernel; entries past `slots` are
// counted, not stored; the scatter checks counts and row sums).
struct PlanOut {
    int* counts;
    fugal_plan_entry* entries;
    int slots;
};

// q = exp(L + u_i + v_j); P += alpha (q - P); gap += (q - P) * (-reg (L - U_i - V_j)).
// Rows grid-strided over the blocks, each row's columns in chunks of 1024 (one
// float4 per thread per chunk); every block reduces its gap once at the end (one
// FP64 atomic per block).  EMIT: each q > 0 also takes a slot of its row through
// a global atomic on the row's count (a few per row, no barrier).
template <bool EMIT>
__global__ void __launch_bounds__(kEwThreads) fw_update_kernel(float* __restrict__ P, long long ldp,
                                                               const float* __restrict__ L, long long ldl,
                                                               const float* __restrict__ u,
                                                               const float* __restrict__ v,
                                                               const double* __restrict__ U,
                                                               const double* __restrict__ V, int n, float alpha,
                                                               double reg, double* gap, PlanOut plan) {
    __shared__ double red[32];
    constexpr int kChunk = kEwThreads * 4;
    double g = 0.0;
    for (int i = blockIdx.x; i < n; i += gridDim.x) {
      const float ui = u[i];
      const double Ui = U ? U[i] : 0.0;
      float* prow = P + static_cast<size_t>(i) * ldp;
    const float* lrow = L + static_cast<size_t>(i) * ldl;
      fugal_plan_entry* slots = EMIT ? plan.entries + static_cast<size_t>(i) * plan.slots : nullptr;
      auto record = [&](int j, float qv) {
          if constexpr (EMIT) {
              if (qv > 0.f) {
                  const int s = atomicAdd(&plan.counts[i], 1);
                  if (s < plan.slots) slots[s] = fugal_plan_entry{j, qv};
              }
          }
      };
      for (int j0 = threadIdx.x * 4; j0 < n; j0 += kChunk) {
        if (j0 + 4 <= n) {
            const float4 l4 = *reinterpret_cast<const float4*>(lrow + j0);
            float4 p4 = *reinterpret_cast<float4*>(prow + j0);
            const float4 v4 = *reinterpret_cast<const float4*>(v + j0);
            const float lv[4] = {l4.x, l4.y, l4.z, l4.w};
            const float vv[4] = {v4.x, v4.y, v4.z, v4.w};
            float pv[4] = {p4.x, p4.y, p4.z, p4.w};
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const float qv = expf(lv[q] + ui + vv[q]);
                const float diff = qv - pv[q];
                const double C = -reg * (static_cast<double>(lv[q]) - Ui - (V ? V[j0 + q] : 0.0));
                g += static_cast<double>(diff) * C;
                pv[q] = fmaf(alpha, diff, pv[q]);
                record(j0 + q, qv);
            }
            p4 = make_float4(pv[0], pv[1], pv[2], pv[3]);
            *reinterpret_cast<float4*>(prow + j0) = p4;
        } else {
            for (int j = j0; j < n; ++j) {
                const float qv = expf(lrow[j] + ui + v[j]);
                const float diff = qv - prow[j];
                const double C = -reg * (static_cast<double>(lrow[j]) - Ui - (V ? V[j] : 0.0));
                g += static_cast<double>(diff) * C;
                prow[j] = fmaf(alpha, diff, prow[j]);
                record(j, qv);
            }
        }
      }
    }
    g = block_sum(g, red);
    if (threadIdx.x == 0) atomicAdd(gap, g);
}

__global__ void commit_duals_kernel(const float* u, const float* v, double* U, double* V, int n) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        U[j] += static_cast<double>(u[j]);
        V[j] += static_cast<double>(v[j]);
    }
}

// Reference form: scaled = exp(K + v_c + u_r); gap += (scaled - P)(K * -reg); P += (scaled - P) alpha.
__global__ void __launch_bounds__(kEwThreads) update_log_kernel(float* __restrict__ P, long long ldp,
                                                                const float* __restrict__ K, long long ldk,
                                                                const float* __restrict__ u,
                                                                const float* __restrict__ v, int n, float alpha,
                                                                float reg, double* gap) {
    __shared__ double red[32];
    const int i = blockIdx.x;
    const int j0 = (blockIdx.y * blockDim.x + threadIdx.x) * 4;
    double g = 0.0;
    for (int j = j0; j < min(n, j0 + 4); ++j) {
        const float k = K[static_cast<size_t>(i) * ldk + j];
        float& p = P[static_cast<size_t>(i) * ldp + j];
        const float scaled = expf(k + v[j] + u[i]);
        const float diff = scaled - p;
        g += static_cast<double>(diff) * static_cast<double>(k * -reg);
        p = __fadd_rn(p, __fmul_rn(diff, alpha));
    }
    g = block_sum(g, red);
    if (threadIdx.x == 0) atomicAdd(gap, g);
}

// gradient += it - (2 it) * P, unfused IEEE operations in the reference's order.
__global__ void regularize_kernel(float* G, long long ldg, const float* P, long long ldp, int n, int it) {
    const int i = blockIdx.x;
    const int j0 = (blockIdx.y * blockDim.x + threadIdx.x) * 4;
    for (int j = j0; j < min(n, j0 + 4); ++j) {
        float& g = G[static_cast<size_t>(i) * ldg + j];
        const float t = __fmul_rn(static_cast<float>(it * 2), P[static_cast<size_t>(i) * ldp + j]);
        g = __fadd_rn(g, __fsub_rn(static_cast<float>(it), t));
    }
}

// out[x][y] += sqrtf(sum_i (s[x][i] - t[y][i])^2), squares of FP32 differences summed in double
// (the reference accumulates into `auto sum = 0.0`).
__global__ void add_distance_kernel(const float* s, const float* t, int n, float* out, long long ldo) {
    const int x = blockIdx.x;
    const int y0 = (blockIdx.y * blockDim.x + threadIdx.x) * 4;
    const float a0 = s[4 * x], a1 = s[4 * x + 1], a2 = s[4 * x + 2], a3 = s[4 * x + 3];
    for (int y = y0; y < min(n, y0 + 4); ++y) {
        double sum = 0.0;
        const float d0 = a0 - t[4 * y], d1 = a1 - t[4 * y + 1], d2 = a2 - t[4 * y + 2], d3 = a3 - t[4 * y + 3];
        sum += __fmul_rn(d0, d0);
        sum += __fmul_rn(d1, d1);
        sum += __fmul_rn(d2, d2);
        sum += __fmul_rn(d3, d3);
        out[static_cast<size_t>(x) * ldo + y] += sqrtf(static_cast<float>(sum));
    }
}

// out[r] = (1-w) out[r] - w LSE_c(K[r,c] + add[c]) (w == 1 within 1e-4: out[r] = -LSE).
__global__ void __launch_bounds__(256) log_step_kernel(const float* K, long long ldk, int cols, const float* add,
                                                       float* out, float w) {
    __shared__ float sm_m[32], sm_s[32];
    const int r = blockIdx.x;
    const float* row = K + static_cast<size_t>(r) * ldk;
    float m = -INFINITY;
    for (int c = threadIdx.x; c < cols; c += blockDim.x) m = fmaxf(m, row[c] + add[c]);
    m = warp_max(m);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (lane == 0) sm_m[warp] = m;
    __syncthreads();
    float M = -INFINITY;
    for (int q = 0; q < nw; ++q) M = fmaxf(M, sm_m[q]);
    const float base = (M == -INFINITY) ? 0.f : M;
    float s = 0.f;
    for (int c = threadIdx.x; c < cols; c += blockDim.x) s += expf(row[c] + add[c] - base);
    s = warp_sum(s);
    if (lane == 0) sm_s[warp] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        float S = 0.f;
        for (int q = 0; q < nw; ++q) S += sm_s[q];
        const float lse = M + logf(S);
        out[r] = (fabsf(w - 1.0f) < 1e-4f) ? -lse : (1.0f - w) * out[r] - w * lse;
    }
}

__global__ void __launch_bounds__(256) marginal_rows_kernel(const float* K, long long ldk, int n, const float* u,
                                                            const float* v, double* result) {
    __shared__ double red[32];
    const int r = blockIdx.x;
    const float* row = K + static_cast<size_t>(r) * ldk;
    double s = 0.0;
    for (int c = threadIdx.x; c < n; c += blockDim.x) s += static_cast<double>(expf(row[c] + u[r] + v[c]));
    s = block_sum(s, red);
    if (threadIdx.x == 0) atomicAdd(result, fabs(s - 1.0));
}

__global__ void __launch_bounds__(256) marginal_cols_kernel(const float* K, long long ldk, int n, const float* u,
                                                            const float* v, double* result) {
    __shared__ double red[32];
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    double dev = 0.0;
    if (c < n) {
        double s = 0.0;
        for (int r = 0; r < n; ++r) s += static_cast<double>(expf(K[static_cast<size_t>(r) * ldk + c] + u[r] + v[c]));
        dev = fabs(s - 1.0);
    }
    dev = block_sum(dev, red);
    if (threadIdx.x == 0) atomicAdd(result, dev);
}

__global__ void count_le_kernel(const float* P, long long ldp, int n, float thr, unsigned long long* count) {
    const int i = blockIdx.x;
    const int j0 = (blockIdx.y * blockDim.x + threadIdx.x) * 4;
    int c = 0;
    for (int j = j0; j < min(n, j0 + 4); ++j) c += (P[static_cast<size_t>(i) * ldp + j] <= thr) ? 1 : 0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, static_cast<unsigned long long>(c));
}

fugal_status check_square(const void* p, int64_t ld, int64_t n, const char* who, const char* what) {
    if (p == nullptr) return fail(FUGAL_BAD_ARGUMENT, "%s: %s is null", who, what);
    if (n <= 0 || n > (1ll << 30)) return fail(FUGAL_BAD_SHAPE, "%s: bad n", who);
    if (ld < n) return fail(FUGAL_BAD_SHAPE, "%s: leading dimension of %s < n", who, what);
    return FUGAL_OK;
}

}  // namespace fugal

using namespace fugal;

namespace {

fugal_status fw_update(int64_t n, float* P, int64_t ldp, const float* cost32, int64_t ld32, const float* u,
                       const float* v, double* U, double* V, double alpha, double regularization, double* gap,
                       int commit, const PlanOut* plan, const char* who, cudaStream_t stream) {
    FUGAL_TRY(check_square(P, ldp, n, who, "P"));
    FUGAL_TRY(check_square(cost32, ld32, n, who, "cost32"));
    if (u == nullptr || v == nullptr || gap == nullptr) return fail(FUGAL_BAD_ARGUMENT, "%s: null duals or gap", who);
    if ((U == nullptr) != (V == nullptr)) return fail(FUGAL_BAD_ARGUMENT, "%s: give both U and V", who);
    if (commit && U == nullptr) return fail(FUGAL_BAD_ARGUMENT, "%s: commit needs U and V", who);
    if ((ldp % 4) || (ld32 % 4) || !aligned16(P) || !aligned16(cost32) || !aligned16(v))
        return fail(FUGAL_BAD_SHAPE, "%s: P, cost32, v need 16-byte rows", who);
    FUGAL_TRY(cuda_check(cudaMemsetAsync(gap, 0, sizeof(double), stream), who));
    {
        LaunchScope scope(FUGAL_KERNEL_UPDATE, stream);
        const int blocks = static_cast<int>(std::min<int64_t>(n, static_cast<int64_t>(sm_count()) * 8));
        if (plan != nullptr)
            fw_update_kernel<true><<<blocks, kEwThreads, 0, stream>>>(P, ldp, cost32, ld32, u, v, U, V,
                                                                      static_cast<int>(n), static_cast<float>(alpha),
                                                                      regularization, gap, *plan);
        else
            fw_update_kernel<false><<<blocks, kEwThreads, 0, stream>>>(P, ldp, cost32, ld32, u, v, U, V,
                                                                       static_cast<int>(n),
                                                                       static_cast<float>(alpha), regularization,
                                                                       gap, PlanOut{});
        FUGAL_TRY(launch_check(who));
    }
    if (commit) {
        LaunchScope scope(FUGAL_KERNEL_OTHER, stream);
        const int blocks = static_cast<int>(std::min<int64_t>((n + 255) / 256, 1024));
        commit_duals_kernel<<<blocks, 256, 0, stream>>>(u, v, U, V, static_cast<int>(n));
        FUGAL_TRY(launch_check("fugal_fw_update: commit"));
    }
    return FUGAL_OK;
}

}  // namespace

extern "C" fugal_status fugal_fw_update(int64_t n, float* P, int64_t ldp, const float* cost32, int64_t ld32,
                                        const float* u, const float* v, double* U, double* V, double alpha,
                                        double regularization, double* gap, int commit, fugal_stream_t stream) {
    return fw_update(n, P, ldp, cost32, ld32, u, v, U, V, alpha, regularization, gap, commit, nullptr,
                     "fugal_fw_update", reinterpret_cast<cudaStream_t>(stream));
}

extern "C" fugal_status fugal_fw_update_collect(int64_t n, float* P, int64_t ldp, const float* cost32, int64_t ld32,
                                                const float* u, const float* v, double* U, double* V, double alpha,
                                                double regularization, double* gap, int commit, int32_t* plan_counts,
                                                fugal_plan_entry* plan_entries, int32_t slots,
                                                fugal_stream_t stream) {
    const char* who = "fugal_fw_update_collect";
    if (plan_counts == nullptr || plan_entries == nullptr)
        return fail(FUGAL_BAD_ARGUMENT, "%s: null plan buffers", who);
    if (slots < 1 || slots > 1024) return fail(FUGAL_BAD_ARGUMENT, "%s: slots must be in [1, 1024]", who);
    FUGAL_TRY(cuda_check(cudaMemsetAsync(plan_counts, 0, static_cast<size_t>(n) * sizeof(int32_t),
                                         reinterpret_cast<cudaStream_t>(stream)),
                         who));
    const PlanOut plan{plan_counts, plan_entries, slots};
    return fw_update(n, P, ldp, cost32, ld32, u, v, U, V, alpha, regularization, gap, commit, &plan, who,
                     reinterpret_cast<cudaStream_t>(stream));
}

extern "C" fugal_status fugal_update_quasi_permutation_log(float* P, int64_t ldp, const float* K, int64_t ldk,
                                                           const float* u, const float* v, int64_t n, float alpha,
                                                           float regularization, double* gap,
                                                           fugal_stream_t stream_) {
    cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
    const char* who = "fugal_update_quasi_permutation_log";
    FUGAL_TRY(check_square(P, ldp, n, who, "P"));
    FUGAL_TRY(check_square(K, ldk, n, who, "K"));
    if (u == nullptr || v == nullptr || gap == nullptr) return fail(FUGAL_BAD_ARGUMENT, "%s: null argument", who);
    FUGAL_TRY(cuda_check(cudaMemsetAsync(gap, 0, sizeof(double), stream), who));
    LaunchScope scope(FUGAL_KERNEL_UPDATE, stream);
    update_log_kernel<<<ew_grid(n), kEwThreads, 0, stream>>>(P, ldp, K, ldk, u, v, static_cast<int>(n), alpha,
                                                              regularization, gap);
    return launch_check(who);
}

extern "C" fugal_status fugal_regularize(float* gradient, int64_t ldg, const float* P, int64_t ldp, int64_t n,
                                         int iteration, fugal_stream_t stream_) {
    cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
    FUGAL_TRY(check_square(gradient, ldg, n, "fugal_regularize", "gradient"));
    FUGAL_TRY(check_square(P, ldp, n, "fugal_regularize", "P"));
    LaunchScope scope(FUGAL_KERNEL_OTHER, stream);
    regularize_kernel<<<ew_grid(n), kEwThreads, 0, stream>>>(gradient, ldg, P, ldp, static_cast<int>(n), iteration);
    return launch_check("fugal_regularize");
}

extern "C" fugal_status fugal_add_distance(const float* source, const float* target, int64_t n, float* out,
                                           int64_t ldo, fugal_stream_t stream_) {
    cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
    FUGAL_TRY(check_square(out, ldo, n, "fugal_add_distance", "out"));
    if (source == nullptr || target == nullptr) return fail(FUGAL_BAD_ARGUMENT, "fugal_add_distance: null features");
    LaunchScope scope(FUGAL_KERNEL_OTHER, stream);
    add_distance_kernel<<<ew_grid(n), kEwThreads, 0, stream>>>(source, target, static_cast<int>(n), out, ldo);
    return launch_check("fugal_add_distance");
}

extern "C" fugal_status fugal_sinkhorn_log_step(const float* K, int64_t rows, int64_t cols, int64_t ldk,
                                                const float* add, float* out, float momentum,
                                                fugal_stream_t stream_) {
    cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
    if (K == nullptr || add == nullptr || out == nullptr)
        return fail(FUGAL_BAD_ARGUMENT, "fugal_sinkhorn_log_step: null argument");
    if (rows <= 0 || cols <= 0 || ldk < cols || rows > (1ll << 31) - 1)
        return fail(FUGAL_BAD_SHAPE, "fugal_sinkhorn_log_step: bad shape");
    LaunchScope scope(FUGAL_KERNEL_OTHER, stream);
    log_step_kernel<<<static_cast<unsigned>(rows), 256, 0, stream>>>(K, ldk, static_cast<int>(cols), add, out,
                                                                      momentum);
    return launch_check("fugal_sinkhorn_log_step");
}

extern "C" fugal_status fugal_sinkhorn_log_marginal(const float* K, int64_t n, int64_t ldk, const float* u,
                                                    const float* v, int axis, double* result,
                                                    fugal_stream_t stream_) {
    cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
    FUGAL_TRY(check_square(K, ldk, n, "fugal_sinkhorn_log_marginal", "K"));
    if (u == nullptr || v == nullptr || result == nullptr)
        return fail(FUGAL_BAD_ARGUMENT, "fugal_sinkhorn_log_marginal: null argument");
    if (axis != 0 && axis != 1) return fail(FUGAL_BAD_ARGUMENT, "fugal_sinkhorn_log_marginal: axis must be 0 or 1");
    FUGAL_TRY(cuda_check(cudaMemsetAsync(result, 0, sizeof(double), stream), "fugal_sinkhorn_log_marginal"));
    LaunchScope scope(FUGAL_KERNEL_OTHER, stream);
    if (axis == 1)
        marginal_rows_kernel<<<static_cast<unsigned>(n), 256, 0, stream>>>(K, ldk, static_cast<int>(n), u, v, result);
    else
        marginal_cols_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, stream>>>(K, ldk, static_cast<int>(n),
                                                                                           u, v, result);
    return launch_check("fugal_sinkhorn_log_marginal");
}

extern "C" fugal_status fugal_count_le(const float* P, int64_t ldp, int64_t n, float threshold, int64_t* count,
                                       fugal_stream_t stream_) {
    cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
    FUGAL_TRY(check_square(P, ldp, n, "fugal_count_le", "P"));
    if (count == nullptr) return fail(FUGAL_BAD_ARGUMENT, "fugal_count_le: null count");
    FUGAL_TRY(cuda_check(cudaMemsetAsync(count, 0, sizeof(int64_t), stream), "fugal_count_le"));
    LaunchScope scope(FUGAL_KERNEL_OTHER, stream);
    count_le_kernel<<<ew_grid(n), kEwThreads, 0, stream>>>(P, ldp, static_cast<int>(n), threshold,
                                                            reinterpret_cast<unsigned long long*>(count));
    return launch_check("fugal_count_le");
}
