// Scaling-form Sinkhorn (the reference's SinkhornMethod.STANDARD,
// cugal/sinkhorn.py:122-144) and its Frank-Wolfe update (cugal/pred.py:77-86,
// 136-141), on the kernel matrix K = exp(-C/reg) (FP32, as the reference).
//
// Per iteration t the reference computes
//     v <- v^(1-w) (1 / (u K + eps))^w,   u <- u^(1-w) (1 / (K v + eps))^w,
// and at t % eval_freq == 0 (t = 0 included) the column-marginal error
//     sum_j | sum_i u_i K_ij v_j - 1 |,
// stopping below the threshold and updating the Lehmann factor w otherwise.
// Here round t launches: column partial sums of u K (the error of iteration
// t-1 uses exactly these sums with the current v, so it costs no extra pass),
// their FP64 merge with the error and the stop / momentum decision on the
// device, the v update, and the row products K v with the u update.  Rounds
// after the decision to stop return at once; the host polls the stop flag with
// a lag of two rounds.  u and v are read and written in place (warm start
// across solves, cugal/sinkhorn.py:51-65).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "fugal_common.cuh"
#include "fugal_host.h"

namespace fugal {

constexpr float kStdEps = 1e-16f;  // M_EPS, cugal/sinkhorn.py:12
constexpr int kStdThreads = 256;

struct StdState {
    int done;
    int final_it;
    int n_err;
    int max_it;
    int eval_freq;
    int momentum_start;
    unsigned int ticket;
    int pad;
    double threshold;
    double omega;
    double err_accum;
    double last_err;
    double errors[FUGAL_MAX_RECORDED_ERRORS];
};

struct StdWs {
    StdState* st;
    float* colsum;    // [n]
    float* partials;  // [chunks][n]
    size_t bytes;
};

int std_chunks(int64_t n) {
    const int col_blocks = static_cast<int>((n + kStdThreads - 1) / kStdThreads);
    int chunks = std::max(1, (sm_count() * 8) / std::max(1, col_blocks));
    return static_cast<int>(std::min<int64_t>(chunks, std::max<int64_t>(1, n / 8)));
}

StdWs std_layout(int64_t n, char* base) {
    StdWs w{};
    size_t off = 0;
    auto take = [&](size_t bytes) {
        char* p = base ? base + off : nullptr;
        off = (off + bytes + 255) / 256 * 256;
        return p;
    };
    w.st = reinterpret_cast<StdState*>(take(sizeof(StdState)));
    w.colsum = reinterpret_cast<float*>(take(n * 4));
    w.partials = reinterpret_cast<float*>(take(static_cast<size_t>(std_chunks(n)) * n * 4));
    w.bytes = off;
    return w;
}

__global__ void std_init_kernel(StdState* st, int max_it, int eval_freq, int momentum_start, double threshold) {
    st->done = 0;
    st->final_it = -1;
    st->n_err = 0;
    st->max_it = max_it;
    st->eval_freq = eval_freq;
    st->momentum_start = momentum_start;
    st->ticket = 0;
    st->threshold = threshold;
    st->omega = 1.0;
    st->err_accum = 0.0;
    st->last_err = 0.0;
}

// partials[c][j] = sum over rows of chunk c of u_i K_ij
__global__ void __launch_bounds__(kStdThreads) std_colpart_kernel(const float* __restrict__ K, long long ldk, int n,
                                                                  const float* __restrict__ u, int rows_per_chunk,
                                                                  float* __restrict__ partials,
                                                                  const StdState* st) {
    if (*reinterpret_cast<const volatile int*>(&st->done)) return;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const int r0 = blockIdx.y * rows_per_chunk;
    const int r1 = min(n, r0 + rows_per_chunk);
    float acc = 0.f;
    for (int i = r0; i < r1; ++i) acc = fmaf(u[i], K[static_cast<size_t>(i) * ldk + j], acc);
    partials[static_cast<size_t>(blockIdx.y) * n + j] = acc;
}

// colsum_j = sum of the chunk partials (FP64); the error of iteration t-1 when
// it was an evaluation point; the last block takes the decision.
__global__ void __launch_bounds__(kStdThreads) std_merge_kernel(const float* __restrict__ partials, int chunks, int n,
                                                                const float* __restrict__ v, float* colsum,
                                                                StdState* st, int t) {
    __shared__ double red[32];
    __shared__ bool last;
    if (*reinterpret_cast<volatile int*>(&st->done)) return;
    const bool eval = t > 0 && ((t - 1) % st->eval_freq == 0);
    double err = 0.0;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        double c = 0.0;
        for (int k = 0; k < chunks; ++k) c += static_cast<double>(partials[static_cast<size_t>(k) * n + j]);
        const float cf = static_cast<float>(c);
        colsum[j] = cf;
        if (eval) err += fabs(static_cast<double>(v[j]) * static_cast<double>(cf) - 1.0);
    }
    err = block_sum(err, red);
    if (threadIdx.x == 0) {
        if (eval) atomicAdd(&st->err_accum, err);
        __threadfence();
        last = atomicAdd(&st->ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last || threadIdx.x != 0) return;
    __threadfence();
    st->ticket = 0;
    bool stop = false;
    if (eval) {
        const double e = *reinterpret_cast<volatile double*>(&st->err_accum);
        st->err_accum = 0.0;
        st->last_err = e;
        if (st->n_err < FUGAL_MAX_RECORDED_ERRORS) st->errors[st->n_err] = e;
        st->n_err += 1;
        if (e < st->threshold)
            stop = true;
        else
            st->omega = lehmann_omega(st->errors, st->n_err, st->eval_freq, st->momentum_start);
    }
    if (stop || t >= st->max_it) {
        st->done = 1;
        st->final_it = t - 1;
    }
}

// v_j <- v_j^(1-w) (1 / (colsum_j + eps))^w
__global__ void std_vupdate_kernel(const float* colsum, float* v, int n, const StdState* st) {
    if (*reinterpret_cast<const volatile int*>(&st->done)) return;
    const double w = st->omega;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const float x = 1.0f / (colsum[j] + kStdEps);
        v[j] = (w == 1.0) ? x : powf(v[j], static_cast<float>(1.0 - w)) * powf(x, static_cast<float>(w));
    }
}

// u_i <- u_i^(1-w) (1 / (sum_j K_ij v_j + eps))^w, one warp per row.
__global__ void __launch_bounds__(kStdThreads) std_rowdot_kernel(const float* __restrict__ K, long long ldk, int n,
                                                                 const float* __restrict__ v, float* u,
                                                                 const StdState* st) {
    if (*reinterpret_cast<const volatile int*>(&st->done)) return;
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    const double w = st->omega;
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
        const float* row = K + static_cast<size_t>(i) * ldk;
        float acc = 0.f;
        for (int j = lane; j < n; j += 32) acc = fmaf(row[j], v[j], acc);
        acc = warp_sum(acc);
        if (lane == 0) {
            const float x = 1.0f / (acc + kStdEps);
            u[i] = (w == 1.0) ? x : powf(u[i], static_cast<float>(1.0 - w)) * powf(x, static_cast<float>(w));
        }
    }
}

__global__ void std_record_kernel(const StdState* st, fugal_solve_record* rec) {
    if (threadIdx.x == 0) {
        rec->iteration_count = st->final_it + 1;
        rec->n_errors = min(st->n_err, FUGAL_MAX_RECORDED_ERRORS);
        rec->status = 0;
        rec->polish_count = 0;
        rec->last_error = st->last_err;
        rec->polish_error = 0.0;
    }
    for (int k = threadIdx.x; k < FUGAL_MAX_RECORDED_ERRORS; k += blockDim.x) rec->errors[k] = st->errors[k];
}

// out = exp(scale * C)
__global__ void exp_scale_kernel(const float* __restrict__ C, long long ldc, int n, float scale, float* out,
                                 long long ldo) {
    for (int i = blockIdx.y; i < n; i += gridDim.y)
        for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
            out[static_cast<size_t>(i) * ldo + j] = expf(C[static_cast<size_t>(i) * ldc + j] * scale);
}

// q = (K_ij v_j) u_i;  P += alpha (q - P);  gap += C (q - P)  (FP64)
__global__ void __launch_bounds__(kStdThreads) std_update_kernel(float* P, long long ldp, const float* K, long long ldk,
                                                                 const float* u, const float* v, const float* C,
                                                                 long long ldc, int n, float alpha, double* gap) {
    __shared__ double red[32];
    double g = 0.0;
    for (int i = blockIdx.y; i < n; i += gridDim.y) {
        const float ui = u[i];
        for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
            const float q = (K[static_cast<size_t>(i) * ldk + j] * v[j]) * ui;
            float* pp = P + static_cast<size_t>(i) * ldp + j;
            const float diff = q - *pp;
            g += static_cast<double>(C[static_cast<size_t>(i) * ldc + j]) * static_cast<double>(diff);
            *pp = fmaf(alpha, diff, *pp);
        }
    }
    g = block_sum(g, red);
    if (threadIdx.x == 0) atomicAdd(gap, g);
}

}  // namespace fugal

using namespace fugal;

extern "C" fugal_status fugal_sinkhorn_standard_workspace_size(int64_t n, size_t* bytes) {
    if (bytes == nullptr) return fail(FUGAL_BAD_ARGUMENT, "fugal_sinkhorn_standard_workspace_size: null output");
    if (n <= 0 || n > (1ll << 30)) return fail(FUGAL_BAD_SHAPE, "fugal_sinkhorn_standard_workspace_size: bad n");
    *bytes = std_layout(n, nullptr).bytes;
    return FUGAL_OK;
}

namespace {
constexpr int kStdPinnedSlots = 64;
constexpr int kStdPollLag = 2;
thread_local int* g_std_pinned = nullptr;
thread_local int g_std_next = 0;
}  // namespace

extern "C" fugal_status fugal_sinkhorn_standard_solve(const float* K, int64_t ldk, int64_t n, float* u, float* v,
                                                      int max_iterations, double threshold, int eval_freq,
                                                      int momentum_start, void* record, void* workspace,
                                                      size_t workspace_bytes, fugal_stream_t stream_) {
    cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
    size_t need = 0;
    FUGAL_TRY(fugal_sinkhorn_standard_workspace_size(n, &need));
    if (K == nullptr || u == nullptr || v == nullptr || workspace == nullptr)
        return fail(FUGAL_BAD_ARGUMENT, "fugal_sinkhorn_standard_solve: null argument");
    if (ldk < n) return fail(FUGAL_BAD_SHAPE, "fugal_sinkhorn_standard_solve: ldk < n");
    if (max_iterations <= 0 || eval_freq <= 0)
        return fail(FUGAL_BAD_ARGUMENT, "fugal_sinkhorn_standard_solve: max_iterations and eval_freq must be positive");
    if (workspace_bytes < need)
        return fail(FUGAL_WORKSPACE_TOO_SMALL, "fugal_sinkhorn_standard_solve: workspace %zu < %zu", workspace_bytes,
                    need);
    StdWs w = std_layout(n, static_cast<char*>(workspace));
    const int nn = static_cast<int>(n);
    const int chunks = std_chunks(n);
    const int rows_per_chunk = (nn + chunks - 1) / chunks;
    const int vec_blocks = static_cast<int>(std::min<int64_t>((n + kStdThreads - 1) / kStdThreads, 4 * sm_count()));
    const int row_blocks = static_cast<int>(std::min<int64_t>((n * 32 + kStdThreads - 1) / kStdThreads, 16 * sm_count()));
    {
        LaunchScope scope(FUGAL_KERNEL_OTHER, stream);
        std_init_kernel<<<1, 1, 0, stream>>>(w.st, max_iterations, eval_freq, momentum_start < 0 ? -1 : momentum_start,
                                             threshold);
        FUGAL_TRY(launch_check("sinkhorn standard: init"));
    }
    if (g_std_pinned == nullptr) {
        void* p = nullptr;
        FUGAL_TRY(cuda_check(cudaHostAlloc(&p, kStdPinnedSlots * sizeof(int), cudaHostAllocPortable),
                             "sinkhorn standard: pinned flags"));
        g_std_pinned = static_cast<int*>(p);
    }
    int* pinned = g_std_pinned + g_std_next;
    g_std_next = (g_std_next + 2) % kStdPinnedSlots;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    FUGAL_TRY(cuda_check(cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming), "sinkhorn standard: event"));
    FUGAL_TRY(cuda_check(cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming), "sinkhorn standard: event"));
    fugal_status status = FUGAL_OK;
    int slot = 0, poll_slot = -1, poll_t = 0;
    // round t evaluates iteration t-1 (if it was an evaluation point) and, unless
    // the solve stopped, runs iteration t
    for (int t = 0; t <= max_iterations && status == FUGAL_OK; ++t) {
        {
            LaunchScope scope(FUGAL_KERNEL_COLUMN_PASS, stream);
            std_colpart_kernel<<<dim3((nn + kStdThreads - 1) / kStdThreads, chunks), kStdThreads, 0, stream>>>(
                K, ldk, nn, u, rows_per_chunk, w.partials, w.st);
            status = launch_check("sinkhorn standard: column partials");
        }
        if (status != FUGAL_OK) break;
        {
            LaunchScope scope(FUGAL_KERNEL_FINALIZE, stream);
            std_merge_kernel<<<vec_blocks, kStdThreads, 0, stream>>>(w.partials, chunks, nn, v, w.colsum, w.st, t);
            status = launch_check("sinkhorn standard: merge");
        }
        if (status != FUGAL_OK || t == max_iterations) break;
        {
            LaunchScope scope(FUGAL_KERNEL_OTHER, stream);
            std_vupdate_kernel<<<vec_blocks, kStdThreads, 0, stream>>>(w.colsum, v, nn, w.st);
            status = launch_check("sinkhorn standard: v update");
        }
        if (status != FUGAL_OK) break;
        {
            LaunchScope scope(FUGAL_KERNEL_SWEEP_F32, stream);
            std_rowdot_kernel<<<row_blocks, kStdThreads, 0, stream>>>(K, ldk, nn, v, u, w.st);
            status = launch_check("sinkhorn standard: u update");
        }
        if (status != FUGAL_OK) break;
        // poll the stop flag written by round t's decision, kStdPollLag rounds later
        if (poll_slot >= 0 && t - poll_t >= kStdPollLag) {
            status = cuda_check(cudaEventSynchronize(ev[poll_slot]), "sinkhorn standard: poll wait");
            timing_poll();
            const bool stop = status == FUGAL_OK && pinned[poll_slot] != 0;
            poll_slot = -1;
            if (stop) break;
        }
        if (poll_slot < 0 && t > 0 && (t - 1) % eval_freq == 0) {
            slot ^= 1;
            status = cuda_check(cudaMemcpyAsync(&pinned[slot], &w.st->done, sizeof(int), cudaMemcpyDeviceToHost, stream),
                                "sinkhorn standard: poll copy");
            if (status == FUGAL_OK) status = cuda_check(cudaEventRecord(ev[slot], stream), "sinkhorn standard: poll event");
            poll_slot = slot;
            poll_t = t;
        }
    }
    if (status == FUGAL_OK && record != nullptr) {
        LaunchScope scope(FUGAL_KERNEL_OTHER, stream);
        std_record_kernel<<<1, 256, 0, stream>>>(w.st, static_cast<fugal_solve_record*>(record));
        status = launch_check("sinkhorn standard: record");
    }
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
    return status;
}

extern "C" fugal_status fugal_exp_scale(const float* C, int64_t ldc, int64_t n, double scale, float* out, int64_t ldo,
                                        fugal_stream_t stream_) {
    cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
    if (C == nullptr || out == nullptr) return fail(FUGAL_BAD_ARGUMENT, "fugal_exp_scale: null argument");
    if (n <= 0 || ldc < n || ldo < n) return fail(FUGAL_BAD_SHAPE, "fugal_exp_scale: bad shape");
    LaunchScope scope(FUGAL_KERNEL_OTHER, stream);
    dim3 grid(static_cast<unsigned>(std::min<int64_t>((n + 255) / 256, 64)),
              static_cast<unsigned>(std::min<int64_t>(n, 65535)));
    exp_scale_kernel<<<grid, 256, 0, stream>>>(C, ldc, static_cast<int>(n), static_cast<float>(scale), out, ldo);
    return launch_check("fugal_exp_scale");
}

extern "C" fugal_status fugal_fw_update_standard(int64_t n, float* P, int64_t ldp, const float* K, int64_t ldk,
                                                 const float* u, const float* v, const float* C, int64_t ldc,
                                                 double alpha, double* gap, fugal_stream_t stream_) {
    cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
    if (P == nullptr || K == nullptr || u == nullptr || v == nullptr || C == nullptr || gap == nullptr)
        return fail(FUGAL_BAD_ARGUMENT, "fugal_fw_update_standard: null argument");
    if (n <= 0 || ldp < n || ldk < n || ldc < n) return fail(FUGAL_BAD_SHAPE, "fugal_fw_update_standard: bad shape");
    FUGAL_TRY(cuda_check(cudaMemsetAsync(gap, 0, sizeof(double), stream), "fugal_fw_update_standard: clear gap"));
    LaunchScope scope(FUGAL_KERNEL_UPDATE, stream);
    dim3 grid(static_cast<unsigned>(std::min<int64_t>((n + 255) / 256, 16)),
              static_cast<unsigned>(std::min<int64_t>(n, 8 * sm_count())));
    std_update_kernel<<<grid, kStdThreads, 0, stream>>>(P, ldp, K, ldk, u, v, C, ldc, static_cast<int>(n),
                                                        static_cast<float>(alpha), gap);
    return launch_check("fugal_fw_update_standard");
}
