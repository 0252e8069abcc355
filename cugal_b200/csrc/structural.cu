// Structural term of the Frank-Wolfe gradient kept across steps (no reference
// counterpart; the reference forms -A P B with two SpMMs every step,
// cugal/pred.py:54-74).  With P' = (1 - alpha) P + alpha q (cugal/pred.py:133-141)
// the term follows M' = (1 - alpha) M + alpha A q B.  M is stored as int64 fixed
// point scaled by a caller-held factor that carries the (1 - alpha) products, so a
// step only adds round(alpha / scale' * 2^frac_bits * q_kl) to the entries
// (i, j), i in N_A(k), j in N_B(l), of each nonzero plan entry q_kl.  The adds are
// integer atomics: their sum does not depend on their order.
//
//   fugal_csr_edge_rows       the row of every CSR edge (the scatter's work list)
//   fugal_structural_scatter  the adds, one half-warp per edge (k, i) of A, lanes over N_B(l)
//
// The dense refresh (two SpMMs into Mq) and the elementwise gradient that reads
// Mq live with the SpMM kernels (spmm.cu); the plan entries come from the update
// (update.cu, fugal_fw_update_collect).
#include <cuda_runtime.h>

#include <algorithm>

#include "fugal_common.cuh"
#include "fugal_host.h"

namespace fugal {

constexpr int kScatterThreads = 256;

// rows[e] = k for rp[k] <= e < rp[k+1]; one warp per row, lanes over its edges.
__global__ void csr_edge_rows_kernel(const int* __restrict__ rp, int n, int* __restrict__ rows) {
    const int lane = threadIdx.x & 31;
    const int warps = gridDim.x * (blockDim.x >> 5);
    for (int k = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); k < n; k += warps) {
        const int e0 = rp[k], e1 = rp[k + 1];
        for (int e = e0 + lane; e < e1; e += 32) rows[e] = k;
    }
}

// One half-warp per edge e = (k, i) of A: for each recorded plan entry (l, q) of
// row k, the 16 lanes add round(q * inc_scale) to Mq[i][j] for j in N_B(l).
// Entries of a row are few, so a half-warp walks them in turn; hub rows of A or
// B spread over many half-warps (one per edge of A) and many lane steps (N_B(l)
// in chunks of 16).  The warp's trip count over edge pairs is uniform, so the
// row-sum shuffles always see all 32 lanes.
__global__ void __launch_bounds__(kScatterThreads) structural_scatter_kernel(
    const int* __restrict__ a_col, const int* __restrict__ a_rows, long long nnz_a, const int* __restrict__ b_rp,
    const int* __restrict__ b_col, const int* __restrict__ counts, const fugal_plan_entry* __restrict__ entries,
    int slots, double inc_scale, unsigned long long* __restrict__ Mq, long long ldm, int* flags) {
    if (flags[0] != 0 || flags[1] != 0) return;  // stale term: the next gradient refreshes Mq
    const int lane = threadIdx.x & 31;
    const int hl = lane & 15;
    const long long warps = static_cast<long long>(gridDim.x) * (blockDim.x >> 5);
    const long long pairs = (nnz_a + 1) / 2;
    for (long long pr = static_cast<long long>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); pr < pairs;
         pr += warps) {
        const long long e = 2 * pr + (lane >> 4);
        const bool valid = e < nnz_a;
        const int k = valid ? a_rows[e] : 0;
        const int i = valid ? a_col[e] : 0;
        const int cnt = valid ? counts[k] : 0;
        const fugal_plan_entry* ent = entries + static_cast<size_t>(k) * slots;
        // a row this step cannot add exactly: flag it (the next gradient recomputes Mq)
        float rsum = 0.f;
        for (int s = hl; s < min(cnt, slots); s += 16) rsum += ent[s].value;
#pragma unroll
        for (int o = 8; o > 0; o >>= 1) rsum += __shfl_xor_sync(0xffffffffu, rsum, o, 16);
        if (!valid) continue;
        if (cnt > slots || !(rsum <= FUGAL_PLAN_ROW_SUM_MAX)) {
            if (hl == 0) atomicOr(flags, 1);
            continue;
        }
        unsigned long long* mrow = Mq + static_cast<unsigned long long>(static_cast<unsigned>(i)) *
                                            static_cast<unsigned long long>(ldm);
        for (int s = 0; s < cnt; ++s) {
            const fugal_plan_entry pe = ent[s];
            const unsigned long long inc =
                static_cast<unsigned long long>(__double2ll_rn(static_cast<double>(pe.value) * inc_scale));
            if (inc == 0) continue;
            const int b0 = b_rp[pe.column], b1 = b_rp[pe.column + 1];
            for (int b = b0 + hl; b < b1; b += 16) atomicAdd(mrow + b_col[b], inc);
        }
    }
}

}  // namespace fugal

using namespace fugal;

extern "C" fugal_status fugal_csr_edge_rows(const int32_t* row_pointers, int64_t n, int64_t nnz, int32_t* rows,
                                            fugal_stream_t stream_) {
    cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
    const char* who = "fugal_csr_edge_rows";
    if (row_pointers == nullptr || (rows == nullptr && nnz > 0))
        return fail(FUGAL_BAD_ARGUMENT, "%s: null pointer", who);
    if (n <= 0 || n > (1ll << 30) || nnz < 0 || nnz >= (1ll << 31)) return fail(FUGAL_BAD_SHAPE, "%s: bad n or nnz", who);
    if (nnz == 0) return FUGAL_OK;
    LaunchScope scope(FUGAL_KERNEL_OTHER, stream);
    const int blocks = static_cast<int>(std::min<int64_t>((n + 7) / 8, static_cast<int64_t>(sm_count()) * 16));
    csr_edge_rows_kernel<<<blocks, 256, 0, stream>>>(row_pointers, static_cast<int>(n), rows);
    return launch_check(who);
}

extern "C" fugal_status fugal_structural_scatter(int64_t n, const int32_t* a_col_indices, const int32_t* a_edge_rows,
                                                 int64_t a_nnz, const int32_t* b_row_pointers,
                                                 const int32_t* b_col_indices, const int32_t* plan_counts,
                                                 const fugal_plan_entry* plan_entries, int32_t slots,
                                                 double increment_scale, int64_t* Mq, int64_t ldm,
                                                 const int32_t* flags, fugal_stream_t stream_) {
    cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
    const char* who = "fugal_structural_scatter";
    if (n <= 0 || n > (1ll << 30)) return fail(FUGAL_BAD_SHAPE, "%s: bad n", who);
    if (a_nnz < 0 || a_nnz >= (1ll << 31)) return fail(FUGAL_BAD_SHAPE, "%s: bad a_nnz", who);
    if (a_nnz == 0) return FUGAL_OK;
    if (a_col_indices == nullptr || a_edge_rows == nullptr || b_row_pointers == nullptr || b_col_indices == nullptr ||
        plan_counts == nullptr || plan_entries == nullptr || Mq == nullptr || flags == nullptr)
        return fail(FUGAL_BAD_ARGUMENT, "%s: null pointer", who);
    if (slots < 1 || slots > 1024) return fail(FUGAL_BAD_ARGUMENT, "%s: slots must be in [1, 1024]", who);
    if (ldm < n || ldm >= (1ll << 32)) return fail(FUGAL_BAD_SHAPE, "%s: ldm must be in [n, 2^32)", who);
    if (!(increment_scale >= 0.0) || !(increment_scale * FUGAL_PLAN_ROW_SUM_MAX < 4503599627370496.0))
        return fail(FUGAL_BAD_ARGUMENT, "%s: increment_scale out of range", who);
    LaunchScope scope(FUGAL_KERNEL_GRADIENT, stream);
    const int64_t pairs = (a_nnz + 1) / 2;
    const int blocks = static_cast<int>(std::min<int64_t>((pairs + kScatterThreads / 32 - 1) / (kScatterThreads / 32),
                                                          static_cast<int64_t>(sm_count()) * 16));
    structural_scatter_kernel<<<blocks, kScatterThreads, 0, stream>>>(
        a_col_indices, a_edge_rows, a_nnz, b_row_pointers, b_col_indices, plan_counts, plan_entries, slots,
        increment_scale, reinterpret_cast<unsigned long long*>(Mq), ldm, const_cast<int32_t*>(flags));
    return launch_check(who);
}
