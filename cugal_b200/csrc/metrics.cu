// Alignment quality metrics of the reference's experiment harness
// (benchmark/experiment.py:115-144): edge correctness (EC), induced conserved
// structure (ICS) and the symmetric substructure score (S3) all derive from one
// integer, the overlap
//     |{(i, j) : A[answer_i][answer_j] = 1 and B[truth_i][truth_j] = 1}|,
// which the reference counts on dense n x n numpy adjacency matrices.  Here it
// is counted on the CSR graphs: every stored entry (x, y) of A is an (i, j) pair
// with i = answer^-1(x), j = answer^-1(y), and B[truth_i][truth_j] is a binary
// search in B's sorted row truth_i.  Requires `answer` to be a permutation; the
// kernel reports whether it is one (otherwise the caller uses the dense form).
#include <cuda_runtime.h>

#include <algorithm>

#include "fugal_common.cuh"
#include "fugal_host.h"

namespace fugal {

// flags: bit 0 = answer is not a permutation of 0..n-1, bit 1 = truth has an entry outside 0..n-1
__global__ void invert_mapping_kernel(const long long* answer, const long long* truth, int n, int* inverse,
                                      int* not_permutation) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (truth[i] < 0 || truth[i] >= n) atomicOr(not_permutation, 2);
        const long long x = answer[i];
        if (x < 0 || x >= n) {
            atomicOr(not_permutation, 1);
            continue;
        }
        if (atomicCAS(&inverse[x], -1, i) != -1) atomicOr(not_permutation, 1);
    }
}

__device__ __forceinline__ bool row_contains(const int* rp, const int* col, int row, int key) {
    int lo = rp[row], hi = rp[row + 1];
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        const int c = col[mid];
        if (c == key) return true;
        if (c < key) lo = mid + 1;
        else hi = mid;
    }
    return false;
}

// One warp per row x of A; lanes over its stored entries.
__global__ void overlap_kernel(const int* __restrict__ a_rp, const int* __restrict__ a_col,
                               const int* __restrict__ b_rp, const int* __restrict__ b_col, int n,
                               const int* __restrict__ inverse, const long long* __restrict__ truth,
                               const int* not_permutation, unsigned long long* count) {
    if (*not_permutation) return;
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    unsigned long long local = 0;
    for (int x = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; x < n; x += warps) {
        const int i = inverse[x];
        const int ti = static_cast<int>(truth[i]);
        for (int e = a_rp[x] + lane; e < a_rp[x + 1]; e += 32) {
            const int j = inverse[a_col[e]];
            if (row_contains(b_rp, b_col, ti, static_cast<int>(truth[j]))) ++local;
        }
    }
    local = __reduce_add_sync(0xffffffffu, static_cast<unsigned>(local));
    if (lane == 0 && local) atomicAdd(count, local);
}

}  // namespace fugal

using namespace fugal;

extern "C" fugal_status fugal_alignment_overlap_workspace_size(int64_t n, size_t* bytes) {
    if (bytes == nullptr) return fail(FUGAL_BAD_ARGUMENT, "fugal_alignment_overlap_workspace_size: null output");
    if (n <= 0 || n > (1ll << 30)) return fail(FUGAL_BAD_SHAPE, "fugal_alignment_overlap_workspace_size: bad n");
    *bytes = (static_cast<size_t>(n) * 4 + 255) / 256 * 256 + 256;
    return FUGAL_OK;
}

extern "C" fugal_status fugal_alignment_overlap(const int32_t* a_row_pointers, const int32_t* a_col_indices,
                                                const int32_t* b_row_pointers, const int32_t* b_col_indices,
                                                int64_t n, const int64_t* answer, const int64_t* truth,
                                                uint64_t* overlap, int32_t* not_permutation, void* workspace,
                                                size_t workspace_bytes, fugal_stream_t stream_) {
    cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
    size_t need = 0;
    FUGAL_TRY(fugal_alignment_overlap_workspace_size(n, &need));
    if (a_row_pointers == nullptr || b_row_pointers == nullptr || answer == nullptr || truth == nullptr ||
        overlap == nullptr || not_permutation == nullptr || workspace == nullptr)
        return fail(FUGAL_BAD_ARGUMENT, "fugal_alignment_overlap: null argument");
    if (workspace_bytes < need)
        return fail(FUGAL_WORKSPACE_TOO_SMALL, "fugal_alignment_overlap: workspace %zu < %zu", workspace_bytes, need);
    int* inverse = static_cast<int*>(workspace);
    const int nn = static_cast<int>(n);
    FUGAL_TRY(cuda_check(cudaMemsetAsync(inverse, 0xff, static_cast<size_t>(n) * 4, stream), "overlap: clear"));
    FUGAL_TRY(cuda_check(cudaMemsetAsync(overlap, 0, 8, stream), "overlap: clear count"));
    FUGAL_TRY(cuda_check(cudaMemsetAsync(not_permutation, 0, 4, stream), "overlap: clear flag"));
    const int blocks = static_cast<int>(std::min<int64_t>((n + 255) / 256, 8 * sm_count()));
    {
        LaunchScope scope(FUGAL_KERNEL_OTHER, stream);
        invert_mapping_kernel<<<blocks, 256, 0, stream>>>(reinterpret_cast<const long long*>(answer),
                                                          reinterpret_cast<const long long*>(truth), nn, inverse,
                                                          not_permutation);
        FUGAL_TRY(launch_check("fugal_alignment_overlap: invert"));
    }
    {
        LaunchScope scope(FUGAL_KERNEL_OTHER, stream);
        const int oblocks = static_cast<int>(std::min<int64_t>((n * 32 + 255) / 256, 16 * sm_count()));
        overlap_kernel<<<oblocks, 256, 0, stream>>>(a_row_pointers, a_col_indices, b_row_pointers, b_col_indices, nn,
                                                    inverse, reinterpret_cast<const long long*>(truth),
                                                    not_permutation, reinterpret_cast<unsigned long long*>(overlap));
        FUGAL_TRY(launch_check("fugal_alignment_overlap: count"));
    }
    return FUGAL_OK;
}
